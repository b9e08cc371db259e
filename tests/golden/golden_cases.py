"""Seeded cases whose outputs are committed as golden fixtures (oracle_digests.json).

Each case drives a volume through the reference's public sequence (configure, enable_multigrid,
set_free_surface / set_velocity, a projection or steps) and returns the reports and every field the
reference publishes: eta and its roundoff, u, v, w and p.  The same function drives the oracle
(OracleVolume) and the library (Volume3 in the ordered-f32 reduction mode, whose fields are
bit-identical to the oracle's), through the small adapters below.  The fixtures store SHA-256
digests of the fields' bits, so a test can check either side against the committed values without
running the other.

make_golden.py (beside this file) writes the fixtures from the oracle.
"""
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("eta", "roundoff", "u", "v", "w", "p")


def known_answers() -> dict:
    """The reference's published known answers (known_answers.json)."""
    with open(os.path.join(HERE, "known_answers.json")) as f:
        return json.load(f)


def oracle_digests() -> dict:
    """The oracle's outputs on CASES (oracle_digests.json, written by make_golden.py)."""
    with open(os.path.join(HERE, "oracle_digests.json")) as f:
        return json.load(f)


class OracleSide:
    """The oracle behind the case API."""

    def __init__(self):
        from oracle import oracle as O
        self.O = O

    def volume(self, nx, ny, nz, dx, rho, g, bottom=None, solid=None):
        return self.O.OracleVolume(nx, ny, nz, dx, rho, g, bottom=bottom, solid=solid)

    @staticmethod
    def step(v, dt_us, max_iters):
        return v.step_surface_mobile(dt_us, max_iters)

    @staticmethod
    def project(v, scale, k1, max_iters):
        return v.project_mobile(scale, k1, max_iters)

    @staticmethod
    def step_linear(v, dt_us, max_iters):
        return v.step_surface_linear(dt_us, max_iters)

    @staticmethod
    def fields(v):
        e, r = v.surface()
        return dict(zip(FIELDS, [e, r, *v.velocity(), v.pressure()]))

    @staticmethod
    def close(v):
        del v


class DeviceSide:
    """The sm_100a library behind the case API, ordered-f32 reductions."""

    def __init__(self):
        from fluidisim_b200 import delta3d as D
        self.D = D

    def volume(self, nx, ny, nz, dx, rho, g, bottom=None, solid=None):
        V = self.D.Volume3
        if solid is not None:
            d = V.configure_with_solid(nx, ny, nz, dx, rho, g, bottom, solid)
        elif bottom is not None:
            d = V.configure_with_bottom(nx, ny, nz, dx, rho, g, bottom)
        else:
            d = V.configure(nx, ny, nz, dx, rho, g)
        d.set_options(reduction=self.D.REDUCE_ORDERED_F32)
        return d

    @staticmethod
    def step(v, dt_us, max_iters):
        return v.step_surface_mobile(dt_us, max_iters).as_dict()

    @staticmethod
    def project(v, scale, k1, max_iters):
        return v.project_mobile3(scale, k1, max_iters).as_dict()

    @staticmethod
    def step_linear(v, dt_us, max_iters):
        return v.step_surface_linear(dt_us, max_iters).as_dict()

    @staticmethod
    def fields(v):
        e, r = v.surface_and_roundoff()
        return dict(zip(FIELDS, [e, r, *v.velocity(), v.pressure()]))

    @staticmethod
    def close(v):
        v.close()


def _s385(side, nx, bump, steps):
    """The S385 bench (examples/delta3d_multigrille.rs:26-94): first steps from rest, multigrid."""
    from fluidisim_b200 import scenes
    s = scenes.s385_case(nx, bump)
    v = side.volume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"])
    v.enable_multigrid()
    v.set_free_surface(s["eta"], s["rest"])
    reports = [side.step(v, s["dt_us"], 20000) for _ in range(steps)]
    return v, reports


def _lake(side, mg):
    """A 32^3 lake around four solid spheres, seed 1, random faces: one projection."""
    from fluidisim_b200 import scenes
    s = scenes.sphere_lake(32, seed=1, spheres=4)
    v = side.volume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    if mg:
        v.enable_multigrid()
    v.set_free_surface(s["eta"], s["rest"])
    v.set_velocity(s["u"], s["v"], s["w"])
    scale, k1 = scenes.projection_scalars(s)
    return v, [side.project(v, scale, k1, 4000)]


def _sparse(side):
    """A 32 x 24 window holding two rectangles of columns, a bump in each, ten mobile steps
    (tests_delta3d_sparse.rs:264-290 shapes)."""
    from fluidisim_b200 import scenes
    nx, ny = 32, 24
    v = side.volume(nx, ny, scenes.SPARSE_NZ, scenes.SPARSE_DX, 1000.0, 9.81)
    v.set_free_surface(np.full(nx * ny, scenes.SPARSE_REST, np.float32), scenes.SPARSE_REST)
    v.enable_multigrid()
    v.enable_sparse()
    mask = scenes.rect_mask(nx, ny, [(0, 12, 0, 24), (16, 32, 4, 20)])
    v.set_active_columns(mask)
    v.set_free_surface(scenes.bumps_in(nx, ny, mask, [(6.0, 11.0), (23.0, 12.0)]), scenes.SPARSE_REST)
    return v, [side.step(v, 20_000, 20_000) for _ in range(10)]


def _linear(side, nx):
    """The cut-bump bench (FACES-COUPEES-3D-S324.md, S326 Jacobi): one linear step."""
    from fluidisim_b200 import scenes
    s = scenes.s324_case(nx, True)
    v = side.volume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"])
    v.set_precondition_cut(True)
    v.set_surface(s["eta"])
    return v, [side.step_linear(v, s["dt_us"], 20000)]


CASES = {
    "s385_32_flat_first_step": lambda side: _s385(side, 32, False, 1),
    "s385_32_bump_first_step": lambda side: _s385(side, 32, True, 1),
    "s385_64_bump_first_step": lambda side: _s385(side, 64, True, 1),
    "s385_32_bump_ten_steps": lambda side: _s385(side, 32, True, 10),
    "sphere_lake_32_mg_projection": lambda side: _lake(side, True),
    "sphere_lake_32_jacobi_projection": lambda side: _lake(side, False),
    "sparse_two_rectangles_ten_steps": _sparse,
    "s326_cut_bump_32_linear_step": lambda side: _linear(side, 32),
}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).tobytes()).hexdigest()


def report_keys(name):
    return LINEAR_KEYS if "linear" in name else None


def run(side, name):
    """Runs one case; returns {"reports": [...], "fields": {name: sha256}, "sizes": {name: n}}."""
    v, reports = CASES[name](side)
    f = side.fields(v)
    out = {"reports": reports, "fields": {k: digest(a) for k, a in f.items()},
           "sizes": {k: int(np.asarray(a).size) for k, a in f.items()}}
    side.close(v)
    return out


# The linear path's report is compared on these keys only, the divergence to 1e-12 relative: the
# device sums that path's report metrics in another order than the oracle.
LINEAR_KEYS = ("iterations", "degraded", "divergence")


def same_report(got: dict, want: dict, keys=None) -> bool:
    """Counts and flags exactly; the f64 report metrics to 1e-12 relative."""
    if keys is None:
        if set(got) != set(want):
            return False
        keys = want.keys()
    for k in keys:
        w, g = want[k], got[k]
        if isinstance(w, float):
            if not abs(g - w) <= 1e-12 * max(abs(w), 1e-300):
                return False
        elif g != w:
            return False
    return True
