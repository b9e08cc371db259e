"""The second-order advection term (delta3d_advection.rs) on the GPU, through the C ABI (needs a GPU).

The predictor with the term must be bit-identical to the oracle's on a flat box, a cut lake with
solid spheres and a sparse set; mobile steps with the term must stay bit-identical in the ordered
mode; and the four-cell mode of tests_delta3d.rs:2182-2193 must stop growing.
"""
import numpy as np
import pytest

import golden_cases as G
from fluidisim_b200 import scenes
from fluidisim_b200.delta3d import REDUCE_ORDERED_F32, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_bits(a, b, what):
    a, b = bits(a), bits(b)
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{what}: {bad.size} differ, first at {bad[:5]}"


def test_the_term_is_off_by_default():
    d = Volume3.configure(8, 4, 6, 0.25, 1025.0, 9.81)
    assert not d.advection_correction()
    d.enable_advection_correction()
    assert d.advection_correction()


@pytest.mark.parametrize("scene", ["flat", "lake", "sparse"])
def test_the_corrected_predictor_is_bit_identical_to_the_oracle(scene):
    if scene == "lake":
        s = scenes.sphere_lake(32, seed=1, spheres=4)
        n, dx = 32, s["dx"]
        o = O.OracleVolume(n, n, n, dx, s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
        d = Volume3.configure_with_solid(n, n, n, dx, s["rho"], s["g"], s["bottom"], s["solid"])
        shape = (n, n, n)
    else:
        shape = (24, 20, 12)
        o = O.OracleVolume(*shape, 0.25, 1000.0, 9.81)
        d = Volume3.configure(*shape, 0.25, 1000.0, 9.81)
    rng = np.random.default_rng(11)
    u, v, w = (rng.uniform(-1, 1, m).astype(np.float32) for m in scenes.face_counts(*shape))
    for x in (o, d):
        if scene == "sparse":
            x.enable_sparse()
            x.set_active_columns(scenes.rect_mask(24, 20, [(0, 16, 0, 8), (0, 8, 8, 20), (16, 24, 12, 20)]))
        x.enable_advection_correction()
        x.set_velocity(u, v, w)
    for _ in range(3):
        o.advect_for_tests(0.02)
        d.advect_for_tests(0.02)
    for a, b, name in zip(o.velocity(), d.velocity(), "uvw"):
        assert_bits(a, b, name)


def test_steps_with_the_term_are_bit_identical_to_the_oracle():
    nx, ny, nz = 24, 16, 12
    eta = scenes.bumps_in(nx, ny, np.ones(nx * ny), [(9.0, 7.0)])
    o = O.OracleVolume(nx, ny, nz, 0.25, 1000.0, 9.81)
    d = Volume3.configure(nx, ny, nz, 0.25, 1000.0, 9.81)
    d.set_options(reduction=REDUCE_ORDERED_F32)
    for x in (o, d):
        x.set_free_surface(eta, 2.0)
        x.enable_advection_correction()
    for s in range(15):
        a, b = o.step_surface_mobile(20_000, 20_000), d.step_surface_mobile(20_000, 20_000)
        assert a["iterations"] == b.iterations, s
    e, r = o.surface()
    de, dr = d.surface_and_roundoff()
    for a, b, name in zip([e, r, *o.velocity(), o.pressure()], [de, dr, *d.velocity(), d.pressure()],
                          ["eta", "roundoff", "u", "v", "w", "p"]):
        assert_bits(a, b, name)


def advection_only(corrected, amplitude, steps):
    d = Volume3.configure(128, 4, 6, 0.25, 1025.0, 9.81)
    if corrected:
        d.enable_advection_correction()
    u = np.zeros((6, 4, 129), np.float32)
    i = np.arange(1, 128, dtype=np.float32)
    u[:, :, 1:128] = np.float32(2.0) + np.float32(amplitude) * np.sin(np.float32(np.pi / 2) * i).astype(np.float32)
    d.set_velocity(u.ravel(), np.zeros(d.nx * 5 * 6, np.float32), np.zeros(128 * 4 * 7, np.float32))
    for _ in range(steps):
        d.advect_for_tests(0.033)
    return d.velocity()[0].reshape(6, 4, 129)


def test_second_order_advection_stops_the_ftcs_growth():
    """tests_delta3d.rs:2182-2193: FTCS x5..10 over 60 steps, corrected < 0.5."""
    def growth(corrected):
        a, b = advection_only(corrected, 1e-3, 60), advection_only(corrected, 0.0, 60)
        s = c = 0.0
        for i in range(48, 80):
            x = float(a[2, 2, i]) - float(b[2, 2, i])
            s += x * np.sin(np.pi / 2 * i)
            c += x * np.cos(np.pi / 2 * i)
        return float(np.hypot(s, c)) / (1e-3 * 32 / 2)
    ftcs, corrected = growth(False), growth(True)
    want = G.known_answers()["advection_four_cell_mode"]
    lo, hi = want["ftcs_growth_between"]
    assert lo < ftcs < hi, ftcs
    assert corrected < want["corrected_growth_below"], corrected
