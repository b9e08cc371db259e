"""The four-cells-per-thread fine kernels (fd3_options.kernels = 4; the default family on volumes of
2^23 cells or more) against the other families and the oracle, through the C ABI.

Every family evaluates each cell with the same f32 expressions in the same order, so a V-cycle
(which holds no reduction) gives the same bits whichever family runs it, and the same bits as the
oracle's v_cycle3 (delta3d_multigrid.rs:393-429).  A projection differs between families only in
the order of its f64 partial sums.  The shapes cover both tilings (16 and 32 lanes per row), tiles
cut by the domain's edge in x and in y, and non-cubic volumes.
"""
import numpy as np
import pytest

from fluidisim_b200 import batch, scenes
from fluidisim_b200.delta3d import REDUCE_F64, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (nx, ny, nz): QX = 16 below nx = 128, 32 from it; 40, 48, 96 and 24-row sides cut the tiles
SHAPES = [(64, 64, 64), (128, 32, 32), (96, 40, 24), (48, 24, 32), (40, 56, 16), (256, 16, 8)]


def lake(nx, ny, nz, seed=3):
    rng = scenes.SplitMix64(seed)
    d = 0.1
    centres, radii = [], []
    for _ in range(3 if nz >= 16 else 0):  # spheres clear of the walls and 4 cells below the surface
        r = rng.uniform(2.0, max(2.5, min(nx, ny, nz) / 5))
        top = 0.6 * nz - 1.5 - 4.0 - r
        if top < r + 1.0:
            continue
        centres.append((rng.uniform(r + 1, nx - r - 1) * d, rng.uniform(r + 1, ny - r - 1) * d,
                        rng.uniform(r + 1, top) * d))
        radii.append(r * d)
    sdf = scenes.spheres_sdf(nx, ny, nz, d, centres, radii) if centres else \
        np.full((nx + 1) * (ny + 1) * (nz + 1), 1e3, np.float32)
    i = np.arange(nx) + 0.5
    j = np.arange(ny) + 0.5
    eta = (0.6 * nz + 1.5 * np.sin(2 * np.pi * i[None, :] / nx) * np.cos(2 * np.pi * j[:, None] / ny)) * d
    nu, nv, nw = scenes.face_counts(nx, ny, nz)
    return dict(nx=nx, ny=ny, nz=nz, dx=d, rho=1025.0, g=9.81, bottom=np.zeros(nx * ny, np.float32), solid=sdf,
                eta=eta.astype(np.float32).ravel(), rest=float(np.float32(0.6 * nz * d)),
                u=rng.uniform_array(nu, -1.0, 1.0), v=rng.uniform_array(nv, -1.0, 1.0),
                w=rng.uniform_array(nw, -1.0, 1.0), dt=1.0 / 60.0)


def device(s, kernels):
    d = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    d.set_options(reduction=REDUCE_F64, kernels=kernels)
    d.enable_multigrid()
    d.set_free_surface(s["eta"], s["rest"])
    d.set_velocity(s["u"], s["v"], s["w"])
    return d


@pytest.mark.parametrize("shape", SHAPES)
def test_vcycle_bits_are_the_same_in_every_family_and_the_oracle(shape):
    s = lake(*shape)
    x = scenes.noise(s["nx"] * s["ny"] * s["nz"], 5)
    zs = {}
    for kernels in (0, 1, 2, 3, 4, 5):
        d = device(s, kernels)
        zs[kernels] = d.vcycle_for_tests(x)
        d.close()
    o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    o.enable_multigrid()
    o.set_free_surface(s["eta"], s["rest"])
    zo = o.vcycle_for_tests(x)
    assert np.abs(zo).max() > 0
    for kernels, z in zs.items():
        bad = np.nonzero(z.view(np.uint32) != zo.view(np.uint32))[0]
        assert bad.size == 0, f"kernels={kernels}: {bad.size} cells differ, first {bad[:5]}"


@pytest.mark.parametrize("shape", SHAPES[:4])
def test_projection_matches_the_two_cell_family(shape):
    s = lake(*shape)
    scale, k1 = scenes.projection_scalars(s)
    out = {}
    for kernels in (4, 3):
        d = device(s, kernels)
        r = d.project_mobile3(scale, k1, 4000)
        out[kernels] = (r, d.pressure().astype(np.float64))
        d.close()
    (r4, p4), (r2, p2) = out[4], out[3]
    assert not r4.degraded and r4.residual <= 1e-6 and r4.divergence_plain <= 1e-5, r4
    assert abs(r4.iterations - r2.iterations) <= 1
    assert np.abs(p4 - p2).max() <= 1e-5 * np.abs(p2).max()


def test_quad_family_through_a_batch_of_patches():
    """Patches whose nx is a multiple of 4 and of 8: the batched entry point on the four-cell family."""
    ps = batch.patch_scenes(6, seed=11, hi=48)
    vols = [batch.configure(p, kernels=4) for p in ps]
    sk = [scenes.projection_scalars(p) for p in ps]
    reps, st = batch.project_batch(vols, [a for a, _ in sk], [b for _, b in sk], threads=3)
    assert st == [0] * len(ps)
    for p, v, r in zip(ps, vols, reps):
        assert not r.degraded and r.residual <= 1e-6 and r.divergence_plain <= 1e-5, r
        v.close()
