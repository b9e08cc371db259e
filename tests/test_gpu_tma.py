"""The TMA-staged fine kernels (fd3_options.kernels = 5, fd3_tmarch.cuh) through the C ABI.

Their layers arrive by cp.async.bulk.tensor copies into shared memory, but each cell is evaluated
with the same f32 expressions in the same order as in every other family.  So a V-cycle gives the
oracle's bits (tests/test_gpu_quad.py runs that comparison on six shapes, this family included), and a
projection differs from the two-cells-per-thread family's only in the order of its f64 partial sums:
iterations within 1, pressure within 1e-5 relative, the reference's acceptance met.  The shapes
cover tiles cut by the volume's edge in x (nx = 40, 96) and y (ny = 24, 40, 56), both layer depths
per CTA (4, and 8 from two waves of CTAs), and the volumes the family refuses.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from fluidisim_b200.delta3d import REDUCE_F64, STORAGE_F16, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P_TOL = 1e-5


def _lake(nx, ny, nz, seed=3):
    from test_gpu_quad import lake  # the seeded sphere lake of the four-cell family's tests
    return lake(nx, ny, nz, seed)


def _device(s, kernels):
    d = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    d.set_options(reduction=REDUCE_F64, kernels=kernels)
    d.enable_multigrid()
    d.set_free_surface(s["eta"], s["rest"])
    d.set_velocity(s["u"], s["v"], s["w"])
    return d


def _project(s, kernels):
    scale, k1 = scenes.projection_scalars(s)
    d = _device(s, kernels)
    r = d.project_mobile3(scale, k1, 4000)
    p = d.pressure().astype(np.float64)
    uvw = d.velocity()
    d.close()
    return r, p, uvw


@pytest.mark.parametrize("shape", [(64, 64, 64), (96, 40, 24), (40, 56, 16), (128, 32, 32)])
def test_projection_matches_the_two_cell_family(shape):
    s = _lake(*shape)
    rt, pt, _ = _project(s, 5)
    r2, p2, _ = _project(s, 3)
    assert not rt.degraded and rt.residual <= 1e-6 and rt.divergence_plain <= 1e-5, rt
    assert abs(rt.iterations - r2.iterations) <= 1, (rt.iterations, r2.iterations)
    assert np.abs(pt - p2).max() <= P_TOL * np.abs(p2).max()


def test_box_basin_128_against_the_oracle():
    """The bench's scene (128^3 basin, 16 boxes) on this family against the reference's projection."""
    s = scenes.box_basin(128)
    r, p, _ = _project(s, 5)
    O.build()
    O.set_threads(O.max_threads("f32"), "f32")
    o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    o.enable_multigrid()
    o.set_free_surface(s["eta"], s["rest"])
    o.set_velocity(s["u"], s["v"], s["w"])
    scale, k1 = scenes.projection_scalars(s)
    ro = o.project_mobile(scale, k1, 4000)
    po = o.pressure().astype(np.float64)
    assert not r.degraded and r.residual <= 1e-6 and r.divergence_plain <= 1e-5, r
    assert abs(r.iterations - ro["iterations"]) <= 1, (r.iterations, ro["iterations"])
    assert np.abs(p - po).max() <= P_TOL * np.abs(po).max()


def test_breaking_wave_256_matches_the_four_cell_family():
    """256^3 (eight layers per CTA): against the default family at this size, four cells per thread."""
    s = scenes.breaking_wave(256)
    rt, pt, _ = _project(s, 5)
    r4, p4, _ = _project(s, 4)
    assert not rt.degraded and rt.residual <= 1e-6 and rt.divergence_plain <= 1e-5, rt
    assert abs(rt.iterations - r4.iterations) <= 1, (rt.iterations, r4.iterations)
    assert np.abs(pt - p4).max() <= P_TOL * np.abs(p4).max()


def test_two_projections_from_the_same_state_give_the_same_bits():
    s = _lake(64, 64, 64)
    a = _project(s, 5)
    b = _project(s, 5)
    assert a[0].as_dict() == b[0].as_dict()
    assert np.array_equal(a[1], b[1])
    for x, y in zip(a[2], b[2]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_volumes_the_family_cannot_take_are_refused():
    """nx % 8 != 0 (a tensor map's row stride must be a multiple of 16 bytes), and FP16 storage."""
    d = Volume3.configure(36, 32, 32, 0.1, 1000.0, 9.81)
    with pytest.raises(Exception):
        d.set_options(reduction=REDUCE_F64, kernels=5)
    d.close()
    d = Volume3.configure(64, 32, 32, 0.1, 1000.0, 9.81)
    with pytest.raises(Exception):
        d.set_options(reduction=REDUCE_F64, kernels=5, storage=STORAGE_F16)
    d.set_options(reduction=REDUCE_F64, kernels=5)  # accepted on its own
    d.close()
