"""The FP16-storage V-cycle (fd3_options.storage = FD3_STORAGE_F16) on the GPU, through the C ABI.

The V-cycle's vectors (fine z, coarse x and r) are stored in FP16 with f32 arithmetic; CG vectors
stay f32 and the dots, alpha/beta and the true residual FP64.  The projection must reach the
reference's acceptance (relative residual <= 1e-6, plain divergence <= 1e-5), its pressure must
match the reference's own CPU projection (the f32 oracle) to 1e-5 relative in L-infinity, and its
error against an FP64 oracle solve (relative residual 1e-12) must be no worse than that of f32
storage.  That error is the algebraic error of stopping at a relative residual of 1e-6: on the
64^3 basin the reference's own f32 projection is 1.5e-5 away from the FP64 solution, so it is
compared with f32 storage's, not with a fixed bar.
"""
import numpy as np
import pytest

from fluidisim_b200 import scenes
from fluidisim_b200.delta3d import REDUCE_F64, REDUCE_ORDERED_F32, STORAGE_F16, STORAGE_F32, Delta3dError, Volume3
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P_TOL = 1e-5  # pressure L-inf difference to the FP64 solve, relative to its L-inf


def device(s, storage, **opts):
    d = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    d.set_options(storage=storage, **opts)
    d.enable_multigrid()
    d.set_free_surface(s["eta"], s["rest"])
    d.set_velocity(s["u"], s["v"], s["w"])
    return d


def oracle_pressure(s, real):
    """The oracle's projection: f32 (the reference, relative residual 1e-6) or f64 to 1e-12."""
    O.set_threads(O.max_threads(real), real)
    o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"],
                       real=real)
    o.enable_multigrid()
    o.set_free_surface(s["eta"], s["rest"])
    o.set_velocity(s["u"], s["v"], s["w"])
    if real == "f64":
        o.set_tolerance(1e-24)
    scale, k1 = scenes.projection_scalars(s)
    o.project_mobile(scale, k1, 4000)
    return o.pressure().astype(np.float64)


def test_fp16_storage_needs_the_paired_f64_kernels():
    d = Volume3.configure(16, 16, 16, 0.1)
    with pytest.raises(Delta3dError) as e:
        d.set_options(storage=STORAGE_F16, reduction=REDUCE_ORDERED_F32)
    assert e.value.kind == "Domain"
    with pytest.raises(Delta3dError):
        d.set_options(storage=STORAGE_F16, kernels=1)
    with pytest.raises(Delta3dError):
        d.set_options(storage=2)
    d.set_options(storage=STORAGE_F16)
    d.close()
    odd = Volume3.configure(15, 16, 16, 0.1)
    with pytest.raises(Delta3dError):
        odd.set_options(storage=STORAGE_F16)
    odd.close()


def test_fp16_vcycle_tracks_the_f32_vcycle():
    s = scenes.sphere_lake(32, spheres=4)
    x = scenes.noise(s["nx"] * s["ny"] * s["nz"], 7)
    z = {}
    for st in (STORAGE_F32, STORAGE_F16):
        d = device(s, st)
        z[st] = d.vcycle_for_tests(x).astype(np.float64)
        d.close()
    ref = z[STORAGE_F32]
    assert np.abs(ref).max() > 0
    assert np.abs(z[STORAGE_F16] - ref).max() <= 2e-3 * np.abs(ref).max()


@pytest.mark.parametrize("scene,n", [("box", 64), ("lake", 64), ("box", 128)])
def test_fp16_projection_meets_the_acceptance_and_the_fp64_solution(scene, n):
    s = scenes.box_basin(n) if scene == "box" else scenes.sphere_lake(n)
    scale, k1 = scenes.projection_scalars(s)
    reps, ps = {}, {}
    for st in (STORAGE_F32, STORAGE_F16):
        d = device(s, st)
        reps[st] = d.project_mobile3(scale, k1, 4000)
        ps[st] = d.pressure().astype(np.float64)
        d.close()
    r = reps[STORAGE_F16]
    assert not r.degraded and r.residual <= 1e-6 and r.divergence_plain <= 1e-5, r
    assert r.iterations <= reps[STORAGE_F32].iterations + 2, (r.iterations, reps[STORAGE_F32].iterations)
    pref = oracle_pressure(s, "f32")
    assert np.abs(ps[STORAGE_F16] - pref).max() <= P_TOL * np.abs(pref).max()
    p64 = oracle_pressure(s, "f64")
    pmax = np.abs(p64).max()
    if scene == "box":  # the basin's pressure does not fit FP16: the V-cycle's scaling keeps it in range
        assert pmax > 65504.0
    err16 = np.abs(ps[STORAGE_F16] - p64).max() / pmax
    err32 = np.abs(ps[STORAGE_F32] - p64).max() / pmax
    assert err16 <= 1.5 * err32 + 5e-6, (err16, err32)


def test_fp16_graph_and_stream_loops_agree():
    s = scenes.box_basin(64)
    scale, k1 = scenes.projection_scalars(s)
    out = []
    for graphs in (0, 1):
        d = device(s, STORAGE_F16, use_graphs=graphs)
        rep = d.project_mobile3(scale, k1, 4000)
        out.append((rep.as_dict(), d.pressure()))
        d.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))


def test_fp16_surface_follows_f32_over_warm_steps():
    s = scenes.s385_case(64, bump=True)
    etas = {}
    for st in (STORAGE_F32, STORAGE_F16):
        d = Volume3.configure_with_bottom(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"])
        d.set_options(storage=st)
        d.enable_multigrid()
        d.set_free_surface(s["eta"], s["rest"])
        for _ in range(5):
            rep = d.step_surface_mobile(s["dt_us"], 4000)
            assert not rep.degraded
        etas[st] = d.surface().astype(np.float64)
        d.close()
    assert np.abs(etas[STORAGE_F16] - etas[STORAGE_F32]).max() <= 1e-6  # metres, as tests_delta3d.rs:1875
