"""The learned projection end to end on the GPU: FCG with the network as the preconditioner,
multigrid PCG as the fallback, trained by the library's own kernels (needs a GPU)."""
import numpy as np
import pytest

from fluidisim_b200 import learned, scenes
from fluidisim_b200.delta3d import REDUCE_F64, Volume3

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def lake(n, seed, mg=True):
    s = scenes.sphere_lake(n, seed=seed, spheres=4)
    v = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    v.set_options(reduction=REDUCE_F64)
    if mg:
        v.enable_multigrid()
    v.set_free_surface(s["eta"], s["rest"])
    v.set_velocity(s["u"], s["v"], s["w"])
    return v, s


@pytest.fixture(scope="module")
def trained():
    n = 32
    vols = [lake(n, seed)[0] for seed in range(11, 17)]
    s = scenes.sphere_lake(n, seed=11, spheres=4)
    scale, _ = scenes.projection_scalars(s)
    net = learned.UNet(4, n, n, n)
    net.set_params(learned.init_params(0))
    untrained = net.params()
    tr = learned.Trainer(net, vols, scale, batch=4, seed=5)
    rng = np.random.default_rng(0)
    losses = [tr.step(2e-3, rng) for _ in range(300)]
    return net, untrained, losses


def test_learned_projection_reaches_the_reference_acceptance(trained):
    net, _, _ = trained
    v, s = lake(32, 3)
    scale, k1 = scenes.projection_scalars(s)
    r = learned.project_learned(v, net, scale, k1, 4000, 200)
    assert not r.report.degraded
    assert r.report.residual <= 1e-6 and r.report.divergence_plain <= 1e-5
    p = v.pressure()
    ref, _ = lake(32, 3)
    rr = ref.project_mobile3(scale, k1, 4000)
    assert not rr.degraded
    pr = ref.pressure()
    # Both pressures meet the reference's acceptance (relative residual <= 1e-6).  Their difference
    # is the algebraic error of stopping there, which this ghost-heavy operator (coefficients up to
    # 1/theta_min = 1000) amplifies: about 1e-4 relative was seen, so the bar is 1e-3.
    assert np.max(np.abs(p - pr)) <= 1e-3 * np.max(np.abs(pr))


def test_training_lowers_the_loss(trained):
    _, _, losses = trained
    first, last = np.mean(losses[:20]), np.mean(losses[-20:])
    assert last < 0.5 * first, (first, last)


def test_trained_network_cuts_fcg_iterations(trained):
    """What the network gains: FCG iterations to the reference tolerance with the trained network,
    against the untrained one and against the Jacobi-PCG of the same projection without multigrid."""
    net, untrained, _ = trained
    v, s = lake(32, 99)
    scale, k1 = scenes.projection_scalars(s)
    r = learned.project_learned(v, net, scale, k1, 4000, 400)
    assert not r.report.degraded
    fresh = learned.UNet(1, 32, 32, 32)
    fresh.set_params(untrained)
    v2, _ = lake(32, 99)
    r0 = learned.project_learned(v2, fresh, scale, k1, 4000, 400)
    jac, _ = lake(32, 99, mg=False)
    rj = jac.project_mobile3(scale, k1, 4000)
    trained_cost = r.fcg_iterations + r.report.iterations
    print(f"FCG iterations: trained {r.fcg_iterations} (+{r.report.iterations} fallback), untrained "
          f"{r0.fcg_iterations} (+{r0.report.iterations}), Jacobi-PCG {rj.iterations}")
    # the trained network beats the projection without a multigrid by a wide margin, and leaves the
    # multigrid fallback no more to do than the untrained one (after a stall the fallback starts
    # from the original pressure, so it is then the plain multigrid projection)
    assert trained_cost < rj.iterations // 3
    assert r.report.iterations <= r0.report.iterations


# ----------------------------------------------- learned FCG against plain MGPCG (the headline's solver)
def _timed(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    best, out = float("inf"), None
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best, out


@pytest.fixture(scope="module")
def trained64():
    """Networks trained at 64^3 on sphere lakes: on right-hand sides (MODE_NET) and on the residuals
    a V-cycle leaves (MODE_VCYCLE_PLUS_NET)."""
    nets = {}
    for mode, kind in ((learned.MODE_NET, "rhs"), (learned.MODE_VCYCLE_PLUS_NET, "vcycle")):
        vols = [lake(64, 1000 + q)[0] for q in range(4)]
        s = scenes.sphere_lake(64, seed=1000, spheres=4)
        scale, _ = scenes.projection_scalars(s)
        net = learned.UNet(8, 64, 64, 64)
        net.set_params(learned.init_params(0))
        tr = learned.Trainer(net, vols, scale, batch=8, seed=2, samples=kind)
        rng = np.random.default_rng(1)
        losses = [tr.step(1e-3, rng) for _ in range(150)]
        nets[mode] = (net.params(), float(np.mean(losses[:5])), float(np.mean(losses[-5:])))
        net.close()
    return nets


@pytest.mark.parametrize("n", [64, 128])
def test_learned_fcg_against_plain_mgpcg(trained64, n):
    """Iterations and event-timed ms of plain MGPCG and of learned FCG in both modes on the same
    scene.  What holds by design, and is asserted: each meets the reference's acceptance; after a
    stall the MGPCG fallback restarts from the pressure the call started with, so it runs plain
    MGPCG's iterations and the learned call costs at most the FCG attempt more than plain MGPCG.
    The measured comparison is printed (and is in the bench line's learned_fcg key): neither mode
    is faster than plain MGPCG at these sizes, because one network application costs several
    MGPCG iterations."""
    if n == 64:
        s = scenes.sphere_lake(64, seed=2000, spheres=4)
    else:
        s = scenes.box_basin(128)
    scale, k1 = scenes.projection_scalars(s)
    v = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    v.set_options(reduction=REDUCE_F64)
    v.enable_multigrid()
    v.set_free_surface(s["eta"], s["rest"])

    def plain():
        v.set_velocity(s["u"], s["v"], s["w"])
        v.reset_pressure()
        return v.project_mobile3(scale, k1, 4000)
    plain_ms, rp = _timed(plain)
    assert not rp.degraded and rp.residual <= 1e-6
    p_plain = v.pressure().astype(np.float64)
    # one network application at this size
    net = learned.UNet(1, s["nz"], s["ny"], s["nx"])
    x = torch.zeros(3 * v.cells, dtype=torch.float32, device="cuda")
    y = torch.empty(v.cells, dtype=torch.float32, device="cuda")
    net_ms, _ = _timed(lambda: net.forward(1, s["nz"], s["ny"], s["nx"], x.data_ptr(), 1.0, 1.0, y.data_ptr()) or net.sync())
    out = {"plain": {"ms": plain_ms, "iterations": rp.iterations}, "network_ms": net_ms}
    for mode, (params, l0, l1) in trained64.items():
        assert l1 < 0.5 * l0, (mode, l0, l1)
        net.set_params(params)
        net.set_mode(mode)

        def run():
            v.set_velocity(s["u"], s["v"], s["w"])
            v.reset_pressure()
            return learned.project_learned(v, net, scale, k1, 4000, 100)
        ms, r = _timed(run)
        out[f"mode{mode}"] = {"ms": ms, "fcg": r.fcg_iterations, "fallback": r.report.iterations,
                              "fell_back": r.fell_back, "speed_vs_plain": plain_ms / ms}
        assert not r.report.degraded and r.report.residual <= 1e-6 and r.report.divergence_plain <= 1e-5
        assert np.max(np.abs(v.pressure() - p_plain)) <= 1e-3 * np.max(np.abs(p_plain))
        if r.fell_back:
            assert abs(r.report.iterations - rp.iterations) <= 1
            # the attempt's cost: per FCG iteration one network application (plus a V-cycle in
            # the hybrid mode) and a few vector passes with host round trips
            per_it = net_ms + (plain_ms / max(rp.iterations, 1) if mode == learned.MODE_VCYCLE_PLUS_NET else 0.0) + 0.5
            assert ms <= plain_ms + (r.fcg_iterations + 1) * per_it + 2.0, out
    print(out)
    net.close()
    v.close()
