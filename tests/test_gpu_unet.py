"""The learned preconditioner's network on the GPU against its FP64 oracle (needs a GPU).

The GPU stores activations, weights and activation gradients in BF16 and accumulates in FP32.
Two comparisons: against the oracle with the same BF16 storage rounding (the GPU's arithmetic must
agree up to accumulation order: tight tolerances), and against the plain FP64 oracle (the error
that BF16 storage costs: loose tolerances).  Errors are relative L2 norms of whole vectors.
"""
import numpy as np
import pytest

from fluidisim_b200 import learned
from oracle import unet_oracle as U

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# against the BF16-storage oracle
FWD_TOL = 5e-3
GRAD_TOL = 2e-2
BIAS_TOL = 5e-2  # a bias gradient is a sum over every cell, with cancellation
# against the plain FP64 oracle
FWD_TOL_64 = 5e-2
GRAD_TOL_64 = 0.2


def oracle_params(flat):
    p, off = {}, 0
    for name, cin, cout, _ in learned.LAYERS:
        n = 27 * cout * cin
        p[name + ".w"] = flat[off:off + n].astype(np.float64).reshape(27, cout, cin)
        off += n
        p[name + ".b"] = flat[off:off + cout].astype(np.float64)
        off += cout
    return p


def oracle_flat_grads(g):
    return np.concatenate([np.concatenate([g[name + ".w"].ravel(), g[name + ".b"].ravel()])
                           for name, _, _, _ in learned.LAYERS])


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_param_layout_matches_the_oracle():
    assert learned.param_count() == sum(v.size for v in U.init_params(0).values())


@pytest.mark.parametrize("conv", ["tcgen05", "mma.sync"])
@pytest.mark.parametrize("shape,batch", [((8, 8, 8), 2), ((4, 12, 8), 3)])
def test_forward_and_backward_match_the_fp64_oracle(shape, batch, conv):
    Z, Y, X = shape
    rng = np.random.default_rng(7)
    flat = learned.init_params(3)
    flat = flat + (0.02 * rng.standard_normal(flat.size)).astype(np.float32)  # non-zero biases
    net = learned.UNet(batch, Z, Y, X)
    net.set_conv_kernels(conv == "tcgen05")
    net.set_params(flat)
    assert np.array_equal(net.params(), flat)
    cells = Z * Y * X
    x = rng.standard_normal((batch, cells, 3)).astype(np.float32)
    x[..., 1:] = (x[..., 1:] > 0).astype(np.float32)  # the mask channels are 0/1
    gy = rng.standard_normal((batch, cells)).astype(np.float32)
    dx = torch.from_numpy(x.ravel()).cuda()
    dy = torch.empty(batch * cells, dtype=torch.float32, device="cuda")
    dg = torch.from_numpy(gy.ravel()).cuda()
    in_s = np.array([0.5 + k for k in range(batch)], np.float32)
    out_s = np.array([2.0 - 0.25 * k for k in range(batch)], np.float32)
    net.forward(batch, Z, Y, X, dx.data_ptr(), in_s, out_s, dy.data_ptr())
    net.backward(dg.data_ptr())
    net.sync()
    y = dy.cpu().numpy().reshape(batch, cells)
    grads = net.grads()
    P = oracle_params(flat)
    for round_bf16, ftol, gtol, btol in ((True, FWD_TOL, GRAD_TOL, BIAS_TOL),
                                         (False, FWD_TOL_64, GRAD_TOL_64, GRAD_TOL_64)):
        ref_y, ref_g = [], 0
        for k in range(batch):
            xo = x[k].astype(np.float64).reshape(Z, Y, X, 3).copy()
            xo[..., 0] = (x[k, :, 0] * in_s[k]).astype(np.float32).reshape(Z, Y, X)
            o = U.UNet(P, round_bf16=round_bf16)
            ref_y.append(o.forward(xo)[..., 0].ravel() * out_s[k])
            gk = (gy[k] * out_s[k]).astype(np.float32).astype(np.float64)
            ref_g = ref_g + oracle_flat_grads(o.backward(gk.reshape(Z, Y, X, 1)))
        ref_y = np.stack(ref_y)
        errs = {"y": rel(y, ref_y)}
        off = 0
        for name, cin, cout, _ in learned.LAYERS:
            n = 27 * cout * cin
            errs[name + ".w"] = rel(grads[off:off + n], ref_g[off:off + n])
            off += n
            errs[name + ".b"] = rel(grads[off:off + cout], ref_g[off:off + cout])
            off += cout
        print("bf16 storage" if round_bf16 else "fp64", {k: round(v, 5) for k, v in errs.items()})
        assert errs["y"] < ftol, errs
        for name, _, _, _ in learned.LAYERS:  # per layer, so a wrong layer cannot hide behind a large one
            assert errs[name + ".w"] < gtol, (name, errs)
            assert errs[name + ".b"] < btol, (name, errs)
    assert np.all(net.grads() == 0)  # consumed


def test_adam_step_moves_the_parameters_against_the_gradient():
    net = learned.UNet(1, 8, 8, 8)
    flat = learned.init_params(1)
    net.set_params(flat)
    rng = np.random.default_rng(2)
    x = torch.from_numpy(rng.standard_normal(512 * 3).astype(np.float32)).cuda()
    y = torch.empty(512, dtype=torch.float32, device="cuda")
    g = torch.ones(512, dtype=torch.float32, device="cuda")
    net.forward(1, 8, 8, 8, x.data_ptr(), 1.0, 1.0, y.data_ptr())
    net.backward(g.data_ptr())
    net.adam(1e-3)
    net.sync()
    moved = net.params() - flat
    head_b = learned.param_count() - 1
    assert moved[head_b] == pytest.approx(-1e-3, rel=1e-3)  # d(sum y)/d(head bias) > 0: the bias goes down


@pytest.mark.parametrize("shape,batch", [((4, 8, 128), 1), ((8, 16, 64), 2), ((8, 8, 256), 1)])
def test_tcgen05_convolutions_match_mma_sync(shape, batch):
    """The tcgen05 convolutions (several M tiles per CTA, rows of up to 256 cells) against the
    mma.sync ones on the same network and input: forward output and every parameter gradient.
    Both store BF16 and accumulate in FP32; only the order of the accumulation differs."""
    Z, Y, X = shape
    rng = np.random.default_rng(11)
    flat = learned.init_params(5) + (0.02 * rng.standard_normal(learned.param_count())).astype(np.float32)
    cells = Z * Y * X
    x = rng.standard_normal((batch, cells, 3)).astype(np.float32)
    x[..., 1:] = (x[..., 1:] > 0).astype(np.float32)
    gy = rng.standard_normal(batch * cells).astype(np.float32)
    out = {}
    for tc in (True, False):
        net = learned.UNet(batch, Z, Y, X)
        net.set_conv_kernels(tc)
        net.set_params(flat)
        dx = torch.from_numpy(x.ravel()).cuda()
        dy = torch.empty(batch * cells, dtype=torch.float32, device="cuda")
        dg = torch.from_numpy(gy).cuda()
        net.forward(batch, Z, Y, X, dx.data_ptr(), 1.0, 1.0, dy.data_ptr())
        net.backward(dg.data_ptr())
        net.sync()
        out[tc] = (dy.cpu().numpy(), net.grads())
    assert rel(out[True][0], out[False][0]) < 5e-3
    off = 0
    for name, cin, cout, _ in learned.LAYERS:
        n = 27 * cout * cin
        assert rel(out[True][1][off:off + n], out[False][1][off:off + n]) < 2e-2, name
        off += n + cout


@pytest.mark.parametrize("tiles", [5, 3])
@pytest.mark.parametrize("shape,batch", [((4, 8, 128), 1), ((8, 16, 64), 2), ((8, 8, 256), 1), ((16, 16, 16), 4)])
def test_pipelined_convolutions_give_the_same_bits(shape, batch, tiles):
    """The warp-specialised tcgen05 convolutions (set_conv_kernels(2)) against the one-phase-at-a-time
    ones: the same MMAs in the same order, so the forward output has the same bits.  The parameter
    gradients agree to the weight-gradient kernel's own reproducibility (it merges its per-CTA
    partials with float atomics, whose order varies from run to run).  Rows of 256 cells leave no
    room for two stage slots of the wide layers: those layers fall back."""
    Z, Y, X = shape
    rng = np.random.default_rng(13)
    flat = learned.init_params(7) + (0.02 * rng.standard_normal(learned.param_count())).astype(np.float32)
    cells = Z * Y * X
    x = rng.standard_normal((batch, cells, 3)).astype(np.float32)
    x[..., 1:] = (x[..., 1:] > 0).astype(np.float32)
    gy = rng.standard_normal(batch * cells).astype(np.float32)
    out = {}
    for mode in (1, 2):
        net = learned.UNet(batch, Z, Y, X)
        net.set_conv_kernels(mode)
        net.set_conv_tiles(tiles)
        net.set_params(flat)
        dx = torch.from_numpy(x.ravel()).cuda()
        dy = torch.empty(batch * cells, dtype=torch.float32, device="cuda")
        dg = torch.from_numpy(gy).cuda()
        for _ in range(2):  # twice: the second call reuses the persistent CTAs' barriers from a fresh launch
            net.forward(batch, Z, Y, X, dx.data_ptr(), 1.0, 1.0, dy.data_ptr())
        net.backward(dg.data_ptr())
        net.sync()
        out[mode] = (dy.cpu().numpy(), net.grads())
        net.close()
    assert np.array_equal(out[1][0].view(np.uint32), out[2][0].view(np.uint32))
    off = 0
    for name, cin, cout, _ in learned.LAYERS:
        n = 27 * cout * cin
        assert rel(out[2][1][off:off + n], out[1][1][off:off + n]) < 1e-5, name
        off += n + cout
