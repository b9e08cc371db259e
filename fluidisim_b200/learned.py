"""The learned preconditioner: the U-Net of libfluidisim_delta3d.so, its training loop and the
learned projection (flexible CG with the network, multigrid PCG as the fallback).

There is no reference counterpart.  The network maps (residual, solid mask, liquid mask) to an
approximate solution of A z = r.  It is trained on the GPU by the library's own forward and
backward kernels, on right-hand sides that the library assembles from seeded random scenes.  The
loss is the squared residual norm |A M(r) - r|^2 / |r|^2, averaged over a batch.

Layers, in execution order (3x3x3 convolutions, ReLU after every one but the head):
    e0 3->16, pool, e1 16->32, pool, b 32->64, up+cat(e1), d1 96->32, up+cat(e0), d0 48->16, head 16->1.
Parameters per layer: w[27][cout][cin] then b[cout] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from .delta3d import Delta3dError, Report, Volume3, _Report, library

LAYERS = [("e0", 3, 16, True), ("e1", 16, 32, True), ("b", 32, 64, True), ("d1", 96, 32, True),
          ("d0", 48, 16, True), ("head", 16, 1, False)]


def param_count() -> int:
    return sum(27 * cin * cout + cout for _, cin, cout, _ in LAYERS)


def init_params(seed: int = 0) -> np.ndarray:
    """He initialisation (N(0, 2/fan_in), fan_in = 27 cin), zero biases; the head a tenth of that."""
    rng = np.random.default_rng(seed)
    out = []
    for _, cin, cout, relu in LAYERS:
        std = np.sqrt(2.0 / (27 * cin)) * (1.0 if relu else 0.1)
        out.append(rng.normal(0.0, std, size=27 * cout * cin))
        out.append(np.zeros(cout))
    return np.concatenate(out).astype(np.float32)


def _bind(L: C.CDLL) -> C.CDLL:
    if getattr(L, "_learned_bound", False):
        return L
    vp, f32, i32, u32, sz = C.c_void_p, C.c_float, C.c_int, C.c_uint32, C.c_size_t
    fp = C.POINTER(C.c_float)
    L.fd3_unet_create.argtypes = [i32, i32, i32, i32, C.POINTER(vp)]
    L.fd3_unet_destroy.argtypes = [vp]
    L.fd3_unet_destroy.restype = None
    L.fd3_unet_set_stream.argtypes = [vp, vp]
    L.fd3_unet_param_count.argtypes = [vp]
    L.fd3_unet_param_count.restype = C.c_uint64
    L.fd3_unet_set_params.argtypes = [vp, fp, sz]
    L.fd3_unet_get_params.argtypes = [vp, fp, sz]
    L.fd3_unet_get_grads.argtypes = [vp, fp, sz]
    L.fd3_unet_forward.argtypes = [vp, i32, i32, i32, i32, vp, fp, fp, vp]
    L.fd3_unet_backward.argtypes = [vp, vp]
    L.fd3_unet_adam.argtypes = [vp, f32, f32, f32, f32]
    L.fd3_unet_sync.argtypes = [vp]
    L.fd3_unet_set_conv_kernels.argtypes = [vp, i32]
    L.fd3_unet_set_conv_tiles.argtypes = [vp, i32]
    L.fd3_unet_kernel_launches.argtypes = [vp]
    L.fd3_unet_kernel_launches.restype = C.c_uint64
    L.fd3_assemble_device.argtypes = [vp, f32]
    L.fd3_problem_device.argtypes = [vp, C.POINTER(vp), C.POINTER(vp)]
    L.fd3_apply_device.argtypes = [vp, vp, vp]
    L.fd3_learned_input.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
    L.fd3_unet_set_mode.argtypes = [vp, i32]
    L.fd3_vcycle_residual_device.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
    L.fd3_residual_loss.argtypes = [vp, vp, vp, f32, vp, C.POINTER(C.c_double)]
    L.fd3_project_learned.argtypes = [vp, vp, f32, f32, u32, u32, C.POINTER(_Report), C.POINTER(u32),
                                      C.POINTER(i32)]
    L._learned_bound = True
    return L


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class UNet:
    """The network object of the library: parameters, Adam state and activations for up to
    `max_batch` samples of nz x ny x nx cells (each a multiple of 4)."""

    def __init__(self, max_batch: int, nz: int, ny: int, nx: int):
        self._L = _bind(library())
        h = C.c_void_p()
        e = self._L.fd3_unet_create(max_batch, nz, ny, nx, C.byref(h))
        if e:
            raise Delta3dError(e, "fd3_unet_create", self._L.fd3_last_cuda_error().decode())
        self._h = h
        self.max_batch, self.shape = max_batch, (nz, ny, nx)
        self.nparams = int(self._L.fd3_unet_param_count(self._h))

    def close(self):
        if self._h:
            self._L.fd3_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, e, where):
        if e:
            raise Delta3dError(e, where, self._L.fd3_last_cuda_error().decode())

    def set_stream(self, stream: int):
        self._check(self._L.fd3_unet_set_stream(self._h, C.c_void_p(stream)), "set_stream")

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self._L.fd3_unet_set_params(self._h, _fp(p), p.size), "set_params")

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, np.float32)
        self._check(self._L.fd3_unet_get_params(self._h, _fp(out), out.size), "params")
        return out

    def grads(self) -> np.ndarray:
        """The accumulated parameter gradient (then cleared)."""
        out = np.empty(self.nparams, np.float32)
        self._check(self._L.fd3_unet_get_grads(self._h, _fp(out), out.size), "grads")
        return out

    def forward(self, batch: int, nz: int, ny: int, nx: int, d_in: int, in_scale, out_scale, d_out: int):
        """y = out_scale[b] * net(x); x [batch*cells][3] and y [batch*cells] are device pointers."""
        a = np.ascontiguousarray(np.broadcast_to(np.float32(in_scale), (batch,)), np.float32)
        b = np.ascontiguousarray(np.broadcast_to(np.float32(out_scale), (batch,)), np.float32)
        self._check(self._L.fd3_unet_forward(self._h, batch, nz, ny, nx, C.c_void_p(d_in), _fp(a), _fp(b),
                                             C.c_void_p(d_out)), "forward")

    def backward(self, d_gout: int):
        self._check(self._L.fd3_unet_backward(self._h, C.c_void_p(d_gout)), "backward")

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self._check(self._L.fd3_unet_adam(self._h, lr, beta1, beta2, eps), "adam")

    def sync(self):
        self._check(self._L.fd3_unet_sync(self._h), "sync")

    def set_conv_kernels(self, tcgen05):
        """True or 1: convolutions on tcgen05.mma, one phase at a time (default); 2: the pipelined
        tcgen05 kernel (the same bits); False or 0: on mma.sync (for cross-checks)."""
        self._check(self._L.fd3_unet_set_conv_kernels(self._h, int(tcgen05)), "set_conv_kernels")

    def set_conv_tiles(self, tiles: int):
        """Budget of 128-row output tiles per CTA of the tcgen05 convolutions (1..5, default 5)."""
        self._check(self._L.fd3_unet_set_conv_tiles(self._h, int(tiles)), "set_conv_tiles")

    def kernel_launches(self) -> int:
        return int(self._L.fd3_unet_kernel_launches(self._h))

    def set_mode(self, mode: int):
        """How project_learned uses the network: MODE_NET (the preconditioner is the network) or
        MODE_VCYCLE_PLUS_NET (the V-cycle plus the network's correction of the residual it leaves)."""
        self._check(self._L.fd3_unet_set_mode(self._h, int(mode)), "set_mode")


MODE_NET = 0
MODE_VCYCLE_PLUS_NET = 1


# ------------------------------------------------------------------- the volume's learned hooks
def assemble_device(vol: Volume3, scale: float):
    L = _bind(vol._L)
    vol._check(L.fd3_assemble_device(vol._h, np.float32(scale)), "assemble_device")


def problem_device(vol: Volume3):
    """(rhs, codes) device pointers of the last assembly."""
    L = _bind(vol._L)
    r, c = C.c_void_p(), C.c_void_p()
    vol._check(L.fd3_problem_device(vol._h, C.byref(r), C.byref(c)), "problem_device")
    return r.value, c.value


def apply_device(vol: Volume3, d_x: int, d_out: int):
    L = _bind(vol._L)
    vol._check(L.fd3_apply_device(vol._h, C.c_void_p(d_x), C.c_void_p(d_out)), "apply_device")


def learned_input(vol: Volume3, d_r: int, d_in3: int) -> float:
    """The network input (r, solid, liquid) of a residual; returns |r|^2."""
    L = _bind(vol._L)
    rr = C.c_double()
    vol._check(L.fd3_learned_input(vol._h, C.c_void_p(d_r), C.c_void_p(d_in3), C.byref(rr)), "learned_input")
    return rr.value


def vcycle_residual(vol: Volume3, d_r: int, d_rho: int) -> float:
    """rho = r - A V(r), the residual a multigrid V-cycle leaves (d_rho may be d_r); returns |rho|^2."""
    L = _bind(vol._L)
    rr = C.c_double()
    vol._check(L.fd3_vcycle_residual_device(vol._h, C.c_void_p(d_r), C.c_void_p(d_rho), C.byref(rr)),
               "vcycle_residual")
    return rr.value


def residual_loss(vol: Volume3, d_z: int, d_b: int, weight: float, d_grad: int) -> float:
    L = _bind(vol._L)
    loss = C.c_double()
    vol._check(L.fd3_residual_loss(vol._h, C.c_void_p(d_z), C.c_void_p(d_b), np.float32(weight), C.c_void_p(d_grad),
                                   C.byref(loss)), "residual_loss")
    return loss.value


@dataclass
class LearnedReport:
    report: Report
    fcg_iterations: int
    fell_back: bool


def project_learned(vol: Volume3, net: UNet, scale: float, k1: float, max_iters: int = 4000,
                    max_fcg: int = 100) -> LearnedReport:
    """project_mobile3 with the learned FCG in front (us = u); see fd3_project_learned."""
    L = _bind(vol._L)
    r = _Report()
    it = C.c_uint32()
    fb = C.c_int()
    vol._check(L.fd3_project_learned(vol._h, net._h, np.float32(scale), np.float32(k1), max_iters, max_fcg,
                                     C.byref(r), C.byref(it), C.byref(fb)), "project_learned")
    return LearnedReport(Report._from(r), int(it.value), bool(fb.value))


# ------------------------------------------------------------------------------------ training
class Trainer:
    """Trains `net` on right-hand sides assembled by the library from `volumes` (one geometry each,
    all of the same shape) with seeded random face velocities U[-1, 1], in batches.  With
    samples="vcycle" each sample is instead the residual a V-cycle leaves of such a right-hand
    side, r - A V(r): what the network corrects in MODE_VCYCLE_PLUS_NET.

    Device buffers are torch tensors (memory only); every computation is a library kernel."""

    def __init__(self, net: UNet, volumes, scale: float, batch: int, seed: int = 0, samples: str = "rhs"):
        import torch
        self.torch = torch
        self.net, self.vols, self.scale, self.batch = net, list(volumes), scale, batch
        v0 = self.vols[0]
        self.shape = (v0.nz, v0.ny, v0.nx)
        self.cells = v0.nz * v0.ny * v0.nx
        dev = torch.device("cuda")
        self.x = torch.empty(batch * self.cells * 3, dtype=torch.float32, device=dev)
        self.y = torch.empty(batch * self.cells, dtype=torch.float32, device=dev)
        self.g = torch.empty(batch * self.cells, dtype=torch.float32, device=dev)
        self.b = torch.empty(batch * self.cells, dtype=torch.float32, device=dev)
        self.gen = torch.Generator(device=dev)
        self.gen.manual_seed(seed)
        self.dx2 = float(np.float32(v0.dx) ** 2)
        self.samples = 0
        if samples not in ("rhs", "vcycle"):
            raise ValueError(samples)
        self.kind = samples

    def _sample(self, k: int, vol: Volume3):
        """Random velocity on vol, its rhs into slot k of the batch, the input into x."""
        t = self.torch
        u = t.rand(vol.nu, generator=self.gen, device="cuda") * 2 - 1
        v = t.rand(vol.nv, generator=self.gen, device="cuda") * 2 - 1
        w = t.rand(vol.nw, generator=self.gen, device="cuda") * 2 - 1
        t.cuda.synchronize()  # the volume's stream reads them next
        vol.set_velocity_device(u.data_ptr(), v.data_ptr(), w.data_ptr())
        assemble_device(vol, self.scale)
        rhs, _ = problem_device(vol)
        n = self.cells
        bk = self.b[k * n:(k + 1) * n]
        t.cuda.synchronize()
        bk.copy_(_as_tensor(rhs, n))
        if self.kind == "vcycle":
            t.cuda.synchronize()
            vcycle_residual(vol, bk.data_ptr(), bk.data_ptr())
        rr = learned_input(vol, bk.data_ptr(), self.x[3 * k * n:3 * (k + 1) * n].data_ptr())
        return rr

    def step(self, lr: float, rng: np.random.Generator) -> float:
        """One batch: forward, residual loss and its gradient per sample, backward, Adam."""
        n, B = self.cells, self.batch
        picks = rng.integers(0, len(self.vols), size=B)
        rrs = [self._sample(k, self.vols[int(q)]) for k, q in enumerate(picks)]
        s = np.sqrt(np.maximum(np.array(rrs), 1e-300) / n)
        nz, ny, nx = self.shape
        self.net.forward(B, nz, ny, nx, self.x.data_ptr(), 1.0 / s, s * self.dx2, self.y.data_ptr())
        self.net.sync()
        loss = 0.0
        for k, q in enumerate(picks):
            vol = self.vols[int(q)]
            # A and the rhs of this sample: reassemble (the volume may have served another sample)
            w = 1.0 / (max(rrs[k], 1e-300) * B)
            yk, bk, gk = (self.y[k * n:(k + 1) * n], self.b[k * n:(k + 1) * n], self.g[k * n:(k + 1) * n])
            loss += residual_loss(vol, yk.data_ptr(), bk.data_ptr(), w, gk.data_ptr())
        self.net.backward(self.g.data_ptr())
        self.net.adam(lr)
        self.samples += B
        return loss


def _as_tensor(ptr: int, n: int):
    """A torch view of n f32 at a device pointer (through the CUDA array interface)."""
    import torch

    class _Blob:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Blob(), device="cuda")


def _forward_case(argv=None):
    """`python -m fluidisim_b200.learned forward [batch] [n] [repeat] [kernels] [tiles]`: U-Net
    forward passes of `batch` samples of n^3 cells (He-initialised weights, random input) on the
    convolution kernels `kernels` (0 mma.sync, 1 one-phase tcgen05, 2 pipelined tcgen05) with
    `tiles` 128-row tiles per CTA; prints the best CUDA-event time of one forward. Also a small
    case for a profiler's capture of the convolutions."""
    import json
    import sys

    import torch
    args = list(sys.argv[1:] if argv is None else argv)
    if not args or args[0] != "forward":
        raise SystemExit("usage: python -m fluidisim_b200.learned forward "
                         "[batch] [n] [repeat] [kernels] [tiles]")
    batch = int(args[1]) if len(args) > 1 else 4
    n = int(args[2]) if len(args) > 2 else 64
    repeat = int(args[3]) if len(args) > 3 else 3
    kernels = int(args[4]) if len(args) > 4 else 1
    tiles = int(args[5]) if len(args) > 5 else 5
    net = UNet(batch, n, n, n)
    net.set_params(init_params(0))
    net.set_conv_kernels(kernels)
    net.set_conv_tiles(tiles)
    x = torch.randn(batch * n ** 3 * 3, device="cuda")
    y = torch.empty(batch * n ** 3, device="cuda")
    stream = torch.cuda.Stream()
    net.set_stream(stream.cuda_stream)  # the events below see the launches
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(repeat):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        net.forward(batch, n, n, n, x.data_ptr(), 1.0, 1.0, y.data_ptr())
        b.record(stream)
        net.sync()
        best = min(best, a.elapsed_time(b))
    print(json.dumps({"batch": batch, "n": n, "kernels": kernels, "tiles": tiles,
                      "forward_ms": round(best, 3), "max_abs": float(y.abs().max())}))
    net.close()


if __name__ == "__main__":
    _forward_case()

