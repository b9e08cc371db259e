"""Many independent δ patches projected together: the batched entry point, the patch scenes, and
the autotuner that picks the solver options per size class.

There is no reference counterpart (the reference projects one `Volume3` at a time).  Each patch
is an ordinary volume; `project_batch` hands them all to `fd3_project_batch`, which runs their
device-side PCG loops concurrently on their own streams from a pool of host workers.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import scenes
from .delta3d import REDUCE_F64, Delta3dError, Report, Volume3, _Report, library

SIZE_CLASSES = [("small", 0, 48 ** 3), ("medium", 48 ** 3, 80 ** 3), ("large", 80 ** 3, 1 << 62)]
# (kernels, mg_max_levels): fine-level kernel family and V-cycle depth (0 = every level)
CANDIDATES = [(0, 0), (1, 0), (2, 0), (0, 3), (1, 3)]


def _bind(L):
    if not getattr(L, "_batch_bound", False):
        L.fd3_project_batch.argtypes = [C.POINTER(C.c_void_p), C.c_size_t, C.POINTER(C.c_float),
                                        C.POINTER(C.c_float), C.c_uint32, C.c_int, C.POINTER(_Report),
                                        C.POINTER(C.c_int)]
        vpp = C.POINTER(C.c_void_p)
        L.fd3_batch_create.argtypes = [vpp, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]
        L.fd3_batch_destroy.argtypes = [C.c_void_p]
        L.fd3_batch_destroy.restype = None
        L.fd3_batch_clusters.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.fd3_batch_kernel_launches.argtypes = [C.c_void_p]
        L.fd3_batch_kernel_launches.restype = C.c_uint64
        L.fd3_batch_project.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint32, C.c_int,
                                        vpp, vpp, vpp, C.POINTER(_Report), C.POINTER(C.c_int)]
        L._batch_bound = True
    return L


def size_class(cells: int) -> str:
    for name, lo, hi in SIZE_CLASSES:
        if lo <= cells < hi:
            return name
    return SIZE_CLASSES[-1][0]


def patch_scene(rng: scenes.SplitMix64, lo: int = 16, hi: int = 96, quantum: int = 8, dx: float = 0.1) -> dict:
    """One patch: sides log-uniform in [lo, hi] per axis, rounded to a multiple of `quantum` (so the
    reference's coarsening rule, which halves while every side is even, gives a multigrid), solid
    spheres (radius U[2, 6] cells, clear of the walls, the bottom layer and the lid layer) added
    until 5-15 % of the cells are solid (the target drawn U[0.05, 0.15]), fill fraction U[0.3, 0.8],
    faces U[-1, 1] m/s."""
    def side():
        s = np.exp(rng.uniform(np.log(lo), np.log(hi)))
        return int(max(quantum, quantum * round(s / quantum)))
    nx, ny, nz = side(), side(), side()
    d = float(np.float32(dx))
    target = rng.uniform(0.05, 0.15)
    fill = rng.uniform(0.3, 0.8)
    centres, radii = [], []
    cells = nx * ny * nz
    solid = 0.0
    for _ in range(400):
        if solid >= target * cells:
            break
        r = rng.uniform(2.0, 6.0)
        r = min(r, (min(nx, ny) - 2.5) / 2.0, (nz - 3.5) / 2.0)
        if r < 1.0:
            break
        cx = rng.uniform(r + 1.0, nx - r - 1.0)
        cy = rng.uniform(r + 1.0, ny - r - 1.0)
        cz = rng.uniform(r + 1.0, nz - r - 2.0)
        centres.append((cx * d, cy * d, cz * d))
        radii.append(r * d)
        solid += 4.0 / 3.0 * np.pi * r ** 3
    sdf = scenes.spheres_sdf(nx, ny, nz, dx, centres, radii) if centres else \
        np.full((nx + 1) * (ny + 1) * (nz + 1), 1e3, np.float32)
    nu, nv, nw = scenes.face_counts(nx, ny, nz)
    eta = np.full(nx * ny, np.float32(fill * nz * d), np.float32)
    return dict(nx=nx, ny=ny, nz=nz, dx=d, rho=1025.0, g=9.81, bottom=np.zeros(nx * ny, np.float32), solid=sdf,
                eta=eta, rest=float(eta[0]), u=rng.uniform_array(nu, -1.0, 1.0), v=rng.uniform_array(nv, -1.0, 1.0),
                w=rng.uniform_array(nw, -1.0, 1.0), dt=1.0 / 60.0, fill=fill, solid_target=target)


def patch_scenes(count: int = 256, seed: int = 3, **kw) -> list:
    rng = scenes.SplitMix64(seed)
    return [patch_scene(rng, **kw) for _ in range(count)]


def configure(scene: dict, kernels: int = 0, levels: int = 0) -> Volume3:
    v = Volume3.configure_with_solid(scene["nx"], scene["ny"], scene["nz"], scene["dx"], scene["rho"], scene["g"],
                                     scene["bottom"], scene["solid"])
    v.set_options(reduction=REDUCE_F64, kernels=kernels, mg_max_levels=levels)
    v.enable_multigrid()
    v.set_free_surface(scene["eta"], scene["rest"])
    v.set_velocity(scene["u"], scene["v"], scene["w"])
    return v


def project_batch(volumes, scales, k1s, max_iters: int = 4000, threads: int = 0):
    """fd3_project_batch: returns (reports, statuses); a status is 0 or the volume's refusal."""
    vols = list(volumes)
    n = len(vols)
    L = _bind(library())
    arr = (C.c_void_p * n)(*[v._h.value for v in vols])
    sc = np.ascontiguousarray(scales, np.float32)
    kk = np.ascontiguousarray(k1s, np.float32)
    reps = (_Report * n)()
    st = (C.c_int * n)()
    e = L.fd3_project_batch(arr, n, sc.ctypes.data_as(C.POINTER(C.c_float)), kk.ctypes.data_as(C.POINTER(C.c_float)),
                            max_iters, threads, reps, st)
    if e:
        raise Delta3dError(e, "fd3_project_batch")
    return [Report._from(reps[i]) for i in range(n)], [int(st[i]) for i in range(n)]


class PersistentBatch:
    """fd3_batch: the volumes projected by one persistent kernel launch (thread-block clusters as
    independent solvers, each taking its share of the volumes, largest first).  Create once (all
    allocations happen there), project many times; close before the volumes."""

    def __init__(self, volumes, cluster_size: int = 4):
        self.vols = list(volumes)
        L = _bind(library())
        self._L = L
        arr = (C.c_void_p * len(self.vols))(*[v._h.value for v in self.vols])
        h = C.c_void_p()
        e = L.fd3_batch_create(arr, len(self.vols), int(cluster_size), C.byref(h))
        if e:
            raise Delta3dError(e, "fd3_batch_create", L.fd3_last_cuda_error().decode() if e >= 100 else "")
        self._h = h
        n, cs = C.c_int(), C.c_int()
        L.fd3_batch_clusters(h, C.byref(n), C.byref(cs))
        self.clusters, self.cluster_size = n.value, cs.value

    def project(self, scales, k1s, max_iters: int = 4000, reset_pressure: bool = False, inputs=None):
        """Returns (reports, statuses).  inputs: None, or per volume a (u, v, w) of device pointers
        copied into the volume's velocity first."""
        n = len(self.vols)
        sc = np.ascontiguousarray(scales, np.float32)
        kk = np.ascontiguousarray(k1s, np.float32)
        reps = (_Report * n)()
        st = (C.c_int * n)()
        if inputs is not None:
            iu = (C.c_void_p * n)(*[x[0] for x in inputs])
            iv = (C.c_void_p * n)(*[x[1] for x in inputs])
            iw = (C.c_void_p * n)(*[x[2] for x in inputs])
        else:
            iu = iv = iw = None
        e = self._L.fd3_batch_project(self._h, sc.ctypes.data_as(C.POINTER(C.c_float)),
                                      kk.ctypes.data_as(C.POINTER(C.c_float)), int(max_iters),
                                      1 if reset_pressure else 0, iu, iv, iw, reps, st)
        if e:
            raise Delta3dError(e, "fd3_batch_project", self._L.fd3_last_cuda_error().decode() if e >= 100 else "")
        return [Report._from(reps[i]) for i in range(n)], [int(st[i]) for i in range(n)]

    def kernel_launches(self) -> int:
        return int(self._L.fd3_batch_kernel_launches(self._h))

    def close(self):
        if self._h:
            self._L.fd3_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Tuned:
    kernels: int
    levels: int
    ms: float


def autotune(scenes_by_class: dict, repeats: int = 3, timer=None) -> dict:
    """Per size class, time every candidate (kernel family, V-cycle depth) on the class's largest
    patch (best of `repeats` projections) and keep the fastest.  `timer(scene, kernels, levels)`
    replaces the measurement (tests); by default it configures the patch and times
    fd3_project_mobile with device synchronisation around each call."""
    def measure(scene, kernels, levels):
        v = configure(scene, kernels, levels)
        scale, k1 = scenes.projection_scalars(scene)
        best = float("inf")
        for _ in range(repeats + 1):
            v.set_velocity(scene["u"], scene["v"], scene["w"])
            v.reset_pressure()
            t0 = time.perf_counter()
            v.project_mobile3(scale, k1, 4000)
            best = min(best, time.perf_counter() - t0)
        v.close()
        return best * 1e3
    timer = timer or measure
    out = {}
    for name, group in scenes_by_class.items():
        if not group:
            continue
        big = max(group, key=lambda s: s["nx"] * s["ny"] * s["nz"])
        times = {(k, l): timer(big, k, l) for k, l in CANDIDATES}
        (k, l), ms = min(times.items(), key=lambda kv: kv[1])
        out[name] = Tuned(k, l, ms)
    return out


def snake_owner(k: int, world: int) -> int:
    """Rank of the k-th patch in decreasing cost: 0, 1, ..., w-1, w-1, ..., 0, 0, 1, ..."""
    q, r = divmod(k, world)
    return r if q % 2 == 0 else world - 1 - r


def deal(cells, world: int, rank: int) -> list:
    """The indices of the patches rank `rank` projects: patches sorted by decreasing cell count
    (ties by index) and dealt in snake order, so each rank gets every patch once and the ranks'
    cell loads differ by at most one patch.  No data moves between ranks."""
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    return [i for k, i in enumerate(order) if snake_owner(k, world) == rank]


def reduce_totals(ms: float, cells_iterations: float, world: int, device="cpu"):
    """The two collectives of the sharded patch run: the slowest rank's device time (max) and the
    cells x iterations of all ranks (sum).  One rank returns its own values unchanged."""
    if world == 1:
        return float(ms), float(cells_iterations)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells_iterations)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def by_class(scene_list) -> dict:
    out = {name: [] for name, _, _ in SIZE_CLASSES}
    for s in scene_list:
        out[size_class(s["nx"] * s["ny"] * s["nz"])].append(s)
    return out
