"""Python mirror of water-core's `Volume3` projection API over the C ABI of libfluidisim_delta3d.so.

Same method names, argument meanings and refusals as the reference
(code/water-core/src/delta3d.rs, delta3d_mobile.rs, delta3d_multigrid.rs): a refusal raises
`Delta3dError` whose `kind` is the reference's `Error` variant (Domain, NotFinite, Shape,
Convergence, ...), and leaves the published fields untouched.

The CUDA library is mandatory: importing works anywhere, but constructing a volume without the
built library or without a GPU raises; there is no CPU path behind this API.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluidisim_delta3d.so")

STATUS = {0: "Ok", 1: "Domain", 2: "NotFinite", 3: "Shape", 4: "Budget", 5: "Clock", 6: "Convergence",
          7: "BackgroundContext", 8: "NonPlanar", 100: "Cuda", 101: "NoDevice", 102: "InvalidArgument",
          103: "OutOfMemory"}

REDUCE_F64 = 0
REDUCE_ORDERED_F32 = 1
# storage of the V-cycle vectors (fd3_storage)
STORAGE_F32 = 0
STORAGE_F16 = 1


class Delta3dError(Exception):
    """A refusal of the projection API; `kind` names the reference's `Error` variant."""

    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        self.kind = STATUS.get(code, str(code))
        super().__init__(f"{where}: {self.kind}" + (f" ({detail})" if detail else ""))


class _Domain(C.Structure):
    _fields_ = [("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64), ("dx", C.c_float)]


class _Report(C.Structure):
    _fields_ = [("refinements", C.c_uint32), ("iterations", C.c_uint32), ("degraded", C.c_uint8),
                ("floor", C.c_uint8), ("pad", C.c_uint8 * 6), ("residual", C.c_double),
                ("divergence", C.c_double), ("backward_error", C.c_double), ("divergence_plain", C.c_double)]


class _Options(C.Structure):
    _fields_ = [("reduction", C.c_uint32), ("mg_max_levels", C.c_uint32), ("use_graphs", C.c_uint32),
                ("kernels", C.c_uint32), ("no_overlap", C.c_uint32), ("storage", C.c_uint32),
                ("no_tile_skip", C.c_uint32), ("reserved", C.c_uint32 * 1)]


class _SparseChange(C.Structure):
    _fields_ = [("activated", C.c_uint64), ("deactivated", C.c_uint64), ("active_columns", C.c_uint64),
                ("volume_removed", C.c_double), ("height_removed", C.c_float), ("velocity_removed", C.c_float)]


@dataclass
class SparseChange:
    """SparseChange (delta3d_sparse.rs:85-99): what a change of the sparse column set did."""
    activated: int
    deactivated: int
    active_columns: int
    volume_removed: float
    height_removed: float
    velocity_removed: float

    @staticmethod
    def _from(c: _SparseChange) -> "SparseChange":
        return SparseChange(int(c.activated), int(c.deactivated), int(c.active_columns), float(c.volume_removed),
                            float(c.height_removed), float(c.velocity_removed))


BLOCK = 8  # side of a block of the shared lattice, in columns (domain_blocks.rs:18)


class _LevelChange(C.Structure):
    _fields_ = [("volume_before", C.c_double), ("volume_after", C.c_double)]


@dataclass
class Report:
    """Report (delta_projection.rs:164-189)."""
    refinements: int
    iterations: int
    degraded: bool
    residual: float
    divergence: float
    floor: bool
    backward_error: float
    divergence_plain: float

    @staticmethod
    def _from(r: _Report) -> "Report":
        return Report(int(r.refinements), int(r.iterations), bool(r.degraded), float(r.residual),
                      float(r.divergence), bool(r.floor), float(r.backward_error), float(r.divergence_plain))

    def as_dict(self) -> dict:
        return dict(self.__dict__)


_LIB = None


def library() -> C.CDLL:
    """Load libfluidisim_delta3d.so (built in-tree by fluidisim_b200.build)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m fluidisim_b200.build` (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    vp, u64, f32, u32, sz = C.c_void_p, C.c_uint64, C.c_float, C.c_uint32, C.c_size_t
    fp = C.POINTER(C.c_float)
    L.fd3_version.restype = C.c_char_p
    L.fd3_last_cuda_error.restype = C.c_char_p
    L.fd3_configure.argtypes = [C.POINTER(_Domain), f32, f32, C.POINTER(vp)]
    L.fd3_configure_with_bottom.argtypes = [C.POINTER(_Domain), f32, f32, fp, sz, C.POINTER(vp)]
    L.fd3_configure_with_solid.argtypes = [C.POINTER(_Domain), f32, f32, fp, sz, fp, sz, C.POINTER(vp)]
    L.fd3_destroy.argtypes = [vp]
    L.fd3_destroy.restype = None
    L.fd3_set_options.argtypes = [vp, C.POINTER(_Options)]
    L.fd3_get_options.argtypes = [vp, C.POINTER(_Options)]
    L.fd3_set_stream.argtypes = [vp, vp]
    L.fd3_enable_multigrid.argtypes = [vp]
    L.fd3_multigrid_levels.argtypes = [vp]
    L.fd3_set_free_surface.argtypes = [vp, fp, sz, f32]
    L.fd3_set_surface.argtypes = [vp, fp, sz]
    L.fd3_set_velocity.argtypes = [vp, fp, sz, fp, sz, fp, sz]
    L.fd3_set_velocity_device.argtypes = [vp, vp, vp, vp]
    L.fd3_reset_pressure.argtypes = [vp]
    L.fd3_project_mobile.argtypes = [vp, f32, f32, u32, C.POINTER(_Report)]
    L.fd3_refine_mobile.argtypes = [vp, f32, f32, u32, C.POINTER(_Report)]
    L.fd3_set_solid_rigid.argtypes = [vp, fp, C.c_size_t, fp, fp, fp]
    L.fd3_set_solid.argtypes = [vp, fp, C.c_size_t, fp]
    L.fd3_step_surface_mobile.argtypes = [vp, u64, u32, C.POINTER(_Report)]
    L.fd3_last_refused_report.argtypes = [vp, C.POINTER(_Report)]
    L.fd3_project_linear.argtypes = [vp, f32, f32, u32, C.POINTER(_Report)]
    L.fd3_step_surface_linear.argtypes = [vp, u64, u32, C.POINTER(_Report)]
    L.fd3_set_precondition_cut.argtypes = [vp, C.c_int]
    L.fd3_enable_sparse.argtypes = [vp]
    L.fd3_set_active_columns.argtypes = [vp, vp, sz, C.POINTER(_SparseChange)]
    L.fd3_set_active_blocks.argtypes = [vp, vp, sz, C.c_int32, C.c_int32, C.POINTER(_SparseChange)]
    L.fd3_active_columns.argtypes = [vp, vp, sz]
    L.fd3_sparse_cells.argtypes = [vp]
    L.fd3_sparse_cells.restype = u64
    L.fd3_resample_from.argtypes = [vp, vp, C.POINTER(_LevelChange)]
    L.fd3_perturbation_volume.argtypes = [vp, C.POINTER(C.c_double)]
    L.fd3_enable_advection_correction.argtypes = [vp]
    L.fd3_advection_correction.argtypes = [vp]
    L.fd3_advect_for_tests.argtypes = [vp, f32]
    L.fd3_get_pressure.argtypes = [vp, fp, sz]
    L.fd3_get_velocity.argtypes = [vp, fp, sz, fp, sz, fp, sz]
    L.fd3_get_surface.argtypes = [vp, fp, fp, sz]
    L.fd3_device_fields.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    L.fd3_get_geometry.argtypes = [vp, fp, fp, fp, fp, fp]
    L.fd3_wet_cells.argtypes = [vp]
    L.fd3_wet_cells.restype = u64
    L.fd3_apply_pressure_operator_for_trials.argtypes = [vp, fp, fp, sz]
    L.fd3_assemble_pressure_problem_for_trials.argtypes = [vp, fp, f32, fp, fp, sz]
    L.fd3_vcycle_for_tests.argtypes = [vp, fp, fp, sz]
    L.fd3_level_geometry.argtypes = [vp, u32, fp, fp, fp, fp, fp]
    L.fd3_kernel_launches.argtypes = [vp]
    L.fd3_kernel_launches.restype = u64
    L.fd3_profile.argtypes = [vp, C.c_int]
    L.fd3_profile_count.argtypes = [vp]
    L.fd3_profile_entry.argtypes = [vp, C.c_int, C.c_char_p, sz, C.POINTER(u64), C.POINTER(C.c_double)]
    _LIB = L
    return L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Volume3:
    """One delta volume on the GPU: a flat bottom, a cut bottom, or a cut bottom plus a solid."""

    def __init__(self, handle, nx, ny, nz, dx, cut):
        self._h = handle
        self._L = library()
        self.nx, self.ny, self.nz, self.dx = nx, ny, nz, float(np.float32(dx))
        self.cut = cut
        self.cells = nx * ny * nz
        self.nu, self.nv, self.nw = (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)

    # ---- configure (delta3d.rs:210, 300, 327)
    @classmethod
    def configure(cls, nx, ny, nz, dx, rho=1025.0, g_eff=9.81) -> "Volume3":
        return cls._make(nx, ny, nz, dx, rho, g_eff, None, None)

    @classmethod
    def configure_with_bottom(cls, nx, ny, nz, dx, rho, g_eff, bottom) -> "Volume3":
        return cls._make(nx, ny, nz, dx, rho, g_eff, bottom, None)

    @classmethod
    def configure_with_solid(cls, nx, ny, nz, dx, rho, g_eff, bottom, solid) -> "Volume3":
        return cls._make(nx, ny, nz, dx, rho, g_eff, bottom, solid)

    @classmethod
    def _make(cls, nx, ny, nz, dx, rho, g_eff, bottom, solid):
        L = library()
        dom = _Domain(int(nx), int(ny), int(nz), np.float32(dx))
        h = C.c_void_p()
        if solid is not None:
            b = _f32(bottom if bottom is not None else np.zeros(int(nx) * int(ny)))
            s = _f32(solid)
            e = L.fd3_configure_with_solid(C.byref(dom), rho, g_eff, _fp(b), b.size, _fp(s), s.size, C.byref(h))
        elif bottom is not None:
            b = _f32(bottom)
            e = L.fd3_configure_with_bottom(C.byref(dom), rho, g_eff, _fp(b), b.size, C.byref(h))
        else:
            e = L.fd3_configure(C.byref(dom), rho, g_eff, C.byref(h))
        if e:
            raise Delta3dError(e, "configure", L.fd3_last_cuda_error().decode() if e >= 100 else "")
        return cls(h, int(nx), int(ny), int(nz), dx, bottom is not None or solid is not None)

    def close(self):
        if self._h:
            self._L.fd3_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, e, where):
        if e:
            raise Delta3dError(e, where, self._L.fd3_last_cuda_error().decode() if e >= 100 else "")

    # ---- options
    def set_options(self, reduction=None, mg_max_levels=None, use_graphs=None, kernels=None, no_overlap=None,
                    storage=None, no_tile_skip=None):
        o = _Options()
        self._check(self._L.fd3_get_options(self._h, C.byref(o)), "get_options")
        if reduction is not None:
            o.reduction = int(reduction)
        if mg_max_levels is not None:
            o.mg_max_levels = int(mg_max_levels)
        if use_graphs is not None:
            o.use_graphs = int(use_graphs)
        if kernels is not None:
            o.kernels = int(kernels)
        if no_overlap is not None:
            o.no_overlap = int(no_overlap)
        if storage is not None:
            o.storage = int(storage)
        if no_tile_skip is not None:
            o.no_tile_skip = int(no_tile_skip)
        self._check(self._L.fd3_set_options(self._h, C.byref(o)), "set_options")

    def set_stream(self, stream_ptr: int):
        self._check(self._L.fd3_set_stream(self._h, C.c_void_p(stream_ptr)), "set_stream")

    # ---- multigrid (delta3d_multigrid.rs:339, 353)
    def enable_multigrid(self):
        self._check(self._L.fd3_enable_multigrid(self._h), "enable_multigrid")

    def multigrid_levels(self):
        n = self._L.fd3_multigrid_levels(self._h)
        return None if n < 0 else n

    # ---- inputs
    def set_solid_rigid(self, solid, velocity=(0.0, 0.0, 0.0), angular=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)):
        """Volume3::set_solid_rigid (delta3d.rs:382-509): the solid's new signed distance at the nodes and
        its rigid motion (translation, rotation in rad/s about `center`)."""
        a = _f32(solid)
        vel, ang, cen = _f32(velocity), _f32(angular), _f32(center)
        self._check(self._L.fd3_set_solid_rigid(self._h, _fp(a), a.size, _fp(vel), _fp(ang), _fp(cen)),
                    "set_solid_rigid")

    def set_solid(self, solid, velocity=(0.0, 0.0, 0.0)):
        """Volume3::set_solid (delta3d.rs:376-378)."""
        a = _f32(solid)
        vel = _f32(velocity)
        self._check(self._L.fd3_set_solid(self._h, _fp(a), a.size, _fp(vel)), "set_solid")

    def set_free_surface(self, eta, rest):
        a = _f32(eta)
        self._check(self._L.fd3_set_free_surface(self._h, _fp(a), a.size, np.float32(rest)), "set_free_surface")

    def set_surface(self, eta):
        a = _f32(eta)
        self._check(self._L.fd3_set_surface(self._h, _fp(a), a.size), "set_surface")

    def set_velocity(self, u, v, w):
        a, b, c = _f32(u), _f32(v), _f32(w)
        self._check(self._L.fd3_set_velocity(self._h, _fp(a), a.size, _fp(b), b.size, _fp(c), c.size),
                    "set_velocity")

    def set_velocity_device(self, du: int, dv: int, dw: int):
        self._check(self._L.fd3_set_velocity_device(self._h, C.c_void_p(du), C.c_void_p(dv), C.c_void_p(dw)),
                    "set_velocity_device")

    def reset_pressure(self):
        self._check(self._L.fd3_reset_pressure(self._h), "reset_pressure")

    # ---- the sparse column set (delta3d_sparse.rs)
    def enable_sparse(self):
        """Volume3::enable_sparse (delta3d_sparse.rs:105): reserve the set, every column in it."""
        self._check(self._L.fd3_enable_sparse(self._h), "enable_sparse")

    def set_active_columns(self, mask) -> SparseChange:
        """Volume3::set_active_columns (delta3d_sparse.rs:147): mask[j*nx + i] != 0 puts column (i, j) in
        the set; a column that leaves goes to rest."""
        m = np.ascontiguousarray(np.asarray(mask).reshape(-1) != 0, dtype=np.uint8)
        ch = _SparseChange()
        self._check(self._L.fd3_set_active_columns(self._h, m.ctypes.data, m.size, C.byref(ch)), "set_active_columns")
        return SparseChange._from(ch)

    def set_active_blocks(self, blocks, origin=(0, 0)) -> SparseChange:
        """Volume3::set_active_blocks (delta3d_sparse.rs:163): the set from (i, j) blocks of BLOCK x BLOCK
        columns, relative to the block `origin` whose window starts at column (0, 0)."""
        b = np.ascontiguousarray(np.asarray(blocks, dtype=np.int32).reshape(-1, 2))
        ch = _SparseChange()
        self._check(self._L.fd3_set_active_blocks(self._h, b.ctypes.data, b.shape[0], int(origin[0]), int(origin[1]),
                                                  C.byref(ch)), "set_active_blocks")
        return SparseChange._from(ch)

    def active_columns(self):
        """Volume3::active_columns (delta3d_sparse.rs:129): one byte per column, or None without a set."""
        out = np.empty(self.nx * self.ny, np.uint8)
        e = self._L.fd3_active_columns(self._h, out.ctypes.data, out.size)
        if e == 1:
            return None
        self._check(e, "active_columns")
        return out

    def sparse_cells(self) -> int:
        """Volume3::sparse_cells (delta3d_sparse.rs:135)."""
        return int(self._L.fd3_sparse_cells(self._h))

    # ---- the level change (delta3d_levels.rs)
    def resample_from(self, src: "Volume3") -> dict:
        """Volume3::resample_from (delta3d_levels.rs:43): receive the state of `src`, the same window at
        another dx.  Returns LevelChange as {volume_before, volume_after}."""
        ch = _LevelChange()
        self._check(self._L.fd3_resample_from(self._h, src._h, C.byref(ch)), "resample_from")
        return {"volume_before": float(ch.volume_before), "volume_after": float(ch.volume_after)}

    def perturbation_volume(self) -> float:
        """Volume3::perturbation_volume (delta3d_balance.rs:105), m^3."""
        out = C.c_double()
        self._check(self._L.fd3_perturbation_volume(self._h, C.byref(out)), "perturbation_volume")
        return float(out.value)

    # ---- steps
    def project_mobile3(self, scale, k1, max_iters=4000) -> Report:
        """project_mobile3 of the current velocity (us = u), as tests_delta3d.rs:389-400 does."""
        r = _Report()
        self._check(self._L.fd3_project_mobile(self._h, np.float32(scale), np.float32(k1), int(max_iters),
                                               C.byref(r)), "project_mobile3")
        return Report._from(r)

    def refine_mobile3(self, scale, k1, max_iters=4000) -> Report:
        """refine_mobile3 (delta3d_coupling.rs:226-248): project the current field again from p = 0 with
        homogeneous ghosts and add the increment to the current pressure."""
        r = _Report()
        self._check(self._L.fd3_refine_mobile(self._h, np.float32(scale), np.float32(k1), int(max_iters),
                                              C.byref(r)), "refine_mobile3")
        return Report._from(r)

    def step_surface_mobile(self, duration_us, max_iters=4000) -> Report:
        r = _Report()
        self._check(self._L.fd3_step_surface_mobile(self._h, int(duration_us), int(max_iters), C.byref(r)),
                    "step_surface_mobile")
        return Report._from(r)

    def enable_advection_correction(self):
        """Volume3::enable_advection_correction (delta3d_advection.rs:19): the second-order advection term."""
        self._check(self._L.fd3_enable_advection_correction(self._h), "enable_advection_correction")

    def advection_correction(self) -> bool:
        return bool(self._L.fd3_advection_correction(self._h))

    def advect_for_tests(self, dt):
        """The predictor alone (tests_delta3d.rs:2136-2160): advection over dt, the second-order term when on,
        then u = us."""
        self._check(self._L.fd3_advect_for_tests(self._h, np.float32(dt)), "advect_for_tests")

    def last_refused_report(self):
        r = _Report()
        return None if self._L.fd3_last_refused_report(self._h, C.byref(r)) else Report._from(r)

    # ---- the linear (fixed-lid) path (delta3d.rs:1060-1357)
    def project(self, scale, k1, max_iters=4000) -> Report:
        """project (delta3d.rs:1060) of the current velocity (us = u), as tests_delta3d.rs:143-148 does."""
        r = _Report()
        self._check(self._L.fd3_project_linear(self._h, np.float32(scale), np.float32(k1), int(max_iters),
                                               C.byref(r)), "project")
        return Report._from(r)

    def step_surface_linear(self, duration_us, max_iters=4000) -> Report:
        r = _Report()
        self._check(self._L.fd3_step_surface_linear(self._h, int(duration_us), int(max_iters), C.byref(r)),
                    "step_surface_linear")
        return Report._from(r)

    def set_precondition_cut(self, on: bool):
        """set_precondition_cut (delta3d.rs:526): Jacobi on the linear path's cut bottom."""
        self._check(self._L.fd3_set_precondition_cut(self._h, 1 if on else 0), "set_precondition_cut")

    # ---- outputs (delta3d.rs:647-661)
    def pressure(self) -> np.ndarray:
        out = np.empty(self.cells, np.float32)
        self._check(self._L.fd3_get_pressure(self._h, _fp(out), out.size), "pressure")
        return out

    def velocity(self):
        u, v, w = np.empty(self.nu, np.float32), np.empty(self.nv, np.float32), np.empty(self.nw, np.float32)
        self._check(self._L.fd3_get_velocity(self._h, _fp(u), u.size, _fp(v), v.size, _fp(w), w.size), "velocity")
        return u, v, w

    def velocity_u(self):
        return self.velocity()[0]

    def velocity_v(self):
        return self.velocity()[1]

    def velocity_w(self):
        return self.velocity()[2]

    def surface(self) -> np.ndarray:
        return self.surface_and_roundoff()[0]

    def surface_and_roundoff(self):
        e, r = np.empty(self.nx * self.ny, np.float32), np.empty(self.nx * self.ny, np.float32)
        self._check(self._L.fd3_get_surface(self._h, _fp(e), _fp(r), e.size), "surface")
        return e, r

    def device_fields(self):
        p, u, v, w = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._check(self._L.fd3_device_fields(self._h, C.byref(p), C.byref(u), C.byref(v), C.byref(w)),
                    "device_fields")
        return p.value, u.value, v.value, w.value

    def geometry(self):
        """(frac, open_u, open_v, open_w, floor) of a cut volume (delta3d.rs:595-602)."""
        out = (np.empty(self.cells, np.float32), np.empty(self.nu, np.float32), np.empty(self.nv, np.float32),
               np.empty(self.nw, np.float32), np.empty(self.nx * self.ny, np.float32))
        self._check(self._L.fd3_get_geometry(self._h, *[_fp(o) for o in out]), "geometry")
        return out

    def wet_cells(self) -> int:
        return int(self._L.fd3_wet_cells(self._h))

    # ---- trial hooks (delta3d_mobile.rs:936, 960) and the V-cycle
    def apply_pressure_operator_for_trials(self, p) -> np.ndarray:
        a = _f32(p)
        out = np.empty(self.cells, np.float32)
        self._check(self._L.fd3_apply_pressure_operator_for_trials(self._h, _fp(a), _fp(out), a.size),
                    "apply_pressure_operator_for_trials")
        return out

    def assemble_pressure_problem_for_trials(self, divergence, scale):
        a = _f32(divergence)
        rhs, prec = np.empty(self.cells, np.float32), np.empty(self.cells, np.float32)
        self._check(self._L.fd3_assemble_pressure_problem_for_trials(self._h, _fp(a), np.float32(scale), _fp(rhs),
                                                                     _fp(prec), a.size),
                    "assemble_pressure_problem_for_trials")
        return rhs, prec

    def vcycle_for_tests(self, x) -> np.ndarray:
        a = _f32(x)
        z = np.empty(self.cells, np.float32)
        self._check(self._L.fd3_vcycle_for_tests(self._h, _fp(a), _fp(z), a.size), "vcycle_for_tests")
        return z

    def level_geometry(self, level: int):
        L = self._level_dims(level)
        cx, cy, cz = L
        out = (np.empty(cx * cy * cz, np.float32), np.empty(cx * cy * cz, np.float32),
               np.empty((cx + 1) * cy * cz, np.float32), np.empty(cx * (cy + 1) * cz, np.float32),
               np.empty(cx * cy * (cz + 1), np.float32))
        self._check(self._L.fd3_level_geometry(self._h, level, *[_fp(o) for o in out]), "level_geometry")
        return out

    def _level_dims(self, level):
        x, y, z = self.nx, self.ny, self.nz
        for _ in range(level + 1):
            x, y, z = x // 2, y // 2, z // 2
        return x, y, z

    def kernel_launches(self) -> int:
        return int(self._L.fd3_kernel_launches(self._h))

    def profile(self, on: bool):
        """Per-kernel CUDA-event timing of every launch of this volume (graph replay bypassed)."""
        self._check(self._L.fd3_profile(self._h, 1 if on else 0), "profile")

    def profile_entries(self):
        """[(kernel name, launches, total ms)] accumulated since profile(True)."""
        out = []
        for q in range(self._L.fd3_profile_count(self._h)):
            name = C.create_string_buffer(128)
            n, ms = C.c_uint64(), C.c_double()
            self._check(self._L.fd3_profile_entry(self._h, q, name, 128, C.byref(n), C.byref(ms)), "profile_entry")
            out.append((name.value.decode(), int(n.value), float(ms.value)))
        return out
