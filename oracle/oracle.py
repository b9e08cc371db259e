"""ctypes binding of the CPU oracle (oracle/delta3d_oracle.cpp).

TEST INFRASTRUCTURE ONLY: this module is the parity checker and the timed CPU baseline.  The
product package (fluidisim_b200) never imports it; only tests/, the smoke check and bench.py's
CPU-baseline leg do.

`OracleVolume` mirrors water-core's `Volume3` projection API (code/water-core/src/delta3d.rs,
delta3d_mobile.rs, delta3d_multigrid.rs) one call per method.  The f32 build restates the
reference bit for bit; the f64 build (`real="f64"`) runs the same algorithm in double precision
and serves as the error reference.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

ERRORS = {0: "Ok", 1: "Domain", 2: "NotFinite", 3: "Shape", 4: "Budget", 5: "Clock",
          6: "Convergence", 102: "InvalidArgument"}


class OracleError(Exception):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}")
        self.code = code
        self.kind = ERRORS.get(code, str(code))


class _Domain(C.Structure):
    _fields_ = [("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64), ("dx", C.c_float)]


def build() -> None:
    """Compile the oracle libraries (f32 and f64) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_LIBS: dict[str, C.CDLL] = {}


def lib(real: str = "f32") -> C.CDLL:
    if real in _LIBS:
        return _LIBS[real]
    path = os.path.join(BUILD, f"liboracle_delta3d_{real}.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, u64, f32, u32 = C.c_void_p, C.c_uint64, C.c_float, C.c_uint32
    fp = C.POINTER(C.c_float)
    L.od3_configure.argtypes = [C.POINTER(_Domain), f32, f32, C.POINTER(vp)]
    L.od3_configure_with_bottom.argtypes = [C.POINTER(_Domain), f32, f32, fp, u64, C.POINTER(vp)]
    L.od3_configure_with_solid.argtypes = [C.POINTER(_Domain), f32, f32, fp, u64, fp, u64, C.POINTER(vp)]
    L.od3_destroy.argtypes = [vp]
    L.od3_destroy.restype = None
    L.od3_enable_multigrid.argtypes = [vp, u32]
    L.od3_multigrid_levels.argtypes = [vp]
    L.od3_level_count3.argtypes = [u64, u64, u64]
    L.od3_level_count3.restype = u64
    L.od3_hierarchy_floats3.argtypes = [u64, u64, u64]
    L.od3_hierarchy_floats3.restype = u64
    L.od3_set_free_surface.argtypes = [vp, fp, u64, f32]
    L.od3_set_surface.argtypes = [vp, fp, u64]
    L.od3_set_velocity.argtypes = [vp, fp, u64, fp, u64, fp, u64]
    L.od3_set_tolerance.argtypes = [vp, f32]
    dp = C.POINTER(C.c_double)
    L.od3_project_mobile.argtypes = [vp, f32, f32, u32, dp]
    L.od3_step_surface_mobile.argtypes = [vp, u64, u32, dp]
    L.od3_last_refused_report.argtypes = [vp, dp]
    L.od3_get_pressure.argtypes = [vp, vp, u64]
    L.od3_get_velocity.argtypes = [vp, vp, u64, vp, u64, vp, u64]
    L.od3_get_surface.argtypes = [vp, vp, vp, u64]
    L.od3_get_rhs_prec.argtypes = [vp, vp, vp, u64]
    L.od3_get_geometry.argtypes = [vp, vp, vp, vp, vp, vp]
    L.od3_wet_cells.argtypes = [vp]
    L.od3_wet_cells.restype = u64
    L.od3_apply_pressure_operator_for_trials.argtypes = [vp, fp, vp, u64]
    L.od3_assemble_pressure_problem_for_trials.argtypes = [vp, fp, f32, vp, vp, u64]
    L.od3_vcycle_for_tests.argtypes = [vp, fp, vp, u64]
    L.od3_level_geometry.argtypes = [vp, u32, vp, vp, vp, vp, vp]
    L.od3_fingerprint.argtypes = [fp, u64]
    L.od3_fingerprint.restype = u64
    L.od3_set_threads.argtypes = [C.c_int]
    L.od3_set_threads.restype = None
    L.od3_max_threads.restype = C.c_int
    L.od3_set_smoother.argtypes = [C.c_int]
    L.od3_set_smoother.restype = None
    L.od3_set_transfer.argtypes = [C.c_int]
    L.od3_set_transfer.restype = None
    L.od3_set_storage.argtypes = [C.c_int]
    L.od3_set_storage.restype = None
    L.od3_take_zmax.argtypes = []
    L.od3_take_zmax.restype = C.c_double
    L.od3_project_linear.argtypes = [vp, f32, f32, u32, dp]
    L.od3_refine_mobile.argtypes = [vp, f32, f32, u32, dp]
    L.od3_set_solid_rigid.argtypes = [vp, fp, u64, fp, fp, fp]
    L.od3_step_surface_linear.argtypes = [vp, u64, u32, dp]
    L.od3_set_precondition_cut.argtypes = [vp, C.c_int]
    L.od3_enable_sparse.argtypes = [vp]
    L.od3_set_active_columns.argtypes = [vp, vp, u64, dp]
    L.od3_set_active_blocks.argtypes = [vp, vp, u64, C.c_int32, C.c_int32, dp]
    L.od3_active_columns.argtypes = [vp, vp, u64]
    L.od3_sparse_cells.argtypes = [vp]
    L.od3_sparse_cells.restype = u64
    L.od3_resample_from.argtypes = [vp, vp, dp]
    L.od3_perturbation_volume.argtypes = [vp]
    L.od3_perturbation_volume.restype = C.c_double
    L.od3_enable_advection_correction.argtypes = [vp]
    L.od3_advect_for_tests.argtypes = [vp, f32]
    _LIBS[real] = L
    return L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


REPORT_KEYS = ("refinements", "iterations", "degraded", "residual", "divergence", "floor",
               "backward_error", "divergence_plain")


def report_dict(rep) -> dict:
    d = dict(zip(REPORT_KEYS, [float(x) for x in rep]))
    d["refinements"] = int(d["refinements"])
    d["iterations"] = int(d["iterations"])
    d["degraded"] = bool(d["degraded"])
    d["floor"] = bool(d["floor"])
    return d


CHANGE_KEYS = ("activated", "deactivated", "active_columns", "volume_removed", "height_removed",
               "velocity_removed")


def change_dict(ch) -> dict:
    """SparseChange (delta3d_sparse.rs:85-99) from the six doubles the oracle writes."""
    d = dict(zip(CHANGE_KEYS, [float(x) for x in ch]))
    for k in ("activated", "deactivated", "active_columns"):
        d[k] = int(d[k])
    d["height_removed"] = float(np.float32(d["height_removed"]))
    d["velocity_removed"] = float(np.float32(d["velocity_removed"]))
    return d


def set_threads(n: int, real: str = "f32") -> None:
    lib(real).od3_set_threads(int(n))


def set_smoother(smoother: int, real: str = "f32") -> None:
    """0: damped Jacobi on every level, the reference's (omega = 6/7); 1: red-black Gauss-Seidel on
    every level, red first going down and black first coming up (a symmetric V-cycle); 2: red-black
    on the fine level only; 3: red-black on the coarse levels only."""
    lib(real).od3_set_smoother(int(smoother))


def set_transfer(transfer: int, real: str = "f32") -> None:
    """0: the reference's 8-child mean and injection; 1: trilinear prolongation from the active coarse
    cells (renormalised) and its adjoint restriction (full weighting)."""
    lib(real).od3_set_transfer(int(transfer))


def set_storage(storage: int, real: str = "f32") -> None:
    """0: f32 V-cycle storage (the reference); 1: emulate the library's FP16 storage mode."""
    lib(real).od3_set_storage(int(storage))


def take_zmax(real: str = "f32") -> float:
    """Largest |z| a V-cycle returned in the FP16 mode since the last call."""
    return float(lib(real).od3_take_zmax())


def max_threads(real: str = "f32") -> int:
    return int(lib(real).od3_max_threads())


def level_count3(nx, ny, nz) -> int:
    return int(lib().od3_level_count3(nx, ny, nz))


def hierarchy_floats3(nx, ny, nz) -> int:
    return int(lib().od3_hierarchy_floats3(nx, ny, nz))


def fingerprint(p) -> int:
    a = _f32(p)
    return int(lib().od3_fingerprint(_fptr(a), a.size))


class OracleVolume:
    """One reference `Volume3` (flat bottom, cut bottom, or cut bottom plus a solid SDF)."""

    def __init__(self, nx, ny, nz, dx, rho=1025.0, g=9.81, bottom=None, solid=None, real="f32"):
        self.L = lib(real)
        self.dtype = np.float32 if real == "f32" else np.float64
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(np.float32(dx))
        dom = _Domain(self.nx, self.ny, self.nz, np.float32(dx))
        h = C.c_void_p()
        if solid is not None:
            b = _f32(bottom if bottom is not None else np.zeros(self.nx * self.ny))
            s = _f32(solid)
            e = self.L.od3_configure_with_solid(C.byref(dom), rho, g, _fptr(b), b.size, _fptr(s), s.size, C.byref(h))
        elif bottom is not None:
            b = _f32(bottom)
            e = self.L.od3_configure_with_bottom(C.byref(dom), rho, g, _fptr(b), b.size, C.byref(h))
        else:
            e = self.L.od3_configure(C.byref(dom), rho, g, C.byref(h))
        if e:
            raise OracleError(e, "configure")
        self.h = h
        self.cut = bottom is not None or solid is not None
        n = self.nx * self.ny * self.nz
        self.cells = n
        self.nu = (self.nx + 1) * self.ny * self.nz
        self.nv = self.nx * (self.ny + 1) * self.nz
        self.nw = self.nx * self.ny * (self.nz + 1)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.od3_destroy(h)
            self.h = None

    def _check(self, e, where):
        if e:
            raise OracleError(e, where)

    def enable_multigrid(self, max_levels: int = 0):
        self._check(self.L.od3_enable_multigrid(self.h, max_levels), "enable_multigrid")

    def multigrid_levels(self):
        n = self.L.od3_multigrid_levels(self.h)
        return None if n < 0 else n

    def set_free_surface(self, eta, rest):
        a = _f32(eta)
        self._check(self.L.od3_set_free_surface(self.h, _fptr(a), a.size, np.float32(rest)), "set_free_surface")

    def set_surface(self, eta):
        a = _f32(eta)
        self._check(self.L.od3_set_surface(self.h, _fptr(a), a.size), "set_surface")

    def set_velocity(self, u, v, w):
        a, b, c = _f32(u), _f32(v), _f32(w)
        self._check(self.L.od3_set_velocity(self.h, _fptr(a), a.size, _fptr(b), b.size, _fptr(c), c.size),
                    "set_velocity")

    def set_tolerance(self, tol2: float):
        self._check(self.L.od3_set_tolerance(self.h, tol2), "set_tolerance")

    def project_mobile(self, scale, k1, max_iters=4000) -> dict:
        rep = (C.c_double * 8)()
        self._check(self.L.od3_project_mobile(self.h, np.float32(scale), np.float32(k1), max_iters, rep),
                    "project_mobile")
        return report_dict(rep)

    def set_solid_rigid(self, solid, velocity=(0.0, 0.0, 0.0), angular=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)):
        """set_solid_rigid (delta3d.rs:382-509): the solid's new signed distance at the nodes."""
        a = _f32(solid)
        vel, ang, cen = _f32(velocity), _f32(angular), _f32(center)
        self._check(self.L.od3_set_solid_rigid(self.h, _fptr(a), a.size, _fptr(vel), _fptr(ang), _fptr(cen)),
                    "set_solid_rigid")

    def refine_mobile(self, scale, k1, max_iters=4000) -> dict:
        """refine_mobile3 (delta3d_coupling.rs:226-248) of the current state."""
        rep = (C.c_double * 8)()
        self._check(self.L.od3_refine_mobile(self.h, np.float32(scale), np.float32(k1), max_iters, rep),
                    "refine_mobile")
        return report_dict(rep)

    def step_surface_mobile(self, duration_us, max_iters=4000) -> dict:
        rep = (C.c_double * 8)()
        self._check(self.L.od3_step_surface_mobile(self.h, duration_us, max_iters, rep), "step_surface_mobile")
        return report_dict(rep)

    def project_linear(self, scale, k1, max_iters=4000) -> dict:
        """project (delta3d.rs:1060-1196) of the current velocity field, as tests_delta3d.rs:143-148."""
        rep = (C.c_double * 8)()
        self._check(self.L.od3_project_linear(self.h, np.float32(scale), np.float32(k1), max_iters, rep),
                    "project_linear")
        return report_dict(rep)

    def step_surface_linear(self, duration_us, max_iters=4000) -> dict:
        rep = (C.c_double * 8)()
        self._check(self.L.od3_step_surface_linear(self.h, duration_us, max_iters, rep), "step_surface_linear")
        return report_dict(rep)

    def set_precondition_cut(self, on: bool):
        self._check(self.L.od3_set_precondition_cut(self.h, 1 if on else 0), "set_precondition_cut")

    # The sparse column set (delta3d_sparse.rs:101-178).
    def enable_sparse(self):
        self._check(self.L.od3_enable_sparse(self.h), "enable_sparse")

    def set_active_columns(self, mask) -> dict:
        m = np.ascontiguousarray(np.asarray(mask) != 0, dtype=np.uint8)
        ch = (C.c_double * 6)()
        self._check(self.L.od3_set_active_columns(self.h, m.ctypes.data, m.size, ch), "set_active_columns")
        return change_dict(ch)

    def set_active_blocks(self, blocks, origin=(0, 0)) -> dict:
        b = np.ascontiguousarray(np.asarray(blocks, dtype=np.int32).reshape(-1, 2))
        ch = (C.c_double * 6)()
        self._check(self.L.od3_set_active_blocks(self.h, b.ctypes.data, b.shape[0], int(origin[0]), int(origin[1]),
                                                 ch), "set_active_blocks")
        return change_dict(ch)

    def active_columns(self) -> np.ndarray:
        out = np.empty(self.nx * self.ny, np.uint8)
        self._check(self.L.od3_active_columns(self.h, out.ctypes.data, out.size), "active_columns")
        return out

    def sparse_cells(self) -> int:
        return int(self.L.od3_sparse_cells(self.h))

    # The level change (delta3d_levels.rs:38-69).
    def resample_from(self, src: "OracleVolume") -> dict:
        out = (C.c_double * 2)()
        self._check(self.L.od3_resample_from(self.h, src.h, out), "resample_from")
        return {"volume_before": float(out[0]), "volume_after": float(out[1])}

    def enable_advection_correction(self):
        """enable_advection_correction (delta3d_advection.rs:17-21): the second-order term of the advection."""
        self._check(self.L.od3_enable_advection_correction(self.h), "enable_advection_correction")

    def advect_for_tests(self, dt):
        self._check(self.L.od3_advect_for_tests(self.h, np.float32(dt)), "advect_for_tests")

    def perturbation_volume(self) -> float:
        return float(self.L.od3_perturbation_volume(self.h))

    def last_refused_report(self):
        rep = (C.c_double * 8)()
        return None if self.L.od3_last_refused_report(self.h, rep) else report_dict(rep)

    def pressure(self) -> np.ndarray:
        out = np.empty(self.cells, self.dtype)
        self._check(self.L.od3_get_pressure(self.h, out.ctypes.data, out.size), "pressure")
        return out

    def velocity(self):
        u, v, w = np.empty(self.nu, self.dtype), np.empty(self.nv, self.dtype), np.empty(self.nw, self.dtype)
        self._check(self.L.od3_get_velocity(self.h, u.ctypes.data, u.size, v.ctypes.data, v.size, w.ctypes.data,
                                            w.size), "velocity")
        return u, v, w

    def surface(self):
        e, r = np.empty(self.nx * self.ny, self.dtype), np.empty(self.nx * self.ny, self.dtype)
        self._check(self.L.od3_get_surface(self.h, e.ctypes.data, r.ctypes.data, e.size), "surface")
        return e, r

    def rhs_prec(self):
        r, p = np.empty(self.cells, self.dtype), np.empty(self.cells, self.dtype)
        self._check(self.L.od3_get_rhs_prec(self.h, r.ctypes.data, p.ctypes.data, r.size), "rhs_prec")
        return r, p

    def geometry(self):
        """(frac, open_u, open_v, open_w, floor) of a cut volume."""
        out = (np.empty(self.cells, self.dtype), np.empty(self.nu, self.dtype), np.empty(self.nv, self.dtype),
               np.empty(self.nw, self.dtype), np.empty(self.nx * self.ny, self.dtype))
        self._check(self.L.od3_get_geometry(self.h, *[o.ctypes.data for o in out]), "geometry")
        return out

    def wet_cells(self) -> int:
        return int(self.L.od3_wet_cells(self.h))

    def apply_pressure_operator_for_trials(self, p) -> np.ndarray:
        a = _f32(p)
        out = np.empty(self.cells, self.dtype)
        self._check(self.L.od3_apply_pressure_operator_for_trials(self.h, _fptr(a), out.ctypes.data, a.size),
                    "apply_pressure_operator_for_trials")
        return out

    def assemble_pressure_problem_for_trials(self, divergence, scale):
        a = _f32(divergence)
        rhs, prec = np.empty(self.cells, self.dtype), np.empty(self.cells, self.dtype)
        self._check(self.L.od3_assemble_pressure_problem_for_trials(self.h, _fptr(a), np.float32(scale),
                                                                    rhs.ctypes.data, prec.ctypes.data, a.size),
                    "assemble_pressure_problem_for_trials")
        return rhs, prec

    def vcycle_for_tests(self, x) -> np.ndarray:
        a = _f32(x)
        z = np.empty(self.cells, self.dtype)
        self._check(self.L.od3_vcycle_for_tests(self.h, _fptr(a), z.ctypes.data, a.size), "vcycle")
        return z
