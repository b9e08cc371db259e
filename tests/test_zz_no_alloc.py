"""fd3_assemble_pressure_problem_noalloc: the pressure-problem assembly for callers that cannot
allocate device memory when they call (a host whose arena is sealed after set-up, or a real-time
loop where cudaMalloc would stall a frame).  Its scratch is a static device array inside the
library, so it must give what the allocating path gives, call after call, although every call
reuses the same scratch.

This file is collected last on purpose: if it fails, a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(lib):
    f = lib.fd3_assemble_pressure_problem_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


def test_noalloc_assembly_matches_the_allocating_path_on_two_calls():
    import torch

    from fluidisim_b200 import scenes
    from fluidisim_b200.delta3d import Volume3, library

    s = scenes.sphere_lake(32, seed=1, spheres=4)
    v = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    v.set_free_surface(s["eta"], s["rest"])
    scale, _ = scenes.projection_scalars(s)
    entry = _entry(library())

    for call, seed in enumerate((9, 10)):
        div = scenes.noise(v.cells, seed) * np.float32(3.0)
        rhs_ref, prec_ref = v.assemble_pressure_problem_for_trials(div, scale)  # the existing entry point
        d_div = torch.from_numpy(div).cuda()
        d_rhs = torch.full((v.cells,), float("nan"), dtype=torch.float32, device="cuda")
        d_prec = torch.full((v.cells,), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        norm2 = C.c_double(-1.0)
        e = entry(v._h, d_div.data_ptr(), np.float32(scale), d_rhs.data_ptr(), d_prec.data_ptr(), v.cells,
                  C.byref(norm2))
        assert e == 0, f"call {call}: status {e}"
        torch.cuda.synchronize()
        rhs, prec = d_rhs.cpu().numpy(), d_prec.cpu().numpy()
        # the same f32 arithmetic: the tolerance of the assembly parity tests is bit equality
        assert np.array_equal(rhs.view(np.uint32), rhs_ref.view(np.uint32)), f"call {call}: rhs differs"
        assert np.array_equal(prec.view(np.uint32), prec_ref.view(np.uint32)), f"call {call}: prec differs"
        want = float(np.sum(rhs_ref.astype(np.float64) ** 2))
        assert want > 0 and abs(norm2.value - want) <= 1e-12 * want, (call, norm2.value, want)

    # a wrong length is refused before anything runs
    norm2 = C.c_double(0.0)
    assert entry(v._h, d_div.data_ptr(), np.float32(scale), d_rhs.data_ptr(), d_prec.data_ptr(), v.cells - 1,
                 C.byref(norm2)) == 1
    v.close()


def test_noalloc_assembly_reports_a_nan_and_the_next_call_is_clean():
    """One NaN in the divergence gives NotFinite (2); the finiteness flag lives in the shared scratch,
    so the clean call after it must return Ok with the allocating path's bits."""
    import torch

    from fluidisim_b200 import scenes
    from fluidisim_b200.delta3d import Volume3, library

    s = scenes.sphere_lake(32, seed=2, spheres=4)
    v = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    v.set_free_surface(s["eta"], s["rest"])
    scale, _ = scenes.projection_scalars(s)
    entry = _entry(library())
    div = scenes.noise(v.cells, 21) * np.float32(2.0)
    bad = div.copy()
    bad[v.cells // 3] = np.nan
    d_rhs = torch.empty(v.cells, dtype=torch.float32, device="cuda")
    d_prec = torch.empty(v.cells, dtype=torch.float32, device="cuda")
    norm2 = C.c_double(0.0)
    d_bad = torch.from_numpy(bad).cuda()
    torch.cuda.synchronize()
    assert entry(v._h, d_bad.data_ptr(), np.float32(scale), d_rhs.data_ptr(), d_prec.data_ptr(), v.cells,
                 C.byref(norm2)) == 2
    rhs_ref, prec_ref = v.assemble_pressure_problem_for_trials(div, scale)
    d_div = torch.from_numpy(div).cuda()
    torch.cuda.synchronize()
    assert entry(v._h, d_div.data_ptr(), np.float32(scale), d_rhs.data_ptr(), d_prec.data_ptr(), v.cells,
                 C.byref(norm2)) == 0
    torch.cuda.synchronize()
    assert np.array_equal(d_rhs.cpu().numpy().view(np.uint32), rhs_ref.view(np.uint32))
    assert np.array_equal(d_prec.cpu().numpy().view(np.uint32), prec_ref.view(np.uint32))
    want = float(np.sum(rhs_ref.astype(np.float64) ** 2))
    assert abs(norm2.value - want) <= 1e-12 * want
    v.close()
