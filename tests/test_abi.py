"""The C-ABI library loads and exports every entry point include/fluidisim_delta3d.h declares
(no GPU needed: nothing is called)."""
import ctypes
import os
import re

from fluidisim_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fluidisim_delta3d.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fd3_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_volume3_api():
    names = declared_symbols()
    for want in ["fd3_configure", "fd3_configure_with_bottom", "fd3_configure_with_solid", "fd3_enable_multigrid",
                 "fd3_set_free_surface", "fd3_set_velocity", "fd3_project_mobile", "fd3_step_surface_mobile",
                 "fd3_project_linear", "fd3_step_surface_linear",
                 "fd3_get_pressure", "fd3_get_velocity", "fd3_apply_pressure_operator_for_trials",
                 "fd3_assemble_pressure_problem_for_trials", "fd3_destroy"]:
        assert want in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(B.build())
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_names_without_a_device():
    lib = ctypes.CDLL(B.build())
    buf = ctypes.create_string_buffer(32)
    lib.fd3_status_name(6, buf, 32)
    assert buf.value == b"Convergence"
    lib.fd3_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.fd3_version()
