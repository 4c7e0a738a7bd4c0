"""The C-ABI library loads here (no GPU) and exports every declared entry point."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "vortex_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(vt_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("vt_create", "vt_destroy", "vt_step_rk4", "vt_step_euler", "vt_rhs",
                 "vt_upload_state", "vt_download_state", "vt_read_input_file", "vt_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(vt):
    lib = vt.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_no_cuda_device_reports_error_not_crash(vt):
    """Without a GPU, context creation fails with a status instead of exiting."""
    import torch
    if torch.cuda.is_available():
        return
    pb = vt.Problem(vt.make_params(4, 4, p=1))
    try:
        vt.Solver(pb)
    except vt.VortexError as e:
        assert e.status in (vt.VT_ERR_CUDA, vt.VT_ERR_NO_MEMORY)
    else:
        raise AssertionError("expected a CUDA error without a device")


def test_oracle_library_is_separate(vt):
    """The product library does not link the oracle."""
    import subprocess
    out = subprocess.run(["nm", "-D", vt.LIB_PATH], capture_output=True, text=True).stdout
    assert "vto_" not in out
