"""The C-ABI library loads, exports every symbol its header declares, and
rejects bad arguments -- without launching anything on a GPU."""
import ctypes

import pytest

from broccoli_b200 import _lib as L


def test_header_declares_entry_points():
    syms = L.header_symbols()
    for name in ("brc_ctx_create", "brc_filter3d", "brc_normal_equations", "brc_solve_affine_fp64",
                 "brc_warp_affine", "brc_smooth3d", "brc_register_linear_batched", "brc_motion_correct"):
        assert name in syms


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    missing = [s for s in L.header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_exports_the_nifti_header():
    import os
    path = os.path.join(os.path.dirname(L.HEADER_PATH), "broccoli_nifti.h")
    syms = L.header_symbols(path)
    assert {"brc_nifti_read", "brc_nifti_write", "brc_nifti_free", "brc_nifti_error"} <= set(syms)
    lib = L.lib()
    assert all(hasattr(lib, s) for s in syms)


def test_status_strings_and_version():
    assert L.status_string(L.BRC_OK) == "ok"
    assert "invalid" in L.status_string(L.BRC_ERR_INVALID)
    assert L.lib().brc_version().decode().startswith("broccoli_b200")


def test_null_context_is_rejected():
    lib = L.lib()
    assert lib.brc_ctx_destroy(None) == L.BRC_ERR_INVALID
    assert lib.brc_filter3d(None, None, 1, 1, 1, 1, 1, None, 3, 0, None) == L.BRC_ERR_INVALID
    assert lib.brc_ctx_create(0, None) == L.BRC_ERR_INVALID


def test_no_device_reports_nodevice():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert L.lib().brc_ctx_create(0, ctypes.byref(h)) == L.BRC_ERR_NODEVICE


def test_default_options():
    o = L.LinearOpts()
    L.lib().brc_linear_opts_default(ctypes.byref(o), 20)
    assert (o.iterations, o.type, o.precision, o.use_graph, o.certainty_sigma_x100) == (20, L.AFFINE, 0, 1, 0)
    assert o.tolerance == 0.0
