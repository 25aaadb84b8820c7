"""The class members beyond the registration results (DEBUG outputs, skull
strip, pre-centring, the parameter inverse) on the CPU: the oracle's
restatement composed as the reference composes them equals the reference's
own kernels (tests/golden/boundary.npz, tests/golden/make_golden_boundary.py),
and the library's host-side inverse equals the reference's Eigen inverse.
The same fixtures pin the GPU path in test_gpu_boundary.py."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN
from broccoli_b200 import _lib as L


@pytest.fixture(scope="module")
def boundary():
    return dict(np.load(os.path.join(GOLDEN, "boundary.npz")))


def test_debug_outputs_restatement_exact(orc, golden, boundary, lin_filters):
    series = golden["mc_series"]
    qref = orc.filter3d(series[0], lin_filters).astype(np.complex64)
    qlast = orc.filter3d(series[-1], lin_filters).astype(np.complex64)
    for k in range(3):
        assert np.array_equal(qref[k], boundary[f"mc_dbg_q{k + 1}"])
    pd, pc, pg = orc.phase_volumes(qref[2], qlast[2], 2)
    assert np.array_equal(pd, boundary["mc_dbg_pd"])
    assert np.array_equal(pc, boundary["mc_dbg_pc"])
    assert np.array_equal(pg, boundary["mc_dbg_pg"])
    # the gradient's first and last z planes are the zero fill
    assert not pg[0].any() and not pg[-1].any()


def test_library_inverse_matches_reference_eigen(golden, boundary):
    p = np.ascontiguousarray(golden["r2v_params"], np.float32)
    inv = np.zeros(12, np.float32)
    L.lib().brc_invert_affine_parameters(p.ctypes.data_as(ctypes.c_void_p), inv.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_allclose(inv, boundary["r2v_inverse"], rtol=1e-6, atol=1e-7)
    # and it is an inverse: composing both gives the identity transform
    back = np.zeros(12, np.float32)
    L.lib().brc_invert_affine_parameters(inv.ctypes.data_as(ctypes.c_void_p), back.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_allclose(back, p, rtol=1e-5, atol=1e-6)


def test_skull_strip_restatement_exact(orc, golden, boundary):
    assert np.array_equal(golden["r2v_aligned_nonlinear"] * boundary["r2v_mask"], boundary["r2v_skull"])
    back = orc.transform_affine(boundary["r2v_mask"], boundary["r2v_inverse"], interp=0)[0]
    assert np.array_equal(golden["r2v_interpolated"] * back, boundary["r2v_skull_original"])


def test_precenter_restatement_exact(orc, golden, boundary, bank):
    c1, _ = orc.center_volumes(golden["r2v_subject"], 1)
    c2, _ = orc.center_volumes(c1[0], 1)
    r = orc.register_two_volumes(c2[0], golden["r2v_voxel"], golden["r2v_template"], (1.0, 1.0, 1.0), bank, 6, 4,
                                 2, mm_z_cut=3)
    for k in ("params", "interpolated", "aligned_linear", "aligned_nonlinear", "field"):
        assert np.array_equal(r[k], boundary["pc_" + k]), k
    # pre-centring changes the result
    assert not np.array_equal(boundary["pc_params"], golden["r2v_params"])
