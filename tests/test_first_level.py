"""The first-level preprocessing chain on the CPU: the oracle's composition
(oracle.first_level_preprocess, the stages of PerformFirstLevelAnalysisWrapper,
broccoli_lib.cpp:8480-8733) and its two new steps -- CalculateTensorMagnitude
(:5658-5746) and SegmentEPIData (:11008-11030) -- against the golden fixture
that tests/golden/make_golden.py records from the reference's own kernels,
and the host-only FWHM filters of the library against the oracle's."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from broccoli_b200 import _lib as L
from broccoli_b200.api import Context


@pytest.fixture(scope="module")
def fl():
    return dict(np.load(os.path.join(GOLDEN, "first_level.npz")))


def cfg(fl):
    """The chain's settings stored with the fixture (cfg_* entries)."""
    return {k[4:]: (tuple(float(x) for x in v) if v.ndim else v.item()) for k, v in fl.items()
            if k.startswith("cfg_")}


def _run(orc, fl, bank, prec):
    c = cfg(fl)
    return orc.first_level_preprocess(fl["in_fmri"], c["epi_voxel"], fl["in_t1"], c["t1_voxel"], fl["in_mni"],
                                      c["mni_voxel"], bank, c["lin_iter"], c["nl_iter"], c["coarsest_t1_mni"],
                                      c["coarsest_epi_t1"], c["mm_t1_z_cut"], c["motion_iter"],
                                      c["smoothing_fwhm"], prec=prec)


def test_oracle_chain_equals_reference_kernels(orc, fl, bank):
    """The FP32 restatement reproduces every output of the chain on the
    reference's kernels bit for bit."""
    out = _run(orc, fl, bank, "f32")
    keys = [k[4:] for k in fl if k.startswith("out_")]
    assert set(keys) == set(out)
    for k in keys:
        assert np.array_equal(np.asarray(out[k], np.float32), fl["out_" + k], equal_nan=True), k


def test_oracle_steps_equal_reference_kernels(orc, fl, bank):
    c = cfg(fl)
    assert np.array_equal(orc.tensor_magnitude(fl["in_t1"], bank), fl["tensor_magnitude_t1"])
    mask = orc.segment_epi(fl["in_fmri"][0], c["epi_voxel"])
    assert np.array_equal(mask, fl["segment_epi0"])
    assert set(np.unique(mask)) == {np.float32(1.0), np.float32(0.001)}


def test_oracle_fp64_chain_close(orc, fl, bank):
    """The FP64 oracle agrees with the FP32 chain to float accuracy (no
    discrete decision -- mass-match rounding, mask threshold -- flips)."""
    out = _run(orc, fl, bank, "f64")
    for k, v in out.items():
        ref = fl["out_" + k].astype(np.float64)
        err = np.abs(np.asarray(v) - ref).max() / max(1.0, np.abs(ref).max())
        assert err < 1e-4, (k, err)


def test_fwhm_filters_equal_oracle(orc):
    for fwhm, vs in ((4.0, (3.0, 3.0, 3.5)), (6.0, (2.0, 2.5, 3.0)), (8.0, (1.0, 1.0, 1.0))):
        got = Context.smoothing_filters_fwhm(fwhm, vs)
        want = orc.smoothing_filter_fwhm(fwhm, vs)
        for g, w in zip(got, want):
            assert np.array_equal(g, w)


def test_first_level_opts_default():
    import ctypes
    o = L.FirstLevelOpts()
    L.lib().brc_first_level_opts_default(ctypes.byref(o))
    assert (o.linear_iterations, o.nonlinear_iterations, o.motion_iterations) == (10, 10, 5)
    assert (o.coarsest_scale_t1_mni, o.coarsest_scale_epi_t1, o.mm_t1_z_cut) == (4, 4, 0)
    assert (o.apply_motion_correction, o.apply_smoothing, o.smoothing_fwhm) == (1, 1, 6.0)
    assert o.precision == L.PREC_FP32


def test_null_context_is_rejected():
    import ctypes
    assert L.lib().brc_first_level_preprocess(None, None, None, None) == L.BRC_ERR_INVALID
    assert L.lib().brc_segment_epi(None, None, 1, 1, 1, None, None) == L.BRC_ERR_INVALID
    assert L.lib().brc_tensor_magnitude(None, None, 1, 1, 1, None, None, 0, None) == L.BRC_ERR_INVALID
    del ctypes
