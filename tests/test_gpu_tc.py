"""BF16X3 precision: the 7^3 filtering on the tcgen05 tensor cores with
split-BF16 operands (x = x_hi + x_lo, three products per tap) and FP32
accumulation in tensor memory.

Bars:
  filter responses  max |gpu - oracle_f64| <= 2e-5 * max |oracle_f64|
                    (a split product carries ~2^-16 relative error)
  registrations     RMS displacement vs the FP64 oracle <= 0.05 voxel (the
                    mixed-precision target), and within 0.01 voxel of the
                    FP32 path on the same inputs
  nonlinear fields  max |field_bf16x3 - field_fp32| <= 0.02 voxel
"""
import numpy as np
import pytest
import torch

from conftest import rel_err
from broccoli_b200 import _lib as L
from broccoli_b200 import synthetic as S

pytestmark = pytest.mark.gpu
FTOL = 2e-5


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("shape", [(5, 17, 33), (11, 9, 7), (9, 40, 65), (33, 64, 64), (4, 3, 2),
                                   (13, 230, 21), (40, 12, 31)])
@pytest.mark.parametrize("nf", [3, 6])
def test_tc_filter_vs_fp64_oracle(ctx, orc, bank, shape, nf):
    rng = np.random.default_rng(sum(shape) + 7 * nf)
    vol = (rng.standard_normal(shape) * 50 + 100).astype(np.float32)
    flt = bank["linear"] if nf == 3 else bank["nonlinear"]
    ref = orc.filter3d(vol, flt, prec="f64")
    got = ctx.filter3d(cuda(vol), flt, precision=L.PREC_BF16X3).cpu().numpy()[0]
    ctx.synchronize()
    assert got.shape == ref.shape
    assert rel_err(got, ref) < FTOL


@pytest.mark.parametrize("nf", [3, 6])
def test_tc_filter_non_symmetric_bank(ctx, orc, nf):
    rng = np.random.default_rng(60 + nf)
    flt = rng.standard_normal((nf, 2, 7, 7, 7)).astype(np.float32)
    vol = rng.standard_normal((14, 22, 37)).astype(np.float32)
    ref = orc.filter3d(vol, flt, prec="f64")
    got = ctx.filter3d(cuda(vol), flt, precision=L.PREC_BF16X3).cpu().numpy()[0]
    assert rel_err(got, ref) < FTOL


def test_tc_filter_batch_matches_single(ctx, lin_filters):
    rng = np.random.default_rng(8)
    vols = rng.standard_normal((5, 15, 22, 30)).astype(np.float32)
    qb = ctx.filter3d(cuda(vols), lin_filters, precision=L.PREC_BF16X3).cpu().numpy()
    for b in range(5):
        qs = ctx.filter3d(cuda(vols[b]), lin_filters, precision=L.PREC_BF16X3).cpu().numpy()[0]
        assert np.array_equal(qb[b], qs)


def test_tc_affine_registration_vs_fp64_oracle(ctx, orc, lin_filters):
    base, moved, truth = S.affine_pair((33, 64, 64))
    r = ctx.register_linear(cuda(base), cuda(moved)[None], lin_filters, 20, L.AFFINE,
                            precision=L.PREC_BF16X3)
    r32 = ctx.register_linear(cuda(base), cuda(moved)[None], lin_filters, 20, L.AFFINE)
    ctx.synchronize()
    p = r["params"].cpu().numpy()[0].astype(np.float64)
    p32 = r32["params"].cpu().numpy()[0].astype(np.float64)
    p64, _, _ = orc.align_linear(base, moved, lin_filters, 20, L.AFFINE, prec="f64")
    assert S.rms_displacement_error(p, p64, base.shape) <= 0.05
    assert S.rms_displacement_error(p, p32, base.shape) <= 0.01


def test_tc_batched_motion_correction_close_to_fp32(ctx, lin_filters):
    series, _ = S.motion_series(T=24)
    ref = cuda(series[0])
    mov = cuda(series[1:])
    r = ctx.register_linear(ref, mov, lin_filters, 20, L.RIGID, tolerance=1e-3, precision=L.PREC_BF16X3)
    r32 = ctx.register_linear(ref, mov, lin_filters, 20, L.RIGID, tolerance=1e-3)
    ctx.synchronize()
    p = r["params"].cpu().numpy().astype(np.float64)
    p32 = r32["params"].cpu().numpy().astype(np.float64)
    err = max(S.rms_displacement_error(p[i], p32[i], series.shape[1:]) for i in range(len(p)))
    assert err <= 0.01


def test_tc_nonlinear_close_to_fp32(ctx, bank):
    sub, tpl, _ = S.t1_template_pair((40, 48, 44), (40, 48, 44), seed=5)
    f, a = ctx.register_nonlinear(cuda(tpl), cuda(sub), bank, 4, coarsest_scale=2,
                                  precision=L.PREC_BF16X3)
    f32, a32 = ctx.register_nonlinear(cuda(tpl), cuda(sub), bank, 4, coarsest_scale=2)
    ctx.synchronize()
    d = np.abs(f.cpu().numpy() - f32.cpu().numpy()).max()
    assert d <= 0.02


def test_bounded_wait_reports_timeout_and_context_survives(ctx, orc, lin_filters):
    """A device-side wait that runs out (a barrier nothing completes) sets
    the context's flag; synchronize() reports BRC_ERR_TIMEOUT once, then the
    context keeps working."""
    ctx.synchronize()
    ctx.selftest_bounded_wait(50)
    with pytest.raises(L.BrcError) as e:
        ctx.synchronize()
    assert e.value.status == L.BRC_ERR_TIMEOUT
    ctx.synchronize()  # flag cleared
    vol = np.random.default_rng(3).standard_normal((9, 12, 15)).astype(np.float32)
    got = ctx.filter3d(cuda(vol), lin_filters, precision=L.PREC_BF16X3).cpu().numpy()[0]
    ctx.synchronize()
    assert rel_err(got, orc.filter3d(vol, lin_filters, prec="f64")) < FTOL


# ---- TF32 (BRC_PREC_TF32): one tf32 product per tap ----------------------
# Bars: responses max |gpu - oracle_f64| <= 2e-3 max |oracle_f64| (data and
# taps rounded to a 10-bit mantissa: ~2^-11 relative each); registrations
# within 0.05 voxel RMS of the FP64 oracle and 0.01 of the FP32 path.
TF32_TOL = 2e-3


@pytest.mark.parametrize("shape", [(5, 17, 33), (11, 9, 7), (33, 64, 64), (4, 3, 2), (13, 230, 21), (40, 12, 31)])
@pytest.mark.parametrize("nf", [3, 6])
def test_tf32_filter_vs_fp64_oracle(ctx, orc, bank, shape, nf):
    rng = np.random.default_rng(sum(shape) + 11 * nf)
    vol = (rng.standard_normal(shape) * 50 + 100).astype(np.float32)
    flt = bank["linear"] if nf == 3 else bank["nonlinear"]
    ref = orc.filter3d(vol, flt, prec="f64")
    got = ctx.filter3d(cuda(vol), flt, precision=L.PREC_TF32).cpu().numpy()[0]
    ctx.synchronize()
    assert got.shape == ref.shape
    assert rel_err(got, ref) < TF32_TOL
    # and it is not the BF16X3 result (the precision switch is honoured)
    b3 = ctx.filter3d(cuda(vol), flt, precision=L.PREC_BF16X3).cpu().numpy()[0]
    assert rel_err(b3, ref) < rel_err(got, ref)


def test_tf32_non_symmetric_bank_and_batch(ctx, orc, lin_filters):
    rng = np.random.default_rng(61)
    flt = rng.standard_normal((3, 2, 7, 7, 7)).astype(np.float32)
    vols = rng.standard_normal((4, 14, 22, 37)).astype(np.float32)
    qb = ctx.filter3d(cuda(vols), flt, precision=L.PREC_TF32).cpu().numpy()
    for b in range(4):
        assert rel_err(qb[b], orc.filter3d(vols[b], flt, prec="f64")) < TF32_TOL
        qs = ctx.filter3d(cuda(vols[b]), flt, precision=L.PREC_TF32).cpu().numpy()[0]
        assert np.array_equal(qb[b], qs)


def test_tf32_affine_registration_vs_fp64_oracle(ctx, orc, lin_filters):
    base, moved, truth = S.affine_pair((33, 64, 64))
    r = ctx.register_linear(cuda(base), cuda(moved)[None], lin_filters, 20, L.AFFINE, precision=L.PREC_TF32)
    r32 = ctx.register_linear(cuda(base), cuda(moved)[None], lin_filters, 20, L.AFFINE)
    ctx.synchronize()
    p = r["params"].cpu().numpy()[0].astype(np.float64)
    p32 = r32["params"].cpu().numpy()[0].astype(np.float64)
    p64, _, _ = orc.align_linear(base, moved, lin_filters, 20, L.AFFINE, prec="f64")
    assert S.rms_displacement_error(p, p64, base.shape) <= 0.05
    assert S.rms_displacement_error(p, p32, base.shape) <= 0.01


def test_tf32_batched_motion_correction_close_to_fp32(ctx, lin_filters):
    series, _ = S.motion_series(T=24)
    ref = cuda(series[0])
    mov = cuda(series[1:])
    r = ctx.register_linear(ref, mov, lin_filters, 20, L.RIGID, tolerance=1e-3, precision=L.PREC_TF32)
    r32 = ctx.register_linear(ref, mov, lin_filters, 20, L.RIGID, tolerance=1e-3)
    ctx.synchronize()
    p = r["params"].cpu().numpy().astype(np.float64)
    p32 = r32["params"].cpu().numpy().astype(np.float64)
    err = max(S.rms_displacement_error(p[i], p32[i], series.shape[1:]) for i in range(len(p)))
    assert err <= 0.01


def test_tf32_nonlinear_close_to_fp32(ctx, bank):
    sub, tpl, _ = S.t1_template_pair((40, 48, 44), (40, 48, 44), seed=5)
    f, a = ctx.register_nonlinear(cuda(tpl), cuda(sub), bank, 4, coarsest_scale=2, precision=L.PREC_TF32)
    f32, a32 = ctx.register_nonlinear(cuda(tpl), cuda(sub), bank, 4, coarsest_scale=2)
    ctx.synchronize()
    d = np.abs(f.cpu().numpy() - f32.cpu().numpy()).max()
    assert d <= 0.02
