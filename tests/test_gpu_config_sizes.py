"""Whole-path parity at the workload sizes, not only on the small golden
cases: every result compared with the CPU oracle run on the same seeded
inputs, and every mixed-precision result scored against the FP64 oracle.

Cases
  * one plain FP32 AFFINE registration of a 64x64x33 volume (3 mm EPI-like
    base volume and a copy under a seeded affine), 20 iterations, no early
    exit, with the reference's shipped filters and with the lognormal
    u0 = pi/3, 2-octave bank;
  * a batch of 8 volumes of the 64x64x33 rigid motion-correction series
    (Rician noise, SNR 50), FP32, with and without the 3x3x3 certainty
    smoothing, against the oracle one volume at a time;
  * one T1-to-template normalisation at half the workload's resolution
    (subject 128x128x85, template 91x109x91, both 2 mm; affine then
    nonlinear over the scales 8, 4, 2, 1; 10 + 10 iterations; the six
    shipped nonlinear filters).

Bars
  FP32 parity (the reference's 1e-4 relative):
    parameters  max |p - p_oracle| <= 1e-4 * max(1, max |p_oracle|)
    volumes and displacement fields  max |v - v_oracle| <= 1e-4 * max |v_oracle|
  mixed precision (BF16X3 or TF32 filtering, FP64 solves) against the FP64 oracle:
    RMS displacement error <= 0.05 voxel (affine: over all voxels of the
    grid; nonlinear: RMS over voxels of the length of the difference of the
    combined affine + nonlinear displacement fields)
"""
import numpy as np
import pytest
import torch

from conftest import rel_err
from broccoli_b200 import _lib as L
from broccoli_b200 import filters as F
from broccoli_b200 import synthetic as S

pytestmark = pytest.mark.gpu
TOL = 1e-4
RMS_BAR = 0.05


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def param_err(p, ref):
    p = np.asarray(p, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(p - ref).max() / max(1.0, np.abs(ref).max()))


def field_rms(f, ref):
    d = np.asarray(f, np.float64) - np.asarray(ref, np.float64)
    return float(np.sqrt((d * d).sum(0).mean()))


@pytest.fixture(scope="module")
def affine_case():
    return S.affine_pair((33, 64, 64))


@pytest.mark.parametrize("which", ["shipped", "lognormal"])
def test_affine_64x64x33_fp32_matches_oracle(ctx, orc, bank, affine_case, which):
    base, moved, truth = affine_case
    flt = bank["linear"] if which == "shipped" else F.linear_registration_filters()
    r = ctx.register_linear(cuda(base), cuda(moved)[None], flt, 20, L.AFFINE)
    p = r["params"].cpu().numpy()[0]
    assert int(r["iterations"].cpu()[0]) == 20
    p32, al32, _ = orc.align_linear(base, moved, flt, 20, orc.AFFINE)
    assert param_err(p, p32) < TOL
    assert rel_err(r["aligned"].cpu().numpy()[0], al32) < TOL
    p64, _, _ = orc.align_linear(base, moved, flt, 20, orc.AFFINE, prec="f64")
    assert S.rms_displacement_error(p, p64, base.shape) < RMS_BAR
    # the registration recovers the applied affine
    err0 = S.rms_displacement_error(np.zeros(12), truth, base.shape)
    assert S.rms_displacement_error(p, truth, base.shape) < 0.2 * err0


@pytest.mark.parametrize("prec", [L.PREC_BF16X3, L.PREC_TF32], ids=["bf16x3", "tf32"])
@pytest.mark.parametrize("which", ["shipped", "lognormal"])
def test_affine_64x64x33_mixed_vs_fp64_oracle(ctx, orc, bank, affine_case, which, prec):
    base, moved, _ = affine_case
    flt = bank["linear"] if which == "shipped" else F.linear_registration_filters()
    r = ctx.register_linear(cuda(base), cuda(moved)[None], flt, 20, L.AFFINE, precision=prec)
    p = r["params"].cpu().numpy()[0]
    p64, _, _ = orc.align_linear(base, moved, flt, 20, orc.AFFINE, prec="f64")
    assert S.rms_displacement_error(p, p64, base.shape) < RMS_BAR
    p32 = ctx.register_linear(cuda(base), cuda(moved)[None], flt, 20, L.AFFINE)["params"].cpu().numpy()[0]
    assert S.rms_displacement_error(p, p32, base.shape) < 0.01


@pytest.fixture(scope="module")
def series8():
    vols, _ = S.motion_series(T=9, shape=(33, 64, 64), snr=50.0)
    return vols


@pytest.mark.parametrize("cert_sigma", [0.0, 1.0])
def test_motion_batch_64x64x33_fp32_matches_oracle(ctx, orc, series8, cert_sigma):
    flt = F.linear_registration_filters()
    vols = series8
    r = ctx.register_linear(cuda(vols[0]), cuda(vols[1:]), flt, 20, L.RIGID, certainty_sigma=cert_sigma)
    got = r["params"].cpu().numpy()
    al = r["aligned"].cpu().numpy()
    for i in range(vols.shape[0] - 1):
        p32, a32, _ = orc.align_linear(vols[0], vols[i + 1], flt, 20, orc.RIGID, cert_sigma=cert_sigma)
        assert param_err(got[i], p32) < TOL, i
        assert rel_err(al[i], a32) < TOL, i


@pytest.mark.parametrize("prec", [L.PREC_BF16X3, L.PREC_TF32], ids=["bf16x3", "tf32"])
def test_motion_batch_64x64x33_workload_vs_fp64_oracle(ctx, orc, series8, prec):
    """The timed workload's form (tensor-core filtering, certainty smoothing
    sigma 1, early exit at 1e-3 voxel) against the FP64 oracle running all
    20 iterations."""
    flt = F.linear_registration_filters()
    vols = series8
    r = ctx.register_linear(cuda(vols[0]), cuda(vols[1:]), flt, 20, L.RIGID, tolerance=1e-3,
                            precision=prec, certainty_sigma=1.0)
    got = r["params"].cpu().numpy()
    for i in range(vols.shape[0] - 1):
        p64, _, _ = orc.align_linear(vols[0], vols[i + 1], flt, 20, orc.RIGID, prec="f64", cert_sigma=1.0)
        assert S.rms_displacement_error(got[i], p64, vols.shape[1:]) < RMS_BAR, i


@pytest.fixture(scope="module")
def t1_half():
    tpl = S.head_phantom((91, 109, 91), seed=2)
    sub = S.warp_with_field(S.head_phantom((85, 128, 128), seed=1),
                            S.smooth_field((85, 128, 128), seed=200, max_mm=3.0, sigma=4.0))
    return np.ascontiguousarray(sub, np.float32), tpl


@pytest.fixture(scope="module")
def t1_half_oracle(orc, bank, t1_half):
    sub, tpl = t1_half
    two = (2.0, 2.0, 2.0)
    return {prec: orc.register_two_volumes(sub, two, tpl, two, bank, 10, 10, 8, prec=prec)
            for prec in ("f32", "f64")}


def test_t1_to_template_half_size_fp32_matches_oracle(ctx, bank, t1_half, t1_half_oracle):
    sub, tpl = t1_half
    two = (2.0, 2.0, 2.0)
    o = t1_half_oracle["f32"]
    r = ctx.register_two_volumes(cuda(sub), two, cuda(tpl), two, bank, 10, 10, 8)
    assert param_err(r["params"], o["params"]) < TOL
    for k in ("interpolated", "aligned_linear", "aligned_nonlinear", "field"):
        assert rel_err(r[k].cpu().numpy(), o[k]) < TOL, k


@pytest.mark.parametrize("prec", [L.PREC_BF16X3, L.PREC_TF32], ids=["bf16x3", "tf32"])
def test_t1_to_template_half_size_mixed_vs_fp64_oracle(ctx, bank, t1_half, t1_half_oracle, prec):
    sub, tpl = t1_half
    two = (2.0, 2.0, 2.0)
    o = t1_half_oracle["f64"]
    r = ctx.register_two_volumes(cuda(sub), two, cuda(tpl), two, bank, 10, 10, 8, precision=prec,
                                 solve_fp64=True)
    f = r["field"].cpu().numpy()
    assert field_rms(f, o["field"]) < RMS_BAR
    assert S.rms_displacement_error(r["params"], o["params"], tpl.shape) < RMS_BAR
    # the FP32 path is as close to the FP64 oracle
    r32 = ctx.register_two_volumes(cuda(sub), two, cuda(tpl), two, bank, 10, 10, 8)
    assert field_rms(r32["field"].cpu().numpy(), o["field"]) < RMS_BAR
