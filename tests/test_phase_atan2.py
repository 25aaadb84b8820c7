"""The arctangent of the phase kernels (phase_atan2 in csrc/common.cuh).

The reference's phase-difference and phase-gradient kernels call OpenCL's
atan2 (kernelRegistration.cpp:173-382); the CUDA kernels use a polynomial
fit with the hardware reciprocal instead.  Checked here:
  CPU: the fit script reproduces the coefficients the header holds, and
       their float32 evaluation is within 1.5e-7 relative of atan on [0, 1];
  GPU: against atan2 in float64 over six decades of magnitude and every
       quadrant, absolute error <= 5e-7 rad, relative error <= 5e-7 where the
       angle is reduced without a reflection (|y| < |x|, x > 0), and the
       axis and zero cases exactly.
"""
import os
import re

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def header_coefficients():
    src = open(os.path.join(ROOT, "broccoli_b200", "csrc", "common.cuh")).read()
    body = src[src.index("float phase_atan2("):]
    body = body[:body.index("return copysignf")]
    first = re.search(r"float p = ([-0-9.e+]+)f;", body).group(1)
    rest = re.findall(r"p = fmaf\(p, s, ([-0-9.e+]+)f\);", body)
    return np.array([float(v) for v in [first] + rest][::-1], np.float32)


def test_fit_reproduces_header_coefficients():
    from broccoli_b200 import fit_atan
    c = fit_atan.fit()
    np.testing.assert_array_equal(c, header_coefficients())
    t = np.concatenate([np.logspace(-8, 0, 50001), np.linspace(0, 1, 100001)[1:]]).astype(np.float32)
    ref = np.arctan(t.astype(np.float64))
    r = fit_atan.eval_f32(c, t).astype(np.float64)
    assert np.max(np.abs(r - ref) / ref) < 1.5e-7


@pytest.mark.gpu
def test_phase_atan2_error_bound(ctx):
    import torch
    rng = np.random.default_rng(7)
    n = 1 << 20
    mag = 10.0 ** rng.uniform(-3, 3, n)
    ang = rng.uniform(-np.pi, np.pi, n)
    y = (mag * np.sin(ang)).astype(np.float32)
    x = (mag * np.cos(ang)).astype(np.float32)
    # near-axis and near-diagonal arguments
    y[: n // 8] *= np.float32(1e-5)
    x[n // 8: n // 4] *= np.float32(1e-5)
    x[n // 4: n // 4 + 1000] = y[n // 4: n // 4 + 1000]
    got = ctx.phase_atan2(torch.from_numpy(y).cuda(), torch.from_numpy(x).cuda()).cpu().numpy().astype(np.float64)
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    err = np.abs(got - ref)
    assert err.max() <= 5e-7, err.max()
    direct = (np.abs(y) < np.abs(x)) & (x > 0) & (y != 0)
    assert np.max(err[direct] / np.abs(ref[direct])) <= 5e-7


@pytest.mark.gpu
def test_phase_atan2_axes_and_zero(ctx):
    import torch
    y = np.array([0.0, 0.0, -0.0, 0.0, 2.5, -2.5, 1.0, -1.0, 3.0, 1e-20], np.float32)
    x = np.array([0.0, 1.0, 1.0, -1.0, 0.0, 0.0, 1.0, -1.0, 3.0, 1e-20], np.float32)
    got = ctx.phase_atan2(torch.from_numpy(y).cuda(), torch.from_numpy(x).cuda()).cpu().numpy()
    want = np.array([0.0, 0.0, -0.0, np.pi, np.pi / 2, -np.pi / 2, np.pi / 4, -3 * np.pi / 4, np.pi / 4, np.pi / 4],
                    np.float32)
    np.testing.assert_allclose(got, want, rtol=0, atol=3e-7)
    assert np.signbit(got[2]) and not np.signbit(got[0])
    assert ctx.phase_atan2(torch.zeros(0).cuda(), torch.zeros(0).cuda()).numel() == 0
