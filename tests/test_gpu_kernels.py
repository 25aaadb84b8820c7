"""Kernel-level parity of the CUDA path (through the C-ABI) with the oracle
and with the golden fixtures made by the reference's own kernels.

Tolerance (FP32 parity, the reference's 1e-4 relative): for every volume
output, max |gpu - ref| <= 1e-4 * max |ref| (norm-wise relative error)."""
import numpy as np
import pytest
import torch

from conftest import rel_err
from broccoli_b200 import _lib as L
from broccoli_b200 import filters as F

pytestmark = pytest.mark.gpu
TOL = 1e-4


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_filter_matches_golden(ctx, golden, lin_filters):
    q = ctx.filter3d(cuda(np.stack([golden["base"], golden["moved"]])), lin_filters).cpu().numpy()
    assert rel_err(q[0], golden["q1"]) < TOL
    assert rel_err(q[1], golden["q2"]) < TOL


@pytest.mark.parametrize("shape", [(5, 17, 33), (11, 9, 7), (9, 40, 65), (33, 64, 64), (4, 3, 2)])
@pytest.mark.parametrize("nf", [3, 6])
@pytest.mark.parametrize("prec", [L.PREC_FP32, L.PREC_FP32_GENERAL])
def test_filter_odd_shapes_vs_oracle(ctx, orc, bank, shape, nf, prec):
    """FP32 (even/odd half-tap kernel for these quadrature banks) and
    FP32_GENERAL (all 343 taps) against the oracle."""
    rng = np.random.default_rng(sum(shape) + nf)
    vol = (rng.standard_normal(shape) * 50 + 100).astype(np.float32)
    flt = bank["linear"] if nf == 3 else bank["nonlinear"]
    ref = orc.filter3d(vol, flt)
    got = ctx.filter3d(cuda(vol), flt, precision=prec).cpu().numpy()[0]
    assert got.shape == ref.shape
    assert rel_err(got, ref) < TOL


@pytest.mark.parametrize("nf", [3, 6])
def test_filter_non_symmetric_bank(ctx, orc, nf):
    """A bank without even/odd symmetry takes the general kernel."""
    rng = np.random.default_rng(40 + nf)
    flt = rng.standard_normal((nf, 2, 7, 7, 7)).astype(np.float32)
    vol = rng.standard_normal((12, 20, 36)).astype(np.float32)
    ref = orc.filter3d(vol, flt)
    got = ctx.filter3d(cuda(vol), flt).cpu().numpy()[0]
    assert rel_err(got, ref) < TOL


def test_filter_batch_matches_single(ctx, lin_filters):
    rng = np.random.default_rng(5)
    vols = rng.standard_normal((4, 9, 12, 20)).astype(np.float32)
    qb = ctx.filter3d(cuda(vols), lin_filters).cpu().numpy()
    for b in range(4):
        qs = ctx.filter3d(cuda(vols[b]), lin_filters).cpu().numpy()[0]
        assert np.array_equal(qb[b], qs)


def test_lognormal_filters_are_quadrature(ctx):
    flt = F.linear_registration_filters()
    # a plane wave along x: filter 0 responds with a constant-magnitude
    # analytic signal, the other two barely respond.
    x = np.arange(40)
    vol = np.broadcast_to(np.cos(np.pi / 3 * x), (20, 24, 40)).astype(np.float32)
    q = ctx.filter3d(cuda(vol), flt).cpu().numpy()[0]
    inner = q[:, 8:-8, 8:-8, 8:-8]
    mag = np.abs(inner[0])
    assert mag.std() / mag.mean() < 0.05
    assert np.abs(inner[1]).mean() < 0.05 * mag.mean()


def test_normal_equations_match_golden(ctx, golden):
    q1 = torch.from_numpy(golden["q1"]).cuda()
    q2 = torch.from_numpy(golden["q2"]).cuda()
    A, h = ctx.normal_equations(q1, q2[None])
    A = A.cpu().numpy()[0]
    h = h.cpu().numpy()[0]
    assert rel_err(A, golden["A"]) < TOL
    assert rel_err(h, golden["h"]) < TOL
    # zero structure identical
    assert np.array_equal(A != 0, golden["A"] != 0)


def test_solve_matches_golden(ctx, golden):
    A = torch.from_numpy(golden["A"].astype(np.float64)).cuda()
    h = torch.from_numpy(golden["h"].astype(np.float64)).cuda()
    p = ctx.solve(A, h).cpu().numpy()[0]
    np.testing.assert_allclose(p, golden["p_solve"], rtol=1e-6, atol=1e-7)


def test_solve_zero_system(ctx):
    A = torch.zeros((2, 12, 12), dtype=torch.float64, device="cuda")
    h = torch.zeros((2, 12), dtype=torch.float64, device="cuda")
    p = ctx.solve(A, h).cpu().numpy()
    assert np.all(p == 0)


def test_warp_affine_matches_golden(ctx, golden):
    out = ctx.warp_affine(cuda(golden["moved"]), torch.from_numpy(golden["p_solve"]).cuda())
    assert rel_err(out.cpu().numpy()[0], golden["warp_affine"]) < TOL


def test_warp_field_matches_golden(ctx, golden):
    out = ctx.warp_field(cuda(golden["moved"]), cuda(golden["field_x"]), cuda(golden["field_y"]),
                         cuda(golden["field_z"]))
    assert rel_err(out.cpu().numpy(), golden["warp_field"]) < TOL


def test_warp_identity_is_exact(ctx, golden):
    v = cuda(golden["moved"])
    out = ctx.warp_affine(v, torch.zeros(12, device="cuda"))
    assert torch.equal(out[0], v)


def test_smoothing_matches_golden(ctx, golden):
    fs = golden["smooth_filter"]
    out = ctx.smooth3d(cuda(golden["moved"]), fs, fs, fs).cpu().numpy()
    assert rel_err(out, golden["smooth"]) < TOL
    out = ctx.smooth3d(cuda(golden["moved"]), fs, fs, fs, cert=cuda(golden["cert"]),
                       smoothed_cert=cuda(golden["smooth_cert"])).cpu().numpy()
    assert rel_err(out, golden["smooth_normalized"]) < TOL


def test_smoothing_in_place_and_ragged_sizes(ctx, orc):
    """The fused smoothing (one kernel, z-marching) on sizes that are not
    multiples of its 32 x 8 x 32 tile, batched, against the oracle's three
    passes; and written over its own input (the output then goes through a
    temporary) with the same result."""
    import ctypes
    rng = np.random.default_rng(4)
    vols = rng.standard_normal((3, 37, 21, 45)).astype(np.float32)
    fx, fy, fz = (orc.smoothing_filter_sigma(s) for s in (1.0, 2.0, 3.0))
    got = ctx.smooth3d(cuda(vols), fx, fy, fz).cpu().numpy()
    for b in range(3):
        assert rel_err(got[b], orc.smooth3d(vols[b], fx, fy, fz)) < TOL
    v = cuda(vols)
    taps = [np.ascontiguousarray(f, np.float32) for f in (fx, fy, fz)]
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    assert L.lib().brc_smooth3d(ctx.handle, P(v), 45, 21, 37, 3, *[t.ctypes.data_as(ctypes.c_void_p) for t in taps],
                                None, None, P(v)) == 0
    torch.cuda.synchronize()
    assert torch.equal(v.cpu(), torch.from_numpy(got))


def test_rescale_matches_golden(ctx, golden):
    out = ctx.rescale_linear(cuda(golden["moved"]), (11, 13, 17)).cpu().numpy()
    assert rel_err(out, golden["rescale"]) < TOL


def test_smooth_normalized_matches_golden(ctx):
    """brc_smooth_normalized against the reference kernels' output: the same
    NaN voxels, the rest within 1e-4 of the largest value."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "smooth_normalized.npz"))
    fs = g["filter"]
    out = ctx.smooth_normalized(cuda(g["vols"]), cuda(g["mask"]), fs, fs, fs).cpu().numpy()
    ref = g["out"]
    assert np.array_equal(np.isnan(out), np.isnan(ref))
    fin = np.isfinite(ref)
    assert np.abs(out[fin] - ref[fin]).max() <= TOL * np.abs(ref[fin]).max()
