"""Whole-path parity of batched registration and motion correction on the
GPU (through the C-ABI) with the golden fixtures of the reference's own
kernels and with the CPU oracle.

Tolerances (FP32 parity, the reference's 1e-4 relative):
  parameters: max_i |p_gpu - p_ref| <= 1e-4 * max(1, max_i |p_ref|)
              (norm-wise relative; translations are in voxels)
  volumes:    max |v_gpu - v_ref| <= 1e-4 * max |v_ref|
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


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def param_err(p, ref):
    p = np.asarray(p, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(p - ref).max() / max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("typ,name", [(0, "translation"), (1, "rigid"), (2, "affine")])
@pytest.mark.parametrize("graph", [True, False])
def test_align_matches_golden(ctx, golden, lin_filters, typ, name, graph):
    r = ctx.register_linear(cuda(golden["base"]), cuda(golden["moved"])[None], lin_filters, 10, typ,
                            use_graph=graph)
    p = r["params"].cpu().numpy()[0]
    assert param_err(p, golden[f"align_{name}_p"]) < TOL
    assert rel_err(r["aligned"].cpu().numpy()[0], golden[f"align_{name}_vol"]) < TOL
    assert int(r["iterations"].cpu()[0]) == 10
    if typ == 1:
        np.testing.assert_allclose(r["rotations"].cpu().numpy()[0], golden["align_rigid_rot"],
                                   atol=1e-3)


def test_batched_equals_one_at_a_time(ctx, lin_filters):
    base = S.base_volume((13, 20, 24), seed=2)
    rng = np.random.default_rng(0)
    movs = []
    for _ in range(5):
        A = S._rotation(*np.deg2rad(rng.uniform(-3, 3, 3)))
        movs.append(S.transform_volume(base, A, rng.uniform(-1.5, 1.5, 3)))
    movs = np.stack(movs)
    rb = ctx.register_linear(cuda(base), cuda(movs), lin_filters, 6, L.RIGID)
    pb = rb["params"].cpu().numpy()
    for i in range(5):
        ri = ctx.register_linear(cuda(base), cuda(movs[i])[None], lin_filters, 6, L.RIGID)
        assert np.array_equal(ri["params"].cpu().numpy()[0], pb[i])
    # per-instance references (stride) give the same as the shared one
    rs = ctx.register_linear(cuda(np.stack([base] * 5)), cuda(movs), lin_filters, 6, L.RIGID)
    assert np.array_equal(rs["params"].cpu().numpy(), pb)


def test_batched_matches_oracle(ctx, orc, lin_filters):
    vols, _ = S.motion_series(T=4, shape=(11, 22, 18), snr=50.0)
    r = ctx.register_linear(cuda(vols[0]), cuda(vols[1:]), lin_filters, 5, L.AFFINE)
    for i in range(3):
        p, vol, _ = orc.align_linear(vols[0], vols[i + 1], lin_filters, 5, 2)
        assert param_err(r["params"].cpu().numpy()[i], p) < TOL
        assert rel_err(r["aligned"].cpu().numpy()[i], vol) < TOL


def test_motion_correction_matches_golden(ctx, golden, lin_filters):
    corr, motion = ctx.motion_correct(golden["mc_series"], golden["mc_voxel"], lin_filters, 5)
    gm = golden["mc_motion"]
    for t in range(gm.shape[1]):
        assert param_err(motion[:3, t] / golden["mc_voxel"], gm[:3, t] / golden["mc_voxel"]) < TOL
    np.testing.assert_allclose(motion[3:], gm[3:], atol=2e-3)
    assert np.array_equal(corr[0], golden["mc_series"][0])
    assert rel_err(corr, golden["mc_corrected"]) < TOL


@pytest.mark.parametrize("prec", [L.PREC_FP32, L.PREC_BF16X3])
def test_chunked_host_motion_correction_equals_device_batch(ctx, lin_filters, prec):
    """A 70-volume series goes through brc_motion_correct in three chunks
    (6 / 57 / 6 registrations) with overlapped copies; every volume's
    parameters and corrected volume equal
    those of the device-resident batch of all 69 registrations (the
    instances are independent, so the split does not change any result)."""
    vols, _ = S.motion_series(T=70, shape=(13, 18, 20), snr=50.0)
    vs = np.array([3.0, 3.0, 3.5], np.float32)
    corr, motion = ctx.motion_correct(vols, vs, lin_filters, 8, tolerance=1e-3, precision=prec,
                                      certainty_sigma=1.0)
    r = ctx.register_linear(cuda(vols[0]), cuda(vols[1:]), lin_filters, 8, L.RIGID, tolerance=1e-3,
                            precision=prec, certainty_sigma=1.0)
    p = r["params"].cpu().numpy()
    assert np.array_equal(motion[:3, 1:].T, p[:, :3] * vs)
    assert np.array_equal(motion[3:, 1:].T, r["rotations"].cpu().numpy())
    assert np.array_equal(corr[1:], r["aligned"].cpu().numpy())
    assert np.array_equal(corr[0], vols[0])


def test_early_exit_stops_converged_instances(ctx, lin_filters):
    vols, _ = S.motion_series(T=6, shape=(17, 32, 32), snr=50.0)
    full = ctx.register_linear(cuda(vols[0]), cuda(vols[1:]), lin_filters, 30, L.RIGID)
    early = ctx.register_linear(cuda(vols[0]), cuda(vols[1:]), lin_filters, 30, L.RIGID, tolerance=1e-3)
    it = early["iterations"].cpu().numpy()
    assert it.min() >= 1 and it.max() <= 30 and it.min() < 30
    pf = full["params"].cpu().numpy()
    pe = early["params"].cpu().numpy()
    for i in range(5):
        assert S.rms_displacement_error(pe[i], pf[i], vols.shape[1:]) < 5e-3


def test_ground_truth_recovery_config0_shape(ctx):
    """64x64x33 affine pair, lognormal filters (u0 = pi/3, 2 octaves):
    20 iterations recover the applied affine."""
    flt = F.linear_registration_filters()
    base, moved, truth = S.affine_pair((33, 64, 64))
    r = ctx.register_linear(cuda(base), cuda(moved)[None], flt, 20, L.AFFINE)
    p = r["params"].cpu().numpy()[0]
    err0 = S.rms_displacement_error(np.zeros(12), truth, base.shape)
    err = S.rms_displacement_error(p, truth, base.shape)
    assert err < 0.2 * err0 and err < 0.5


def test_constant_volume(ctx, lin_filters):
    v = torch.full((12, 14, 16), 3.0, device="cuda")
    r = ctx.register_linear(v, v[None], lin_filters, 3, L.AFFINE)
    assert torch.all(r["params"] == 0)
    assert torch.equal(r["aligned"][0], v)


def test_tiny_volume(ctx, lin_filters):
    v = cuda(np.random.default_rng(0).standard_normal((5, 4, 6)))
    r = ctx.register_linear(v, v[None], lin_filters, 2, L.RIGID)
    assert torch.all(r["params"] == 0)


def test_zero_iterations_copies_moving(ctx, lin_filters):
    v = cuda(np.random.default_rng(1).standard_normal((8, 9, 10)))
    r = ctx.register_linear(v, (v * 2)[None], lin_filters, 0, L.AFFINE)
    assert torch.equal(r["aligned"][0], v * 2)
    assert torch.all(r["params"] == 0)


def test_invalid_arguments_raise(ctx, lin_filters):
    v = torch.zeros((8, 8, 8), device="cuda")
    with pytest.raises(L.BrcError) as e:
        ctx.register_linear(v, v[None], lin_filters, -1, L.AFFINE)
    assert e.value.status == L.BRC_ERR_INVALID
    with pytest.raises(L.BrcError) as e:
        ctx.register_linear(v, v[None], lin_filters, 2, 7)
    assert e.value.status == L.BRC_ERR_INVALID
    with pytest.raises(ValueError):
        ctx.filter3d(v, np.zeros((3, 2, 5, 5, 5), np.float32))


def test_kernel_launch_counter(ctx, lin_filters):
    v = cuda(np.random.default_rng(2).standard_normal((9, 10, 11)))
    before = ctx.kernel_launches
    ctx.register_linear(v, v[None], lin_filters, 4, L.AFFINE)
    torch.cuda.synchronize()
    # active-set initialisation, reference filtering, 4 x (filter, normal
    # equations, solve, warp): without early exit every iteration is a node
    assert ctx.kernel_launches - before == 2 + 4 * 4


@pytest.mark.parametrize("use_graph", [True, False])
def test_loop_stops_when_every_instance_converged(ctx, lin_filters, use_graph):
    """A volume registered to itself converges at iteration 0.  As a graph
    with early exit, iteration 0 and the loop's WHILE node, which runs one
    more (empty) iteration and stops on the device (five kernels each, with
    the control kernel); the eager loop runs all ten iterations (four
    kernels each) over an empty active set.  Both give the same (zero)
    parameters and one iteration per instance."""
    v = cuda(np.random.default_rng(3).standard_normal((12, 14, 13)))
    before = ctx.kernel_launches
    r = ctx.register_linear(v, torch.stack([v, v]), lin_filters, 10, L.AFFINE, tolerance=1e-3, use_graph=use_graph)
    torch.cuda.synchronize()
    n = ctx.kernel_launches - before
    assert n == (2 + 2 * 5 if use_graph else 2 + 10 * 4)
    assert np.array_equal(r["iterations"].cpu().numpy(), [1, 1])
    assert np.abs(r["params"].cpu().numpy()).max() == 0.0


def test_certainty_smoothing_one_iteration_matches_oracle(ctx, orc, golden, lin_filters):
    """The certainty-smoothing switch (3x3x3 Gaussian of the certainties
    before the sums): one AFFINE iteration equals the oracle's solve of the
    smoothed-certainty normal equations."""
    q1 = orc.filter3d(golden["base"], lin_filters)
    q2 = orc.filter3d(golden["moved"], lin_filters)
    A, h = orc.normal_equations_smoothcert(q1, q2, 1.0, prec="f64")
    p = orc.solve(A, h, prec="f64")
    r = ctx.register_linear(cuda(golden["base"]), cuda(golden["moved"])[None], lin_filters, 1, L.AFFINE,
                            certainty_sigma=1.0)
    assert param_err(r["params"].cpu().numpy()[0], p) < TOL
    # and it differs from the unsmoothed solve
    r0 = ctx.register_linear(cuda(golden["base"]), cuda(golden["moved"])[None], lin_filters, 1, L.AFFINE)
    assert param_err(r0["params"].cpu().numpy()[0], p) > 10 * TOL
