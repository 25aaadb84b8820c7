"""Nonlinear registration and the multi-scale drivers on the GPU against
the golden fixtures of the reference's own kernels.

Tolerance (FP32 parity): displacement fields and volumes within
max |gpu - ref| <= 1e-4 * max |ref|; parameters as in
test_gpu_registration (norm-wise 1e-4 with a 1-voxel floor)."""
import numpy as np
import pytest
import torch

from conftest import rel_err
from broccoli_b200 import _lib as L
from broccoli_b200 import synthetic as S

pytestmark = pytest.mark.gpu
TOL = 1e-4


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def param_err(p, ref):
    p = np.asarray(p, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(p - ref).max() / max(1.0, np.abs(ref).max()))


def test_filter_six_matches_golden(ctx, golden, bank):
    q = ctx.filter3d(cuda(golden["nl_base"]), bank["nonlinear"]).cpu().numpy()[0]
    assert rel_err(q, golden["nl_q1"]) < TOL


def test_nonlinear_step_matches_golden(ctx, golden, bank):
    q1 = torch.from_numpy(golden["nl_q1"]).cuda()
    q2 = torch.from_numpy(golden["nl_q2"]).cuda()
    D, H, W = golden["nl_base"].shape
    field = torch.zeros((3, D, H, W), device="cuda")
    ctx.nonlinear_step(q1, q2, bank, field)
    assert rel_err(field.cpu().numpy(), golden["nl_field1"]) < TOL
    # the step adds into the field
    ctx.nonlinear_step(q1, q2, bank, field)
    assert rel_err(field.cpu().numpy(), 2 * golden["nl_field1"]) < TOL


def test_register_nonlinear_single_scale(ctx, golden, bank):
    f, a = ctx.register_nonlinear(cuda(golden["nl_base"]), cuda(golden["nl_moved"]), bank, 6)
    # coarsest scale 1 runs ceil(6/2) = 3 iterations
    assert rel_err(f.cpu().numpy(), golden["nl_field3"]) < TOL
    assert rel_err(a.cpu().numpy(), golden["nl_aligned3"]) < TOL


def test_register_nonlinear_scales(ctx, golden, bank):
    f, a = ctx.register_nonlinear(cuda(golden["nl_base"]), cuda(golden["nl_moved"]), bank, 3,
                                  coarsest_scale=2)
    assert rel_err(f.cpu().numpy(), golden["nl_scales_field"]) < TOL
    assert rel_err(a.cpu().numpy(), golden["nl_scales_aligned"]) < TOL


def test_nonlinear_fp64_solve_close(ctx, golden, bank):
    f32, _ = ctx.register_nonlinear(cuda(golden["nl_base"]), cuda(golden["nl_moved"]), bank, 6)
    f64, _ = ctx.register_nonlinear(cuda(golden["nl_base"]), cuda(golden["nl_moved"]), bank, 6,
                                    solve_fp64=True)
    assert rel_err(f64.cpu().numpy(), f32.cpu().numpy()) < 1e-3


@pytest.mark.parametrize("typ,name", [(1, "rigid"), (2, "affine")])
def test_linear_scales_match_golden(ctx, golden, lin_filters, typ, name):
    r = ctx.register_linear_scales(cuda(golden["sc_base"]), cuda(golden["sc_moved"])[None], lin_filters, 8,
                                   2, typ)
    assert param_err(r["params"].cpu().numpy()[0], golden[f"sc_{name}_p"]) < TOL
    assert rel_err(r["aligned"].cpu().numpy()[0], golden[f"sc_{name}_vol"]) < TOL
    if typ == 1:
        np.testing.assert_allclose(r["rotations"].cpu().numpy()[0], golden["sc_rigid_rot"], atol=2e-3)


def test_nonlinear_invalid_arguments(ctx, bank):
    v = torch.zeros((8, 8, 8), device="cuda")
    with pytest.raises(L.BrcError):
        ctx.register_nonlinear(v, v, bank, 2, coarsest_scale=16)
    with pytest.raises(L.BrcError):
        ctx.register_nonlinear(v, v, bank, 2, tsigma=0.0)


def test_change_resolution_and_size_matches_golden(ctx, golden):
    out = ctx.change_resolution_and_size(cuda(golden["r2v_subject"]), golden["r2v_voxel"],
                                         golden["r2v_template"].shape, (1.0, 1.0, 1.0), 3)
    assert rel_err(out.cpu().numpy(), golden["r2v_crs"]) < TOL


def test_center_of_mass(ctx, golden, orc):
    c = ctx.center_of_mass(cuda(golden["r2v_template"]))
    D, H, W = golden["r2v_template"].shape
    ref = np.zeros(3, np.float64)
    import ctypes
    v = np.ascontiguousarray(golden["r2v_template"], np.float64)
    orc.orc_lib().orc_center_of_mass_f64(v.ctypes.data_as(ctypes.c_void_p), W, H, D,
                                         ref.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_allclose(c, ref, rtol=1e-5)


def test_register_two_volumes_matches_golden(ctx, golden, bank):
    r = ctx.register_two_volumes(cuda(golden["r2v_subject"]), golden["r2v_voxel"], cuda(golden["r2v_template"]),
                                 (1.0, 1.0, 1.0), bank, 6, 4, 2, mm_z_cut=3)
    assert param_err(r["params"], golden["r2v_params"]) < TOL
    for k in ("interpolated", "aligned_linear", "aligned_nonlinear", "field"):
        assert rel_err(r[k].cpu().numpy(), golden["r2v_" + k]) < TOL, k


@pytest.mark.parametrize("prec", [L.PREC_FP32, L.PREC_BF16X3])
def test_cohort_equals_two_volumes_per_subject(ctx, golden, bank, prec):
    """brc_register_cohort: three subjects of different sizes and voxel
    sizes (one ragged resample launch, one batched affine stage, nonlinear
    per subject) give, subject by subject, exactly what
    brc_register_two_volumes gives."""
    tpl = golden["r2v_template"]
    subs, vox = [], []
    for i, (shape, vs) in enumerate((((30, 36, 34), (1.1, 0.9, 1.2)), ((27, 40, 31), (1.2, 1.0, 1.0)),
                                     ((33, 34, 37), (0.9, 1.1, 0.95)))):
        sub, _, _ = S.t1_template_pair(shape, tpl.shape, seed=10 + i)
        subs.append(sub.astype(np.float32))
        vox.append(vs)
    c = ctx.register_cohort([cuda(v) for v in subs], vox, cuda(tpl), (1.0, 1.0, 1.0), bank, 6, 3, 2, mm_z_cut=3,
                            precision=prec)
    for i in range(3):
        r = ctx.register_two_volumes(cuda(subs[i]), vox[i], cuda(tpl), (1.0, 1.0, 1.0), bank, 6, 3, 2, mm_z_cut=3,
                                     precision=prec)
        assert np.array_equal(c["params"][i], r["params"]), i
        assert np.array_equal(c["aligned_linear"][i].cpu().numpy(), r["aligned_linear"].cpu().numpy()), i
        assert np.array_equal(c["aligned_nonlinear"][i].cpu().numpy(), r["aligned_nonlinear"].cpu().numpy()), i
        assert np.array_equal(c["fields"][i].cpu().numpy(), r["field"].cpu().numpy()), i
