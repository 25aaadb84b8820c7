"""The CPU oracle against the golden fixtures made by the reference's own
kernels (tests/golden/make_golden.py), plus its behaviour on edge cases.

The float restatement keeps the reference's operation order, so most
comparisons are exact."""
import numpy as np
import pytest

from conftest import rel_err
from broccoli_b200 import synthetic as S


def test_filter_responses_exact(orc, golden, lin_filters):
    q1 = orc.filter3d(golden["base"], lin_filters)
    q2 = orc.filter3d(golden["moved"], lin_filters)
    assert np.array_equal(q1.astype(np.complex64), golden["q1"])
    assert np.array_equal(q2.astype(np.complex64), golden["q2"])


def test_normal_equations_exact(orc, golden):
    A, h = orc.normal_equations(golden["q1"], golden["q2"])
    assert np.array_equal(A, golden["A"])
    assert np.array_equal(h, golden["h"])
    # block structure: 30 distinct entries, three decoupled 4x4 systems
    assert np.count_nonzero(np.tril(A)) == 30


def test_solve_and_parameter_algebra(orc, golden):
    p = orc.solve(golden["A"], golden["h"])
    np.testing.assert_allclose(p, golden["p_solve"], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(orc.remove_scaling(golden["p_solve"]), golden["p_rigid"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(orc.add_affine(golden["p_solve"], 0.5 * golden["p_solve"]),
                               golden["p_compose"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(orc.rotation_angles(golden["p_rigid"]), golden["rot"], rtol=1e-6, atol=1e-6)


def test_rigid_projection_is_orthogonal(orc, golden):
    p = orc.remove_scaling(golden["p_solve"], prec="f64")
    R = np.eye(3) + p[3:].reshape(3, 3)
    np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-12)


def test_warps_exact(orc, golden):
    assert np.array_equal(orc.warp_affine(golden["moved"], golden["p_solve"]), golden["warp_affine"])
    w = orc.warp_field(golden["moved"], golden["field_x"], golden["field_y"], golden["field_z"])
    assert np.array_equal(w, golden["warp_field"])


def test_smoothing_and_rescale(orc, golden):
    fs = orc.smoothing_filter_sigma(2.0)
    assert np.array_equal(fs, golden["smooth_filter"])
    assert np.array_equal(orc.smooth3d(golden["moved"], fs, fs, fs), golden["smooth"])
    sn = orc.smooth3d(golden["moved"], fs, fs, fs, cert=golden["cert"], smoothed_cert=golden["smooth_cert"])
    assert np.array_equal(sn, golden["smooth_normalized"])
    assert np.array_equal(orc.rescale_linear(golden["moved"], (11, 13, 17)), golden["rescale"])


@pytest.mark.parametrize("typ,name", [(0, "translation"), (1, "rigid"), (2, "affine")])
def test_align_linear_exact(orc, golden, lin_filters, typ, name):
    p, vol, rot = orc.align_linear(golden["base"], golden["moved"], lin_filters, 10, typ)
    assert np.array_equal(p, golden[f"align_{name}_p"])
    assert np.array_equal(vol, golden[f"align_{name}_vol"])
    if typ == 1:
        assert np.array_equal(rot, golden["align_rigid_rot"])


def test_motion_correction_exact(orc, golden, lin_filters):
    corr, motion = orc.motion_correct(golden["mc_series"], golden["mc_voxel"], lin_filters, 5)
    assert np.array_equal(corr, golden["mc_corrected"])
    assert np.array_equal(motion, golden["mc_motion"])
    assert np.all(motion[:, 0] == 0)


def test_fp64_oracle_close_to_fp32(orc, golden, lin_filters):
    p32, _, _ = orc.align_linear(golden["base"], golden["moved"], lin_filters, 10, 2)
    p64, _, _ = orc.align_linear(golden["base"], golden["moved"], lin_filters, 10, 2, prec="f64")
    assert S.rms_displacement_error(p32, p64, golden["base"].shape) < 1e-3


def test_constant_volume_gives_zero_parameters(orc, lin_filters):
    v = np.full((12, 14, 16), 5.0, np.float32)
    p, al, _ = orc.align_linear(v, v, lin_filters, 3, 2)
    assert np.all(np.isfinite(p))
    assert np.all(p == 0)


def test_volume_smaller_than_filter_border(orc, lin_filters):
    rng = np.random.default_rng(3)
    v = rng.standard_normal((5, 6, 5)).astype(np.float32)
    p, _, _ = orc.align_linear(v, v, lin_filters, 2, 2)
    assert np.all(p == 0)


def test_ground_truth_recovery(orc, lin_filters):
    """Known-motion recovery, the reference's validation design
    (Matlab_Wrapper/test_motioncorrection.m:115-186, :417-423)."""
    base, moved, truth = S.affine_pair((20, 24, 22))
    p, _, _ = orc.align_linear(base, moved, lin_filters, 10, 2, prec="f64")
    err0 = S.rms_displacement_error(np.zeros(12), truth, base.shape)
    err = S.rms_displacement_error(p, truth, base.shape)
    assert err < 0.25 * err0


def test_reference_build_agrees_on_fresh_case(orc, lin_filters):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    rng = np.random.default_rng(11)
    a = rng.standard_normal((9, 13, 17)).astype(np.float32) * 100
    b = np.roll(a, 1, axis=2)
    pr, vr, _ = orc.ref_align_linear(a, b, lin_filters, 3, 1)
    po, vo, _ = orc.align_linear(a, b, lin_filters, 3, 1)
    assert np.array_equal(pr, po)
    assert np.array_equal(vr, vo)


def test_nonlinear_exact(orc, golden, bank):
    f1, _ = orc.align_nonlinear(golden["nl_base"], golden["nl_moved"], bank, 1)
    assert np.array_equal(f1, golden["nl_field1"])
    f3, a3 = orc.align_nonlinear(golden["nl_base"], golden["nl_moved"], bank, 3)
    assert np.array_equal(f3, golden["nl_field3"])
    assert np.array_equal(a3, golden["nl_aligned3"])


def test_nonlinear_scales_exact(orc, golden, bank):
    f, a = orc.align_nonlinear_scales(golden["nl_base"], golden["nl_moved"], bank, 3, 2)
    assert np.array_equal(f, golden["nl_scales_field"])
    assert np.array_equal(a, golden["nl_scales_aligned"])


@pytest.mark.parametrize("typ,name", [(1, "rigid"), (2, "affine")])
def test_linear_scales_exact(orc, golden, lin_filters, typ, name):
    p, v, r = orc.align_linear_scales(golden["sc_base"], golden["sc_moved"], lin_filters, 8, 2, typ)
    assert np.array_equal(p, golden[f"sc_{name}_p"])
    assert np.array_equal(v, golden[f"sc_{name}_vol"])
    assert np.array_equal(r, golden[f"sc_{name}_rot"])


def test_nonlinear_fp64_close(orc, golden, bank):
    f32, _ = orc.align_nonlinear(golden["nl_base"], golden["nl_moved"], bank, 3)
    f64, _ = orc.align_nonlinear(golden["nl_base"], golden["nl_moved"], bank, 3, prec="f64")
    assert rel_err(f32, f64) < 1e-3


def test_register_two_volumes_exact(orc, golden, bank):
    r = orc.register_two_volumes(golden["r2v_subject"], golden["r2v_voxel"], golden["r2v_template"],
                                 (1.0, 1.0, 1.0), bank, 6, 4, 2, mm_z_cut=3)
    for k in ("params", "interpolated", "aligned_linear", "aligned_nonlinear", "field"):
        assert np.array_equal(r[k], golden["r2v_" + k]), k
    crs = orc.change_resolution_and_size(golden["r2v_subject"], golden["r2v_voxel"],
                                         golden["r2v_template"].shape, (1.0, 1.0, 1.0), 3)
    assert np.array_equal(crs, golden["r2v_crs"])


def test_smooth_normalized_matches_reference_kernels():
    """Normalised-convolution smoothing (PerformSmoothingNormalizedWrapper):
    the FP32 restatement equals the reference's kernels bit for bit,
    including the NaN voxels of the unguarded division."""
    import os
    import oracle as O
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "smooth_normalized.npz"))
    fs = g["filter"]
    out = O.smooth_normalized(g["vols"], g["mask"], fs, fs, fs)
    assert np.array_equal(out, g["out"], equal_nan=True)
    assert np.isnan(out).any() and np.isfinite(out[:, 8, 9, 10]).all()


@pytest.fixture(scope="module")
def golden_tf():
    import os
    from conftest import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "transforms.npz")))


@pytest.mark.parametrize("interp,tag", [(0, "nearest"), (1, "linear")])
def test_transforms_match_reference_kernels(orc, golden_tf, interp, tag):
    """TransformVolumesLinear / NonLinear, CenterVolumesWrapper and
    ChangeVolumesResolutionAndSize of a 3-volume series: the restatement
    equals the reference's kernels (golden vectors) bit for bit."""
    g = golden_tf
    v = g["vols"]
    assert np.array_equal(orc.transform_affine(v, g["p12"], interp), g["affine_" + tag])
    assert np.array_equal(orc.transform_field(v, *g["field"], interp=interp), g["field_" + tag])
    c, p = orc.center_volumes(v, interp)
    assert np.array_equal(p, g["center_p12_" + tag])
    assert np.array_equal(c, g["center_" + tag])
    r = orc.change_resolution_and_size_interp(v, g["vin"], tuple(g["shape2"]), g["vnew"], int(g["zcut"]), interp)
    assert np.array_equal(r, g["resize_" + tag])


def test_combined_field_matches_reference_kernel(orc, golden_tf):
    g = golden_tf
    f = np.ascontiguousarray(g["field"], np.float32).copy()
    D, H, W = f.shape[1:]
    orc.orc_lib().orc_add_linear_nonlinear_f32(f.ctypes.data_as(orc._P), W, H, D,
                                               np.ascontiguousarray(g["p12"]).ctypes.data_as(orc._P))
    assert np.array_equal(f, g["combined_field"])
