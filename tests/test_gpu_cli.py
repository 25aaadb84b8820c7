"""The command-line tools (broccoli_b200/bin/MotionCorrection,
RegisterTwoVolumes, built from broccoli_b200/cli/ on the BROCCOLI_LIB class)
on NIfTI files: their outputs equal the library's on the same data, and the
motion-parameter and affine-matrix files hold the reference's columns
(Bash_Wrapper/MotionCorrection.cpp:747-775, RegisterTwoVolumes.cpp:1220-1246)."""
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import GOLDEN, ROOT, rel_err
from broccoli_b200 import _lib as L
from broccoli_b200 import nifti
from broccoli_b200 import synthetic as S

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "broccoli_b200", "bin")
FILTERS = os.path.join(GOLDEN, "filters")


def run(args):
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    return r


def header_with_voxels(vs):
    """A NiftiImage header template with the given voxel sizes."""
    import struct
    h = bytearray(348)
    struct.pack_into("<i", h, 0, 348)
    struct.pack_into("<8f", h, 76, 1.0, *vs, 1.0, 1.0, 1.0, 1.0)
    h[344:348] = b"n+1\0"
    return nifti.NiftiImage(None, bytes(h), [1.0, *vs, 1, 1, 1, 1], 16)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_motion_correction_cli_equals_library(ctx, tmp_path, bank, precision):
    vols, _ = S.motion_series(T=8, shape=(18, 22, 20), snr=50.0)
    vs = (3.0, 3.0, 3.5)
    path = os.path.join(tmp_path, "run1.nii.gz")
    nifti.write(path, vols, header_with_voxels(vs))
    run([os.path.join(BIN, "MotionCorrection"), path, "-filters", FILTERS, "-iterations", "6", "-precision",
         precision, "-quiet"])
    out = nifti.read(os.path.join(tmp_path, "run1_mc.nii.gz"))
    prec = L.PREC_FP32 if precision == "fp32" else L.PREC_BF16X3
    corr, motion = ctx.motion_correct(vols, vs, bank["linear"], 6, precision=prec)
    assert np.array_equal(out.data, corr)
    assert out.voxel_size == vs
    cols = np.loadtxt(os.path.join(tmp_path, "run1_motionparameters.1D"))
    expect = np.stack([motion[4], -motion[3], motion[5], -motion[2], -motion[0], -motion[1]], 1)
    np.testing.assert_allclose(cols, expect, rtol=1e-5, atol=1e-6)  # printed with 6 significant digits


def test_motion_correction_cli_reference_volume_and_output_name(ctx, tmp_path, bank):
    vols, _ = S.motion_series(T=5, shape=(14, 16, 18), snr=50.0)
    vs = (2.0, 2.0, 2.0)
    series = os.path.join(tmp_path, "series.nii")
    refp = os.path.join(tmp_path, "ref.nii")
    nifti.write(series, vols, header_with_voxels(vs))
    nifti.write(refp, vols[2], header_with_voxels(vs))
    outp = os.path.join(tmp_path, "corrected.nii")
    run([os.path.join(BIN, "MotionCorrection"), series, "-filters", FILTERS, "-iterations", "4",
         "-referencevolume", refp, "-output", outp, "-quiet"])
    corr, _ = ctx.motion_correct(vols, vs, bank["linear"], 4, reference=vols[2])
    assert np.array_equal(nifti.read(outp).data, corr)
    assert os.path.exists(os.path.join(tmp_path, "corrected_motionparameters.1D"))


def test_register_two_volumes_cli_equals_library(ctx, tmp_path, bank):
    subj = S.head_phantom((22, 26, 24), seed=4).astype(np.float32)
    tpl = np.ascontiguousarray(subj[1:-1, 2:-1, 1:-2])
    vin, vtpl = (2.0, 2.0, 2.0), (2.2, 2.1, 2.3)
    sp = os.path.join(tmp_path, "t1.nii")
    tp = os.path.join(tmp_path, "template.nii.gz")
    nifti.write(sp, subj, header_with_voxels(vin))
    nifti.write(tp, tpl, header_with_voxels(vtpl))
    run([os.path.join(BIN, "RegisterTwoVolumes"), sp, tp, "-filters", FILTERS, "-iterationslinear", "4",
         "-iterationsnonlinear", "2", "-lowestscale", "2", "-sigma", "4.0", "-savematrix", "-savefield",
         "-saveinterpolated", "-quiet"])
    r = ctx.register_two_volumes(torch.from_numpy(subj).cuda(), vin, torch.from_numpy(tpl).cuda(), vtpl, bank,
                                 4, 2, 2, 0, 4.0, 4.0, 4.0)
    names = {"interpolated": "t1_interpolated.nii", "aligned_linear": "t1_aligned_linear.nii",
             "aligned_nonlinear": "t1_aligned_nonlinear.nii"}
    for k, n in names.items():
        img = nifti.read(os.path.join(tmp_path, n))
        assert np.array_equal(img.data, r[k].cpu().numpy()), k
        assert img.data.shape == tpl.shape and img.voxel_size == tuple(np.float32(vtpl))
    f = r["field"].cpu().numpy()
    for a, ax in enumerate("xyz"):
        assert np.array_equal(nifti.read(os.path.join(tmp_path, f"t1_displacement_{ax}.nii")).data, f[a])
    m = np.loadtxt(os.path.join(tmp_path, "t1_affinematrix.txt"))
    p = r["params"]
    expect = np.array([[p[3] + 1, p[4], p[5], p[0]], [p[6], p[7] + 1, p[8], p[1]], [p[9], p[10], p[11] + 1, p[2]],
                       [0, 0, 0, 1]])
    np.testing.assert_allclose(m, expect, rtol=1e-5, atol=1e-6)


def test_cli_errors(tmp_path):
    bad = os.path.join(tmp_path, "nope.nii")
    r = subprocess.run([os.path.join(BIN, "MotionCorrection"), bad, "-filters", FILTERS, "-quiet"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Could not read" in r.stderr
    r = subprocess.run([os.path.join(BIN, "RegisterTwoVolumes"), bad, bad, "-mask", "m.nii"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Could not read" in r.stderr


@pytest.mark.parametrize("maskopt", ["-mask", "-maskoriginal"])
def test_register_two_volumes_cli_precenter_mask_debug(ctx, tmp_path, bank, maskopt):
    """-precenter, -mask / -maskoriginal and -debug (RegisterTwoVolumes.cpp:
    364-392, :410, :1088-1160, :1292-1318): the masked volume is the
    library's aligned (or interpolated) volume times the (carried back)
    mask, and the debug volumes are the template's responses."""
    subj = S.head_phantom((22, 26, 24), seed=4).astype(np.float32)
    tpl = np.ascontiguousarray(subj[1:-1, 2:-1, 1:-2])
    mask = (tpl > 400).astype(np.float32)
    vin, vtpl = (2.0, 2.0, 2.0), (2.2, 2.1, 2.3)
    sp = os.path.join(tmp_path, "t1.nii")
    tp = os.path.join(tmp_path, "template.nii")
    mp = os.path.join(tmp_path, "mask.nii")
    nifti.write(sp, subj, header_with_voxels(vin))
    nifti.write(tp, tpl, header_with_voxels(vtpl))
    nifti.write(mp, mask, header_with_voxels(vtpl))
    run([os.path.join(BIN, "RegisterTwoVolumes"), sp, tp, "-filters", FILTERS, "-iterationslinear", "4",
         "-iterationsnonlinear", "2", "-lowestscale", "2", "-sigma", "4.0", "-precenter", maskopt, mp, "-debug",
         "-quiet"])
    r = ctx.register_two_volumes(torch.from_numpy(subj).cuda(), vin, torch.from_numpy(tpl).cuda(), vtpl, bank,
                                 4, 2, 2, 0, 4.0, 4.0, 4.0, precenter=True)
    lin = nifti.read(os.path.join(tmp_path, "t1_aligned_linear.nii")).data
    assert np.array_equal(lin, r["aligned_linear"].cpu().numpy())
    masked = nifti.read(os.path.join(tmp_path, "t1_masked.nii")).data
    m = torch.from_numpy(mask).cuda()
    if maskopt == "-mask":
        expect = r["aligned_nonlinear"] * m
    else:
        from broccoli_b200.api import Context
        inv = Context.invert_affine_parameters(r["params"])
        back = ctx.transform_volumes_linear(m, inv, 0)
        expect = r["interpolated"] * back.reshape(m.shape)
    assert np.array_equal(masked, expect.cpu().numpy())
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import oracle
    qt = oracle.filter3d(tpl, bank["linear"])
    for k in range(3):
        re = nifti.read(os.path.join(tmp_path, f"t1_quadrature_filter_response_{k + 1}_real.nii")).data
        im = nifti.read(os.path.join(tmp_path, f"t1_quadrature_filter_response_{k + 1}_imag.nii")).data
        assert rel_err(re + 1j * im, qt[k]) < 1e-4
    for n in ("phase_differences", "phase_certainties", "phase_gradients"):
        assert os.path.exists(os.path.join(tmp_path, f"t1_{n}.nii"))


@pytest.mark.parametrize("mode", ["ones", "mask", "automask"])
def test_smoothing_cli_equals_library(ctx, tmp_path, mode):
    """Smoothing (Bash_Wrapper/Smoothing.cpp): normalised smoothing with a
    mask, with the all-ones certainty, or with the library's EPI mask
    (written as _mask)."""
    vols, _ = S.motion_series(T=3, shape=(12, 16, 14), snr=50.0)
    vs = (3.0, 3.0, 3.5)
    path = os.path.join(tmp_path, "epi.nii")
    nifti.write(path, vols, header_with_voxels(vs))
    args = [os.path.join(BIN, "Smoothing"), path, "-fwhm", "8", "-quiet"]
    mask = np.ones(vols.shape[1:], np.float32)
    if mode == "mask":
        mask = (S.head_phantom(vols.shape[1:], seed=3) > 200).astype(np.float32)
        nifti.write(os.path.join(tmp_path, "mask.nii"), mask, header_with_voxels(vs))
        args += ["-mask", os.path.join(tmp_path, "mask.nii")]
    if mode == "automask":
        args += ["-automask"]
        mask = ctx.segment_epi(torch.from_numpy(vols[0]).cuda(), vs).cpu().numpy()
    run(args)
    fx, fy, fz = ctx.smoothing_filters_fwhm(8.0, vs)
    want = ctx.smooth_normalized(torch.from_numpy(vols).cuda(), torch.from_numpy(mask).cuda(), fx, fy, fz)
    out = nifti.read(os.path.join(tmp_path, "epi_sm.nii"))
    assert np.array_equal(out.data, want.cpu().numpy(), equal_nan=True)
    assert out.voxel_size == vs
    if mode == "automask":
        assert np.array_equal(nifti.read(os.path.join(tmp_path, "epi_mask.nii")).data, mask)


def test_transform_volume_cli_equals_library(ctx, tmp_path):
    """TransformVolume (Bash_Wrapper/TransformVolume.cpp): a 4x4 matrix file,
    a scaling, a centring and a displacement field, each on the reference
    volume's grid, equal to the library's transform calls."""
    from broccoli_b200 import _lib as L
    rng = np.random.default_rng(7)
    vols = np.stack([S.head_phantom((20, 24, 22), seed=s) for s in (1, 2)]).astype(np.float32)
    vin, vref = (2.0, 2.0, 2.5), (2.5, 2.2, 2.4)
    ref = np.zeros((18, 22, 20), np.float32)
    src = os.path.join(tmp_path, "vol.nii")
    refp = os.path.join(tmp_path, "ref.nii.gz")
    nifti.write(src, vols, header_with_voxels(vin))
    nifti.write(refp, ref, header_with_voxels(vref))
    resampled = ctx.change_resolution_and_size_batch(torch.from_numpy(vols).cuda(), vin, ref.shape, vref, 0,
                                                     L.INTERP_LINEAR)
    # matrix (rows a11 a12 a13 tx ...), nearest neighbour
    p = np.array([1.5, -0.75, 0.5, 0.02, -0.01, 0.015, 0.01, -0.02, 0.005, -0.012, 0.01, 0.018], np.float32)
    mat = np.array([[p[3] + 1, p[4], p[5], p[0]], [p[6], p[7] + 1, p[8], p[1]], [p[9], p[10], p[11] + 1, p[2]],
                    [0, 0, 0, 1]])
    np.savetxt(os.path.join(tmp_path, "m.txt"), mat, fmt="%.9g")
    run([os.path.join(BIN, "TransformVolume"), src, refp, "-matrix", os.path.join(tmp_path, "m.txt"),
         "-interpolation", "0", "-quiet"])
    resampled0 = ctx.change_resolution_and_size_batch(torch.from_numpy(vols).cuda(), vin, ref.shape, vref, 0,
                                                      L.INTERP_NEAREST)
    pm = np.array([mat[0, 3], mat[1, 3], mat[2, 3], mat[0, 0] - 1, mat[0, 1], mat[0, 2], mat[1, 0], mat[1, 1] - 1,
                   mat[1, 2], mat[2, 0], mat[2, 1], mat[2, 2] - 1], np.float32)
    want = ctx.transform_volumes_linear(resampled0, pm, L.INTERP_NEAREST).cpu().numpy()
    out = nifti.read(os.path.join(tmp_path, "vol_warped.nii"))
    assert np.array_equal(out.data, want) and out.voxel_size == tuple(np.float32(vref))
    # scaling on the input's own grid
    run([os.path.join(BIN, "TransformVolume"), src, src, "-scaling", "1.25", "-output",
         os.path.join(tmp_path, "scaled.nii"), "-quiet"])
    same = ctx.change_resolution_and_size_batch(torch.from_numpy(vols).cuda(), vin, vols.shape[1:], vin, 0,
                                                L.INTERP_LINEAR)
    ps = np.zeros(12, np.float32)
    ps[[3, 7, 11]] = np.float32(1.0) / np.float32(1.25) - np.float32(1.0)
    want = ctx.transform_volumes_linear(same, ps, L.INTERP_LINEAR).cpu().numpy()
    assert np.array_equal(nifti.read(os.path.join(tmp_path, "scaled.nii")).data, want)
    # centring (input grid)
    run([os.path.join(BIN, "TransformVolume"), src, src, "-centering", "-quiet"])
    want, _ = ctx.center_volumes(torch.from_numpy(vols).cuda())
    assert np.array_equal(nifti.read(os.path.join(tmp_path, "vol_centered.nii")).data, want.cpu().numpy())
    # displacement field on the reference grid
    field = (rng.standard_normal((3,) + ref.shape) * 0.8).astype(np.float32)
    fps = []
    for a, ax in enumerate("xyz"):
        fps.append(os.path.join(tmp_path, f"f_{ax}.nii"))
        nifti.write(fps[-1], field[a], header_with_voxels(vref))
    run([os.path.join(BIN, "TransformVolume"), src, refp, "-field", *fps, "-output",
         os.path.join(tmp_path, "fw.nii.gz"), "-quiet"])
    f = torch.from_numpy(field).cuda()
    want = ctx.transform_volumes_nonlinear(resampled, f[0], f[1], f[2], L.INTERP_LINEAR).cpu().numpy()
    assert np.array_equal(nifti.read(os.path.join(tmp_path, "fw.nii.gz")).data, want)


def test_new_cli_errors(tmp_path):
    vol = os.path.join(tmp_path, "v.nii")
    nifti.write(vol, np.ones((4, 5, 6), np.float32), header_with_voxels((1.0, 1.0, 1.0)))
    r = subprocess.run([os.path.join(BIN, "TransformVolume"), vol, vol, "-scaling", "2", "-centering"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "exactly one" in r.stderr
    r = subprocess.run([os.path.join(BIN, "Smoothing"), vol, "-fwhm", "-1"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode != 0 and "positive" in r.stderr


def test_first_level_cli_preprocessing_equals_library(ctx, tmp_path, bank):
    """FirstLevelAnalysis -preprocessingonly (Bash_Wrapper/FirstLevelAnalysis.cpp)
    on NIfTI files: the saved matrices, motion parameters and volumes equal
    brc_first_level_preprocess on the same data (coarsest scale 1 for this
    template: fewer than 32 voxels along an axis)."""
    fmri, t1, mni, _ = S.first_level_dataset(4, (12, 14, 14), (3.0, 3.0, 3.0), (24, 28, 26), (1.5, 1.5, 1.5),
                                             (18, 22, 20), (2.0, 2.0, 2.0), seed=2)
    fp, tp, mp = (os.path.join(tmp_path, n) for n in ("run.nii", "t1.nii.gz", "mni.nii"))
    nifti.write(fp, fmri, header_with_voxels((3.0, 3.0, 3.0)))
    nifti.write(tp, t1, header_with_voxels((1.5, 1.5, 1.5)))
    nifti.write(mp, mni, header_with_voxels((2.0, 2.0, 2.0)))
    run([os.path.join(BIN, "FirstLevelAnalysis"), fp, tp, mp, "-preprocessingonly", "-filters", FILTERS,
         "-iterationslinear", "3", "-iterationsnonlinear", "2", "-iterationsmc", "3", "-smoothing", "6",
         "-saveall", "-quiet"])
    want = ctx.first_level_preprocess(fmri, (3.0, 3.0, 3.0), t1, (1.5, 1.5, 1.5), mni, (2.0, 2.0, 2.0), bank, 3, 2,
                                      3, 1, 1, smoothing_fwhm=6.0)
    vols = {"t1_interpolated.nii.gz": "interpolated_t1", "t1_aligned_mni_linear.nii.gz": "aligned_t1_linear",
            "t1_aligned_mni_nonlinear.nii.gz": "aligned_t1_nonlinear", "run_aligned_t1.nii": "aligned_epi_t1",
            "run_aligned_mni_linear.nii": "aligned_epi_mni_linear",
            "run_aligned_mni_nonlinear.nii": "aligned_epi_mni_nonlinear", "run_motion_corrected.nii": "motion_corrected",
            "run_smoothed.nii": "smoothed", "run_mask.nii": "epi_mask"}
    for name, k in vols.items():
        got = nifti.read(os.path.join(tmp_path, name)).data
        assert np.array_equal(got, want[k]), name
    for name, k in (("t1_affinematrix_t1_mni.txt", "params_t1_mni"), ("run_affinematrix_epi_t1.txt", "params_epi_t1"),
                    ("run_affinematrix_epi_mni.txt", "params_epi_mni")):
        m = np.loadtxt(os.path.join(tmp_path, name))
        p = want[k]
        expect = np.array([[p[3] + 1, p[4], p[5], p[0]], [p[6], p[7] + 1, p[8], p[1]],
                           [p[9], p[10], p[11] + 1, p[2]], [0, 0, 0, 1]])
        np.testing.assert_allclose(m, expect, rtol=1e-5, atol=1e-6)
    cols = np.loadtxt(os.path.join(tmp_path, "run_motionparameters.1D"))
    mo = want["motion_parameters"]
    np.testing.assert_allclose(cols, np.stack([mo[4], -mo[3], mo[5], -mo[2], -mo[0], -mo[1]], 1), rtol=1e-5,
                               atol=1e-6)
    r = subprocess.run([os.path.join(BIN, "FirstLevelAnalysis"), fp, tp, mp, "regressors.txt"], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode != 0 and "statistical analysis" in r.stderr
