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

from conftest import GOLDEN, ROOT
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
    assert r.returncode != 0 and "not supported" in r.stderr
