"""The drop-in BROCCOLI_LIB C++ class (include/broccoli_lib.h), driven by a
small C++ program written the way the reference's MotionCorrection CLI
uses the class.  The build (compile + link against libbroccoli_b200) is a
CPU test; running it is a GPU test compared with the golden fixtures of the
reference's own kernels (tolerances as in test_gpu_registration)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err

SRC = os.path.join(ROOT, "tests", "cpp", "broccoli_lib_mc.cpp")


def build_program(out_dir):
    exe = os.path.join(out_dir, "broccoli_lib_mc")
    libdir = os.path.join(ROOT, "broccoli_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-L", libdir,
                           "-lbroccoli_b200", f"-Wl,-rpath,{libdir}", "-o", exe])
    return exe


def test_class_program_builds(tmp_path):
    exe = build_program(str(tmp_path))
    assert os.path.exists(exe)


def test_class_reports_missing_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    exe = build_program(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_class_motion_correction_matches_golden(tmp_path, golden, lin_filters):
    exe = build_program(str(tmp_path))
    series = np.ascontiguousarray(golden["mc_series"], np.float32)
    T, D, H, W = series.shape
    vs = golden["mc_voxel"]
    p_in = tmp_path / "series.f32"
    p_f = tmp_path / "filters.f32"
    series.tofile(p_in)
    np.ascontiguousarray(lin_filters, np.float32).tofile(p_f)
    p_out = tmp_path / "out.f32"
    p_mot = tmp_path / "motion.f32"
    r = subprocess.run([exe, str(p_in), str(W), str(H), str(D), str(T), str(vs[0]), str(vs[1]), str(vs[2]),
                        str(p_f), "5", str(p_out), str(p_mot)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    corr = np.fromfile(p_out, np.float32).reshape(T, D, H, W)
    motion = np.fromfile(p_mot, np.float32).reshape(6, T)
    assert rel_err(corr, golden["mc_corrected"]) < 1e-4
    gm = golden["mc_motion"]
    tr = np.abs(motion[:3] - gm[:3]).max() / max(1.0, np.abs(gm[:3]).max())
    assert tr < 1e-4 * max(vs)
    np.testing.assert_allclose(motion[3:], gm[3:], atol=2e-3)


SMOOTH_SRC = os.path.join(ROOT, "tests", "cpp", "broccoli_lib_smooth.cpp")


def build_smoothing_program(out_dir):
    exe = os.path.join(out_dir, "broccoli_lib_smooth")
    libdir = os.path.join(ROOT, "broccoli_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SMOOTH_SRC, "-L",
                           libdir, "-lbroccoli_b200", f"-Wl,-rpath,{libdir}", "-o", exe])
    return exe


def test_smoothing_program_builds(tmp_path):
    assert os.path.exists(build_smoothing_program(str(tmp_path)))


@pytest.mark.gpu
def test_class_normalized_smoothing_matches_golden(tmp_path):
    """The Smoothing CLI's calls (PerformSmoothingNormalizedHostWrapper, FWHM
    from the fixture's sigma at 3 mm voxels) against the reference kernels'
    output: same NaN voxels, the rest within 1e-4 of the largest value."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "smooth_normalized.npz"))
    vols, mask, ref = g["vols"], g["mask"], g["out"]
    T, D, H, W = vols.shape
    exe = build_smoothing_program(str(tmp_path))
    p_in, p_c, p_out = tmp_path / "vols.f32", tmp_path / "cert.f32", tmp_path / "out.f32"
    np.ascontiguousarray(vols, np.float32).tofile(p_in)
    np.ascontiguousarray(mask, np.float32).tofile(p_c)
    fwhm = 1.5 * 2.354 * 3.0  # sigma 1.5 voxels at 3 mm
    r = subprocess.run([exe, str(p_in), str(p_c), str(W), str(H), str(D), str(T), "3", "3", "3", repr(fwhm),
                        str(p_out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(p_out, np.float32).reshape(vols.shape)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = np.isfinite(ref)
    assert np.abs(got[fin] - ref[fin]).max() <= 1e-4 * np.abs(ref[fin]).max()
