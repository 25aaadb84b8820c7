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


@pytest.mark.gpu
def test_class_auto_mask_smoothing(tmp_path):
    """SetAutoMask(true): the certainty is the library's mask of the first
    volume (SegmentEPIData), written back to the certainty array, and the
    series is smoothed with it."""
    import torch
    from broccoli_b200 import synthetic as S
    from broccoli_b200.api import Context
    vols, _ = S.motion_series(T=3, shape=(12, 16, 14), snr=50.0)
    T, D, H, W = vols.shape
    exe = build_smoothing_program(str(tmp_path))
    p_in, p_out = tmp_path / "vols.f32", tmp_path / "out.f32"
    np.ascontiguousarray(vols, np.float32).tofile(p_in)
    r = subprocess.run([exe, str(p_in), "auto", str(W), str(H), str(D), str(T), "3", "3", "3.5", "6.0",
                        str(p_out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(p_out, np.float32).reshape(vols.shape)
    mask = np.fromfile(str(p_out) + ".mask", np.float32).reshape(D, H, W)
    ctx = Context(0)
    want_mask = ctx.segment_epi(torch.from_numpy(vols[0]).cuda(), (3.0, 3.0, 3.5))
    assert np.array_equal(mask, want_mask.cpu().numpy())
    fx, fy, fz = Context.smoothing_filters_fwhm(6.0, (3.0, 3.0, 3.5))
    want = ctx.smooth_normalized(torch.from_numpy(vols).cuda(), want_mask, fx, fy, fz).cpu().numpy()
    ctx.close()
    assert np.array_equal(got, want)


FIRST_LEVEL_SRC = os.path.join(ROOT, "tests", "cpp", "broccoli_lib_first_level.cpp")


def build_first_level_program(out_dir):
    exe = os.path.join(out_dir, "broccoli_lib_first_level")
    libdir = os.path.join(ROOT, "broccoli_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), FIRST_LEVEL_SRC, "-L",
                           libdir, "-lbroccoli_b200", f"-Wl,-rpath,{libdir}", "-o", exe])
    return exe


def test_first_level_program_builds(tmp_path):
    assert os.path.exists(build_first_level_program(str(tmp_path)))


@pytest.mark.gpu
def test_class_first_level_equals_library(tmp_path, bank):
    """PerformFirstLevelAnalysisWrapper on the class (set up as the
    reference's FirstLevelAnalysis tool does) equals
    brc_first_level_preprocess through the Python API on the same inputs,
    and refuses to run without SetPreprocessingOnly(true)."""
    from broccoli_b200.api import Context
    from test_first_level import cfg
    fl = dict(np.load(os.path.join(ROOT, "tests", "golden", "first_level.npz")))
    c = cfg(fl)
    fmri, t1, mni = fl["in_fmri"], fl["in_t1"], fl["in_mni"]
    d = str(tmp_path)
    for name, a in (("fmri", fmri), ("t1", t1), ("mni", mni), ("filters3", bank["linear"]),
                    ("filters6", bank["nonlinear"]), ("tensors", bank["projection_tensors"]),
                    ("dirs", bank["directions"])):
        np.ascontiguousarray(a, np.float32).tofile(os.path.join(d, name + ".f32"))
    exe = build_first_level_program(d)
    T, D1, H1, W1 = fmri.shape
    D2, H2, W2 = t1.shape
    D3, H3, W3 = mni.shape
    args = [W1, H1, D1, T, W2, H2, D2, W3, H3, D3, *c["epi_voxel"], *c["t1_voxel"], *c["mni_voxel"],
            c["lin_iter"], c["nl_iter"], c["motion_iter"], c["coarsest_t1_mni"], c["coarsest_epi_t1"],
            c["smoothing_fwhm"]]
    r = subprocess.run([exe, d] + [str(x) for x in args], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    ctx = Context(0)
    want = ctx.first_level_preprocess(fmri, c["epi_voxel"], t1, c["t1_voxel"], mni, c["mni_voxel"], bank,
                                      c["lin_iter"], c["nl_iter"], c["motion_iter"], c["coarsest_t1_mni"],
                                      c["coarsest_epi_t1"], 0, smoothing_fwhm=c["smoothing_fwhm"])
    ctx.close()
    files = {"params_t1_mni": "params_t1_mni", "params_epi_t1": "params_epi_t1", "params_epi_mni": "params_epi_mni",
             "motion_parameters": "motion", "interpolated_t1": "interpolated_t1",
             "aligned_t1_linear": "aligned_t1_linear", "aligned_t1_nonlinear": "aligned_t1_nonlinear",
             "aligned_epi_t1": "aligned_epi_t1", "aligned_epi_mni_linear": "aligned_epi_mni_linear",
             "aligned_epi_mni_nonlinear": "aligned_epi_mni_nonlinear", "motion_corrected": "motion_corrected",
             "epi_mask": "epi_mask", "smoothed": "smoothed", "fmri": "fmri"}
    for k, f in files.items():
        got = np.fromfile(os.path.join(d, f + ".f32"), np.float32)
        assert np.array_equal(got, want[k].reshape(-1)), k
