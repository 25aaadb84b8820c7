"""The BROCCOLI_LIB members beyond the registration results on the GPU,
through a C++ caller of the class (tests/cpp/broccoli_lib_boundary.cpp) and
the Python binding, against the reference's own kernels
(tests/golden/boundary.npz) and the oracle:

  SetDebug + SetOutputQuadratureFilterResponses (three and six arrays) +
  SetOutputPhaseDifferences / Certainties / Gradients, SetPrecenter-
  Registration, SetDoSkullstrip / SetDoSkullstripOriginal with
  SetInputMNIBrainMask and SetOutputSkullstrippedT1Volume, the
  GetOpenCLCreateKernelErrors / CreateBufferErrors getters, and the C-ABI
  entries under them (brc_ctx_set_debug_outputs, brc_phase_volumes,
  brc_multiply_volumes, brc_invert_affine_parameters).

Tolerances (FP32 parity): volumes and responses max |a - b| <= 1e-4 max |b|;
parameters norm-wise 1e-4 with a 1-voxel floor; angles (phase differences
and gradients) compared modulo 2 pi within 1e-4 * pi.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import GOLDEN, ROOT, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4
SRC = os.path.join(ROOT, "tests", "cpp", "broccoli_lib_boundary.cpp")


def param_err(p, ref):
    p = np.asarray(p, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(p - ref).max() / max(1.0, np.abs(ref).max()))


def angle_err(a, b):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return float(np.minimum(d, 2 * np.pi - d).max())


@pytest.fixture(scope="module")
def boundary():
    return dict(np.load(os.path.join(GOLDEN, "boundary.npz")))


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("bin")
    out = str(d / "broccoli_lib_boundary")
    libdir = os.path.join(ROOT, "broccoli_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-L", libdir,
                           "-lbroccoli_b200", f"-Wl,-rpath,{libdir}", "-o", out])
    return out


def _f(path, a, dt=np.float32):
    np.ascontiguousarray(a, dt).tofile(path)
    return str(path)


def test_class_debug_outputs_of_motion_correction(exe, tmp_path, golden, boundary, lin_filters):
    series = golden["mc_series"]
    T, D, H, W = series.shape
    r = subprocess.run([exe, "mc", _f(tmp_path / "s.f32", series), str(W), str(H), str(D), str(T),
                        _f(tmp_path / "f.f32", lin_filters), "5", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for k in range(3):
        q = np.fromfile(tmp_path / f"q{k + 1}.c64", np.complex64).reshape(D, H, W)
        assert rel_err(q, boundary[f"mc_dbg_q{k + 1}"]) < TOL, k
    pd = np.fromfile(tmp_path / "pd.f32", np.float32).reshape(D, H, W)
    pc = np.fromfile(tmp_path / "pc.f32", np.float32).reshape(D, H, W)
    pg = np.fromfile(tmp_path / "pg.f32", np.float32).reshape(D, H, W)
    assert angle_err(pd, boundary["mc_dbg_pd"]) < TOL * np.pi
    assert rel_err(pc, boundary["mc_dbg_pc"]) < TOL
    assert angle_err(pg, boundary["mc_dbg_pg"]) < TOL * np.pi
    assert not pg[0].any() and not pg[-1].any()


def _r2v_args(exe, tmp_path, golden, bank, precenter, strip, mask, debug):
    sub = golden["r2v_subject"]
    tpl = golden["r2v_template"]
    D, H, W = sub.shape
    D2, H2, W2 = tpl.shape
    vs = golden["r2v_voxel"]
    f6 = np.ascontiguousarray(bank["nonlinear"], np.float32)
    return [exe, "r2v", _f(tmp_path / "sub.f32", sub), str(W), str(H), str(D), str(vs[0]), str(vs[1]), str(vs[2]),
            _f(tmp_path / "tpl.f32", tpl), str(W2), str(H2), str(D2), _f(tmp_path / "f3.f32", bank["linear"]),
            _f(tmp_path / "f6.f32", f6), _f(tmp_path / "m.f32", bank["projection_tensors"]),
            _f(tmp_path / "d.f32", bank["directions"]), "6", "4", "2", "3", str(precenter), str(strip),
            _f(tmp_path / "mask.f32", mask) if strip in (1, 2) else "-", str(debug), str(tmp_path)]


def _r2v_outputs(tmp_path, shape):
    D2, H2, W2 = shape
    out = {"params": np.fromfile(tmp_path / "params.f32", np.float32)}
    for k in ("interpolated", "aligned_linear", "aligned_nonlinear"):
        out[k] = np.fromfile(tmp_path / f"{k}.f32", np.float32).reshape(D2, H2, W2)
    out["field"] = np.fromfile(tmp_path / "field.f32", np.float32).reshape(3, D2, H2, W2)
    return out


@pytest.mark.parametrize("precenter", [0, 1])
def test_class_two_volumes_skull_strip_and_precenter(exe, tmp_path, golden, boundary, bank, orc, precenter):
    tpl = golden["r2v_template"]
    r = subprocess.run(_r2v_args(exe, tmp_path, golden, bank, precenter, 1, boundary["r2v_mask"], 3),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = _r2v_outputs(tmp_path, tpl.shape)
    pre = "pc_" if precenter else "r2v_"
    assert param_err(out["params"], boundary["pc_params"] if precenter else golden["r2v_params"]) < TOL
    for k in ("interpolated", "aligned_linear", "aligned_nonlinear", "field"):
        ref = boundary[pre + k] if precenter else golden[pre + k]
        assert rel_err(out[k], ref) < TOL, k
    skull = np.fromfile(tmp_path / "skull.f32", np.float32).reshape(tpl.shape)
    # the skull strip is the product of this run's aligned volume and the mask
    assert np.array_equal(skull, out["aligned_nonlinear"] * boundary["r2v_mask"])
    if not precenter:
        assert rel_err(skull, boundary["r2v_skull"]) < TOL
    # debug: the last linear call's reference volume is the template at full size
    qt = orc.filter3d(tpl, bank["linear"])
    for k in range(3):
        q = np.fromfile(tmp_path / f"q{k + 1}.c64", np.complex64).reshape(tpl.shape)
        assert rel_err(q, qt[k]) < TOL, k


def test_class_two_volumes_skull_strip_original(exe, tmp_path, golden, boundary, bank, orc):
    tpl = golden["r2v_template"]
    r = subprocess.run(_r2v_args(exe, tmp_path, golden, bank, 0, 2, boundary["r2v_mask"], 6),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = _r2v_outputs(tmp_path, tpl.shape)
    skull = np.fromfile(tmp_path / "skull.f32", np.float32).reshape(tpl.shape)
    # the mask carried back by the inverse of this run's parameters (NEAREST)
    from broccoli_b200.api import Context
    inv = Context.invert_affine_parameters(out["params"])
    back = orc.transform_affine(boundary["r2v_mask"], inv, interp=0)[0]
    assert np.array_equal(skull, out["interpolated"] * back)
    # against the reference's own result: NEAREST may round a sample that
    # lies within the parameters' rounding of a half-voxel the other way
    bad = np.abs(skull - boundary["r2v_skull_original"]) > TOL * np.abs(boundary["r2v_skull_original"]).max()
    assert bad.mean() < 1e-3
    # six responses: the nonlinear reference (the template) at the finest scale
    qt = orc.filter3d(tpl, bank["nonlinear"])
    for k in range(6):
        q = np.fromfile(tmp_path / f"q{k + 1}.c64", np.complex64).reshape(tpl.shape)
        assert rel_err(q, qt[k]) < TOL, k


def test_class_skull_strip_without_mask_fails_loudly(exe, tmp_path, golden, bank, boundary):
    # SetDoSkullstrip(true) without SetInputMNIBrainMask: an error, not a
    # silently unwritten output
    r = subprocess.run(_r2v_args(exe, tmp_path, golden, bank, 0, 3, boundary["r2v_mask"], 0), capture_output=True,
                       text=True)
    assert r.returncode == 1
    assert "SetInputMNIBrainMask" in r.stderr


def test_python_debug_outputs_of_linear_registration(ctx, orc, golden, lin_filters):
    base, moved = golden["base"], golden["moved"]
    D, H, W = base.shape
    outs = {"quadrature_responses": [np.zeros((D, H, W), np.complex64) for _ in range(3)],
            "phase_differences": np.zeros((D, H, W), np.float32),
            "phase_certainties": np.zeros((D, H, W), np.float32),
            "phase_gradients": np.zeros((D, H, W), np.float32)}
    ctx.set_debug_outputs(outs)
    try:
        ctx.register_linear(torch.from_numpy(base).cuda(), torch.from_numpy(moved).cuda()[None], lin_filters, 4, 2)
    finally:
        ctx.set_debug_outputs(None)
    q1 = orc.filter3d(base, lin_filters)
    q2 = orc.filter3d(moved, lin_filters)
    for k in range(3):
        assert rel_err(outs["quadrature_responses"][k], q1[k]) < TOL
    pd, pc, pg = orc.phase_volumes(q1[2], q2[2], 2)
    assert angle_err(outs["phase_differences"], pd) < TOL * np.pi
    assert rel_err(outs["phase_certainties"], pc) < TOL
    assert angle_err(outs["phase_gradients"], pg) < TOL * np.pi


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_phase_volumes_match_oracle(ctx, orc, golden, axis):
    q1, q2 = golden["q1"][axis], golden["q2"][axis]
    pd, pc, pg = ctx.phase_volumes(torch.from_numpy(q1).cuda(), torch.from_numpy(q2).cuda(), axis)
    rd, rc, rg = orc.phase_volumes(q1, q2, axis)
    assert angle_err(pd.cpu().numpy(), rd) < TOL * np.pi
    assert rel_err(pc.cpu().numpy(), rc) < TOL
    assert angle_err(pg.cpu().numpy(), rg) < TOL * np.pi


def test_multiply_volumes(ctx):
    rng = np.random.default_rng(3)
    v = rng.standard_normal((3, 7, 9, 11)).astype(np.float32)
    m = (rng.random((7, 9, 11)) > 0.5).astype(np.float32)
    t = torch.from_numpy(v).cuda()
    ctx.multiply_volumes(t, torch.from_numpy(m).cuda())
    assert np.array_equal(t.cpu().numpy(), v * m[None])
