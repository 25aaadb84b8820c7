"""ctypes bindings of the CPU oracle.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` import this module, as the checker.  The
product package ``broccoli_b200`` never imports it.

Two libraries are bound:

* ``liborc.so`` -- the C restatement (``orc_impl.h``), float (``*_f32``, the
  FP32 parity target) and double (``*_f64``, the accuracy oracle).
* ``_ref/libbroccoli_ref.so`` -- the reference's own OpenCL C kernels compiled
  for the CPU through ``clshim.hpp`` with the host loops restated
  (``ref_shim.cpp``).  Present only where it was built.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "libbroccoli_ref.so")

TRANSLATION, RIGID, AFFINE = 0, 1, 2

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_long
_D = ctypes.c_double


def build(ref: bool = False) -> None:
    """Compile liborc.so (and _ref/ when the reference tree is present)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])


_orc = None
_ref = None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def orc_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_PATH):
            build()
        _orc = ctypes.CDLL(ORC_PATH)
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_PATH)
    return _ref


def _dt(prec: str):
    return (np.float32, "_f32") if prec == "f32" else (np.float64, "_f64")


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def num_threads() -> int:
    return orc_lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    """OpenMP threads of the oracle and of the reference-kernel build (one
    OpenMP runtime per process)."""
    fn = orc_lib().orc_set_num_threads
    fn.argtypes = [_I]
    fn.restype = None
    fn(int(n))


# --------------------------------------------------------------------------
# restatement (liborc.so)
# --------------------------------------------------------------------------

def filter3d(vol: np.ndarray, filters: np.ndarray, prec: str = "f32") -> np.ndarray:
    """Complex responses of `vol` (D,H,W) to nfilt 7^3 filters.

    `filters` has shape (nfilt, 2, 7, 7, 7) (re/im, z, y, x).  Returns
    complex array (nfilt, D, H, W)."""
    dt, s = _dt(prec)
    D, H, W = vol.shape
    f = _arr(filters, dt)
    nf = f.shape[0]
    v = _arr(vol, dt)
    out = np.empty((nf, D, H, W, 2), dt)
    getattr(orc_lib(), "orc_filter3d" + s)(_ptr(v), W, H, D, _ptr(f), nf, _ptr(out))
    return out[..., 0] + 1j * out[..., 1]


def _interleave(q: np.ndarray, dt) -> np.ndarray:
    out = np.empty(q.shape + (2,), dt)
    out[..., 0] = q.real
    out[..., 1] = q.imag
    return out


def normal_equations(q1: np.ndarray, q2: np.ndarray, prec: str = "f32"):
    """A (12x12) and h (12) of one affine iteration from (3,D,H,W) complex
    responses of the reference (q1) and aligned (q2) volumes."""
    dt, s = _dt(prec)
    _, D, H, W = q1.shape
    a = _interleave(q1, dt)
    c = _interleave(q2, dt)
    A = np.zeros(144, dt)
    h = np.zeros(12, dt)
    getattr(orc_lib(), "orc_normal_equations" + s)(_ptr(a), _ptr(c), W, H, D, _ptr(A), _ptr(h))
    return A.reshape(12, 12).T.copy(), h


def solve(A: np.ndarray, h: np.ndarray, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    n = h.shape[0]
    Acm = _arr(np.asarray(A).T, dt)  # column-major
    hv = _arr(h, dt)
    p = np.zeros(n, dt)
    getattr(orc_lib(), "orc_solve" + s)(_ptr(Acm), _ptr(hv), n, _ptr(p))
    return p


def remove_scaling(p: np.ndarray, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    q = _arr(p, dt).copy()
    getattr(orc_lib(), "orc_remove_scaling" + s)(_ptr(q))
    return q


def add_affine(old: np.ndarray, new: np.ndarray, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    o = _arr(old, dt).copy()
    n = _arr(new, dt)
    getattr(orc_lib(), "orc_add_affine" + s)(_ptr(o), _ptr(n))
    return o


def rotation_angles(p: np.ndarray, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    q = _arr(p, dt)
    r = np.zeros(3, dt)
    getattr(orc_lib(), "orc_rotation_angles" + s)(_ptr(q), _ptr(r))
    return r


def warp_affine(src: np.ndarray, p12: np.ndarray, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    D, H, W = src.shape
    v = _arr(src, dt)
    p = _arr(p12, dt)
    out = np.empty_like(v)
    getattr(orc_lib(), "orc_warp_affine" + s)(_ptr(v), W, H, D, _ptr(p), _ptr(out))
    return out


def warp_field(src: np.ndarray, dx, dy, dz, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    D, H, W = src.shape
    v = _arr(src, dt)
    fx, fy, fz = (_arr(a, dt) for a in (dx, dy, dz))
    out = np.empty_like(v)
    getattr(orc_lib(), "orc_warp_field" + s)(_ptr(v), W, H, D, _ptr(fx), _ptr(fy), _ptr(fz), _ptr(out))
    return out


def align_linear(ref: np.ndarray, moving: np.ndarray, filters: np.ndarray, niter: int,
                 type_: int = AFFINE, prec: str = "f32", cert_sigma: float = 0.0):
    """Single-scale linear registration of `moving` to `ref`; cert_sigma > 0
    smooths the certainties by the separable 3x3x3 Gaussian of that sigma.

    Returns (params12, aligned volume, rotations in degrees or None)."""
    dt, s = _dt(prec)
    D, H, W = ref.shape
    r = _arr(ref, dt)
    orig = _arr(moving, dt).copy()
    aligned = orig.copy()
    f = _arr(filters, dt)
    p = np.zeros(12, dt)
    rot = np.zeros(3, dt)
    fn = getattr(orc_lib(), "orc_align_linear_cs" + s)
    fn.argtypes = [_P, _P, _P, _I, _I, _I, _P, _I, _I, _D, _P, _P]
    fn(_ptr(r), _ptr(aligned), _ptr(orig), W, H, D, _ptr(f), niter, type_, float(cert_sigma), _ptr(p), _ptr(rot))
    return p, aligned, (rot if type_ == RIGID else None)


def motion_correct(vols: np.ndarray, voxel_size, filters: np.ndarray, niter: int, prec: str = "f32"):
    """Rigid motion correction of a (T,D,H,W) series to volume 0.

    Returns (corrected series, motion parameters (6,T): mm then degrees)."""
    dt, s = _dt(prec)
    T, D, H, W = vols.shape
    v = _arr(vols, dt).copy()
    vs = _arr(voxel_size, dt)
    f = _arr(filters, dt)
    m = np.zeros(6 * T, dt)
    getattr(orc_lib(), "orc_motion_correct" + s)(_ptr(v), W, H, D, T, _ptr(vs), _ptr(f), niter, _ptr(m))
    return v, m.reshape(6, T)


def smoothing_filter_sigma(sigma: float, size: int = 9, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    f = np.zeros(size, dt)
    fn = getattr(orc_lib(), "orc_smoothing_filter_sigma" + s)
    fn.argtypes = [_I, _D, _P]
    fn(size, float(sigma), _ptr(f))
    return f


def smooth_normalized(vols: np.ndarray, mask: np.ndarray, fx, fy, fz, prec: str = "f32") -> np.ndarray:
    """Normalised-convolution smoothing of a (T,D,H,W) series with one
    certainty volume (PerformSmoothingNormalizedWrapper,
    broccoli_lib.cpp:11227-11272; PerformSmoothingNormalized, :11359-11450):
    smoothed mask = smoothing of the mask; each volume is smoothed with the
    mask as certainty, divided by the smoothed mask in the last pass (no
    guard: 0/0 gives NaN), then multiplied by the mask."""
    sm = smooth3d(mask, fx, fy, fz, prec=prec)
    dt, _ = _dt(prec)
    m = _arr(mask, dt)
    with np.errstate(invalid="ignore"):
        return np.stack([smooth3d(v, fx, fy, fz, mask, sm, prec=prec) * m for v in vols])


def smooth3d(vol: np.ndarray, fx, fy, fz, cert=None, smoothed_cert=None, prec: str = "f32"):
    dt, s = _dt(prec)
    D, H, W = vol.shape
    v = _arr(vol, dt)
    c = _arr(cert, dt) if cert is not None else None
    sc = _arr(smoothed_cert, dt) if smoothed_cert is not None else None
    fxa, fya, fza = (_arr(a, dt) for a in (fx, fy, fz))
    out = np.empty_like(v)
    getattr(orc_lib(), "orc_smooth3d" + s)(_ptr(v), _ptr(c) if c is not None else None,
                                           _ptr(sc) if sc is not None else None, W, H, D,
                                           _ptr(fxa), _ptr(fya), _ptr(fza), _ptr(out))
    return out


def rescale_linear(src: np.ndarray, shape, prec: str = "f32") -> np.ndarray:
    dt, s = _dt(prec)
    D, H, W = src.shape
    D2, H2, W2 = shape
    v = _arr(src, dt)
    out = np.empty((D2, H2, W2), dt)
    getattr(orc_lib(), "orc_rescale_linear" + s)(_ptr(v), W, H, D, W2, H2, D2, _ptr(out))
    return out


def align_linear_scales(ref: np.ndarray, moving: np.ndarray, filters: np.ndarray, niter: int,
                        coarsest: int, type_: int = AFFINE, prec: str = "f32"):
    """Multi-scale linear registration.  Returns (params12, aligned, rot3)."""
    dt, s = _dt(prec)
    D, H, W = ref.shape
    r = _arr(ref, dt)
    aligned = _arr(moving, dt).copy()
    f = _arr(filters, dt)
    p = np.zeros(12, dt)
    rot = np.zeros(3, dt)
    getattr(orc_lib(), "orc_align_linear_scales" + s)(_ptr(r), _ptr(aligned), W, H, D, coarsest, _ptr(f),
                                                      niter, type_, _ptr(p), _ptr(rot))
    return p, aligned, rot


def _nl_args(bank: dict, dt):
    f6 = _arr(bank["nonlinear"], dt)
    m = _arr(bank["projection_tensors"], dt)
    d = _arr(bank["directions"], dt)
    return f6, m, d


def align_nonlinear(ref: np.ndarray, moving: np.ndarray, bank: dict, niter: int, tsigma=5.0,
                    esigma=5.0, dsigma=5.0, prec: str = "f32"):
    """Single-scale nonlinear registration.  `bank` is the dict of
    broccoli_b200.filters.load_filter_dir.  Returns (field (3,D,H,W),
    aligned)."""
    dt, s = _dt(prec)
    D, H, W = ref.shape
    r = _arr(ref, dt)
    orig = _arr(moving, dt).copy()
    aligned = orig.copy()
    f6, m, d = _nl_args(bank, dt)
    field = np.zeros((3, D, H, W), dt)
    fn = getattr(orc_lib(), "orc_align_nonlinear" + s)
    fn.argtypes = [_P, _P, _P, _I, _I, _I, _P, _P, _P, _I, _D, _D, _D, _P]
    fn(_ptr(r), _ptr(aligned), _ptr(orig), W, H, D, _ptr(f6), _ptr(m), _ptr(d), niter, tsigma, esigma,
       dsigma, _ptr(field))
    return field, aligned


def align_nonlinear_scales(ref: np.ndarray, moving: np.ndarray, bank: dict, niter: int, coarsest: int,
                           tsigma=5.0, esigma=5.0, dsigma=5.0, prec: str = "f32"):
    dt, s = _dt(prec)
    D, H, W = ref.shape
    r = _arr(ref, dt)
    aligned = _arr(moving, dt).copy()
    f6, m, d = _nl_args(bank, dt)
    field = np.zeros((3, D, H, W), dt)
    fn = getattr(orc_lib(), "orc_align_nonlinear_scales" + s)
    fn.argtypes = [_P, _P, _I, _I, _I, _I, _P, _P, _P, _I, _D, _D, _D, _P]
    fn(_ptr(r), _ptr(aligned), W, H, D, coarsest, _ptr(f6), _ptr(m), _ptr(d), niter, tsigma, esigma,
       dsigma, _ptr(field))
    return field, aligned


# --------------------------------------------------------------------------
# the reference's own kernels (oracle/_ref/libbroccoli_ref.so), float only
# --------------------------------------------------------------------------

def ref_align_nonlinear(ref: np.ndarray, moving: np.ndarray, bank: dict, niter: int, tsigma=5.0,
                        esigma=5.0, dsigma=5.0):
    D, H, W = ref.shape
    r = _arr(ref, np.float32)
    orig = _arr(moving, np.float32).copy()
    aligned = orig.copy()
    f6, m, d = _nl_args(bank, np.float32)
    field = np.zeros((3, D, H, W), np.float32)
    fn = ref_lib().ref_align_nonlinear
    fn.argtypes = [_P, _P, _P, _I, _I, _I, _P, _P, _P, _I, _D, _D, _D, _P]
    fn(_ptr(r), _ptr(aligned), _ptr(orig), W, H, D, _ptr(f6), _ptr(m), _ptr(d), niter, tsigma, esigma,
       dsigma, _ptr(field))
    return field, aligned

def ref_filter3d(vol: np.ndarray, filters: np.ndarray) -> np.ndarray:
    D, H, W = vol.shape
    v = _arr(vol, np.float32)
    f = _arr(filters, np.float32)
    assert f.shape[0] == 3
    out = np.empty((3, D, H, W, 2), np.float32)
    ref_lib().ref_filter3d(_ptr(v), W, H, D, _ptr(f), _ptr(out))
    return out[..., 0] + 1j * out[..., 1]


def ref_normal_equations(q1: np.ndarray, q2: np.ndarray):
    _, D, H, W = q1.shape
    a = _interleave(q1, np.float32)
    c = _interleave(q2, np.float32)
    A = np.zeros(144, np.float32)
    h = np.zeros(12, np.float32)
    ref_lib().ref_normal_equations(_ptr(a), _ptr(c), W, H, D, _ptr(A), _ptr(h))
    return A.reshape(12, 12).T.copy(), h


def ref_solve(A: np.ndarray, h: np.ndarray) -> np.ndarray:
    n = h.shape[0]
    Acm = _arr(np.asarray(A).T, np.float32)
    hv = _arr(h, np.float32)
    p = np.zeros(n, np.float32)
    ref_lib().ref_solve(_ptr(Acm), _ptr(hv), n, _ptr(p))
    return p


def ref_remove_scaling(p: np.ndarray) -> np.ndarray:
    q = _arr(p, np.float32).copy()
    ref_lib().ref_remove_scaling(_ptr(q))
    return q


def ref_add_affine(old: np.ndarray, new: np.ndarray) -> np.ndarray:
    o = _arr(old, np.float32).copy()
    n = _arr(new, np.float32)
    ref_lib().ref_add_affine(_ptr(o), _ptr(n))
    return o


def ref_rotation_angles(p: np.ndarray) -> np.ndarray:
    q = _arr(p, np.float32)
    r = np.zeros(3, np.float32)
    ref_lib().ref_rotation_angles(_ptr(q), _ptr(r))
    return r


def ref_warp_affine(src: np.ndarray, p12: np.ndarray) -> np.ndarray:
    D, H, W = src.shape
    v = _arr(src, np.float32)
    p = _arr(p12, np.float32)
    out = np.empty_like(v)
    ref_lib().ref_warp_affine(_ptr(v), W, H, D, _ptr(p), _ptr(out))
    return out


def ref_warp_field(src: np.ndarray, dx, dy, dz) -> np.ndarray:
    D, H, W = src.shape
    v = _arr(src, np.float32)
    fx, fy, fz = (_arr(a, np.float32) for a in (dx, dy, dz))
    out = np.empty_like(v)
    ref_lib().ref_warp_field(_ptr(v), W, H, D, _ptr(fx), _ptr(fy), _ptr(fz), _ptr(out))
    return out


def ref_rescale_linear(src: np.ndarray, shape) -> np.ndarray:
    D, H, W = src.shape
    D2, H2, W2 = shape
    v = _arr(src, np.float32)
    out = np.empty((D2, H2, W2), np.float32)
    ref_lib().ref_rescale_linear(_ptr(v), W, H, D, W2, H2, D2, _ptr(out))
    return out


def ref_align_linear(ref: np.ndarray, moving: np.ndarray, filters: np.ndarray, niter: int,
                     type_: int = AFFINE):
    D, H, W = ref.shape
    r = _arr(ref, np.float32)
    orig = _arr(moving, np.float32).copy()
    aligned = orig.copy()
    f = _arr(filters, np.float32)
    p = np.zeros(12, np.float32)
    rot = np.zeros(3, np.float32)
    ref_lib().ref_align_linear(_ptr(r), _ptr(aligned), _ptr(orig), W, H, D, _ptr(f), niter, type_,
                               _ptr(p), _ptr(rot))
    return p, aligned, (rot if type_ == RIGID else None)


def ref_motion_correct(vols: np.ndarray, voxel_size, filters: np.ndarray, niter: int):
    T, D, H, W = vols.shape
    v = _arr(vols, np.float32).copy()
    vs = _arr(voxel_size, np.float32)
    f = _arr(filters, np.float32)
    m = np.zeros(6 * T, np.float32)
    ref_lib().ref_motion_correct(_ptr(v), W, H, D, T, _ptr(vs), _ptr(f), niter, _ptr(m))
    return v, m.reshape(6, T)


def ref_smooth_normalized(vols: np.ndarray, mask: np.ndarray, fx, fy, fz) -> np.ndarray:
    """PerformSmoothingNormalizedWrapper (broccoli_lib.cpp:11227-11272) on
    the reference's own kernels: the smoothed mask, then every volume
    smoothed with the mask as certainty over the smoothed mask, times the
    mask (PerformSmoothingNormalized, :11359-11450)."""
    sm = ref_smooth3d(mask, fx, fy, fz)
    with np.errstate(invalid="ignore"):
        return np.stack([ref_smooth3d(v, fx, fy, fz, mask, sm) * np.asarray(mask, np.float32) for v in vols])


def ref_smooth3d(vol: np.ndarray, fx, fy, fz, cert=None, smoothed_cert=None):
    D, H, W = vol.shape
    v = _arr(vol, np.float32)
    c = _arr(cert, np.float32) if cert is not None else None
    sc = _arr(smoothed_cert, np.float32) if smoothed_cert is not None else None
    fxa, fya, fza = (_arr(a, np.float32) for a in (fx, fy, fz))
    out = np.empty_like(v)
    ref_lib().ref_smooth3d(_ptr(v), _ptr(c) if c is not None else None,
                           _ptr(sc) if sc is not None else None, W, H, D,
                           _ptr(fxa), _ptr(fya), _ptr(fza), _ptr(out))
    return out


def ref_align_linear_scales(ref: np.ndarray, moving: np.ndarray, filters: np.ndarray, niter: int,
                            coarsest: int, type_: int = AFFINE):
    D, H, W = ref.shape
    r = _arr(ref, np.float32)
    aligned = _arr(moving, np.float32).copy()
    f = _arr(filters, np.float32)
    p = np.zeros(12, np.float32)
    rot = np.zeros(3, np.float32)
    ref_lib().ref_align_linear_scales(_ptr(r), _ptr(aligned), W, H, D, coarsest, _ptr(f), niter, type_,
                                      _ptr(p), _ptr(rot))
    return p, aligned, rot


def ref_align_nonlinear_scales(ref: np.ndarray, moving: np.ndarray, bank: dict, niter: int, coarsest: int,
                               tsigma=5.0, esigma=5.0, dsigma=5.0):
    D, H, W = ref.shape
    r = _arr(ref, np.float32)
    aligned = _arr(moving, np.float32).copy()
    f6, m, d = _nl_args(bank, np.float32)
    field = np.zeros((3, D, H, W), np.float32)
    fn = ref_lib().ref_align_nonlinear_scales
    fn.argtypes = [_P, _P, _I, _I, _I, _I, _P, _P, _P, _I, _D, _D, _D, _P]
    fn(_ptr(r), _ptr(aligned), W, H, D, coarsest, _ptr(f6), _ptr(m), _ptr(d), niter, tsigma, esigma,
       dsigma, _ptr(field))
    return field, aligned


def _r2v_args(bank):
    return (_arr(bank["linear"], np.float32), _arr(bank["nonlinear"], np.float32),
            _arr(bank["projection_tensors"], np.float32), _arr(bank["directions"], np.float32))


def _register_two_volumes(lib_fn, dt, subject, vin, template, vtpl, bank, lin_iter, nl_iter, coarsest,
                          mm_z_cut=0, tsigma=5.0, esigma=5.0, dsigma=5.0):
    D, H, W = subject.shape
    D2, H2, W2 = template.shape
    s = _arr(subject, dt)
    t = _arr(template, dt)
    f3, f6, m, d = (_arr(a, dt) for a in _r2v_args(bank))
    v1 = np.asarray(vin, np.float32)
    v2 = np.asarray(vtpl, np.float32)
    p = np.zeros(12, dt)
    interp = np.zeros((D2, H2, W2), dt)
    al = np.zeros_like(interp)
    anl = np.zeros_like(interp)
    field = np.zeros((3, D2, H2, W2), dt)
    lib_fn.argtypes = [_P, _I, _I, _I, _P, _P, _I, _I, _I, _P, _I, _I, _I, _I, _P, _P, _P, _P, _D, _D, _D,
                       _P, _P, _P, _P, _P]
    lib_fn(_ptr(s), W, H, D, _ptr(v1), _ptr(t), W2, H2, D2, _ptr(v2), mm_z_cut, coarsest, lin_iter, nl_iter,
           _ptr(f3), _ptr(f6), _ptr(m), _ptr(d), tsigma, esigma, dsigma, _ptr(p), _ptr(interp), _ptr(al),
           _ptr(anl), _ptr(field))
    return {"params": p, "interpolated": interp, "aligned_linear": al, "aligned_nonlinear": anl,
            "field": field}


def register_two_volumes(subject, vin, template, vtpl, bank, lin_iter, nl_iter, coarsest, mm_z_cut=0,
                         prec="f32", **kw):
    """T1-to-template normalisation (restatement)."""
    dt, s = _dt(prec)
    return _register_two_volumes(getattr(orc_lib(), "orc_register_two_volumes" + s), dt, subject, vin,
                                 template, vtpl, bank, lin_iter, nl_iter, coarsest, mm_z_cut, **kw)


def ref_register_two_volumes(subject, vin, template, vtpl, bank, lin_iter, nl_iter, coarsest, mm_z_cut=0,
                             **kw):
    """T1-to-template normalisation with the reference's kernels."""
    return _register_two_volumes(ref_lib().ref_register_two_volumes, np.float32, subject, vin, template,
                                 vtpl, bank, lin_iter, nl_iter, coarsest, mm_z_cut, **kw)


def change_resolution_and_size(src, vin, shape, vnew, mm_z_cut=0, prec="f32"):
    dt, s = _dt(prec)
    D, H, W = src.shape
    D2, H2, W2 = shape
    v = _arr(src, dt)
    out = np.zeros((D2, H2, W2), dt)
    fn = getattr(orc_lib(), "orc_change_resolution_and_size" + s)
    fn.argtypes = [_P, _I, _I, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P, _I, _I, _I,
                   ctypes.c_float, ctypes.c_float, ctypes.c_float, _I]
    fn(_ptr(v), W, H, D, *[float(a) for a in vin], _ptr(out), W2, H2, D2, *[float(a) for a in vnew], mm_z_cut)
    return out


def ref_change_resolution_and_size(src, vin, shape, vnew, mm_z_cut=0):
    D, H, W = src.shape
    D2, H2, W2 = shape
    v = _arr(src, np.float32)
    out = np.zeros((D2, H2, W2), np.float32)
    fn = ref_lib().ref_change_resolution_and_size
    fn.argtypes = [_P, _I, _I, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P, _I, _I, _I,
                   ctypes.c_float, ctypes.c_float, ctypes.c_float, _I]
    fn(_ptr(v), W, H, D, *[float(a) for a in vin], _ptr(out), W2, H2, D2, *[float(a) for a in vnew], mm_z_cut)
    return out


def normal_equations_smoothcert(q1: np.ndarray, q2: np.ndarray, sigma: float, prec: str = "f32"):
    """Normal equations with 3x3x3-smoothed certainties (the certainty
    smoothing switch of the motion-correction workload)."""
    dt, s = _dt(prec)
    _, D, H, W = q1.shape
    a = _interleave(q1, dt)
    c = _interleave(q2, dt)
    A = np.zeros(144, dt)
    h = np.zeros(12, dt)
    fn = getattr(orc_lib(), "orc_normal_equations_smoothcert" + s)
    fn.argtypes = [_P, _P, _I, _I, _I, _D, _P, _P]
    fn(_ptr(a), _ptr(c), W, H, D, float(sigma), _ptr(A), _ptr(h))
    return A.reshape(12, 12).T.copy(), h


def registration_objective(moving, ref, filters, sigma, params=None, field=None, prec="f64"):
    """Filter-response SSD of the smoothed moving volume warped by `params`
    (12,) or `field` (3,D,H,W) against the smoothed reference, evaluated with
    the oracle's kernels in double (the finite-difference reference of the
    differentiable registration)."""
    taps = np.exp(-(np.arange(9) - 4.0) ** 2 / (2.0 * sigma * sigma))
    taps = taps / taps.sum()
    sm = smooth3d(moving, taps, taps, taps, prec=prec)
    sr = smooth3d(ref, taps, taps, taps, prec=prec)
    if params is not None:
        w = warp_affine(sm, params, prec=prec)
    else:
        w = warp_field(sm, field[0], field[1], field[2], prec=prec)
    qm = filter3d(w, filters, prec=prec)
    qr = filter3d(sr, filters, prec=prec)
    d = qm - qr
    return float((d.real ** 2 + d.imag ** 2).sum())


# ---- 4D transforms with NEAREST (0) / LINEAR (1) interpolation ------------

def _vols4(src):
    v = np.asarray(src)
    return v[None] if v.ndim == 3 else v


def transform_affine(src, p12, interp=1, prec="f32"):
    """TransformVolumesLinear: one parameter vector applied to (T, D, H, W)."""
    dt, s = _dt(prec)
    v = _arr(_vols4(src), dt)
    T, D, H, W = v.shape
    p = _arr(p12, dt)
    out = np.empty_like(v)
    getattr(orc_lib(), "orc_transform_affine" + s)(_ptr(v), W, H, D, T, _ptr(p), int(interp), _ptr(out))
    return out


def transform_field(src, dx, dy, dz, interp=1, prec="f32"):
    """TransformVolumesNonLinear: one displacement field applied to (T, D, H, W)."""
    dt, s = _dt(prec)
    v = _arr(_vols4(src), dt)
    T, D, H, W = v.shape
    fx, fy, fz = (_arr(a, dt) for a in (dx, dy, dz))
    out = np.empty_like(v)
    getattr(orc_lib(), "orc_transform_field" + s)(_ptr(v), W, H, D, T, _ptr(fx), _ptr(fy), _ptr(fz),
                                                   int(interp), _ptr(out))
    return out


def center_volumes(src, interp=1, prec="f32"):
    """CenterVolumesWrapper: (centred volumes, 12 parameters)."""
    dt, s = _dt(prec)
    v = _arr(_vols4(src), dt)
    T, D, H, W = v.shape
    out = np.empty_like(v)
    p = np.zeros(12, dt)
    getattr(orc_lib(), "orc_center_volumes" + s)(_ptr(v), W, H, D, T, int(interp), _ptr(out), _ptr(p))
    return out, p


def change_resolution_and_size_interp(src, vin, shape, vnew, mm_z_cut=0, interp=1, prec="f32"):
    """ChangeVolumesResolutionAndSize of (T, D, H, W) volumes with an interpolation mode."""
    dt, s = _dt(prec)
    v = _arr(_vols4(src), dt)
    T, D, H, W = v.shape
    D2, H2, W2 = shape
    out = np.zeros((T, D2, H2, W2), dt)
    fn = getattr(orc_lib(), "orc_change_resolution_and_size_interp" + s)
    fn.argtypes = [_P, _I, _I, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P, _I, _I, _I,
                   ctypes.c_float, ctypes.c_float, ctypes.c_float, _I, _I]
    V, V2 = D * H * W, D2 * H2 * W2
    for t in range(T):
        src_t = v[t]
        out_t = np.zeros((D2, H2, W2), dt)
        fn(_ptr(src_t), W, H, D, *[float(a) for a in vin], _ptr(out_t), W2, H2, D2, *[float(a) for a in vnew],
           int(mm_z_cut), int(interp))
        out[t] = out_t
    return out


def ref_transform_affine(src, p12, interp=1):
    v = _arr(_vols4(src), np.float32)
    T, D, H, W = v.shape
    p = _arr(p12, np.float32)
    out = np.empty_like(v)
    ref_lib().ref_transform_linear(_ptr(v), W, H, D, T, _ptr(p), int(interp), _ptr(out))
    return out


def ref_transform_field(src, dx, dy, dz, interp=1):
    v = _arr(_vols4(src), np.float32)
    T, D, H, W = v.shape
    fx, fy, fz = (_arr(a, np.float32) for a in (dx, dy, dz))
    out = np.empty_like(v)
    ref_lib().ref_transform_nonlinear(_ptr(v), W, H, D, T, _ptr(fx), _ptr(fy), _ptr(fz), int(interp), _ptr(out))
    return out


def ref_center_volumes(src, interp=1):
    v = _arr(_vols4(src), np.float32)
    T, D, H, W = v.shape
    out = np.empty_like(v)
    p = np.zeros(12, np.float32)
    ref_lib().ref_center_volumes(_ptr(v), W, H, D, T, int(interp), _ptr(out), _ptr(p))
    return out, p


def ref_change_resolution_and_size_interp(src, vin, shape, vnew, mm_z_cut=0, interp=1):
    v = _arr(_vols4(src), np.float32)
    T, D, H, W = v.shape
    D2, H2, W2 = shape
    out = np.zeros((T, D2, H2, W2), np.float32)
    fn = ref_lib().ref_change_resolution_and_size_interp
    fn.argtypes = [_P, _I, _I, _I, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P, _I, _I, _I,
                   ctypes.c_float, ctypes.c_float, ctypes.c_float, _I, _I]
    fn(_ptr(v), W, H, D, T, *[float(a) for a in vin], _ptr(out), W2, H2, D2, *[float(a) for a in vnew],
       int(mm_z_cut), int(interp))
    return out


def match_volume_masses(v1, v2, prec="f32"):
    """MatchVolumeMasses: (v1 translated so its centre of mass meets v2's, 12 parameters)."""
    dt, s = _dt(prec)
    D, H, W = v1.shape
    a = _arr(v1, dt).copy()
    b = _arr(v2, dt)
    p = np.zeros(12, dt)
    getattr(orc_lib(), "orc_match_volume_masses" + s)(_ptr(a), _ptr(b), W, H, D, _ptr(p))
    return a, p


def smoothing_filter_fwhm(fwhm, voxel_size, size=9, prec="f32"):
    """CreateSmoothingFilters from a FWHM in mm: (fx, fy, fz)."""
    dt, s = _dt(prec)
    f = [np.zeros(size, dt) for _ in range(3)]
    fn = getattr(orc_lib(), "orc_smoothing_filter_fwhm" + s)
    fn.argtypes = [_I, _D, _D, _D, _D, _P, _P, _P]
    fn(size, float(fwhm), *[float(v) for v in voxel_size], *[_ptr(a) for a in f])
    return tuple(f)


def tensor_magnitude(vol, bank, prec="f32"):
    """CalculateTensorMagnitude of one (D, H, W) volume."""
    dt, s = _dt(prec)
    D, H, W = vol.shape
    v = _arr(vol, dt)
    f6, m, _ = _nl_args(bank, dt)
    out = np.zeros_like(v)
    getattr(orc_lib(), "orc_tensor_magnitude" + s)(_ptr(v), W, H, D, _ptr(f6), _ptr(m), _ptr(out))
    return out


def segment_epi(vol, voxel_size, prec="f32"):
    """SegmentEPIData of one (D, H, W) volume: the 1 / 0.001 mask."""
    dt, s = _dt(prec)
    D, H, W = vol.shape
    v = _arr(vol, dt)
    out = np.zeros_like(v)
    fn = getattr(orc_lib(), "orc_segment_epi" + s)
    fn.argtypes = [_P, _I, _I, _I, _D, _D, _D, _P]
    fn(_ptr(v), W, H, D, *[float(a) for a in voxel_size], _ptr(out))
    return out


def ref_match_volume_masses(v1, v2):
    D, H, W = v1.shape
    a = _arr(v1, np.float32).copy()
    b = _arr(v2, np.float32)
    p = np.zeros(12, np.float32)
    ref_lib().ref_match_volume_masses(_ptr(a), _ptr(b), W, H, D, _ptr(p))
    return a, p


def ref_tensor_magnitude(vol, bank):
    D, H, W = vol.shape
    v = _arr(vol, np.float32)
    f6, m, _ = _nl_args(bank, np.float32)
    out = np.zeros_like(v)
    ref_lib().ref_tensor_magnitude(_ptr(v), W, H, D, _ptr(f6), _ptr(m), _ptr(out))
    return out


def ref_segment_epi(vol, voxel_size):
    D, H, W = vol.shape
    v = _arr(vol, np.float32)
    out = np.zeros_like(v)
    fn = ref_lib().ref_segment_epi
    fn.argtypes = [_P, _I, _I, _I, _D, _D, _D, _P]
    fn(_ptr(v), W, H, D, *[float(a) for a in voxel_size], _ptr(out))
    return out


class _Steps:
    """The steps of the first-level preprocessing chain, from the C
    restatement (prec "f32" / "f64") or from the reference's own kernels
    (prec "ref", float)."""

    def __init__(self, prec):
        self.ref = prec == "ref"
        self.prec = "f32" if self.ref else prec
        self.dt = np.float32 if self.ref else _dt(prec)[0]

    def center(self, v):
        return (ref_center_volumes(v, 1) if self.ref else center_volumes(v, 1, self.prec))[0][0]

    def resize(self, v, vin, shape, vnew, zcut):
        if self.ref:
            return ref_change_resolution_and_size(v, vin, shape, vnew, zcut)
        return change_resolution_and_size(v, vin, shape, vnew, zcut, self.prec)

    def match(self, v1, v2):
        return ref_match_volume_masses(v1, v2) if self.ref else match_volume_masses(v1, v2, self.prec)

    def scales(self, ref, moving, filters, niter, coarsest, type_):
        if self.ref:
            return ref_align_linear_scales(ref, moving, filters, niter, coarsest, type_)
        return align_linear_scales(ref, moving, filters, niter, coarsest, type_, self.prec)

    def nonlinear(self, ref, moving, bank, niter, coarsest, ts, es, ds):
        if self.ref:
            return ref_align_nonlinear_scales(ref, moving, bank, niter, coarsest, ts, es, ds)
        return align_nonlinear_scales(ref, moving, bank, niter, coarsest, ts, es, ds, self.prec)

    def compose(self, old, new):
        return ref_add_affine(old, new) if self.ref else add_affine(old, new, self.prec)

    def affine(self, v, p):
        return (ref_transform_affine(v, p, 1) if self.ref else transform_affine(v, p, 1, self.prec))[0]

    def field(self, v, f):
        if self.ref:
            return ref_transform_field(v, f[0], f[1], f[2], 1)[0]
        return transform_field(v, f[0], f[1], f[2], 1, self.prec)[0]

    def tensor_magnitude(self, v, bank):
        return ref_tensor_magnitude(v, bank) if self.ref else tensor_magnitude(v, bank, self.prec)

    def motion(self, vols, vs, filters, niter):
        return ref_motion_correct(vols, vs, filters, niter) if self.ref else motion_correct(vols, vs, filters,
                                                                                             niter, self.prec)

    def segment(self, v, vs):
        return ref_segment_epi(v, vs) if self.ref else segment_epi(v, vs, self.prec)

    def smooth(self, vols, mask, f):
        if self.ref:
            return ref_smooth_normalized(vols, mask, *f)
        return smooth_normalized(vols, mask, *f, prec=self.prec).astype(self.dt)


def first_level_preprocess(fmri, vs_epi, t1, vs_t1, mni, vs_mni, bank, lin_iter=10, nl_iter=10,
                           coarsest_t1_mni=4, coarsest_epi_t1=4, mm_t1_z_cut=0, motion_iter=5,
                           smoothing_fwhm=6.0, apply_motion=True, apply_smoothing=True, tsigma=5.0,
                           esigma=5.0, dsigma=5.0, prec="f32"):
    """The registration, motion-correction, segmentation and smoothing stages
    of PerformFirstLevelAnalysisWrapper (broccoli_lib.cpp:8480-8733), with
    slice-timing correction off, composed in the reference's order from the
    oracle's steps (prec "f32" / "f64") or from the reference's kernels
    (prec "ref").  fmri (T, D, H, W), t1 and mni (D, H, W) volumes; voxel
    sizes (x, y, z) in mm.  Returns a dict of the outputs."""
    op = _Steps(prec)
    lin = bank["linear"]
    out = {}
    # T1 to MNI: PerformRegistrationT1MNINoSkullstrip, :8226-8273
    mni_t1 = op.resize(op.center(t1), vs_t1, mni.shape, vs_mni, mm_t1_z_cut)
    mni_t1, start_t1_mni = op.match(mni_t1, mni)
    skull = mni_t1.copy()
    out["interpolated_t1"] = skull
    p_t1_mni, mni_t1, _ = op.scales(mni, mni_t1, lin, lin_iter, coarsest_t1_mni, AFFINE)
    out["aligned_t1_linear"] = mni_t1
    field = None
    if nl_iter > 0:
        field, out["aligned_t1_nonlinear"] = op.nonlinear(mni, mni_t1, bank, nl_iter, coarsest_t1_mni, tsigma,
                                                          esigma, dsigma)
        out["field"] = field
    out["params_t1_mni"] = op.compose(p_t1_mni, start_t1_mni)  # :8510
    # EPI to T1 on the MNI grid: PerformRegistrationEPIT1, :7853-7915
    epi0 = np.asarray(fmri[0])
    t1_epi = op.resize(op.center(epi0), vs_epi, mni.shape, vs_mni, 0)
    t1_epi, start_epi_t1 = op.match(t1_epi, skull)
    p_epi_t1, t1_epi, _ = op.scales(skull, t1_epi, lin, lin_iter, coarsest_epi_t1, AFFINE)
    out["aligned_epi_t1"] = t1_epi
    epi_mni = op.affine(t1_epi, p_t1_mni)  # :8547-8556
    out["aligned_epi_mni_linear"] = epi_mni
    if field is not None:
        out["aligned_epi_mni_nonlinear"] = op.field(epi_mni, field)
    epi_t1_out = op.compose(p_epi_t1, start_epi_t1)  # :8574-8575
    out["params_epi_mni"] = op.compose(p_t1_mni, epi_t1_out)
    # EPI to the original T1: PerformRegistrationEPIT1Original, :7917-7970
    t1o = np.asarray(t1)
    t1_epi_o = op.resize(epi0, vs_epi, t1o.shape, vs_t1, 0)
    t1_epi_o, start_o = op.match(t1_epi_o, t1o)
    tm_epi = op.tensor_magnitude(t1_epi_o, bank)
    tm_t1 = op.tensor_magnitude(t1o, bank)
    aff = np.zeros(12, op.dt)
    for type_ in (TRANSLATION, RIGID):
        p, t1_epi_o, _ = op.scales(t1o, t1_epi_o, lin, lin_iter, coarsest_epi_t1 * 2, type_)
        tm_epi = op.affine(tm_epi, p)
        aff = op.compose(aff, p)
    for type_ in (RIGID, AFFINE):
        p, tm_epi, _ = op.scales(tm_t1, tm_epi, lin, lin_iter, 2, type_)
        t1_epi_o = op.affine(t1_epi_o, p)
        aff = op.compose(aff, p)
    out["params_epi_t1"] = op.compose(aff, start_o)  # :8601
    # motion correction (PerformMotionCorrectionHost, :10723-10787), the EPI
    # mask of the first corrected volume (SegmentEPIData, :11008-11030) and
    # normalised smoothing with that mask (:8700-8733)
    vols = _arr(fmri, op.dt).copy()
    if apply_motion:
        vols, out["motion_parameters"] = op.motion(vols, vs_epi, lin, motion_iter)
        out["motion_corrected"] = vols.copy()
    mask = op.segment(vols[0], vs_epi)
    out["epi_mask"] = mask
    if apply_smoothing:
        vols = op.smooth(vols, mask, smoothing_filter_fwhm(smoothing_fwhm, vs_epi, 9, op.prec))
        out["smoothed"] = vols
    out["fmri"] = vols
    return out


# --------------------------------------------------------------------------
# debug outputs and parameter inversion
# --------------------------------------------------------------------------

def phase_volumes(q1: np.ndarray, q2: np.ndarray, axis: int = 2, prec: str = "f32"):
    """Phase difference, certainty and phase gradient along `axis` of one pair
    of complex (D,H,W) responses (restatement; kernelRegistration.cpp:173-382),
    zeros where the gradient kernels write nothing."""
    dt, s = _dt(prec)
    D, H, W = q1.shape
    a = _interleave(q1, dt)
    c = _interleave(q2, dt)
    V = D * H * W
    pd = np.zeros(V, dt)
    cert = np.zeros(V, dt)
    grad = np.zeros(V, dt)
    fn = getattr(orc_lib(), "orc_phase_diff_cert" + s)
    fn.argtypes = [_P, _P, _L, _P, _P]
    fn(_ptr(a), _ptr(c), V, _ptr(pd), _ptr(cert))
    fn = getattr(orc_lib(), "orc_phase_grad" + s)
    fn.argtypes = [_P, _P, _I, _I, _I, _I, _P]
    fn(_ptr(a), _ptr(c), int(axis), W, H, D, _ptr(grad))
    return pd.reshape(D, H, W), cert.reshape(D, H, W), grad.reshape(D, H, W)


def ref_phase_volumes(q1: np.ndarray, q2: np.ndarray, axis: int = 2):
    """The same with the reference's kernels (zero-filled outputs)."""
    D, H, W = q1.shape
    a = _interleave(q1, np.float32)
    c = _interleave(q2, np.float32)
    out = [np.empty((D, H, W), np.float32) for _ in range(3)]
    fn = ref_lib().ref_phase_volumes
    fn.argtypes = [_P, _P, _I, _I, _I, _I, _P, _P, _P]
    fn(_ptr(a), _ptr(c), W, H, D, int(axis), *(_ptr(o) for o in out))
    return tuple(out)


def ref_invert_affine(p12) -> np.ndarray:
    """InvertAffineRegistrationParameters (broccoli_lib.cpp:7186-7250) with
    the reference's Eigen."""
    p = _arr(p12, np.float32)
    out = np.zeros(12, np.float32)
    fn = ref_lib().ref_invert_affine
    fn.argtypes = [_P, _P]
    fn(_ptr(p), _ptr(out))
    return out
