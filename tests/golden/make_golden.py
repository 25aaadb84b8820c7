"""Generates the golden fixtures of this directory from the reference itself.

Run where the BROCCOLI sources are present, naming their root in
BROCCOLI_REF (the directory holding code/ and filters/):

    BROCCOLI_REF=/path/to/BROCCOLI python tests/golden/make_golden.py

1. Copies the reference's shipped filter coefficients (``filters/*.bin``:
   quadrature filters, projection tensors, filter directions) into
   ``tests/golden/filters/`` -- they are input data of the path.
2. Builds ``oracle/_ref`` (the reference's own OpenCL C kernels compiled for
   the CPU, see oracle/ref_shim.cpp) and records its outputs on small seeded
   inputs into ``golden_small.npz``: filter responses, normal equations,
   solve, rigid projection, composition, angles, warps, smoothing, rescale,
   full single-scale registrations of every type and a short motion
   correction.

The reference ships no output vectors for this path; these fixtures are the
reference's kernels run here on fixed inputs, and the inputs are stored with
them so the tests never regenerate data.
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from broccoli_b200 import filters as F  # noqa: E402
from broccoli_b200 import synthetic as S  # noqa: E402

REF = os.environ.get("BROCCOLI_REF", "")


def main() -> None:
    if not REF or not os.path.isdir(os.path.join(REF, "code", "Kernels")):
        sys.exit("make_golden.py: set BROCCOLI_REF to the root of the BROCCOLI sources")
    src = os.path.join(REF, "filters")
    dst = os.path.join(HERE, "filters")
    os.makedirs(dst, exist_ok=True)
    for name in sorted(os.listdir(src)):
        if name.endswith(".bin"):
            shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))

    os.environ.setdefault("REF", REF)
    O.build(ref=True)
    bank = F.load_filter_dir(dst)
    flt = bank["linear"]

    g = {}
    shape = (20, 24, 22)  # D, H, W -- odd/even mix, not tile multiples
    base, moved, truth = S.affine_pair(shape, base_seed=0, motion_seed=1)
    g["base"], g["moved"], g["truth"] = base, moved, truth
    q1 = O.ref_filter3d(base, flt)
    q2 = O.ref_filter3d(moved, flt)
    g["q1"], g["q2"] = q1.astype(np.complex64), q2.astype(np.complex64)
    A, h = O.ref_normal_equations(q1, q2)
    g["A"], g["h"] = A, h
    p = O.ref_solve(A, h)
    g["p_solve"] = p
    g["p_rigid"] = O.ref_remove_scaling(p)
    g["p_compose"] = O.ref_add_affine(p, 0.5 * p)
    g["rot"] = O.ref_rotation_angles(g["p_rigid"])
    g["warp_affine"] = O.ref_warp_affine(moved, p)
    rng = np.random.Generator(np.random.PCG64(7))
    fld = [(rng.standard_normal(shape) * 2.0).astype(np.float32) for _ in range(3)]
    g["field_x"], g["field_y"], g["field_z"] = fld
    g["warp_field"] = O.ref_warp_field(moved, *fld)
    fs = O.smoothing_filter_sigma(2.0)
    g["smooth_filter"] = fs
    g["smooth"] = O.ref_smooth3d(moved, fs, fs, fs)
    cert = (rng.uniform(0.2, 1.0, shape)).astype(np.float32)
    scert = O.ref_smooth3d(cert, fs, fs, fs)
    g["cert"], g["smooth_cert"] = cert, scert
    g["smooth_normalized"] = O.ref_smooth3d(moved, fs, fs, fs, cert=cert, smoothed_cert=scert)
    g["rescale"] = O.ref_rescale_linear(moved, (11, 13, 17))
    for typ, name in ((0, "translation"), (1, "rigid"), (2, "affine")):
        pp, al, rr = O.ref_align_linear(base, moved, flt, 10, typ)
        g[f"align_{name}_p"] = pp
        g[f"align_{name}_vol"] = al
        if rr is not None:
            g[f"align_{name}_rot"] = rr

    # nonlinear: six filters, projection tensors and directions
    nshape = (18, 22, 20)
    nbase, nmoved, _ = S.affine_pair(nshape, base_seed=4, motion_seed=5)
    g["nl_base"], g["nl_moved"] = nbase, nmoved
    f6 = bank["nonlinear"]
    g["nl_q1"] = np.concatenate([O.ref_filter3d(nbase, f6[:3]), O.ref_filter3d(nbase, f6[3:])]).astype(np.complex64)
    g["nl_q2"] = np.concatenate([O.ref_filter3d(nmoved, f6[:3]), O.ref_filter3d(nmoved, f6[3:])]).astype(np.complex64)
    fld1, _ = O.ref_align_nonlinear(nbase, nmoved, bank, 1)
    g["nl_field1"] = fld1
    fld3, al3 = O.ref_align_nonlinear(nbase, nmoved, bank, 3)
    g["nl_field3"], g["nl_aligned3"] = fld3, al3
    fs, als = O.ref_align_nonlinear_scales(nbase, nmoved, bank, 3, 2)
    g["nl_scales_field"], g["nl_scales_aligned"] = fs, als

    # pyramid linear registration
    sshape = (26, 30, 28)
    sbase, smoved, _ = S.affine_pair(sshape, base_seed=6, motion_seed=7)
    g["sc_base"], g["sc_moved"] = sbase, smoved
    for typ, name in ((1, "rigid"), (2, "affine")):
        pp, al, rr = O.ref_align_linear_scales(sbase, smoved, flt, 8, 2, typ)
        g[f"sc_{name}_p"], g[f"sc_{name}_vol"], g[f"sc_{name}_rot"] = pp, al, rr

    # T1-to-template normalisation on a small synthetic head pair, with
    # anisotropic input voxels and a z cut
    sub, tpl, _ = S.t1_template_pair((30, 36, 34), (32, 38, 32), seed=0)
    g["r2v_subject"], g["r2v_template"] = sub, tpl
    g["r2v_voxel"] = np.array([1.1, 0.9, 1.2], np.float32)
    g["r2v_crs"] = O.ref_change_resolution_and_size(sub, g["r2v_voxel"], tpl.shape, (1.0, 1.0, 1.0), 3)
    r2v = O.ref_register_two_volumes(sub, g["r2v_voxel"], tpl, (1.0, 1.0, 1.0), bank, 6, 4, 2, mm_z_cut=3)
    for k, v in r2v.items():
        g["r2v_" + k] = v

    series, _ = S.motion_series(T=4, shape=(14, 18, 16), snr=50.0)
    g["mc_series"] = series
    g["mc_voxel"] = np.array([3.0, 3.0, 3.5], np.float32)
    corr, motion = O.ref_motion_correct(series, g["mc_voxel"], flt, 5)
    g["mc_corrected"], g["mc_motion"] = corr, motion

    np.savez_compressed(os.path.join(HERE, "golden_small.npz"), **g)
    print("wrote", os.path.join(HERE, "golden_small.npz"), "with", len(g), "arrays")


def main_smooth_normalized() -> None:
    """Normalised-convolution smoothing of a short series with a binary
    ellipsoid mask (PerformSmoothingNormalizedWrapper) on the reference's
    kernels; the corners lie more than 4 voxels from the mask, where the
    reference's unguarded division leaves NaN."""
    shape = (16, 18, 20)
    rng = np.random.Generator(np.random.PCG64(11))
    vols = (rng.standard_normal((3,) + shape) * 10 + 100).astype(np.float32)
    z, y, x = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    c = [(n - 1) / 2.0 for n in shape]
    r = ((z - c[0]) / 5.0) ** 2 + ((y - c[1]) / 6.0) ** 2 + ((x - c[2]) / 6.5) ** 2
    mask = (r <= 1.0).astype(np.float32)
    fs = O.smoothing_filter_sigma(1.5)
    out = O.ref_smooth_normalized(vols, mask, fs, fs, fs)
    np.savez_compressed(os.path.join(HERE, "smooth_normalized.npz"), vols=vols, mask=mask, filter=fs, out=out)
    print("wrote smooth_normalized.npz; NaN voxels per volume:", int(np.isnan(out[0]).sum()))


def main_transforms() -> None:
    """The 4D transforms on the reference's kernels (TransformVolumesLinear /
    NonLinear, CenterVolumesWrapper, ChangeVolumesResolutionAndSize with
    NEAREST = 0 and LINEAR = 1), on a short series of smooth volumes with
    an off-centre blob."""
    shape = (11, 14, 17)
    rng = np.random.Generator(np.random.PCG64(21))
    z, y, x = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    blob = np.exp(-(((z - 3.5) / 3.0) ** 2 + ((y - 9.0) / 4.0) ** 2 + ((x - 5.0) / 3.5) ** 2)) * 500.0
    vols = (blob[None] + rng.standard_normal((3,) + shape) * 5 + 100).astype(np.float32)
    p12 = np.array([1.37, -0.81, 0.55, 0.031, -0.012, 0.024, 0.018, -0.027, 0.011, -0.022, 0.016, 0.013],
                   np.float32)
    field = (rng.standard_normal((3,) + shape) * 1.7).astype(np.float32)
    vin, vnew, shape2, zcut = (2.0, 2.5, 3.0), (1.5, 2.0, 3.5), (14, 12, 10), 2
    g = {"vols": vols, "p12": p12, "field": field, "vin": np.array(vin, np.float32),
         "vnew": np.array(vnew, np.float32), "shape2": np.array(shape2, np.int32), "zcut": np.int32(zcut)}
    for interp, tag in ((0, "nearest"), (1, "linear")):
        g["affine_" + tag] = O.ref_transform_affine(vols, p12, interp)
        g["field_" + tag] = O.ref_transform_field(vols, *field, interp=interp)
        g["center_" + tag], g["center_p12_" + tag] = O.ref_center_volumes(vols, interp)
        g["resize_" + tag] = O.ref_change_resolution_and_size_interp(vols, vin, shape2, vnew, zcut, interp)
    f2 = field.copy()
    O.ref_lib().ref_add_linear_nonlinear(f2.ctypes.data_as(O._P), shape[2], shape[1], shape[0],
                                         p12.ctypes.data_as(O._P))
    g["combined_field"] = f2
    np.savez_compressed(os.path.join(HERE, "transforms.npz"), **g)
    print("wrote transforms.npz")


FIRST_LEVEL = dict(epi_shape=(12, 14, 14), epi_voxel=(3.0, 3.0, 3.0), t1_shape=(24, 28, 26),
                   t1_voxel=(1.5, 1.5, 1.5), mni_shape=(18, 22, 20), mni_voxel=(2.0, 2.0, 2.0), T=4, seed=2,
                   lin_iter=4, nl_iter=2, coarsest_t1_mni=2, coarsest_epi_t1=2, mm_t1_z_cut=0, motion_iter=4,
                   smoothing_fwhm=6.0)


def main_first_level() -> None:
    """The preprocessing stages of a first-level analysis (T1 to template,
    EPI to T1 on the template grid and to the original T1, motion
    correction, EPI mask, normalised smoothing) composed from the
    reference's kernels (oracle.first_level_preprocess with prec "ref") on
    first_level_dataset inputs, plus the tensor magnitude of the T1 and the
    mask of the first EPI volume on their own."""
    c = FIRST_LEVEL
    fmri, t1, mni, _ = S.first_level_dataset(c["T"], c["epi_shape"], c["epi_voxel"], c["t1_shape"], c["t1_voxel"],
                                             c["mni_shape"], c["mni_voxel"], seed=c["seed"])
    bank = F.load_filter_dir(os.path.join(HERE, "filters"))
    out = O.first_level_preprocess(fmri, c["epi_voxel"], t1, c["t1_voxel"], mni, c["mni_voxel"], bank,
                                   c["lin_iter"], c["nl_iter"], c["coarsest_t1_mni"], c["coarsest_epi_t1"],
                                   c["mm_t1_z_cut"], c["motion_iter"], c["smoothing_fwhm"], prec="ref")
    g = {"in_fmri": fmri, "in_t1": t1, "in_mni": mni,
         "tensor_magnitude_t1": O.ref_tensor_magnitude(t1, bank),
         "segment_epi0": O.ref_segment_epi(fmri[0], c["epi_voxel"])}
    g.update({"cfg_" + k: np.asarray(v) for k, v in c.items() if not k.endswith("_shape")})
    g.update({"out_" + k: np.asarray(v, np.float32) for k, v in out.items()})
    np.savez_compressed(os.path.join(HERE, "first_level.npz"), **g)
    print("wrote first_level.npz")


if __name__ == "__main__":
    main()
    main_smooth_normalized()
    main_transforms()
    main_first_level()
