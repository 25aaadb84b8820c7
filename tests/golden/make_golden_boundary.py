"""Generates tests/golden/boundary.npz from the reference itself: the outputs
of the class members beyond the registration results -- the DEBUG outputs,
the skull strip and the pre-centring -- on the inputs of golden_small.npz.

Run where the BROCCOLI sources are present, naming their root in
BROCCOLI_REF (oracle/_ref is built from them):

    BROCCOLI_REF=/path/to/BROCCOLI python tests/golden/make_golden_boundary.py

Fixtures (all from oracle/_ref, the reference's own OpenCL C kernels run on
the CPU, with Eigen where the reference uses it):

  mc_dbg_q{1,2,3}       the three responses of the motion-correction series'
                        volume 0 (the reference volume of every
                        AlignTwoVolumesLinear call; broccoli_lib.cpp:5285-5289)
  mc_dbg_pd/pc/pg       iteration 0 of the last call (volume T-1 aligned to
                        volume 0, whose aligned volume at iteration 0 is the
                        volume itself): phase difference, certainty and z
                        phase gradient of the third filter pair
                        (broccoli_lib.cpp:5349-5354), unwritten samples 0
  r2v_inverse           InvertAffineRegistrationParameters of r2v_params
  r2v_mask              a seeded binary brain mask on the template grid
  r2v_skull             DO_SKULLSTRIP: r2v_aligned_nonlinear * r2v_mask
                        (MultiplyVolumes, broccoli_lib.cpp:8066-8079)
  r2v_skull_original    DO_SKULLSTRIP_ORIGINAL: r2v_interpolated * the mask
                        carried back by r2v_inverse with NEAREST
                        (broccoli_lib.cpp:8081-8103)
  pc_*                  PerformRegistrationTwoVolumesWrapper with
                        PRECENTER_REGISTRATION: the subject centred twice by
                        its centre of mass (CenterVolumeMass, LINEAR,
                        broccoli_lib.cpp:8003-8007), then the same
                        registration as r2v_* (6 linear and 4 nonlinear
                        iterations, coarsest scale 2, 3 mm z cut)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from broccoli_b200 import filters as F  # noqa: E402

REF = os.environ.get("BROCCOLI_REF", "")


def main() -> None:
    if not REF or not os.path.isdir(os.path.join(REF, "code", "Kernels")):
        sys.exit("make_golden_boundary.py: set BROCCOLI_REF to the root of the BROCCOLI sources")
    os.environ.setdefault("REF", REF)
    O.build(ref=True)
    g = dict(np.load(os.path.join(HERE, "golden_small.npz")))
    bank = F.load_filter_dir(os.path.join(HERE, "filters"))
    flt = bank["linear"]
    out = {}

    series = g["mc_series"]
    qref = O.ref_filter3d(series[0], flt)
    qlast = O.ref_filter3d(series[-1], flt)
    for k in range(3):
        out[f"mc_dbg_q{k + 1}"] = qref[k].astype(np.complex64)
    out["mc_dbg_pd"], out["mc_dbg_pc"], out["mc_dbg_pg"] = O.ref_phase_volumes(qref[2], qlast[2], 2)

    tpl = g["r2v_template"]
    D2, H2, W2 = tpl.shape
    z, y, x = np.meshgrid(np.arange(D2), np.arange(H2), np.arange(W2), indexing="ij")
    rng = np.random.Generator(np.random.PCG64(400))
    c = np.array([D2, H2, W2]) / 2.0 + rng.uniform(-1.5, 1.5, 3)
    r = np.array([D2, H2, W2]) * rng.uniform(0.3, 0.4, 3)
    mask = ((((z - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((x - c[2]) / r[2]) ** 2) <= 1.0)
    out["r2v_mask"] = mask.astype(np.float32)
    inv = O.ref_invert_affine(g["r2v_params"])
    out["r2v_inverse"] = inv
    out["r2v_skull"] = (g["r2v_aligned_nonlinear"] * out["r2v_mask"]).astype(np.float32)
    back = O.ref_transform_affine(out["r2v_mask"], inv, interp=0)[0]
    out["r2v_skull_original"] = (g["r2v_interpolated"] * back).astype(np.float32)

    sub = g["r2v_subject"]
    c1, _ = O.ref_center_volumes(sub, 1)
    c2, _ = O.ref_center_volumes(c1[0], 1)
    pc = O.ref_register_two_volumes(c2[0], g["r2v_voxel"], tpl, (1.0, 1.0, 1.0), bank, 6, 4, 2, mm_z_cut=3)
    for k, v in pc.items():
        out["pc_" + k] = v

    path = os.path.join(HERE, "boundary.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {sorted(out)}")


if __name__ == "__main__":
    main()
