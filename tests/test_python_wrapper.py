"""The Python mirror of BROCCOLI's Python wrapper (broccoli_b200.broccoli_lib):
the packing convention (the reference's own round-trip check,
broccoli_common.py:9-11) on the CPU, and motion correction through it on the
GPU against the golden fixtures of the reference's kernels."""
import numpy as np
import pytest

from conftest import rel_err
from broccoli_b200 import broccoli_lib as BL


def to_wrapper_layout(vol_zyx):
    """(D, H, W) or (T, D, H, W) arrays (x fastest) in the wrapper's input
    convention, which packVolume undoes (flipud + transpose)."""
    if vol_zyx.ndim == 3:
        return np.flipud(vol_zyx.transpose(1, 2, 0))
    return np.flipud(vol_zyx.transpose(2, 3, 1, 0))


def test_pack_unpack_round_trip():
    B = BL.BROCCOLI_LIB()
    rng = np.random.default_rng(0)
    a = rng.standard_normal((5, 6, 7)).astype(np.float32)
    packed = B.packVolume(a)
    assert np.array_equal(B.unpackOutputVolume(packed.copy(), a.shape), a)
    # 4D: the reference's unpack flips the second axis of the packed
    # (T, D, H, W) array (fliplr), not the H axis that packing flipped; the
    # mirror keeps that behaviour, so the round trip differs by a z flip.
    a4 = rng.standard_normal((4, 5, 6, 3)).astype(np.float32)
    un = B.unpackOutputVolume(B.packVolume(a4).copy(), a4.shape)
    assert np.array_equal(np.flipud(np.fliplr(un.transpose(3, 2, 0, 1))).shape, a4.transpose(3, 2, 0, 1).shape)
    packed4 = B.packVolume(a4).reshape(3, 6, 4, 5)
    assert np.array_equal(np.fliplr(un.transpose(3, 2, 0, 1)), packed4)


def test_pack_matches_layout(golden):
    B = BL.BROCCOLI_LIB()
    series = golden["mc_series"]
    packed = B.packVolume(to_wrapper_layout(series))
    assert np.array_equal(packed, series.reshape(-1))


@pytest.mark.gpu
def test_perform_motion_correction_matches_golden(golden, lin_filters):
    series = golden["mc_series"]
    filters = [to_wrapper_layout(lin_filters[k, 0]) + 1j * to_wrapper_layout(lin_filters[k, 1])
               for k in range(3)]
    corrected, motion = BL.performMotionCorrection(to_wrapper_layout(series), golden["mc_voxel"], filters, 5)
    gm = golden["mc_motion"]
    assert np.abs(motion[:3] - gm[:3]).max() < 1e-4 * max(1.0, np.abs(gm[:3]).max()) * golden["mc_voxel"].max()
    np.testing.assert_allclose(motion[3:], gm[3:], atol=2e-3)
    # undo unpackOutputVolume (transpose back, flip the second axis back)
    back = np.fliplr(corrected.transpose(3, 2, 0, 1))
    assert rel_err(back, golden["mc_corrected"]) < 1e-4


def test_fwhm_filters_match_oracle():
    """CreateSmoothingFilters from a FWHM: the wrapper's taps equal the
    oracle's restatement bit for bit."""
    import oracle as O
    vox = (3.0, 3.0, 3.5)
    fx, fy, fz = BL.fwhm_filters(6.0, vox)
    for f, v in zip((fx, fy, fz), vox):
        assert np.array_equal(f, O.smoothing_filter_sigma(6.0 / 2.354 / v))


@pytest.mark.gpu
def test_perform_smoothing_normalized_matches_golden():
    """PerformSmoothingNormalizedWrapper through the wrapper class (RANDOM
    filters = the fixture's taps) against the reference kernels' output."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "smooth_normalized.npz"))
    vols, mask, fs, ref = g["vols"], g["mask"], g["filter"], g["out"]
    B = BL.BROCCOLI_LIB(0, 0)
    B.SetfMRIData(to_wrapper_layout(vols), (3.0, 3.0, 3.0))
    B.SetEPIMask(B.packVolume(to_wrapper_layout(mask)))
    B.SetSmoothingType(BL.RANDOM)
    B.SetSmoothingFilters(fs, fs, fs)
    out = B.createOutputArray(to_wrapper_layout(vols).shape)
    B.SetOutputSmoothedfMRIVolumes(out)
    B.PerformSmoothingNormalizedWrapper()
    got = out.reshape(vols.shape)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = np.isfinite(ref)
    assert np.abs(got[fin] - ref[fin]).max() <= 1e-4 * np.abs(ref[fin]).max()


@pytest.mark.gpu
def test_perform_first_level_preprocessing_equals_library(bank):
    """firstlevel.py's preprocessing through the wrapper class (fMRI flipped
    up-down, template brain divided by its maximum, packVolume layouts)
    equals brc_first_level_preprocess on the same volumes."""
    import os
    from conftest import GOLDEN
    from test_first_level import cfg
    from broccoli_b200.api import Context
    fl = dict(np.load(os.path.join(GOLDEN, "first_level.npz")))
    c = cfg(fl)
    fmri, t1, mni = fl["in_fmri"], fl["in_t1"], fl["in_mni"]
    wrap3 = to_wrapper_layout
    filters = {k: [to_wrapper_layout(bank[k][i, 0]) + 1j * to_wrapper_layout(bank[k][i, 1])
                   for i in range(len(bank[k]))] for k in ("linear", "nonlinear")}
    # performFirstLevelAnalysis flips the fMRI data up-down before packing it
    r = BL.performFirstLevelPreprocessing(
        np.flipud(to_wrapper_layout(fmri)), c["epi_voxel"], wrap3(t1), c["t1_voxel"], wrap3(mni), c["mni_voxel"],
        filters["linear"], filters["nonlinear"], bank["projection_tensors"], list(bank["directions"]),
        c["lin_iter"], c["nl_iter"], c["motion_iter"], c["coarsest_t1_mni"], c["coarsest_epi_t1"], 0,
        c["smoothing_fwhm"])
    ctx = Context(0)
    want = ctx.first_level_preprocess(fmri, c["epi_voxel"], t1, c["t1_voxel"], mni / mni.max(), c["mni_voxel"],
                                      bank, c["lin_iter"], c["nl_iter"], c["motion_iter"], c["coarsest_t1_mni"],
                                      c["coarsest_epi_t1"], 0, smoothing_fwhm=c["smoothing_fwhm"])
    ctx.close()
    assert np.array_equal(r["T1_MNI_registration_parameters"], want["params_t1_mni"])
    assert np.array_equal(r["EPI_T1_registration_parameters"], want["params_epi_t1"])
    assert np.array_equal(r["EPI_MNI_registration_parameters"], want["params_epi_mni"])
    assert np.array_equal(r["motion_parameters"], want["motion_parameters"])
    assert np.array_equal(r["EPI_mask"], wrap3(want["epi_mask"]))
    assert np.array_equal(r["aligned_T1_volume"], wrap3(want["aligned_t1_linear"]))


@pytest.mark.gpu
@pytest.mark.parametrize("strip", ["mask", "original"])
def test_two_volumes_precenter_skull_strip_debug(golden, bank, strip):
    """The Python mirror's SetPrecenterRegistration, SetDoSkullstrip(Original)
    with SetInputMNIBrainMask / SetOutputSkullstrippedT1Volume, and SetDebug
    with three response arrays, against the reference kernels' fixtures
    (tests/golden/boundary.npz; 6 linear and 4 nonlinear iterations, coarsest
    scale 2, 3 mm z cut as there)."""
    import os
    import oracle
    from conftest import GOLDEN
    bd = dict(np.load(os.path.join(GOLDEN, "boundary.npz")))
    sub, tpl = golden["r2v_subject"], golden["r2v_template"]
    D, H, W = sub.shape
    D2, H2, W2 = tpl.shape
    B = BL.BROCCOLI_LIB(0, 0)
    B.SetT1Width(W), B.SetT1Height(H), B.SetT1Depth(D)
    vs = golden["r2v_voxel"]
    B.SetT1VoxelSizeX(vs[0]), B.SetT1VoxelSizeY(vs[1]), B.SetT1VoxelSizeZ(vs[2])
    B.SetMNIWidth(W2), B.SetMNIHeight(H2), B.SetMNIDepth(D2)
    B.SetInputT1Volume(np.ascontiguousarray(sub).reshape(-1))
    B.SetInputMNIBrainVolume(np.ascontiguousarray(tpl).reshape(-1))
    B.linear_filters = np.ascontiguousarray(bank["linear"], np.float32)
    B.nonlinear_filters = np.ascontiguousarray(bank["nonlinear"], np.float32)
    B.projection_tensors = np.asarray(bank["projection_tensors"], np.float32).reshape(6, 6)
    B.directions = np.asarray(bank["directions"], np.float32).reshape(3, 6)
    B.SetNumberOfIterationsForLinearImageRegistration(6)
    B.SetNumberOfIterationsForNonLinearImageRegistration(4)
    B.SetCoarsestScaleT1MNI(2)
    B.SetMMT1ZCUT(3)
    B.SetPrecenterRegistration(True)
    params = np.zeros(12, np.float32)
    nonlin = np.zeros(D2 * H2 * W2, np.float32)
    interp = np.zeros(D2 * H2 * W2, np.float32)
    skull = np.zeros(D2 * H2 * W2, np.float32)
    B.SetOutputT1MNIRegistrationParameters(params)
    B.SetOutputAlignedT1VolumeNonLinear(nonlin)
    B.SetOutputInterpolatedT1Volume(interp)
    B.SetInputMNIBrainMask(bd["r2v_mask"].reshape(-1))
    B.SetOutputSkullstrippedT1Volume(skull)
    B.SetDoSkullstrip(strip == "mask")
    B.SetDoSkullstripOriginal(strip == "original")
    q = [np.zeros(D2 * H2 * W2, np.complex64) for _ in range(3)]
    B.SetDebug(True)
    B.SetOutputQuadratureFilterResponses(*q)
    B.PerformRegistrationTwoVolumesWrapper()
    assert np.abs(params - bd["pc_params"]).max() < 1e-4 * max(1.0, np.abs(bd["pc_params"]).max())
    assert rel_err(nonlin.reshape(D2, H2, W2), bd["pc_aligned_nonlinear"]) < 1e-4
    mask = bd["r2v_mask"]
    if strip == "mask":
        assert np.array_equal(skull, nonlin * mask.reshape(-1))
    else:
        from broccoli_b200.api import Context
        back = oracle.transform_affine(mask, Context.invert_affine_parameters(params), interp=0)[0]
        assert np.array_equal(skull, interp * back.reshape(-1))
    qt = oracle.filter3d(tpl, bank["linear"])
    for k in range(3):
        assert rel_err(q[k].reshape(D2, H2, W2), qt[k]) < 1e-4
