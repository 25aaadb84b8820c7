"""Python mirror of BROCCOLI's Python wrapper for the registration path.

The reference's wrapper (code/Python_Wrapper/broccoli/broccoli_common.py:
55-200) subclasses the SWIG-bound C++ class; its helpers pack numpy volumes
(flipud, then transpose (2, 0, 1) so x is fastest) and its module functions
(motion_correction.py:4-73, registration.py) drive the class.  This module
keeps those names and conventions and runs the path through the C-ABI of
libbroccoli_b200 with host arrays (no torch needed).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

_pack_permutation = (2, 0, 1)
_pack_permutation_4d = (3, 2, 0, 1)

TRANSLATION, RIGID, AFFINE = 0, 1, 2
NEAREST, LINEAR, CUBIC = 0, 1, 2
LOWPASS, RANDOM = 0, 1  # smoothing types (broccoli_constants.h)


def _permute(permutation, array):
    return [array[permutation[i]] for i in range(len(array))]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class BROCCOLI_LIB:
    """Setter/wrapper interface of BROCCOLI_LIB for this path, on the C-ABI."""

    def __init__(self, *args):
        self._ctx = None
        self._initiated = False
        self._init_error = ""
        self._input_arrays = []
        self.epi = [0, 0, 0, 1]
        self.t1 = [0, 0, 0]
        self.t1_t = 1
        self.interpolation = LINEAR
        self.center_parameters = np.zeros(12, np.float32)
        self.mni = [0, 0, 0]
        self.epi_vox = [1.0, 1.0, 1.0]
        self.t1_vox = [1.0, 1.0, 1.0]
        self.mni_vox = [1.0, 1.0, 1.0]
        self.fmri = None
        self.t1_volume = None
        self.mni_volume = None
        self.linear_filters = None
        self.nonlinear_filters = None
        self.projection_tensors = np.zeros((6, 6), np.float32)
        self.directions = None
        self.it_linear, self.it_nonlinear, self.it_mc = 10, 10, 5
        self.coarsest = 4
        self.mm_z_cut = 0
        self.sigmas = [5.0, 5.0, 5.0]
        self.mc_tolerance = 0.0
        self.precision = L.PREC_FP32
        self.out = {}
        self.save = {}
        self.coarsest_epi_t1 = 4
        self.apply_mc, self.apply_smoothing, self.apply_slice_timing = True, True, False
        self.preprocessing_only = False
        if len(args) == 2:
            self.OpenCLInitiate(*args)

    # ---- runtime ----------------------------------------------------------

    def OpenCLInitiate(self, platform, device):
        """Binds a CUDA device (platform must be 0)."""
        if platform != 0:
            self._init_error = "platform must be 0"
            return False
        h = ctypes.c_void_p()
        s = L.lib().brc_ctx_create(int(device), ctypes.byref(h))
        if s != L.BRC_OK:
            self._init_error = L.status_string(s)
            return False
        self._ctx = h
        self._initiated = True
        return True

    def GetOpenCLInitiated(self):
        return 1 if self._initiated else 0

    def GetOpenCLInitializationError(self):
        return self._init_error

    def __del__(self):
        if getattr(self, "_ctx", None):
            L.lib().brc_ctx_destroy(self._ctx)
            self._ctx = None

    def _check(self, s):
        if s != L.BRC_OK:
            msg = L.lib().brc_last_error(self._ctx).decode() if self._ctx else ""
            raise L.BrcError(s, f"{L.status_string(s)}: {msg}")

    # ---- packing (broccoli_common.py:144-200) -----------------------------

    def packArray(self, array):
        return np.ascontiguousarray(array, dtype=np.float32)

    def packVolume(self, array):
        if len(array.shape) == 3:
            t = np.flipud(array).transpose(_pack_permutation)
        elif len(array.shape) == 4:
            t = np.flipud(array).transpose(_pack_permutation_4d)
        else:
            t = array
        t = self.packArray(t.flatten())
        self._input_arrays.append(t)
        return t

    def createOutputArray(self, shape, dtype=np.float32):
        return np.empty(shape=shape, dtype=dtype).flatten()

    def unpackOutputArray(self, array, shape):
        return array.reshape(shape)

    def unpackOutputVolume(self, array, shape=None):
        unpack = None
        if shape:
            if len(shape) == 3:
                t_shape = _permute(_pack_permutation, shape)
                unpack = np.argsort(_pack_permutation)
            elif len(shape) == 4:
                t_shape = _permute(_pack_permutation_4d, shape)
                unpack = np.argsort(_pack_permutation_4d)
            else:
                t_shape = shape
            array = self.unpackOutputArray(array, t_shape)
            array = np.fliplr(array)
        return array.transpose(unpack) if unpack is not None else array

    # ---- data setters (broccoli_common.py:75-127) --------------------------

    def SetEPIData(self, array, voxel_sizes):
        self.SetEPIHeight(array.shape[0])
        self.SetEPIWidth(array.shape[1])
        self.SetEPIDepth(array.shape[2])
        self.SetInputEPIVolume(self.packVolume(array))
        self.SetEPIVoxelSizeX(voxel_sizes[0])
        self.SetEPIVoxelSizeY(voxel_sizes[1])
        self.SetEPIVoxelSizeZ(voxel_sizes[2])

    def SetT1Data(self, array, voxel_sizes):
        self.SetT1Height(array.shape[0])
        self.SetT1Width(array.shape[1])
        self.SetT1Depth(array.shape[2])
        self.SetInputT1Volume(self.packVolume(array))
        self.SetT1VoxelSizeX(voxel_sizes[0])
        self.SetT1VoxelSizeY(voxel_sizes[1])
        self.SetT1VoxelSizeZ(voxel_sizes[2])

    def SetMNIData(self, array, voxel_sizes):
        self.SetMNIHeight(array.shape[0])
        self.SetMNIWidth(array.shape[1])
        self.SetMNIDepth(array.shape[2])
        self.SetInputMNIVolume(self.packVolume(array))
        self.SetMNIVoxelSizeX(voxel_sizes[0])
        self.SetMNIVoxelSizeY(voxel_sizes[1])
        self.SetMNIVoxelSizeZ(voxel_sizes[2])

    def SetfMRIData(self, array, voxel_sizes):
        self.SetEPIHeight(array.shape[0])
        self.SetEPIWidth(array.shape[1])
        self.SetEPIDepth(array.shape[2])
        self.SetEPITimepoints(array.shape[3])
        self.SetInputfMRIVolumes(self.packVolume(array))
        self.SetEPIVoxelSizeX(voxel_sizes[0])
        self.SetEPIVoxelSizeY(voxel_sizes[1])
        self.SetEPIVoxelSizeZ(voxel_sizes[2])

    def SetParametricImageRegistrationFilters(self, filters):
        """Three complex 7x7x7 arrays (linear registration)."""
        bank = np.zeros((3, 2, 7, 7, 7), np.float32)
        for i in range(3):
            bank[i, 0] = self.packVolume(np.real(filters[i])).reshape(7, 7, 7)
            bank[i, 1] = self.packVolume(np.imag(filters[i])).reshape(7, 7, 7)
        self.linear_filters = bank

    def SetNonParametricImageRegistrationFilters(self, filters):
        bank = np.zeros((6, 2, 7, 7, 7), np.float32)
        for i in range(6):
            bank[i, 0] = self.packVolume(np.real(filters[i])).reshape(7, 7, 7)
            bank[i, 1] = self.packVolume(np.imag(filters[i])).reshape(7, 7, 7)
        self.nonlinear_filters = bank

    def SetProjectionTensorMatrixFilters(self, filters):
        for k in range(6):
            self.projection_tensors[k] = np.asarray(filters[k], np.float32)

    def SetFilterDirections(self, x, y, z):
        self.directions = np.stack([np.asarray(a, np.float32).reshape(6) for a in (x, y, z)])

    # ---- raw setters with the C++ class's names ----------------------------

    def SetEPIWidth(self, w): self.epi[0] = int(w)
    def SetEPIHeight(self, h): self.epi[1] = int(h)
    def SetEPIDepth(self, d): self.epi[2] = int(d)
    def SetEPITimepoints(self, t): self.epi[3] = int(t)
    def SetEPIVoxelSizeX(self, v): self.epi_vox[0] = float(v)
    def SetEPIVoxelSizeY(self, v): self.epi_vox[1] = float(v)
    def SetEPIVoxelSizeZ(self, v): self.epi_vox[2] = float(v)
    def SetT1Width(self, w): self.t1[0] = int(w)
    def SetT1Height(self, h): self.t1[1] = int(h)
    def SetT1Depth(self, d): self.t1[2] = int(d)
    def SetT1VoxelSizeX(self, v): self.t1_vox[0] = float(v)
    def SetT1VoxelSizeY(self, v): self.t1_vox[1] = float(v)
    def SetT1VoxelSizeZ(self, v): self.t1_vox[2] = float(v)
    def SetMNIWidth(self, w): self.mni[0] = int(w)
    def SetMNIHeight(self, h): self.mni[1] = int(h)
    def SetMNIDepth(self, d): self.mni[2] = int(d)
    def SetMNIVoxelSizeX(self, v): self.mni_vox[0] = float(v)
    def SetMNIVoxelSizeY(self, v): self.mni_vox[1] = float(v)
    def SetMNIVoxelSizeZ(self, v): self.mni_vox[2] = float(v)
    def SetInputfMRIVolumes(self, a): self.fmri = a
    def SetInputEPIVolume(self, a): self.fmri = a
    def SetInputT1Volume(self, a): self.t1_volume = a
    def SetInputMNIVolume(self, a): self.mni_volume = a
    def SetInputMNIBrainVolume(self, a): self.mni_volume = a
    def SetImageRegistrationFilterSize(self, n):
        if int(n) != 7:
            raise ValueError("filter size must be 7")
    def SetNumberOfIterationsForLinearImageRegistration(self, n): self.it_linear = int(n)
    def SetNumberOfIterationsForParametricImageRegistration(self, n): self.it_linear = int(n)
    def SetNumberOfIterationsForNonLinearImageRegistration(self, n): self.it_nonlinear = int(n)
    def SetNumberOfIterationsForNonParametricImageRegistration(self, n): self.it_nonlinear = int(n)
    def SetNumberOfIterationsForMotionCorrection(self, n): self.it_mc = int(n)
    def SetCoarsestScaleT1MNI(self, n): self.coarsest = int(n)
    def SetCoarsestScaleEPIT1(self, n): self.coarsest_epi_t1 = int(n)
    def SetApplyMotionCorrection(self, b): self.apply_mc = bool(b)
    def SetApplySmoothing(self, b): self.apply_smoothing = bool(b)
    def SetApplySliceTimingCorrection(self, b): self.apply_slice_timing = bool(b)
    def SetPreprocessingOnly(self, b): self.preprocessing_only = bool(b)
    def SetOutputEPIT1RegistrationParameters(self, a): self.out["params_epi_t1"] = a
    def SetOutputEPIMNIRegistrationParameters(self, a): self.out["params_epi_mni"] = a
    def SetOutputAlignedEPIVolumeT1(self, a): self.out["aligned_epi_t1"] = a
    def SetOutputAlignedEPIVolumeMNILinear(self, a): self.out["aligned_epi_mni_linear"] = a
    def SetOutputAlignedEPIVolumeMNINonlinear(self, a): self.out["aligned_epi_mni_nonlinear"] = a
    def SetOutputEPIMask(self, a): self.out["epi_mask"] = a
    def SetSaveInterpolatedT1(self, b): self.save["interpolated_t1"] = bool(b)
    def SetSaveAlignedT1MNILinear(self, b): self.save["aligned_t1_linear"] = bool(b)
    def SetSaveAlignedT1MNINonLinear(self, b): self.save["aligned_t1_nonlinear"] = bool(b)
    def SetSaveAlignedEPIT1(self, b): self.save["aligned_epi_t1"] = bool(b)
    def SetSaveAlignedEPIMNI(self, b): self.save["aligned_epi_mni"] = bool(b)
    def SetSaveEPIMask(self, b): self.save["epi_mask"] = bool(b)
    def SetSaveMotionCorrected(self, b): self.save["motion_corrected"] = bool(b)
    def SetSaveSmoothed(self, b): self.save["smoothed"] = bool(b)
    def SetMMT1ZCUT(self, mm): self.mm_z_cut = int(mm)
    def SetInterpolationMode(self, mode):
        # the registration loops resample linearly whatever the mode (as the
        # reference's loops do); the transform wrappers take NEAREST or LINEAR
        if mode not in (NEAREST, LINEAR):
            raise ValueError("NEAREST or LINEAR interpolation (the reference's CUBIC kernels are not usable)")
        self.interpolation = int(mode)
    def SetT1Timepoints(self, t): self.t1_t = int(t)
    def SetTsigma(self, s): self.sigmas[0] = float(s)
    def SetEsigma(self, s): self.sigmas[1] = float(s)
    def SetDsigma(self, s): self.sigmas[2] = float(s)
    def SetMotionCorrectionTolerance(self, v): self.mc_tolerance = float(v)
    def SetPrecision(self, p): self.precision = int(p)
    def SetSolveFP64(self, b): self.solve_fp64 = bool(b)
    def SetPrecenterRegistration(self, b): self.precenter = bool(b)
    def SetDoSkullstrip(self, b): self.do_skullstrip = bool(b)
    def SetDoSkullstripOriginal(self, b): self.do_skullstrip_original = bool(b)
    def SetInputMNIBrainMask(self, a): self.mni_mask = a
    def SetOutputSkullstrippedT1Volume(self, a): self.out["skullstripped"] = a
    def SetDebug(self, b): self.debug = bool(b)
    def SetOutputQuadratureFilterResponses(self, *arrays):
        """Three arrays (the last linear call's reference responses) or six
        (the nonlinear reference's responses at the finest scale)."""
        if len(arrays) not in (3, 6):
            raise ValueError("SetOutputQuadratureFilterResponses takes 3 or 6 arrays")
        self.out["q"] = list(arrays)
    def SetOutputPhaseDifferences(self, a): self.out["phase_differences"] = a
    def SetOutputPhaseCertainties(self, a): self.out["phase_certainties"] = a
    def SetOutputPhaseGradients(self, a): self.out["phase_gradients"] = a

    def _debug_arrays(self, ctx):
        """Host arrays for the context's debug outputs when SetDebug(True):
        the caller's own arrays where they are contiguous of the right type,
        else staging arrays copied back by _debug_copy_back."""
        if not getattr(self, "debug", False):
            ctx.set_debug_outputs(None)
            return None
        stage = {}

        def host(a, dtype):
            if a is None:
                return None
            if isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous:
                return a
            t = np.zeros(np.asarray(a).size, dtype)
            stage[id(t)] = (t, a)
            return t
        outs = {"quadrature_responses": [host(a, np.complex64) for a in self.out.get("q", [])]}
        for k in ("phase_differences", "phase_certainties", "phase_gradients"):
            outs[k] = host(self.out.get(k), np.float32)
        ctx.set_debug_outputs(outs)
        return stage

    @staticmethod
    def _debug_copy_back(stage):
        for t, a in (stage or {}).values():
            a[...] = t.reshape(np.asarray(a).shape).astype(np.asarray(a).dtype)
    def SetOutputMotionParameters(self, a): self.out["motion"] = a
    def SetOutputMotionCorrectedfMRIVolumes(self, a): self.out["mc"] = a
    def SetOutputT1MNIRegistrationParameters(self, a): self.out["params"] = a
    def SetOutputAlignedT1VolumeLinear(self, a): self.out["aligned_linear"] = a
    def SetOutputAlignedT1VolumeNonLinear(self, a): self.out["aligned_nonlinear"] = a
    def SetOutputInterpolatedT1Volume(self, a): self.out["interpolated"] = a
    def SetOutputDisplacementField(self, x, y, z): self.out["field"] = (x, y, z)
    def SetOutputSmoothedfMRIVolumes(self, a): self.out["smoothed"] = a
    def SetEPISmoothingAmount(self, fwhm_mm): self.epi_fwhm = float(fwhm_mm)
    def SetSmoothingType(self, t): self.smoothing_type = int(t)
    def SetSmoothingFilters(self, fx, fy, fz):
        self.smoothing_filters = [np.ascontiguousarray(f, np.float32).reshape(9) for f in (fx, fy, fz)]
    def SetEPIMask(self, mask): self.epi_mask = mask  # packed like the volumes (packVolume)

    # ---- entry points -------------------------------------------------------

    def PerformMotionCorrectionWrapper(self):
        if getattr(self, "debug", False):
            return self._motion_correction_debug()
        W, H, D, T = self.epi
        vols = np.ascontiguousarray(self.fmri, np.float32)
        opts = L.LinearOpts()
        L.lib().brc_linear_opts_default(ctypes.byref(opts), self.it_mc)
        opts.type = RIGID
        opts.tolerance = self.mc_tolerance
        opts.precision = self.precision
        motion = np.zeros(6 * T, np.float32)
        vs = np.asarray(self.epi_vox, np.float32)
        bank = np.ascontiguousarray(self.linear_filters, np.float32)
        self._check(L.lib().brc_motion_correct(self._ctx, _ptr(vols), W, H, D, T, _ptr(vs), _ptr(bank),
                                               ctypes.byref(opts), None, _ptr(motion)))
        if self.fmri is not vols:
            self.fmri[...] = vols.reshape(self.fmri.shape)
        if "motion" in self.out:
            self.out["motion"][...] = motion.reshape(self.out["motion"].shape)
        if "mc" in self.out:
            self.out["mc"][...] = vols.reshape(self.out["mc"].shape)

    def _motion_correction_debug(self):
        """Motion correction through a Context, so that SetDebug's outputs
        are filled (the last volume's registration to volume 0)."""
        from .api import Context
        W, H, D, T = self.epi
        ctx = Context(0)
        stage = self._debug_arrays(ctx)
        vols = np.ascontiguousarray(self.fmri, np.float32).reshape(T, D, H, W)
        corrected, motion = ctx.motion_correct(vols, self.epi_vox, self.linear_filters, self.it_mc,
                                               precision=self.precision, tolerance=self.mc_tolerance)
        ctx.close()
        self._debug_copy_back(stage)
        self.fmri[...] = np.asarray(corrected, np.float32).reshape(self.fmri.shape)
        if "motion" in self.out:
            self.out["motion"][...] = np.asarray(motion, np.float32).reshape(self.out["motion"].shape)
        if "mc" in self.out:
            self.out["mc"][...] = np.asarray(corrected, np.float32).reshape(self.out["mc"].shape)

    def _smoothing_taps(self):
        if getattr(self, "smoothing_type", LOWPASS) == RANDOM:
            return self.smoothing_filters
        return fwhm_filters(getattr(self, "epi_fwhm", 0.0), self.epi_vox)

    def _smooth(self, normalized: bool):
        import torch
        from .api import Context
        W, H, D, T = self.epi
        ctx = Context(0)
        vols = torch.from_numpy(np.ascontiguousarray(self.fmri, np.float32).reshape(T, D, H, W)).cuda()
        fx, fy, fz = self._smoothing_taps()
        if normalized:
            mask = torch.from_numpy(np.ascontiguousarray(self.epi_mask, np.float32).reshape(D, H, W)).cuda()
            out = ctx.smooth_normalized(vols, mask, fx, fy, fz)
        else:
            out = ctx.smooth3d(vols, fx, fy, fz)
        if "smoothed" in self.out:
            self.out["smoothed"][...] = out.cpu().numpy().reshape(self.out["smoothed"].shape)
        ctx.close()

    def PerformSmoothingWrapper(self):
        """PerformSmoothingWrapper (broccoli_lib.cpp:11122-11210)."""
        self._smooth(False)

    def PerformSmoothingNormalizedWrapper(self):
        """PerformSmoothingNormalizedWrapper (broccoli_lib.cpp:11227-11272):
        the EPI mask is the certainty."""
        self._smooth(True)

    def PerformRegistrationTwoVolumesWrapper(self):
        import torch
        from .api import Context
        ctx = Context(0)
        W, H, D = self.t1
        W2, H2, D2 = self.mni
        sub = torch.from_numpy(np.ascontiguousarray(self.t1_volume, np.float32).reshape(D, H, W)).cuda()
        tpl = torch.from_numpy(np.ascontiguousarray(self.mni_volume, np.float32).reshape(D2, H2, W2)).cuda()
        bank = {"linear": self.linear_filters, "nonlinear": self.nonlinear_filters,
                "projection_tensors": self.projection_tensors, "directions": self.directions}
        nonlinear = self.it_nonlinear if self.nonlinear_filters is not None else 0
        strip = getattr(self, "do_skullstrip", False) or (getattr(self, "do_skullstrip_original", False) and
                                                            self.it_linear > 0)
        if strip and (getattr(self, "mni_mask", None) is None or "skullstripped" not in self.out):
            raise L.BrcError(L.BRC_ERR_INVALID, "PerformRegistrationTwoVolumesWrapper: skull strip needs "
                                                "SetInputMNIBrainMask and SetOutputSkullstrippedT1Volume")
        stage = self._debug_arrays(ctx)
        r = ctx.register_two_volumes(sub, self.t1_vox, tpl, self.mni_vox, bank, self.it_linear, nonlinear,
                                     self.coarsest, self.mm_z_cut, *self.sigmas,
                                     solve_fp64=getattr(self, "solve_fp64", False), precision=self.precision,
                                     precenter=getattr(self, "precenter", False))
        self._debug_copy_back(stage)
        if "params" in self.out:
            self.out["params"][: 12] = r["params"]
        for k in ("aligned_linear", "aligned_nonlinear", "interpolated"):
            if k in self.out:
                self.out[k][...] = r[k].cpu().numpy().reshape(self.out[k].shape)
        if "field" in self.out:
            f = r["field"].cpu().numpy()
            for a in range(3):
                self.out["field"][a][...] = f[a].reshape(self.out["field"][a].shape)
        if strip:
            # broccoli_lib.cpp:8064-8105: the aligned volume times the mask, or
            # the interpolated volume times the mask carried back (NEAREST)
            mask = torch.from_numpy(np.ascontiguousarray(self.mni_mask, np.float32).reshape(D2, H2, W2)).cuda()
            if getattr(self, "do_skullstrip", False):
                vol = (r["aligned_nonlinear"] if nonlinear > 0 else r["aligned_linear"]).clone()
            else:
                inv = Context.invert_affine_parameters(r["params"])
                mask = ctx.transform_volumes_linear(mask, inv, L.INTERP_NEAREST).reshape(D2, H2, W2).contiguous()
                vol = r["interpolated"].clone()
            ctx.multiply_volumes(vol, mask)
            self.out["skullstripped"][...] = vol.cpu().numpy().reshape(self.out["skullstripped"].shape)
        ctx.close()

    def PerformFirstLevelAnalysisWrapper(self):
        """The preprocessing of PerformFirstLevelAnalysisWrapper
        (broccoli_lib.cpp:8466-8733) on brc_first_level_preprocess: the
        fMRI volumes are replaced by the preprocessed series; the parameter
        vectors and motion parameters are written always, the volumes when
        their SetSave* flag is on.  The statistics are not part of this
        library (SetPreprocessingOnly(True) is required) and slice-timing
        correction must be off."""
        from .api import Context
        if not self.preprocessing_only:
            raise L.BrcError(L.BRC_ERR_UNSUPPORTED, "PerformFirstLevelAnalysisWrapper: the statistical analysis "
                                                    "is not part of this library; call SetPreprocessingOnly(True)")
        if self.apply_slice_timing:
            raise L.BrcError(L.BRC_ERR_UNSUPPORTED,
                             "PerformFirstLevelAnalysisWrapper: slice-timing correction is not supported")
        W, H, D, T = self.epi
        W2, H2, D2 = self.t1
        W3, H3, D3 = self.mni
        ctx = Context(0)
        bank = {"linear": self.linear_filters, "nonlinear": self.nonlinear_filters,
                "projection_tensors": self.projection_tensors, "directions": self.directions}
        r = ctx.first_level_preprocess(
            np.asarray(self.fmri, np.float32).reshape(T, D, H, W), self.epi_vox,
            np.asarray(self.t1_volume, np.float32).reshape(D2, H2, W2), self.t1_vox,
            np.asarray(self.mni_volume, np.float32).reshape(D3, H3, W3), self.mni_vox, bank, self.it_linear,
            self.it_nonlinear, self.it_mc, self.coarsest, self.coarsest_epi_t1, self.mm_z_cut, self.apply_mc,
            self.apply_smoothing, getattr(self, "epi_fwhm", 8.0), *self.sigmas, precision=self.precision)
        ctx.close()
        self.fmri[...] = r["fmri"].reshape(self.fmri.shape)
        written = {"params": "params_t1_mni", "params_epi_t1": "params_epi_t1", "params_epi_mni": "params_epi_mni"}
        if self.apply_mc:
            written["motion"] = "motion_parameters"
        flags = {"interpolated": ("interpolated_t1", "interpolated_t1"),
                 "aligned_linear": ("aligned_t1_linear", "aligned_t1_linear"),
                 "aligned_nonlinear": ("aligned_t1_nonlinear", "aligned_t1_nonlinear"),
                 "aligned_epi_t1": ("aligned_epi_t1", "aligned_epi_t1"),
                 "aligned_epi_mni_linear": ("aligned_epi_mni", "aligned_epi_mni_linear"),
                 "aligned_epi_mni_nonlinear": ("aligned_epi_mni", "aligned_epi_mni_nonlinear"),
                 "epi_mask": ("epi_mask", "epi_mask"), "mc": ("motion_corrected", "motion_corrected"),
                 "smoothed": ("smoothed", "smoothed")}
        for k, (flag, key) in flags.items():
            if self.save.get(flag, False):
                written[k] = key
        for k, key in written.items():
            if k in self.out:
                dst = self.out[k]
                dst[...] = np.asarray(r[key], np.float32).reshape(-1)[: dst.size].reshape(dst.shape)

    # ---- 4D transforms (TransformVolumesLinear/NonLinearWrapper,
    # CenterVolumesWrapper, broccoli_lib.cpp:8145-8245) ------------------------

    def _t1_volumes(self, ctx):
        import torch
        W, H, D = self.t1
        a = np.ascontiguousarray(self.t1_volume, np.float32).reshape(self.t1_t, D, H, W)
        return torch.from_numpy(a).cuda()

    def _t1_to_mni(self, ctx, vols):
        W2, H2, D2 = self.mni
        return ctx.change_resolution_and_size_batch(vols, self.t1_vox, (D2, H2, W2), self.mni_vox, self.mm_z_cut,
                                                    self.interpolation)

    def TransformVolumesLinearWrapper(self):
        """The T1 volumes resampled onto the MNI grid, then transformed by the
        parameters of SetOutputT1MNIRegistrationParameters; result in the
        array of SetOutputInterpolatedT1Volume."""
        from .api import Context
        ctx = Context(0)
        mni = self._t1_to_mni(ctx, self._t1_volumes(ctx))
        out = ctx.transform_volumes_linear(mni, np.asarray(self.out["params"], np.float32)[:12], self.interpolation)
        self.out["interpolated"][...] = out.cpu().numpy().reshape(self.out["interpolated"].shape)
        ctx.close()

    def TransformVolumesNonLinearWrapper(self):
        """As TransformVolumesLinearWrapper with the displacement field of
        SetOutputDisplacementField."""
        import torch
        from .api import Context
        ctx = Context(0)
        W2, H2, D2 = self.mni
        mni = self._t1_to_mni(ctx, self._t1_volumes(ctx))
        f = [torch.from_numpy(np.ascontiguousarray(a, np.float32).reshape(D2, H2, W2)).cuda()
             for a in self.out["field"]]
        out = ctx.transform_volumes_nonlinear(mni, *f, interpolation=self.interpolation)
        self.out["interpolated"][...] = out.cpu().numpy().reshape(self.out["interpolated"].shape)
        ctx.close()

    def CenterVolumesWrapper(self):
        """The T1 volumes centred by the first one's centre of mass (T1 size)."""
        from .api import Context
        ctx = Context(0)
        out, p = ctx.center_volumes(self._t1_volumes(ctx), self.interpolation)
        self.center_parameters[:] = p
        self.out["interpolated"][...] = out.cpu().numpy().reshape(self.out["interpolated"].shape)
        ctx.close()


def fwhm_filters(fwhm_mm: float, voxel_sizes):
    """9-tap Gaussians for a FWHM in mm along x, y, z: sigma = FWHM / 2.354 /
    voxel size, weights exp(-u^2 / 2 sigma^2) in double, stored float and
    normalised by their float sum (CreateSmoothingFilters,
    broccoli_lib.cpp:11093-11121)."""
    out = []
    for a in range(3):
        sigma = float(fwhm_mm) / 2.354 / float(voxel_sizes[a])
        u = np.arange(9, dtype=np.float64) - 4
        f = np.exp(-(u ** 2) / (2.0 * sigma * sigma)).astype(np.float32)
        s = np.float32(0)
        for v in f:
            s = np.float32(s + v)
        out.append((f / s).astype(np.float32))
    return out


def performSmoothingNormalized(h_fMRI_Volumes, h_EPI_Mask, h_fMRI_Voxel_Sizes, fwhm_mm,
                               OPENCL_PLATFORM=0, OPENCL_DEVICE=0):
    """Normalised-convolution smoothing of an fMRI series with a mask
    (PerformSmoothingNormalizedWrapper) through the wrapper class.  Returns
    the smoothed volumes in the wrapper's output layout."""
    B = BROCCOLI_LIB(OPENCL_PLATFORM, OPENCL_DEVICE)
    if not B.GetOpenCLInitiated():
        raise RuntimeError("initialisation failed: " + B.GetOpenCLInitializationError())
    shape = h_fMRI_Volumes.shape
    B.SetfMRIData(h_fMRI_Volumes, h_fMRI_Voxel_Sizes)
    B.SetEPIMask(B.packVolume(h_EPI_Mask))
    B.SetEPISmoothingAmount(fwhm_mm)
    B.SetSmoothingType(LOWPASS)
    out = B.createOutputArray(shape)
    B.SetOutputSmoothedfMRIVolumes(out)
    B.PerformSmoothingNormalizedWrapper()
    return B.unpackOutputVolume(out, shape)


def performMotionCorrection(h_fMRI_Volumes, h_fMRI_Voxel_Sizes, h_Quadrature_Filters, iterations,
                            OPENCL_PLATFORM=0, OPENCL_DEVICE=0):
    """motion_correction.py:performMotionCorrection on the C-ABI.  Returns
    (corrected volumes, motion parameters (6, T))."""
    B = BROCCOLI_LIB(OPENCL_PLATFORM, OPENCL_DEVICE)
    if not B.GetOpenCLInitiated():
        raise RuntimeError("initialisation failed: " + B.GetOpenCLInitializationError())
    shape = h_fMRI_Volumes.shape
    T = shape[3]
    B.SetfMRIData(h_fMRI_Volumes, h_fMRI_Voxel_Sizes)
    B.SetImageRegistrationFilterSize(len(h_Quadrature_Filters[0]))
    B.SetParametricImageRegistrationFilters(h_Quadrature_Filters)
    B.SetNumberOfIterationsForMotionCorrection(iterations)
    corrected = B.createOutputArray(shape)
    B.SetOutputMotionCorrectedfMRIVolumes(corrected)
    motion = B.createOutputArray((6, T))
    B.SetOutputMotionParameters(motion)
    B.PerformMotionCorrectionWrapper()
    return B.unpackOutputVolume(corrected, shape), B.unpackOutputArray(motion, (6, T))


def performFirstLevelPreprocessing(fMRI_data, fMRI_voxel_sizes, T1_data, T1_voxel_sizes, MNI_brain_data,
                                   MNI_voxel_sizes, parametric_filters, nonparametric_filters, projection_tensor,
                                   filter_directions, iterations_parametric, iterations_nonparametric,
                                   iterations_motion_correction, coarsest_scale_T1_MNI, coarsest_scale_EPI_T1,
                                   mm_T1_z_cut, EPI_smoothing, opencl_platform=0, opencl_device=0):
    """The registration, motion-correction and smoothing stages of
    firstlevel.py:performFirstLevelAnalysis (Python_Wrapper/broccoli/
    firstlevel.py:21-181) through the wrapper class with
    SetPreprocessingOnly(True): the same packing (fMRI flipped up-down, the
    template brain divided by its maximum) and parameter setters.  Returns a
    dict: T1_MNI_registration_parameters, EPI_T1_registration_parameters,
    EPI_MNI_registration_parameters, motion_parameters (6, T),
    motion_corrected_fMRI_data, smoothed_fMRI_data, EPI_mask,
    aligned_T1_volume, aligned_T1_volume_nonparametric and
    aligned_EPI_volume (template space, linear)."""
    B = BROCCOLI_LIB(opencl_platform, opencl_device)
    if not B.GetOpenCLInitiated():
        raise RuntimeError("initialisation failed: " + B.GetOpenCLInitializationError())
    fMRI_data = np.flipud(fMRI_data)
    MNI_brain_data = MNI_brain_data / MNI_brain_data.max()
    B.SetfMRIData(fMRI_data, fMRI_voxel_sizes)
    B.SetT1Data(T1_data, T1_voxel_sizes)
    B.SetMNIData(MNI_brain_data, MNI_voxel_sizes)
    B.SetInputMNIBrainVolume(B.packVolume(MNI_brain_data))
    B.SetNumberOfIterationsForParametricImageRegistration(iterations_parametric)
    B.SetNumberOfIterationsForNonParametricImageRegistration(iterations_nonparametric)
    B.SetImageRegistrationFilterSize(parametric_filters[0][0].shape[0])
    B.SetParametricImageRegistrationFilters(parametric_filters)
    B.SetNonParametricImageRegistrationFilters(nonparametric_filters)
    B.SetProjectionTensorMatrixFilters(projection_tensor)
    B.SetFilterDirections(*[B.packArray(f) for f in filter_directions])
    B.SetNumberOfIterationsForMotionCorrection(iterations_motion_correction)
    B.SetCoarsestScaleT1MNI(coarsest_scale_T1_MNI)
    B.SetCoarsestScaleEPIT1(coarsest_scale_EPI_T1)
    B.SetMMT1ZCUT(mm_T1_z_cut)
    B.SetEPISmoothingAmount(EPI_smoothing)
    B.SetPreprocessingOnly(True)
    T = fMRI_data.shape[3]
    r = {"T1_MNI_registration_parameters": B.createOutputArray(12),
         "EPI_T1_registration_parameters": B.createOutputArray(12),
         "EPI_MNI_registration_parameters": B.createOutputArray(12),
         "motion_parameters": B.createOutputArray(6 * T),
         "motion_corrected_fMRI_data": B.createOutputArray(fMRI_data.shape),
         "smoothed_fMRI_data": B.createOutputArray(fMRI_data.shape),
         "EPI_mask": B.createOutputArray(fMRI_data.shape[0:3]),
         "aligned_T1_volume": B.createOutputArray(MNI_brain_data.shape),
         "aligned_T1_volume_nonparametric": B.createOutputArray(MNI_brain_data.shape),
         "aligned_EPI_volume": B.createOutputArray(MNI_brain_data.shape)}
    B.SetOutputT1MNIRegistrationParameters(r["T1_MNI_registration_parameters"])
    B.SetOutputEPIT1RegistrationParameters(r["EPI_T1_registration_parameters"])
    B.SetOutputEPIMNIRegistrationParameters(r["EPI_MNI_registration_parameters"])
    B.SetOutputMotionParameters(r["motion_parameters"])
    B.SetOutputMotionCorrectedfMRIVolumes(r["motion_corrected_fMRI_data"])
    B.SetOutputSmoothedfMRIVolumes(r["smoothed_fMRI_data"])
    B.SetOutputEPIMask(r["EPI_mask"])
    B.SetOutputAlignedT1VolumeLinear(r["aligned_T1_volume"])
    B.SetOutputAlignedT1VolumeNonLinear(r["aligned_T1_volume_nonparametric"])
    B.SetOutputAlignedEPIVolumeMNILinear(r["aligned_EPI_volume"])
    for save in (B.SetSaveMotionCorrected, B.SetSaveSmoothed, B.SetSaveEPIMask, B.SetSaveAlignedT1MNILinear,
                 B.SetSaveAlignedT1MNINonLinear, B.SetSaveAlignedEPIMNI):
        save(True)
    B.PerformFirstLevelAnalysisWrapper()
    r["motion_parameters"] = B.unpackOutputArray(r["motion_parameters"], (6, T))
    for k in ("motion_corrected_fMRI_data", "smoothed_fMRI_data"):
        r[k] = B.unpackOutputVolume(r[k], fMRI_data.shape)
    r["EPI_mask"] = B.unpackOutputVolume(r["EPI_mask"], fMRI_data.shape[0:3])
    for k in ("aligned_T1_volume", "aligned_T1_volume_nonparametric", "aligned_EPI_volume"):
        r[k] = B.unpackOutputVolume(r[k], MNI_brain_data.shape)
    return r
