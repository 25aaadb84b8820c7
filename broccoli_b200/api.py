"""Torch-facing wrappers over the C-ABI.

Device memory and streams come from torch (plumbing only); every operation
runs in libbroccoli_b200's sm_100a kernels.  Volumes are float32 tensors
shaped (D, H, W) or batches (B, D, H, W), x fastest in memory as in the
reference.  Filter banks are numpy/torch arrays shaped (nfilt, 2, 7, 7, 7)
(filter, re/im, z, y, x).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L


def _check(ctx: "Context", status: int) -> None:
    if status != L.BRC_OK:
        msg = L.lib().brc_last_error(ctx.handle).decode() if ctx is not None else ""
        raise L.BrcError(status, f"{L.status_string(status)}: {msg}")


def _host_filters(filters) -> np.ndarray:
    f = filters.detach().cpu().numpy() if isinstance(filters, torch.Tensor) else np.asarray(filters)
    f = np.ascontiguousarray(f, dtype=np.float32)
    if f.ndim != 5 or f.shape[1:] != (2, 7, 7, 7):
        raise ValueError("filter bank must have shape (nfilt, 2, 7, 7, 7)")
    return f


def _vol_batch(t: torch.Tensor):
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
        raise TypeError("volumes must be float32 CUDA tensors")
    if t.dim() == 3:
        t = t.unsqueeze(0)
    if t.dim() != 4:
        raise ValueError("volumes must be (D,H,W) or (B,D,H,W)")
    return t.contiguous()


def _p(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """A library context bound to one CUDA device.  Work is queued on torch's
    current stream of that device at call time."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        s = L.lib().brc_ctx_create(device, ctypes.byref(h))
        if s != L.BRC_OK:
            raise L.BrcError(s, f"brc_ctx_create({device}): {L.status_string(s)}")
        self.handle = h
        self.device = device

    def close(self) -> None:
        if self.handle:
            L.lib().brc_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _bind_stream(self) -> None:
        # torch's default stream is the legacy NULL stream (handle 0), which
        # the C-ABI takes as NULL; other torch streams pass their handle.
        st = torch.cuda.current_stream(self.device).cuda_stream
        _check(self, L.lib().brc_ctx_set_stream(self.handle, ctypes.c_void_p(st) if st else None))

    @property
    def kernel_launches(self) -> int:
        return int(L.lib().brc_ctx_kernel_launches(self.handle))

    @property
    def workspace_bytes(self) -> int:
        return int(L.lib().brc_ctx_workspace_bytes(self.handle))

    def synchronize(self) -> None:
        """Waits for the context's work; raises if a bounded device-side
        wait of a tensor-core kernel gave up since the last check."""
        self._bind_stream()
        _check(self, L.lib().brc_ctx_synchronize(self.handle))

    def selftest_bounded_wait(self, wait_ms: int = 50) -> None:
        """Queues the self-test of the device-side bounded wait: the next
        synchronize() raises a timeout error, after which the context is
        usable again."""
        self._bind_stream()
        _check(self, L.lib().brc_selftest_bounded_wait(self.handle, int(wait_ms)))

    def phase_atan2(self, y: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
        """The arctangent of the phase kernels, element-wise on two float32
        device tensors of one shape."""
        for t in (y, x):
            if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
                raise TypeError("phase_atan2: float32 CUDA tensors")
        if y.shape != x.shape:
            raise ValueError("phase_atan2: y and x differ in shape")
        y, x = y.contiguous(), x.contiguous()
        out = torch.empty_like(y)
        self._bind_stream()
        _check(self, L.lib().brc_selftest_phase_atan2(self.handle, _p(y), _p(x), _p(out), y.numel()))
        return out

    # ---- kernels ---------------------------------------------------------

    def filter3d(self, vol: torch.Tensor, filters, precision: int = L.PREC_FP32) -> torch.Tensor:
        """Complex responses (B, nfilt, D, H, W) of the 7^3 filter bank."""
        v = _vol_batch(vol)
        f = _host_filters(filters)
        B, D, H, W = v.shape
        out = torch.empty((B, f.shape[0], D, H, W, 2), dtype=torch.float32, device=v.device)
        self._bind_stream()
        _check(self, L.lib().brc_filter3d(self.handle, _p(v), W, H, D, B, D * H * W,
                                          f.ctypes.data_as(ctypes.c_void_p), f.shape[0], precision,
                                          _p(out)))
        return torch.view_as_complex(out)

    def normal_equations(self, q1: torch.Tensor, q2: torch.Tensor):
        """A (B,12,12) and h (B,12) in float64 from reference responses q1
        ((3,D,H,W) shared, or (B,3,D,H,W)) and aligned responses q2
        (B,3,D,H,W) (complex64)."""
        if q2.dim() == 4:
            q2 = q2.unsqueeze(0)
        B, nf, D, H, W = q2.shape
        shared = q1.dim() == 4
        a = torch.view_as_real(q1.contiguous()).contiguous()
        c = torch.view_as_real(q2.contiguous()).contiguous()
        A = torch.empty((B, 12, 12), dtype=torch.float64, device=q2.device)
        h = torch.empty((B, 12), dtype=torch.float64, device=q2.device)
        self._bind_stream()
        _check(self, L.lib().brc_normal_equations(self.handle, _p(a), 0 if shared else 6 * D * H * W,
                                                  _p(c), W, H, D, B, _p(A), _p(h)))
        return A.transpose(1, 2), h

    def solve(self, A: torch.Tensor, h: torch.Tensor) -> torch.Tensor:
        if A.dim() == 2:
            A, h = A.unsqueeze(0), h.unsqueeze(0)
        Acm = A.transpose(1, 2).contiguous().to(torch.float64)
        hv = h.contiguous().to(torch.float64)
        p = torch.empty((A.shape[0], 12), dtype=torch.float32, device=A.device)
        self._bind_stream()
        _check(self, L.lib().brc_solve_affine_fp64(self.handle, _p(Acm), _p(hv), A.shape[0], _p(p)))
        return p

    def warp_affine(self, src: torch.Tensor, params: torch.Tensor) -> torch.Tensor:
        v = _vol_batch(src)
        B, D, H, W = v.shape
        p = params.reshape(B, 12).contiguous().to(torch.float32)
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_warp_affine(self.handle, _p(v), W, H, D, B, _p(p), _p(out)))
        return out

    def warp_field(self, src: torch.Tensor, dx, dy, dz) -> torch.Tensor:
        v = src.contiguous()
        D, H, W = v.shape
        fx, fy, fz = (t.contiguous().to(torch.float32) for t in (dx, dy, dz))
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_warp_field(self.handle, _p(v), W, H, D, _p(fx), _p(fy), _p(fz), _p(out)))
        return out

    def smooth3d(self, vol: torch.Tensor, fx, fy, fz, cert=None, smoothed_cert=None) -> torch.Tensor:
        v = _vol_batch(vol)
        B, D, H, W = v.shape
        taps = [np.ascontiguousarray(np.asarray(f, np.float32).reshape(9)) for f in (fx, fy, fz)]
        out = torch.empty_like(v)
        c = cert.contiguous() if cert is not None else None
        sc = smoothed_cert.contiguous() if smoothed_cert is not None else None
        self._bind_stream()
        _check(self, L.lib().brc_smooth3d(self.handle, _p(v), W, H, D, B,
                                          *[t.ctypes.data_as(ctypes.c_void_p) for t in taps],
                                          _p(c) if c is not None else None,
                                          _p(sc) if sc is not None else None, _p(out)))
        return out if vol.dim() == 4 else out[0]

    def smooth_normalized(self, vols: torch.Tensor, mask: torch.Tensor, fx, fy, fz) -> torch.Tensor:
        """Normalised-convolution smoothing of vols (T,D,H,W) or (D,H,W) with
        the certainty `mask` (D,H,W); NaN where the smoothed mask is 0, as in
        the reference."""
        v = _vol_batch(vols)
        T, D, H, W = v.shape
        m = mask.contiguous()
        taps = [np.ascontiguousarray(np.asarray(f, np.float32).reshape(9)) for f in (fx, fy, fz)]
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_smooth_normalized(self.handle, _p(v), W, H, D, T, _p(m),
                                                   *[t.ctypes.data_as(ctypes.c_void_p) for t in taps], _p(out)))
        return out if vols.dim() == 4 else out[0]

    def rescale_linear(self, src: torch.Tensor, shape) -> torch.Tensor:
        v = src.contiguous()
        D, H, W = v.shape
        D2, H2, W2 = shape
        out = torch.empty((D2, H2, W2), dtype=torch.float32, device=v.device)
        self._bind_stream()
        _check(self, L.lib().brc_rescale_linear(self.handle, _p(v), W, H, D, _p(out), W2, H2, D2))
        return out

    # ---- whole path ------------------------------------------------------

    def register_linear(self, ref: torch.Tensor, moving: torch.Tensor, filters, iterations: int,
                        type_: int = L.AFFINE, tolerance: float = 0.0, use_graph: bool = True,
                        precision: int = L.PREC_FP32, certainty_sigma: float = 0.0):
        """Batched single-scale registration of moving (B,D,H,W) onto ref
        ((D,H,W) shared or (B,D,H,W)).  Returns dict with params (B,12),
        aligned (B,D,H,W), rotations (B,3) and iterations (B,)."""
        m = _vol_batch(moving)
        B, D, H, W = m.shape
        r = ref.contiguous()
        ref_stride = 0 if r.dim() == 3 else D * H * W
        f = _host_filters(filters)
        if f.shape[0] != 3:
            raise ValueError("linear registration uses 3 filters")
        opts = L.LinearOpts()
        L.lib().brc_linear_opts_default(ctypes.byref(opts), iterations)
        opts.type = type_
        opts.tolerance = tolerance
        opts.use_graph = 1 if use_graph else 0
        opts.precision = precision
        opts.certainty_sigma_x100 = int(round(certainty_sigma * 100))
        params = torch.empty((B, 12), dtype=torch.float32, device=m.device)
        aligned = torch.empty_like(m)
        rot = torch.empty((B, 3), dtype=torch.float32, device=m.device)
        iters = torch.empty((B,), dtype=torch.int32, device=m.device)
        self._bind_stream()
        _check(self, L.lib().brc_register_linear_batched(
            self.handle, _p(r), ref_stride, _p(m), W, H, D, B, f.ctypes.data_as(ctypes.c_void_p),
            ctypes.byref(opts), _p(params), _p(aligned), _p(rot), _p(iters)))
        return {"params": params, "aligned": aligned, "rotations": rot, "iterations": iters}

    def register_linear_scales(self, ref: torch.Tensor, moving: torch.Tensor, filters, iterations: int,
                               coarsest_scale: int, type_: int = L.AFFINE):
        """Multi-scale linear registration of moving (B,D,H,W) onto a shared
        ref (D,H,W).  Returns dict with params (B,12), aligned (B,D,H,W) and
        rotations (B,3)."""
        m = _vol_batch(moving)
        B, D, H, W = m.shape
        r = ref.contiguous()
        f = _host_filters(filters)
        opts = L.LinearOpts()
        L.lib().brc_linear_opts_default(ctypes.byref(opts), iterations)
        opts.type = type_
        params = torch.empty((B, 12), dtype=torch.float32, device=m.device)
        aligned = torch.empty_like(m)
        rot = torch.empty((B, 3), dtype=torch.float32, device=m.device)
        self._bind_stream()
        _check(self, L.lib().brc_register_linear_scales(
            self.handle, _p(r), _p(m), W, H, D, B, f.ctypes.data_as(ctypes.c_void_p), ctypes.byref(opts),
            coarsest_scale, _p(params), _p(aligned), _p(rot)))
        return {"params": params, "aligned": aligned, "rotations": rot}

    @staticmethod
    def _nl_consts(bank: dict):
        f6 = np.ascontiguousarray(bank["nonlinear"], np.float32)
        m = np.ascontiguousarray(bank["projection_tensors"], np.float32)
        d = np.ascontiguousarray(bank["directions"], np.float32)
        return f6, m, d

    def nonlinear_step(self, q1: torch.Tensor, q2: torch.Tensor, bank: dict, field: torch.Tensor,
                       tsigma=5.0, esigma=5.0, dsigma=5.0, solve_fp64: bool = False) -> torch.Tensor:
        """Adds one nonlinear update computed from responses q1, q2 (6,D,H,W
        complex64) to `field` (3,D,H,W float32, in place)."""
        _, D, H, W = q2.shape
        a = torch.view_as_real(q1.contiguous()).contiguous()
        c = torch.view_as_real(q2.contiguous()).contiguous()
        _, m, d = self._nl_consts(bank)
        self._bind_stream()
        _check(self, L.lib().brc_nonlinear_step(self.handle, _p(a), _p(c), W, H, D,
                                                m.ctypes.data_as(ctypes.c_void_p),
                                                d.ctypes.data_as(ctypes.c_void_p), tsigma, esigma, dsigma,
                                                1 if solve_fp64 else 0, _p(field)))
        return field

    def register_nonlinear(self, ref: torch.Tensor, moving: torch.Tensor, bank: dict, iterations: int,
                           coarsest_scale: int = 1, tsigma=5.0, esigma=5.0, dsigma=5.0,
                           solve_fp64: bool = False, precision: int = L.PREC_FP32):
        """Multi-scale nonlinear registration.  Returns (field (3,D,H,W),
        aligned (D,H,W))."""
        r = ref.contiguous()
        m = moving.contiguous()
        D, H, W = m.shape
        f6, mt, d = self._nl_consts(bank)
        o = L.NonlinearOpts()
        L.lib().brc_nonlinear_opts_default(ctypes.byref(o), iterations)
        o.coarsest_scale = coarsest_scale
        o.tsigma, o.esigma, o.dsigma = tsigma, esigma, dsigma
        o.solve_fp64 = 1 if solve_fp64 else 0
        o.precision = precision
        field = torch.empty((3, D, H, W), dtype=torch.float32, device=m.device)
        aligned = torch.empty_like(m)
        self._bind_stream()
        _check(self, L.lib().brc_register_nonlinear(self.handle, _p(r), _p(m), W, H, D,
                                                    f6.ctypes.data_as(ctypes.c_void_p),
                                                    mt.ctypes.data_as(ctypes.c_void_p),
                                                    d.ctypes.data_as(ctypes.c_void_p), ctypes.byref(o),
                                                    _p(field), _p(aligned)))
        return field, aligned

    def change_resolution_and_size(self, src: torch.Tensor, voxel_size, shape, new_voxel_size,
                                   mm_z_cut: int = 0) -> torch.Tensor:
        v = src.contiguous()
        D, H, W = v.shape
        D2, H2, W2 = shape
        out = torch.empty((D2, H2, W2), dtype=torch.float32, device=v.device)
        vs = np.ascontiguousarray(voxel_size, np.float32)
        nvs = np.ascontiguousarray(new_voxel_size, np.float32)
        self._bind_stream()
        _check(self, L.lib().brc_change_resolution_and_size(
            self.handle, _p(v), W, H, D, vs.ctypes.data_as(ctypes.c_void_p), _p(out), W2, H2, D2,
            nvs.ctypes.data_as(ctypes.c_void_p), mm_z_cut))
        return out

    # ---- 4D transforms (NEAREST = 0, LINEAR = 1) ------------------------------

    @staticmethod
    def _vols4(t: torch.Tensor) -> torch.Tensor:
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
            raise TypeError("volumes must be float32 CUDA tensors")
        if t.dim() == 3:
            t = t.unsqueeze(0)
        if t.dim() != 4:
            raise ValueError("volumes must be (D,H,W) or (T,D,H,W)")
        return t.contiguous()

    def change_resolution_and_size_batch(self, src: torch.Tensor, voxel_size, shape, new_voxel_size,
                                         mm_z_cut: int = 0, interpolation: int = L.INTERP_LINEAR) -> torch.Tensor:
        """ChangeVolumesResolutionAndSize of (T, D, H, W) volumes onto a
        (D2, H2, W2) grid; returns (T, D2, H2, W2)."""
        v = self._vols4(src)
        T, D, H, W = v.shape
        D2, H2, W2 = shape
        out = torch.empty((T, D2, H2, W2), dtype=torch.float32, device=v.device)
        vs = np.ascontiguousarray(voxel_size, np.float32)
        nvs = np.ascontiguousarray(new_voxel_size, np.float32)
        self._bind_stream()
        _check(self, L.lib().brc_change_resolution_and_size_batch(
            self.handle, _p(v), W, H, D, T, vs.ctypes.data_as(ctypes.c_void_p), _p(out), W2, H2, D2,
            nvs.ctypes.data_as(ctypes.c_void_p), int(mm_z_cut), int(interpolation)))
        return out

    def transform_volumes_linear(self, src: torch.Tensor, params,
                                 interpolation: int = L.INTERP_LINEAR) -> torch.Tensor:
        """TransformVolumesLinear: one 12-parameter vector applied to every
        volume of (T, D, H, W)."""
        v = self._vols4(src)
        T, D, H, W = v.shape
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(12))
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_transform_volumes_linear(self.handle, _p(v), W, H, D, T,
                                                          p.ctypes.data_as(ctypes.c_void_p), int(interpolation),
                                                          _p(out)))
        return out

    def transform_volumes_nonlinear(self, src: torch.Tensor, dx, dy, dz,
                                    interpolation: int = L.INTERP_LINEAR) -> torch.Tensor:
        """TransformVolumesNonLinear: one displacement field (voxels) applied
        to every volume of (T, D, H, W)."""
        v = self._vols4(src)
        T, D, H, W = v.shape
        fx, fy, fz = (f.contiguous().to(torch.float32) for f in (dx, dy, dz))
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_transform_volumes_nonlinear(self.handle, _p(v), W, H, D, T, _p(fx), _p(fy),
                                                             _p(fz), int(interpolation), _p(out)))
        return out

    def combine_displacement_field(self, dx: torch.Tensor, dy: torch.Tensor, dz: torch.Tensor, params) -> None:
        """CreateCombinedDisplacementField: adds the affine displacement of
        params to the field (dx, dy, dz) in place."""
        for f in (dx, dy, dz):
            if not f.is_contiguous() or f.dtype != torch.float32 or not f.is_cuda:
                raise TypeError("field components must be contiguous float32 CUDA tensors")
        D, H, W = dx.shape
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(12))
        self._bind_stream()
        _check(self, L.lib().brc_combine_displacement_field(self.handle, _p(dx), _p(dy), _p(dz), W, H, D,
                                                            p.ctypes.data_as(ctypes.c_void_p)))

    def center_volumes(self, src: torch.Tensor, interpolation: int = L.INTERP_LINEAR):
        """CenterVolumesWrapper: (centred (T, D, H, W) volumes, 12 parameters)."""
        v = self._vols4(src)
        T, D, H, W = v.shape
        out = torch.empty_like(v)
        p = np.zeros(12, np.float32)
        self._bind_stream()
        _check(self, L.lib().brc_center_volumes(self.handle, _p(v), W, H, D, T, int(interpolation), _p(out),
                                                p.ctypes.data_as(ctypes.c_void_p)))
        return out, p

    def center_of_mass(self, vol: torch.Tensor) -> np.ndarray:
        v = vol.contiguous()
        D, H, W = v.shape
        c = np.zeros(3, np.float32)
        self._bind_stream()
        _check(self, L.lib().brc_center_of_mass(self.handle, _p(v), W, H, D, c.ctypes.data_as(ctypes.c_void_p)))
        return c

    def phase_volumes(self, q1: torch.Tensor, q2: torch.Tensor, axis: int = 2):
        """Phase difference, certainty and phase gradient along `axis` of one
        pair of complex (D,H,W) responses (the reference's linear formulas)."""
        a = torch.view_as_real(q1.contiguous()).contiguous() if q1.is_complex() else q1.contiguous()
        c = torch.view_as_real(q2.contiguous()).contiguous() if q2.is_complex() else q2.contiguous()
        D, H, W = a.shape[:3]
        out = torch.empty((3, D, H, W), dtype=torch.float32, device=a.device)
        self._bind_stream()
        _check(self, L.lib().brc_phase_volumes(self.handle, _p(a), _p(c), W, H, D, axis, _p(out[0]), _p(out[1]),
                                               _p(out[2])))
        return out[0], out[1], out[2]

    def multiply_volumes(self, vols: torch.Tensor, mask: torch.Tensor) -> None:
        """vols (T,D,H,W) or (D,H,W) *= mask (D,H,W), in place."""
        v = vols if vols.dim() == 4 else vols[None]
        assert v.is_contiguous() and mask.is_contiguous()
        T, D, H, W = v.shape
        self._bind_stream()
        _check(self, L.lib().brc_multiply_volumes(self.handle, _p(v), W, H, D, T, _p(mask)))

    def set_debug_outputs(self, outputs) -> None:
        """Host numpy arrays the linear (and, with six responses, nonlinear)
        registrations fill as the reference does with DEBUG set: a dict with
        any of 'quadrature_responses' (list of 3 or 6 complex64 arrays),
        'phase_differences', 'phase_certainties', 'phase_gradients'
        (float32).  None turns them off.  The arrays must stay alive while
        debug outputs are on."""
        if outputs is None:
            _check(self, L.lib().brc_ctx_set_debug_outputs(self.handle, None))
            self._debug_keep = None
            return
        d = L.DebugOutputs()
        keep = []
        for k, a in enumerate(outputs.get("quadrature_responses", []) or []):
            if a is not None:
                assert a.dtype == np.complex64 and a.flags.c_contiguous
                d.quadrature_responses[k] = a.ctypes.data
                keep.append(a)
        for name in ("phase_differences", "phase_certainties", "phase_gradients"):
            a = outputs.get(name)
            if a is not None:
                assert a.dtype == np.float32 and a.flags.c_contiguous
                setattr(d, name, a.ctypes.data)
                keep.append(a)
        self._debug_keep = keep
        _check(self, L.lib().brc_ctx_set_debug_outputs(self.handle, ctypes.byref(d)))

    @staticmethod
    def invert_affine_parameters(params) -> np.ndarray:
        p = np.ascontiguousarray(params, np.float32)
        out = np.zeros(12, np.float32)
        L.lib().brc_invert_affine_parameters(p.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def register_two_volumes(self, subject: torch.Tensor, voxel_size, template: torch.Tensor,
                             template_voxel_size, bank: dict, linear_iterations: int,
                             nonlinear_iterations: int, coarsest_scale: int, mm_z_cut: int = 0,
                             tsigma=5.0, esigma=5.0, dsigma=5.0, solve_fp64: bool = False,
                             precision: int = L.PREC_FP32, precenter: bool = False):
        """T1-to-template normalisation.  Returns dict: params (12,),
        interpolated, aligned_linear, aligned_nonlinear (template size) and
        field (3, D, H, W).  precenter: centre the subject by its centre of
        mass at its own size first (PRECENTER_REGISTRATION)."""
        s = subject.contiguous()
        t = template.contiguous()
        D, H, W = s.shape
        D2, H2, W2 = t.shape
        f3 = np.ascontiguousarray(bank["linear"], np.float32)
        f6, m, d = self._nl_consts(bank)
        o = L.TwoVolumeOpts()
        L.lib().brc_two_volume_opts_default(ctypes.byref(o))
        o.linear_iterations, o.nonlinear_iterations = linear_iterations, nonlinear_iterations
        o.coarsest_scale, o.mm_z_cut = coarsest_scale, mm_z_cut
        o.tsigma, o.esigma, o.dsigma = tsigma, esigma, dsigma
        o.solve_fp64 = 1 if solve_fp64 else 0
        o.precision = precision
        o.precenter = 1 if precenter else 0
        vs = np.ascontiguousarray(voxel_size, np.float32)
        tvs = np.ascontiguousarray(template_voxel_size, np.float32)
        params = np.zeros(12, np.float32)
        out = {k: torch.empty((D2, H2, W2), dtype=torch.float32, device=t.device)
               for k in ("interpolated", "aligned_linear", "aligned_nonlinear")}
        field = torch.zeros((3, D2, H2, W2), dtype=torch.float32, device=t.device)
        cp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        self._bind_stream()
        _check(self, L.lib().brc_register_two_volumes(
            self.handle, _p(s), W, H, D, cp(vs), _p(t), W2, H2, D2, cp(tvs), cp(f3), cp(f6), cp(m), cp(d),
            ctypes.byref(o), cp(params), _p(out["interpolated"]), _p(out["aligned_linear"]),
            _p(out["aligned_nonlinear"]), _p(field)))
        out["params"] = params
        out["field"] = field
        return out

    def register_cohort(self, subjects, voxel_sizes, template: torch.Tensor, template_voxel_size, bank: dict,
                        linear_iterations: int, nonlinear_iterations: int, coarsest_scale: int,
                        mm_z_cut: int = 0, tsigma=5.0, esigma=5.0, dsigma=5.0, solve_fp64: bool = False,
                        precision: int = L.PREC_FP32, precenter: bool = False):
        """T1-to-template normalisation of a cohort: `subjects` is a list of
        (D,H,W) device volumes of any sizes, `voxel_sizes` a matching list of
        (vx, vy, vz).  Returns dict: params (n,12), aligned_linear,
        aligned_nonlinear (n, template size) and fields (n,3, template size)."""
        subs = [v.contiguous() for v in subjects]
        n = len(subs)
        t = template.contiguous()
        D2, H2, W2 = t.shape
        f3 = np.ascontiguousarray(bank["linear"], np.float32)
        f6, m, d = self._nl_consts(bank)
        o = L.TwoVolumeOpts()
        L.lib().brc_two_volume_opts_default(ctypes.byref(o))
        o.linear_iterations, o.nonlinear_iterations = linear_iterations, nonlinear_iterations
        o.coarsest_scale, o.mm_z_cut = coarsest_scale, mm_z_cut
        o.tsigma, o.esigma, o.dsigma = tsigma, esigma, dsigma
        o.solve_fp64 = 1 if solve_fp64 else 0
        o.precision = precision
        o.precenter = 1 if precenter else 0
        ptrs = (ctypes.c_void_p * n)(*[v.data_ptr() for v in subs])
        sizes = np.ascontiguousarray([[v.shape[2], v.shape[1], v.shape[0]] for v in subs], np.int32)
        vs = np.ascontiguousarray(voxel_sizes, np.float32).reshape(n, 3)
        tvs = np.ascontiguousarray(template_voxel_size, np.float32)
        params = np.zeros((n, 12), np.float32)
        lin = torch.empty((n, D2, H2, W2), dtype=torch.float32, device=t.device)
        nl = torch.empty((n, D2, H2, W2), dtype=torch.float32, device=t.device)
        fields = torch.zeros((n, 3, D2, H2, W2), dtype=torch.float32, device=t.device)
        cp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        self._bind_stream()
        _check(self, L.lib().brc_register_cohort(
            self.handle, n, ctypes.cast(ptrs, ctypes.c_void_p), cp(sizes), cp(vs), _p(t), W2, H2, D2, cp(tvs),
            cp(f3), cp(f6), cp(m), cp(d), ctypes.byref(o), cp(params), _p(lin), _p(nl), _p(fields)))
        return {"params": params, "aligned_linear": lin, "aligned_nonlinear": nl, "fields": fields}

    def motion_correct(self, volumes: np.ndarray, voxel_size, filters, iterations: int,
                       tolerance: float = 0.0, reference: np.ndarray = None, use_graph: bool = True,
                       precision: int = L.PREC_FP32, certainty_sigma: float = 0.0):
        """Host-buffer motion correction of a (T,D,H,W) float32 series.
        Returns (corrected series, motion (6,T): mm then degrees).  The
        input array is not modified (a copy is corrected)."""
        v = np.ascontiguousarray(volumes, dtype=np.float32).copy()
        T, D, H, W = v.shape
        vs = np.ascontiguousarray(voxel_size, dtype=np.float32)
        f = _host_filters(filters)
        motion = np.zeros(6 * T, np.float32)
        opts = L.LinearOpts()
        L.lib().brc_linear_opts_default(ctypes.byref(opts), iterations)
        opts.type = L.RIGID
        opts.tolerance = tolerance
        opts.use_graph = 1 if use_graph else 0
        opts.precision = precision
        opts.certainty_sigma_x100 = int(round(certainty_sigma * 100))
        refp = None
        if reference is not None:
            ref_arr = np.ascontiguousarray(reference, dtype=np.float32)
            refp = ref_arr.ctypes.data_as(ctypes.c_void_p)
        self._bind_stream()
        _check(self, L.lib().brc_motion_correct(
            self.handle, v.ctypes.data_as(ctypes.c_void_p), W, H, D, T, vs.ctypes.data_as(ctypes.c_void_p),
            f.ctypes.data_as(ctypes.c_void_p), ctypes.byref(opts), refp,
            motion.ctypes.data_as(ctypes.c_void_p)))
        return v, motion.reshape(6, T)

    @staticmethod
    def smoothing_filters_fwhm(fwhm: float, voxel_size):
        """Gaussian filters (9 taps per axis) from a FWHM in mm: (fx, fy, fz)."""
        vs = np.ascontiguousarray(voxel_size, np.float32)
        f = [np.zeros(9, np.float32) for _ in range(3)]
        L.lib().brc_smoothing_filters_fwhm(float(fwhm), vs.ctypes.data_as(ctypes.c_void_p),
                                           *[a.ctypes.data_as(ctypes.c_void_p) for a in f])
        return tuple(f)

    def tensor_magnitude(self, vol: torch.Tensor, bank: dict, precision: int = L.PREC_FP32) -> torch.Tensor:
        """Frobenius norm of the structure tensor of one (D,H,W) volume."""
        v = vol.contiguous()
        D, H, W = v.shape
        f6, m, _ = self._nl_consts(bank)
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_tensor_magnitude(self.handle, _p(v), W, H, D, f6.ctypes.data_as(ctypes.c_void_p),
                                                  m.ctypes.data_as(ctypes.c_void_p), precision, _p(out)))
        return out

    def segment_epi(self, vol: torch.Tensor, voxel_size) -> torch.Tensor:
        """Brain mask (1 / 0.001) of one (D,H,W) EPI volume."""
        v = vol.contiguous()
        D, H, W = v.shape
        vs = np.ascontiguousarray(voxel_size, np.float32)
        out = torch.empty_like(v)
        self._bind_stream()
        _check(self, L.lib().brc_segment_epi(self.handle, _p(v), W, H, D, vs.ctypes.data_as(ctypes.c_void_p),
                                             _p(out)))
        return out

    def first_level_preprocess(self, fmri: np.ndarray, epi_voxel_size, t1: np.ndarray, t1_voxel_size,
                               mni: np.ndarray, mni_voxel_size, bank: dict, linear_iterations: int = 10,
                               nonlinear_iterations: int = 10, motion_iterations: int = 5,
                               coarsest_scale_t1_mni: int = 4, coarsest_scale_epi_t1: int = 4,
                               mm_t1_z_cut: int = 0, apply_motion_correction: bool = True,
                               apply_smoothing: bool = True, smoothing_fwhm: float = 6.0, tsigma=5.0, esigma=5.0,
                               dsigma=5.0, solve_fp64: bool = False, precision: int = L.PREC_FP32):
        """The preprocessing stages of a first-level analysis on host arrays:
        fmri (T,D,H,W), t1 and mni (D,H,W), voxel sizes (x, y, z) in mm.
        Returns a dict of every output of brc_first_level_preprocess (as
        numpy arrays) plus "fmri", the preprocessed series (the input array
        is not modified)."""
        v = np.ascontiguousarray(fmri, np.float32).copy()
        T, D1, H1, W1 = v.shape
        t = np.ascontiguousarray(t1, np.float32)
        m = np.ascontiguousarray(mni, np.float32)
        D2, H2, W2 = t.shape
        D3, H3, W3 = m.shape
        f3 = np.ascontiguousarray(bank["linear"], np.float32)
        f6, mt, d = self._nl_consts(bank)
        cp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        inp = L.FirstLevelInput(cp(v), W1, H1, D1, T, L._F3(*epi_voxel_size), cp(t), W2, H2, D2,
                                L._F3(*t1_voxel_size), cp(m), W3, H3, D3, L._F3(*mni_voxel_size), cp(f3), cp(f6),
                                cp(mt), cp(d))
        o = L.FirstLevelOpts()
        L.lib().brc_first_level_opts_default(ctypes.byref(o))
        o.linear_iterations, o.nonlinear_iterations = linear_iterations, nonlinear_iterations
        o.motion_iterations = motion_iterations
        o.coarsest_scale_t1_mni, o.coarsest_scale_epi_t1 = coarsest_scale_t1_mni, coarsest_scale_epi_t1
        o.mm_t1_z_cut = mm_t1_z_cut
        o.apply_motion_correction, o.apply_smoothing = int(apply_motion_correction), int(apply_smoothing)
        o.smoothing_fwhm = smoothing_fwhm
        o.tsigma, o.esigma, o.dsigma = tsigma, esigma, dsigma
        o.precision, o.solve_fp64 = precision, int(solve_fp64)
        shapes = {"params_t1_mni": (12,), "params_epi_t1": (12,), "params_epi_mni": (12,),
                  "motion_parameters": (6, T), "interpolated_t1": (D3, H3, W3),
                  "aligned_t1_linear": (D3, H3, W3), "aligned_t1_nonlinear": (D3, H3, W3),
                  "field": (3, D3, H3, W3), "aligned_epi_t1": (D3, H3, W3), "aligned_epi_mni_linear": (D3, H3, W3),
                  "aligned_epi_mni_nonlinear": (D3, H3, W3), "motion_corrected": (T, D1, H1, W1),
                  "epi_mask": (D1, H1, W1), "smoothed": (T, D1, H1, W1)}
        res = {k: np.zeros(shapes[k], np.float32) for k in L.FIRST_LEVEL_OUTPUTS}
        out = L.FirstLevelOutput(*[cp(res[k]) for k in L.FIRST_LEVEL_OUTPUTS])
        self._bind_stream()
        _check(self, L.lib().brc_first_level_preprocess(self.handle, ctypes.byref(inp), ctypes.byref(o),
                                                        ctypes.byref(out)))
        res["fmri"] = v
        return res
