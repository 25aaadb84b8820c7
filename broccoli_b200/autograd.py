"""Differentiable registration: torch.autograd.Function wrappers whose
forward and backward passes are the library's CUDA kernels.

    smooth3d   Gaussian smoothing (the adjoint is the same smoothing with the
               taps reversed)
    warp_affine / warp_field
               trilinear warps; backward = exact derivative of the
               interpolant for the parameters / field, atomic scatter for
               the source volume
    filter3d   7^3 complex filtering; backward = correlation of the complex
               gradient with the filters (brc_filter3d_adjoint)

`registration_objective` composes them into the filter-response SSD of a
moving volume, warped by 12 affine parameters or a displacement field,
against a reference: L = sum_k sum_x |q_k(warp(S moving)) - q_k(S ref)|^2.
The reference responses are computed once and kept (a checkpoint per
scale when used in a pyramid); torch only holds tensors and stitches the
graph together.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .api import Context, _check, _host_filters, _p

_contexts = {}


def _ctx(device: torch.device) -> Context:
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx not in _contexts:
        _contexts[idx] = Context(idx)
    c = _contexts[idx]
    c._bind_stream()
    return c


def _sig(name, args):
    fn = getattr(L.lib(), name)
    fn.argtypes = args
    fn.restype = ctypes.c_int
    return fn


_P, _I = ctypes.c_void_p, ctypes.c_int


def gaussian_taps(sigma: float) -> np.ndarray:
    """9-tap Gaussian normalised by its float sum (CreateSmoothingFilters,
    broccoli_lib.cpp:11093-11121)."""
    u = np.arange(9, dtype=np.float64) - 4
    f = np.exp(-u ** 2 / (2.0 * sigma * sigma)).astype(np.float32)
    s = np.float32(0)
    for v in f:
        s = np.float32(s + v)
    return (f / s).astype(np.float32)


class Smooth3d(torch.autograd.Function):
    @staticmethod
    def forward(fctx, vol, taps):
        c = _ctx(vol.device)
        fctx.taps = taps
        return c.smooth3d(vol.contiguous(), taps, taps, taps)

    @staticmethod
    def backward(fctx, g):
        c = _ctx(g.device)
        rev = np.ascontiguousarray(fctx.taps[::-1])
        return c.smooth3d(g.contiguous(), rev, rev, rev), None


class WarpAffine(torch.autograd.Function):
    @staticmethod
    def forward(fctx, src, params):
        c = _ctx(src.device)
        s = src.contiguous()
        p = params.detach().reshape(-1, 12).contiguous().to(torch.float32)
        fctx.save_for_backward(s, p)
        return c.warp_affine(s, p)

    @staticmethod
    def backward(fctx, g):
        s, p = fctx.saved_tensors
        c = _ctx(g.device)
        B, D, H, W = (s.shape if s.dim() == 4 else (1,) + tuple(s.shape))
        gp = torch.empty((B, 12), dtype=torch.float64, device=g.device)
        gs = torch.empty((B, D, H, W), dtype=torch.float32, device=g.device) if fctx.needs_input_grad[0] else None
        fn = _sig("brc_warp_affine_backward", [_P, _P, _I, _I, _I, _I, _P, _P, _P, _P])
        _check(c, fn(c.handle, _p(s), W, H, D, B, _p(p), _p(g.contiguous()), _p(gp), _p(gs) if gs is not None else None))
        gsrc = gs.reshape(s.shape) if gs is not None else None
        return gsrc, gp.to(torch.float32).reshape(fctx.saved_tensors[1].shape)


class WarpField(torch.autograd.Function):
    @staticmethod
    def forward(fctx, src, field):
        c = _ctx(src.device)
        s = src.contiguous()
        f = field.detach().contiguous()
        fctx.save_for_backward(s, f)
        return c.warp_field(s, f[0], f[1], f[2])

    @staticmethod
    def backward(fctx, g):
        s, f = fctx.saved_tensors
        c = _ctx(g.device)
        D, H, W = s.shape
        gf = torch.empty_like(f) if fctx.needs_input_grad[1] else None
        gs = torch.empty_like(s) if fctx.needs_input_grad[0] else None
        fn = _sig("brc_warp_field_backward", [_P, _P, _I, _I, _I, _P, _P, _P, _P, _P, _P])
        _check(c, fn(c.handle, _p(s), W, H, D, _p(f[0]), _p(f[1]), _p(f[2]), _p(g.contiguous()),
                     _p(gf) if gf is not None else None, _p(gs) if gs is not None else None))
        return gs, gf


class Filter3d(torch.autograd.Function):
    """Real volumes (B,D,H,W) -> responses (B,nfilt,D,H,W,2) (re, im)."""

    @staticmethod
    def forward(fctx, vol, filters):
        c = _ctx(vol.device)
        f = _host_filters(filters)
        fctx.filters = f
        return torch.view_as_real(c.filter3d(vol, f))

    @staticmethod
    def backward(fctx, g):
        c = _ctx(g.device)
        f = fctx.filters
        B, nf, D, H, W, _ = g.shape
        out = torch.empty((B, D, H, W), dtype=torch.float32, device=g.device)
        fn = _sig("brc_filter3d_adjoint", [_P, _P, _I, _I, _I, _I, _P, _I, _P])
        _check(c, fn(c.handle, _p(g.contiguous()), W, H, D, B, f.ctypes.data_as(ctypes.c_void_p), nf, _p(out)))
        return out, None


def smooth3d(vol, sigma: float):
    return Smooth3d.apply(vol, gaussian_taps(sigma))


def warp_affine(src, params):
    return WarpAffine.apply(src, params)


def warp_field(src, field):
    return WarpField.apply(src, field)


def filter3d(vol, filters):
    return Filter3d.apply(vol, filters)


def reference_responses(ref: torch.Tensor, filters, sigma: float) -> torch.Tensor:
    """Responses of the smoothed reference (kept across iterations; the
    checkpoint of one pyramid scale)."""
    with torch.no_grad():
        return filter3d(smooth3d(ref[None] if ref.dim() == 3 else ref, sigma), filters)


def registration_objective(moving: torch.Tensor, q_ref: torch.Tensor, filters, sigma: float,
                           params: torch.Tensor = None, field: torch.Tensor = None) -> torch.Tensor:
    """SSD of the filter responses of `moving` (D,H,W) smoothed, then warped
    by `params` (12,) or `field` (3,D,H,W), against the reference responses
    `q_ref` (1,nfilt,D,H,W,2).  Differentiable in params / field / moving."""
    s = smooth3d(moving[None], sigma)
    if params is not None:
        w = warp_affine(s, params.reshape(1, 12))
    else:
        w = warp_field(s[0], field)[None]
    q = filter3d(w, filters)
    return ((q - q_ref) ** 2).sum()
