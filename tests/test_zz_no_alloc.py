"""brc_normal_equations_noalloc: the normal equations for callers that
cannot let a library allocate device memory (a pooled or pre-reserved HBM
budget, or a host that plans all memory before it starts).  It keeps its
partial sums in a fixed device array instead of a context workspace.

Checked through the C-ABI against the allocating entry point
brc_normal_equations, on two calls in a row (the fixed array keeps the
previous call's contents, which must not leak into the next result).
Tolerance as in the other kernel tests: max |a - b| <= 1e-4 * max |b|.

This file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_err
from broccoli_b200 import _lib as L

pytestmark = pytest.mark.gpu
TOL = 1e-4
BRC_ERR_SCRATCH_LIMIT = -8  # include/broccoli_b200.h


def _noalloc():
    fn = L.lib().brc_normal_equations_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _responses(seed, B, shape):
    g = torch.Generator().manual_seed(seed)
    q1 = torch.randn((3,) + shape + (2,), generator=g).cuda()
    q2 = (q1[None] + 0.3 * torch.randn((B, 3) + shape + (2,), generator=g).cuda()).contiguous()
    return q1.contiguous(), q2


def _run_noalloc(q1, q2, shared):
    B, _, D, H, W, _ = q2.shape
    A = torch.full((B, 144), float("nan"), dtype=torch.float64, device="cuda")
    h = torch.full((B, 12), float("nan"), dtype=torch.float64, device="cuda")
    stride = 0 if shared else 6 * D * H * W
    st = torch.cuda.current_stream().cuda_stream
    s = _noalloc()(ctypes.c_void_p(st) if st else None, q1.data_ptr(), stride, q2.data_ptr(), W, H, D, B,
                   A.data_ptr(), h.data_ptr())
    assert s == L.BRC_OK, L.status_string(s)
    torch.cuda.synchronize()
    return A.reshape(B, 12, 12).transpose(1, 2).cpu().numpy(), h.cpu().numpy()


def _run_alloc(ctx, q1, q2):
    A, h = ctx.normal_equations(torch.view_as_complex(q1), torch.view_as_complex(q2))
    torch.cuda.synchronize()
    return A.cpu().numpy(), h.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    from broccoli_b200.api import Context
    ctx = Context(0)
    cases = [(1, 5, (33, 64, 64)), (2, 3, (20, 24, 22))]
    for seed, B, shape in cases:  # two calls in a row, different sizes
        q1, q2 = _responses(seed, B, shape)
        A0, h0 = _run_noalloc(q1, q2, shared=True)
        A1, h1 = _run_alloc(ctx, q1, q2)
        assert np.all(np.isfinite(A0)) and np.all(np.isfinite(h0))
        assert rel_err(A0, A1) < TOL
        assert rel_err(h0, h1) < TOL
    ctx.close()


def test_noalloc_rejects_requests_beyond_its_scratch():
    q1, q2 = _responses(3, 1, (33, 64, 64))
    st = torch.cuda.current_stream().cuda_stream
    A = torch.zeros((200, 144), dtype=torch.float64, device="cuda")
    h = torch.zeros((200, 12), dtype=torch.float64, device="cuda")
    # 27 rows per 64x64x33 volume: 200 volumes need 5400 > 3072 rows
    s = _noalloc()(ctypes.c_void_p(st) if st else None, q1.data_ptr(), 0, q2.data_ptr(), 64, 64, 33, 200,
                   A.data_ptr(), h.data_ptr())
    assert s == BRC_ERR_SCRATCH_LIMIT
    assert "scratch" in L.status_string(s)
