"""brc_normal_equations_noalloc: the normal equations for callers that
cannot let a library allocate device memory (a pooled or pre-reserved HBM
budget, or a host that plans all memory before it starts).  It keeps its
partial sums in a fixed device array instead of a context workspace.

Checked through the C-ABI against the allocating entry point
brc_normal_equations, on two calls in a row (the fixed array keeps the
previous call's contents, which must not leak into the next result), with
one reference shared by the batch and with one reference per instance, and
against the CPU oracle's normal equations on one volume.  The device's free
memory is unchanged across a call.  Tolerance as in the other kernel tests:
max |a - b| <= 1e-4 * max |b|.

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


def _stream():
    st = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(st) if st else None


def _setup():
    # batch = 0: resolve the fixed array on this device (allocates it under
    # lazy module loading) and nothing else
    s = _noalloc()(_stream(), None, 0, None, 0, 0, 0, 0, None, None)
    assert s == L.BRC_OK, L.status_string(s)


def _outputs(B):
    A = torch.full((B, 144), float("nan"), dtype=torch.float64, device="cuda")
    h = torch.full((B, 12), float("nan"), dtype=torch.float64, device="cuda")
    return A, h


def _call_noalloc(q1, q2, shared, A, h):
    B, _, D, H, W, _ = q2.shape
    stride = 0 if shared else 6 * D * H * W
    s = _noalloc()(_stream(), q1.data_ptr(), stride, q2.data_ptr(), W, H, D, B, A.data_ptr(), h.data_ptr())
    assert s == L.BRC_OK, L.status_string(s)


def _host(A, h):
    B = A.shape[0]
    return A.reshape(B, 12, 12).transpose(1, 2).cpu().numpy(), h.cpu().numpy()


def _run_alloc(ctx, q1, q2):
    A, h = ctx.normal_equations(torch.view_as_complex(q1), torch.view_as_complex(q2))
    torch.cuda.synchronize()
    return A.cpu().numpy(), h.cpu().numpy()


@pytest.mark.parametrize("shared", [True, False], ids=["shared_reference", "reference_per_instance"])
def test_noalloc_matches_allocating_entry_point_twice(shared):
    from broccoli_b200.api import Context
    _setup()
    ctx = Context(0)
    cases = [(1, 5, (33, 64, 64)), (2, 3, (20, 24, 22))]
    for seed, B, shape in cases:  # two calls in a row, different sizes
        q1, q2 = _responses(seed, B, shape)
        if not shared:  # one reference per instance: B x 3 complex volumes
            g = torch.Generator().manual_seed(seed + 10)
            q1 = (q1[None] + 0.1 * torch.randn((B,) + tuple(q1.shape), generator=g).cuda()).contiguous()
        A, h = _outputs(B)
        _call_noalloc(q1, q2, shared, A, h)
        torch.cuda.synchronize()
        A0, h0 = _host(A, h)
        if shared:
            A1, h1 = _run_alloc(ctx, q1, q2)
        else:  # the allocating entry point one instance at a time
            r = [_run_alloc(ctx, q1[b], q2[b:b + 1]) for b in range(B)]
            A1, h1 = np.concatenate([a for a, _ in r]), np.concatenate([x for _, x in r])
        assert np.all(np.isfinite(A0)) and np.all(np.isfinite(h0))
        assert rel_err(A0, A1) < TOL
        assert rel_err(h0, h1) < TOL
    ctx.close()


def test_noalloc_leaves_free_memory_unchanged_and_matches_oracle():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import oracle
    _setup()
    q1a, q2a = _responses(4, 4, (33, 64, 64))
    q1b, q2b = _responses(5, 2, (21, 30, 26))
    Aa, ha = _outputs(4)
    Ab, hb = _outputs(2)
    _call_noalloc(q1a, q2a, True, Aa, ha)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _call_noalloc(q1b, q2b, True, Ab, hb)  # a second call of another size
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    A0, h0 = _host(Ab, hb)
    c1 = torch.view_as_complex(q1b).cpu().numpy()
    c2 = torch.view_as_complex(q2b).cpu().numpy()
    for b in range(2):
        Ao, ho = oracle.normal_equations(c1, c2[b])
        assert rel_err(A0[b], Ao) < TOL
        assert rel_err(h0[b], ho) < TOL


def test_noalloc_rejects_requests_beyond_its_scratch():
    q1, q2 = _responses(3, 1, (33, 64, 64))
    A = torch.zeros((200, 144), dtype=torch.float64, device="cuda")
    h = torch.zeros((200, 12), dtype=torch.float64, device="cuda")
    # 27 rows per 64x64x33 volume: 200 volumes need 5400 > 3072 rows
    s = _noalloc()(_stream(), q1.data_ptr(), 0, q2.data_ptr(), 64, 64, 33, 200, A.data_ptr(), h.data_ptr())
    assert s == BRC_ERR_SCRATCH_LIMIT
    assert "scratch" in L.status_string(s)
