"""bz2g_rle1_noalloc: the RLE1 entry point that allocates no device memory
(for callers that reserve their device memory up front, or must not take the
synchronisation of cudaMalloc / cudaFree on their path).  Its output must
equal the allocating entry point's (bz2g_rle1) exactly, call after call,
since both share one static scratch array across calls."""
import ctypes

import numpy as np
import pytest

import bzip2gpu_b200 as B
import bzip2gpu_b200.workloads as W

pytestmark = pytest.mark.gpu


def _fn():
    f = B.lib().bz2g_rle1_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                  ctypes.c_void_p]
    return f


def _noalloc(torch, d_in):
    n = d_in.numel()
    out = torch.full((B.lib().bz2g_rle1_bound(n),), 0xAA, dtype=torch.uint8, device="cuda")
    m = ctypes.c_int(-1)
    rc = _fn()(d_in.data_ptr(), n, out.data_ptr(), ctypes.byref(m),
               torch.cuda.current_stream().cuda_stream)
    return rc, out[: max(m.value, 0)], m.value


def _call(torch, d_in, out):
    m = ctypes.c_int(-1)
    rc = _fn()(d_in.data_ptr(), d_in.numel(), out.data_ptr(), ctypes.byref(m),
               torch.cuda.current_stream().cuda_stream)
    return rc, m.value


def test_noalloc_matches_allocating_entry_point_twice(torch_cuda):
    torch = torch_cuda
    inputs = [W.small_markov(1 << 20, seed=41),                       # at the size limit
              np.concatenate([np.full(300000, 7), np.arange(777) % 3,
                              np.full(1037, 9)]).astype(np.uint8)]     # long runs, smaller
    d_ins = [torch.from_numpy(a).cuda() for a in inputs]
    refs = [B.rle1(d) for d in d_ins]
    outs = [torch.full((B.lib().bz2g_rle1_bound(d.numel()),), 0xAA, dtype=torch.uint8,
                       device="cuda") for d in d_ins]
    # set-up call (the scratch's address; the library's kernels loaded)
    assert _call(torch, d_ins[1], outs[1])[0] == 0, B.lib().bz2g_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    res = [_call(torch, d, o) for d, o in zip(d_ins, outs)]  # two calls in a row
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0, f"device memory taken during the calls: {free0 - free1} bytes"
    for (rc, m), ref, o in zip(res, refs, outs):
        assert rc == 0, B.lib().bz2g_last_error()
        assert m == ref.numel()
        assert torch.equal(o[:m], ref)


def test_noalloc_rejects_inputs_over_the_limit(torch_cuda):
    torch = torch_cuda
    d_in = torch.zeros((1 << 20) + 1, dtype=torch.uint8, device="cuda")
    rc, _, _ = _noalloc(torch, d_in)
    assert rc == 5  # BZ2G_ERR_TOO_LARGE
    assert b"exceeds" in B.lib().bz2g_last_error()
