"""The search entry point that allocates nothing (xtn_nn_search_static).

Some callers cannot allocate device memory while they run:
  - a framework's caching allocator already owns the device memory;
  - a latency-critical loop cannot take cudaMalloc's synchronisation;
  - a plugin host forbids allocation on its call path.
xtn_nn_search_static serves them from one fixed device array inside the library.
This test calls it through the C ABI twice in a row, with inputs the caller placed on the
device and output buffers the caller allocated. Each result must equal, bit for bit, what
the context entry point (xtn_context_nn_device) returns for the same input. The second call
is smaller than the first, so state left in the shared array by the first call would show.
The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

import xtn

pytestmark = pytest.mark.gpu


def static_search(lib, torch, chars, offs, d, measure, cap=1 << 16):
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    out_p = torch.zeros((cap, 2), dtype=torch.int32, device="cuda")
    out_d = torch.zeros(cap, dtype=torch.int8, device="cuda")
    n_out = ctypes.c_int64(-1)
    args = xtn.Args(d, measure, 0, 0)
    torch.cuda.synchronize()
    rc = lib.xtn_nn_search_static(ctypes.byref(args), ctypes.c_void_p(dch.data_ptr()), ctypes.c_void_p(dof.data_ptr()),
                                  len(offs) - 1, ctypes.c_void_p(out_p.data_ptr()), ctypes.c_void_p(out_d.data_ptr()),
                                  cap, ctypes.byref(n_out), None)
    assert rc == 0, lib.xtn_last_error().decode()
    m = n_out.value
    return out_p[:m].cpu().numpy(), out_d[:m].cpu().numpy()


def test_static_search_matches_context_search_twice():
    import torch

    lib = xtn.load()
    P = ctypes.c_void_p
    lib.xtn_nn_search_static.argtypes = [ctypes.POINTER(xtn.Args), P, P, ctypes.c_int32, P, P, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int64), P]
    ctx = xtn.Context(0)
    cases = [(xtn.synth_mutants(seed=501, n=4000, mutant_frac=0.25), 2, xtn.LEVENSHTEIN),
             (xtn.synth_mutants(seed=502, n=1500, mutant_frac=0.25), 1, xtn.HAMMING)]
    for (chars, offs), d, m in cases:
        got_p, got_d = static_search(lib, torch, chars, offs, d, m)
        dch = torch.from_numpy(chars).cuda()
        dof = torch.from_numpy(offs.view(np.int32)).cuda()
        torch.cuda.synchronize()
        n = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), len(offs) - 1, distance=d, measure=m)
        ref = ctx.fetch(n)
        assert len(ref.pairs) > 50
        assert np.array_equal(got_p, ref.pairs)
        assert np.array_equal(got_d, ref.distances)
    ctx.close()


def test_static_search_rejects_oversized_input():
    import torch

    lib = xtn.load()
    chars, offs = xtn.synth_mutants(seed=503, n=5000)
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    n_out = ctypes.c_int64(0)
    args = xtn.Args(1, 0, 0, 0)
    rc = lib.xtn_nn_search_static(ctypes.byref(args), ctypes.c_void_p(dch.data_ptr()), ctypes.c_void_p(dof.data_ptr()),
                                  len(offs) - 1, None, None, 0, ctypes.byref(n_out), None)
    assert rc == xtn.ERR_LIMIT
    assert "at most 4096 sequences" in lib.xtn_last_error().decode()
