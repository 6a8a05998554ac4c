"""Error paths of the CUDA library that need a GPU but must never fault it.

* Device-resident inputs are validated on the device: a sequence outside 1..500 residues
  (the reference's MAX_INPUT_LENGTH, xtneighbor_streaming/src/codec.cu:18) is reported as
  XTN_ERR_ARG with its index, before any kernel indexes by length, for every entry point
  that takes device pointers. The host-buffer entry already checks on the host.
* The bounded look-back waits of the single-pass prefix sums: with the context option
  "wait_fault_test" the first tile's status word is never set (a flag that nothing sets), so
  the later tiles' waits run out after "wait_polls" polls. The call must return XTN_ERR_CUDA,
  and the same context must then search correctly.
"""
import ctypes

import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import assert_same_pairs, csr

pytestmark = pytest.mark.gpu


def bad_inputs():
    """Three host-built inputs with one invalid sequence each: 501 residues, empty, and
    decreasing offsets."""
    good = ["CASSLGF", "CASSLGY", "CASRLGF"] * 40
    long_seq = "CAS" + "G" * 497 + "F"  # 501 residues
    a_c, a_o = csr(good[:50] + [long_seq] + good[50:])
    b_c, b_o = csr(good)
    b_o = np.concatenate([b_o[:71], b_o[70:]]).astype(np.uint32)  # offset 70 repeated: row 70 is empty
    c_c, c_o = csr(good)
    c_o = c_o.copy()
    c_o[33] = c_o[35]  # row 32 grows; row 33 now ends before it starts (a negative length)
    return [(a_c, a_o, 50), (b_c, b_o, 70), (c_c, c_o, 33)]


def device(torch, chars, offs):
    dch = torch.from_numpy(np.concatenate([chars, np.zeros(64, np.uint8)])).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    return dch, dof


def test_device_entry_rejects_bad_lengths():
    import torch

    with xtn.Context(0) as ctx:
        for chars, offs, first_bad in bad_inputs():
            dch, dof = device(torch, chars, offs)
            n = len(offs) - 1
            with pytest.raises(xtn.XtnError, match=f"sequence {first_bad} has an invalid length"):
                ctx.nn_device(dch.data_ptr(), dof.data_ptr(), n, distance=2)
            info = np.zeros((n, 3), np.int32)
            info[:, 0] = 1
            info[:, 2] = np.arange(n)
            dinf = torch.from_numpy(info).cuda()
            torch.cuda.synchronize()
            with pytest.raises(xtn.XtnError, match=f"sequence {first_bad} has an invalid length"):
                ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), 1, distance=1)
        # the context is still usable
        chars, offs = xtn.synth_mutants(seed=8, n=3000)
        dch, dof = device(torch, chars, offs)
        m = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), len(offs) - 1, distance=2)
        got = ctx.fetch(m)
        exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
        assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "after rejected inputs")


def test_index_device_entries_reject_bad_lengths():
    import torch

    lib = xtn.load()
    chars, offs = xtn.synth_mutants(seed=9, n=2000)
    with xtn.Index(chars, offs, max_distance=1) as ix:
        for qc, qo, first_bad in bad_inputs():
            dch, dof = device(torch, qc, qo)
            with pytest.raises(xtn.XtnError, match=f"sequence {first_bad} has an invalid length"):
                ix.query_device(dch.data_ptr(), dof.data_ptr(), len(qo) - 1, distance=1)
            h = ctypes.c_void_p()
            rc = lib.xtn_index_create_device(0, ctypes.c_void_p(dch.data_ptr()), ctypes.c_void_p(dof.data_ptr()),
                                             len(qo) - 1, 1, ctypes.byref(h))
            assert rc == xtn.ERR_ARG and not h.value
            assert f"sequence {first_bad} has an invalid length".encode() in lib.xtn_last_error()
        got = ix.query(chars[: offs[100]], offs[:101], distance=1)
        assert len(got.pairs) > 0


def test_static_entry_rejects_bad_lengths():
    import torch

    lib = xtn.load()
    out_p = torch.zeros((1024, 2), dtype=torch.int32, device="cuda")
    out_d = torch.zeros(1024, dtype=torch.int8, device="cuda")
    for chars, offs, first_bad in bad_inputs():
        dch, dof = device(torch, chars, offs)
        n_out = ctypes.c_int64(-1)
        args = xtn.Args(1, 0, 0, 0)
        rc = lib.xtn_nn_search_static(ctypes.byref(args), ctypes.c_void_p(dch.data_ptr()),
                                      ctypes.c_void_p(dof.data_ptr()), len(offs) - 1,
                                      ctypes.c_void_p(out_p.data_ptr()), ctypes.c_void_p(out_d.data_ptr()), 1024,
                                      ctypes.byref(n_out), None)
        assert rc == xtn.ERR_ARG
        assert f"sequence {first_bad} has an invalid length".encode() in lib.xtn_last_error()


def test_lookback_wait_expiry_is_reported_and_recoverable():
    """A look-back wait that runs out is an error the caller sees, not a hang or a wrong result."""
    chars, offs = xtn.synth_clusters(seed=17, n=40_000)  # ~10 tiles in the variant-offset scan
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    with xtn.Context(0, wait_polls=512) as ctx:
        ctx.set_option("wait_fault_test", 1)
        with pytest.raises(xtn.XtnError, match="did not complete in time") as ei:
            ctx.perform(chars, offs, distance=2)
        assert ei.value.code == xtn.ERR_CUDA
        got = ctx.perform(chars, offs, distance=2)  # the option was one-shot
        assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "after the expired wait")
