"""The allocation-free dense matcher (fsb_match_bf_noalloc) gives the same pairs as the
allocating entry point (fsb_match_bf), on two calls in a row.

This entry point exists for callers that cannot call cudaMalloc (processes with a fixed,
pre-reserved device-memory budget, host frameworks that own the CUDA allocator, real-time loops
that must not block in an allocation). Its scratch is a fixed device array inside the library,
shared by every call, so the second call below also checks that nothing left over from the first
call leaks into its result. This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, torch, a, b, ratio, dev):
    da = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    na, nb = len(a), len(b)
    dq = torch.full((max(na, 1),), -7, dtype=torch.int64, device=dev)
    dt = torch.full((max(na, 1),), -7, dtype=torch.int64, device=dev)
    dn = torch.full((1,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = lib.fsb_match_bf_noalloc(ctypes.c_void_p(da.data_ptr()), na, ctypes.c_void_p(db.data_ptr()), nb,
                                  ctypes.c_float(ratio), ctypes.c_void_p(dq.data_ptr()),
                                  ctypes.c_void_p(dt.data_ptr()), ctypes.c_void_p(dn.data_ptr()),
                                  ctypes.c_void_p(stream.cuda_stream))
    assert st == 0, lib.fsb_last_error()
    torch.cuda.synchronize(dev)
    n = int(dn.item())
    return dq[:n].cpu().numpy(), dt[:n].cpu().numpy()


def test_no_alloc_matches_allocating_entry_point_twice():
    import torch

    import fieldstitch_b200 as F
    from fieldstitch_b200 import _lib, synth
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    # first call: 3000 x 2500; second call: smaller A, larger B, other ratio
    for na, nb, seed, ratio in [(3000, 2500, 11, 0.8), (1200, 4000, 12, 0.85)]:
        a, b, _ = synth.synth_descriptors(na, nb, seed)
        q_ref, t_ref = F.matching._ratio_match_bf(a, b, ratio)
        q, t = _call(lib, torch, a, b, ratio, dev)
        assert len(q_ref) > 0
        np.testing.assert_array_equal(q, q_ref)
        np.testing.assert_array_equal(t, t_ref)


def test_no_alloc_at_its_largest_layout():
    """16384 x 16384 fills the per-target key table and the top-2 table to their fixed capacity;
    16384 x 130 runs the most column splits the table allows for a full A side."""
    import torch

    import fieldstitch_b200 as F
    from fieldstitch_b200 import _lib, synth
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    for na, nb, seed, ratio in [(16384, 16384, 13, 0.8), (16384, 130, 14, 0.8)]:
        a, b, _ = synth.synth_descriptors(na, nb, seed)
        q_ref, t_ref = F.matching._ratio_match_bf(a, b, ratio)
        q, t = _call(lib, torch, a, b, ratio, dev)
        assert len(q_ref) > 0
        np.testing.assert_array_equal(q, q_ref)
        np.testing.assert_array_equal(t, t_ref)


@pytest.mark.parametrize("na,nb", [(16385, 10), (10, 16385)])
def test_no_alloc_rejects_sizes_beyond_its_limit(na, nb):
    from fieldstitch_b200 import _lib
    lib = _lib.load()
    # the size check comes before any pointer is used, so placeholder addresses are never touched
    st = lib.fsb_match_bf_noalloc(ctypes.c_void_p(16), na, ctypes.c_void_p(16), nb, ctypes.c_float(0.8),
                                  ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert st == 1
    assert b"16384-row limit" in lib.fsb_last_error()
