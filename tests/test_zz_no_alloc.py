"""The allocation-free entry point, msa_nw_all_pairs_noalloc.

It exists for callers that may not call cudaMalloc when they score sequences
(a runtime that owns all device memory in its own pool, or code that must not
risk the device synchronisation an allocation can cause). The test plays such
a caller: it owns the device buffers (made here with torch) and checks that
two calls in a row produce exactly the scores of the regular entry point,
msa_nw_all_pairs. Scores are integers, so the tolerance is zero.
"""
import ctypes

import numpy as np
import pytest

from msa_b200 import ScoringTable, pairwise
from msa_b200 import _lib
from msa_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device_inputs(wl):
    import torch
    flat, offs, lens = wl.flat_units(pad3=False)
    d_units = torch.from_numpy(flat.copy()).to("cuda:0")
    return flat, offs, lens, d_units


def _noalloc(d_units, offs, lens, n, table, stream):
    import torch
    out = torch.full((n * (n - 1) // 2,), -7, dtype=torch.int32, device="cuda:0")
    u64 = ctypes.POINTER(ctypes.c_uint64)
    rc = _lib.lib().msa_nw_all_pairs_noalloc(ctypes.c_void_p(d_units.data_ptr()), offs.ctypes.data_as(u64),
                                             lens.ctypes.data_as(u64), n, ctypes.byref(table._t),
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    if rc != 0:
        raise _lib.MsaError(rc, (_lib.lib().msa_noalloc_last_error() or b"").decode())
    return out.cpu().numpy()


@pytest.mark.parametrize("case", ["protein_with_end_units", "dna_long"])
def test_noalloc_matches_regular_entry_point_twice(case):
    import torch
    torch.cuda.set_device(0)
    if case == "protein_with_end_units":
        wl = W.random_set(71, 30, 0, 700, extra=b"*\r")   # interior END units and empties
        table = ScoringTable("blosum62")
    else:
        wl = W.random_set(72, 12, 300, 2500, alphabet=b"ACGTN")   # several 512-row strips
        table = ScoringTable("default")
    flat, offs, lens, d_units = _device_inputs(wl)
    want = pairwise.score_units(flat, offs, lens, table, _lib.MSA_NW_PERSISTENT)
    stream = torch.cuda.current_stream().cuda_stream
    first = _noalloc(d_units, offs, lens, wl.n, table, stream)
    second = _noalloc(d_units, offs, lens, wl.n, table, stream)
    assert np.array_equal(first, want)
    assert np.array_equal(second, want)


def test_noalloc_second_call_is_independent_of_the_first():
    import torch
    torch.cuda.set_device(0)
    big = W.random_set(73, 20, 100, 1500, alphabet=b"ACGT")
    small = W.c1()
    stream = torch.cuda.current_stream().cuda_stream
    for wl, name in ((big, "default"), (small, "blosum62")):
        t = ScoringTable(name)
        flat, offs, lens, d_units = _device_inputs(wl)
        got = _noalloc(d_units, offs, lens, wl.n, t, stream)
        assert np.array_equal(got, pairwise.score_units(flat, offs, lens, t, _lib.MSA_NW_PLAIN))


def test_noalloc_rejects_requests_beyond_its_limits():
    import torch
    torch.cuda.set_device(0)
    t = ScoringTable("blosum62")
    d = torch.zeros(16, dtype=torch.uint8, device="cuda:0")
    out = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    n = 70000
    offs = np.zeros(n, np.uint64)
    lens = np.ones(n, np.uint64)
    u64 = ctypes.POINTER(ctypes.c_uint64)
    rc = _lib.lib().msa_nw_all_pairs_noalloc(ctypes.c_void_p(d.data_ptr()), offs.ctypes.data_as(u64),
                                             lens.ctypes.data_as(u64), n, ctypes.byref(t._t),
                                             ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.MSA_ERR_TOO_LARGE
    assert b"65536" in _lib.lib().msa_noalloc_last_error()


def test_noalloc_gap_unit_in_shorter_sequence_is_undefined_like_the_regular_entry_point():
    """With a caller's own table every GAP entry lies outside the reference's
    storage. A GAP unit only in the shorter sequence of a pair must give
    MSA_ERR_UNDEFINED from both entry points, not scores."""
    import torch
    torch.cuda.set_device(0)
    base = ScoringTable("blosum62").matrix().astype(np.int32)
    table = ScoringTable.custom(base, 4)
    wl = W.random_set(74, 6, 60, 120)
    flat, offs, lens = wl.flat_units(pad3=False)
    flat = flat.copy()
    k = int(np.argmin(lens))
    flat[int(offs[k]) + int(lens[k]) // 2] = _lib.UNIT_GAP
    with pytest.raises(_lib.MsaError) as regular:
        pairwise.score_units(flat, offs, lens, table, _lib.MSA_NW_PERSISTENT)
    assert regular.value.status == _lib.MSA_ERR_UNDEFINED
    d_units = torch.from_numpy(flat).to("cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        with pytest.raises(_lib.MsaError) as na:
            _noalloc(d_units, offs, lens, wl.n, table, stream)
        assert na.value.status == _lib.MSA_ERR_UNDEFINED
    # Without the GAP unit the same call scores as before.
    flat2, _, _ = wl.flat_units(pad3=False)
    got = _noalloc(torch.from_numpy(flat2.copy()).to("cuda:0"), offs, lens, wl.n, table, stream)
    assert np.array_equal(got, pairwise.score_units(flat2, offs, lens, table, _lib.MSA_NW_PERSISTENT))
