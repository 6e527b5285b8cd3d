"""All-pairs NW on the GPU through the C ABI, checked bit-exact against the
reference (golden fixtures it produced) and the oracle restatement."""
import ctypes

import numpy as np
import pytest

from msa_b200 import Database, ScoringTable, pairwise
from msa_b200 import _lib
from msa_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = [_lib.MSA_NW_PLAIN, _lib.MSA_NW_PERSISTENT]


def gpu_scores(wl, table, mode, pad3=False):
    flat, offs, lens = wl.flat_units(pad3=pad3)
    t = table if isinstance(table, ScoringTable) else ScoringTable(table)
    return pairwise.score_units(flat, offs, lens, t, mode)


@pytest.fixture(scope="module")
def tables(golden):
    return O.table_block(golden)


def oracle_scores(wl, table, tables, pad3=False):
    flat, offs, lens = wl.flat_units(pad3=pad3)
    return O.oracle_nw_all_pairs(flat, offs, lens, tables, 7, O.TABLE_INDEX[table], O.PENALTY[table])


@pytest.mark.parametrize("mode", MODES)
def test_c1_matches_reference(gpu, golden, mode):
    got = gpu_scores(W.c1(), "blosum62", mode)
    assert np.array_equal(got, np.array(golden["c1"]["scores"], np.int32))


@pytest.mark.parametrize("mode", MODES)
def test_edge_sets_match_reference(gpu, golden, mode):
    for e in golden["edge"]:
        wl = W.random_set(e["seed"], e["n"], e["lo"], e["hi"], alphabet=e["alphabet"].encode(),
                          extra=e["extra"].encode("latin-1"))
        for pad3 in (False, True):
            got = gpu_scores(wl, e["table"], mode, pad3)
            assert np.array_equal(got, np.array(e["scores"], np.int32)), (e["seed"], pad3)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("seed,n,lo,hi,table", [
    (41, 40, 1, 70, "blosum62"),        # single strips, tiny columns
    (42, 12, 480, 1100, "default"),     # strip boundaries at 512 / 1024 rows
    (43, 9, 1500, 2600, "pam250"),      # several strips, wide columns
    (44, 33, 500, 530, "blosum45"),     # odd count: unpaired 16-bit task
    (45, 6, 5000, 7000, "blosum62"),    # 32-bit path (16-bit bound exceeded)
    (46, 51, 300, 560, "blosum62"),     # stacked rows pairs (rows <= 512) beside single ones
    (47, 20, 1, 512, "blosum90"),       # stacked rows pairs of every strip height
])
def test_random_sets_match_oracle(gpu, tables, mode, seed, n, lo, hi, table):
    alpha = b"ACGTN" if table == "default" else b"ARNDCQEGHILKMFPSTWYV"
    wl = W.random_set(seed, n, lo, hi, alphabet=alpha)
    got = gpu_scores(wl, table, mode)
    assert np.array_equal(got, oracle_scores(wl, table, tables))


@pytest.mark.parametrize("table", ["default", "blosum62", "blosum45", "blosum50", "blosum80", "blosum90", "pam250"])
def test_named_tables_take_16bit_lanes(gpu, tables, table):
    # Short sequences of letters fit the 16-bit lanes under every named table
    # (each table's letter block has smin = -g); the batched kernel must run
    # them there and stay exact.
    alpha = b"ACGTN" if table == "default" else b"ARNDCQEGHILKMFPSTWYVBZX"
    wl = W.random_set(60, 24, 200, 900, alphabet=alpha)
    got = gpu_scores(wl, table, _lib.MSA_NW_PERSISTENT)
    assert pairwise.last_stats().narrow_tasks > 0
    assert np.array_equal(got, oracle_scores(wl, table, tables))


def test_plain_and_persistent_agree_on_related_sequences(gpu):
    wl = W.c2(n=300)
    a = gpu_scores(wl, "blosum62", _lib.MSA_NW_PLAIN)
    b = gpu_scores(wl, "blosum62", _lib.MSA_NW_PERSISTENT)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["c2", "c4"])
def test_full_workload_samples_match_reference(gpu, golden, name):
    g = golden[name + "_sample"]
    wl = W.BY_NAME[name]()
    got = gpu_scores(wl, g["table"], _lib.MSA_NW_PERSISTENT)
    i, j = np.array(g["i"], np.int64), np.array(g["j"], np.int64)
    assert np.array_equal(got[i * (i - 1) // 2 + j], np.array(g["scores"], np.int32))


def test_c3_full_plain_equals_persistent_and_reference_sample(gpu, golden):
    g = golden["c3_sample"]
    wl = W.c3()
    pers = gpu_scores(wl, "default", _lib.MSA_NW_PERSISTENT)
    i, j = np.array(g["i"], np.int64), np.array(g["j"], np.int64)
    assert np.array_equal(pers[i * (i - 1) // 2 + j], np.array(g["scores"], np.int32))
    plain = gpu_scores(wl, "default", _lib.MSA_NW_PLAIN)
    assert np.array_equal(plain, pers)


def test_asymmetric_custom_table_uses_reference_orientation(gpu):
    rng = np.random.default_rng(7)
    m = rng.integers(-6, 7, (25, 25)).astype(np.int32)
    t = ScoringTable.custom(m, 3)
    wl = W.random_set(46, 20, 1, 90)
    got = gpu_scores(wl, t, _lib.MSA_NW_PERSISTENT)
    flat, offs, lens = wl.flat_units()
    want = O.oracle_nw_all_pairs(flat, offs, lens, m.reshape(-1), 1, 0, 3)
    assert np.array_equal(got, want)


def test_output_on_device(gpu, golden):
    import torch
    wl = W.c1()
    flat, offs, lens = wl.flat_units()
    lib = _lib.lib()
    h = ctypes.c_uint64()
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    _lib.check(lib.msa_seqs_upload(gpu.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                   lens.ctypes.data_as(u64), wl.n, ctypes.byref(h)), gpu.handle)
    out = torch.zeros(wl.n * (wl.n - 1) // 2, dtype=torch.int32, device="cuda:0")
    t = ScoringTable("blosum62")
    _lib.check(lib.msa_nw_all_pairs(gpu.handle, h.value, ctypes.byref(t._t), _lib.MSA_NW_PERSISTENT,
                                    ctypes.c_void_p(out.data_ptr()), 1), gpu.handle)
    torch.cuda.synchronize()
    lib.msa_seqs_release(gpu.handle, h.value)
    assert np.array_equal(out.cpu().numpy(), np.array(golden["c1"]["scores"], np.int32))


def test_gap_unit_with_pam250_is_rejected(gpu):
    wl = W.random_set(47, 5, 5, 10, extra=b"-")
    flat, offs, lens = wl.flat_units()
    with pytest.raises(_lib.MsaError) as ei:
        pairwise.score_units(flat, offs, lens, ScoringTable("pam250"))
    assert ei.value.status == _lib.MSA_ERR_UNDEFINED


def test_database_run_api(gpu, golden):
    db = Database()
    for k, s in enumerate(W.c1().seqs):
        db.add((f"s{k}", bytes(s)))
    dm = pairwise.run(db, table="blosum62", algorithm="default")
    want = golden["c1"]["scores"]
    assert dm.count == 16
    assert all(dm[i, j] == want[i * (i - 1) // 2 + j] for i in range(1, 16) for j in range(i))
    dm2 = pairwise.run(db, table="blosum62", algorithm="sequential")
    assert np.array_equal(dm.scores, dm2.scores)


def test_stats_and_launch_counts(gpu):
    wl = W.c2(n=200)
    before = gpu.launches
    gpu_scores(wl, "blosum62", _lib.MSA_NW_PERSISTENT)
    s = pairwise.last_stats()
    assert s.pairs == 200 * 199 // 2 and s.cells == wl.cells()
    assert s.launches >= 2 and gpu.launches - before == s.launches
    assert s.narrow_tasks > 0 and s.kernel_ms > 0


@pytest.mark.parametrize("tiles", [(16, 4), (16, 8), (32, 4), (32, 8)])
def test_every_tile_shape_matches_oracle(gpu, tables, tiles):
    wl = W.random_set(48, 23, 30, 2200, alphabet=b"ARNDCQEGHILKMFPSTWYV")
    want = oracle_scores(wl, "blosum62", tables)
    _lib.check(_lib.lib().msa_nw_set_tiles(gpu.handle, *tiles))
    try:
        got = gpu_scores(wl, "blosum62", _lib.MSA_NW_PERSISTENT)
    finally:
        _lib.lib().msa_nw_set_tiles(gpu.handle, 0, 0)
    assert np.array_equal(got, want)


def test_wide_rows_pairs_match_oracle(gpu, tables):
    # blosum62 lengths past the 16-bit bound run the rows pair in 32-bit lanes.
    wl = W.random_set(49, 7, 4200, 5000, alphabet=b"ARNDCQEGHILKMFPSTWYV")
    got = gpu_scores(wl, "blosum62", _lib.MSA_NW_PERSISTENT)
    assert np.array_equal(got, oracle_scores(wl, "blosum62", tables))
    assert pairwise.last_stats().narrow_tasks == 0


def test_repeated_call_replays_graph_with_identical_scores(gpu, tables):
    wl = W.random_set(50, 40, 50, 900)
    flat, offs, lens = wl.flat_units()
    lib = _lib.lib()
    h = ctypes.c_uint64()
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    _lib.check(lib.msa_seqs_upload(gpu.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                   lens.ctypes.data_as(u64), wl.n, ctypes.byref(h)), gpu.handle)
    t = ScoringTable("blosum62")
    outs, graphs = [], []
    for _ in range(3):
        out = np.zeros(wl.n * (wl.n - 1) // 2, np.int32)
        _lib.check(lib.msa_nw_all_pairs(gpu.handle, h.value, ctypes.byref(t._t), _lib.MSA_NW_PERSISTENT,
                                        out.ctypes.data_as(ctypes.c_void_p), 0), gpu.handle)
        outs.append(out)
        graphs.append(pairwise.last_stats().graph)
    lib.msa_seqs_release(gpu.handle, h.value)
    assert graphs == [1, 1, 1]
    want = oracle_scores(wl, "blosum62", tables)
    assert all(np.array_equal(o, want) for o in outs)


def _split_workload():
    # Uneven DNA lengths, plus sequences with END units inside (generic path).
    rng = np.random.Generator(np.random.PCG64(21))
    lens = W.c3_lengths(rng, 150, 0.75) // 4 + 50
    seqs = [W._dna(rng, int(L)) for L in lens]
    for k in (3, 77, 120):
        s = np.array(seqs[k], np.uint8)
        s[len(s) // 2] = ord("*")
        seqs[k] = s
    return W.Workload("split", seqs, "default", 21)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("nparts", [2, 3])
def test_parts_assemble_the_whole_matrix(gpu, mode, nparts):
    wl = _split_workload()
    flat, offs, lens = wl.flat_units()
    table = ScoringTable(wl.table)
    full = pairwise.score_units(flat, offs, lens, table, mode)
    owner = pairwise.part_of_pairs(flat, offs, lens, table, nparts)
    # Host output: each part writes only its own entries.
    acc = np.full_like(full, 0x7eadbeef)
    for p in range(nparts):
        before = acc.copy()
        pairwise.score_units_part(flat, offs, lens, table, p, nparts, out=acc, mode=mode)
        changed = acc != before
        assert not np.any(changed & (owner != p))
        assert np.array_equal(acc[owner == p], full[owner == p])
    assert np.array_equal(acc, full)


def test_parts_on_device_into_one_buffer(gpu):
    import torch

    from msa_b200 import runtime, shard
    wl = _split_workload()
    flat, offs, lens = wl.flat_units()
    table = ScoringTable(wl.table)
    full = pairwise.score_units(flat, offs, lens, table)
    ctx = runtime.context(0)
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    h = ctypes.c_uint64()
    _lib.check(_lib.lib().msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                          lens.ctypes.data_as(u64), wl.n, ctypes.byref(h)), ctx.handle)
    try:
        # Zero-filled partial triangles summed, as the multi-device exchange does.
        total = torch.zeros(len(full), dtype=torch.int32, device="cuda:0")
        for p in range(4):
            part = torch.zeros_like(total)
            torch.cuda.synchronize()   # the library scores on its own stream
            shard.score_part(ctx, h.value, table, p, 4, part.data_ptr())
            total += part
        torch.cuda.synchronize()
        assert np.array_equal(total.cpu().numpy(), full)
    finally:
        _lib.lib().msa_seqs_release(ctx.handle, h.value)


@pytest.mark.parametrize("mode", MODES)
def test_16bit_lanes_near_their_bound(gpu, golden, mode):
    # The 16-bit lanes hold T = H + g(i+j), the sum of s + 2g over an
    # alignment's matched cells. Matches +1, mismatches -2 and gap 1 make
    # s + 2g either 3 or 0: all-A against all-A drives T to 3*lc (0xffff at
    # lc = 21845, the largest column count the bound admits) and all-A against
    # all-C keeps it at 0, the floor. One more column must fall back to 32-bit
    # lanes, and so must a table whose mismatch costs more than two gaps.
    m = np.full((25, 25), -2, np.int32)
    np.fill_diagonal(m, 1)
    edge = ScoringTable.custom(m, 1)
    m = np.full((25, 25), -60, np.int32)
    np.fill_diagonal(m, 1)
    steep = ScoringTable.custom(m, 1)
    for table, lc, narrow in ((edge, 21845, True), (edge, 21846, False), (steep, 4000, False)):
        la = lc + 7
        seqs = [b"A" * la, b"A" * lc, b"C" * (lc - 3)]
        wl = W.Workload("edge", [np.frombuffer(s, np.uint8) for s in seqs], "default", 0)
        flat, offs, lens = wl.flat_units()
        got = pairwise.score_units(flat, offs, lens, table, mode)
        # (1,0): lc matches and 7 gaps; (2,0) and (2,1): every letter against a
        # gap or a mismatch (a mismatch costs at least two gaps).
        want = np.array([lc - (la - lc), -(la + lc - 3), -(lc + lc - 3)], np.int32)
        assert np.array_equal(got, want), (lc, got, want)
        if mode == _lib.MSA_NW_PERSISTENT:
            assert (pairwise.last_stats().narrow_tasks > 0) == narrow, lc


@pytest.mark.parametrize("mode", MODES)
def test_packed_profile_rows_at_their_byte_bound(gpu, mode):
    # Packed profile rows hold s + 2g in one byte. Match +1, mismatch -2 and
    # gap 127 make s + 2g reach 255 on matches, and the 257 columns of the
    # second sequence put T at 257 * 255 = 0xffff: the batched kernel must
    # still take 16-bit lanes (the 600-row strip has R = 20, so some of its
    # rows are packed). Gap 128 pushes s + 2g past a byte: 32-bit lanes.
    m = np.full((25, 25), -2, np.int32)
    np.fill_diagonal(m, 1)
    la, lc, lm = 600, 257, 250
    seqs = [b"A" * la, b"A" * lc, b"C" * lm]
    wl = W.Workload("edge", [np.frombuffer(s, np.uint8) for s in seqs], "default", 0)
    flat, offs, lens = wl.flat_units()
    for g, narrow in ((127, True), (128, False)):
        got = pairwise.score_units(flat, offs, lens, ScoringTable.custom(m, g), mode)
        # (1,0): lc matches and la - lc gaps; (2,0) and (2,1): every C against
        # an A (a mismatch costs less than two gaps), the rest gaps.
        want = np.array([lc - g * (la - lc), -2 * lm - g * (la - lm), -2 * lm - g * (lc - lm)], np.int32)
        assert np.array_equal(got, want), (g, got, want)
        if mode == _lib.MSA_NW_PERSISTENT:
            assert (pairwise.last_stats().narrow_tasks > 0) == narrow, g
