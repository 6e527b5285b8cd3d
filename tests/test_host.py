"""CPU-only tests of the host side: the C ABI library loads and exports every
declared symbol, and the encoder, tables, names and FASTA loading behave like
the reference's (checked against the compiled reference where present and
against the golden fixtures otherwise). No GPU work is issued here."""
import hashlib
import re
from pathlib import Path

import numpy as np
import pytest

import msa_b200
from msa_b200 import Database, ScoringTable, Sequence, encode, pairwise, phylogeny
from msa_b200 import _lib
from msa_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]


def _declared_functions():
    text = (ROOT / "include/msa_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(msa_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = _declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_declares_every_exported_function():
    assert set(_declared_functions()) <= set(_lib.EXPORTED)


def test_library_is_sm100a_only():
    # The embedded image is for sm_100a; cuobjdump-free check via the build flags.
    from msa_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_encoder_matches_reference_for_every_byte(ref):
    from oracle import oracle as O
    lib = O.restatement()
    chars = bytes(range(1, 256))
    got = msa_b200.sequence.encode_units(chars)
    want = np.array([lib.oracle_encode_char(bytes([c])) for c in chars], np.uint8)
    assert np.array_equal(got, want)
    # the compiled reference's packed blocks
    blocks = O.ref_encode_blocks(chars)
    assert np.array_equal(Sequence(chars).packed(), blocks)


@pytest.mark.parametrize("text", [b"", b"A", b"AC", b"ACG", b"acgtn*-xyz", b"MKV\rLL\n", b"-" * 7])
def test_block_packing_round_trip(ref, text):
    from oracle import oracle as O
    s = Sequence(text)
    assert np.array_equal(s.packed(), O.ref_encode_blocks(text))
    assert Sequence.from_blocks(s.packed()) == s


def test_sequence_api_like_reference():
    s = Sequence("MKVLAT")
    assert str(s) == "MKVLAT"
    assert s.length == 6
    assert [s[i] for i in range(6)] == list("MKVLAT")
    with pytest.raises(IndexError):
        s[s.length]
    t = Sequence("ACGTA")
    assert str(t) == "ACGTA*" and t.length == 6
    assert encode("acgTU") == "ACGTX*"
    assert Sequence.padding == "*"


def test_tables_match_golden(golden):
    for t in golden["tables"]:
        st = ScoringTable(t["name"])
        assert st.penalty == t["penalty"]
        assert st.matrix().reshape(-1).tolist() == t["scores"]
    assert ScoringTable.list() == golden["table_list"]
    assert ScoringTable.has("blosum62") and not ScoringTable.has("blosum99")
    with pytest.raises(RuntimeError, match="unknown pairwise scoring table"):
        ScoringTable("nope")


def test_tables_are_symmetric(golden):
    for t in golden["tables"]:
        m = np.array(t["scores"]).reshape(25, 25)
        assert np.array_equal(m, m.T)


def test_table_indexing_by_letter():
    t = ScoringTable("blosum62")
    assert t["W", "W"] == t[17, 17]
    with pytest.raises(RuntimeError):
        t[25, 0]


def test_algorithm_names_match_reference(golden):
    assert pairwise.list() == golden["pairwise_list"]
    assert phylogeny.list() == golden["phylogeny_list"]
    with pytest.raises(RuntimeError, match="unknown pairwise algorithm"):
        pairwise.run(Database(), algorithm="smith-waterman")


def test_distance_matrix_indexing():
    dm = pairwise.DistanceMatrix([1.0, 2.0, 3.0], 3)
    assert dm[0, 0] == 0 and dm[1, 0] == 1.0 and dm[0, 1] == 1.0
    assert dm[2, 0] == 2.0 and dm[2, 1] == 3.0 and dm.count == 3
    assert np.array_equal(dm.full(), dm.full().T)


def test_database_add_merge_only():
    db = Database()
    db.add({"s1": "ACGT", "s2": "MKV*"})
    db.add(("s3", "GG"))
    db.add(["TT", Sequence("CC")])
    assert db.count == 5
    assert db["s2"].description == "s2" and str(db["s2"].contents) == "MKV***"
    other = Database()
    other.add({"s4": "AAA", "s1": "CCC"})
    db.merge(other)
    assert db.count == 7 and str(db["s1"].contents) == "CCC"
    sub = db.only(["s3", "s4"])
    assert sub.count == 2
    with pytest.raises(TypeError):
        db.only(["s3", 1])
    with pytest.raises(RuntimeError):
        db["missing"]


def _write(tmp_path, name, data: bytes) -> str:
    p = tmp_path / name
    p.write_bytes(data)
    return str(p)


FASTA_CASES = {
    "plain.fasta": b">a one\nACGT\nGGCC\n>b\nMKV\n",
    "crlf.fa": b">a\r\nACGT\r\nGG\r\n>b\r\nTT\r\n",
    "blank.fasta": b"junk\n>a\nAC\n\nGT\n>b\nCC\n\n\n>c\nAA",
    "lower.fasta": b">x\nacgt-*1\n>y\n\n>z\nQ\n",
    "noeol.fasta": b">only\nACGTACGT",
}


@pytest.mark.parametrize("name", sorted(FASTA_CASES))
def test_fasta_parser_matches_reference(ref, tmp_path, name):
    from oracle import oracle as O
    fn = _write(tmp_path, name, FASTA_CASES[name])
    want = O.ref_fasta(fn)
    db = Database.load(fn)
    got = [(e.description, str(e.contents)) for e in db]
    assert got == want


def test_fasta_unknown_file_raises():
    with pytest.raises(RuntimeError):
        Database.load("unknown/file/path")


def test_reference_fixture_digests():
    # The reference's own loader test pins MD5s of decoded contents
    # (test/loader.py:16-34); check them where the reference tree is present.
    from oracle.oracle import REFERENCE_ROOT
    fx = REFERENCE_ROOT / "test" / "fixtures"
    if not fx.is_dir():
        pytest.skip("reference fixtures not present")
    db = Database.load(str(fx / "mock2.fasta"))
    assert db.count == 3
    digests = {e.description: hashlib.md5(str(e.contents).encode()).hexdigest() for e in db}
    assert digests["AF241168.1"] == "c638e233669d5a37e88eacfad7e3d435"
    assert digests["NC_001874.1"] == "95bd6fb267dcab96ea781e90dcabfbe4"


def test_workload_letters_encode_like_library():
    wl = W.random_set(3, 5, 10, 20, alphabet=b"ARNDCQEGHILKMFPSTWYVBJZXOU-*acgt")
    for s in wl.seqs:
        assert np.array_equal(W.letters_to_units(s), msa_b200.sequence.encode_units(bytes(s)))


def test_workload_shapes():
    c1 = W.c1()
    assert c1.n == 16 and c1.lengths().min() >= 100 and c1.lengths().max() <= 300
    c3 = W.c3(n=400)
    L = c3.lengths()
    assert L.min() >= 200 and L.max() <= 16000
    assert 1100 < np.median(L) < 2000


@pytest.mark.parametrize("text", [b"", b"A", b"ACGTACG", b"acgtn*-xyz"])
def test_encode_blocks_abi_matches_reference(ref, text):
    import ctypes
    from oracle import oracle as O
    out = np.zeros(max(1, (len(text) + 2) // 3), np.uint16)
    _lib.check(_lib.lib().msa_encode_blocks(text, len(text), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))))
    want = O.ref_encode_blocks(text)
    assert np.array_equal(out[:len(want)], want)


def test_bench_packed_row_fraction_replays_the_strip_plan():
    """bench.py's roofline weighs the batched kernel's packed profile rows by
    replaying its plan; check the replay against a pair-by-pair count on a
    small uneven workload (rows pairs of the length-sorted sequences, strips of
    32R rows with R even and at most 32, 8 floor(R/16) packed rows per lane)."""
    import sys
    root = Path(__file__).resolve().parents[1]
    if str(root) not in sys.path:
        sys.path.insert(0, str(root))
    import bench
    wl = W.random_set(90, 41, 20, 3000, alphabet=b"ACGT")
    e = np.sort(wl.lengths().astype(np.int64))[::-1]
    packed = total = 0.0
    for k in range((len(e) + 1) // 2):
        a1, a2 = 2 * k, min(2 * k + 1, len(e) - 1)
        nst = -(-int(e[a1]) // 1024)
        r = -(-int(e[a1]) // (32 * nst))
        r += r % 2
        for b in range(2 * k + 1, len(e)):
            for a in {a1, a2}:
                cells = float(e[a] * e[b])
                packed += cells * (8 * (r // 16)) / r
                total += cells
    assert bench.packed_row_fraction(wl) == pytest.approx(packed / total, rel=1e-12)
    assert 0.0 <= packed / total <= 0.5


def test_phylogeny_names_select_the_reference_order():
    """src/phylogeny/phylogeny.cpp:26-41: the linear transform for exactly four
    names; an unknown name raises the reference's message."""
    lin = {n for n in phylogeny.list() if phylogeny.order_of(n) == _lib.MSA_NJ_LINEAR}
    assert lin == {"linear", "njoining-linear", "njoining-sequential-linear", "njoining-distributed-linear"}
    assert len(phylogeny.list()) == 14
    with pytest.raises(RuntimeError, match="unknown phylogeny algorithm 'nope'"):
        phylogeny.order_of("nope")
