"""Pins the oracle (the C restatement in oracle/nw_oracle.c) to the reference:
against the committed golden fixtures (made by the reference itself) and, where
the compiled reference is present, against it directly on fresh inputs."""
import numpy as np
import pytest

from msa_b200 import workloads as W
from oracle import oracle as O


def restate(wl, table, pad3=False, tables=None):
    flat, offs, lens = wl.flat_units(pad3=pad3)
    return O.oracle_nw_all_pairs(flat, offs, lens, tables, 7, O.TABLE_INDEX[table], O.PENALTY[table])


@pytest.fixture(scope="module")
def tables(golden):
    return O.table_block(golden)


def test_golden_tables_match_reference(ref, golden):
    assert np.array_equal(O.table_block(golden), O.table_block())
    for t in golden["tables"]:
        assert O.PENALTY[t["name"]] == t["penalty"]


def test_restatement_matches_golden_c1(golden, tables):
    g = golden["c1"]
    got = restate(W.c1(), "blosum62", tables=tables)
    assert np.array_equal(got, np.array(g["scores"], np.int32))


def test_restatement_nj_matches_golden_c1(golden):
    g = golden["c1"]
    tri = np.array(g["scores"], np.float32)
    t = O.oracle_nj(tri, 16)
    for k in ("parent", "child0", "child1", "level"):
        assert t[k].tolist() == g["tree"][k]
    assert t["distance"].view(np.uint32).tolist() == g["tree"]["distance_bits"]


def test_restatement_matches_golden_edge_sets(golden, tables):
    for e in golden["edge"]:
        wl = W.random_set(e["seed"], e["n"], e["lo"], e["hi"], alphabet=e["alphabet"].encode(),
                          extra=e["extra"].encode("latin-1"))
        for pad3 in (False, True):
            got = restate(wl, e["table"], pad3, tables)
            assert np.array_equal(got, np.array(e["scores"], np.int32)), (e["seed"], pad3)


@pytest.mark.parametrize("name", ["c2", "c3", "c4"])
def test_restatement_matches_golden_samples(golden, tables, name):
    g = golden[name + "_sample"]
    wl = W.BY_NAME[name]()
    flat, offs, lens = wl.flat_units(pad3=False)
    tb = tables
    i, j = np.array(g["i"]), np.array(g["j"])
    if name == "c3":
        i, j = i[:12], j[:12]
    for a, b, want in zip(i, j, g["scores"]):
        sub_off = np.array([offs[b], offs[a]], np.uint64)
        sub_len = np.array([lens[b], lens[a]], np.uint64)
        got = O.oracle_nw_all_pairs(flat, sub_off, sub_len, tb, 7, O.TABLE_INDEX[g["table"]],
                                    O.PENALTY[g["table"]])
        assert int(got[0]) == want


@pytest.mark.parametrize("seed,table,extra", [(31, "blosum62", b""), (32, "default", b"*\r"),
                                              (33, "pam250", b"*"), (34, "blosum62", b"-*")])
def test_restatement_matches_reference_fresh(ref, tables, seed, table, extra):
    wl = W.random_set(seed, 22, 0, 50, extra=extra)
    want = O.ref_nw_all_pairs(wl.strings(), table)
    got = restate(wl, table, tables=tables)
    assert np.array_equal(got.astype(np.float32), want)


@pytest.mark.parametrize("n,kind", [(2, "ties"), (3, "ties"), (9, "ties"), (64, "ties"), (150, "wide"),
                                    (300, "neg")])
def test_restatement_nj_matches_reference(ref, n, kind):
    rng = np.random.default_rng(n)
    m = n * (n - 1) // 2
    tri = {"ties": rng.integers(-3, 4, m), "wide": rng.integers(-5000, 5000, m),
           "neg": -rng.integers(0, 100, m)}[kind].astype(np.float32)
    r = O.ref_nj(tri, n)
    o = O.oracle_nj(tri, n)
    for k in ("parent", "child0", "child1", "level"):
        assert np.array_equal(r[k], o[k])
    assert np.array_equal(r["distance"].view(np.uint32), o["distance"].view(np.uint32))


@pytest.mark.parametrize("n,kind", [(2, "ties"), (3, "ties"), (9, "ties"), (17, "ties"), (33, "ties"),
                                    (60, "ties"), (120, "ties"), (60, "wide"), (150, "wide"), (300, "neg")])
def test_restatement_nj_linear_matches_reference(ref, n, kind):
    """The linear removal order (njoining-sequential-linear) against the
    compiled reference; it differs from the symmetric order's tree on most of
    these inputs, so the two orders are told apart."""
    rng = np.random.default_rng(7000 + n)
    m = n * (n - 1) // 2
    tri = {"ties": rng.integers(-3, 4, m), "wide": rng.integers(-5000, 5000, m),
           "neg": -rng.integers(0, 100, m)}[kind].astype(np.float32)
    r = O.ref_nj(tri, n, "njoining-sequential-linear")
    o = O.oracle_nj(tri, n, "linear")
    for k in ("parent", "child0", "child1", "level"):
        assert np.array_equal(r[k], o[k]), k
    assert np.array_equal(r["distance"].view(np.uint32), o["distance"].view(np.uint32))


def test_linear_and_symmetric_orders_differ(ref):
    rng = np.random.default_rng(5)
    n = 33
    tri = rng.integers(-3, 4, n * (n - 1) // 2).astype(np.float32)
    a = O.oracle_nj(tri, n, "linear")
    b = O.oracle_nj(tri, n, "symmetric")
    assert not (np.array_equal(a["parent"], b["parent"]) and
                np.array_equal(a["distance"].view(np.uint32), b["distance"].view(np.uint32)))


def test_reference_scores_are_exact_integers(golden):
    for e in golden["edge"]:
        assert all(isinstance(v, int) for v in e["scores"])


def test_reference_binding_library_loads(ref):
    """The reference-side binding (oracle/ref_b200.cpp) links against the
    reference and libmsa_b200.so and exports its two test entry points."""
    lib = O.binding()
    assert lib is not None
    assert hasattr(lib, "b200_ref_nw_all_pairs") and hasattr(lib, "b200_ref_nj")
