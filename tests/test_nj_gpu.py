"""Neighbor-joining on the GPU through the C ABI, checked bit-exact (joins,
levels and branch-length bits) against the reference's tree (golden) and the
oracle restatement."""
import json
from pathlib import Path

import numpy as np
import pytest

from msa_b200 import _lib, phylogeny
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def assert_same_tree(tree, want: dict):
    assert tree.parent.tolist() == list(want["parent"])
    assert tree.child0.tolist() == list(want["child0"])
    assert tree.child1.tolist() == list(want["child1"])
    assert tree.level.tolist() == list(want["level"])
    bits = want.get("distance_bits")
    if bits is None:
        bits = np.asarray(want["distance"], np.float32).view(np.uint32).tolist()
    assert tree.distance.view(np.uint32).tolist() == list(bits)


def test_c1_tree_matches_reference(gpu, golden):
    tri = np.array(golden["c1"]["scores"], np.int32)
    assert_same_tree(phylogeny.run_triangle(tri, 16), golden["c1"]["tree"])
    # float input of the same values
    assert_same_tree(phylogeny.run_triangle(tri.astype(np.float32), 16), golden["c1"]["tree"])


def _matrix(n, kind, rng):
    m = n * (n - 1) // 2
    if kind == "ties":       # few distinct values: ties decide most joins
        return rng.integers(-3, 4, m).astype(np.float32)
    if kind == "wide":
        return rng.integers(-5000, 5000, m).astype(np.float32)
    if kind == "fraction":   # full 24-bit significands
        return (rng.standard_normal(m) * 1000).astype(np.float32)
    if kind == "tiny":       # subnormal distances: halved updates lose bits, so the
        # new row sum takes the double-precision fold
        return (rng.integers(1, 64, m) * np.float32(1.4e-45)).astype(np.float32)
    raise ValueError(kind)


# Odd sizes exercise row pitches padded to 4 floats; 2100 is larger than the
# pipeline-scale workload.
@pytest.mark.parametrize("n,kind", [(2, "ties"), (3, "ties"), (4, "wide"), (5, "ties"), (6, "wide"), (9, "ties"),
                                    (17, "ties"), (33, "wide"), (130, "fraction"), (200, "ties"), (300, "tiny"),
                                    (700, "wide"), (1100, "ties"), (1500, "wide"), (2100, "fraction")])
def test_random_matrices_match_oracle(gpu, n, kind):
    tri = _matrix(n, kind, np.random.default_rng(1000 + n))
    want = O.oracle_nj(tri, n)
    assert_same_tree(phylogeny.run_triangle(tri, n), want)


LINEAR = _lib.MSA_NJ_LINEAR


def test_c1_linear_tree_matches_reference(gpu, golden):
    """njoining-sequential-linear's tree (the reference's, from the golden
    fixture) through the linear removal order of the device kernel."""
    tri = np.array(golden["c1"]["scores"], np.int32)
    assert_same_tree(phylogeny.run_triangle(tri, 16, order=LINEAR), golden["c1"]["tree_linear"])


@pytest.mark.parametrize("n,kind", [(2, "ties"), (3, "ties"), (4, "wide"), (5, "ties"), (6, "wide"), (9, "ties"),
                                    (17, "ties"), (33, "wide"), (60, "ties"), (120, "ties"), (130, "fraction"),
                                    (200, "ties"), (300, "tiny"), (700, "wide"), (1100, "ties"), (1500, "wide"),
                                    (2100, "fraction")])
def test_random_matrices_linear_order_match_oracle(gpu, n, kind):
    tri = _matrix(n, kind, np.random.default_rng(1000 + n))
    want = O.oracle_nj(tri, n, "linear")
    assert_same_tree(phylogeny.run_triangle(tri, n, order=LINEAR), want)


def test_every_name_runs_its_order(gpu, golden):
    """The four names of the linear transform (src/phylogeny/phylogeny.cpp:30,
    33, 38, 40) give sequential_linear's tree, the ten others
    sequential_symmetric's."""
    from msa_b200 import pairwise
    tri = np.array(golden["c1"]["scores"], np.int32)
    dm = pairwise.DistanceMatrix(tri.astype(np.float32), 16)
    for name in phylogeny.list():
        want = golden["c1"]["tree_linear"] if name in phylogeny.LINEAR else golden["c1"]["tree"]
        assert_same_tree(phylogeny.run(dm, 16, algorithm=name), want)


def test_all_nan_matrix_is_an_error(gpu):
    from msa_b200._lib import MsaError
    tri = np.full(10 * 9 // 2, np.nan, np.float32)
    with pytest.raises(MsaError):
        phylogeny.run_triangle(tri, 10)
    # the context stays usable
    tri = _matrix(10, "wide", np.random.default_rng(7))
    assert_same_tree(phylogeny.run_triangle(tri, 10), O.oracle_nj(tri, 10))


def test_stats_report_the_cluster(gpu):
    import ctypes
    from msa_b200 import _lib, runtime
    tri = _matrix(400, "wide", np.random.default_rng(8))
    phylogeny.run_triangle(tri, 400)
    ns = _lib.MsaNjStats()
    _lib.check(_lib.lib().msa_nj_last_stats(runtime.context(0).handle, ctypes.byref(ns)))
    assert ns.n == 400 and ns.cluster in (2, 4, 8, 16)
    assert ns.kernel_ms > 0 and ns.cycles_fold > 0 and ns.cycles_scan > 0


def test_c4_tree_matches_reference(gpu):
    p = GOLDEN / "golden_c4.json"
    if not p.exists():
        pytest.skip("golden_c4.json not generated")
    g = json.loads(p.read_text())
    import hashlib
    from msa_b200 import ScoringTable, pairwise
    from msa_b200 import workloads as W
    wl = W.c4()
    flat, offs, lens = wl.flat_units()
    tri = pairwise.score_units(flat, offs, lens, ScoringTable("blosum62"))
    assert hashlib.sha256(tri.tobytes()).hexdigest() == g["scores_sha256"]
    assert_same_tree(phylogeny.run_triangle(tri, wl.n), g["tree"])
    if "tree_linear" in g:
        assert_same_tree(phylogeny.run_triangle(tri, wl.n, order=LINEAR), g["tree_linear"])


def test_small_inputs():
    assert len(phylogeny.run_triangle(np.zeros(0, np.float32), 1)) == 0
    assert len(phylogeny.run_triangle(np.zeros(0, np.float32), 0)) == 0


def _set_clusters(clusters, min_count=0, wait_us=0, stall=0):
    from msa_b200 import runtime
    _lib.check(_lib.lib().msa_nj_set_clusters(runtime.context(0).handle, clusters, min_count, wait_us, stall))


def _last_stats():
    import ctypes
    from msa_b200 import runtime
    ns = _lib.MsaNjStats()
    _lib.check(_lib.lib().msa_nj_last_stats(runtime.context(0).handle, ctypes.byref(ns)))
    return ns


@pytest.mark.parametrize("order", [_lib.MSA_NJ_SYMMETRIC, _lib.MSA_NJ_LINEAR])
@pytest.mark.parametrize("n,kind", [(9, "ties"), (60, "ties"), (200, "ties"), (700, "wide"), (1500, "fraction")])
def test_helper_clusters_give_the_same_tree(gpu, order, n, kind):
    """Helper clusters scanning beside the joining one (from 8 OTUs on, so
    small matrices use them too) change nothing in the tree."""
    tri = _matrix(n, kind, np.random.default_rng(3000 + n))
    want = O.oracle_nj(tri, n, "linear" if order == _lib.MSA_NJ_LINEAR else "symmetric")
    try:
        for clusters in (1, 2, 4):
            _set_clusters(clusters, 8)
            assert_same_tree(phylogeny.run_triangle(tri, n, order=order), want)
            if clusters > 1 and n > 9:
                assert _last_stats().helper_clusters >= 1
    finally:
        _set_clusters(0)


def test_wait_between_clusters_runs_out_and_the_context_stays_usable(gpu):
    """With the joining cluster's hand-over withheld (test hook), the helpers'
    wait for it and then the joining cluster's wait for their candidates run
    out: the call fails with MSA_ERR_DEVICE_TIMEOUT, and the next call on the
    same context builds the right tree."""
    n = 300
    tri = _matrix(n, "wide", np.random.default_rng(77))
    raised = None
    try:
        _set_clusters(2, 8, 20000, 1)
        try:
            phylogeny.run_triangle(tri, n)
        except _lib.MsaError as e:
            raised = e
        if _last_stats().helper_clusters == 0:
            pytest.skip("no second cluster could be resident beside the first")
        assert raised is not None and raised.status == _lib.MSA_ERR_DEVICE_TIMEOUT
    finally:
        _set_clusters(0)
    assert_same_tree(phylogeny.run_triangle(tri, n), O.oracle_nj(tri, n))
