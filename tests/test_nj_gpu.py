"""Neighbor-joining on the GPU through the C ABI, checked bit-exact (joins,
levels and branch-length bits) against the reference's tree (golden) and the
oracle restatement."""
import json
from pathlib import Path

import numpy as np
import pytest

from msa_b200 import phylogeny
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


@pytest.mark.parametrize("n,kind", [(2, "ties"), (3, "ties"), (4, "wide"), (17, "ties"), (200, "ties"),
                                    (700, "wide"), (1100, "ties"), (1500, "wide")])
def test_random_matrices_match_oracle(gpu, n, kind):
    rng = np.random.default_rng(1000 + n)
    m = n * (n - 1) // 2
    tri = {"ties": rng.integers(-3, 4, m), "wide": rng.integers(-5000, 5000, m)}[kind].astype(np.float32)
    want = O.oracle_nj(tri, n)
    assert_same_tree(phylogeny.run_triangle(tri, n), want)


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


def test_small_inputs():
    assert len(phylogeny.run_triangle(np.zeros(0, np.float32), 1)) == 0
    assert len(phylogeny.run_triangle(np.zeros(0, np.float32), 0)) == 0
