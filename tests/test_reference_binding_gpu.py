"""The reference-side binding (oracle/ref_b200.cpp): Museqa's own
pairwise::algorithm and phylogeny::algorithm interfaces implemented over
libmsa_b200.so's C ABI and compiled against the reference's headers. The
algorithm objects are called directly on a reference database and matrix and
must return what the reference's sequential algorithms return."""
import numpy as np
import pytest

from msa_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bind():
    if O.binding() is None:
        pytest.skip("reference-side binding (oracle/_ref/libmuseqa_b200.so) not built")
    return O


@pytest.mark.parametrize("case", ["c1", "end_units", "gap_units", "dna"])
def test_needleman_b200_equals_sequential(gpu, bind, case):
    wl, table = {
        "c1": (W.c1(), "blosum62"),
        "end_units": (W.random_set(11, 24, 0, 40, extra=b"*1\r. "), "blosum62"),
        "gap_units": (W.random_set(12, 24, 1, 40, extra=b"-"), "blosum62"),
        "dna": (W.random_set(18, 12, 500, 1100, alphabet=b"ACGT", extra=b"\r"), "default"),
    }[case]
    got, want = bind.binding_nw_all_pairs(wl.strings(), table)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("linear,ref_name", [(False, "sequential"), (True, "njoining-sequential-linear")])
def test_njoining_b200_equals_sequential(gpu, bind, golden, linear, ref_name):
    tri = np.array(golden["c1"]["scores"], np.float32)
    got, want = bind.binding_nj(tri, 16, linear, ref_name)
    assert np.array_equal(got, want)
    rng = np.random.default_rng(33)
    n = 33
    tri = rng.integers(-3, 4, n * (n - 1) // 2).astype(np.float32)   # tie-heavy
    got, want = bind.binding_nj(tri, n, linear, ref_name)
    assert np.array_equal(got, want)
