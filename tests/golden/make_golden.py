"""Generates the golden fixtures in this directory from the reference's own
CPU implementation (oracle/_ref/libmuseqa_ref.so, built from the reference
sources by `make -C oracle ref`).

    python tests/golden/make_golden.py [--c4 | --c4-tri FILE.npy]

Inputs are the seeded synthetic workloads of msa_b200.workloads; outputs are
the reference's float scores (stored as int32, they are integers) and trees.
--c4 also scores the full 2,000-sequence c4 set (about 1e12 cells; minutes
on all host cores) and builds its 2,000-taxon trees (symmetric and linear
removal orders). --c4-tri rebuilds only the trees, from a saved int32
triangle that must hash to the recorded reference matrix.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from msa_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def tri_sha(tri: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(tri, np.int32).tobytes()).hexdigest()


def tree_dict(t: dict) -> dict:
    return {"parent": t["parent"].tolist(), "child0": t["child0"].tolist(), "child1": t["child1"].tolist(),
            "distance_bits": t["distance"].view(np.uint32).tolist(), "level": t["level"].tolist()}


def sample_pairs(n: int, k: int, seed: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    i = rng.integers(1, n, k)
    j = (rng.random(k) * i).astype(np.int64)
    return i.astype(np.int32), j.astype(np.int32)


def full_set(wl, table: str) -> dict:
    tri = O.ref_nw_all_pairs(wl.strings(), table)
    assert np.all(tri == np.round(tri))
    return tri.astype(np.int32)


def edge_sets() -> list:
    """Small sets exercising the reference's END/GAP handling and empties."""
    specs = [
        (11, 24, 0, 40, b"ARNDCQEGHILKMFPSTWYV", b"*1\r. ", "blosum62"),
        (12, 24, 1, 40, b"ARNDCQEGHILKMFPSTWYV", b"-", "blosum62"),
        (13, 20, 0, 30, b"ACGTN", b"-*x", "default"),
        (14, 20, 0, 30, b"ARNDCQEGHILKMFPSTWYVBJZXOU", b"-*", "blosum45"),
        (15, 20, 0, 30, b"ARNDCQEGHILKMFPSTWYV", b"*", "pam250"),
        (16, 16, 0, 8, b"ACGT", b"", "default"),
        (17, 20, 1, 700, b"ARNDCQEGHILKMFPSTWYV", b"", "blosum80"),
        (18, 12, 500, 1100, b"ACGT", b"\r", "default"),
        (19, 20, 1, 60, b"ARNDCQEGHILKMFPSTWYV", b"", "blosum90"),
        (20, 20, 1, 60, b"ARNDCQEGHILKMFPSTWYV", b"", "blosum50"),
    ]
    out = []
    for seed, n, lo, hi, alpha, extra, table in specs:
        wl = W.random_set(seed, n, lo, hi, alphabet=alpha, extra=extra)
        tri = full_set(wl, table)
        out.append({"seed": seed, "n": n, "lo": lo, "hi": hi, "alphabet": alpha.decode(), "extra": extra.decode("latin-1"),
                    "table": table, "scores": tri.tolist()})
    return out


def main() -> None:
    if O.reference() is None:
        sys.exit("build the reference first: make -C oracle ref")
    t0 = time.time()
    gold = {"generator": "tests/golden/make_golden.py", "reference": "Museqa v0.1.1 needleman::sequential, "
            "njoining::sequential_symmetric and sequential_linear (oracle/_ref)"}

    order = ["default", "blosum62", "blosum45", "blosum50", "blosum80", "blosum90", "pam250"]
    gold["tables"] = []
    for name in order:
        t, pen = O.ref_table(name)
        gold["tables"].append({"name": name, "penalty": int(pen), "scores": t.astype(np.int32).reshape(-1).tolist()})
    gold["table_list"] = O.ref_list("table")
    gold["pairwise_list"] = O.ref_list("pairwise")
    gold["phylogeny_list"] = O.ref_list("phylogeny")

    c1 = W.c1()
    tri = full_set(c1, "blosum62")
    gold["c1"] = {"seed": 1, "table": "blosum62", "scores": tri.tolist(),
                  "tree": tree_dict(O.ref_nj(tri.astype(np.float32), c1.n)),
                  "tree_linear": tree_dict(O.ref_nj(tri.astype(np.float32), c1.n, "njoining-sequential-linear"))}
    gold["edge"] = edge_sets()

    # Sampled pairs of the large configurations.
    for name, fn, table, k in (("c2", W.c2, "blosum62", 300), ("c3", W.c3, "default", 48),
                               ("c4", W.c4, "blosum62", 300)):
        wl = fn()
        i, j = sample_pairs(wl.n, k, 100 + int(name[1]))
        if name == "c3":   # keep the CPU time bounded: drop the longest pairs
            L = wl.lengths()
            keep = (L[i] * L[j]) < 3.0e7
            i, j = i[keep], j[keep]
        sc = O.ref_nw_pairs(wl.strings(), i, j, table, threads=os.cpu_count() or 1)
        gold[name + "_sample"] = {"table": table, "i": i.tolist(), "j": j.tolist(),
                                  "scores": sc.astype(np.int32).tolist(), "cells": int(W.Workload.cells(wl))}
    (OUT / "golden.json").write_text(json.dumps(gold))
    print(f"golden.json written in {time.time() - t0:.1f}s")

    if "--c4" in sys.argv:
        # The c4 matrix scored by the reference (about 17 minutes on 8 host
        # threads), then its two guide trees.
        wl = W.c4()
        n = wl.n
        ii, jj = np.tril_indices(n, -1)
        order = np.lexsort((jj, ii))
        ii, jj = ii[order].astype(np.int32), jj[order].astype(np.int32)
        t1 = time.time()
        sc = O.ref_nw_pairs(wl.strings(), ii, jj, "blosum62", threads=os.cpu_count() or 1)
        tri = sc.astype(np.int32)
        t2 = time.time()
        c4 = {"n": n, "table": "blosum62", "scores_sha256": tri_sha(tri), "nw_seconds": t2 - t1,
              "threads": os.cpu_count()}
        c4_trees(c4, tri)
        print(f"golden_c4.json: NW {t2 - t1:.1f}s, NJ {c4['nj_seconds']:.2f}s")
    elif "--c4-tri" in sys.argv:
        # The c4 trees only, from a saved int32 triangle (.npy) whose SHA-256
        # must equal the one recorded when the reference scored c4, so the
        # trees are the reference's on the reference's own matrix.
        path = sys.argv[sys.argv.index("--c4-tri") + 1]
        tri = np.load(path).astype(np.int32)
        c4 = json.loads((OUT / "golden_c4.json").read_text())
        if tri_sha(tri) != c4["scores_sha256"]:
            raise SystemExit(f"{path} is not the reference's c4 matrix (SHA-256 differs)")
        c4_trees(c4, tri)
        print(f"golden_c4.json trees rewritten, NJ {c4['nj_seconds']:.2f}s")


def c4_trees(c4: dict, tri: np.ndarray) -> None:
    """Adds the reference's symmetric (`tree`) and linear (`tree_linear`)
    guide trees of the c4 matrix to `c4` and writes golden_c4.json."""
    n = c4["n"]
    t0 = time.time()
    c4["tree"] = tree_dict(O.ref_nj(tri.astype(np.float32), n))
    c4["nj_seconds"] = time.time() - t0
    c4["tree_linear"] = tree_dict(O.ref_nj(tri.astype(np.float32), n, "njoining-sequential-linear"))
    (OUT / "golden_c4.json").write_text(json.dumps(c4))


if __name__ == "__main__":
    main()
