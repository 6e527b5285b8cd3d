"""Phylogeny module: neighbor-joining guide trees with the names and result
shape of src/phylogeny/phylogeny.{cuh,cpp} and src/phylogeny/njoining/. Every
name runs the device kernel of libmsa_b200.so."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import runtime
from ._lib import (MSA_NJ_LINEAR, MSA_NJ_SYMMETRIC, MSA_TRI_F32_HOST, MSA_TRI_I32_HOST, UNDEFINED_REF, MsaOtu,
                   check, lib)
from .pairwise import DistanceMatrix

# src/phylogeny/phylogeny.cpp:26-41. The four names that select the linear
# matrix transform (hybrid_linear, sequential_linear: lines 30, 33, 38, 40)
# run the linear removal order; every other name the symmetric one.
ALGORITHMS = [
    "default", "distributed", "hybrid", "linear", "njoining", "njoining-distributed",
    "njoining-distributed-linear", "njoining-hybrid", "njoining-linear", "njoining-sequential",
    "njoining-sequential-linear", "njoining-symmetric", "sequential", "symmetric",
]
LINEAR = {"linear", "njoining-linear", "njoining-sequential-linear", "njoining-distributed-linear"}


def order_of(algorithm: str) -> int:
    """The removal order a phylogeny algorithm name selects."""
    if algorithm not in ALGORITHMS:
        raise RuntimeError(f"unknown phylogeny algorithm '{algorithm}'")
    return MSA_NJ_LINEAR if algorithm in LINEAR else MSA_NJ_SYMMETRIC

undefined = UNDEFINED_REF


@dataclass
class Node:
    """otu + hierarchy (src/phylogeny/phylogeny.cuh:171-180, src/hierarchy.hpp:46-47)."""
    id: int
    parent: int
    child: tuple
    distance: float
    level: int


class GuideTree:
    """2n-1 nodes: leaves 0..n-1, joins n..2n-2, root 2n-2 (src/phylogeny/tree.cuh)."""

    def __init__(self, parent, child0, child1, distance, level, leaves: int):
        self.parent = np.asarray(parent, np.uint32)
        self.child0 = np.asarray(child0, np.uint32)
        self.child1 = np.asarray(child1, np.uint32)
        self.distance = np.asarray(distance, np.float32)
        self.level = np.asarray(level, np.uint32)
        self.leaves = leaves

    def __len__(self) -> int:
        return len(self.parent)

    def __getitem__(self, ref: int) -> Node:
        return Node(int(ref), int(self.parent[ref]), (int(self.child0[ref]), int(self.child1[ref])),
                    float(self.distance[ref]), int(self.level[ref]))

    @property
    def root(self) -> int:
        return len(self.parent) - 1 if len(self.parent) else undefined

    def newick(self, names=None) -> str:
        if not len(self.parent):
            return ";"
        names = names or [str(k) for k in range(self.leaves)]

        def rec(r: int) -> str:
            if r < self.leaves:
                s = names[r]
            else:
                s = "(" + rec(int(self.child0[r])) + "," + rec(int(self.child1[r])) + ")"
            if r != self.root:
                s += ":" + repr(float(self.distance[r]))
            return s
        import sys
        sys.setrecursionlimit(max(10000, 4 * len(self.parent)))
        return rec(self.root) + ";"


def list() -> "list[str]":  # noqa: A001
    return sorted(ALGORITHMS)


def run_triangle(tri: np.ndarray, n: int, device: int | None = None, order: int = MSA_NJ_SYMMETRIC) -> GuideTree:
    """Neighbor-joining over a packed lower triangle (float32 or int32), in
    the symmetric (default) or linear removal order."""
    ctx = runtime.context(device)
    if n < 2:
        return GuideTree([], [], [], [], [], n)
    tri = np.ascontiguousarray(tri)
    if tri.dtype == np.int32:
        kind = MSA_TRI_I32_HOST
    else:
        tri = np.ascontiguousarray(tri, np.float32)
        kind = MSA_TRI_F32_HOST
    nodes = (MsaOtu * (2 * n - 1))()
    check(lib().msa_nj_order(ctx.handle, tri.ctypes.data_as(ctypes.c_void_p), kind, n, order, nodes), ctx.handle)
    arr = np.frombuffer(nodes, dtype=np.dtype([("parent", "<u4"), ("c0", "<u4"), ("c1", "<u4"),
                                               ("distance", "<f4"), ("level", "<u4")]))
    return GuideTree(arr["parent"], arr["c0"], arr["c1"], arr["distance"], arr["level"], n)


def run(matrix: DistanceMatrix, count: int | None = None, algorithm: str = "default",
        device: int | None = None) -> GuideTree:
    """phylogeny::run (src/phylogeny/phylogeny.cuh:245-258)."""
    order = order_of(algorithm)
    n = matrix.count if count is None else int(count)
    tri = getattr(matrix, "int_scores", None)
    if tri is None:
        tri = matrix.scores
    return run_triangle(tri, n, device, order)
