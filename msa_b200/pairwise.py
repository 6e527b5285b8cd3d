"""Pairwise module: scoring tables, the distance matrix and `run`, with the
names and behaviour of src/pairwise/pairwise.{cuh,cpp}, src/pairwise/table.cu
and src/python/pairwise.pyx. Every algorithm name runs on the GPU through
libmsa_b200.so; there is no CPU implementation behind any of them.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Union

import numpy as np

from . import runtime
from ._lib import (MSA_NW_PERSISTENT, MSA_NW_PLAIN, MsaNwStats, MsaTable, check, lib)
from .database import Database
from .sequence import encode_units

# Algorithm names of the reference's dispatcher (src/pairwise/pairwise.cpp:26-35).
# The "sequential"/"distributed" family selects the plain per-bucket kernel, the
# rest the persistent batched kernel; both give identical scores.
ALGORITHMS = {
    "default": MSA_NW_PERSISTENT,
    "needleman": MSA_NW_PERSISTENT,
    "hybrid": MSA_NW_PERSISTENT,
    "needleman-hybrid": MSA_NW_PERSISTENT,
    "sequential": MSA_NW_PLAIN,
    "distributed": MSA_NW_PLAIN,
    "needleman-sequential": MSA_NW_PLAIN,
    "needleman-distributed": MSA_NW_PLAIN,
}


def list() -> "list[str]":  # noqa: A001 - mirrors pairwise.list() of the reference
    return sorted(ALGORITHMS)


def has(name: str) -> bool:
    return name in ALGORITHMS


class ScoringTable:
    """A substitution table plus linear gap penalty (src/pairwise/pairwise.cuh:124-182)."""

    def __init__(self, name: str | None = None):
        name = name if name is not None else "default"
        t = MsaTable()
        rc = lib().msa_table_make(name.encode("ascii"), ctypes.byref(t))
        if rc != 0:
            raise RuntimeError(f"unknown pairwise scoring table '{name}'")
        self.name = name
        self._t = t

    @classmethod
    def custom(cls, scores, penalty: int) -> "ScoringTable":
        obj = cls.__new__(cls)
        t = MsaTable()
        arr = np.asarray(scores, np.int32).reshape(625)
        for k in range(625):
            t.score[k] = int(arr[k])
        t.penalty = int(penalty)
        t.index = -1
        obj.name = "custom"
        obj._t = t
        return obj

    def __getitem__(self, offset: tuple):
        x, y = offset
        x = int(encode_units(x)[0]) if isinstance(x, str) else int(x)
        y = int(encode_units(y)[0]) if isinstance(y, str) else int(y)
        if x >= 25 or y >= 25 or x < 0 or y < 0:
            raise RuntimeError("scoring table offset out of range")
        return float(self._t.score[x * 25 + y])

    @property
    def penalty(self) -> float:
        return float(self._t.penalty)

    def matrix(self) -> np.ndarray:
        return np.array(self._t.score[:], np.int32).reshape(25, 25)

    @staticmethod
    def list() -> "list[str]":
        names = (ctypes.c_char_p * 32)()
        k = lib().msa_table_list(names, 32)
        return [names[i].decode() for i in range(k)]

    @staticmethod
    def has(name: str) -> bool:
        return bool(lib().msa_table_has(name.encode("ascii")))


class DistanceMatrix:
    """Packed strict lower triangle of pair scores (src/pairwise/pairwise.cuh:53-117):
    [i, j] reads buf[max*(max-1)/2 + min], 0 on the diagonal."""

    def __init__(self, score=(), count: int = 0):
        self.scores = np.asarray(score, np.float32).reshape(-1)
        self._count = int(count)

    @classmethod
    def from_int32(cls, tri: np.ndarray, count: int) -> "DistanceMatrix":
        m = cls((), count)
        m.scores = tri.astype(np.float32)   # exact: |score| < 2^24
        m.int_scores = tri
        return m

    def __getitem__(self, offset: tuple) -> float:
        a, b = int(offset[0]), int(offset[1])
        hi, lo = max(a, b), min(a, b)
        if hi == lo:
            return 0.0
        return float(self.scores[hi * (hi - 1) // 2 + lo])

    @property
    def count(self) -> int:
        return self._count

    def full(self) -> np.ndarray:
        n = self._count
        out = np.zeros((n, n), np.float32)
        if n > 1:
            ii, jj = np.tril_indices(n, -1)
            out[ii, jj] = self.scores[ii * (ii - 1) // 2 + jj]
            out[jj, ii] = out[ii, jj]
        return out


def last_stats(device: int | None = None) -> MsaNwStats:
    ctx = runtime.context(device)
    s = MsaNwStats()
    check(lib().msa_nw_last_stats(ctx.handle, ctypes.byref(s)))
    return s


def score_units(flat: np.ndarray, offs: np.ndarray, lens: np.ndarray, table: ScoringTable,
                mode: int = MSA_NW_PERSISTENT, device: int | None = None) -> np.ndarray:
    """Uploads unit sequences and scores all pairs; returns the int32 triangle."""
    ctx = runtime.context(device)
    n = len(lens)
    flat = np.ascontiguousarray(flat, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    lens = np.ascontiguousarray(lens, np.uint64)
    h = ctypes.c_uint64()
    u8 = ctypes.POINTER(ctypes.c_uint8)
    u64 = ctypes.POINTER(ctypes.c_uint64)
    check(lib().msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    try:
        out = np.zeros(n * (n - 1) // 2, np.int32)
        check(lib().msa_nw_all_pairs(ctx.handle, h.value, ctypes.byref(table._t), mode,
                                     out.ctypes.data_as(ctypes.c_void_p), 0), ctx.handle)
    finally:
        lib().msa_seqs_release(ctx.handle, h.value)
    return out


def part_of_pairs(flat: np.ndarray, offs: np.ndarray, lens: np.ndarray, table: ScoringTable,
                  nparts: int) -> np.ndarray:
    """The part (0..nparts-1) that scores each pair when a job is split over
    `nparts` devices (msa_nw_part_of_pairs); host only, no device needed."""
    n = len(lens)
    flat = np.ascontiguousarray(flat, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    lens = np.ascontiguousarray(lens, np.uint64)
    out = np.zeros(max(n * (n - 1) // 2, 1), np.uint32)
    check(lib().msa_nw_part_of_pairs(flat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                     offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                     lens.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n, ctypes.byref(table._t),
                                     nparts, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))))
    return out[: n * (n - 1) // 2]


def score_units_part(flat: np.ndarray, offs: np.ndarray, lens: np.ndarray, table: ScoringTable, part: int,
                     nparts: int, out: np.ndarray | None = None, mode: int = MSA_NW_PERSISTENT,
                     device: int | None = None) -> np.ndarray:
    """Scores the pairs of one part (msa_nw_all_pairs_part) into `out` (host
    int32 triangle; a zero-filled one if None); other entries are kept."""
    ctx = runtime.context(device)
    n = len(lens)
    flat = np.ascontiguousarray(flat, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    lens = np.ascontiguousarray(lens, np.uint64)
    if out is None:
        out = np.zeros(n * (n - 1) // 2, np.int32)
    h = ctypes.c_uint64()
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    check(lib().msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    try:
        check(lib().msa_nw_all_pairs_part(ctx.handle, h.value, ctypes.byref(table._t), mode, part, nparts,
                                          out.ctypes.data_as(ctypes.c_void_p), 0), ctx.handle)
    finally:
        lib().msa_seqs_release(ctx.handle, h.value)
    return out


def run(db: Database, table: Union[ScoringTable, str, None] = None,
        algorithm: Union[str, Callable] = "default", **kwargs) -> DistanceMatrix:
    """pairwise::run (src/pairwise/pairwise.cuh:231-244; src/python/pairwise.pyx:88-98)."""
    if table is None:
        table = ScoringTable()
    elif not isinstance(table, ScoringTable):
        table = ScoringTable(table)
    if callable(algorithm):
        return algorithm(db, table=table)
    if algorithm not in ALGORITHMS:
        raise RuntimeError(f"unknown pairwise algorithm '{algorithm}'")
    flat, offs, lens = db.units()
    tri = score_units(flat, offs, lens, table, ALGORITHMS[algorithm], kwargs.get("device"))
    return DistanceMatrix.from_int32(tri, db.count)
