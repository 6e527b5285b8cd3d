"""ORACLE — test infrastructure only.

ctypes access to the two checkers built by oracle/Makefile:
  * liboracle.so          — the plain-C restatement (nw_oracle.c);
  * _ref/libmuseqa_ref.so — the reference's own CPU code (Museqa's
    needleman::sequential and njoining::sequential_symmetric, compiled from
    its sources; ref_harness.cpp drives it).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or to time the reference.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# The reference project's root (its src/, test/ and db/ directories), present
# only where the checker libraries are built; MSA_REFERENCE overrides it.
REFERENCE_ROOT = Path(os.environ.get("MSA_REFERENCE", "/root/reference"))
RESTATEMENT = HERE / "liboracle.so"
REFERENCE = HERE / "_ref" / "libmuseqa_ref.so"
# The reference-side binding of libmsa_b200.so (ref_b200.cpp): Museqa's own
# algorithm interfaces implemented over the C ABI, linked with the reference.
BINDING = HERE / "_ref" / "libmuseqa_b200.so"

_vp = ctypes.c_void_p


def _load(path: Path):
    if not path.exists():
        return None
    return ctypes.CDLL(str(path), mode=os.RTLD_LOCAL)


_ref = None
_res = None


def reference():
    """The compiled reference, or None when it was not built."""
    global _ref
    if _ref is None:
        _ref = _load(REFERENCE)
        if _ref is not None:
            _ref.ref_last_error.restype = ctypes.c_char_p
            _ref.ref_nw_all_pairs.argtypes = [ctypes.c_int, _vp, _vp, ctypes.c_char_p, _vp]
            _ref.ref_nw_pairs.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_char_p, ctypes.c_int, _vp]
            _ref.ref_nj.argtypes = [ctypes.c_int, _vp, ctypes.c_char_p, _vp, _vp, _vp, _vp, _vp]
            _ref.ref_encode.argtypes = [ctypes.c_char_p, ctypes.c_uint64, _vp]
            _ref.ref_encode.restype = ctypes.c_int64
            _ref.ref_fasta.argtypes = [ctypes.c_char_p, _vp, ctypes.c_uint64, _vp, ctypes.c_uint64]
            _ref.ref_fasta.restype = ctypes.c_int64
            _ref.ref_table.argtypes = [ctypes.c_char_p, _vp, _vp]
            for f in ("ref_table_list", "ref_pairwise_list", "ref_phylogeny_list"):
                getattr(_ref, f).argtypes = [_vp, ctypes.c_uint64]
                getattr(_ref, f).restype = ctypes.c_int64
    return _ref


_bind = None


def binding():
    """The reference-side binding library, or None when it was not built."""
    global _bind
    if _bind is None:
        if reference() is None:
            return None
        _bind = _load(BINDING)
        if _bind is not None:
            _bind.b200_ref_last_error.restype = ctypes.c_char_p
            _bind.b200_ref_nw_all_pairs.argtypes = [ctypes.c_int, _vp, _vp, ctypes.c_char_p, _vp, _vp]
            _bind.b200_ref_nj.argtypes = [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_char_p, _vp, _vp]
    return _bind


def binding_nw_all_pairs(seqs: list, table: str):
    """(scores of the needleman_b200 algorithm object, scores of
    pairwise::run(db, table, "sequential")) on the same reference database."""
    lib = binding()
    n = len(seqs)
    arr, lens = _cstrs(seqs)
    a = np.zeros(n * (n - 1) // 2, np.float32)
    b = np.zeros(n * (n - 1) // 2, np.float32)
    if lib.b200_ref_nw_all_pairs(n, ctypes.cast(arr, _vp), _ptr(lens), table.encode(), _ptr(a), _ptr(b)):
        raise RuntimeError(lib.b200_ref_last_error().decode())
    return a, b


def binding_nj(tri: np.ndarray, n: int, linear: bool, ref_name: str):
    """(tree of the njoining_b200 algorithm object, tree of
    phylogeny::run(matrix, n, ref_name)), each as 2n-1 rows of (parent,
    child0, child1, distance bits, level)."""
    lib = binding()
    tri = np.ascontiguousarray(tri, np.float32)
    m = max(2 * n - 1, 1)
    a = np.zeros((m, 5), np.uint32)
    b = np.zeros((m, 5), np.uint32)
    if lib.b200_ref_nj(n, _ptr(tri), int(linear), ref_name.encode(), _ptr(a), _ptr(b)):
        raise RuntimeError(lib.b200_ref_last_error().decode())
    return a, b


def restatement():
    global _res
    if _res is None:
        _res = _load(RESTATEMENT)
        if _res is not None:
            _res.oracle_nw_pair.argtypes = [_vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int32, _vp]
            _res.oracle_nw_all_pairs.argtypes = [ctypes.c_int64, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int32, _vp]
            _res.oracle_nj.argtypes = [ctypes.c_int64, _vp] + [_vp] * 7
            _res.oracle_nj_order.argtypes = [ctypes.c_int64, _vp, ctypes.c_int] + [_vp] * 7
            _res.oracle_encode_char.argtypes = [ctypes.c_char]
            _res.oracle_encode_char.restype = ctypes.c_uint8
    return _res


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


# ------------------------------------------------------------ reference calls

def _cstrs(seqs):
    arr = (ctypes.c_char_p * len(seqs))(*[bytes(s) for s in seqs])
    lens = np.array([len(s) for s in seqs], np.uint64)
    return arr, lens


def ref_nw_all_pairs(seqs: list, table: str) -> np.ndarray:
    lib = reference()
    n = len(seqs)
    arr, lens = _cstrs(seqs)
    out = np.zeros(n * (n - 1) // 2, np.float32)
    rc = lib.ref_nw_all_pairs(n, ctypes.cast(arr, _vp), _ptr(lens), table.encode(), _ptr(out))
    if rc:
        raise RuntimeError(lib.ref_last_error().decode())
    return out


def ref_nw_pairs(seqs: list, first: np.ndarray, second: np.ndarray, table: str, threads: int = 1) -> np.ndarray:
    lib = reference()
    arr, lens = _cstrs(seqs)
    first = np.ascontiguousarray(first, np.int32)
    second = np.ascontiguousarray(second, np.int32)
    out = np.zeros(len(first), np.float32)
    rc = lib.ref_nw_pairs(ctypes.cast(arr, _vp), _ptr(lens), _ptr(first), _ptr(second), len(first),
                          table.encode(), threads, _ptr(out))
    if rc:
        raise RuntimeError(lib.ref_last_error().decode())
    return out


def ref_nj(tri: np.ndarray, n: int, algorithm: str = "sequential") -> dict:
    lib = reference()
    tri = np.ascontiguousarray(tri, np.float32)
    m = max(2 * n - 1, 1)
    P, C0, C1, L = (np.zeros(m, np.uint32) for _ in range(4))
    D = np.zeros(m, np.float32)
    rc = lib.ref_nj(n, _ptr(tri), algorithm.encode(), _ptr(P), _ptr(C0), _ptr(C1), _ptr(D), _ptr(L))
    if rc:
        raise RuntimeError(lib.ref_last_error().decode())
    return {"parent": P, "child0": C0, "child1": C1, "distance": D, "level": L}


def ref_table(name: str):
    lib = reference()
    t = np.zeros(625, np.float32)
    p = np.zeros(1, np.float32)
    if lib.ref_table(name.encode(), _ptr(t), _ptr(p)):
        raise RuntimeError(lib.ref_last_error().decode())
    return t.reshape(25, 25), float(p[0])


def ref_list(kind: str) -> list:
    lib = reference()
    buf = ctypes.create_string_buffer(8192)
    k = getattr(lib, f"ref_{kind}_list")(ctypes.cast(buf, _vp), 8192)
    return [s.decode() for s in buf.raw.split(b"\0")[:k]]


def ref_encode_blocks(text: bytes) -> np.ndarray:
    lib = reference()
    out = np.zeros(len(text) // 3 + 2, np.uint16)
    k = lib.ref_encode(text, len(text), _ptr(out))
    return out[:k]


def ref_fasta(filename: str):
    lib = reference()
    cap = 1 << 26
    d = ctypes.create_string_buffer(cap)
    c = ctypes.create_string_buffer(cap)
    k = lib.ref_fasta(filename.encode(), ctypes.cast(d, _vp), cap, ctypes.cast(c, _vp), cap)
    if k < 0:
        raise RuntimeError(lib.ref_last_error().decode())
    descs = [s.decode("latin-1") for s in d.raw.split(b"\0")[:k]]
    conts = [s.decode("latin-1") for s in c.raw.split(b"\0")[:k]]
    return list(zip(descs, conts))


# ------------------------------------------------------------ restatement calls

def table_block(golden: dict | None = None) -> np.ndarray:
    """The seven built-in tables in the reference's storage order, int32 [7*625]:
    from the golden fixture (written by the reference) or the compiled reference."""
    if golden is not None:
        return np.concatenate([np.array(t["scores"], np.int32) for t in golden["tables"]])
    order = ["default", "blosum62", "blosum45", "blosum50", "blosum80", "blosum90", "pam250"]
    return np.concatenate([ref_table(n)[0].reshape(-1) for n in order]).astype(np.int32)


def oracle_nw_all_pairs(units: np.ndarray, offs: np.ndarray, lens: np.ndarray, tables: np.ndarray,
                        ntables: int, table: int, penalty: int) -> np.ndarray:
    lib = restatement()
    n = len(lens)
    out = np.zeros(n * (n - 1) // 2, np.int32)
    units = np.ascontiguousarray(units, np.uint8)
    offs = np.ascontiguousarray(offs, np.uint64)
    lens = np.ascontiguousarray(lens, np.uint64)
    tables = np.ascontiguousarray(tables, np.int32)
    rc = lib.oracle_nw_all_pairs(n, _ptr(units), _ptr(offs), _ptr(lens), _ptr(tables), ntables, table,
                                 penalty, _ptr(out))
    if rc:
        raise RuntimeError(f"oracle_nw_all_pairs failed ({rc})")
    return out


NJ_ORDER = {"symmetric": 0, "linear": 1}


def oracle_nj(tri: np.ndarray, n: int, order: str = "symmetric") -> dict:
    """The restated NJ; `order` is the removal order: "symmetric"
    (sequential_symmetric) or "linear" (sequential_linear)."""
    lib = restatement()
    tri = np.ascontiguousarray(tri, np.float32)
    m = max(2 * n - 1, 1)
    P, C0, C1, L = (np.zeros(m, np.uint32) for _ in range(4))
    D = np.zeros(m, np.float32)
    jx = np.zeros(max(n - 1, 1), np.uint32)
    jy = np.zeros(max(n - 1, 1), np.uint32)
    rc = lib.oracle_nj_order(n, _ptr(tri), NJ_ORDER[order], _ptr(P), _ptr(C0), _ptr(C1), _ptr(D), _ptr(L),
                             _ptr(jx), _ptr(jy))
    if rc:
        raise RuntimeError(f"oracle_nj failed ({rc})")
    return {"parent": P, "child0": C0, "child1": C1, "distance": D, "level": L}


TABLE_INDEX = {"default": 0, "blosum62": 1, "blosum45": 2, "blosum50": 3, "blosum80": 4, "blosum90": 5,
               "pam250": 6}
PENALTY = {"default": 1, "blosum62": 4, "blosum45": 5, "blosum50": 5, "blosum80": 6, "blosum90": 6, "pam250": 8}
