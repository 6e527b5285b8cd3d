"""Sequence database (src/database.{hpp,cpp}) and FASTA loading
(src/io/loader/parser/fasta.cpp:26-70, src/io/loader/database.cpp:31-34)."""
from __future__ import annotations

import itertools
from collections import namedtuple
from pathlib import Path

import numpy as np

from .sequence import Sequence

_anonymous = itertools.count(1)


class Database:
    """Ordered sequences with a description -> offset map (src/database.hpp:25-210)."""

    entry = namedtuple("entry", ["description", "contents"])

    def __init__(self):
        self._entries: list[Database.entry] = []
        self._index: dict[str, int] = {}

    # -- lookup
    def __getitem__(self, key):
        if isinstance(key, (int, np.integer)):
            if key < 0 or key >= len(self._entries):
                raise RuntimeError("database offset out of range")
            return self._entries[int(key)]
        if isinstance(key, bytes):
            key = key.decode()
        if isinstance(key, str):
            if key not in self._index:
                raise RuntimeError("cannot find key in database")
            return self._entries[self._index[key]]
        raise TypeError("could not find sequence")

    @property
    def count(self) -> int:
        return len(self._entries)

    def __len__(self) -> int:
        return len(self._entries)

    def __iter__(self):
        return iter(self._entries)

    # -- insertion (database::add, src/database.hpp:99-122)
    def _add(self, description: str, seq: Sequence) -> None:
        self._index[description] = len(self._entries)
        self._entries.append(Database.entry(description, seq))

    def add(self, target) -> None:
        if isinstance(target, dict):
            for item in target.items():
                self.add(item)
        elif isinstance(target, tuple):
            description, contents = target
            self._add(str(description), contents if isinstance(contents, Sequence) else Sequence(contents))
        elif isinstance(target, list):
            for item in target:
                self.add(item)
        elif isinstance(target, Sequence):
            self._add(f"anonymous#{next(_anonymous)}", target)
        elif isinstance(target, (str, bytes)):
            self._add(f"anonymous#{next(_anonymous)}", Sequence(target))
        else:
            raise TypeError("could not add sequence to database")

    def merge(self, other: "Database") -> None:
        start = len(self._entries)
        self._entries.extend(other._entries)
        for k in range(start, len(self._entries)):
            self._index[self._entries[k].description] = k

    def only(self, keys: list) -> "Database":
        if not all(type(k) is type(keys[0]) for k in keys):
            raise TypeError("cannot select sequences via different key types")
        out = Database()
        for key in sorted(set(keys)):
            e = self[key]
            out._add(e.description, e.contents)
        return out

    # -- device view
    def units(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Concatenated units, offsets and (padded) lengths, the flattened form
        of pairwise::database (src/pairwise/database.cu:24-50)."""
        lens = np.array([len(e.contents.units) for e in self._entries], np.uint64)
        offs = np.zeros(len(lens), np.uint64)
        if len(lens) > 1:
            offs[1:] = np.cumsum(lens[:-1])
        flat = np.concatenate([e.contents.units for e in self._entries]) if self._entries else np.zeros(0, np.uint8)
        return np.ascontiguousarray(flat, np.uint8), offs, lens

    # -- loading
    @staticmethod
    def load(*filenames) -> "Database":
        result = Database()
        for filename in filenames:
            result.merge(load_file(str(filename)))
        return result


def _extension(filename: str) -> str:
    # utils::extension (src/utils.hpp:263-267): text after the last '.', or the
    # whole name when there is none.
    return filename[filename.rfind(".") + 1:] if filename else ""


def load_file(filename: str) -> Database:
    ext = _extension(filename)
    if ext not in ("fa", "fasta"):
        raise RuntimeError(f"unknown database parser '{ext}'")
    return parse_fasta(filename)


def parse_fasta(filename: str) -> Database:
    """parser::fasta (src/io/loader/parser/fasta.cpp:26-70), with its stream
    semantics: a record's contents are the lines after its '>' line up to the
    next '>' line or the first empty line; '\\r' stays in the line."""
    p = Path(filename)
    if not p.is_file():
        raise RuntimeError(f"file does not exist or cannot be read '{filename}'")
    data = p.read_bytes()
    db = Database()
    pos = 0
    n = len(data)
    eof = False

    def getline():
        nonlocal pos, eof
        if pos >= n:
            eof = True
            return None
        k = data.find(b"\n", pos)
        if k < 0:
            line = data[pos:]
            pos = n
            eof = True
            return line
        line = data[pos:k]
        pos = k + 1
        return line

    while not eof:
        line = b""
        found = True
        while len(line) < 1 or line[0] != 0x3E:
            if eof:
                found = False
                break
            got = getline()
            if got is None:
                found = False
                break
            line = got
        if not found:
            break
        description = line[1:].decode("latin-1")
        contents = bytearray()
        while True:
            if pos < n and data[pos] == 0x3E:
                break
            got = getline()
            if got is None or len(got) == 0:
                break
            contents += got
        db._add(description, Sequence(bytes(contents)))
    return db
