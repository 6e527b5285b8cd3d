"""Encoded sequences: the Python face of src/sequence.hpp and src/encoder.{hpp,cpp}.

Units are one byte each (codes 0..25); a sequence is padded with END units to
a multiple of 3, the reference's 3-units-per-block granularity
(src/sequence.hpp:101-104).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import UNIT_END, check, lib

BLOCK = 3


def encode_units(text: str | bytes) -> np.ndarray:
    """encoder::encode(char) per character (src/encoder.cpp:46-57), unpadded."""
    data = text.encode("ascii") if isinstance(text, str) else bytes(text)
    out = np.empty(len(data), np.uint8)
    if len(data):
        check(lib().msa_encode(data, len(data), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
    return out


def decode_units(units: np.ndarray) -> str:
    units = np.ascontiguousarray(units, np.uint8)
    buf = ctypes.create_string_buffer(len(units) + 1)
    if len(units):
        check(lib().msa_decode(units.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), len(units), buf))
    return buf.raw[: len(units)].decode("ascii")


def pad_units(units: np.ndarray) -> np.ndarray:
    pad = (-len(units)) % BLOCK
    if pad:
        units = np.concatenate([units, np.full(pad, UNIT_END, np.uint8)])
    return units


def encode(sequence: str) -> str:
    """Encodes and decodes back, padded to a block multiple (src/python/sequence.pyx `encode`)."""
    return decode_units(pad_units(encode_units(sequence)))


class Sequence:
    """An encoded sequence (src/sequence.hpp:24-129)."""

    padding = "*"   # decode of the END unit

    __slots__ = ("units", "raw_length")

    def __init__(self, contents: str | bytes | np.ndarray = b""):
        if isinstance(contents, np.ndarray):
            units = np.ascontiguousarray(contents, np.uint8)
        elif isinstance(contents, (str, bytes)):
            units = encode_units(contents)
        else:
            raise TypeError("unexpected argument type")
        self.raw_length = len(units)
        self.units = pad_units(units)

    def __getitem__(self, offset: int) -> str:
        if offset < 0 or offset >= len(self.units):
            raise IndexError("sequence offset out of range")
        return decode_units(self.units[offset:offset + 1])

    def __str__(self) -> str:
        return decode_units(self.units)

    def __len__(self) -> int:
        return len(self.units)

    @property
    def length(self) -> int:
        """Padded length, 3 * blocks (src/sequence.hpp:101-104)."""
        return len(self.units)

    @property
    def blocks(self) -> int:
        return len(self.units) // BLOCK

    def packed(self) -> np.ndarray:
        """The reference's packed blocks: units at bits 1, 6, 11 of a uint16,
        bit 0 set on a block that runs past the sequence (src/encoder.cpp:76-98)."""
        u = self.units.reshape(-1, BLOCK).astype(np.uint16)
        out = (u[:, 0] << 1) | (u[:, 1] << 6) | (u[:, 2] << 11)
        if len(out) and self.raw_length % BLOCK:
            out[-1] |= 1
        return out.astype(np.uint16)

    @classmethod
    def from_blocks(cls, blocks: np.ndarray) -> "Sequence":
        blocks = np.ascontiguousarray(blocks, np.uint16)
        units = np.empty(3 * len(blocks), np.uint8)
        if len(blocks):
            check(lib().msa_unpack_blocks(blocks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), len(blocks),
                                          units.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        seq = cls(units)
        if len(blocks) and blocks[-1] & 1:
            # sequence::unpadded (src/sequence.hpp:110-119): trailing END units of
            # the flagged last block are padding.
            k = len(units)
            while k > len(units) - BLOCK + 1 and units[k - 1] == UNIT_END:
                k -= 1
            seq.raw_length = k
        return seq

    def __eq__(self, other) -> bool:
        return isinstance(other, Sequence) and np.array_equal(self.units, other.units)

    def __repr__(self) -> str:
        return f"Sequence({str(self)!r})"
