"""Seeded synthetic workloads with the shapes of the five benchmark
configurations (no public dataset is involved; every input is generated here
from an explicit seed with numpy's PCG64).

    c1  16 protein sequences, lengths U[100,300], iid residues; blosum62.
    c2  1,000 proteins derived from one 500-residue ancestor: per-descendant
        substitution rate U[0.10,0.30], indel rate 0.02 (50/50 insertion/
        deletion, lengths geometric with mean 3); blosum62.
    c3  4,000 DNA sequences over ACGT with 1% N, lengths log-normal with median
        1,500 and sigma 0.75, clipped to [200,16000]; the +1/-1 `default` table.
    c4  2,000 proteins in 20 clades of 100: clade ancestors diverge 40% from a
        1,200-residue root and are cut or extended to a clade length
        U[200,1200]; members diverge 10% with indel rate 0.02; blosum62.
    c5  serving jobs: n U[8,512], lengths U[50,2000], half protein (blosum62,
        as c1) and half DNA (`default`, as c3), one seed per job.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

AMINO = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", np.uint8)
DNA = np.frombuffer(b"ACGT", np.uint8)

# Letter -> unit (encoder::encode, src/encoder.cpp:27-57), vectorised.
_LUT = np.full(256, 0x18, np.uint8)
for _i, _u in enumerate([0x00, 0x14, 0x01, 0x06, 0x08, 0x0E, 0x03, 0x09, 0x0A, 0x15, 0x0C, 0x0B, 0x0D,
                         0x05, 0x17, 0x0F, 0x07, 0x04, 0x10, 0x02, 0x17, 0x13, 0x11, 0x17, 0x12, 0x16]):
    _LUT[ord("A") + _i] = _u
    _LUT[ord("a") + _i] = _u
_LUT[ord("-")] = 0x19


def letters_to_units(letters: np.ndarray) -> np.ndarray:
    return _LUT[letters]


@dataclass
class Workload:
    name: str
    seqs: list            # list of uint8 letter arrays
    table: str
    seed: int

    @property
    def n(self) -> int:
        return len(self.seqs)

    def lengths(self) -> np.ndarray:
        return np.array([len(s) for s in self.seqs], np.int64)

    def cells(self) -> int:
        """Sum over pairs of L_i * L_j with unpadded lengths (the GCUPS numerator)."""
        L = self.lengths().astype(np.float64)
        return int(round((L.sum() ** 2 - (L * L).sum()) / 2))

    def flat_units(self, pad3: bool = True):
        """Concatenated units, offsets, lengths (each padded to a multiple of 3 with END)."""
        parts, lens = [], []
        for s in self.seqs:
            u = letters_to_units(s)
            if pad3 and len(u) % 3:
                u = np.concatenate([u, np.full(3 - len(u) % 3, 0x18, np.uint8)])
            parts.append(u)
            lens.append(len(u))
        lens = np.array(lens, np.uint64)
        offs = np.zeros(len(lens), np.uint64)
        if len(lens) > 1:
            offs[1:] = np.cumsum(lens[:-1])
        flat = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
        return np.ascontiguousarray(flat), offs, lens

    def strings(self) -> list:
        return [bytes(s) for s in self.seqs]


def _mutate(rng, seq, sub_rate, indel_rate, alphabet):
    s = seq.copy()
    if sub_rate > 0:
        m = rng.random(len(s)) < sub_rate
        s[m] = alphabet[rng.integers(0, len(alphabet), int(m.sum()))]
    if indel_rate <= 0:
        return s
    out = []
    events = np.nonzero(rng.random(len(s)) < indel_rate)[0]
    last = 0
    for pos in events:
        if pos < last:
            continue
        out.append(s[last:pos])
        length = int(rng.geometric(1.0 / 3.0))
        if rng.random() < 0.5:   # insertion before pos
            out.append(alphabet[rng.integers(0, len(alphabet), length)])
            last = pos
        else:                    # deletion of `length` residues from pos
            last = min(len(s), pos + length)
    out.append(s[last:])
    r = np.concatenate(out) if out else s[:0]
    return r if len(r) else alphabet[rng.integers(0, len(alphabet), 1)]


def c1(seed: int = 1) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = rng.integers(100, 301, 16)
    return Workload("c1", [AMINO[rng.integers(0, 20, int(L))] for L in lens], "blosum62", seed)


def c2(seed: int = 2, n: int = 1000) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    anc = AMINO[rng.integers(0, 20, 500)]
    seqs = [_mutate(rng, anc, float(rng.uniform(0.10, 0.30)), 0.02, AMINO) for _ in range(n)]
    return Workload("c2", seqs, "blosum62", seed)


def c3_lengths(rng, n: int, sigma: float = 0.75) -> np.ndarray:
    z = rng.standard_normal(n)
    return np.clip(np.round(np.exp(np.log(1500.0) + sigma * z)), 200, 16000).astype(np.int64)


def _dna(rng, L: int) -> np.ndarray:
    s = DNA[rng.integers(0, 4, L)]
    s[rng.random(L) < 0.01] = ord("N")
    return s


def c3(seed: int = 3, n: int = 4000, sigma: float = 0.75) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = c3_lengths(rng, n, sigma)
    return Workload("c3", [_dna(rng, int(L)) for L in lens], "default", seed)


def c4(seed: int = 4, clades: int = 20, members: int = 100) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    root = AMINO[rng.integers(0, 20, 1200)]
    seqs = []
    for _ in range(clades):
        anc = _mutate(rng, root, 0.40, 0.0, AMINO)
        target = int(rng.integers(200, 1201))
        if target <= len(anc):
            anc = anc[:target]
        else:
            anc = np.concatenate([anc, AMINO[rng.integers(0, 20, target - len(anc))]])
        for _ in range(members):
            seqs.append(_mutate(rng, anc, 0.10, 0.02, AMINO))
    return Workload("c4", seqs, "blosum62", seed)


def c5_job(job_seed: int) -> Workload:
    rng = np.random.Generator(np.random.PCG64(job_seed))
    n = int(rng.integers(8, 513))
    lens = rng.integers(50, 2001, n)
    if rng.random() < 0.5:
        return Workload("c5-protein", [AMINO[rng.integers(0, 20, int(L))] for L in lens], "blosum62", job_seed)
    return Workload("c5-dna", [_dna(rng, int(L)) for L in lens], "default", job_seed)


def random_set(seed: int, n: int, lo: int, hi: int, alphabet: bytes = b"ARNDCQEGHILKMFPSTWYV",
               extra: bytes = b"") -> Workload:
    """Small random sets for parity tests; `extra` characters are sprinkled in
    (non-letters become END units, '-' the GAP unit)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    alpha = np.frombuffer(alphabet, np.uint8)
    seqs = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = alpha[rng.integers(0, len(alpha), L)] if L else np.zeros(0, np.uint8)
        if extra and L:
            ex = np.frombuffer(extra, np.uint8)
            m = rng.random(L) < 0.05
            s[m] = ex[rng.integers(0, len(ex), int(m.sum()))]
        seqs.append(s)
    return Workload(f"random{seed}", seqs, "blosum62", seed)


BY_NAME = {"c1": c1, "c2": c2, "c3": c3, "c4": c4}
