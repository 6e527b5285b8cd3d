"""Autotuner for the persistent NW kernel.

    python -m msa_b200.autotune [--write] [--from-json saved_run.log]

For seeded workloads of several length classes it times every (rows per lane,
warps per CTA) tile shape the library is built with, then, on the fastest
shape, every number of column groups a single-strip task sweeps after one
staging of its profile strip (msa_nw_set_variant's groups_per_task: 1 restages
the strip for every group of W column sequences). It prints the table, and
with --write regenerates csrc/autotune.inc (the choice compiled into the
library) from the fastest setting per class. The measurements behind the
committed choice are kept next to it in autotune.json.
"""
from __future__ import annotations

import ctypes
import json
import sys
import time
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
SHAPES = [(16, 4), (16, 8), (32, 4), (32, 8)]
CHUNKS = [1, 2, 4, 8, 16]
DEFAULT_CHUNK = 4


def classes():
    from . import workloads as W
    rng = np.random.Generator(np.random.PCG64(11))

    def dna(n, lo, hi):
        lens = rng.integers(lo, hi + 1, n)
        return W.Workload("dna", [W.DNA[rng.integers(0, 4, int(L))] for L in lens], "default", 11)

    return [
        ("median<384", dna(1500, 100, 600)),
        ("median<1024", W.c2(n=800)),
        ("median<2048", dna(700, 900, 2400)),
        ("median>=2048", dna(300, 2000, 6000)),
        ("c3-like", W.c3(n=1200)),
    ]


def time_shape(ctx, wl, shape, reps: int = 3, chunk: int = 0) -> float:
    from . import ScoringTable, _lib, pairwise
    lib = _lib.lib()
    _lib.check(lib.msa_nw_set_tiles(ctx.handle, *shape), ctx.handle)
    _lib.check(lib.msa_nw_set_variant(ctx.handle, 0, chunk), ctx.handle)
    flat, offs, lens = wl.flat_units()
    best = 0.0
    try:
        for _ in range(reps):
            pairwise.score_units(flat, offs, lens, ScoringTable(wl.table), _lib.MSA_NW_PERSISTENT)
            st = pairwise.last_stats()
            best = max(best, wl.cells() / st.kernel_ms / 1e6)
    finally:
        lib.msa_nw_set_tiles(ctx.handle, 0, 0)
        lib.msa_nw_set_variant(ctx.handle, 0, 0)
    return best


def main():
    if "--from-json" in sys.argv:
        # Regenerate the committed choice from a saved measurement (the JSON line
        # printed by a GPU run of this module).
        out = json.loads(Path(sys.argv[sys.argv.index("--from-json") + 1]).read_text().strip().splitlines()[-1])
        table = out["classes"]
    else:
        from . import runtime
        ctx = runtime.context(0)
        table = {}
        for name, wl in classes():
            L = wl.lengths()
            row = {f"{r}x{w}": round(time_shape(ctx, wl, (r, w), chunk=DEFAULT_CHUNK), 1) for r, w in SHAPES}
            best = max(SHAPES, key=lambda s: row[f"{s[0]}x{s[1]}"])
            row["groups_per_task"] = {str(g): round(time_shape(ctx, wl, best, chunk=g), 1) for g in CHUNKS}
            row["median_len"] = int(np.median(L))
            table[name] = row
            print(name, row, flush=True)
        out = {"when": time.strftime("%Y-%m-%d %H:%M:%S"), "unit": "GCUPS (kernel time)", "classes": table}
        print(json.dumps(out))
    if "--write" in sys.argv:
        (PKG / "autotune.json").write_text(json.dumps(out, indent=1) + "\n")
        bounds = [("median<384", 384), ("median<1024", 1024), ("median<2048", 2048), ("median>=2048", None)]
        lines = ["// Tile shapes of the batched kernel by median effective length of the clean",
                 "// sequences. Written by msa_b200/autotune.py from measurements on a B200",
                 "// (autotune.json); regenerate with `python -m msa_b200.autotune --write`.",
                 "static Tiles pick_tiles(const SeqStore *st, uint32_t nclean)",
                 "{",
                 "    if(nclean == 0) return {16, 8};",
                 "    const uint32_t med = st->eff[st->clean_sorted[nclean / 2]];"]
        for name, bound in bounds:
            row = table[name]
            best = max(SHAPES, key=lambda s: row[f"{s[0]}x{s[1]}"])
            cond = f"med < {bound}" if bound else "true"
            lines.append(f"    if({cond}) return {{{best[0]}, {best[1]}}};   // {row[f'{best[0]}x{best[1]}']} GCUPS")
        lines += ["    return {32, 8};", "}", "",
                  "// Column groups per single-strip task, by the same classes.",
                  "static uint32_t pick_chunk(const SeqStore *st, uint32_t nclean)",
                  "{",
                  f"    if(nclean == 0) return {DEFAULT_CHUNK};",
                  "    const uint32_t med = st->eff[st->clean_sorted[nclean / 2]];"]
        for name, bound in bounds:
            gpt = table[name].get("groups_per_task")
            g = int(max(gpt, key=gpt.get)) if gpt else DEFAULT_CHUNK
            cond = f"med < {bound}" if bound else "true"
            lines.append(f"    if({cond}) return {g};" + (f"   // {gpt[str(g)]} GCUPS" if gpt else ""))
        lines += [f"    return {DEFAULT_CHUNK};", "}"]
        (PKG / "csrc" / "autotune.inc").write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
