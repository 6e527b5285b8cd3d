"""One rank of the sharded job, for tests/test_partition.py: run under
torch.distributed.run by bench.launch_ranks on CPU ranks (gloo), with the
oracle standing in for the device kernel. Rank 0 writes bench.shard_line's
JSON line to the path given as the first argument."""
import datetime
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main():
    import torch
    import torch.distributed as dist

    import bench
    from msa_b200 import ScoringTable, pairwise, shard
    from msa_b200 import workloads as W
    from oracle import oracle as O

    rank, world, _ = bench._rank_info()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        golden = json.loads((ROOT / "tests/golden/golden.json").read_text())
        wl = W.random_set(13, 40, 20, 300)
        flat, offs, lens = wl.flat_units()
        npairs = wl.n * (wl.n - 1) // 2
        want = O.oracle_nw_all_pairs(flat, offs, lens, O.table_block(golden), 7, O.TABLE_INDEX["blosum62"],
                                     O.PENALTY["blosum62"])
        mine = np.nonzero(pairwise.part_of_pairs(flat, offs, lens, ScoringTable("blosum62"), world) == rank)[0]
        part = torch.from_numpy(want[mine].astype(np.int32))
        idx = torch.from_numpy(mine)
        tri = torch.zeros(npairs, dtype=torch.int32)

        def step():
            tri.zero_()
            tri[idx] = part          # this rank's part (the oracle standing in for the kernel)
            shard.exchange(tri)

        def timer(fn):
            t0 = time.perf_counter()
            fn()
            return (time.perf_counter() - t0) * 1e3

        def maxr(v):
            t = torch.tensor([v], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        step_ms = bench.timed_steps(step, 3, 1, timer, dist.barrier, maxr)
        ok = bool(np.array_equal(tri.numpy(), want)) if rank == 0 else None
        cfg = {"workload": "40 random proteins, blosum62", "sequences": wl.n, "pairs": npairs, "cells": wl.cells()}
        line = bench.shard_line(cfg, world, 3, 1, step_ms, step_ms, flat.nbytes + offs.nbytes + lens.nbytes,
                                npairs * 4, ok, {"sm_mhz": None, "sm_max_mhz": None, "reasons": []})
        if rank == 0:
            Path(sys.argv[1]).write_text(json.dumps(line))
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
