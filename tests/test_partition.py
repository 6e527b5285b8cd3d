"""Splitting one all-pairs job over several devices, host side (no GPU): the
split covers every pair exactly once, balances DP cells, is deterministic,
and the one exchange step (a sum-reduce of zero-filled partial triangles into
rank 0, run here over gloo with two ranks) rebuilds the whole matrix exactly.
bench.py's rank launcher and its sharded line run here on two gloo ranks,
with the oracle standing in for the device kernel."""
import os

import numpy as np
import pytest

from msa_b200 import ScoringTable, pairwise
from msa_b200 import workloads as W
from oracle import oracle as O


def _lognormal_set(seed, n):
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = W.c3_lengths(rng, n, 0.75)
    return W.Workload("split", [W._dna(rng, int(L)) for L in lens], "default", seed)


def _cells(wl):
    L = wl.lengths().astype(np.float64)
    n = len(L)
    i, j = np.tril_indices(n, -1)
    return L[i] * L[j]


@pytest.mark.parametrize("nparts", [1, 2, 3, 5, 8])
def test_split_covers_every_pair_once_and_balances_cells(nparts):
    wl = _lognormal_set(11, 300)
    flat, offs, lens = wl.flat_units()
    part = pairwise.part_of_pairs(flat, offs, lens, ScoringTable("default"), nparts)
    assert part.shape == (300 * 299 // 2,)
    assert part.max() < nparts
    if nparts == 1:
        assert not part.any()
    cells = _cells(wl)
    per = np.bincount(part, weights=cells, minlength=nparts)
    # Parts are cut at rows-pair granularity: off by at most the largest rows pair.
    L = np.sort(wl.lengths())[::-1].astype(np.float64)
    biggest = 2 * L[0] * L.sum()
    assert np.all(np.abs(per - cells.sum() / nparts) <= biggest)
    # Same inputs, same split.
    assert np.array_equal(part, pairwise.part_of_pairs(flat, offs, lens, ScoringTable("default"), nparts))


def test_split_with_generic_pairs_and_an_asymmetric_table():
    # END units inside sequences send their pairs down the generic path; an
    # asymmetric caller table sends every pair there.
    wl = W.random_set(12, 60, 0, 200, extra=b"*\r")
    flat, offs, lens = wl.flat_units()
    for table in (ScoringTable("blosum62"), None):
        if table is None:
            m = np.array([[(a * 7 + b * 3) % 11 - 5 for b in range(25)] for a in range(25)], np.int32)
            table = ScoringTable.custom(m, 3)
        part = pairwise.part_of_pairs(flat, offs, lens, table, 4)
        assert part.max() < 4 and len(part) == 60 * 59 // 2
        counts = np.bincount(part, minlength=4)
        assert np.all(counts > 0)


def _rank_main(rank, world, port, flat, offs, lens, tables, want, nparts, result):
    import torch
    import torch.distributed as dist
    from msa_b200 import ScoringTable, pairwise, shard
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        table = ScoringTable("blosum62")
        mine = pairwise.part_of_pairs(flat, offs, lens, table, nparts) == rank
        # This rank's pairs (the CPU oracle stands in for the device kernel).
        scores = O.oracle_nw_all_pairs(flat, offs, lens, tables, 7, O.TABLE_INDEX["blosum62"], O.PENALTY["blosum62"])
        tri = torch.zeros(len(mine), dtype=torch.int32)
        tri[torch.from_numpy(np.nonzero(mine)[0])] = torch.from_numpy(scores[mine].astype(np.int32))
        shard.exchange(tri)
        # The whole matrix lands on rank 0 (the neighbor-joining device).
        result[rank] = bool(np.array_equal(tri.numpy(), want)) if rank == 0 else True
    finally:
        dist.destroy_process_group()


def test_two_ranks_assemble_the_whole_matrix_over_gloo(golden):
    import socket

    import torch.multiprocessing as mp
    wl = W.random_set(13, 40, 20, 300)
    flat, offs, lens = wl.flat_units()
    tables = O.table_block(golden)
    want = O.oracle_nw_all_pairs(flat, offs, lens, tables, 7, O.TABLE_INDEX["blosum62"], O.PENALTY["blosum62"])
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    result = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, flat, offs, lens, tables, want.astype(np.int32), 2, result))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert result[0] and result[1]


def test_launcher_runs_the_sharded_job_on_two_gloo_ranks(tmp_path):
    import json
    from pathlib import Path
    import bench
    root = Path(__file__).resolve().parents[1]
    out = tmp_path / "line.json"
    rc = bench.launch_ranks(2, str(root / "tests" / "_shard_rank.py"), [str(out)], timeout_s=300)
    assert rc == 0
    line = json.loads(out.read_text())
    assert line["n_gpus"] == 2 and line["scaling"] == "strong" and line["higher_is_better"] is True
    assert line["matches_single_device"] is True
    assert line["value"] > 0 and line["unit"] == "GCUPS" and line["ms_per_step"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] > 0 and line["e2e"]["d2h_bytes_per_step"] == 40 * 39 // 2 * 4
    assert "sum-reduce" in line["config"]["parallelism"] and line["config"]["pairs"] == 40 * 39 // 2
