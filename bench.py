"""Benchmark: all-pairs Needleman-Wunsch GCUPS on one B200 (or N, weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3|c2|c4]
    python bench.py --impl reference ...      # the reference's CPU path

A step is one all-pairs scoring pass over the workload (c3 by default: 4,000
uneven DNA sequences, ~8.0M pairs). `value` is kernel-resident throughput
(inputs already in HBM); `e2e` goes through the public C ABI with host buffers
(sequence upload and score download inside the timed region). GCUPS counts
sum over pairs of L_i * L_j with unpadded lengths.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "all-pairs NW GCUPS (bit-exact) batched vs plain"


def _rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_workload(name: str, rank: int = 0):
    from msa_b200 import workloads as W
    if name == "c3":
        return W.c3(seed=3 + 1000 * rank)
    if name == "c2":
        return W.c2(seed=2 + 1000 * rank)
    if name == "c4":
        return W.c4(seed=4 + 1000 * rank)
    raise SystemExit(f"unknown workload {name}")


def workload_config(name: str, wl) -> dict:
    L = wl.lengths()
    cfg = {"workload": {"c3": "4000 uneven DNA (log-normal median 1500, sigma 0.75, clip [200,16000]), default +1/-1 table, gap 1",
                        "c2": "1000 proteins from a 500-aa ancestor (subst U[0.10,0.30], indel 0.02), blosum62, gap 4",
                        "c4": "2000 proteins, 20 clades of 100, lengths U[200,1200], blosum62, gap 4"}[name],
           "sequences": wl.n, "pairs": wl.n * (wl.n - 1) // 2, "cells": wl.cells(),
           "mean_len": float(L.mean()), "max_len": int(L.max()), "table": wl.table, "seed": wl.seed}
    return cfg


# ---------------------------------------------------------------- CPU reference arm

def cpu_reference_sample(wl, target_cells: float, seed: int = 77):
    """A seeded uniform sample of the workload's pairs holding ~target_cells cells."""
    rng = np.random.Generator(np.random.PCG64(seed))
    L = wl.lengths().astype(np.float64)
    n = wl.n
    mean_cells = (L.sum() ** 2 - (L * L).sum()) / (n * (n - 1))
    k = max(8, int(target_cells / mean_cells))
    i = rng.integers(1, n, k)
    j = (rng.random(k) * i).astype(np.int64)
    cells = float((L[i] * L[j]).sum())
    return i.astype(np.int32), j.astype(np.int32), cells


def run_cpu_reference(wl, steps: int, warmup: int, target_cells: float):
    from oracle import oracle as O
    if O.reference() is None:
        return None
    threads = os.cpu_count() or 1
    strings = wl.strings()
    times, cells_all = [], []
    for s in range(warmup + steps):
        i, j, cells = cpu_reference_sample(wl, target_cells, seed=77 + s)
        t0 = time.perf_counter()
        O.ref_nw_pairs(strings, i, j, wl.table, threads=threads)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
            cells_all.append(cells)
    gcups = sum(cells_all) / sum(times) / 1e9
    return {"value": gcups, "unit": "GCUPS", "cores": threads, "kind": "reference", "cpu": cpu_model(),
            "sample": f"{len(times)} x ~{target_cells:.2g}-cell uniform pair samples of the workload, "
                      f"Museqa needleman::sequential (oracle/_ref) on {threads} host threads",
            "seconds": sum(times)}


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform's processor string."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def reference_arm(args):
    rank, world, _ = _rank_info()
    if rank != 0:
        return
    wl = load_workload(args.workload)
    res = run_cpu_reference(wl, args.steps, args.warmup, args.cpu_cells)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmuseqa_ref.so was not built"}))
        return
    line = {"metric": METRIC, "value": res["value"], "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * res["seconds"] / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": workload_config(args.workload, wl), "impl": "reference",
            "cpu_baseline": res, "e2e": {"value": res["value"], "unit": "GCUPS", "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- NJ leg

def nj_algorithmic_bytes(n: int) -> int:
    """Bytes one NJ run must move at the least: each join with c OTUs reads the
    c(c-1)/2 lower-triangle distances and the c row sums, reads rows x and y
    and writes row and column x and the copy of logical 0 into y (6c floats)."""
    return sum(4 * (c * (c - 1) // 2 + c + 6 * c) for c in range(2, n + 1))


def nj_leg(lib, ctx, steps: int = 3, cpu: bool = True) -> dict:
    """Neighbor-joining of the 2000-taxon pipeline workload: the NW scores stay
    on the device and feed msa_nj directly (int32 triangle). Reports the NJ
    kernel time, algorithmic bytes per second, and the reference's sequential
    NJ on the host for the same matrix (with a topology check)."""
    import ctypes

    import torch

    from msa_b200 import ScoringTable, _lib
    wl = load_workload("c4")
    n = wl.n
    flat, offs, lens = wl.flat_units()
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    h = ctypes.c_uint64()
    _lib.check(lib.msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                   lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    tri = torch.empty(n * (n - 1) // 2, dtype=torch.int32, device=torch.cuda.current_device())
    table = ScoringTable(wl.table)
    _lib.check(lib.msa_nw_all_pairs(ctx.handle, h.value, ctypes.byref(table._t), _lib.MSA_NW_PERSISTENT,
                                    ctypes.c_void_p(tri.data_ptr()), 1), ctx.handle)
    lib.msa_seqs_release(ctx.handle, h.value)
    nodes = (_lib.MsaOtu * (2 * n - 1))()
    kms, tms = [], []
    for s in range(1 + steps):
        _lib.check(lib.msa_nj(ctx.handle, ctypes.c_void_p(tri.data_ptr()), _lib.MSA_TRI_I32_DEVICE, n, nodes),
                   ctx.handle)
        st = _lib.MsaNjStats()
        lib.msa_nj_last_stats(ctx.handle, ctypes.byref(st))
        if s >= 1:
            kms.append(st.kernel_ms)
            tms.append(st.total_ms)
    kernel_ms = float(np.mean(kms))
    alg = nj_algorithmic_bytes(n)
    out = {"workload": "2000 proteins, 20 clades of 100 (c4 scores, int32 on the device)", "otus": n,
           "joins": n - 1, "kernel_ms": kernel_ms, "total_ms": float(np.mean(tms)), "steps": steps,
           "us_per_join": 1e3 * kernel_ms / (n - 1), "algorithmic_bytes": alg,
           "achieved_GBps": alg / (kernel_ms / 1e3) / 1e9, "cluster_ctas": int(st.cluster),
           "note": "the 16 MB distance matrix stays in L2 (126 MB); the bound is per-join latency"}
    if cpu:
        from oracle import oracle as O
        if O.reference() is not None:
            host = tri.cpu().numpy()
            t0 = time.perf_counter()
            ref = O.ref_nj(host.astype(np.float32), n)
            ref_ms = (time.perf_counter() - t0) * 1e3
            arr = np.frombuffer(nodes, dtype=np.dtype([("parent", "<u4"), ("c0", "<u4"), ("c1", "<u4"),
                                                       ("distance", "<f4"), ("level", "<u4")]))
            out["cpu_reference"] = {"ms": ref_ms, "cores": 1, "kind": "reference",
                                    "sample": "Museqa njoining::sequential (symmetric), oracle/_ref, full run"}
            out["tree_matches_reference"] = bool(
                (arr["parent"] == ref["parent"]).all() and (arr["c0"] == ref["child0"]).all()
                and (arr["c1"] == ref["child1"]).all()
                and (arr["distance"].view(np.uint32) == np.asarray(ref["distance"], np.float32).view(np.uint32)).all())
    return out


# ---------------------------------------------------------------- GPU arm

PROBE_OPS = ["iadd", "imnmx", "viaddmax_s32", "vimax3_s32", "vadd2", "viaddmax_s16x2", "vimax3_s16x2",
             "viaddmax_u16x2", "vimax3_u16x2", "vmaxu2", "prmt", "cell_s32", "cell_s16x2", "cell_u16x2_biased",
             "cell_u16x2_gapfree", "lds128_bytes"]


def packed_row_fraction(wl, rmax: int = 32) -> float:
    """Share of the DP cells that the batched kernel scores from packed-byte
    profile rows, by replaying its plan: length-sorted sequences paired into
    rows pairs, strips of 32R rows (R even, at most rmax), and 8 floor(R/16)
    of each lane's R rows packed. Cells are weighted by the pair's unpadded
    cells."""
    e = np.sort(wl.lengths().astype(np.int64))[::-1]
    n = len(e)
    csum = np.concatenate([[0], np.cumsum(e)])       # csum[i] = sum of e[:i]
    packed = total = 0.0
    for k in range((n + 1) // 2):
        a1, a2 = 2 * k, min(2 * k + 1, n - 1)
        cols = float(csum[n] - csum[2 * k + 1])       # columns: sorted 2k+1 .. n-1
        if cols <= 0:
            continue
        e1 = int(e[a1])
        nst = -(-e1 // (32 * rmax))
        r = -(-e1 // (32 * nst))
        r = (r + 1) & ~1
        cells = (e1 + (int(e[a2]) if a2 != a1 else 0)) * cols
        packed += cells * (8 * (r // 16)) / r
        total += cells
    return packed / total if total else 0.0


def probe_rate(ctx, op: int, iters: int = 2048) -> float:
    """Lane-ops (op 15: shared-memory bytes) per SM per clock of one probe form."""
    import ctypes

    from msa_b200 import _lib
    p = _lib.MsaOpProbe()
    _lib.check(_lib.lib().msa_probe_op(ctx.handle, op, iters, ctypes.byref(p)), ctx.handle)
    return float(p.ops_per_clk_sm)


def probe_ops(iters: int = 2048) -> dict:
    """Lane-ops per SM per clock of each integer form (msa_probe_op)."""
    import ctypes

    from msa_b200 import _lib, runtime
    ctx = runtime.context(0)
    res = {}
    for k, name in enumerate(PROBE_OPS):
        p = _lib.MsaOpProbe()
        _lib.check(_lib.lib().msa_probe_op(ctx.handle, k, iters, ctypes.byref(p)), ctx.handle)
        res[name] = {"ops_per_clk_sm": round(p.ops_per_clk_sm, 2), "sm_mhz": round(p.sm_clock_mhz, 1)}
    print(json.dumps(res))
    return res


def serve_bench(args):
    """c5: all-pairs jobs (n U[8,512], lengths U[50,2000], half protein/blosum62,
    half DNA/default) arriving as a Poisson process at `load` x the saturated
    rate; latency = completion - submission per job. The same arrivals are
    served with batch windows (the headline, unless --window-ms 0) and with
    continuous admission, and one at a time by the plain kernel."""
    import ctypes
    import threading

    from msa_b200 import ScoringTable, _lib, pairwise
    from msa_b200 import workloads as W
    from msa_b200.serve import Server
    jobs = [W.c5_job(50_000 + k) for k in range(args.jobs)]
    packed = [(wl.flat_units(), ScoringTable(wl.table), wl.cells()) for wl in jobs]
    total_cells = sum(c for _, _, c in packed)
    mean_cells = total_cells / len(jobs)

    # Saturated throughput: every job submitted at once.
    with Server(device=0) as srv:
        t0 = time.perf_counter()
        ids = [srv.submit(*fu, t) for fu, t, _ in packed]
        for i in ids:
            srv.wait(i)
        sat_s = time.perf_counter() - t0
    sat_gcups = total_cells / sat_s / 1e9

    rate = args.load * (sat_gcups * 1e9) / mean_cells          # jobs per second

    def arrival_times(seed):
        rng = np.random.Generator(np.random.PCG64(seed))
        return np.cumsum(rng.exponential(1.0 / rate, len(jobs)))

    arrivals = arrival_times(5)

    def run_server(window_ms=0.0, arrivals=arrivals):
        stats = [None] * len(jobs)
        with Server(device=0, batch_window_ms=window_ms) as srv:
            ids = [None] * len(jobs)
            start = time.perf_counter()

            def producer():
                for k, (fu, t, _) in enumerate(packed):
                    delay = arrivals[k] - (time.perf_counter() - start)
                    if delay > 0:
                        time.sleep(delay)
                    ids[k] = srv.submit(*fu, t)
            th = threading.Thread(target=producer)
            th.start()
            for k in range(len(jobs)):
                while ids[k] is None:
                    time.sleep(0.0005)
                stats[k] = srv.wait(ids[k])[1]
            th.join()
        lat = np.array([s["latency_ms"] for s in stats])
        span_ms = max(s["done_ms"] for s in stats) - min(s["submit_ms"] for s in stats)
        return lat, total_cells / (span_ms / 1e3) / 1e9, stats

    def summary(lat, agg, stats):
        return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "p99_over_p50": float(np.percentile(lat, 99) / np.percentile(lat, 50)), "aggregate_gcups": agg,
                "mean_launches_per_job": float(np.mean([s["launches"] for s in stats]))}

    if args.sweep_windows:
        # Window x arrival-seed sweep at the same offered load (no plain leg).
        seeds = [int(x) for x in args.arrival_seeds.split(",")]
        for w in [float(x) for x in args.sweep_windows.split(",")]:
            for seed in seeds:
                lat, agg, st = run_server(w, arrival_times(seed))
                slow = np.argsort(lat)[::-1][:4]
                t0 = min(x["submit_ms"] for x in st)
                tail = [{"latency_ms": round(float(lat[k]), 1), "submit_ms": round(st[k]["submit_ms"] - t0, 1),
                         "admit_wait_ms": round(st[k]["admit_ms"] - st[k]["submit_ms"], 1),
                         "run_ms": round(st[k]["done_ms"] - st[k]["admit_ms"], 1), "cells": int(st[k]["cells"])}
                        for k in slow]
                print(json.dumps({"window_ms": w, "arrival_seed": seed, **summary(lat, agg, st),
                                  "p90_ms": float(np.percentile(lat, 90)), "max_ms": float(lat.max()),
                                  "saturated_gcups": sat_gcups, "arrival_rate_per_s": rate, "slowest": tail}),
                      flush=True)
        return None

    continuous = summary(*run_server())
    windowed = summary(*run_server(args.window_ms)) if args.window_ms > 0 else None

    # Same jobs, same arrivals, one at a time through the plain kernel.
    def run_plain():
        start = time.perf_counter()
        lat_p = []
        for k, (fu, t, _) in enumerate(packed):
            now = time.perf_counter() - start
            if now < arrivals[k]:
                time.sleep(arrivals[k] - now)
            pairwise.score_units(*fu, t, _lib.MSA_NW_PLAIN)
            lat_p.append((time.perf_counter() - start - arrivals[k]) * 1e3)
        span = time.perf_counter() - start - arrivals[0]
        return np.array(lat_p), total_cells / span / 1e9

    lat_p, agg_p = run_plain()
    head = windowed if windowed else continuous
    policy = f"batch windows of {args.window_ms:g} ms" if windowed else "continuous admission"
    line = {"metric": "serve p50/p99 job latency (continuous batching)", "unit": "ms", "policy": policy, **head,
            "saturated_gcups": sat_gcups, "offered_load": args.load, "arrival_rate_per_s": rate, "jobs": len(jobs),
            "mean_cells_per_job": mean_cells}
    if windowed:
        line["continuous_admission"] = continuous
    line["plain_one_at_a_time"] = {"p50_ms": float(np.percentile(lat_p, 50)), "p99_ms": float(np.percentile(lat_p, 99)),
                                   "aggregate_gcups": agg_p}
    line["data"] = "synthetic (seeded c5 jobs)"
    print(json.dumps(line))
    return line


def profile_run(args):
    """One scoring call (after warm-up) for ncu captures; prints its stats."""
    import ctypes

    from msa_b200 import ScoringTable, _lib, pairwise
    wl = load_workload(args.workload)
    if args.n:
        wl.seqs = wl.seqs[:args.n]
    flat, offs, lens = wl.flat_units()
    if args.profile == "nj":
        from msa_b200 import phylogeny
        tri = pairwise.score_units(flat, offs, lens, ScoringTable(wl.table))
        times = []
        for _ in range(args.warmup + 1):
            t0 = time.perf_counter()
            phylogeny.run_triangle(tri, wl.n)
            times.append((time.perf_counter() - t0) * 1e3)
        import ctypes
        from msa_b200 import runtime
        ns = _lib.MsaNjStats()
        _lib.lib().msa_nj_last_stats(runtime.context(0).handle, ctypes.byref(ns))
        stats = {f: getattr(ns, f) for f, _ in ns._fields_}
        print(json.dumps({"workload": args.workload, "n": wl.n, "mode": "nj", "wall_ms": times, "stats": stats}))
        return
    mode = _lib.MSA_NW_PERSISTENT if args.profile == "persistent" else _lib.MSA_NW_PLAIN
    for _ in range(args.warmup + 1):
        pairwise.score_units(flat, offs, lens, ScoringTable(wl.table), mode)
    st = pairwise.last_stats()
    print(json.dumps({"workload": args.workload, "n": wl.n, "mode": args.profile, "cells": wl.cells(),
                      "kernel_ms": st.kernel_ms, "gcups": wl.cells() / st.kernel_ms / 1e6,
                      "launches": st.launches, "narrow_tasks": st.narrow_tasks}))


def shard_bench(args):
    """One c3 job split over all ranks (one GPU each): every rank scores its
    part of equal DP cells into a zero-filled device triangle, and one NCCL
    sum all-reduce assembles the whole matrix on every rank. Strong scaling:
    the job is the same for any number of ranks. Timed per step from before
    the part to after the exchange, max over ranks."""
    import ctypes

    import torch
    import torch.distributed as dist

    from msa_b200 import ScoringTable, _lib, runtime, shard
    rank, world, local = _rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=600))
    lib = _lib.lib()
    ctx = runtime.context(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    wl = load_workload(args.workload, 0)          # the same job on every rank
    cfg = workload_config(args.workload, wl)
    table = ScoringTable(wl.table)
    flat, offs, lens = wl.flat_units()
    n = wl.n
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    h = ctypes.c_uint64()
    _lib.check(lib.msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                   lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    tri = torch.zeros(n * (n - 1) // 2, dtype=torch.int32, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        tri.zero_()
        shard.score_part(ctx, h.value, table, rank, world, tri.data_ptr())
        if world > 1:
            dist.all_reduce(tri, op=dist.ReduceOp.SUM)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    barrier()
    clocks = sampler.stop()
    t = torch.tensor([float(np.mean(ms))], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms = float(t.item())
    # Whole matrix on every rank: check it once against the one-device result.
    ok = None
    if rank == 0:
        full = torch.empty_like(tri)
        torch.cuda.synchronize()
        _lib.check(lib.msa_nw_all_pairs(ctx.handle, h.value, ctypes.byref(table._t), _lib.MSA_NW_PERSISTENT,
                                        ctypes.c_void_p(full.data_ptr()), 1), ctx.handle)
        ok = bool(torch.equal(full, tri))
        value = cfg["cells"] / (step_ms / 1e3) / 1e9
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int32/int16x2", "data": "synthetic (seeded)",
            "config": dict(cfg, parallelism=f"one job split over {world} GPU(s): equal-cell parts, one NCCL "
                                            f"sum all-reduce of the int32 triangle",
                           l2="flushed (256 MB write) before every timed step"),
            "matches_single_device": ok, "clocks": clocks}))
    lib.msa_seqs_release(ctx.handle, h.value)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c3", "c2", "c4"])
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--cpu-cells", type=float, default=1.5e10)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-nj", action="store_true", help="skip the neighbor-joining leg")
    ap.add_argument("--shard", action="store_true",
                    help="one job split over all ranks with an NCCL exchange (strong scaling)")
    ap.add_argument("--profile", choices=["persistent", "plain", "nj"], default=None,
                    help="profiling run: --warmup calls then one call, on the first --n sequences")
    ap.add_argument("--n", type=int, default=0, help="with --profile: use the first N sequences")
    ap.add_argument("--probe", action="store_true", help="integer-op throughput probes (lane-ops/clk/SM)")
    ap.add_argument("--serve", action="store_true", help="serving loop: Poisson arrivals of c5 jobs")
    ap.add_argument("--jobs", type=int, default=400)
    ap.add_argument("--load", type=float, default=0.8, help="offered load as a fraction of saturated throughput")
    ap.add_argument("--sweep-windows", default="",
                    help="with --serve: comma-separated batch windows (ms, 0 = continuous) to sweep instead")
    ap.add_argument("--arrival-seeds", default="5,6,7", help="with --sweep-windows: Poisson arrival seeds")
    ap.add_argument("--window-ms", type=float, default=60.0,
                    help="with --serve: batch window of the headline serving run (0: continuous admission only)")
    args = ap.parse_args()
    if args.probe:
        return probe_ops()
    if args.serve:
        return serve_bench(args)
    if args.impl == "reference":
        return reference_arm(args)
    if args.shard:
        return shard_bench(args)
    if args.profile:
        return profile_run(args)

    import ctypes

    import torch
    import torch.distributed as dist

    rank, world, local = _rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=600))

    from msa_b200 import ScoringTable, _lib, runtime
    lib = _lib.lib()
    ctx = runtime.context(local)
    stream = torch.cuda.Stream()          # a capturable stream: repeated calls replay a CUDA graph
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    wl = load_workload(args.workload, rank)
    cfg = workload_config(args.workload, wl)
    table = ScoringTable(wl.table)
    flat, offs, lens = wl.flat_units()
    n = wl.n
    npairs = n * (n - 1) // 2
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)

    h = ctypes.c_uint64()
    _lib.check(lib.msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                   lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    out = torch.empty(npairs, dtype=torch.int32, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")   # > 126 MB L2

    def run(mode):
        _lib.check(lib.msa_nw_all_pairs(ctx.handle, h.value, ctypes.byref(table._t), mode,
                                        ctypes.c_void_p(out.data_ptr()), 1), ctx.handle)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(mode, steps, warmup):
        for _ in range(warmup):
            run(mode)
        barrier()
        ms, kms = [], []
        launches0 = ctx.launches
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run(mode)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            st = _lib.MsaNwStats()
            lib.msa_nw_last_stats(ctx.handle, ctypes.byref(st))
            kms.append(st.kernel_ms)
        barrier()
        return ms, kms, ctx.launches - launches0, st

    sampler = ClockSampler(local)
    sampler.start()
    ms, kms, launches, st = timed(_lib.MSA_NW_PERSISTENT, args.steps, args.warmup)
    clocks = sampler.stop()
    plain_ms, plain_kms, _, _ = timed(_lib.MSA_NW_PLAIN, args.plain_steps, 1)

    # Bit-exact cross-check of the two kernels on this workload.
    run(_lib.MSA_NW_PERSISTENT)
    a = out.clone()
    run(_lib.MSA_NW_PLAIN)
    agree = bool(torch.equal(a, out))

    # End to end through the public C ABI: pinned host units in, host scores out.
    pin_units = torch.from_numpy(flat).pin_memory()
    host_out = torch.empty(npairs, dtype=torch.int32).pin_memory()
    e2e_ms = []
    for s in range(1 + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(stream)
        h2 = ctypes.c_uint64()
        _lib.check(lib.msa_seqs_upload(ctx.handle, ctypes.cast(pin_units.data_ptr(), u8), offs.ctypes.data_as(u64),
                                       lens.ctypes.data_as(u64), n, ctypes.byref(h2)), ctx.handle)
        _lib.check(lib.msa_nw_all_pairs(ctx.handle, h2.value, ctypes.byref(table._t), _lib.MSA_NW_PERSISTENT,
                                        ctypes.c_void_p(host_out.data_ptr()), 0), ctx.handle)
        e1.record(stream)
        e1.synchronize()
        lib.msa_seqs_release(ctx.handle, h2.value)
        if s >= 1:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_ok = bool(torch.equal(host_out, a.cpu()))

    # Max over ranks.
    def maxr(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    step_ms = maxr(float(np.mean(ms)))
    kern_ms = maxr(float(np.mean(kms)))
    plain_step = maxr(float(np.mean(plain_ms)))
    e2e_step = maxr(float(np.mean(e2e_ms)))
    cells_all = cfg["cells"] * world
    value = cells_all / (step_ms / 1e3) / 1e9
    kernel_gcups = cfg["cells"] / (kern_ms / 1e3) / 1e9
    plain_gcups = cells_all / (plain_step / 1e3) / 1e9
    e2e_gcups = cells_all / (e2e_step / 1e3) / 1e9

    if rank == 0:
        props = torch.cuda.get_device_properties(local)
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        nsm = props.multi_processor_count
        # DRAM traffic and counted instructions per cell of this kernel on this
        # workload, from the committed ncu summaries.
        traffic = inst_per_cell = None
        tp = ROOT / "profiles" / "nw_traffic.json"
        if tp.exists():
            try:
                tj = json.loads(tp.read_text())
                traffic = tj.get(args.workload)
                inst_per_cell = tj.get(args.workload + "_inst_per_cell")
            except Exception:
                traffic = inst_per_cell = None
        # Ceilings of the batched kernel from rates measured here per SM clock
        # (msa_probe_op). A cell reads its score from shared memory: 2 bytes in
        # a 16-bit profile row, 1 byte in a packed row (a share f of the cells,
        # from the kernel's plan), so 2 - f bytes per cell. The ALU pipe
        # (64 lanes/clk/SM) carries one vimax3 per two cells and one PRMT per
        # two cells of a packed row: (1 + f) / 2 lane-ops per cell. The lowest
        # ceiling (these two, and issue below) is the roofline.
        lds = probe_rate(ctx, 15)
        cell_ops = probe_rate(ctx, 14)
        f_packed = packed_row_fraction(wl)
        smem_peak = nsm * (lds / (2.0 - f_packed)) * sm_mhz * 1e6 / 1e9
        alu_peak = nsm * (64.0 / ((1.0 + f_packed) / 2.0)) * sm_mhz * 1e6 / 1e9
        cell_peak = nsm * (2.0 * cell_ops) * sm_mhz * 1e6 / 1e9
        # Issue: 4 warp-instructions (128 lane-instructions) per SM per clock
        # over the lane-instructions per cell that ncu counted for this kernel
        # on this workload (profiles/nw_traffic.json), when there is a count.
        issue_peak = nsm * (128.0 / inst_per_cell) * sm_mhz * 1e6 / 1e9 if inst_per_cell else None
        ceilings = {"smem": smem_peak, "alu": alu_peak}
        if issue_peak:
            ceilings["issue"] = issue_peak
        bound = min(ceilings, key=ceilings.get)
        roof = ceilings[bound]
        # The four-op int32 issue figure (two max operations per cell on the ALU
        # pipe, 64 lanes/clk/SM): 32 cells/clk/SM.
        peak = nsm * 64 * sm_mhz * 1e6 / 2 / 1e9
        cpu = None
        if not args.no_cpu:
            cpu = run_cpu_reference(wl, 1, 0, args.cpu_cells)
        line = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32/int16x2", "data": "synthetic (seeded)",
            "config": dict(cfg, parallelism=f"{world} independent replicas (weak)" if world > 1 else "1 GPU",
                           l2="flushed (256 MB write) before every timed step"),
            "kernel_gcups": kernel_gcups, "narrow_tasks": int(st.narrow_tasks), "graph_replay": bool(st.graph),
            "plain": {"value": plain_gcups, "ms_per_step": plain_step, "steps": args.plain_steps,
                      "speedup_persistent_vs_plain": value / plain_gcups, "bit_identical": agree},
            "e2e": {"value": e2e_gcups, "unit": "GCUPS", "ms_per_step": e2e_step,
                    "h2d_bytes_per_step": int(flat.nbytes + offs.nbytes + lens.nbytes),
                    "d2h_bytes_per_step": int(npairs * 4), "scores_match": e2e_ok},
            "gpu_launches": int(launches),
            "roofline": {"bound": bound, "achieved": kernel_gcups,
                         "peak": roof, "unit": "GCUPS", "frac": kernel_gcups / roof, "traffic": traffic,
                         "frac_int32_issue": kernel_gcups / peak,
                         "packed_row_fraction": f_packed, "inst_per_cell_counted": inst_per_cell,
                         "ceilings_gcups": {"smem_profile_reads": smem_peak, "alu_pipe": alu_peak,
                                            "issue_counted_instructions": issue_peak,
                                            "cell_ops_16x2_probe": cell_peak, "int32_issue_4ops_per_cell": peak},
                         "measured_per_sm_clk": {"lds_bytes": lds, "cell_16x2_lane_ops": cell_ops},
                         "peak_basis": f"min of {nsm} SM x {lds:.1f} shared-memory bytes/clk (measured, "
                                       f"ld.shared.v4) / (2 - {f_packed:.3f}) bytes of profile per cell, "
                                       f"{nsm} SM x 64 ALU lanes/clk / ((1 + {f_packed:.3f}) / 2) lane-ops per cell"
                                       + (f" and {nsm} SM x 128 issued lane-instructions/clk / {inst_per_cell} "
                                          f"counted per cell" if inst_per_cell else "")
                                       + f", x {sm_mhz:.0f} MHz (median sampled); frac_int32_issue is against "
                                         f"{nsm} SM x 64 ALU lanes/clk / 2 max-ops per cell"},
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        if not args.no_nj:
            line["nj"] = nj_leg(lib, ctx, cpu=not args.no_cpu)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
