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
    def run_nj(order):
        nodes = (_lib.MsaOtu * (2 * n - 1))()
        kms, tms = [], []
        for s in range(1 + steps):
            _lib.check(lib.msa_nj_order(ctx.handle, ctypes.c_void_p(tri.data_ptr()), _lib.MSA_TRI_I32_DEVICE, n,
                                        order, nodes), ctx.handle)
            st = _lib.MsaNjStats()
            lib.msa_nj_last_stats(ctx.handle, ctypes.byref(st))
            if s >= 1:
                kms.append(st.kernel_ms)
                tms.append(st.total_ms)
        return nodes, kms, tms, st

    def same_tree(nodes, ref):
        arr = np.frombuffer(nodes, dtype=np.dtype([("parent", "<u4"), ("c0", "<u4"), ("c1", "<u4"),
                                                   ("distance", "<f4"), ("level", "<u4")]))
        return bool((arr["parent"] == ref["parent"]).all() and (arr["c0"] == ref["child0"]).all()
                    and (arr["c1"] == ref["child1"]).all() and (arr["level"] == ref["level"]).all()
                    and (arr["distance"].view(np.uint32)
                         == np.asarray(ref["distance"], np.float32).view(np.uint32)).all())

    nodes, kms, tms, st = run_nj(_lib.MSA_NJ_SYMMETRIC)
    lin_nodes, lin_kms, _, _ = run_nj(_lib.MSA_NJ_LINEAR)
    kernel_ms = float(np.mean(kms))
    alg = nj_algorithmic_bytes(n)
    out = {"workload": "2000 proteins, 20 clades of 100 (c4 scores, int32 on the device)", "otus": n,
           "joins": n - 1, "kernel_ms": kernel_ms, "total_ms": float(np.mean(tms)), "steps": steps,
           "us_per_join": 1e3 * kernel_ms / (n - 1), "algorithmic_bytes": alg,
           "achieved_GBps": alg / (kernel_ms / 1e3) / 1e9, "cluster_ctas": int(st.cluster),
           "phase_cycles": {f: int(getattr(st, f)) for f, _ in st._fields_ if f.startswith("cycles")},
           "linear_order": {"kernel_ms": float(np.mean(lin_kms)),
                            "us_per_join": 1e3 * float(np.mean(lin_kms)) / (n - 1)},
           "note": "the 16 MB distance matrix stays in L2 (126 MB); the bound is per-join latency"}
    if cpu:
        from oracle import oracle as O
        if O.reference() is not None:
            host = tri.cpu().numpy()
            t0 = time.perf_counter()
            ref = O.ref_nj(host.astype(np.float32), n)
            ref_ms = (time.perf_counter() - t0) * 1e3
            out["cpu_reference"] = {"ms": ref_ms, "cores": 1, "kind": "reference",
                                    "sample": "Museqa njoining::sequential (symmetric), oracle/_ref, full run"}
            out["tree_matches_reference"] = same_tree(nodes, ref)
            t0 = time.perf_counter()
            ref_lin = O.ref_nj(host.astype(np.float32), n, "njoining-sequential-linear")
            out["linear_order"]["cpu_reference_ms"] = (time.perf_counter() - t0) * 1e3
            out["linear_order"]["tree_matches_reference"] = same_tree(lin_nodes, ref_lin)
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


def nw_ceilings(wl, workload: str, nsm: int, sm_mhz: float, lds: float) -> tuple:
    """Ceilings (GCUPS) of the batched kernel on a workload from rates measured
    per SM clock: shared-memory profile reads at 2 - f bytes per cell (f: the
    packed-row share of the cells, from the kernel's plan), the ALU pipe at
    (1 + f) / 2 lane-ops per cell (64 lanes/clk/SM), and issue at the
    lane-instructions per cell that ncu counted for this kernel on this
    workload (profiles/nw_traffic.json), when there is a count. Returns the
    ceilings, the binding one, f, the counted instructions per cell and the
    DRAM traffic of one launch."""
    traffic = inst = None
    tp = ROOT / "profiles" / "nw_traffic.json"
    if tp.exists():
        try:
            tj = json.loads(tp.read_text())
            traffic = tj.get(workload)
            inst = tj.get(workload + "_inst_per_cell")
        except Exception:
            traffic = inst = None
    f = packed_row_fraction(wl)
    c = {"smem": nsm * (lds / (2.0 - f)) * sm_mhz * 1e6 / 1e9,
         "alu": nsm * (64.0 / ((1.0 + f) / 2.0)) * sm_mhz * 1e6 / 1e9}
    if inst:
        c["issue"] = nsm * (128.0 / inst) * sm_mhz * 1e6 / 1e9
    bound = min(c, key=c.get)
    return c, bound, f, inst, traffic


class Scorer:
    """One workload uploaded to the device store of `ctx`, scored into a
    device triangle with CUDA-event timing on `stream` after an L2 flush."""

    def __init__(self, lib, ctx, stream, wl, device: int):
        import ctypes

        import torch

        from msa_b200 import ScoringTable, _lib
        self.lib, self.ctx, self.stream, self.wl = lib, ctx, stream, wl
        self._lib = _lib
        self.table = ScoringTable(wl.table)
        flat, offs, lens = wl.flat_units()
        n = wl.n
        u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
        self.h = ctypes.c_uint64()
        _lib.check(lib.msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                       lens.ctypes.data_as(u64), n, ctypes.byref(self.h)), ctx.handle)
        self.out = torch.empty(n * (n - 1) // 2, dtype=torch.int32, device=f"cuda:{device}")
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")   # > 126 MB L2

    def run(self, mode):
        import ctypes
        self._lib.check(self.lib.msa_nw_all_pairs(self.ctx.handle, self.h.value, ctypes.byref(self.table._t), mode,
                                                  ctypes.c_void_p(self.out.data_ptr()), 1), self.ctx.handle)

    def timed(self, mode, steps: int, warmup: int):
        """Mean step ms (events around the call) and kernel ms (the library's
        own events around the scoring kernels) over `steps` calls."""
        import ctypes

        import torch
        for _ in range(warmup):
            self.run(mode)
        torch.cuda.synchronize()
        ms, kms = [], []
        for _ in range(steps):
            self.flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            self.run(mode)
            e1.record(self.stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            st = self._lib.MsaNwStats()
            self.lib.msa_nw_last_stats(self.ctx.handle, ctypes.byref(st))
            kms.append(st.kernel_ms)
        return float(np.mean(ms)), float(np.mean(kms)), st

    def release(self):
        self.lib.msa_seqs_release(self.ctx.handle, self.h.value)


def side_workload(lib, ctx, stream, name: str, steps: int, plain_steps: int, sm_mhz: float, lds: float,
                  device: int) -> dict:
    """c2 or c4 beside the headline: the persistent kernel and the plain
    one-launch-per-bucket kernel on the same device store, their bit-identity,
    and the persistent kernel's roofline fraction at this workload's own
    packed-row share."""
    import torch

    from msa_b200 import _lib
    wl = load_workload(name)
    sc = Scorer(lib, ctx, stream, wl, device)
    ms, kms, st = sc.timed(_lib.MSA_NW_PERSISTENT, steps, 3)
    a = sc.out.clone()
    pms, pkms, _ = sc.timed(_lib.MSA_NW_PLAIN, plain_steps, 1)
    agree = bool(torch.equal(a, sc.out))
    sc.release()
    cells = wl.cells()
    nsm = torch.cuda.get_device_properties(device).multi_processor_count
    c, bound, f, inst, traffic = nw_ceilings(wl, name, nsm, sm_mhz, lds)
    kg = cells / (kms / 1e3) / 1e9
    return {"config": workload_config(name, wl), "value": cells / (ms / 1e3) / 1e9, "unit": "GCUPS",
            "ms_per_step": ms, "steps": steps, "kernel_gcups": kg,
            "plain": {"value": cells / (pms / 1e3) / 1e9, "ms_per_step": pms, "steps": plain_steps},
            "speedup_persistent_vs_plain": pms / ms, "bit_identical": agree,
            "roofline": {"bound": bound, "achieved": kg, "peak": c[bound], "unit": "GCUPS", "frac": kg / c[bound],
                         "packed_row_fraction": f, "inst_per_cell_counted": inst, "traffic": traffic,
                         "ceilings_gcups": c}}


def ablation(lib, ctx, sc, steps: int) -> dict:
    """What each part of the batched kernel contributes on the headline
    workload, beside the plain kernel and the committed kernel (filled in by
    the caller): the persistent kernel forced to 32-bit lanes; on 16-bit lanes
    without packed-byte profile rows; and restaging its strip for every column
    group. Each is a library variant (msa_nw_set_variant) with the same
    scores, checked against the committed kernel's."""
    import torch

    from msa_b200 import _lib
    cells = sc.wl.cells()
    sc.run(_lib.MSA_NW_PERSISTENT)
    want = sc.out.clone()
    out = {}
    for key, flags, chunk in (("persistent_int32_gcups", _lib.MSA_NW_VARIANT_INT32, 0),
                              ("persistent_16bit_no_packed_rows_gcups", _lib.MSA_NW_VARIANT_NO_PACKED, 0),
                              ("persistent_restage_every_group_gcups", 0, 1)):
        _lib.check(lib.msa_nw_set_variant(ctx.handle, flags, chunk), ctx.handle)
        try:
            ms, _, _ = sc.timed(_lib.MSA_NW_PERSISTENT, steps, 1)
            out[key] = cells / (ms / 1e3) / 1e9
            out[key.replace("_gcups", "_bit_identical")] = bool(torch.equal(want, sc.out))
        finally:
            _lib.check(lib.msa_nw_set_variant(ctx.handle, 0, 0), ctx.handle)
    out["steps"] = steps
    return out


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


def serve_bench(args, emit: bool = True):
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

    def run_server(window_ms=0.0, arrivals=arrivals, age_ms=0.0):
        stats = [None] * len(jobs)
        with Server(device=0, batch_window_ms=window_ms, age_weight_ms=age_ms) as srv:
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

    if args.sweep_age:
        # Continuous admission with age-weighted shares: weight x arrival-seed sweep.
        seeds = [int(x) for x in args.arrival_seeds.split(",")]
        for a in [float(x) for x in args.sweep_age.split(",")]:
            for seed in seeds:
                lat, agg, st = run_server(0.0, arrival_times(seed), a)
                print(json.dumps({"age_weight_ms": a, "arrival_seed": seed, **summary(lat, agg, st),
                                  "p90_ms": float(np.percentile(lat, 90)), "max_ms": float(lat.max()),
                                  "saturated_gcups": sat_gcups, "arrival_rate_per_s": rate}), flush=True)
        return None

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
    aged = summary(*run_server(0.0, arrivals, args.age_ms)) if args.age_ms > 0 else None
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
    if aged:
        line["continuous_age_weighted"] = dict(aged, age_weight_ms=args.age_ms)
    line["plain_one_at_a_time"] = {"p50_ms": float(np.percentile(lat_p, 50)), "p99_ms": float(np.percentile(lat_p, 99)),
                                   "aggregate_gcups": agg_p}
    line["data"] = "synthetic (seeded c5 jobs)"
    if emit:
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


def shard_line(cfg: dict, world: int, steps: int, warmup: int, step_ms: float, e2e_ms: float, h2d: int, d2h: int,
               ok, clocks: dict, launches=None, weak=None, roofline=None) -> dict:
    """The bench line of one job split over `world` ranks (strong scaling:
    the same job for any number of ranks). `value` is the whole job's GCUPS
    from the max-over-ranks step time (every part scored, then the exchange
    into rank 0); `e2e` the same through the public C ABI from pinned host
    units to the whole matrix in rank 0's host memory."""
    line = {
        "metric": METRIC, "value": cfg["cells"] / (step_ms / 1e3) / 1e9, "unit": "GCUPS", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "int32/int16x2", "data": "synthetic (seeded)",
        "config": dict(cfg, parallelism=f"one job split over {world} GPU(s): equal-cell parts of the kernels' task "
                                        f"list, one NCCL sum-reduce of the disjoint int32 parts into rank 0 "
                                        f"(the neighbor-joining device)",
                       l2="flushed (256 MB write) before every timed step"),
        "matches_single_device": ok,
        "e2e": {"value": cfg["cells"] / (e2e_ms / 1e3) / 1e9, "unit": "GCUPS", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "clocks": clocks,
    }
    if launches is not None:
        line["gpu_launches"] = int(launches)
    if roofline is not None:
        line["roofline"] = roofline
    if weak is not None:
        line["weak_replicas"] = weak
    return line


def timed_steps(step, steps: int, warmup: int, timer, barrier, maxr) -> float:
    """Mean ms of `steps` calls of step() after `warmup` untimed ones, each
    timed by timer(step) on this rank; barriers on both sides; the max over
    ranks of the mean."""
    for _ in range(warmup):
        step()
    barrier()
    ms = [timer(step) for _ in range(steps)]
    barrier()
    return maxr(float(np.mean(ms)))


def launch_ranks(nproc: int, script: str, argv: list, timeout_s: int = 3600) -> int:
    """Runs `script argv` as `nproc` ranks of one node under
    torch.distributed.run (rendezvous on 127.0.0.1, a free port); returns its
    exit code. The whole group is killed if it outlives timeout_s."""
    import signal
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(script), *argv]
    p = subprocess.Popen(cmd, start_new_session=True)
    try:
        return p.wait(timeout=timeout_s)
    except subprocess.TimeoutExpired:
        os.killpg(p.pid, signal.SIGTERM)
        try:
            p.wait(timeout=60)
        except subprocess.TimeoutExpired:
            os.killpg(p.pid, signal.SIGKILL)
        return 124


def shard_bench(args):
    """One job split over all ranks (one GPU each): every rank scores its part
    of equal DP cells into a zero-filled device triangle, and one NCCL
    sum-reduce assembles the whole matrix on rank 0, the device that runs
    neighbor-joining. Strong scaling: the job is the same for any number of
    ranks. Timed per step from before the part to after the exchange, max over
    ranks. Beside it, `weak_replicas`: every rank scores its own job of the
    same shape (no data-path collective)."""
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
    npairs = n * (n - 1) // 2
    u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
    h = ctypes.c_uint64()
    _lib.check(lib.msa_seqs_upload(ctx.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                   lens.ctypes.data_as(u64), n, ctypes.byref(h)), ctx.handle)
    tri = torch.zeros(npairs, dtype=torch.int32, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        tri.zero_()
        shard.score_part(ctx, h.value, table, rank, world, tri.data_ptr())
        shard.exchange(tri)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def maxr(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timer(fn):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    sampler = ClockSampler(local)
    sampler.start()
    launches0 = ctx.launches
    step_ms = timed_steps(step, args.steps, args.warmup, timer, barrier, maxr)
    launches = (ctx.launches - launches0) // max(args.steps + args.warmup, 1)
    clocks = sampler.stop()

    # Whole matrix on rank 0: checked against the one-device result.
    ok = None
    if rank == 0:
        full = torch.empty_like(tri)
        torch.cuda.synchronize()
        _lib.check(lib.msa_nw_all_pairs(ctx.handle, h.value, ctypes.byref(table._t), _lib.MSA_NW_PERSISTENT,
                                        ctypes.c_void_p(full.data_ptr()), 1), ctx.handle)
        ok = bool(torch.equal(full, tri))
    lib.msa_seqs_release(ctx.handle, h.value)

    # End to end: pinned host units uploaded on every rank, the part, the
    # exchange, and the whole matrix read back into rank 0's host memory.
    pin_units = torch.from_numpy(flat).pin_memory()
    host_out = torch.empty(npairs, dtype=torch.int32).pin_memory()

    def e2e_step():
        h2 = ctypes.c_uint64()
        _lib.check(lib.msa_seqs_upload(ctx.handle, ctypes.cast(pin_units.data_ptr(), u8), offs.ctypes.data_as(u64),
                                       lens.ctypes.data_as(u64), n, ctypes.byref(h2)), ctx.handle)
        tri.zero_()
        shard.score_part(ctx, h2.value, table, rank, world, tri.data_ptr())
        shard.exchange(tri)
        if rank == 0:
            host_out.copy_(tri, non_blocking=True)
        lib.msa_seqs_release(ctx.handle, h2.value)

    e2e_ms = timed_steps(e2e_step, args.steps, 1, timer, barrier, maxr)

    # Weak replicas: each rank its own job of the same shape, no collective.
    weak = None
    if world > 1 and not args.no_extra:
        own = load_workload(args.workload, rank)
        sc = Scorer(lib, ctx, stream, own, local)
        wms = timed_steps(lambda: sc.run(_lib.MSA_NW_PERSISTENT), 1, 1, timer, barrier, maxr)
        sc.release()
        weak = {"value": own.cells() * world / (wms / 1e3) / 1e9, "unit": "GCUPS", "ms_per_step": wms,
                "scaling": "weak", "steps": 1,
                "parallelism": f"{world} independent replicas, each its own job of this shape (per-rank seed)"}

    if rank == 0:
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        lds = probe_rate(ctx, 15)
        c, bound, f, inst, traffic = nw_ceilings(wl, args.workload, nsm, sm_mhz, lds)
        per_gpu = cfg["cells"] / (step_ms / 1e3) / 1e9 / world
        roof = {"bound": bound, "achieved": per_gpu, "peak": c[bound], "unit": "GCUPS", "frac": per_gpu / c[bound],
                "traffic": traffic, "ceilings_gcups": c, "packed_row_fraction": f,
                "note": "per GPU: whole-job GCUPS / n_gpus against one GPU's ceilings"}
        line = shard_line(cfg, world, args.steps, args.warmup, step_ms, e2e_ms,
                          flat.nbytes + offs.nbytes + lens.nbytes, npairs * 4, ok, clocks, launches, weak, roof)
        print(json.dumps(line))
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
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the c2/c4 legs, the ablation and the serving leg of the default line")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg of the default line")
    ap.add_argument("--side-steps", type=int, default=10, help="timed steps of the c2 and c4 legs")
    ap.add_argument("--shard", action="store_true",
                    help="one job split over all ranks with an NCCL exchange (strong scaling; the default "
                         "when more than one rank runs)")
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
    ap.add_argument("--sweep-age", default="",
                    help="with --serve: comma-separated age weights (ms) of continuous admission to sweep instead")
    ap.add_argument("--age-ms", type=float, default=3.0,
                    help="with --serve: age weight (ms) of the age-weighted continuous run (0: skip it)")
    ap.add_argument("--window-ms", type=float, default=60.0,
                    help="with --serve: batch window of the headline serving run (0: continuous admission only)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # One process per GPU: start the ranks here when not launched by torchrun.
        sys.exit(launch_ranks(args.gpus, __file__, sys.argv[1:]))
    if args.probe:
        return probe_ops()
    if args.serve:
        return serve_bench(args)
    if args.impl == "reference":
        return reference_arm(args)
    if args.shard or _rank_info()[1] > 1:
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

    sc = Scorer(lib, ctx, stream, wl, local)
    out, flush, run = sc.out, sc.flush, sc.run

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
    # Attribution of the persistent kernel's speed-up (rank 0 only, outside
    # every timed region).
    abl = None
    if rank == 0 and not args.no_extra:
        abl = ablation(lib, ctx, sc, args.plain_steps)

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
        if abl is not None:
            line["ablation"] = dict(abl, plain_gcups=plain_gcups, committed_gcups=value)
        if not args.no_extra:
            for name in ("c2", "c4"):
                if name != args.workload:
                    line[name] = side_workload(lib, ctx, stream, name, args.side_steps, args.plain_steps, sm_mhz, lds,
                                               local)
        if not args.no_nj:
            line["nj"] = nj_leg(lib, ctx, cpu=not args.no_cpu)
        if not args.no_extra and not args.no_serve:
            line["serve"] = serve_bench(args, emit=False)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
