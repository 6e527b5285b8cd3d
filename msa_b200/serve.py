"""Serving loop client: continuous batching of all-pairs NW jobs (msa_serve_*).

    with Server(device=0) as srv:
        a = srv.submit_workload(wl1)
        b = srv.submit_workload(wl2)
        scores_a, stats_a = srv.wait(a)

Jobs are admitted while their device footprint fits the HBM budget; every
merged launch takes tasks from all admitted jobs. Scores are those of
msa_nw_all_pairs for the same job alone.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import MsaJobStats, MsaServeConfig, check, lib
from .pairwise import ScoringTable


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_jobs: int = 0, quantum_mcells: int = 0,
                 batch_window_ms: float = 0.0, age_weight_ms: float = 0.0):
        """batch_window_ms > 0 admits jobs at window boundaries (msa_serve_config.batch_window_us);
        under continuous admission, age_weight_ms > 0 weights each job's share
        of a launch by 1 + age / age_weight_ms (msa_serve_config.age_weight_us)."""
        cfg = MsaServeConfig(device, hbm_budget_bytes, max_jobs, quantum_mcells, int(round(batch_window_ms * 1000)),
                             int(round(age_weight_ms * 1000)))
        h = ctypes.c_void_p()
        check(lib().msa_serve_start(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        self._sizes: dict[int, int] = {}

    def submit(self, flat: np.ndarray, offs: np.ndarray, lens: np.ndarray, table: ScoringTable) -> int:
        flat = np.ascontiguousarray(flat, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        lens = np.ascontiguousarray(lens, np.uint64)
        jid = ctypes.c_uint64()
        u8, u64 = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64)
        check(lib().msa_serve_submit(self.handle, flat.ctypes.data_as(u8), offs.ctypes.data_as(u64),
                                     lens.ctypes.data_as(u64), len(lens), ctypes.byref(table._t), ctypes.byref(jid)))
        self._sizes[jid.value] = len(lens)
        return jid.value

    def submit_workload(self, wl, table: ScoringTable | None = None) -> int:
        flat, offs, lens = wl.flat_units()
        return self.submit(flat, offs, lens, table or ScoringTable(wl.table))

    def wait(self, job_id: int, timeout_ms: int = -1):
        n = self._sizes[job_id]
        out = np.zeros(max(n * (n - 1) // 2, 1), np.int32)
        st = MsaJobStats()
        rc = lib().msa_serve_wait(self.handle, job_id, timeout_ms, out.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.byref(st))
        check(rc)
        del self._sizes[job_id]
        stats = {"submit_ms": st.submit_ms, "admit_ms": st.admit_ms, "done_ms": st.done_ms, "cells": st.cells,
                 "n": st.n, "launches": st.launches, "latency_ms": st.done_ms - st.submit_ms}
        return out[: n * (n - 1) // 2], stats

    def poll(self, job_id: int) -> int:
        """Status of a job without waiting: MSA_ERR_DEVICE_TIMEOUT while it runs."""
        n = self._sizes[job_id]
        out = np.zeros(max(n * (n - 1) // 2, 1), np.int32)
        rc = lib().msa_serve_wait(self.handle, job_id, 0, out.ctypes.data_as(ctypes.c_void_p), None)
        if rc != 7:
            del self._sizes[job_id]
        return rc

    def stop(self) -> None:
        if self.handle:
            lib().msa_serve_stop(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()
