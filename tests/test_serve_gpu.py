"""Serving loop on the GPU: jobs submitted together are admitted by HBM
budget, share merged launches, and each job's scores equal the same job
scored alone (msa_nw_all_pairs) — integers, so exactly."""
import threading

import numpy as np
import pytest

from msa_b200 import ScoringTable, pairwise
from msa_b200 import _lib
from msa_b200 import workloads as W
from msa_b200.serve import Server
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _alone(wl, table=None):
    flat, offs, lens = wl.flat_units()
    return pairwise.score_units(flat, offs, lens, table or ScoringTable(wl.table))


def _mixed_jobs():
    jobs = [W.c5_job(1000 + k) for k in range(6)]
    # keep the test quick: trim the larger jobs
    for wl in jobs:
        wl.seqs = wl.seqs[:120]
    jobs.append(W.random_set(81, 40, 0, 300, extra=b"*\r"))   # END units: reference-orientation path
    jobs.append(W.random_set(82, 1, 10, 20))                   # a single sequence: no pairs
    jobs.append(W.random_set(83, 2, 5, 30, alphabet=b"ACGT"))
    return jobs


def test_jobs_in_the_mix_equal_jobs_alone(gpu):
    jobs = _mixed_jobs()
    with Server(device=0) as srv:
        ids = [srv.submit_workload(wl) for wl in jobs]
        results = [srv.wait(i) for i in ids]
    for wl, (scores, stats) in zip(jobs, results):
        if wl.n >= 2:
            assert np.array_equal(scores, _alone(wl)), wl.name
        assert stats["n"] == wl.n and stats["done_ms"] >= stats["admit_ms"] >= stats["submit_ms"]
    # Work of different jobs overlapped on the device: some job was admitted
    # before another one finished.
    spans = sorted((s["admit_ms"], s["done_ms"]) for _, s in results if s["cells"] > 0)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))


def test_small_job_matches_reference_oracle(gpu, golden):
    tables = O.table_block(golden)
    wl = W.random_set(84, 30, 20, 400)
    flat, offs, lens = wl.flat_units()
    want = O.oracle_nw_all_pairs(flat, offs, lens, tables, 7, O.TABLE_INDEX["blosum62"], O.PENALTY["blosum62"])
    with Server(device=0) as srv:
        scores, _ = srv.wait(srv.submit_workload(wl, ScoringTable("blosum62")))
    assert np.array_equal(scores, want)


def test_budget_admits_one_job_at_a_time_and_stays_exact(gpu):
    jobs = [W.c5_job(2000 + k) for k in range(4)]
    for wl in jobs:
        wl.seqs = wl.seqs[:60]
    with Server(device=0, hbm_budget_bytes=1 << 20) as srv:   # smaller than any one job
        ids = [srv.submit_workload(wl) for wl in jobs]
        results = [srv.wait(i) for i in ids]
    for wl, (scores, _) in zip(jobs, results):
        assert np.array_equal(scores, _alone(wl))
    spans = sorted((s["admit_ms"], s["done_ms"]) for _, s in results)
    assert all(spans[k + 1][0] >= spans[k][1] - 1e-6 for k in range(len(spans) - 1))


def test_submissions_from_several_threads(gpu):
    jobs = [W.c5_job(3000 + k) for k in range(8)]
    for wl in jobs:
        wl.seqs = wl.seqs[:50]
    out = {}
    with Server(device=0) as srv:
        def client(k):
            jid = srv.submit_workload(jobs[k])
            out[k] = srv.wait(jid)[0]
        threads = [threading.Thread(target=client, args=(k,)) for k in range(len(jobs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    for k, wl in enumerate(jobs):
        assert np.array_equal(out[k], _alone(wl))


def test_wait_with_timeout_and_unknown_job(gpu):
    with Server(device=0) as srv:
        wl = W.c5_job(4000)
        jid = srv.submit_workload(wl)
        rc = srv.poll(jid)
        assert rc in (_lib.MSA_OK, _lib.MSA_ERR_DEVICE_TIMEOUT)
        if rc == _lib.MSA_ERR_DEVICE_TIMEOUT:
            srv.wait(jid)
        assert _lib.lib().msa_serve_wait(srv.handle, 987654, 0, None, None) == _lib.MSA_ERR_QUEUE


def test_windowed_admission_starts_jobs_on_window_boundaries(gpu):
    """batch_window_ms > 0: a job is admitted at the first window boundary
    after its submission (counted from server start), and its scores are
    still those of the job alone."""
    jobs = [W.c5_job(4000 + k) for k in range(5)]
    for wl in jobs:
        wl.seqs = wl.seqs[:60]
    window = 30.0
    with Server(device=0, batch_window_ms=window) as srv:
        ids = []
        for wl in jobs:
            ids.append(srv.submit_workload(wl))
        results = [srv.wait(i) for i in ids]
    for wl, (scores, stats) in zip(jobs, results):
        assert np.array_equal(scores, _alone(wl))
        boundary = np.ceil(stats["submit_ms"] / window) * window
        assert stats["admit_ms"] >= boundary - 1e-3


def test_reference_orientation_jobs_interleaved_with_resident_jobs(gpu):
    """Jobs with END units are scored at admission, in the reference's
    orientation, on the admission stream (which may capture a CUDA graph for
    them) while merged launches finish other jobs. Finished jobs' memory must
    not be released on that stream: a release enqueued during a capture would
    become part of the graph and the job's scores or memory would be lost.
    Several rounds of such jobs interleaved with resident ones, every job equal
    to the job alone."""
    for rnd in range(3):
        jobs = []
        for k in range(6):
            wl = W.c5_job(6000 + 10 * rnd + k)
            wl.seqs = wl.seqs[:80]
            jobs.append(wl)
            jobs.append(W.random_set(600 + 10 * rnd + k, 24, 0, 260, extra=b"*\r"))
        with Server(device=0) as srv:
            ids = [srv.submit_workload(wl) for wl in jobs]
            results = [srv.wait(i) for i in ids]
        for wl, (scores, _) in zip(jobs, results):
            assert np.array_equal(scores, _alone(wl)), (rnd, wl.name)
