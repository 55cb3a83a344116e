"""Serving loop: admission by memory footprint, continuous batching, p50/p99, and (on the
GPU) results that are the same alone and in the mix."""
import threading
import time

import numpy as np
import pytest

from green_gpu_b200 import serve


def test_admission_respects_budget_and_slots_cpu():
    # fake executor: no device; records concurrent memory use
    state = {"used": 0, "peak": 0, "running": 0, "max_running": 0}
    lock = threading.Lock()
    sizes = {"a": 40, "b": 50, "c": 30, "d": 70, "huge": 500}

    def fp(job):
        return sizes[job.name]

    def ex(job, dev):
        with lock:
            state["used"] += fp(job)
            state["running"] += 1
            state["peak"] = max(state["peak"], state["used"])
            state["max_running"] = max(state["max_running"], state["running"])
        time.sleep(0.05)
        with lock:
            state["used"] -= fp(job)
            state["running"] -= 1
        r = serve.Result(job)
        r.sigma = [np.zeros(1)] * job.iterations
        return r

    srv = serve.Server(budget_bytes=100, slots=2, executor=ex, footprint_fn=fp)
    futs = [srv.submit(serve.Job(name=n, iterations=2)) for n in ("a", "b", "huge", "c", "d")]
    res = [f.result(timeout=10) for f in futs]
    srv.close()
    assert res[2].error and "rejected" in res[2].error
    assert all(r.error is None for i, r in enumerate(res) if i != 2)
    assert state["peak"] <= 100
    assert state["max_running"] <= 2
    st = srv.stats()
    assert st["jobs"] == 4 and st["rejected"] == 1 and st["p99_s"] >= st["p50_s"] > 0


def test_large_jobs_of_the_serving_mix_are_rejected_with_reason_cpu():
    jobs = serve.config5_mix(n_jobs=40, seed=3, large_fraction=0.5)
    big = [j for j in jobs if j.name.startswith("large")]
    assert big
    srv = serve.Server(budget_bytes=150 * 2**30, slots=2, executor=lambda j, d: serve.Result(j),
                       footprint_fn=serve.footprint)
    r = srv.submit(big[0]).result(timeout=10)
    srv.close()
    assert r.error and "cannot be resident" in r.error


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix():
    jobs = [serve.Job(mesh=(2, 2, 1), nao=8, NQ=24, seed=1, iterations=2, name="j1"),
            serve.Job(mesh=(2, 2, 2), nao=12, NQ=40, seed=2, iterations=2, name="j2", precision="fp64"),
            serve.Job(mesh=(3, 1, 1), nao=10, NQ=32, seed=3, iterations=3, name="j3"),
            serve.Job(mesh=(2, 2, 1), nao=16, NQ=48, seed=4, iterations=2, name="j4")]
    alone = [serve.run_job(j) for j in jobs]
    srv = serve.Server(slots=3)
    futs = serve.poisson_stream(srv, [serve.Job(**{k: getattr(j, k) for k in
                                                   ("mesh", "nao", "NQ", "seed", "iterations", "precision",
                                                    "slices", "damping", "name")}) for j in jobs], rate_hz=20.0)
    mixed = [f.result(timeout=600) for f in futs]
    srv.close()
    for a, m in zip(alone, mixed):
        assert m.error is None, m.error
        for x, y in zip(a.sigma, m.sigma):
            assert np.abs(x - y).max() <= 1e-12 * np.abs(x).max()
        for x, y in zip(a.fock, m.fock):
            assert np.abs(x - y).max() <= 1e-12 * np.abs(x).max()
    st = srv.stats()
    assert st["jobs"] == 4 and st["p99_s"] is not None
