"""Serving benchmark: a Poisson stream of HF + GW self-consistent jobs through serve.Server.

    python -m green_gpu_b200.serve_bench [--jobs 12] [--rate 20] [--iterations 5] [--slots 4]
                                         [--scale small|mix] [--precision split|fp64] [--overlap]

``--scale mix`` draws the batched-system mix (k meshes 2x2x2..4x4x4, nao 20..80,
NQ = 6..8 nao) plus 10 % of 6x6x6 k, nao 104, NQ 800 jobs; the latter need ~3.2 TB of
resident integrals and are rejected by admission.  ``--scale small`` keeps the same
structure with meshes up to 2x2x2 and nao up to 36 so that a run ends within a minute.
Every job's inputs are synthesised before the stream starts, so a job's latency (arrival to
last iteration) holds its admission wait, making its state resident and its iterations.
Prints one JSON line with p50 / p99 latency, GW builds/s and the admission log.
``--overlap`` replays the same stream with one slot (jobs run one after another) and with
``--slots`` slots, and adds both makespans and the sum of the builds' device times: with the
concurrent makespan below both the serial makespan and the summed device time, the jobs'
device work overlapped.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import serve


def small_mix(n_jobs, seed, iterations, precision):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n_jobs):
        if rng.random() < 0.1:
            jobs.append(serve.Job(mesh=(6, 6, 6), nao=104, NQ=800, seed=i, name=f"large{i}", iterations=iterations,
                                  precision=precision))
            continue
        nao = int(rng.choice([20, 26, 36]))
        mesh = [(2, 1, 1), (2, 2, 1), (2, 2, 2)][int(rng.integers(3))]
        jobs.append(serve.Job(mesh=mesh, nao=nao, NQ=int(nao * rng.choice([6, 7, 8])), seed=i, name=f"job{i}",
                              iterations=iterations, precision=precision))
    return jobs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=12)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--iterations", type=int, default=5)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--scale", default="small", choices=["small", "mix"])
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--overlap", action="store_true")
    a = ap.parse_args(argv)

    def jobs_():
        if a.scale == "small":
            jobs = small_mix(a.jobs, a.seed, a.iterations, a.precision)
        else:
            jobs = serve.config5_mix(a.jobs, a.seed)
            for j in jobs:
                j.iterations = a.iterations
                j.precision = a.precision
        for j in jobs:  # the requests' inputs exist before they arrive
            if serve.footprint(j) < 2 ** 40:
                j.inputs = serve.make_inputs(j)
        return jobs

    def stream(slots):
        jobs = jobs_()  # before the server starts, so that its log times start at the stream
        srv = serve.Server(slots=slots)
        futs = serve.poisson_stream(srv, jobs, a.rate, seed=a.seed)
        results = [f.result() for f in futs]
        srv.close()
        return srv, results

    srv, results = stream(a.slots)
    st = srv.stats()
    st.update({"scale": a.scale, "rate_hz": a.rate, "slots": a.slots, "precision": a.precision,
               "iterations": a.iterations, "errors": [r.error for r in results if r.error],
               "log": srv.log})
    if a.overlap:
        srv1, _ = stream(1)
        s1 = srv1.stats()
        st["overlap"] = {"makespan_serial_s": s1["span_s"], "makespan_concurrent_s": st["span_s"],
                         "device_s_sum": st["device_s"], "speedup": s1["span_s"] / st["span_s"]}
    print(json.dumps(st))


if __name__ == "__main__":
    main()
