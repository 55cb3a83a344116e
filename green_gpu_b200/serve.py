"""Continuous-batching service for HF + GW self-energy evaluations on one B200.

Requests are self-consistent jobs: a system (k mesh, nao, NQ, seed) and a number of
iterations.  Each iteration evaluates the HF Fock matrix and the GW self-energy of the
current G with the system's integrals, IR transforms and work space resident in HBM (one
gg_context per job, created when the job is admitted and kept until its last iteration).
The self-consistency update of G belongs to the caller (green-mbpt); by default a job
applies a fixed damped update G <- (1 - damping) G between iterations so that every
iteration sees a different input.

Scheduling:
* jobs arrive at any time (``submit``) and wait in a FIFO queue;
* a job is admitted when a slot is free and its device footprint (gg_estimate_bytes: the
  resident integrals plus the un-chunked work space) fits the free part of the memory
  budget; jobs that could never fit are rejected with the reason;
* admitted jobs run concurrently, each on its own context and CUDA stream, so their
  kernels can overlap on the device (``serve_bench --overlap`` measures it: the same stream
  with one slot and with several); a finished job frees its slot and its memory at once
  and the queue is re-examined (continuous batching, not a run-to-completion queue).

``Server.stats()`` reports per-job latency (arrival to last iteration) p50 / p99,
builds/s and the admission log.
"""
from __future__ import annotations

import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np


@dataclass
class Job:
    mesh: tuple = (2, 2, 2)
    nao: int = 26
    NQ: int = 120
    seed: int = 0
    iterations: int = 5
    precision: str = "split"
    slices: int = 5
    damping: float = 0.01
    name: str = ""
    # the request's inputs (a synth.System-like object); built by the executor when absent
    inputs: object = None
    # filled by the server
    arrival: float = 0.0
    start: float = 0.0
    end: float = 0.0
    footprint: int = 0
    device_s: float = 0.0  # device time of the job's builds (CUDA events inside the library)


@dataclass
class Result:
    job: Job
    sigma: List[np.ndarray] = field(default_factory=list)   # one Sigma(tau) per iteration
    fock: List[np.ndarray] = field(default_factory=list)    # one Fock per iteration
    error: Optional[str] = None


def footprint(job: Job) -> int:
    """Device bytes of a resident job (integrals + un-chunked GW work space)."""
    from . import native
    nk = int(np.prod(job.mesh))
    npairs = nk * (nk + 1) // 2
    return native.estimate_bytes(nk, nk, nk, job.nao, job.NQ, 1, 72, 69, npairs)


def make_inputs(job: Job):
    """The request's inputs (seeded synthetic G, V, symmetry and IR transforms)."""
    from . import synth
    return synth.make_system(mesh=job.mesh, nao=job.nao, NQ=job.NQ, seed=job.seed)


def run_job(job: Job, device: int = 0) -> Result:
    """Execute one job on the GPU (default executor): make its state resident (context,
    integrals, IR transforms), run its iterations, release the state."""
    from . import native
    s = job.inputs if job.inputs is not None else make_inputs(job)
    ctx = native.context_for(s, device=device)
    ctx.set_split_slices(job.slices)
    prec = native.PREC_SPLIT if job.precision == "split" else native.PREC_FP64
    ctx.set_hf_precision(prec)
    res = Result(job)
    G = s.G_tskij.copy()
    for _ in range(job.iterations):
        res.fock.append(ctx.hf_fock(G[s.nts - 1], s.S_k, s.madelung))
        res.sigma.append(ctx.gw_sigma(G, precision=prec))
        job.device_s += ctx.timings().get("e2e", 0.0)
        G = (1.0 - job.damping) * G
    ctx.close()
    return res


class Server:
    def __init__(self, budget_bytes: Optional[int] = None, slots: int = 4, device: int = 0,
                 executor: Callable[[Job, int], Result] = run_job,
                 footprint_fn: Callable[[Job], int] = footprint):
        if budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            budget_bytes = int(0.8 * free)
        self.budget = int(budget_bytes)
        self.slots = int(slots)
        self.device = device
        self.executor = executor
        self.footprint_fn = footprint_fn
        self._queue: List[tuple] = []
        self._running = 0
        self._used = 0
        self._lock = threading.Condition()
        self._done: List[Result] = []
        self.log: List[str] = []
        self._t0 = time.perf_counter()
        self._stop = False
        self._sched = threading.Thread(target=self._schedule, daemon=True)
        self._sched.start()

    # -- public API ---------------------------------------------------------------
    def submit(self, job: Job) -> Future:
        fut: Future = Future()
        job.arrival = time.perf_counter()
        job.footprint = self.footprint_fn(job)
        with self._lock:
            if job.footprint > self.budget:
                msg = (f"rejected {job.name or job.mesh}: needs {job.footprint / 2**30:.1f} GiB resident, "
                       f"budget {self.budget / 2**30:.1f} GiB (integrals cannot be resident)")
                self.log.append(msg)
                res = Result(job, error=msg)
                self._done.append(res)
                fut.set_result(res)
                return fut
            self._queue.append((job, fut))
            self._lock.notify_all()
        return fut

    def close(self, wait: bool = True):
        with self._lock:
            if wait:
                while self._queue or self._running:
                    self._lock.wait(0.05)
            self._stop = True
            self._lock.notify_all()
        self._sched.join(timeout=5)

    def stats(self) -> dict:
        done = [r for r in self._done if r.error is None]
        lat = [r.job.end - r.job.arrival for r in done]
        builds = sum(len(r.sigma) for r in done)
        span = (max(r.job.end for r in done) - min(r.job.arrival for r in done)) if done else 0.0
        return {"jobs": len(done), "rejected": sum(1 for r in self._done if r.error),
                "p50_s": float(np.percentile(lat, 50)) if lat else None,
                "p99_s": float(np.percentile(lat, 99)) if lat else None,
                "gw_builds_per_s": builds / span if span > 0 else None, "builds": builds, "span_s": span,
                "device_s": float(sum(r.job.device_s for r in done))}

    # -- scheduling -------------------------------------------------------------------
    def _schedule(self):
        while True:
            with self._lock:
                while not self._stop and not self._admissible():
                    self._lock.wait(0.05)
                if self._stop:
                    return
                job, fut = self._queue.pop(0)
                self._running += 1
                self._used += job.footprint
                self.log.append(f"admit {job.name or job.mesh} at {job.arrival - self._t0:.3f}s "
                                f"({job.footprint / 2**30:.2f} GiB, {self._running} running)")
            threading.Thread(target=self._run, args=(job, fut), daemon=True).start()

    def _admissible(self) -> bool:
        if not self._queue or self._running >= self.slots:
            return False
        job = self._queue[0]
        return self._used + job[0].footprint <= self.budget

    def _run(self, job: Job, fut: Future):
        job.start = time.perf_counter()
        try:
            res = self.executor(job, self.device)
        except Exception as e:  # the job fails, the server keeps serving
            res = Result(job, error=f"{type(e).__name__}: {e}")
        job.end = time.perf_counter()
        with self._lock:
            self._running -= 1
            self._used -= job.footprint
            self._done.append(res)
            self._lock.notify_all()
        fut.set_result(res)


def poisson_stream(server: Server, jobs: List[Job], rate_hz: float, seed: int = 0) -> List[Future]:
    """Submit `jobs` with exponential inter-arrival times of mean 1 / rate_hz."""
    rng = np.random.default_rng(seed)
    futs = []
    for j in jobs:
        time.sleep(float(rng.exponential(1.0 / rate_hz)))
        futs.append(server.submit(j))
    return futs


def config5_mix(n_jobs: int = 20, seed: int = 0, large_fraction: float = 0.1) -> List[Job]:
    """The serving mix: systems of the batched mix plus a fraction of 6x6x6 k, nao 104, NQ 800 jobs."""
    rng = np.random.default_rng(seed)
    meshes = [(2, 2, 2), (2, 2, 2), (3, 3, 3), (4, 4, 4)]
    naos = [20, 36, 52, 80]
    jobs = []
    for i in range(n_jobs):
        if rng.random() < large_fraction:
            jobs.append(Job(mesh=(6, 6, 6), nao=104, NQ=800, seed=i, name=f"large{i}"))
            continue
        nao = int(rng.choice(naos))
        jobs.append(Job(mesh=tuple(meshes[int(rng.integers(len(meshes)))]), nao=nao,
                        NQ=int(nao * rng.choice([6, 7, 8])), seed=i, name=f"job{i}"))
    return jobs
