"""Benchmark: GW self-energy builds per second on B200 (one HF-exchange / GW iteration path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config cfg2|cfg1] [--precision split|fp64]

One step = one full GW Sigma build (G unfold, P0, IR transforms, FP64 Dyson, Sigma) of the
configured system with V, G and the IR transforms already resident in HBM.  The default
workload is the 4x4x4 k-mesh, nao = 52, NQ = 400, 72 tau / 69 bosonic frequencies system
(full BZ, identity symmetry) with seeded synthetic G and V; V (36 GB) is larger than L2.

Prints one JSON line (rank 0).  For N > 1 (torchrun), the irreducible q points are
distributed round-robin over ranks and the partial Sigma are summed with an NCCL
all-reduce, as the reference distributes q over device ranks and all-reduces Sigma.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "cfg1": dict(mesh=(2, 2, 2), nao=26, NQ=120),
    "cfg2": dict(mesh=(4, 4, 4), nao=52, NQ=400),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = str(device_index)
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.dev, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def make_inputs(cfg, device, seed=0):
    """Seeded synthetic system; V generated directly in HBM (36 GB for cfg2)."""
    import torch
    from green_gpu_b200 import synth
    s = synth.make_system(seed=seed, with_V=False, **CONFIGS[cfg])
    npairs = int(s.irre_pos_kpair.max()) + 1
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    V = torch.empty((npairs, s.NQ, s.nao, s.nao, 2), dtype=torch.float64, device=device)
    chunk = max(1, npairs // 16)
    scale = torch.exp(-0.1 * torch.arange(s.NQ, device=device, dtype=torch.float64)).view(1, s.NQ, 1, 1, 1)
    for p0 in range(0, npairs, chunk):
        blk = V[p0:p0 + chunk]
        blk.normal_(generator=g)
        blk.mul_(scale / np.sqrt(2.0))
    # V(k,k) must be Hermitian in (i, j): symmetrise the diagonal k-pairs on the device
    for k in range(s.nk):
        p = int(s.irre_pos_kpair[k * (k + 1) // 2 + k])
        Vc = torch.view_as_complex(V[p])
        Vc.copy_(0.5 * (Vc + Vc.conj().transpose(-1, -2)))
    torch.cuda.synchronize(device)
    return s, V


def _blas_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [d.get("num_threads") for d in threadpool_info() if d.get("user_api") == "blas"]
        if n and n[0]:
            return int(n[0])
    except Exception:
        pass
    return os.cpu_count()


class CpuSample:
    """The FP64 oracle on a bounded sample of one GW build of the configured system.

    Set-up (once): a system with the configured nao / NQ / tau grid and a 2-pair k store (the
    per-pair cost does not depend on the k mesh), the full-BZ G and one W~(tau).  One sample
    times one P0 (q, k) pair, one q of IR transforms + Dyson (all nw_b frequencies) and one
    Sigma (k, q') pair; a build is nk^2 P0 pairs + nq q steps + nk * nq Sigma pairs (full BZ,
    identity symmetry), so the extrapolated build time is nk^2 (t_p0 + t_sigma) + nk t_q.
    """

    def __init__(self, cfg):
        import oracle.gw as ogw
        from green_gpu_b200 import synth
        from oracle.symmetry import coulomb
        self.ogw = ogw
        c = CONFIGS[cfg]
        self.cfg = cfg
        self.NK = int(np.prod(c["mesh"]))
        if cfg == "cfg1":
            s = synth.make_system(seed=1, **c)
        else:
            s = synth.make_system(mesh=(2, 1, 1), nao=c["nao"], NQ=c["NQ"], seed=1)
        self.s = s
        self.Gf = ogw.g_full(s)
        self.pairs = []
        for k in range(s.nk):
            k1 = int(s.k1_from_k2q[k * s.nq + 0])
            self.pairs.append((k, k1, coulomb(s, k, k1)))
        P0 = np.zeros((s.nts, s.NQ, s.NQ), np.complex128)
        for t in range(s.nts):
            X = np.random.default_rng(t).standard_normal((s.NQ, s.NQ)) * 1e-3
            P0[t] = -(X @ X.T)
        self.P0 = P0
        self.Wt = ogw.transform_wt(ogw.dyson(ogw.transform_tw(P0, s.Tnt_BF)), s.Ttn_FB)
        n, N, T = s.nao, s.NQ, s.nts
        # reference FLOP model (8MNK + 12MN per complex GEMM, src/green/gpu/common_defs.h:121-125)
        self.f_p0 = (T // 2) * (2 * (8.0 * n * N * n * n) + 8.0 * N * N * n * n)
        self.f_sg = T * (2 * (8.0 * N * n * n * n) + 8.0 * N * N * n * n)
        self.i = 0

    def step(self):
        s, ogw = self.s, self.ogw
        nts = s.nts
        tt = np.arange(nts // 2)
        k, k1, V = self.pairs[self.i % len(self.pairs)]
        self.i += 1
        t0 = time.perf_counter()
        ogw.p0_pair(V, self.Gf[k1, 0, tt], self.Gf[k, 0, nts - 1 - tt], -2.0)
        t1 = time.perf_counter()
        ogw.transform_wt(ogw.dyson(ogw.transform_tw(self.P0, s.Tnt_BF)), s.Ttn_FB)
        t2 = time.perf_counter()
        ogw.sigma_pair(V, self.Gf[k1, 0], self.Wt)
        t3 = time.perf_counter()
        t_p0, t_q, t_sg = t1 - t0, t2 - t1, t3 - t2
        return {"t_p0": t_p0, "t_q": t_q, "t_sigma": t_sg,
                "seconds_per_build": self.NK * self.NK * (t_p0 + t_sg) + self.NK * t_q,
                "sample_s": t3 - t0}

    def describe(self, steps):
        tp = statistics.median([x["t_p0"] for x in steps])
        ts = statistics.median([x["t_sigma"] for x in steps])
        tq = statistics.median([x["t_q"] for x in steps])
        return (f"numpy FP64 oracle (OpenBLAS, {_blas_threads()} threads), {self.cfg}: per sample 1 P0 (q,k) pair "
                f"({tp:.2f} s, {self.f_p0 / tp / 1e9:.0f} GFLOP/s), 1 q of IR + Dyson over {self.s.nw_b} "
                f"frequencies ({tq:.2f} s), 1 Sigma (k,q') pair ({ts:.2f} s, {self.f_sg / ts / 1e9:.0f} GFLOP/s); "
                f"build = {self.NK}^2 x (P0 + Sigma pair) + {self.NK} q steps; {len(steps)} samples")


def oracle_cpu_baseline(cfg, samples=3, sampler=None):
    """Timed CPU baseline (rank 0, N = 1): a few samples of the oracle, extrapolated to builds/s."""
    cs = sampler or CpuSample(cfg)
    steps = [cs.step() for _ in range(samples)]
    t_build = statistics.median([x["seconds_per_build"] for x in steps])
    return {"value": 1.0 / t_build, "unit": "builds/s", "cores": _blas_threads(), "kind": "port",
            "sample": cs.describe(steps), "seconds_per_build": t_build}


def run_reference(args):
    """Reference arm: the reference's CPU path is the oracle port here (the reference itself
    cannot be built: MPI, HDF5, Eigen and the green-* repositories are absent).  Each step is
    one bounded sample of the build (one P0 pair, one q of IR + Dyson, one Sigma pair),
    extrapolated to a whole build."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cs = CpuSample(args.config)
    steps = [cs.step() for _ in range(args.warmup + args.steps)]
    timed = steps[args.warmup:]
    t_build = [x["seconds_per_build"] for x in timed]
    v = len(t_build) / sum(t_build)
    line = {"metric": "GW Sigma builds/s", "value": v, "unit": "builds/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(t_build) / len(t_build),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic (seeded G from random Hermitian Fock, Gaussian V*exp(-0.1Q))",
            "impl": "reference",
            "config": {"workload": f"GW Sigma build {args.config}",
                       "mesh": "x".join(map(str, CONFIGS[args.config]["mesh"])), "nao": CONFIGS[args.config]["nao"],
                       "NQ": CONFIGS[args.config]["NQ"], "precision": "fp64"},
            "cpu_baseline": {"value": v, "unit": "builds/s", "cores": _blas_threads(), "kind": "port",
                             "sample": cs.describe(timed)},
            "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="split", choices=["fp64", "split"])
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--solver", default="cholesky", choices=["cholesky", "lu"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="eager builds instead of graph replays")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 build of the same system")
    ap.add_argument("--no-autotune", action="store_true", help="tile widths and split-K by the rules only")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from green_gpu_b200 import native
    from green_gpu_b200.synth import gw_flop_model, gw_flop_parts

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=5), device_id=dev)

    s, V = make_inputs(args.config, dev)
    ctx = native.Context(s.nk, s.ink, s.inq, s.nao, s.NQ, s.ns, s.nts, s.nw_b, device=local)
    ctx.set_symmetry(s.k_full_to_reduced, s.k_reduced_to_full, s.k_tr_conj, s.q_full_to_reduced,
                     s.q_reduced_to_full, s.q_tr_conj, s.k1_from_k2q, s.k2_from_k1q)
    ctx.set_kpairs(int(s.irre_pos_kpair.max()) + 1, s.conj_kpair_list, s.trans_kpair_list, s.irre_pos_kpair)
    ctx.set_coulomb_device(V.data_ptr(), V)
    ctx.set_ir(s.Ttn_FB, s.Tnt_BF)
    ctx.set_q_shard(rank, world)
    ctx.set_split_slices(args.slices)
    prec = native.PREC_SPLIT if args.precision == "split" else native.PREC_FP64
    solver = native.SOLVER_CHOLESKY if args.solver == "cholesky" else native.SOLVER_LU
    G_host = torch.from_numpy(s.G_tskij.view(np.float64)).pin_memory()
    G = G_host.to(dev)
    Sigma = torch.empty_like(G)
    stream = torch.cuda.current_stream(dev)

    def step():
        ctx.gw_sigma_device(G.data_ptr(), Sigma.data_ptr(), solver=solver, precision=prec,
                            stream=stream.cuda_stream)
        if world > 1:
            dist.all_reduce(Sigma)

    # graph mode: the first warm-up build runs eagerly and is captured; the later builds replay
    # the captured graph (one launch per build).  No profiling events inside the timed region.
    ctx.set_graph(not args.no_graph)
    if args.precision == "split" and not args.no_autotune:
        ctx.set_autotune(True)  # the first warm-up build times the tile candidates of every shape
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lat = []
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            lat.append(a.elapsed_time(b) * 1e-3)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    elapsed = e0.elapsed_time(e1) * 1e-3
    if world > 1:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = args.steps / elapsed

    # one profiled build after the timed region (eager, CUDA events around every launch of the
    # dominant contractions): the per-kernel figures of the roofline and the launch count
    ctx.set_profiling(True)
    step()
    torch.cuda.synchronize(dev)
    ctx.set_profiling(False)
    launches_per_build = ctx.launch_count()
    phases = ctx.timings()
    kstats = {w: [0, 0.0, 0.0] for w in (0, 1, 2)}
    for w in (0, 1, 2):
        st = ctx.kernel_stats(w)
        kstats[w] = [st["launches"], st["seconds"], st["flops"]]

    # end to end through the host-buffer C ABI call (H2D of G from pinned memory, D2H of Sigma)
    e2e_vals = []
    out_host = np.empty_like(s.G_tskij)
    G_pinned_np = G_host.numpy().view(np.complex128).reshape(s.G_tskij.shape)
    Sigma_pinned = torch.empty_like(G_host).pin_memory() if world > 1 else None
    for _ in range(max(1, min(2, args.steps))):
        if world == 1:
            # the host-buffer C ABI call: H2D of G, the build, D2H of Sigma, timed inside
            ctx.gw_sigma(G_pinned_np, solver=solver, precision=prec)
            e2e_vals.append(ctx.timings().get("e2e", 0.0))
        else:
            # every rank: H2D of G from pinned memory, its q share, the all-reduce, D2H of Sigma;
            # CUDA events on the launching stream, max over ranks
            dist.barrier()
            torch.cuda.synchronize(dev)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            G.copy_(G_host, non_blocking=True)
            step()
            Sigma_pinned.copy_(Sigma, non_blocking=True)
            b.record(stream)
            b.synchronize()
            t = torch.tensor([a.elapsed_time(b) * 1e-3], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_vals.append(float(t.item()))
    e2e_t = [x for x in e2e_vals if x]
    gbytes = s.G_tskij.nbytes

    # roofline of the dominant contraction (largest device time)
    pk, pk_src = peaks()
    dom = max((0, 1, 2), key=lambda w: kstats[w][1])
    n_l, sec, fl = kstats[dom]
    achieved = fl / sec / 1e12 if sec > 0 else 0.0
    # the dominant kernels run inside a build of tens of seconds: sustained peaks
    fp64_peak = float(os.environ.get("GG_FP64_PEAK_TFLOPS", "37.0"))
    kname = ("p0_contraction", "sigma_contraction", "sigma_final_contraction")[dom]
    if args.precision == "fp64" or dom == 2:
        # the final product with V^+ is FP64 in both precisions
        peak, peak_note = fp64_peak, ("FP64 tensor (DMMA) rate measured on this pool's B200 with a register-only "
                                      "mma.sync f64 loop (37 TF/s; not part of MEASURED_PEAKS.json)")
        unit = "TFLOP/s"
        kname += " (FP64 DMMA zgemm)"
    else:
        # executed INT8 work: S(S+1)/2 slice pairs, each a real GEMM of 8MNK ops per complex GEMM
        pairs = args.slices * (args.slices + 1) // 2
        achieved *= pairs
        peak, peak_note = (2.0 * pk["bf16_tflops_sustained"],
                           f"2x {pk_src} bf16 sustained (dense INT8 rate; the kernel runs inside a long build)")
        unit = "TOP/s (int8)"
        kname += f" (slicing + tcgen05 INT8 GEMM, {args.slices} slices)"
    roof = {"bound": "tensor", "kernel": kname,
            "achieved": achieved, "peak": peak, "unit": unit, "frac": achieved / peak if peak else None,
            "traffic": None, "launches": n_l, "avg_launch_ms": 1e3 * sec / max(n_l, 1), "peak_source": peak_note,
            "model_tflops": fl / sec / 1e12 if sec > 0 else None}
    traffic_file = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            tr = json.load(f).get(f"{roof['kernel']}_{args.precision}_{args.config}")
        if tr:
            roof["traffic"] = tr["bytes_per_launch"]
            roof["traffic_unit"] = "bytes per launch (DRAM read + write, ncu)"
            roof["traffic_note"] = tr["note"]

    flops_build = gw_flop_model(s.nk, s.ink, s.inq, s.ns, s.nts, s.nw_b, s.nao, s.NQ)
    line = {
        "metric": "GW Sigma builds/s", "value": value, "unit": "builds/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "c128" if args.precision == "fp64" else "c128 in/out, int8 slices on tensor cores",
        "data": "synthetic (seeded G from random Hermitian Fock, Gaussian V*exp(-0.1Q))",
        "config": {"workload": f"GW Sigma build {args.config}", "mesh": "x".join(map(str, CONFIGS[args.config]["mesh"])),
                   "nao": s.nao, "NQ": s.NQ, "nts": s.nts, "nw_b": s.nw_b, "precision": args.precision,
                   "slices": args.slices if args.precision == "split" else None,
                   "solver": args.solver, "l2": "inputs larger than L2 (V = %.1f GB)" % (V.numel() * 8 / 1e9),
                   "parallelism": f"q-shard x{world}" if world > 1 else "1 GPU"},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "model_tflops": flops_build * value / 1e12,
        "phases_s": phases,
        "roofline": roof,
        "gpu_launches": launches_per_build * args.steps,
        "timed_region": ("graph replays, no profiling events" if not args.no_graph else "eager builds, no profiling "
                         "events") + "; phases_s and roofline from one profiled eager build after it",
        "autotune": ctx.autotune_report().splitlines() if args.precision == "split" and not args.no_autotune else None,
        "clocks": clk.summary(),
        "e2e": {"value": (1.0 / statistics.mean(e2e_t)) if e2e_t else None, "unit": "builds/s",
                "h2d_bytes_per_step": gbytes, "d2h_bytes_per_step": gbytes},
    }
    if world == 1 and args.precision == "split" and not args.no_fp64:
        # the same build in plain FP64 on the same inputs: its speed and the split path's error
        # against it (Sigma and the HF exchange K of the benchmarked system)
        ctx.set_graph(False)
        Sigma64 = torch.empty_like(G)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.gw_sigma_device(G.data_ptr(), Sigma64.data_ptr(), solver=solver, precision=native.PREC_FP64,
                            stream=stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        t64 = a.elapsed_time(b) * 1e-3
        sc = torch.view_as_complex(Sigma.view(-1, 2))
        s64 = torch.view_as_complex(Sigma64.view(-1, 2))
        err = float((sc - s64).abs().max() / s64.abs().max())
        ctx.set_hf_precision(native.PREC_FP64)
        K64 = ctx.hf_exchange(s.dm)
        ctx.set_hf_precision(native.PREC_SPLIT)
        Ksp = ctx.hf_exchange(s.dm)
        ctx.set_hf_precision(native.PREC_FP64)
        line["fp64"] = {"value": 1.0 / t64, "unit": "builds/s", "ms_per_step": 1e3 * t64, "steps": 1,
                        "note": "one eager FP64 build of the same system on the same inputs, CUDA events",
                        "split_speedup": value * t64}
        line["accuracy"] = {"sigma_max_rel_err_vs_fp64": err,
                            "k_max_rel_err_vs_fp64": float(np.abs(Ksp - K64).max() / np.abs(K64).max()),
                            "system": f"{args.config} (the benchmarked system)", "slices": args.slices,
                            "tolerance": 1e-8}
        del Sigma64
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = oracle_cpu_baseline(args.config)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
