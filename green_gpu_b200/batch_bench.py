"""Batched uneven systems in one CUDA graph (gg_batch_*): eager one-by-one builds against one
replay of all systems' builds.

    python -m green_gpu_b200.batch_bench [--systems 24] [--precision split|fp64] [--max-v-gb 1.5]

The mix follows the batched-systems configuration: nao in {20, 36, 52, 80}, NQ = 6..8 nao,
k meshes 2x2x2 to 4x4x4 with time-reversal symmetry, IR Lambda in {1e3, 1e4}; shapes whose
resident footprint exceeds the per-system share of the device memory are drawn again, so that
the whole batch stays resident.  Prints one JSON line: per-system shapes, the sum of the eager build
times (CUDA events), the replay time of the batch graph, the speed-up and the largest relative
difference between a batched and an eager result.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import native, synth


def mix(n, seed=0, budget_gb=None):
    """n shapes drawn from the configuration's ranges; a draw whose resident footprint
    (gg_estimate_bytes: integrals + un-chunked work space) does not fit the budget left for it
    and the systems still to draw is drawn again, so that the whole batch stays resident."""
    rng = np.random.default_rng(seed)
    meshes = [(2, 2, 2), (3, 3, 3), (4, 4, 4)]
    left = budget_gb or 1e9

    def footprint(mesh, nao, NQ):
        nk = int(np.prod(mesh))
        return native.estimate_bytes(nk, nk, nk, nao, NQ, 1, 72, 69, nk * (nk + 1) // 2) / 2**30

    fmin = footprint((2, 2, 2), 20, 120)
    if fmin * n > left:
        raise ValueError(f"{n} systems do not fit {left:.1f} GB")
    out, tries = [], 0
    while len(out) < n:
        tries += 1
        if tries > 100000:
            raise RuntimeError("no mix fits the budget")
        nao = int(rng.choice([20, 36, 52, 80]))
        NQ = int(nao * rng.choice([6, 7, 8]))
        lam = float(rng.choice([1e3, 1e4]))
        mesh = meshes[int(rng.integers(len(meshes)))]
        fp = footprint(mesh, nao, NQ)
        # keep room for the remaining systems at the smallest footprint of the ranges
        if fp <= left - fmin * (n - len(out) - 1):
            out.append(dict(mesh=mesh, nao=nao, NQ=NQ, lam=lam, seed=seed * 1000 + len(out), footprint_gb=fp))
            left -= fp
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=24)
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--budget-gb", type=float, default=None, help="device memory for the batch (default 75%% of free)")
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    import torch
    dev = torch.device("cuda:0")
    prec = native.PREC_SPLIT if a.precision == "split" else native.PREC_FP64
    # the footprint estimate leaves out the split engine's slice planes: keep more room for them
    share = 0.5 if prec == native.PREC_SPLIT else 0.75
    budget = a.budget_gb or share * torch.cuda.mem_get_info(dev)[0] / 2**30
    shapes = mix(a.systems, a.seed, budget)
    items, bufs, ctxs, syss = [], [], [], []
    t0 = time.time()
    for sh in shapes:
        s = synth.make_system(mesh=sh["mesh"], nao=sh["nao"], NQ=sh["NQ"], ns=1, beta=100.0, lam=sh["lam"],
                              seed=sh["seed"], symmetry="tr")
        ctx = native.context_for(s)
        ctx.set_split_slices(a.slices)
        G = torch.from_numpy(s.G_tskij.view(np.float64)).to(dev)
        S = torch.zeros_like(G)
        items.append((ctx, G.data_ptr(), S.data_ptr()))
        bufs.append((G, S))
        ctxs.append(ctx)
        syss.append(s)
    setup_s = time.time() - t0
    torch.cuda.synchronize()
    # eager builds one after the other (each on its context stream, timed with CUDA events)
    eager_ms, eager_out = [], []
    for (ctx, gp, sp), (G, S) in zip(items, bufs):
        st = torch.cuda.Stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for rep in range(2):  # the first build allocates and builds tables
            e0.record(st)
            ctx.gw_sigma_device(gp, sp, precision=prec, stream=st.cuda_stream)
            e1.record(st)
            e1.synchronize()
        eager_ms.append(e0.elapsed_time(e1))
        eager_out.append(S.clone())
    batch = native.Batch(items, precision=prec)
    for (G, S) in bufs:
        S.zero_()
    torch.cuda.synchronize()
    reps = 3
    t = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream(dev)
        e0.record(st)
        batch.run(stream=st.cuda_stream)
        e1.record(st)
        e1.synchronize()
        t.append(e0.elapsed_time(e1))
    diff = max(float((S - E).abs().max() / E.abs().max()) for (G, S), E in zip(bufs, eager_out))
    batch.close()
    for c in ctxs:
        c.close()
    res = {"systems": len(shapes), "precision": a.precision, "slices": a.slices if prec == native.PREC_SPLIT else None,
           "shapes": [{"mesh": "x".join(map(str, d["mesh"])), "nao": d["nao"], "NQ": d["NQ"], "lambda": d["lam"],
                       "nts": s.nts, "nw_b": s.nw_b, "footprint_gb": round(d["footprint_gb"], 2)}
                      for d, s in zip(shapes, syss)],
           "eager_sum_ms": float(np.sum(eager_ms)), "batch_graph_ms": float(np.median(t)),
           "speedup": float(np.sum(eager_ms) / np.median(t)), "max_rel_diff_batch_vs_eager": diff,
           "setup_s": setup_s}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
