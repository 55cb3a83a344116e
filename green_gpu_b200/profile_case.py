"""Run one GW build (and one HF exchange) on a seeded synthetic system - the command that
profiling runs wrap, e.g.

    python -m green_gpu_b200.profile_case --mesh 2,2,1 --nao 52 --NQ 400 --precision fp64
"""
from __future__ import annotations

import argparse

import numpy as np

from . import native, synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", default="2,2,1")
    ap.add_argument("--nao", type=int, default=52)
    ap.add_argument("--NQ", type=int, default=400)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    ap.add_argument("--slices", type=int, default=5)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--fused-tail", action="store_true", help="Sigma tail as one kernel (gg_set_fused_tail)")
    a = ap.parse_args(argv)
    mesh = tuple(int(x) for x in a.mesh.split(","))
    s = synth.make_system(mesh=mesh, nao=a.nao, NQ=a.NQ, ns=1, seed=3)
    ctx = native.context_for(s)
    ctx.set_split_slices(a.slices)
    ctx.set_fused_tail(a.fused_tail)
    prec = native.PREC_SPLIT if a.precision == "split" else native.PREC_FP64
    for _ in range(a.repeat):
        out = ctx.gw_sigma(s.G_tskij, precision=prec)
    print("ok", float(np.abs(out).max()), ctx.timings(), ctx.launch_count())
    ctx.close()


if __name__ == "__main__":
    main()
