"""Split-precision accuracy study: errors of Sigma, P0, K and two energies against FP64.

    python -m green_gpu_b200.accuracy [--mesh 2,2,2] [--nao 52] [--NQ 400] [--slices 2,3,4,5,6]

For each slice count the GW build (split P0 and Sigma contractions) and the HF exchange
(split exchange contraction) are compared with the FP64 engine on the same inputs:
* Sigma, P0, K: max |x - x_fp64| / max |x_fp64|;
* E_x = (1/nk) Re sum_{s,k} Tr(D_s(k) K_s(k)) (exchange energy) and
  E_GW = (1/nk) Re sum_{s,k} int_0^beta Tr(G(beta - tau) Sigma(tau)) dtau (trapezoid rule on
  the tau nodes; a Galitskii-Migdal-type correlation energy): relative error.
The energy reductions themselves are done in FP64.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import native, synth


def energies(s, K, Sigma):
    ex = np.einsum("skij,skji->", s.dm, K).real / s.nk
    tau = s.tau
    w = np.zeros(len(tau))
    dt = np.diff(tau)
    w[:-1] += 0.5 * dt
    w[1:] += 0.5 * dt
    G = s.G_tskij
    egw = 0.0
    for t in range(s.nts):
        egw += w[t] * np.einsum("skij,skji->", G[s.nts - 1 - t], Sigma[t]).real
    return ex, egw / s.nk


def run(mesh=(2, 2, 2), nao=52, NQ=400, slices=(2, 3, 4, 5, 6), seed=11):
    s = synth.make_system(mesh=mesh, nao=nao, NQ=NQ, ns=1, seed=seed)
    ctx = native.context_for(s)
    ref, cap = ctx.gw_sigma(s.G_tskij, precision=native.PREC_FP64, capture=True)
    ctx.set_hf_precision(native.PREC_FP64)
    Kref = ctx.hf_exchange(s.dm)
    e_ref = energies(s, Kref, ref)
    rows = []
    for S in slices:
        ctx.set_split_slices(S)
        out, c2 = ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT, capture=True)
        ctx.set_hf_precision(native.PREC_SPLIT)
        K = ctx.hf_exchange(s.dm)
        ctx.set_hf_precision(native.PREC_FP64)
        e = energies(s, K, out)
        rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
        rows.append({"slices": S, "sigma": rel(out, ref), "p0": rel(c2["P0"], cap["P0"]), "k": rel(K, Kref),
                     "e_x": abs(e[0] - e_ref[0]) / abs(e_ref[0]), "e_gw": abs(e[1] - e_ref[1]) / abs(e_ref[1])})
    ctx.close()
    return {"system": {"mesh": list(mesh), "nao": nao, "NQ": NQ, "nts": s.nts, "nw_b": s.nw_b},
            "energies_fp64": {"e_x": e_ref[0], "e_gw": e_ref[1]}, "rows": rows}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", default="2,2,2")
    ap.add_argument("--nao", type=int, default=52)
    ap.add_argument("--NQ", type=int, default=400)
    ap.add_argument("--slices", default="2,3,4,5,6")
    a = ap.parse_args(argv)
    res = run(tuple(int(x) for x in a.mesh.split(",")), a.nao, a.NQ, tuple(int(x) for x in a.slices.split(",")))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
