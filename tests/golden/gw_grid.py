"""The imaginary-time grid of the reference's GW fixture, recovered from the fixture itself.

The reference's GW test (test/cu_solver_test.cpp:226-288) reads its transforms Ttn_FB / Tnt_BF
from green-grids' ``ir/1e4.h5`` (beta = 100, Lambda = 1e4; nts = ncoeff + 2 = 110 at :260-264),
which is not in the reference tree.  Its ``G_tau`` (test/data/GW/data.h5) is the mean-field G
of ``HF/Fock-k`` and ``HF/S-k`` (test/data/GW/input.h5, the same arrays as the HF fixture):
with F x_n = e_n S x_n (x_n^+ S x_m = delta_nm),

    d_n(tau) = -x_n^+ S G(tau) S x_n = exp(-(e_n - mu) tau) / (1 + exp(-beta (e_n - mu)))

and the off-diagonal elements vanish (checked below).  So every tau node follows from the
diagonal d_n(tau) once mu is known, and mu is the value for which one tau fits all orbitals
of all k points and spins.  Each orbital gives tau_n = -(ln d_n + ln(1 + e^{-beta x_n})) / x_n
(x_n = e_n - mu), accurate where d_n is not small; the nodes are the weighted means with
weights (d_n |x_n|)^2.  The transforms on these nodes then come from
``green_gpu_b200.ir.ir_matrices_on_grid``.
"""
import numpy as np
import scipy.linalg as sla
from scipy.optimize import minimize_scalar

BETA = 100.0
LAMBDA = 1e4


def _orbital_occupations(G, F, S, ibz):
    """d_n(tau) for every (spin, IBZ k, orbital): [nts][ns * ink * nao], energies alike."""
    nts, ns, ink = G.shape[:3]
    eps, dv, off = [], [], 0.0
    for s in range(ns):
        for ik, k in enumerate(ibz):
            e, X = sla.eigh(F[s, k], S[s, k])
            XS = X.conj().T @ S[s, k]
            D = -np.einsum("ia,tab,bj->tij", XS, G[:, s, ik], XS.conj().T)
            off = max(off, float(np.abs(D - np.einsum("tii->ti", D)[:, :, None] * np.eye(len(e))).max()))
            eps.extend(e)
            dv.append(np.einsum("tii->ti", D).real)
    return np.array(eps), np.concatenate(dv, axis=1), off


def _taus(eps, dv, mu, beta):
    x = eps - mu
    # ln(1 + e^{-beta x}) without overflow
    lg = np.where(x >= 0, np.log1p(np.exp(-beta * np.abs(x))), -beta * x + np.log1p(np.exp(-beta * np.abs(x))))
    with np.errstate(divide="ignore", invalid="ignore"):
        est = -(np.log(np.clip(dv, 1e-300, None)) + lg[None, :]) / x[None, :]
    w = (np.clip(dv, 0.0, None) * np.abs(x)[None, :]) ** 2
    tau = (w * est).sum(axis=1) / w.sum(axis=1)
    spread = np.sqrt((w * (est - tau[:, None]) ** 2).sum(axis=1) / w.sum(axis=1))
    return tau, spread


def recover_tau(G, F, S, ibz, beta=BETA):
    """(tau nodes incl. 0 and beta, mu, largest off-diagonal element of the MO-basis G)."""
    eps, dv, off = _orbital_occupations(G, F, S, ibz)
    lo, hi = eps[eps < 0].max(), eps[eps > 0].min()
    r = minimize_scalar(lambda mu: float((_taus(eps, dv, mu, beta)[1] ** 2).sum()), bounds=(lo + 1e-4, hi - 1e-4),
                        method="bounded", options={"xatol": 1e-13})
    tau, _ = _taus(eps, dv, r.x, beta)
    tau = 0.5 * (tau + (beta - tau[::-1]))  # the grid is symmetric under tau -> beta - tau
    tau[0], tau[-1] = 0.0, beta
    return tau, float(r.x), off


def fixture_transforms(nw_b=81):
    """(tau, Ttn_FB, Tnt_BF) for the reference's GW fixture (hf_h2_27k.npz)."""
    import os

    from green_gpu_b200.ir import ir_matrices_on_grid
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "hf_h2_27k.npz"))
    ibz = d["k_ibz2bz"].astype(np.int64)
    tau, _, _ = recover_tau(d["G_tau_gw"], d["Fock_k_full"], d["S_k_full"], ibz)
    Ttn, Tnt = ir_matrices_on_grid(tau, BETA, LAMBDA, nw_b)
    return tau, Ttn, Tnt
