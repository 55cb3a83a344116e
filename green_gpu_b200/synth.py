"""Seeded synthetic inputs for the HF-exchange / GW self-energy path.

A :class:`System` bundles everything one HF + GW build consumes, in the
layouts the reference passes across its plugin boundary:

* ``G_tskij``  [nts][ns][ink][nao][nao] complex128 - G(tau) on the IBZ
  (``gpu_factory.h:78-89``, ``gw_gpu_kernel.cpp:431-441``);
* ``V_stored`` [num_kpair_stored][NQ][nao][nao] complex128 - density-fitted
  Coulomb integrals for the irreducible k-pairs ``k1 >= k2``
  (``df_integral_t.h:96-129, 175-235``);
* ``Ttn_FB`` [nts][nw_b], ``Tnt_BF`` [nw_b][nts-2] - IR transforms
  (``cuda_common.cu:93-108``);
* the k/q symmetry maps and AO / auxiliary rotations
  (``cu_symmetry.h:41-66``, ``gw_gpu_kernel.cpp:34-91``);
* ``S_k``, ``madelung`` for the HF Ewald term (``hf_gpu_kernel.cpp:188-201``).

Construction (matching the stated benchmark recipe): a random Hermitian Fock
matrix per (s, k) with eigenvalues uniform in [-2, 2] Ha at mu = 0 gives
``G_k(tau) = -U diag(e^{-eps tau} / (1 + e^{-beta eps})) U^+``; ``V^Q_ij(k1,k2)``
is complex Gaussian scaled by ``exp(-0.1 Q)`` with
``V^Q_ij(k1,k2) = conj(V^Q_ji(k2,k1))``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .ir import ir_matrices


def tri(k1: int, k2: int) -> int:
    """Triangular k-pair index used by the integral store (df_integral_t.h:68-70)."""
    return k1 * (k1 + 1) // 2 + k2 if k1 >= k2 else k2 * (k2 + 1) // 2 + k1


@dataclass
class System:
    nk: int
    ink: int
    nq: int
    inq: int
    nao: int
    NQ: int
    ns: int
    nts: int
    nw_b: int
    beta: float
    # k-mesh symmetry (cu_symmetry_data)
    k_full_to_reduced: np.ndarray
    k_reduced_to_full: np.ndarray
    k_tr_conj: np.ndarray
    k_stars: List[np.ndarray]
    q_full_to_reduced: np.ndarray
    q_reduced_to_full: np.ndarray
    q_tr_conj: np.ndarray
    q_stars: List[np.ndarray]
    k1_from_k2q: np.ndarray   # flat [k * nq + q] -> k + q
    k2_from_k1q: np.ndarray   # flat [k * nq + q] -> k - q
    U_k: Optional[np.ndarray]  # [nk][nao][nao] or None (identity)
    U_q: Optional[np.ndarray]  # [nq][NQ][NQ] or None (identity)
    # k-pair store (df_integral_t)
    conj_kpair_list: np.ndarray
    trans_kpair_list: np.ndarray
    irre_pos_kpair: np.ndarray
    V_stored: np.ndarray
    # inputs of one iteration
    G_tskij: np.ndarray
    Ttn_FB: np.ndarray
    Tnt_BF: np.ndarray
    tau: Optional[np.ndarray] = None
    S_k: Optional[np.ndarray] = None
    madelung: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def num_kpair_stored(self) -> int:
        return int(self.V_stored.shape[0])

    @property
    def dm(self) -> np.ndarray:
        """Density-matrix argument of the HF callback: G(tau = beta) (cu_solver_test.cpp:91)."""
        return self.G_tskij[self.nts - 1]

    def flops_gw(self) -> float:
        """The reference's GW operation count (gw_gpu_kernel.cpp:93-136)."""
        return gw_flop_model(self.nk, self.ink, self.inq, self.ns, self.nts, self.nw_b, self.nao, self.NQ)

    def flops_hf(self) -> float:
        """The reference's HF exchange operation count (hf_gpu_kernel.cpp:211-227)."""
        return hf_flop_model(self.nk, self.ink, self.ns, self.nao, self.NQ)


def matmul_cost(M, N, K):
    """8MNK + 12MN, the reference's complex GEMM cost (common_defs.h:121-125)."""
    return 8.0 * M * N * K + 12.0 * M * N


def gw_flop_model(nk, ink, inq, ns, nts, nw_b, nao, NQ):
    naosq = nao * nao
    NQsq = float(NQ) * NQ
    first = inq * nk * ns * nts / 2.0 * (matmul_cost(nao * NQ, nao, nao) + matmul_cost(NQ * nao, nao, nao)
                                         + matmul_cost(NQ, naosq, NQ))
    per_transform = 2.0 * ns * nts * matmul_cost(nao, nao, nao)
    transforms = inq * nk * 2.0 * per_transform + ink * nk * per_transform
    fourier = inq * (matmul_cost(NQsq, nts, nw_b) + matmul_cost(NQsq, nw_b, nts))
    solver = 2.0 / 3.0 * inq * nw_b * (NQsq * NQ + NQsq)
    second = ink * nk * ns * nts * (matmul_cost(NQ * nao, nao, nao) + matmul_cost(naosq, NQ, NQ)
                                    + matmul_cost(nao, NQ * nao, nao))
    return first + transforms + fourier + solver + second


def gw_flop_parts(nk, ink, inq, ns, nts, nw_b, nao, NQ):
    naosq = nao * nao
    NQsq = float(NQ) * NQ
    return {
        "p0": inq * nk * ns * nts / 2.0 * (matmul_cost(nao * NQ, nao, nao) + matmul_cost(NQ * nao, nao, nao)
                                           + matmul_cost(NQ, naosq, NQ)),
        "p0_main": inq * nk * ns * nts / 2.0 * matmul_cost(NQ, naosq, NQ),
        "sigma": ink * nk * ns * nts * (matmul_cost(NQ * nao, nao, nao) + matmul_cost(naosq, NQ, NQ)
                                        + matmul_cost(nao, NQ * nao, nao)),
        "sigma_main": ink * nk * ns * nts * matmul_cost(naosq, NQ, NQ),
        "fourier": inq * (matmul_cost(NQsq, nts, nw_b) + matmul_cost(NQsq, nw_b, nts)),
        "solver": 2.0 / 3.0 * inq * nw_b * (NQsq * NQ + NQsq),
    }


def hf_flop_model(nk, ink, ns, nao, NQ):
    naosq = nao * nao
    return ink * ns * nk * (matmul_cost(NQ * nao, nao, nao) + matmul_cost(nao, nao, NQ * nao)) \
        + ink * ns * matmul_cost(1, naosq, nk)


def _mesh_maps(mesh):
    n1, n2, n3 = mesh
    nk = n1 * n2 * n3
    idx = np.arange(nk)
    c = np.stack([idx // (n2 * n3), (idx // n3) % n2, idx % n3], axis=1)

    def index(v):
        v = v % np.array(mesh)
        return (v[..., 0] * n2 + v[..., 1]) * n3 + v[..., 2]

    k1_from_k2q = index(c[:, None, :] + c[None, :, :]).reshape(-1)   # [k2*nq + q] = k2 + q
    k2_from_k1q = index(c[:, None, :] - c[None, :, :]).reshape(-1)   # [k1*nq + q] = k1 - q
    minus = index(-c)
    return nk, k1_from_k2q.astype(np.int64), k2_from_k1q.astype(np.int64), minus.astype(np.int64)


def _green_tau(F, tau, beta):
    """-U diag(e^{-eps tau}/(1+e^{-beta eps})) U^+ for Hermitian F, overflow-free."""
    eps, U = np.linalg.eigh(F)
    tau = np.asarray(tau)[:, None]
    e = eps[None, :]
    pos = e >= 0
    ep = np.where(pos, e, 0.0)
    en = np.where(pos, 0.0, e)
    g = np.where(pos, np.exp(-tau * ep) / (1.0 + np.exp(-beta * ep)),
                 np.exp((beta - tau) * en) / (1.0 + np.exp(beta * en)))
    return -np.einsum("ia,ta,ja->tij", U, g, U.conj())


def make_system(mesh=(2, 2, 2), nao=26, NQ=120, ns=1, beta=100.0, lam=1e4, nts=72, nw_b=69,
                seed=0, symmetry="none", with_V=True) -> System:
    """Build a seeded synthetic system.

    ``symmetry='none'``: identity maps (ink = nk, inq = nq, U = I, no TR).
    ``symmetry='tr'``: time reversal only; k and -k form a star, G(-k) = conj G(k),
    V(-k1,-k2) = conj V(k1,k2), handled through the conjugated k-pair list exactly as
    the integral store does (df_integral_t.h:153-173).
    """
    rng = np.random.default_rng(seed)
    nk, k1_from_k2q, k2_from_k1q, minus = _mesh_maps(mesh)
    if symmetry == "none":
        rep = np.arange(nk)
        tr = np.zeros(nk, np.int64)
    elif symmetry == "tr":
        rep = np.minimum(np.arange(nk), minus)
        tr = (np.arange(nk) != rep).astype(np.int64)
    else:
        raise ValueError(symmetry)
    reduced_to_full = np.unique(rep)
    ink = len(reduced_to_full)
    pos = {int(k): i for i, k in enumerate(reduced_to_full)}
    full_to_reduced = np.array([pos[int(r)] for r in rep], np.int64)
    stars = [np.array([k for k in range(nk) if rep[k] == r], np.int64) for r in reduced_to_full]

    # Fock matrices on the IBZ reps, G(tau) on the tau grid
    tau, Ttn_FB, Tnt_BF = ir_matrices(beta, lam, nts, nw_b)
    G = np.empty((nts, ns, ink, nao, nao), np.complex128)
    S_k = np.empty((ns, ink, nao, nao), np.complex128)
    for s in range(ns):
        for ik in range(ink):
            X = rng.standard_normal((nao, nao)) + 1j * rng.standard_normal((nao, nao))
            if symmetry == "tr" and minus[reduced_to_full[ik]] == reduced_to_full[ik]:
                X = X.real  # a time-reversal invariant k (k = -k) has a real Fock matrix
            Q, _ = np.linalg.qr(X)
            eps = rng.uniform(-2.0, 2.0, nao)
            F = (Q * eps) @ Q.conj().T
            F = 0.5 * (F + F.conj().T)
            G[:, s, ik] = _green_tau(F, tau, beta)
            Y = rng.standard_normal((nao, nao)) + 1j * rng.standard_normal((nao, nao))
            S_k[s, ik] = np.eye(nao) + 0.05 * (Y @ Y.conj().T) / nao

    # k-pair store: irreducible pairs k1 >= k2 (and, under TR, one of (k1,k2)/(-k1,-k2))
    npairs = nk * (nk + 1) // 2
    conj_list = np.arange(npairs, dtype=np.int64)
    trans_list = np.arange(npairs, dtype=np.int64)
    if symmetry == "tr":
        for k1 in range(nk):
            for k2 in range(k1 + 1):
                idx = tri(k1, k2)
                m1, m2 = minus[k1], minus[k2]
                # V(k1,k2) = conj V(-k1,-k2).  If -k1 >= -k2 the partner is stored as
                # (-k1,-k2) itself (conjugated pair); otherwise as (-k2,-k1), and
                # conj V(-k1,-k2) = V(-k2,-k1)^T (transposed pair).
                partner = tri(m1, m2)
                if partner < idx:
                    if m1 >= m2:
                        conj_list[idx] = partner
                    else:
                        trans_list[idx] = partner
    # pairs mapped onto themselves by time reversal: (-k1,-k2) = (k1,k2) needs a real V,
    # (-k1,-k2) = (k2,k1) needs V^Q symmetric in (i,j)
    self_real, self_sym = set(), set()
    if symmetry == "tr":
        for k1 in range(nk):
            for k2 in range(k1 + 1):
                m1, m2 = minus[k1], minus[k2]
                if (m1, m2) == (k1, k2):
                    self_real.add(tri(k1, k2))
                elif (m1, m2) == (k2, k1):
                    self_sym.add(tri(k1, k2))
    irre = np.array([i for i in range(npairs) if conj_list[i] == i and trans_list[i] == i], np.int64)
    irre_pos = -np.ones(npairs, np.int64)
    irre_pos[irre] = np.arange(len(irre))
    V = None
    if with_V:
        scale = np.exp(-0.1 * np.arange(NQ))[None, :, None, None]
        V = (rng.standard_normal((len(irre), NQ, nao, nao))
             + 1j * rng.standard_normal((len(irre), NQ, nao, nao))) * (scale / np.sqrt(2.0))
        # diagonal pairs (k,k) must be Hermitian in (i,j): V(k,k) = V(k,k)^+
        kp_of = {}
        for k1 in range(nk):
            for k2 in range(k1 + 1):
                kp_of[tri(k1, k2)] = (k1, k2)
        for p, idx in enumerate(irre):
            k1, k2 = kp_of[int(idx)]
            if int(idx) in self_real:
                V[p] = V[p].real
            if int(idx) in self_sym:
                V[p] = 0.5 * (V[p] + np.swapaxes(V[p], -1, -2))
            if k1 == k2:
                V[p] = 0.5 * (V[p] + np.conj(np.swapaxes(V[p], -1, -2)))
        V = np.ascontiguousarray(V)
        # a conj-related diagonal pair (k,k) ~ (-k,-k) is consistent only if the stored
        # partner is itself Hermitian, which holds by construction above.
    sys_ = System(
        nk=nk, ink=ink, nq=nk, inq=ink, nao=nao, NQ=NQ, ns=ns, nts=nts, nw_b=nw_b, beta=beta,
        k_full_to_reduced=full_to_reduced, k_reduced_to_full=reduced_to_full.astype(np.int64),
        k_tr_conj=tr, k_stars=stars,
        q_full_to_reduced=full_to_reduced.copy(), q_reduced_to_full=reduced_to_full.astype(np.int64).copy(),
        q_tr_conj=tr.copy(), q_stars=[s_.copy() for s_ in stars],
        k1_from_k2q=k1_from_k2q, k2_from_k1q=k2_from_k1q, U_k=None, U_q=None,
        conj_kpair_list=conj_list, trans_kpair_list=trans_list, irre_pos_kpair=irre_pos,
        V_stored=V if V is not None else np.zeros((len(irre), NQ, nao, nao), np.complex128)[:0],
        G_tskij=G, Ttn_FB=Ttn_FB, Tnt_BF=Tnt_BF, tau=tau, S_k=S_k, madelung=0.15,
        meta={"mesh": tuple(mesh), "seed": seed, "symmetry": symmetry, "lambda": lam},
    )
    return sys_


def unfold_kpairs(sys_: System) -> System:
    """Return the same system with every k-pair stored explicitly (no k-pair symmetry).

    Used to check that the symmetry-reduced store and the explicit one agree.
    """
    from copy import copy
    nk = sys_.nk
    npairs = nk * (nk + 1) // 2
    out = copy(sys_)
    V = np.empty((npairs, sys_.NQ, sys_.nao, sys_.nao), np.complex128)
    for k1 in range(nk):
        for k2 in range(k1 + 1):
            V[tri(k1, k2)] = coulomb_pair(sys_, k1, k2)
    out.V_stored = V
    out.conj_kpair_list = np.arange(npairs, dtype=np.int64)
    out.trans_kpair_list = np.arange(npairs, dtype=np.int64)
    out.irre_pos_kpair = np.arange(npairs, dtype=np.int64)
    return out


def kpair_lookup(sys_: System, k1: int, k2: int):
    """(stored position, dagger, conj, transpose) for V(k1,k2) (df_integral_t.h:153-235)."""
    idx = tri(k1, k2)
    dagger = k1 < k2
    conj = trans = False
    if sys_.conj_kpair_list[idx] != idx:
        idx = int(sys_.conj_kpair_list[idx])
        conj = True
    elif sys_.trans_kpair_list[idx] != idx:
        idx = int(sys_.trans_kpair_list[idx])
        trans = True
    pos = int(sys_.irre_pos_kpair[idx])
    if pos < 0:
        raise KeyError(f"k-pair ({k1},{k2}) maps to a non-stored pair {idx}")
    return pos, dagger, conj, trans


def coulomb_pair(sys_: System, k1: int, k2: int) -> np.ndarray:
    """V^Q(k1,k2) [NQ][nao][nao] built from the store like df_integral_t::symmetrize."""
    pos, dagger, conj, trans = kpair_lookup(sys_, k1, k2)
    V = sys_.V_stored[pos]
    if dagger:
        V = np.conj(np.swapaxes(V, -1, -2))
    if conj:
        V = np.conj(V)
    elif trans:
        V = np.swapaxes(V, -1, -2)
    return np.ascontiguousarray(V)


def make_x2c_system(mesh=(2, 1, 1), nao=6, NQ=20, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=0,
                    spin_orbit=0.3) -> System:
    """Two-component system: the scalar system's integrals, IR transforms and identity symmetry,
    with spinor G(tau) [nts][1][ink][2 nao][2 nao] from random Hermitian spinor Fock matrices
    whose spin blocks are coupled (the ab block scaled by ``spin_orbit``) and a spin-independent
    overlap S_k = diag(S, S).  ``nao`` counts orbitals per spin."""
    base = make_system(mesh=mesh, nao=nao, NQ=NQ, ns=1, beta=beta, lam=lam, nts=nts, nw_b=nw_b, seed=seed,
                       symmetry="none")
    rng = np.random.default_rng(seed + 1000)
    n2 = 2 * nao
    G = np.zeros((nts, 1, base.ink, n2, n2), np.complex128)
    S = np.zeros((1, base.ink, n2, n2), np.complex128)
    for ik in range(base.ink):
        X = rng.standard_normal((n2, n2)) + 1j * rng.standard_normal((n2, n2))
        X[:nao, nao:] *= spin_orbit
        X[nao:, :nao] *= spin_orbit
        Fk = 0.5 * (X + X.conj().T)
        eps, Q = np.linalg.eigh(Fk)
        F = (Q * rng.uniform(-2.0, 2.0, n2)) @ Q.conj().T
        F = 0.5 * (F + F.conj().T)
        G[:, 0, ik] = _green_tau(F, base.tau, beta)
        S[0, ik, :nao, :nao] = base.S_k[0, ik]
        S[0, ik, nao:, nao:] = base.S_k[0, ik]
    base.G_tskij = G
    base.S_k = S
    base.meta = dict(base.meta, x2c=True)
    return base
