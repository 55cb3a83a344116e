"""Oracle: one GW self-energy build in FP64 numpy (test infrastructure only).

Restates src/cugw_utils.cu:104-202 (loop structure), src/cugw_qkpt.cu:203-338
(contractions), src/cugw_qpt.cu:179-358 (scaling, IR transforms, Dyson solve),
src/cuda_common.cu:249-281 (Hermitian symmetrisation) and
src/gw_gpu_kernel.cpp:185-188, 431-441 (tau reversal, division by nk).
"""
import numpy as np
import scipy.linalg as sla

from .symmetry import coulomb, unfold_ao


def g_full(sys_):
    """G(k_full) for every full-BZ k: [nk][ns][nts][nao][nao].

    G_tskij is [t][s][k_ibz][i][j] (gw_gpu_kernel.cpp:431-441); the rotation is
    cu_symmetry.cu:183-233.
    """
    G = np.moveaxis(sys_.G_tskij, 2, 0)  # [ink][t][s][i][j]
    out = np.empty((sys_.nk, sys_.ns, sys_.nts, sys_.nao, sys_.nao), np.complex128)
    for k in range(sys_.nk):
        kr = sys_.k_full_to_reduced[k]
        X = G[kr]  # [t][s][i][j]
        if sys_.U_k is not None:
            U = sys_.U_k[k]
            X = U @ X @ U.conj().T
        if sys_.k_tr_conj[k]:
            X = np.conj(X)
        out[k] = np.swapaxes(X, 0, 1)
    return out


def p0_pair(V, G1, G0m, pref):
    """One (q,k) P0 contribution for all t < nt/2 (src/cugw_qkpt.cu:203-234).

    V = V(k, k1) [NQ][n][n]; G1 = G^{k1}(tau_t) [nt2][n][n];
    G0m = G^k(tau_{nt-1-t}) [nt2][n][n].
    X1[t][a][b][Q'] = sum_p G0m_{ap} V^{Q'}_{pb}  (cugw_qkpt.cu:214, with V_pmQ = V^T from :125)
    X2[t][Q][a][b]  = sum_l G1_{bl} conj(V^Q_{al}) (cugw_qkpt.cu:220, conj from :128)
    P0[t][Q'][Q]    = pref sum_{ab} X2[Q][ab] X1[ab][Q']  (cugw_qkpt.cu:225)
    """
    NQ, n, _ = V.shape
    nt = len(G1)
    # every contraction is a BLAS matmul: A[t] = G0m[t] @ V_(p, Q b), B[t] = conj(V)_(Q a, l) @ G1[t]^T
    Vp = np.ascontiguousarray(V.transpose(1, 0, 2)).reshape(n, NQ * n)  # [p][(Q, b)]
    A = np.matmul(G0m, Vp).reshape(nt, n, NQ, n).transpose(0, 2, 1, 3).reshape(nt, NQ, n * n)
    Vc = np.conj(V).reshape(NQ * n, n)  # [(Q, a)][l]
    B = np.matmul(Vc, np.swapaxes(G1, 1, 2)).reshape(nt, NQ, n * n)  # [t][Q][(a, b)]
    return pref * np.matmul(A, np.swapaxes(B, 1, 2))


def p0_q(sys_, Gf, q_full):
    """Bare polarisation for one q (P0 loop of src/cugw_utils.cu:118-149), unscaled, t < nt/2."""
    ns, nts = sys_.ns, sys_.nts
    nt2 = nts // 2
    pref = -2.0 if ns == 1 else -1.0
    P0 = np.zeros((nt2, sys_.NQ, sys_.NQ), np.complex128)
    tt = np.arange(nt2)
    for k in range(sys_.nk):
        k1 = sys_.k1_from_k2q[k * sys_.nq + q_full]
        V = coulomb(sys_, k, k1)
        for s in range(ns):
            P0 += p0_pair(V, Gf[k1, s, tt], Gf[k, s, nts - 1 - tt], pref)
    return P0


def scale_mirror(P0_half, nk, nts):
    """P0 *= 1/nk for t < nt/2, then P0[nt-1-t] = P0[t] (src/cugw_qpt.cu:179-191)."""
    P0 = np.empty((nts,) + P0_half.shape[1:], np.complex128)
    P0[: nts // 2] = P0_half / nk
    for t in range(nts // 2):
        P0[nts - t - 1] = P0[t]
    return P0


def transform_tw(P0, Tnt_BF):
    """P~[w] = sum_{t=1}^{nt-2} Tnt_BF[w][t-1] P0[t] (src/cugw_qpt.cu:329-339)."""
    nts = P0.shape[0]
    return np.tensordot(Tnt_BF, P0[1:nts - 1], axes=(1, 0))


def transform_wt(Pw, Ttn_FB):
    """W~[t] = sum_w Ttn_FB[t][w] W~[w] (src/cugw_qpt.cu:341-358)."""
    return np.tensordot(Ttn_FB, Pw, axes=(1, 0))


def hermitian_symmetrize(M):
    """Lower triangle averaged with the conjugate upper one; real diagonal.

    src/cuda_common.cu:249-265: for i>j, M[i][j] <- (M[i][j] + conj M[j][i])/2,
    M[j][i] <- conj of that; M[i][i] <- Re M[i][i].
    """
    n = M.shape[-1]
    L = np.tril(M, -1)
    U = np.triu(M, 1)
    low = 0.5 * (L + np.conj(np.swapaxes(U, -1, -2)))
    out = low + np.conj(np.swapaxes(low, -1, -2))
    d = np.real(np.diagonal(M, axis1=-2, axis2=-1))
    out[..., np.arange(n), np.arange(n)] = d
    return out


def dyson(Pw, solver="cholesky"):
    """W~[w] = solve((I - P~), P~) per frequency (src/cugw_qpt.cu:223-322).

    The reference hands row-major buffers to column-major cuSOLVER/cuBLAS, so the
    solved quantity is X_rm = P~ (I - P~)^{-1}; P~ is Hermitian-symmetrised first
    (cuda_common.cu:249-281) and the LU result is symmetrised again (cugw_qpt.cu:314-316).
    """
    n = Pw.shape[-1]
    out = np.empty_like(Pw)
    I = np.eye(n)
    for w in range(Pw.shape[0]):
        P = hermitian_symmetrize(Pw[w])
        A = I - P
        # column-major view: A_cm = A^T, B_cm = P^T; X_cm = A_cm^{-1} B_cm; X_rm = X_cm^T
        if solver == "cholesky":
            c = sla.cho_factor(A.T, lower=True)
            X = sla.cho_solve(c, P.T).T
        else:
            lu = sla.lu_factor(A.T)
            X = sla.lu_solve(lu, P.T).T
            X = hermitian_symmetrize(X)
        out[w] = X
    return out


def sigma_pair(V, G1, Wt, ns_pref=-1.0):
    """Sigma contribution of one (k, q') pair for all t (src/cugw_qkpt.cu:248-338).

    Y1[t][Q][j][c] = (V^Q G1_t)_{jc}       (cugw_qkpt.cu:297)
    Y2[t][(j,c)][Q] = sum_P W[t][P][Q] Y1[t][P][j][c]   (cugw_qkpt.cu:322; row-major W)
    Sigma[t][j][i] = -sum_{c,Q} Y2[t][(j,c)][Q] conj(V^Q_{ic})  (cugw_qkpt.cu:329)
    """
    NQ, n, _ = V.shape
    nt = len(G1)
    # the three contractions as BLAS matmuls (an einsum with a shared batch index does not
    # reach BLAS): Y1[t] = V_(Q j, l) @ G1[t]; Y2[t] = W[t]^T @ Y1[t]_(P, j c);
    # Sigma[t] = Y2[t]_(j, Q c) @ conj(V)_(Q c, i)
    Y1 = np.matmul(V.reshape(NQ * n, n), G1).reshape(nt, NQ, n * n)
    Y2 = np.matmul(np.swapaxes(Wt, 1, 2), Y1).reshape(nt, NQ, n, n)
    Y2 = np.ascontiguousarray(Y2.transpose(0, 2, 1, 3)).reshape(nt, n, NQ * n)
    Vh = np.ascontiguousarray(np.conj(V).transpose(0, 2, 1)).reshape(NQ * n, n)  # [(Q, c)][i]
    return ns_pref * np.matmul(Y2, Vh)


def rotate_w(sys_, Wt, q_deg):
    """W for a star member: U_q W U_q^+ or conj of it for TR partners (src/cugw_utils.cu:240-269,
    cugw_qkpt.cu:297-318 with U / U_conj chosen by the caller)."""
    out = Wt
    if sys_.U_q is not None:
        U = sys_.U_q[q_deg]
        out = U @ out @ U.conj().T
    if sys_.q_tr_conj[q_deg]:
        out = np.conj(out)
    return out


def gw_build(sys_, solver="cholesky", keep=None, q_subset=None):
    """Full GW self-energy build; returns Sigma [nts][ns][ink][nao][nao] (already / nk).

    src/cugw_utils.cu:104-202 for the q loop, src/gw_gpu_kernel.cpp:185-188 for / nk.
    If ``keep`` is a dict, intermediates P0 [inq][nts][NQ][NQ], Pw, Wt are stored in it.
    ``q_subset`` restricts the irreducible q points (one device rank's share,
    cugw_utils.cu:115); the partial results of all ranks sum to the full Sigma.
    """
    Gf = g_full(sys_)
    Sigma = np.zeros((sys_.nts, sys_.ns, sys_.ink, sys_.nao, sys_.nao), np.complex128)
    if keep is not None:
        keep["P0"], keep["Pw"], keep["Wt"] = [], [], []
    for iq in (range(sys_.inq) if q_subset is None else q_subset):
        q_ir = sys_.q_reduced_to_full[iq]
        P0 = scale_mirror(p0_q(sys_, Gf, q_ir), sys_.nk, sys_.nts)
        Pw = transform_tw(P0, sys_.Tnt_BF)
        Ww = dyson(Pw, solver)
        Wt = transform_wt(Ww, sys_.Ttn_FB)
        if keep is not None:
            keep["P0"].append(P0)
            keep["Pw"].append(Pw)
            keep["Wt"].append(Wt)
        for kr in range(sys_.ink):
            k = sys_.k_reduced_to_full[kr]
            for q_deg in sys_.q_stars[iq]:
                k1 = sys_.k2_from_k1q[k * sys_.nq + q_deg]
                V = coulomb(sys_, k, k1)
                Wq = rotate_w(sys_, Wt, q_deg)
                for s in range(sys_.ns):
                    Sigma[:, s, kr] += sigma_pair(V, Gf[k1, s], Wq)
    return Sigma / sys_.nk
