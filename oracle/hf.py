"""Oracle: one HF Fock build (exchange + direct + Ewald) in FP64 numpy (test infrastructure only).

Restates src/cuhf_utils.cu:108-159 (exchange), src/hf_gpu_kernel.cpp:141-186
(direct), :188-201 (Ewald), :203-209 (density unfolding) and :66-104 (solve).
"""
import numpy as np

from .symmetry import coulomb, ibz_to_full, unfold_ao


def exchange(sys_, dm):
    """K_s(k) = pref/nk sum_k2 sum_Q V^Q(k,k2) D_s(k2) V^Q(k,k2)^+ for every IBZ k.

    src/cuhf_utils.cu:108-134: X = V^Q D (GEMM at :118), Y(k2) = sum_{Q,a} X_{ja}
    conj(V^Q_{ia}) (:127), F += pref * (1/nk) * sum_k2 Y (:131); pref = -0.5 (ns=1) or -1.
    """
    ns, nk, ink = sys_.ns, sys_.nk, sys_.ink
    pref = -0.5 if ns == 1 else -1.0
    D = ibz_to_full(sys_, dm)  # [ns][nk][n][n]
    F = np.zeros((ns, ink, sys_.nao, sys_.nao), np.complex128)
    for kr in range(ink):
        k = sys_.k_reduced_to_full[kr]
        for k2 in range(nk):
            V = coulomb(sys_, k, k2)
            for s in range(ns):
                X = V @ D[s, k2]
                F[s, kr] += pref / nk * np.einsum("Qja,Qia->ji", X, np.conj(V), optimize=True)
    return F


def direct(sys_, dm):
    """Hartree term (src/hf_gpu_kernel.cpp:141-186).

    c_Q = (1/nk) sum_{s,k'} sum_{ab} V^Q(k',k')_{ab} D_s(k')_{ba};
    F_s(k) += sum_Q c_Q V^Q(k,k) for every IBZ k (k taken at its full-BZ representative).
    """
    ns, nk = sys_.ns, sys_.nk
    c = np.zeros(sys_.NQ, np.complex128)
    for kp in range(nk):
        V = coulomb(sys_, kp, kp)
        for s in range(ns):
            Dk = unfold_ao(sys_, dm[s], kp)
            c += np.einsum("Qab,ba->Q", V, Dk)
    c /= nk
    F = np.zeros((ns, sys_.ink, sys_.nao, sys_.nao), np.complex128)
    for kr in range(sys_.ink):
        k = sys_.k_reduced_to_full[kr]
        V = coulomb(sys_, k, k)
        J = np.tensordot(c, V, axes=(0, 0))
        for s in range(ns):
            F[s, kr] += J
    return F


def ewald(sys_, dm):
    """-c * madelung * S D S per (s, IBZ k), c = 0.5 (ns=1) or 1 (src/hf_gpu_kernel.cpp:188-201)."""
    c = 1.0 if sys_.ns == 2 else 0.5
    S = sys_.S_k
    return -c * sys_.madelung * (S @ dm @ S)


def hf_build(sys_, dm=None):
    """Returned Fock of hf_gpu_kernel::solve: exchange + direct + Ewald (hf_gpu_kernel.cpp:66-104)."""
    if dm is None:
        dm = sys_.dm
    return exchange(sys_, dm) + direct(sys_, dm) + ewald(sys_, dm)
