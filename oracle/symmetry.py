"""Oracle: k-pair integral lookup and k-point symmetry unfolding (test infrastructure only)."""
import numpy as np


def tri(k1, k2):
    """Triangular k-pair index (src/green/gpu/df_integral_t.h:68-70)."""
    return k1 * (k1 + 1) // 2 + k2 if k1 >= k2 else k2 * (k2 + 1) // 2 + k1


def coulomb(sys_, k1, k2):
    """V^Q(k1,k2) [NQ][nao][nao] as df_integral_t::symmetrize builds it.

    Follows src/green/gpu/df_integral_t.h:153-173 (symmetry type) and :211-235
    (conjugate-transpose when k1 < k2, then conj or transpose).
    """
    idx = tri(k1, k2)
    sign = 1 if k1 >= k2 else -1
    kind = "direct"
    if sys_.conj_kpair_list[idx] != idx:
        kind = "conjugated"
        idx = sys_.conj_kpair_list[idx]
    elif sys_.trans_kpair_list[idx] != idx:
        kind = "transposed"
        idx = sys_.trans_kpair_list[idx]
    pos = sys_.irre_pos_kpair[idx]
    V = np.array(sys_.V_stored[pos], dtype=np.complex128)
    if sign < 0:
        V = np.conj(np.swapaxes(V, 1, 2))
    if kind == "conjugated":
        V = np.conj(V)
    elif kind == "transposed":
        V = np.swapaxes(V, 1, 2)
    return np.ascontiguousarray(V)


def unfold_ao(sys_, X_ibz, k_full):
    """X(k_full) = U_k X(k_ibz) U_k^+, conjugated for time-reversal partners.

    src/cu_symmetry.cu:183-233 (transform_k_ao_device); X_ibz has the IBZ index
    in its third-from-last axis.
    """
    k_ibz = sys_.k_full_to_reduced[k_full]
    X = X_ibz[..., k_ibz, :, :]
    if sys_.U_k is not None:
        U = sys_.U_k[k_full]
        X = U @ X @ U.conj().T
    if sys_.k_tr_conj[k_full]:
        X = np.conj(X)
    return X


def ibz_to_full(sys_, X_ibz):
    """[..., ink, n, n] -> [..., nk, n, n] (hf_gpu_kernel.cpp:203-209 via value_AO)."""
    return np.stack([unfold_ao(sys_, X_ibz, k) for k in range(sys_.nk)], axis=-3)
