"""Oracle: two-component (X2C) HF and GW in FP64 numpy (test infrastructure only).

Restates the reference's X2C kernels, which reuse the scalar contractions on spin blocks:
* HF (src/hf_gpu_kernel.cpp:229-338): the density is cut into the aa, bb, ab blocks
  (get_dm_fbz, :326-336) and the exchange runs with pseudo-spin 3 (prefactor -1,
  src/cuhf_utils.cu:111); the Fock matrix is reassembled with ba = ab^+
  (copy_2c_Fock_from_device_to_host, src/cuda_common.cu:176-201).  The Hartree term uses the
  density of aa + bb and is added to the aa and bb blocks (:262-309); Ewald subtracts
  madelung * S_aa D_block S_aa per block, the ba block getting the adjoint of the ab term
  (:311-323).
* GW (src/gw_gpu_kernel.cpp:457-551): G is cut into the aa, bb, ab, ba blocks (copy_Gk_2c,
  minus_t = false) and the scalar contractions run with pseudo-spin 4 (P0 prefactor -1,
  src/cugw_qkpt.cu:206); for G(-tau) the blocks are taken transposed in spin (minus_t = true:
  pseudo-spin ab pairs with the ba block), Sigma is computed per block and reassembled
  (copy_Sigma_2c, src/cugw_qkpt.cu:382-403).
Only the identity k/q symmetry is restated: the spinor form of a space-group or time-reversal
operation lives in green-symmetry, which is not part of the reference tree.
"""
import numpy as np

from .gw import dyson, p0_pair, scale_mirror, sigma_pair, transform_tw, transform_wt
from .symmetry import coulomb

# (row block, column block) of each pseudo-spin: aa, bb, ab, ba
BLOCKS = ((0, 0), (1, 1), (0, 1), (1, 0))
# pseudo-spin of the G(-tau) operand paired with pseudo-spin s of G(tau) (blocks transposed)
PERM_MINUS_T = (0, 1, 3, 2)


def split(M, nblk):
    """[..., 2n, 2n] -> [..., nblk, n, n] with the blocks of BLOCKS[:nblk]."""
    n = M.shape[-1] // 2
    return np.stack([M[..., a * n:(a + 1) * n, b * n:(b + 1) * n] for a, b in BLOCKS[:nblk]], axis=-3)


def merge(X, adjoint_ba=False):
    """[..., nblk, n, n] -> [..., 2n, 2n]; with 3 blocks (or adjoint_ba) ba = ab^+."""
    nblk, n = X.shape[-3], X.shape[-1]
    out = np.zeros(X.shape[:-3] + (2 * n, 2 * n), np.complex128)
    for s, (a, b) in enumerate(BLOCKS[:nblk]):
        out[..., a * n:(a + 1) * n, b * n:(b + 1) * n] = X[..., s, :, :]
    if nblk == 3 or adjoint_ba:
        out[..., n:, :n] = np.conj(np.swapaxes(X[..., 2, :, :], -1, -2))
    return out


def _check_identity(sys_):
    if sys_.U_k is not None or sys_.U_q is not None or np.any(sys_.k_tr_conj) or np.any(sys_.q_tr_conj):
        raise ValueError("x2c oracle: only the identity k/q symmetry")


def hf_build(sys_, dm):
    """Fock [1][ink][2n][2n] of x2c_hf_gpu_kernel::solve (exchange + direct + Ewald)."""
    _check_identity(sys_)
    nk, ink, n = sys_.nk, sys_.ink, sys_.nao
    D = split(dm[0], 3)  # [ink][3][n][n]; identity symmetry: full BZ k = k_reduced_to_full
    Dfull = np.zeros((nk, 3, n, n), np.complex128)
    for kr in range(ink):
        Dfull[sys_.k_reduced_to_full[kr]] = D[kr]
    K = np.zeros((ink, 3, n, n), np.complex128)
    for kr in range(ink):
        k = sys_.k_reduced_to_full[kr]
        for k2 in range(nk):
            V = coulomb(sys_, k, k2)
            for s in range(3):
                X = V @ Dfull[k2, s]
                K[kr, s] += -1.0 / nk * np.einsum("Qja,Qia->ji", X, np.conj(V), optimize=True)
    F = merge(K)  # [ink][2n][2n]
    # Hartree term from the aa + bb density
    c = np.zeros(sys_.NQ, np.complex128)
    for kp in range(nk):
        V = coulomb(sys_, kp, kp)
        c += np.einsum("Qab,ba->Q", V, Dfull[kp, 0] + Dfull[kp, 1])
    c /= nk
    for kr in range(ink):
        k = sys_.k_reduced_to_full[kr]
        J = np.tensordot(c, coulomb(sys_, k, k), axes=(0, 0))
        F[kr, :n, :n] += J
        F[kr, n:, n:] += J
    # Ewald per block with the AO overlap S_aa
    for kr in range(ink):
        Saa = sys_.S_k[0, kr, :n, :n]
        for a, b in BLOCKS[:3]:
            E = sys_.madelung * Saa @ dm[0, kr, a * n:(a + 1) * n, b * n:(b + 1) * n] @ Saa
            F[kr, a * n:(a + 1) * n, b * n:(b + 1) * n] -= E
            if a != b:
                F[kr, n:, :n] -= np.conj(E.T)
    return F[None]


def gw_build(sys_, G2c, solver="cholesky"):
    """Sigma [nts][1][ink][2n][2n] of x2c_gw_gpu_kernel::compute_2c_gw_selfenergy (already / nk)."""
    _check_identity(sys_)
    nk, ink, nts, n = sys_.nk, sys_.ink, sys_.nts, sys_.nao
    G4 = split(G2c[:, 0], 4)  # [nts][ink][4][n][n]
    Gf = np.zeros((nk, 4, nts, n, n), np.complex128)
    for kr in range(ink):
        Gf[sys_.k_reduced_to_full[kr]] = np.moveaxis(G4[:, kr], 0, 1)
    nt2 = nts // 2
    tt = np.arange(nt2)
    Sigma4 = np.zeros((nts, ink, 4, n, n), np.complex128)
    for iq in range(sys_.inq):
        q = sys_.q_reduced_to_full[iq]
        P0h = np.zeros((nt2, sys_.NQ, sys_.NQ), np.complex128)
        for k in range(nk):
            k1 = sys_.k1_from_k2q[k * sys_.nq + q]
            V = coulomb(sys_, k, k1)
            for s in range(4):
                P0h += p0_pair(V, Gf[k1, s, tt], Gf[k, PERM_MINUS_T[s], nts - 1 - tt], -1.0)
        P0 = scale_mirror(P0h, nk, nts)
        Wt = transform_wt(dyson(transform_tw(P0, sys_.Tnt_BF), solver), sys_.Ttn_FB)
        for kr in range(ink):
            k = sys_.k_reduced_to_full[kr]
            for qd in sys_.q_stars[iq]:
                k1 = sys_.k2_from_k1q[k * sys_.nq + qd]
                V = coulomb(sys_, k, k1)
                for s in range(4):
                    Sigma4[:, kr, s] += sigma_pair(V, Gf[k1, s], Wt)
    return merge(Sigma4 / nk)[:, None]
