"""Oracle: FP64 energy and chemical-potential reductions (test infrastructure only).

green-gpu's kernels return Sigma(tau) and the Fock matrix; the energies and the chemical
potential are reduced from them by its caller (green-mbpt) in FP64.  These are plain numpy
statements of the definitions the library's reductions implement:

* k weights: w_k = |star(k)| / nk over the irreducible k points (the IBZ sums of
  src/gw_gpu_kernel.cpp:34-91's symmetry tables); spin factor f = 2 for ns = 1 (closed
  shell, matrices per spin), 1 for ns = 2 and for two-component matrices;
* E_1b = f sum_{s,k} w_k Re Tr(D_s(k) H_s(k)),  E_HF = (f / 2) sum_{s,k} w_k Re Tr(D_s(k) (H_s(k) + F_s(k)));
* E_GW = -(f / 2) sum_{s,k} w_k int_0^beta Re Tr(Sigma_s(k, tau) G_s(k, beta - tau)) dtau
  (Galitskii-Migdal form), with the integral as the bilinear quadrature
  sum_{t,t'} M[t][t'] Re Tr(Sigma(tau_t) G(tau_t')) that the caller supplies;
* mu: the root of N(mu) = f sum_{s,k} w_k sum_n 1 / (1 + exp(beta (e_skn - mu))) - n_elec, with
  e_skn the eigenvalues of F_s(k) x = e S_s(k) x.
"""
import numpy as np
import scipy.linalg as sla


def kweights(sys_):
    return np.array([len(st) for st in sys_.k_stars], np.float64) / sys_.nk


def spin_factor(ns, x2c=False):
    return 2.0 if (ns == 1 and not x2c) else 1.0


def _tr(A, B):
    """Re Tr(A B) for every leading index: [..., n, n] x [..., n, n] -> [...]."""
    return np.einsum("...ij,...ji->...", A, B).real


def e_hf(sys_, dm, H, F, x2c=False):
    f = spin_factor(sys_.ns, x2c)
    w = kweights(sys_)
    e1 = f * float((w[None, :] * _tr(dm, H)).sum())
    ehf = 0.5 * f * float((w[None, :] * _tr(dm, H + F)).sum())
    return e1, ehf


def e_gw(sys_, G, Sigma, M, x2c=False):
    """G, Sigma [nts][ns][ink][n][n]; M [nts][nts] real."""
    f = spin_factor(sys_.ns, x2c)
    w = kweights(sys_)
    C = np.einsum("tskij,uskji->sktu", Sigma, G).real  # Re Tr(Sigma(t) G(t'))
    return -0.5 * f * float(np.einsum("k,sktu,tu->", w, C, M))


def eigenvalues(F, S):
    ns, ink = F.shape[:2]
    return np.array([[sla.eigh(F[s, k], S[s, k], eigvals_only=True) for k in range(ink)] for s in range(ns)])


def particle_number(eps, w, mu, beta, f):
    x = beta * (eps - mu)
    occ = np.where(x > 0, np.exp(-np.abs(x)) / (1.0 + np.exp(-np.abs(x))), 1.0 / (1.0 + np.exp(-np.abs(x))))
    return f * float((w[None, :, None] * occ).sum())


def chemical_potential(sys_, F, S, beta, nelec, x2c=False):
    """Bisection to FP64 resolution on the mean-field particle number."""
    eps = eigenvalues(F, S)
    w = kweights(sys_)
    f = spin_factor(sys_.ns, x2c)
    lo, hi = eps.min() - 50.0 / beta, eps.max() + 50.0 / beta
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid <= lo or mid >= hi:
            break
        if particle_number(eps, w, mid, beta, f) < nelec:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)
