"""Imaginary-time / Matsubara transformation matrices for the GW path.

The reference receives two dense matrices from green-grids' ``transformer_t``
(``Ttn_FB`` and ``Tnt_BF``, consumed at ``src/cugw_qpt.cu:329-358`` through
``src/cuda_common.cu:93-108``).  green-grids reads them from an IR basis file
(``ir/1e4.h5``) that is not part of the reference, so this module builds an
equivalent pair from first principles:

* the logistic kernel ``K(tau, w) = exp(-tau w) / (1 + exp(-beta w))`` on
  ``tau in [0, beta]``, ``w in [-wmax, wmax]`` with ``Lambda = beta * wmax``
  is discretised with composite Gauss-Legendre rules refined geometrically
  towards ``tau = 0, beta`` and ``w = 0`` (bosonic functions are logistic
  transforms of ``rho_B(w) coth(beta w / 2)``, so the same singular functions
  span them);
* its weighted SVD gives singular functions ``u_l(tau)``; their exact
  bosonic Matsubara transforms follow from ``int_0^beta exp(i W_n tau)
  K(tau, w) dtau = tanh(beta w / 2) / (w - i W_n)``;
* the sampling times are the ``nts - 2`` interior roots of ``u_{nts-2}``
  (mirrored so that ``tau_i = beta - tau_{nts-1-i}``) plus the two end points,
  and the bosonic frequencies form a set symmetric under ``n -> -n`` whose
  positive members are chosen by a column-pivoted QR (so the transforms commute
  with complex conjugation, which time-reversal symmetry relies on).

``Tnt_BF`` (``nw_b x (nts-2)``) fits a function sampled on the interior times
and evaluates it on the bosonic frequencies; ``Ttn_FB`` (``nts x nw_b``)
maps frequency samples back to all ``nts`` times.  Both are complex128,
row-major, exactly the shapes and meaning the reference uses.
"""
from __future__ import annotations

import numpy as np


def _composite_gauss(edges, order):
    x, w = np.polynomial.legendre.leggauss(order)
    xs, ws = [], []
    for a, b in zip(edges[:-1], edges[1:]):
        xs.append(0.5 * (b - a) * x + 0.5 * (b + a))
        ws.append(0.5 * (b - a) * w)
    return np.concatenate(xs), np.concatenate(ws)


def _geometric_edges(lo, hi, smallest, toward_lo=True, toward_hi=True):
    """Panel edges on [lo, hi] refined geometrically towards the chosen ends."""
    mid = 0.5 * (lo + hi)
    half = 0.5 * (hi - lo)
    n = max(1, int(np.ceil(np.log2(half / smallest))))
    g = half * 0.5 ** np.arange(n + 1)  # half, half/2, ..., ~smallest
    left = lo + g[::-1] if toward_lo else np.linspace(lo, mid, 4)
    right = hi - g if toward_hi else np.linspace(mid, hi, 4)
    edges = np.unique(np.concatenate([[lo], left, [mid], right, [hi]]))
    return edges


def _kernel_tau(tau, w, beta):
    """Logistic kernel K(tau, w) = e^{-tau w} / (1 + e^{-beta w}), overflow-free."""
    tau = np.asarray(tau, dtype=np.float64)[:, None]
    w = np.asarray(w, dtype=np.float64)[None, :]
    pos = w >= 0
    wp = np.where(pos, w, 0.0)
    wn = np.where(pos, 0.0, w)
    kp = np.exp(-tau * wp) / (1.0 + np.exp(-beta * wp))
    kn = np.exp((beta - tau) * wn) / (1.0 + np.exp(beta * wn))
    return np.where(pos, kp, kn)


def _kernel_iw(n, w, beta):
    """Bosonic Matsubara transform of K: tanh(beta w / 2) / (w - i W_n), W_n = 2 pi n / beta."""
    Wn = 2.0 * np.pi * np.asarray(n, dtype=np.float64)[:, None] / beta
    w = np.asarray(w, dtype=np.float64)[None, :]
    den = w - 1j * Wn
    zero = (den == 0)
    return np.where(zero, 0.5 * beta + 0j, np.tanh(0.5 * beta * w) / np.where(zero, 1.0, den))


class IRBasis:
    """Bosonic singular-value basis and the two transformation matrices.

    Parameters
    ----------
    beta : inverse temperature (Ha^-1)
    lam : dimensionless cutoff Lambda = beta * wmax
    nts : number of imaginary-time points including tau = 0 and tau = beta
    nw_b : number of bosonic Matsubara frequencies (nw_b <= nts - 2)
    """

    def __init__(self, beta: float = 100.0, lam: float = 1e4, nts: int = 72, nw_b: int = 69,
                 order: int = 24, tau=None):
        """``tau`` (optional): a given grid of nts points, 0 and beta included and symmetric
        under tau -> beta - tau (for example the sampling points of an IR basis file, which
        come from an extended-precision expansion beyond the reach of this double-precision
        SVD); the transforms are then built on it instead of on roots of u_{nts-2}."""
        if tau is not None:
            tau = np.asarray(tau, dtype=np.float64)
            nts = len(tau)
            if tau[0] != 0.0 or tau[-1] != beta or np.any(np.diff(tau) <= 0):
                raise ValueError("tau must rise from 0 to beta")
            if np.abs(tau + tau[::-1] - beta).max() > 1e-6 * beta:
                raise ValueError("tau must be symmetric under tau -> beta - tau")
        if nts % 2:
            raise ValueError("nts must be even (tau grid symmetric about beta/2)")
        if nw_b > nts - 2:
            raise ValueError("need nw_b <= nts - 2")
        if nw_b % 2 == 0:
            raise ValueError("nw_b must be odd: n = 0 plus (nw_b - 1) / 2 pairs +-n")
        self.beta = float(beta)
        self.lam = float(lam)
        self.nts = int(nts)
        self.nw_b = int(nw_b)
        wmax = lam / beta
        t_edges = _geometric_edges(0.0, beta, smallest=0.05 / wmax)
        # refine w towards 0 (scale 1/beta)
        half = wmax
        n = int(np.ceil(np.log2(half * beta / 0.05)))
        g = half * 0.5 ** np.arange(n + 1)
        w_edges = np.unique(np.concatenate([-g, [0.0], g[::-1]]))
        tx, tw = _composite_gauss(t_edges, order)
        wx, ww = _composite_gauss(w_edges, order)
        K = _kernel_tau(tx, wx, beta)
        M = np.sqrt(tw)[:, None] * K * np.sqrt(ww)[None, :]
        U, s, Vt = np.linalg.svd(M, full_matrices=False)
        self._wx, self._ww = wx, ww
        self._tx, self._tw = tx, tw
        self._s = s
        self._V = Vt.T
        L = nts - 2
        self.L = L
        if tau is not None:
            self.tau = tau.copy()
            self._finish(tau[1:-1], nw_b, lam)
            return
        # sampling times: interior roots of u_L (the (L+1)-th singular function)
        dense = np.unique(np.concatenate([np.linspace(0, beta / 2, 20001)[1:],
                                          np.geomspace(1e-7 * beta, beta / 2, 20001)]))
        uL = self.u(dense, [L])[:, 0]
        sgn = np.sign(uL)
        idx = np.nonzero(sgn[:-1] * sgn[1:] < 0)[0]
        roots = []
        for i in idx:
            a, b = dense[i], dense[i + 1]
            fa = uL[i]
            for _ in range(60):
                m = 0.5 * (a + b)
                fm = self.u(np.array([m]), [L])[0, 0]
                if np.sign(fm) == np.sign(fa):
                    a, fa = m, fm
                else:
                    b = m
            roots.append(0.5 * (a + b))
        roots = np.array(sorted(roots))
        need = L // 2
        if len(roots) < need:
            raise RuntimeError(f"found {len(roots)} roots in (0, beta/2), need {need}")
        # keep the `need` roots closest to the ends are all of them when counts match
        roots = roots[:need] if len(roots) == need else roots[np.linspace(0, len(roots) - 1, need).round().astype(int)]
        interior = np.concatenate([roots, beta - roots[::-1]])
        self.tau = np.concatenate([[0.0], interior, [beta]])
        self._finish(interior, nw_b, lam)

    def _finish(self, interior, nw_b, lam):
        # bosonic frequencies: a set symmetric under n -> -n (n = 0 included when nw_b is
        # odd), so that the transform pair commutes with complex conjugation exactly as
        # the physical Fourier transform of a tau-symmetric function does.  Pairs are
        # picked by column-pivoted QR on the even part of the basis.
        import scipy.linalg as sla
        nmax = int(max(4 * nw_b, 2 * lam))
        cand = np.unique(np.concatenate([np.arange(1, 64), np.unique(np.geomspace(1, nmax, 4000).astype(int))]))
        npair = nw_b // 2
        basis = range(nw_b)
        even = [l for l in basis if l % 2 == 0]
        Ue = self.uhat(cand, even)
        # remove the n = 0 row's direction before choosing pairs
        u0 = self.uhat(np.array([0]), even)[0]
        u0 = u0 / np.linalg.norm(u0)
        Ue = Ue - np.outer(Ue @ u0.conj(), u0)
        _, _, piv = sla.qr(Ue.T, pivoting=True, mode="economic")
        pos_n = np.sort(cand[piv[:npair]])
        wn = np.concatenate([-pos_n[::-1], [0], pos_n]).astype(np.int64)
        self.wn = wn
        # transformation matrices
        U_int = self.u(interior, range(nw_b))          # (nts-2) x nw_b
        U_all = self.u(self.tau, range(nw_b))          # nts x nw_b
        Uh_w = self.uhat(self.wn, range(nw_b))         # nw_b x nw_b
        # fit: coefficients c = pinv(U_int) f(tau_int); evaluate: f(iW) = Uh_w c
        self.Tnt_BF = (Uh_w @ np.linalg.pinv(U_int)).astype(np.complex128)      # nw_b x (nts-2)
        self.Ttn_FB = (U_all @ np.linalg.inv(Uh_w)).astype(np.complex128)       # nts x nw_b
        self.cond_fit = np.linalg.cond(U_int)
        self.cond_freq = np.linalg.cond(Uh_w)

    def u(self, tau, ls):
        ls = list(ls)
        K = _kernel_tau(np.asarray(tau, dtype=np.float64), self._wx, self.beta)
        return (K * np.sqrt(self._ww)[None, :]) @ self._V[:, ls] / self._s[ls][None, :]

    def uhat(self, n, ls):
        ls = list(ls)
        K = _kernel_iw(np.asarray(n), self._wx, self.beta)
        return (K * np.sqrt(self._ww)[None, :]) @ self._V[:, ls] / self._s[ls][None, :]


def tau_quadrature(tau, beta: float = 100.0, lam: float = 1e4, nl=None, cutoff: float = 1e-13):
    """Real matrix M [nts][nts] with int_0^beta f(tau) g(beta - tau) dtau = f^T M g for functions
    f, g sampled on the grid `tau` (0 and beta included) and spanned by the first nl singular
    functions u_l of the logistic kernel: M = Fit^T O Fit with Fit the least-squares fit of
    the coefficients from the samples and O_ll' = int u_l(tau) u_l'(beta - tau) dtau (computed
    on the kernel's own quadrature; (-1)^l delta_ll' for the exact functions).  By default nl
    keeps the functions with s_l / s_0 > cutoff, at most nts - 2."""
    tau = np.asarray(tau, dtype=np.float64)
    nts = len(tau)
    b = IRBasis(beta, lam, nts, 1, tau=tau)
    if nl is None:
        nl = int(min(nts - 2, np.count_nonzero(b._s / b._s[0] > cutoff)))
    ls = range(nl)
    U = b.u(tau, ls)
    fit = np.linalg.pinv(U)
    uq = b.u(b._tx, ls)
    ur = b.u(beta - b._tx, ls)
    O = (uq * b._tw[:, None]).T @ ur
    return fit.T @ O @ fit


_CACHE: dict = {}


def ir_matrices_on_grid(tau, beta: float = 100.0, lam: float = 1e4, nw_b: int = 81):
    """(Ttn_FB, Tnt_BF) on a given tau grid (0 and beta included, symmetric), nw_b bosonic
    basis functions fitted on its interior points."""
    b = IRBasis(beta, lam, len(tau), nw_b, tau=tau)
    return b.Ttn_FB.copy(), b.Tnt_BF.copy()


def ir_matrices(beta: float = 100.0, lam: float = 1e4, nts: int = 72, nw_b: int = 69):
    """Return (tau, Ttn_FB, Tnt_BF) for the given grid, memoised per process."""
    key = (float(beta), float(lam), int(nts), int(nw_b))
    if key not in _CACHE:
        b = IRBasis(beta, lam, nts, nw_b)
        _CACHE[key] = (b.tau.copy(), b.Ttn_FB.copy(), b.Tnt_BF.copy())
    return _CACHE[key]
