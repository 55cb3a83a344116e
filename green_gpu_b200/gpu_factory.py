"""Host-side mirror of the reference's plugin surface (src/green/gpu/gpu_factory.h).

green-mbpt obtains its GPU kernels through three factory functions; this module keeps
their names, argument order and meaning, and forwards the work to libgreen_b200.so:

* ``custom_kernel_parameters(p)``  - gpu_factory.h:95-102 (same parameter names/defaults)
* ``custom_hf_kernel(X2C, p, nao, nso, ns, NQ, madelung, bz_utils, S_k)`` -> (kernel, callback)
  with ``callback(dm) -> F``, F = exchange + direct + Ewald (hf_gpu_kernel.cpp:66-104)
* ``custom_gw_kernel(X2C, p, nao, nso, ns, NQ, ft, bz_utils, S_k)`` -> (kernel, callback)
  with ``callback(g, sigma)`` overwriting sigma with Sigma(tau) (gw_gpu_kernel.cpp:163-205)

Differences forced by the environment, kept explicit:
* ``bz_utils`` is any object exposing the symmetry tables of green-symmetry's
  brillouin_zone_utils used by the reference (k/q full<->reduced maps, TR flags, k+-q maps,
  AO / auxiliary rotations, k-pair lists) - e.g. :class:`green_gpu_b200.synth.System`;
* the integrals are passed in memory (``p["dfintegral"]`` / ``p["dfintegral_hf"]``: the
  stored k-pair array [num_kpair_stored][NQ][nao][nao]) or read from the reference's HDF5
  chunk files (``p["dfintegral_file"]`` / ``p["dfintegral_hf_file"]``, see df_integral.py);
* ``ft`` is any object with ``Ttn_FB`` [nts][nw_b] and ``Tnt_BF`` [nw_b][nts-2].
X2C (two-component) kernels (``X2C=True``, nso = 2 nao, ns = 1) run the C ABI's X2C mode
(gg_set_x2c): the spin blocks as pseudo-spins, identity k/q symmetry only.
"""
from __future__ import annotations

import numpy as np

from . import native

LinearSolverType = {"Cholesky": native.SOLVER_CHOLESKY, "LU": native.SOLVER_LU}


def custom_kernel_parameters(p: dict) -> None:
    """Register the GPU-kernel parameters with the reference's names and defaults."""
    p.setdefault("verbose", 0)
    p.setdefault("cuda_linear_solver", "LU")
    p.setdefault("cuda_low_gpu_memory", False)
    p.setdefault("cuda_low_cpu_memory", False)
    p.setdefault("nt_batch", 0)
    # B200-specific: split-precision contractions (replaces P_sp / Sigma_sp single precision)
    p.setdefault("P_sp", False)
    p.setdefault("Sigma_sp", False)
    p.setdefault("split_slices", native.DEFAULT_SPLIT_SLICES)


def _coulomb(p, key_mem, key_file, bz_utils, nao, NQ):
    if p.get(key_mem) is not None:
        return np.ascontiguousarray(p[key_mem], dtype=np.complex128)
    if p.get(key_file):
        from .df_integral import read_stored
        return read_stored(p[key_file], nao, NQ)
    V = getattr(bz_utils, "V_stored", None)
    if V is None:
        raise ValueError(f"no integrals: set p['{key_mem}'] or p['{key_file}']")
    return V


def _context(p, nao, ns, NQ, bz_utils, nts=4, nw_b=0, V=None, device=0):
    ctx = native.Context(bz_utils.nk, bz_utils.ink, bz_utils.inq, nao, NQ, ns, nts, nw_b, device)
    ctx.set_symmetry(bz_utils.k_full_to_reduced, bz_utils.k_reduced_to_full, bz_utils.k_tr_conj,
                     bz_utils.q_full_to_reduced, bz_utils.q_reduced_to_full, bz_utils.q_tr_conj,
                     bz_utils.k1_from_k2q, bz_utils.k2_from_k1q,
                     getattr(bz_utils, "U_k", None), getattr(bz_utils, "U_q", None))
    ctx.set_kpairs(V.shape[0], bz_utils.conj_kpair_list, bz_utils.trans_kpair_list, bz_utils.irre_pos_kpair)
    ctx.set_coulomb(V)
    return ctx


class scalar_hf_gpu_kernel:
    """hf_gpu_kernel / scalar_hf_gpu_kernel (src/green/gpu/hf_gpu_kernel.h:41-100)."""

    def __init__(self, p, nao, nso, ns, NQ, madelung, bz_utils, S_k, verbose=1):
        self._p = p
        self._ns = ns
        self._madelung = float(madelung)
        self._S_k = np.ascontiguousarray(S_k, dtype=np.complex128)
        V = _coulomb(p, "dfintegral_hf", "dfintegral_hf_file", bz_utils, nao, NQ)
        self._ctx = _context(p, nao, ns, NQ, bz_utils, V=V)

    def solve(self, dm):
        """Return F = K + J - Ewald for the IBZ density dm [ns][ink][nso][nso]."""
        return self._ctx.hf_fock(dm, self._S_k, self._madelung)


class x2c_hf_gpu_kernel(scalar_hf_gpu_kernel):
    """x2c_hf_gpu_kernel (src/green/gpu/hf_gpu_kernel.h:68-100): spinor dm / Fock [1][ink][nso][nso]."""

    def __init__(self, p, nao, nso, ns, NQ, madelung, bz_utils, S_k, verbose=1):
        if nso != 2 * nao or ns != 1:
            raise ValueError("x2c: nso = 2 nao and ns = 1")
        super().__init__(p, nao, nso, ns, NQ, madelung, bz_utils, S_k, verbose)
        self._ctx.set_x2c(True)


class scalar_gw_gpu_kernel:
    """gw_gpu_kernel / scalar_gw_gpu_kernel (src/green/gpu/gw_gpu_kernel.h:40-206)."""

    def __init__(self, p, nao, nso, ns, NQ, ft, bz_utils, cuda_lin_solver="LU", verbose=1):
        nts = int(np.asarray(ft.Ttn_FB).shape[0])
        nw_b = int(np.asarray(ft.Ttn_FB).shape[1])
        if nts % 2:
            # gw_gpu_kernel.h:67
            raise RuntimeError("Number of tau points should be even number")
        self._solver = LinearSolverType[cuda_lin_solver] if isinstance(cuda_lin_solver, str) else int(cuda_lin_solver)
        sp = bool(p.get("P_sp", False)) and bool(p.get("Sigma_sp", False))
        self._precision = native.PREC_SPLIT if sp else native.PREC_FP64
        V = _coulomb(p, "dfintegral", "dfintegral_file", bz_utils, nao, NQ)
        self._ctx = _context(p, nao, ns, NQ, bz_utils, nts=nts, nw_b=nw_b, V=V)
        self._ctx.set_ir(ft.Ttn_FB, ft.Tnt_BF)
        self._ctx.set_split_slices(int(p.get("split_slices", native.DEFAULT_SPLIT_SLICES)))

    def solve(self, g, sigma):
        """Overwrite sigma [nts][ns][ink][nso][nso] with Sigma(tau) for G(tau) g."""
        out = self._ctx.gw_sigma(g, solver=self._solver, precision=self._precision)
        sigma[...] = out


class x2c_gw_gpu_kernel(scalar_gw_gpu_kernel):
    """x2c_gw_gpu_kernel (src/green/gpu/gw_gpu_kernel.h:131-206): spinor G / Sigma [nts][1][ink][nso][nso]."""

    def __init__(self, p, nao, nso, ns, NQ, ft, bz_utils, cuda_lin_solver="LU", verbose=1):
        if nso != 2 * nao or ns != 1:
            raise ValueError("x2c: nso = 2 nao and ns = 1")
        super().__init__(p, nao, nso, ns, NQ, ft, bz_utils, cuda_lin_solver, verbose)
        self._ctx.set_x2c(True)


def custom_hf_kernel(X2C, p, nao, nso, ns, NQ, madelung, bz_utils, S_k):
    cls = x2c_hf_gpu_kernel if X2C else scalar_hf_gpu_kernel
    kernel = cls(p, nao, nso, ns, NQ, madelung, bz_utils, S_k)
    return kernel, kernel.solve


def custom_gw_kernel(X2C, p, nao, nso, ns, NQ, ft, bz_utils, S_k):
    cls = x2c_gw_gpu_kernel if X2C else scalar_gw_gpu_kernel
    kernel = cls(p, nao, nso, ns, NQ, ft, bz_utils, p.get("cuda_linear_solver", "LU"), p.get("verbose", 0))
    return kernel, kernel.solve
