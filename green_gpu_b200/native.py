"""ctypes binding of libgreen_b200.so (the C ABI declared in include/green_b200.h).

There is no fallback: if the library is missing or CUDA is unavailable, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libgreen_b200.so")

GG_OK = 0
GG_ERR_ARG = 1
GG_ERR_CUDA = 2
GG_ERR_NOT_HPD = 3
GG_ERR_SINGULAR = 4
GG_ERR_STATE = 5
GG_ERR_MEMORY = 6
GG_ERR_INTERNAL = 7

SOLVER_CHOLESKY = 0
SOLVER_LU = 1
PREC_FP64 = 0
PREC_SPLIT = 1
# slice count of GG_PREC_SPLIT unless set (GG_DEFAULT_SPLIT_SLICES in include/green_b200.h)
DEFAULT_SPLIT_SLICES = 5

EXPORTS = [
    "gg_create", "gg_destroy", "gg_last_error", "gg_set_symmetry", "gg_set_kpairs", "gg_set_coulomb",
    "gg_set_coulomb_device", "gg_set_ir", "gg_set_split_slices", "gg_gw_sigma", "gg_gw_sigma_device",
    "gg_set_capture", "gg_hf_exchange", "gg_hf_fock", "gg_symmetry_unfold", "gg_last_timings", "gg_version",
    "gg_set_profiling", "gg_kernel_stats", "gg_last_launch_count", "gg_set_q_shard", "gg_zgemm",
    "gg_zgemm_noalloc", "gg_set_hf_precision", "gg_estimate_bytes", "gg_set_x2c", "gg_set_graph",
    "gg_batch_create", "gg_batch_run", "gg_batch_destroy", "gg_q_shard_points", "gg_energy_hf", "gg_energy_gw",
    "gg_energy_gw_device", "gg_chemical_potential", "gg_arm_split_timeout_test", "gg_set_autotune",
    "gg_autotune_report", "gg_set_fused_tail",
]


class GreenError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Shape(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("nk", "ink", "nq", "inq", "nao", "NQ", "ns", "nts", "nw_b", "reserved")]


_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} not found: build it with `python -m green_gpu_b200.build`")
    lib = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    I64 = C.POINTER(C.c_int64)
    sig = {
        "gg_create": (C.c_int, [C.POINTER(Shape), C.c_int, C.POINTER(P)]),
        "gg_destroy": (None, [P]),
        "gg_last_error": (C.c_char_p, [P]),
        "gg_set_symmetry": (C.c_int, [P, I64, I64, I64, I64, I64, I64, I64, I64, D, D]),
        "gg_set_kpairs": (C.c_int, [P, C.c_int64, I64, I64, I64]),
        "gg_set_coulomb": (C.c_int, [P, D]),
        "gg_set_coulomb_device": (C.c_int, [P, P]),
        "gg_set_ir": (C.c_int, [P, D, D]),
        "gg_set_split_slices": (C.c_int, [P, C.c_int]),
        "gg_gw_sigma": (C.c_int, [P, D, D, C.c_int, C.c_int]),
        "gg_gw_sigma_device": (C.c_int, [P, P, P, C.c_int, C.c_int, P]),
        "gg_set_capture": (C.c_int, [P, D, D, D]),
        "gg_hf_exchange": (C.c_int, [P, D, D]),
        "gg_hf_fock": (C.c_int, [P, D, D, C.c_double, D]),
        "gg_symmetry_unfold": (C.c_int, [P, D, C.c_int64, D]),
        "gg_last_timings": (C.c_int, [P, D, C.c_int]),
        "gg_version": (C.c_char_p, []),
        "gg_set_profiling": (C.c_int, [P, C.c_int]),
        "gg_kernel_stats": (C.c_int, [P, C.c_int, I64, D, D]),
        "gg_last_launch_count": (C.c_int64, [P]),
        "gg_set_q_shard": (C.c_int, [P, C.c_int, C.c_int]),
        "gg_zgemm": (C.c_int, [P, C.c_int64, C.c_int64, C.c_int64, D, D, D, C.c_int]),
        "gg_zgemm_noalloc": (C.c_int, [C.c_int64, C.c_int64, C.c_int64, P, P, P, P]),
        "gg_set_hf_precision": (C.c_int, [P, C.c_int]),
        "gg_set_x2c": (C.c_int, [P, C.c_int]),
        "gg_set_graph": (C.c_int, [P, C.c_int]),
        "gg_batch_create": (C.c_int, [C.POINTER(P), C.c_int, C.POINTER(P), C.POINTER(P), C.c_int, C.c_int,
                                      C.POINTER(P)]),
        "gg_batch_run": (C.c_int, [P, P]),
        "gg_batch_destroy": (None, [P]),
        "gg_estimate_bytes": (C.c_int, [C.POINTER(Shape), C.c_int64, C.POINTER(C.c_int64)]),
        "gg_q_shard_points": (C.c_int, [C.c_int32, C.c_int, C.c_int, C.POINTER(C.c_int32), C.c_int32,
                                        C.POINTER(C.c_int32)]),
        "gg_energy_hf": (C.c_int, [P, D, D, D, D]),
        "gg_arm_split_timeout_test": (C.c_int, [P]),
        "gg_set_autotune": (C.c_int, [P, C.c_int]),
        "gg_set_fused_tail": (C.c_int, [P, C.c_int]),
        "gg_autotune_report": (C.c_char_p, [P]),
        "gg_energy_gw": (C.c_int, [P, D, D, D, D]),
        "gg_energy_gw_device": (C.c_int, [P, P, P, D, D, P]),
        "gg_chemical_potential": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, D, D, D, C.c_double, C.c_double,
                                            C.c_double, D, D]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _d(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _c128(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
    return a


class Context:
    """One system's device state: symmetry, integrals, IR transforms and work space."""

    def __init__(self, nk, ink, inq, nao, NQ, ns, nts, nw_b, device=0):
        self.lib = load()
        self.shape = Shape(nk, ink, nk, inq, nao, NQ, ns, nts, nw_b, 0)
        h = C.c_void_p()
        rc = self.lib.gg_create(C.byref(self.shape), int(device), C.byref(h))
        if rc != GG_OK:
            raise GreenError(rc, self.lib.gg_last_error(None).decode())
        self.h = h
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.gg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != GG_OK:
            raise GreenError(rc, self.lib.gg_last_error(self.h).decode())

    # --- inputs -------------------------------------------------------------------
    def set_symmetry(self, k_f2r, k_r2f, k_tr, q_f2r, q_r2f, q_tr, k1_from_k2q, k2_from_k1q, U_k=None, U_q=None):
        s = self.shape
        arrs = [np.ascontiguousarray(x, dtype=np.int64) for x in
                (k_f2r, k_r2f, k_tr, q_f2r, q_r2f, q_tr, k1_from_k2q, k2_from_k1q)]
        Uk = _c128(U_k, (s.nk, s.nao, s.nao)) if U_k is not None else None
        Uq = _c128(U_q, (s.nq, s.NQ, s.NQ)) if U_q is not None else None
        self._check(self.lib.gg_set_symmetry(self.h, *[_i64(a) for a in arrs],
                                             _d(Uk.view(np.float64)) if Uk is not None else None,
                                             _d(Uq.view(np.float64)) if Uq is not None else None))

    def set_kpairs(self, num_stored, conj_list, trans_list, irre_pos):
        arrs = [np.ascontiguousarray(x, dtype=np.int64) for x in (conj_list, trans_list, irre_pos)]
        self._check(self.lib.gg_set_kpairs(self.h, int(num_stored), *[_i64(a) for a in arrs]))

    def set_coulomb(self, V_stored):
        V = _c128(V_stored)
        self._check(self.lib.gg_set_coulomb(self.h, _d(V.view(np.float64))))

    def set_coulomb_device(self, ptr: int, keepalive=None):
        self._keep.append(keepalive)
        self._check(self.lib.gg_set_coulomb_device(self.h, C.c_void_p(int(ptr))))

    def set_ir(self, Ttn_FB, Tnt_BF):
        s = self.shape
        a = _c128(Ttn_FB, (s.nts, s.nw_b))
        b = _c128(Tnt_BF, (s.nw_b, s.nts - 2))
        self._check(self.lib.gg_set_ir(self.h, _d(a.view(np.float64)), _d(b.view(np.float64))))

    def set_q_shard(self, rank: int, size: int):
        self._check(self.lib.gg_set_q_shard(self.h, int(rank), int(size)))

    def set_hf_precision(self, precision: int):
        self._check(self.lib.gg_set_hf_precision(self.h, int(precision)))

    def set_x2c(self, enable: bool = True):
        """Two-component mode: G / Sigma / dm / S_k / Fock are spinor matrices of order 2 nao."""
        self._check(self.lib.gg_set_x2c(self.h, int(bool(enable))))
        self.x2c = bool(enable)

    def set_graph(self, enable: bool = True):
        """Capture the GW build into a CUDA graph after its first eager run and replay it."""
        self._check(self.lib.gg_set_graph(self.h, int(bool(enable))))

    def _mat(self):
        """(spin blocks, matrix order) of the caller's G / dm layout."""
        s = self.shape
        return (1, 2 * s.nao) if getattr(self, "x2c", False) else (s.ns, s.nao)

    def set_split_slices(self, slices: int):
        self._check(self.lib.gg_set_split_slices(self.h, int(slices)))

    # --- compute --------------------------------------------------------------------
    def gw_sigma(self, G_tskij, solver=SOLVER_CHOLESKY, precision=PREC_FP64, capture=False):
        s = self.shape
        ns_, m = self._mat()
        shp = (s.nts, ns_, s.ink, m, m)
        G = _c128(G_tskij, shp)
        out = np.empty(shp, np.complex128)
        cap = None
        if capture:
            cap = {"P0": np.empty((s.inq, s.nts, s.NQ, s.NQ), np.complex128),
                   "Pw": np.empty((s.inq, s.nw_b, s.NQ, s.NQ), np.complex128),
                   "Wt": np.empty((s.inq, s.nts, s.NQ, s.NQ), np.complex128)}
            self._check(self.lib.gg_set_capture(self.h, _d(cap["P0"].view(np.float64)),
                                                _d(cap["Pw"].view(np.float64)), _d(cap["Wt"].view(np.float64))))
        try:
            self._check(self.lib.gg_gw_sigma(self.h, _d(G.view(np.float64)), _d(out.view(np.float64)),
                                             int(solver), int(precision)))
        finally:
            if capture:
                self.lib.gg_set_capture(self.h, None, None, None)
        return (out, cap) if capture else out

    def gw_sigma_device(self, G_ptr: int, Sigma_ptr: int, solver=SOLVER_CHOLESKY, precision=PREC_FP64, stream=0):
        self._check(self.lib.gg_gw_sigma_device(self.h, C.c_void_p(int(G_ptr)), C.c_void_p(int(Sigma_ptr)),
                                                int(solver), int(precision), C.c_void_p(int(stream))))

    def hf_exchange(self, dm):
        s = self.shape
        ns_, m = self._mat()
        shp = (ns_, s.ink, m, m)
        D = _c128(dm, shp)
        out = np.empty(shp, np.complex128)
        self._check(self.lib.gg_hf_exchange(self.h, _d(D.view(np.float64)), _d(out.view(np.float64))))
        return out

    def hf_fock(self, dm, S_k, madelung):
        s = self.shape
        ns_, m = self._mat()
        shp = (ns_, s.ink, m, m)
        D = _c128(dm, shp)
        S = _c128(S_k, shp)
        out = np.empty(shp, np.complex128)
        self._check(self.lib.gg_hf_fock(self.h, _d(D.view(np.float64)), _d(S.view(np.float64)), float(madelung),
                                        _d(out.view(np.float64))))
        return out

    def symmetry_unfold(self, X_ibz):
        s = self.shape
        X = _c128(X_ibz)
        nmat = X.size // (s.ink * s.nao * s.nao)
        X = X.reshape(nmat, s.ink, s.nao, s.nao)
        out = np.empty((nmat, s.nk, s.nao, s.nao), np.complex128)
        self._check(self.lib.gg_symmetry_unfold(self.h, _d(X.view(np.float64)), nmat, _d(out.view(np.float64))))
        return out

    def set_fused_tail(self, enable: bool = True):
        self._check(self.lib.gg_set_fused_tail(self.h, 1 if enable else 0))

    def set_autotune(self, enable: bool = True):
        self._check(self.lib.gg_set_autotune(self.h, 1 if enable else 0))

    def autotune_report(self) -> str:
        return (self.lib.gg_autotune_report(self.h) or b"").decode()

    def arm_split_timeout_test(self):
        self._check(self.lib.gg_arm_split_timeout_test(self.h))

    def set_profiling(self, on=True):
        self._check(self.lib.gg_set_profiling(self.h, 1 if on else 0))

    def kernel_stats(self, which):
        n = C.c_int64()
        sec = C.c_double()
        fl = C.c_double()
        self._check(self.lib.gg_kernel_stats(self.h, int(which), C.byref(n), C.byref(sec), C.byref(fl)))
        return {"launches": n.value, "seconds": sec.value, "flops": fl.value}

    def launch_count(self):
        return int(self.lib.gg_last_launch_count(self.h))

    def zgemm(self, A, B, precision=PREC_FP64):
        A = _c128(A)
        B = _c128(B)
        M, K = A.shape
        K2, N = B.shape
        if K != K2:
            raise ValueError("inner dimensions differ")
        out = np.empty((M, N), np.complex128)
        self._check(self.lib.gg_zgemm(self.h, M, N, K, _d(A.view(np.float64)), _d(B.view(np.float64)),
                                      _d(out.view(np.float64)), int(precision)))
        return out

    def energy_hf(self, dm, H, F):
        """(E_1b, E_HF) in FP64 (gg_energy_hf)."""
        out = np.zeros(2)
        self._check(self.lib.gg_energy_hf(self.h, _d(_c128(dm).view(np.float64)), _d(_c128(H).view(np.float64)),
                                          _d(_c128(F).view(np.float64)), _d(out)))
        return float(out[0]), float(out[1])

    def energy_gw(self, G_tskij, Sigma_tskij, M):
        """Galitskii-Migdal E_GW in FP64 with the tau quadrature M (gg_energy_gw)."""
        e = np.zeros(1)
        Mq = np.ascontiguousarray(M, dtype=np.float64)
        self._check(self.lib.gg_energy_gw(self.h, _d(_c128(G_tskij).view(np.float64)),
                                          _d(_c128(Sigma_tskij).view(np.float64)), _d(Mq), _d(e)))
        return float(e[0])

    def energy_gw_device(self, G_ptr: int, Sigma_ptr: int, M, stream=0):
        e = np.zeros(1)
        Mq = np.ascontiguousarray(M, dtype=np.float64)
        self._check(self.lib.gg_energy_gw_device(self.h, C.c_void_p(int(G_ptr)), C.c_void_p(int(Sigma_ptr)), _d(Mq),
                                                 _d(e), C.c_void_p(int(stream))))
        return float(e[0])

    def timings(self):
        buf = np.zeros(8)
        n = self.lib.gg_last_timings(self.h, _d(buf), 8)
        keys = ["total", "unfold", "p0", "ir_fwd", "dyson", "ir_back", "sigma", "e2e"]
        return dict(zip(keys[:n], buf[:n].tolist()))


def q_shard_points(inq: int, rank: int, size: int) -> list:
    """Irreducible q points of one shard, from the library (host-only; no device needed)."""
    lib = load()
    buf = (C.c_int32 * max(inq, 1))()
    n = C.c_int32(0)
    rc = lib.gg_q_shard_points(int(inq), int(rank), int(size), buf, max(inq, 1), C.byref(n))
    if rc != GG_OK:
        raise GreenError(rc, lib.gg_last_error(None).decode())
    return [int(buf[i]) for i in range(n.value)]


def chemical_potential(F, S, weights, beta, nelec, spin_factor):
    """(mu, N(mu)) of a mean-field state (gg_chemical_potential; host-only, no device needed)."""
    lib = load()
    F = _c128(F)
    S = _c128(S)
    ns, ink, n = F.shape[0], F.shape[1], F.shape[-1]
    w = np.ascontiguousarray(weights, dtype=np.float64)
    mu = C.c_double(0.0)
    nat = C.c_double(0.0)
    rc = lib.gg_chemical_potential(ns, ink, n, _d(w), _d(F.view(np.float64)), _d(S.view(np.float64)), float(beta),
                                   float(spin_factor), float(nelec), C.byref(mu), C.byref(nat))
    if rc != GG_OK:
        raise GreenError(rc, lib.gg_last_error(None).decode())
    return mu.value, nat.value


def estimate_bytes(nk, ink, inq, nao, NQ, ns, nts, nw_b, num_kpair_stored) -> int:
    """Device bytes of a resident context of this shape (gg_estimate_bytes)."""
    lib = load()
    sh = Shape(nk, ink, nk, inq, nao, NQ, ns, nts, nw_b, 0)
    out = C.c_int64()
    rc = lib.gg_estimate_bytes(C.byref(sh), int(num_kpair_stored), C.byref(out))
    if rc != GG_OK:
        raise GreenError(rc, lib.gg_last_error(None).decode())
    return int(out.value)


def context_for(sys_, device=0, upload_V=True) -> Context:
    """Build a Context from a synth.System-like object (all inputs set)."""
    ctx = Context(sys_.nk, sys_.ink, sys_.inq, sys_.nao, sys_.NQ, sys_.ns, sys_.nts, sys_.nw_b, device)
    ctx.set_symmetry(sys_.k_full_to_reduced, sys_.k_reduced_to_full, sys_.k_tr_conj, sys_.q_full_to_reduced,
                     sys_.q_reduced_to_full, sys_.q_tr_conj, sys_.k1_from_k2q, sys_.k2_from_k1q, sys_.U_k, sys_.U_q)
    ctx.set_kpairs(sys_.num_kpair_stored, sys_.conj_kpair_list, sys_.trans_kpair_list, sys_.irre_pos_kpair)
    if upload_V:
        ctx.set_coulomb(sys_.V_stored)
    if sys_.nw_b > 0 and sys_.Ttn_FB.size:
        ctx.set_ir(sys_.Ttn_FB, sys_.Tnt_BF)
    return ctx


class Batch:
    """Several systems' GW builds in one CUDA graph (gg_batch_create / gg_batch_run).

    ``items`` are (Context, G_device_ptr, Sigma_device_ptr) triples; creating the batch runs each
    build once eagerly, ``run()`` replays all of them."""

    def __init__(self, items, solver=SOLVER_CHOLESKY, precision=PREC_FP64):
        self.lib = load()
        n = len(items)
        P = C.c_void_p
        ctxs = (P * n)(*[it[0].h for it in items])
        gs = (P * n)(*[int(it[1]) for it in items])
        ss = (P * n)(*[int(it[2]) for it in items])
        self._keep = items
        h = P()
        rc = self.lib.gg_batch_create(ctxs, n, gs, ss, int(solver), int(precision), C.byref(h))
        if rc != GG_OK:
            raise GreenError(rc, self.lib.gg_last_error(None).decode())
        self.h = h

    def run(self, stream=0):
        rc = self.lib.gg_batch_run(self.h, C.c_void_p(int(stream)))
        if rc != GG_OK:
            raise GreenError(rc, self.lib.gg_last_error(None).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.gg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
