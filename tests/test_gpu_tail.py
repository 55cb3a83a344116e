"""GPU checks of the fused Sigma tail (Z = X G and the reduction of Z V^+ in one kernel, Z in
registers) against the two-GEMM form with Z in device memory, and against the FP64 oracle.

Both forms sum in a fixed order; they differ in the FP64 summation order only, so they agree
to 1e-13 relative (norm-wise) in both precisions (in a split build both tails read the same
INT8 contraction output).  Orbital counts cover one to seven 8-wide tiles, counts that are not
multiples of 4 or 8, the largest fused count (52) and one above it (the two-GEMM fallback)."""
import numpy as np
import pytest

import fixture
from green_gpu_b200 import native, synth
from oracle import gw as ogw

pytestmark = pytest.mark.gpu

TOL_FORMS = 1e-13


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def small(nao, NQ, symm="tr", ns=1, mesh=(2, 1, 1), seed=5):
    return synth.make_system(mesh=mesh, nao=nao, NQ=NQ, ns=ns, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=seed,
                             symmetry=symm)


@pytest.mark.parametrize("precision", [native.PREC_FP64, native.PREC_SPLIT])
@pytest.mark.parametrize("nao,NQ,ns,symm", [(3, 17, 1, "tr"), (8, 24, 2, "none"), (13, 40, 1, "tr"),
                                            (26, 100, 1, "none"), (45, 64, 1, "tr"), (52, 60, 2, "tr")])
def test_fused_tail_matches_two_gemm_form(nao, NQ, ns, symm, precision):
    s = small(nao, NQ, symm=symm, ns=ns, seed=nao)
    ctx = native.context_for(s)
    try:
        ctx.set_fused_tail(False)
        two = ctx.gw_sigma(s.G_tskij, precision=precision)
        ctx.set_fused_tail(True)
        fused = ctx.gw_sigma(s.G_tskij, precision=precision)
        again = ctx.gw_sigma(s.G_tskij, precision=precision)
    finally:
        ctx.close()
    assert rel(fused, two) < TOL_FORMS
    assert np.array_equal(fused, again)  # deterministic


@pytest.mark.parametrize("nao", [52, 53])
def test_tail_matches_oracle_at_the_fused_limit(nao):
    # 52: the largest orbital count of the fused kernel; 53: the first that runs two GEMMs
    s = small(nao, 30, symm="tr", mesh=(2, 1, 1), seed=3)
    ctx = native.context_for(s)
    try:
        ctx.set_fused_tail(True)
        out = ctx.gw_sigma(s.G_tskij)
    finally:
        ctx.close()
    assert rel(out, ogw.gw_build(s)) < 1e-10


def test_tail_kernel_statistics():
    s = small(26, 50, symm="none", seed=9)
    ctx = native.context_for(s)
    try:
        stats = {}
        for fused in (False, True):
            ctx.set_fused_tail(fused)
            ctx.set_profiling(True)
            ctx.gw_sigma(s.G_tskij)
            ctx.set_profiling(False)
            stats[fused] = ctx.kernel_stats(2)
    finally:
        ctx.close()
    # entry 2 is the product with V^+ alone, or the fused kernel that also forms Z = X G: one
    # entry per (pair, spin) either way, the fused one with the flops of both products
    n, N, T = s.nao, s.NQ, s.nts
    xg = T * (8.0 * N * n * n * n + 12.0 * N * n * n)
    zv = 8.0 * T * n * n * N * n + 12.0 * T * n * n
    assert stats[True]["launches"] == stats[False]["launches"] > 0
    assert stats[False]["flops"] == pytest.approx(stats[False]["launches"] * zv, rel=1e-12)
    assert stats[True]["flops"] == pytest.approx(stats[True]["launches"] * (xg + zv), rel=1e-12)
    assert stats[True]["seconds"] > 0 and stats[False]["seconds"] > 0


@pytest.mark.parametrize("precision", [native.PREC_FP64, native.PREC_SPLIT])
def test_fused_tail_with_space_group_symmetry(precision):
    # the reference's 27 -> 4 k fixture: rotated W~ (U_q) and k-pair conj/trans lists feed the tail
    s, _ = fixture.load(gw=True)
    nts, nw = s.nts, 41
    rng = np.random.default_rng(11)
    s.nw_b = nw
    s.Ttn_FB = 0.05 * (rng.standard_normal((nts, nw)) + 1j * rng.standard_normal((nts, nw)))
    s.Tnt_BF = 0.05 * (rng.standard_normal((nw, nts - 2)) + 1j * rng.standard_normal((nw, nts - 2)))
    ctx = native.context_for(s)
    try:
        ctx.set_fused_tail(False)
        two = ctx.gw_sigma(s.G_tskij, solver=native.SOLVER_LU, precision=precision)
        ctx.set_fused_tail(True)
        fused = ctx.gw_sigma(s.G_tskij, solver=native.SOLVER_LU, precision=precision)
    finally:
        ctx.close()
    assert rel(fused, two) < TOL_FORMS
