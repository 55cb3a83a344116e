"""GPU checks of the split-precision (Ozaki INT8, tcgen05) engine against FP64 references.

Error metric: max |C - C_ref| / max |C_ref| (norm-wise relative).  The truncation error of
S slices of 7 bits is about 2^(-7S) relative to the row / column maxima, growing with the
reduction length; the bounds below are that estimate with head-room."""
import numpy as np
import pytest

from green_gpu_b200 import native, synth
from oracle import gw as ogw

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def bound(S, K):
    return 2.0 ** (-7 * S + 4) * np.sqrt(K) + 1e-14


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(2, 2, 2, 2, 4, 1, 4, 3)
    yield c
    c.close()


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (130, 70, 300), (400, 400, 2704), (52, 20800 // 8, 52)])
@pytest.mark.parametrize("S", [2, 3, 4, 6])
def test_split_zgemm_error_bound(ctx, M, N, K, S):
    rng = np.random.default_rng(M * 7 + N + K + S)
    A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    # rows / columns of very different magnitude, as in V^Q exp(-0.1 Q)
    A *= np.exp(-0.05 * np.arange(M))[:, None]
    B *= np.exp(-0.03 * np.arange(N))[None, :]
    ref = A @ B
    ctx.set_split_slices(S)
    out = ctx.zgemm(A, B, precision=native.PREC_SPLIT)
    # row-relative error (each row carries its own scale)
    err = np.abs(out - ref).max(axis=1) / np.abs(ref).max(axis=1)
    assert err.max() < bound(S, K), (S, err.max())


def test_fp64_zgemm_matches_numpy(ctx):
    rng = np.random.default_rng(2)
    A = rng.standard_normal((77, 133)) + 1j * rng.standard_normal((77, 133))
    B = rng.standard_normal((133, 91)) + 1j * rng.standard_normal((133, 91))
    assert rel(ctx.zgemm(A, B), A @ B) < 1e-14


def test_split_zgemm_exact_for_small_integers(ctx):
    # integers below 2^5 are represented exactly by the first slice: the result is exact
    rng = np.random.default_rng(3)
    A = rng.integers(-30, 30, (200, 500)) + 1j * rng.integers(-30, 30, (200, 500))
    B = rng.integers(-30, 30, (500, 150)) + 1j * rng.integers(-30, 30, (500, 150))
    ctx.set_split_slices(2)
    out = ctx.zgemm(A.astype(np.complex128), B.astype(np.complex128), precision=native.PREC_SPLIT)
    assert np.array_equal(out, (A @ B).astype(np.complex128))


@pytest.mark.parametrize("S", [4, 6])
def test_gw_split_matches_oracle(S):
    s = synth.make_system(mesh=(2, 2, 1), nao=8, NQ=24, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=9,
                          symmetry="none")
    c = native.context_for(s)
    c.set_split_slices(S)
    out = c.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)
    ref = ogw.gw_build(s)
    assert rel(out, ref) < {4: 1e-6, 6: 1e-9}[S]


@pytest.mark.parametrize("M,N", [(6400, 3072), (2560, 16000)])
def test_fp64_zgemm_tile_runs_match_numpy(ctx, M, N):
    # short reductions (K = 52) over many tiles take the path where one CTA computes a run of
    # consecutive tiles along M (first case) or N (second, with a partial last run)
    rng = np.random.default_rng(M + N)
    K = 52
    A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    assert rel(ctx.zgemm(A, B), A @ B) < 1e-14


def test_autotuner_picks_a_configuration_per_shape_and_keeps_results():
    # the tuned configuration changes only the FP64 order of split-K partial sums, so a tuned
    # GW build equals the untuned one to rounding (1e-13) and the oracle to the split tolerance
    s = synth.make_system(mesh=(2, 2, 1), nao=8, NQ=24, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=9,
                          symmetry="none")
    plain = native.context_for(s)
    ref = plain.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)
    c = native.context_for(s)
    c.set_autotune(True)
    first = c.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)   # tunes every shape
    report = c.autotune_report().splitlines()
    assert report and all("BN" in line and "split-K" in line for line in report)
    second = c.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)  # uses the tuned choices
    assert np.array_equal(first, second)
    assert rel(first, ref) < 1e-13
    assert rel(first, ogw.gw_build(s)) < 1e-8
    assert c.autotune_report().splitlines() == report           # nothing re-tuned
    c.set_graph(True)                                             # tuned shapes also replay in a graph
    g1 = c.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)
    g2 = c.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)
    assert np.array_equal(g1, first) and np.array_equal(g2, first)
    plain.close()
    c.close()


@pytest.mark.parametrize("M,N,K", [(300, 24, 500), (130, 72, 52), (1000, 24, 3000)])
def test_split_zgemm_double_buffered_narrow_tiles(ctx, M, N, K):
    # 2N a multiple of 48 and of no wider tile: the 5-slice engine runs 48-wide tiles with two
    # accumulator sets in TMEM (the next tile's MMAs overlap the previous tile's drain)
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    A *= np.exp(-0.05 * np.arange(M) / 10)[:, None]
    ref = A @ B
    ctx.set_split_slices(5)
    out = ctx.zgemm(A, B, precision=native.PREC_SPLIT)
    err = np.abs(out - ref).max(axis=1) / np.abs(ref).max(axis=1)
    assert err.max() < bound(5, K), err.max()
