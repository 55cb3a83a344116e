"""GPU accuracy of the shipped split-precision default and of the q-sharded CUDA path.

Tolerances (max |x - x_ref| / max |x_ref|, written per test):
* split precision at the default slice count (5): Sigma, P0 and the exchange K within 1e-8 of
  the FP64 oracle - the tolerance the split path is specified to (four slices gives ~5e-8);
* q sharding: the partial Sigma of the shards sum to the unsharded build within 1e-13 (the
  sums differ only in the order of the q contributions).
"""
import numpy as np
import pytest

import fixture
from green_gpu_b200 import native, synth
from oracle import gw as ogw
from oracle import hf as ohf

pytestmark = pytest.mark.gpu

TOL_SPLIT = 1e-8


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def cfg1():
    # the CPU-runnable benchmark configuration: 2x2x2 k, nao 26, NQ 120, 72 tau / 69 Omega
    s = synth.make_system(mesh=(2, 2, 2), nao=26, NQ=120, ns=1, seed=7)
    keep = {}
    ref = ogw.gw_build(s, keep=keep)
    return s, ref, keep


def test_default_slice_count_is_five():
    ctx = native.Context(2, 2, 2, 2, 4, 1, 4, 3)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((96, 300)) + 1j * rng.standard_normal((96, 300))
    B = rng.standard_normal((300, 80)) + 1j * rng.standard_normal((300, 80))
    default = ctx.zgemm(A, B, precision=native.PREC_SPLIT)
    ctx.set_split_slices(5)
    five = ctx.zgemm(A, B, precision=native.PREC_SPLIT)
    ctx.close()
    assert np.array_equal(default, five)


def test_split_default_cfg1_sigma_p0_within_1e8(cfg1):
    s, ref, keep = cfg1
    ctx = native.context_for(s)  # slice count left at the library default
    out, cap = ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT, capture=True)
    assert rel(out, ref) < TOL_SPLIT
    for iq in range(s.inq):
        assert rel(cap["P0"][iq], keep["P0"][iq]) < TOL_SPLIT
        assert rel(cap["Wt"][iq], keep["Wt"][iq]) < TOL_SPLIT
    ctx.close()


def test_split_default_cfg1_exchange_within_1e8(cfg1):
    s, _, _ = cfg1
    ctx = native.context_for(s)
    ctx.set_hf_precision(native.PREC_SPLIT)
    K = ctx.hf_exchange(s.dm)
    assert rel(K, ohf.exchange(s, s.dm)) < TOL_SPLIT
    ctx.close()


def test_split_default_space_group_symmetry():
    # the reference's 27 -> 4 k fixture with rotations U_k (AO) and U_q (auxiliary) and
    # conj/trans k-pair lists, seeded IR transforms of the fixture's shape
    s, _ = fixture.load(gw=True)
    nts, nw = s.nts, 41
    rng = np.random.default_rng(11)
    s.nw_b = nw
    s.Ttn_FB = 0.05 * (rng.standard_normal((nts, nw)) + 1j * rng.standard_normal((nts, nw)))
    s.Tnt_BF = 0.05 * (rng.standard_normal((nw, nts - 2)) + 1j * rng.standard_normal((nw, nts - 2)))
    ctx = native.context_for(s)
    out = ctx.gw_sigma(s.G_tskij, solver=native.SOLVER_LU, precision=native.PREC_SPLIT)
    ref = ogw.gw_build(s, solver="lu")
    assert rel(out, ref) < TOL_SPLIT
    ctx.set_hf_precision(native.PREC_SPLIT)
    K = ctx.hf_exchange(s.dm)
    assert rel(K, ohf.exchange(s, s.dm)) < TOL_SPLIT
    ctx.close()


@pytest.mark.parametrize("precision", [native.PREC_FP64, native.PREC_SPLIT])
def test_q_shards_sum_to_the_full_build(precision):
    # round-robin q distribution of src/cugw_utils.cu:115, partial Sigma summed as the
    # all-reduce of src/gw_gpu_kernel.cpp:187 does
    s = synth.make_system(mesh=(3, 2, 1), nao=6, NQ=20, ns=2, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=12,
                          symmetry="tr")
    assert s.inq >= 3
    full_ctx = native.context_for(s)
    full = full_ctx.gw_sigma(s.G_tskij, precision=precision)
    parts = []
    for rank in range(2):
        c = native.context_for(s)
        c.set_q_shard(rank, 2)
        parts.append(c.gw_sigma(s.G_tskij, precision=precision))
        c.close()
    assert rel(parts[0] + parts[1], full) < 1e-13
    # each shard alone is a proper part (neither is empty nor the whole)
    assert rel(parts[0], full) > 1e-3 and rel(parts[1], full) > 1e-3
    # the same context restored to the full build
    full_ctx.set_q_shard(1, 2)
    full_ctx.gw_sigma(s.G_tskij, precision=precision)
    full_ctx.set_q_shard(0, 1)
    assert rel(full_ctx.gw_sigma(s.G_tskij, precision=precision), full) < 1e-14
    full_ctx.close()
