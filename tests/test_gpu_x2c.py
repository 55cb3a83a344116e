"""GPU checks of the two-component (X2C) mode through the C ABI.

HF is pinned to the reference's own HF_X2C fixture (test/cu_solver_test.cpp:335-337, absolute
1e-8); GW is compared with the X2C oracle (spin blocks as pseudo-spins, oracle/x2c.py) on a
synthetic spin-coupled system, at 1e-10 relative for FP64 and a slice-count bound for split."""
import numpy as np
import pytest

import fixture
from green_gpu_b200 import native, synth
from oracle import x2c

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("precision,tol", [(native.PREC_FP64, 1e-10), (native.PREC_SPLIT, 1e-8)])
def test_x2c_hf_matches_reference_sigma1(precision, tol):
    s, ref = fixture.load_x2c()
    ctx = native.context_for(s)
    ctx.set_x2c(True)
    ctx.set_split_slices(5)
    ctx.set_hf_precision(precision)
    out = -1.0 * ctx.hf_fock(ref["dm"], s.S_k, s.madelung)
    ctx.close()
    assert np.abs(out - ref["Sigma1"]).max() < tol


@pytest.fixture(scope="module")
def sys2c():
    return synth.make_x2c_system(mesh=(2, 1, 1), nao=6, NQ=20, nts=24, nw_b=21, seed=4)


@pytest.mark.parametrize("precision,slices,tol", [(native.PREC_FP64, 4, 1e-10), (native.PREC_SPLIT, 6, 1e-9)])
def test_x2c_gw_matches_oracle(sys2c, precision, slices, tol):
    s = sys2c
    ref = x2c.gw_build(s, s.G_tskij)
    ctx = native.context_for(s)
    ctx.set_x2c(True)
    ctx.set_split_slices(slices)
    out = ctx.gw_sigma(s.G_tskij, precision=precision)
    ctx.close()
    assert out.shape == ref.shape
    assert rel(out, ref) < tol


def test_x2c_hf_exchange_synthetic_matches_oracle(sys2c):
    s = sys2c
    dm = s.G_tskij[-1]
    ctx = native.context_for(s)
    ctx.set_x2c(True)
    out = ctx.hf_fock(dm, s.S_k, 0.37)
    ctx.close()
    s.madelung = 0.37
    assert rel(out, x2c.hf_build(s, dm)) < 1e-12


def test_x2c_rejects_symmetry_reduction():
    # 3x2x1 k: time reversal pairs k with -k != k, so the IBZ is smaller than the mesh
    s = synth.make_system(mesh=(3, 2, 1), nao=4, NQ=10, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=2,
                          symmetry="tr")
    assert s.ink < s.nk and np.any(s.k_tr_conj)
    ctx = native.context_for(s)
    ctx.set_x2c(True)
    G = np.zeros((s.nts, 1, s.ink, 2 * s.nao, 2 * s.nao), np.complex128)
    with pytest.raises(native.GreenError):
        ctx.gw_sigma(G)
    ctx.close()
