"""The split engine's bounded waits, made to run out on purpose (no fault, no hang).

gg_arm_split_timeout_test makes the next split GEMM run with a 0.1 s limit on every barrier
wait while CTA 0 withholds the release of one drained accumulator, so its MMA warp's wait runs
out.  The kernel must record the time-out, let its copies and MMAs in flight complete, free its
tensor memory and return: the call reports GG_ERR_INTERNAL, and the same context then gives
correct results again (split GEMM within its error bound, a GW build equal to the oracle).
"""
import numpy as np
import pytest

from green_gpu_b200 import native, synth
from oracle import gw as ogw

pytestmark = pytest.mark.gpu


def test_split_wait_runs_out_and_the_context_recovers():
    ctx = native.Context(2, 2, 2, 2, 4, 1, 4, 3)
    rng = np.random.default_rng(4)
    # 24 x 10 x 2 tiles of 128 x 96 (more work units than SMs, so CTA 0 gets a second unit)
    M, N, K = 128 * 24, 48 * 10, 256
    A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    ref = A @ B
    ctx.arm_split_timeout_test()
    with pytest.raises(native.GreenError) as e:
        ctx.zgemm(A, B, precision=native.PREC_SPLIT)
    assert e.value.code == native.GG_ERR_INTERNAL
    assert "timed out" in str(e.value)
    # the same context and engine work again
    out = ctx.zgemm(A, B, precision=native.PREC_SPLIT)
    # the engine's error bound at 5 slices: 2^(-7 S + 4) sqrt(K) of the largest element
    assert np.abs(out - ref).max() < 2.0 ** (-7 * 5 + 4) * np.sqrt(K) * np.abs(ref).max()
    ctx.close()
    s = synth.make_system(mesh=(2, 2, 1), nao=8, NQ=24, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=9,
                          symmetry="none")
    c = native.context_for(s)
    got = c.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)
    ref = ogw.gw_build(s)
    assert np.abs(got - ref).max() < 1e-8 * np.abs(ref).max()
    c.close()
