"""GPU checks of graph mode (one GW build captured as a CUDA graph and replayed) and of the
batch of uneven systems built in one graph."""
import numpy as np
import pytest
import torch

from green_gpu_b200 import native, synth
from oracle import gw as ogw

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def tiny(symm="tr", ns=1, seed=3, mesh=(2, 2, 1), nao=8, NQ=24):
    return synth.make_system(mesh=mesh, nao=nao, NQ=NQ, ns=ns, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=seed,
                             symmetry=symm)


@pytest.mark.parametrize("precision,tol", [(native.PREC_FP64, 1e-12), (native.PREC_SPLIT, 1e-7)])
def test_graph_replay_matches_eager(precision, tol):
    s = tiny("tr", ns=2)
    eager = native.context_for(s)
    eager.set_split_slices(5)
    ctx = native.context_for(s)
    ctx.set_split_slices(5)
    ctx.set_graph(True)
    a = ctx.gw_sigma(s.G_tskij, precision=precision)      # eager build, then capture
    b = ctx.gw_sigma(s.G_tskij, precision=precision)      # replay
    assert np.array_equal(a, b)
    G2 = 0.9 * s.G_tskij + 0.05 * s.G_tskij[::-1]
    c = ctx.gw_sigma(G2, precision=precision)             # replay on new input values
    d = eager.gw_sigma(G2, precision=precision)
    assert rel(c, d) < 1e-14
    s2 = tiny("tr", ns=2)
    s2.G_tskij = G2
    assert rel(c, ogw.gw_build(s2)) < tol
    eager.close()
    ctx.close()


def test_graph_replay_reports_dyson_failure_and_stays_usable():
    s = tiny("none", ns=1, seed=4)
    s.V_stored = s.V_stored * 30.0
    ctx = native.context_for(s)
    ctx.set_graph(True)
    ok = ctx.gw_sigma(s.G_tskij, solver=native.SOLVER_CHOLESKY)
    ok2 = ctx.gw_sigma(s.G_tskij, solver=native.SOLVER_CHOLESKY)
    assert np.array_equal(ok, ok2)
    G = s.G_tskij.copy()
    G[: s.nts // 2] *= -1.0
    with pytest.raises(native.GreenError) as e:
        ctx.gw_sigma(G, solver=native.SOLVER_CHOLESKY)
    assert e.value.code == native.GG_ERR_NOT_HPD
    again = ctx.gw_sigma(s.G_tskij, solver=native.SOLVER_CHOLESKY)
    assert np.array_equal(again, ok)
    ctx.close()


def test_setter_drops_the_graph():
    s = tiny("none", ns=1, seed=6)
    ctx = native.context_for(s)
    ctx.set_graph(True)
    a = ctx.gw_sigma(s.G_tskij)
    ctx.gw_sigma(s.G_tskij)
    s.V_stored = 0.5 * s.V_stored
    ctx.set_coulomb(s.V_stored)                           # new integrals: the graph must not replay
    b = ctx.gw_sigma(s.G_tskij)
    assert rel(b, ogw.gw_build(s)) < 1e-12
    assert not np.allclose(a, b)
    ctx.close()


@pytest.mark.parametrize("precision", [native.PREC_FP64, native.PREC_SPLIT])
def test_batch_of_uneven_systems_in_one_graph(precision):
    # systems of different k meshes, orbitals, auxiliary sizes and spin: each result in the
    # batch equals the same system built alone
    systems = [tiny("tr", ns=1, seed=7, mesh=(2, 2, 1), nao=8, NQ=24),
               tiny("none", ns=2, seed=8, mesh=(2, 1, 1), nao=6, NQ=40),
               tiny("tr", ns=1, seed=9, mesh=(3, 1, 1), nao=10, NQ=30),
               tiny("none", ns=1, seed=10, mesh=(1, 1, 1), nao=12, NQ=50)]
    dev = torch.device("cuda:0")
    items, ctxs, bufs, alone = [], [], [], []
    for s in systems:
        ctx = native.context_for(s)
        ctx.set_split_slices(5)
        alone.append(ctx.gw_sigma(s.G_tskij, precision=precision))
        G = torch.from_numpy(s.G_tskij.view(np.float64)).to(dev)
        S = torch.zeros_like(G)
        bufs.append((G, S))
        ctxs.append(ctx)
        items.append((ctx, G.data_ptr(), S.data_ptr()))
    torch.cuda.synchronize()
    batch = native.Batch(items, precision=precision)
    for ctx, (G, S), ref in zip(ctxs, bufs, alone):
        out = S.cpu().numpy().view(np.complex128).reshape(ref.shape)
        assert rel(out, ref) < 1e-14
    # replay on new input values
    for (G, S) in bufs:
        G.mul_(0.8)
        S.zero_()
    torch.cuda.synchronize()
    batch.run()
    for s, ctx, (G, S) in zip(systems, ctxs, bufs):
        out = S.cpu().numpy().view(np.complex128).reshape((s.nts, s.ns, s.ink, s.nao, s.nao))
        ref = ctx.gw_sigma(0.8 * s.G_tskij, precision=precision)
        assert rel(out, ref) < 1e-14
    batch.close()
    for ctx in ctxs:
        ctx.close()


def test_graph_is_recaptured_after_other_entry_points_grow_shared_buffers():
    # the HF exchange, the symmetry unfold and the split GEMM share the context's work buffers
    # with the GW build; when they grow one, the captured graph would address freed memory, so
    # the next build must capture again instead of replaying
    s = tiny("tr", ns=1, seed=13)
    ctx = native.context_for(s)
    ctx.set_graph(True)
    a = ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)  # eager build, then capture
    assert np.array_equal(ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT), a)  # replay
    big = np.repeat(s.G_tskij[:, 0], 40, axis=0)  # [40 nts][ink][nao][nao]: grows the unfold scratch
    ctx.symmetry_unfold(big)
    ctx.set_hf_precision(native.PREC_SPLIT)
    ctx.hf_exchange(s.dm)
    rng = np.random.default_rng(1)
    A = rng.standard_normal((700, 3000)) + 1j * rng.standard_normal((700, 3000))
    ctx.zgemm(A, A.T.copy(), precision=native.PREC_SPLIT)     # grows the split engine's planes
    b = ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)  # eager again, captured again
    c = ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)  # replay of the new graph
    assert np.array_equal(b, a)
    assert np.array_equal(c, a)
    ctx.close()


def test_batch_refuses_to_replay_after_a_member_context_changed():
    systems = [tiny("tr", ns=1, seed=14), tiny("none", ns=1, seed=15, mesh=(2, 1, 1), nao=6, NQ=20)]
    dev = torch.device("cuda:0")
    items, ctxs, bufs = [], [], []
    for s in systems:
        ctx = native.context_for(s)
        G = torch.from_numpy(s.G_tskij.view(np.float64)).to(dev)
        S = torch.zeros_like(G)
        bufs.append((G, S))
        ctxs.append(ctx)
        items.append((ctx, G.data_ptr(), S.data_ptr()))
    batch = native.Batch(items)
    batch.run()
    big = np.repeat(systems[0].G_tskij[:, 0], 40, axis=0)
    ctxs[0].symmetry_unfold(big)                              # reallocates a buffer the graph uses
    with pytest.raises(native.GreenError) as e:
        batch.run()
    assert e.value.code == native.GG_ERR_STATE
    batch.close()
    for ctx in ctxs:
        ctx.close()
