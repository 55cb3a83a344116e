"""CPU checks of the FP64 oracle: pinned against the reference's own golden vectors
and against identities the reference relies on."""
import os

import numpy as np
import pytest

import fixture
from green_gpu_b200 import ir, synth
from oracle import gw, hf, symmetry


def test_hf_oracle_matches_reference_sigma1():
    # test/cu_solver_test.cpp:89-95: Sigma1 = prefactor * solve(dm), prefactor -1 for ns = 2,
    # compared element-wise at an absolute 1e-8.
    s, ref = fixture.load()
    pref = -1.0 if s.ns == 2 else -2.0
    out = pref * hf.hf_build(s)
    assert np.abs(out - ref["Sigma1"]).max() < 1e-8


def test_symmetry_roundtrip_reference_fock():
    # test/cu_symmetry_test.cu:38-130 and cu_solver_test.cpp:343-412 (tolerance 1e-4).
    s, ref = fixture.load()
    Ff = ref["Fock_k_full"]
    un = symmetry.ibz_to_full(s, Ff[:, s.k_reduced_to_full])
    assert np.abs(un - Ff).max() < 1e-4


def test_kpair_lookup_matches_product_host_logic():
    s, _ = fixture.load()
    for k1 in range(s.nk):
        for k2 in range(s.nk):
            np.testing.assert_array_equal(symmetry.coulomb(s, k1, k2), synth.coulomb_pair(s, k1, k2))


def test_ir_transforms_roundtrip():
    b = ir.IRBasis(100.0, 1e4, 72, 69)
    assert b.cond_fit < 1e3 and b.cond_freq < 1e3
    assert np.allclose(b.tau, 100.0 - b.tau[::-1])
    assert np.array_equal(b.wn, -b.wn[::-1])
    for w0 in (0.3, -2.0, 17.0, 0.01):
        f = ir._kernel_tau(b.tau, np.array([w0]), 100.0)[:, 0] / np.tanh(50.0 * w0)
        fw = ir._kernel_iw(b.wn, np.array([w0]), 100.0)[:, 0] / np.tanh(50.0 * w0)
        assert np.abs(b.Tnt_BF @ f[1:-1] - fw).max() < 1e-7 * np.abs(fw).max()
        assert np.abs(b.Ttn_FB @ fw - f).max() < 1e-5 * np.abs(f).max()


def _tiny(symm="tr", ns=1, seed=1):
    return synth.make_system(mesh=(3, 2, 1), nao=4, NQ=10, ns=ns, beta=10.0, lam=100.0, nts=24, nw_b=21,
                             seed=seed, symmetry=symm)


def _unreduced(s):
    full = synth.unfold_kpairs(s)
    nk = s.nk
    ident = np.arange(nk, dtype=np.int64)
    full.k_full_to_reduced = ident
    full.k_reduced_to_full = ident.copy()
    full.k_tr_conj = np.zeros(nk, np.int64)
    full.k_stars = [np.array([k]) for k in range(nk)]
    full.q_full_to_reduced = ident.copy()
    full.q_reduced_to_full = ident.copy()
    full.q_tr_conj = np.zeros(nk, np.int64)
    full.q_stars = [np.array([k]) for k in range(nk)]
    full.ink = full.inq = nk
    full.G_tskij = np.ascontiguousarray(np.moveaxis(gw.g_full(s), 0, 2).swapaxes(0, 1))
    full.S_k = np.stack([np.stack([symmetry.unfold_ao(s, s.S_k[a], k) for k in range(nk)]) for a in range(s.ns)])
    return full


@pytest.mark.parametrize("ns", [1, 2])
def test_gw_oracle_tr_reduced_equals_unreduced(ns):
    s = _tiny("tr", ns=ns)
    full = _unreduced(s)
    a = gw.gw_build(s)
    b = gw.gw_build(full)[:, :, s.k_reduced_to_full]
    assert np.abs(a - b).max() < 1e-10 * np.abs(b).max()


def test_hf_oracle_tr_reduced_equals_unreduced():
    s = _tiny("tr", ns=2)
    full = _unreduced(s)
    a = hf.hf_build(s)
    b = hf.hf_build(full, dm=full.G_tskij[-1])[:, s.k_reduced_to_full]
    assert np.abs(a - b).max() < 1e-12 * np.abs(b).max()


def test_gw_oracle_identities():
    s = _tiny("none")
    keep = {}
    gw.gw_build(s, keep=keep)
    for P0, Pw, Wt in zip(keep["P0"], keep["Pw"], keep["Wt"]):
        # Hermitian P0(tau) with P0(beta - tau) = P0(tau) (cugw_qpt.cu:179-191)
        assert np.abs(P0 - np.conj(np.swapaxes(P0, 1, 2))).max() < 1e-13 * np.abs(P0).max()
        assert np.array_equal(P0, P0[::-1])
        # P0(tau) negative semidefinite at every interior tau
        for t in range(1, s.nts - 1):
            assert np.linalg.eigvalsh(0.5 * (P0[t] + P0[t].conj().T)).max() < 1e-12
        # W~(i Omega) = P (1 - P)^{-1} is Hermitian (cugw_qpt.cu:310-316)
        assert np.abs(Wt - np.conj(np.swapaxes(Wt, 1, 2))).max() < 1e-8 * np.abs(Wt).max()


def test_cholesky_and_lu_agree():
    s = _tiny("none")
    a = gw.gw_build(s, solver="cholesky")
    b = gw.gw_build(s, solver="lu")
    assert np.abs(a - b).max() < 1e-12 * np.abs(a).max()


def test_hermitian_symmetrize_matches_reference_kernel():
    # cuda_common.cu:249-265, written as the reference's per-row loop
    rng = np.random.default_rng(3)
    M = rng.standard_normal((7, 7)) + 1j * rng.standard_normal((7, 7))
    R = M.copy()
    for i in range(7):
        R[i, i] = R[i, i].real
        for j in range(i):
            re = 0.5 * (R[i, j].real + R[j, i].real)
            im = 0.5 * (R[i, j].imag - R[j, i].imag)
            R[i, j] = re + 1j * im
            R[j, i] = re - 1j * im
    assert np.array_equal(gw.hermitian_symmetrize(M), R)


def test_df_integral_reader_matches_fixture():
    # reads the reference's own chunk files when its source tree is named by the
    # GREEN_GPU_REFERENCE environment variable (the golden npz holds the same integrals)
    import os
    root = os.environ.get("GREEN_GPU_REFERENCE")
    if not root:
        pytest.skip("GREEN_GPU_REFERENCE (path of the green-gpu source tree) is not set")
    ref_dir = os.path.join(root, "test", "data", "HF", "df_hf_int")
    if not os.path.isdir(ref_dir):
        pytest.skip(f"{ref_dir} not found")
    from green_gpu_b200 import df_integral
    s, _ = fixture.load()
    V = df_integral.read_stored(ref_dir, s.nao, s.NQ)
    assert np.array_equal(V, s.V_stored)


def test_x2c_hf_oracle_matches_reference_sigma1():
    # test/cu_solver_test.cpp:335-337 (HF_X2C): Sigma1 = -1 * solve(dm), dm = G_tau[last],
    # compared element-wise at an absolute 1e-8.
    from oracle import x2c
    s, ref = fixture.load_x2c()
    out = -1.0 * x2c.hf_build(s, ref["dm"])
    assert np.abs(out - ref["Sigma1"]).max() < 1e-8


def _blockdiag(X, Y):
    n = X.shape[-1]
    out = np.zeros(X.shape[:-2] + (2 * n, 2 * n), np.complex128)
    out[..., :n, :n] = X
    out[..., n:, n:] = Y
    return out


def test_x2c_oracle_spin_diagonal_equals_scalar():
    # with uncoupled spins (ab = ba = 0) the two-component build reduces to the scalar one:
    # P0 sums the aa and bb blocks with prefactor -1 where the scalar build doubles one block
    # with -2; HF takes each spin block at half the scalar (spin-summed) density.
    from oracle import x2c
    s = _tiny("none")
    sig = gw.gw_build(s)
    S2 = _blockdiag(s.G_tskij[:, 0], s.G_tskij[:, 0])[:, None]
    out = x2c.gw_build(s, S2)
    assert np.abs(out - _blockdiag(sig[:, 0], sig[:, 0])[:, None]).max() < 1e-12 * np.abs(sig).max()
    dm = s.G_tskij[-1]
    F = hf.hf_build(s, dm)
    s2 = _tiny("none")
    s2.S_k = _blockdiag(s.S_k, s.S_k)
    F2 = x2c.hf_build(s2, _blockdiag(0.5 * dm, 0.5 * dm))
    assert np.abs(F2 - _blockdiag(F, F)).max() < 1e-12 * np.abs(F).max()


def test_x2c_split_merge_roundtrip():
    from oracle import x2c
    rng = np.random.default_rng(5)
    M = rng.standard_normal((3, 8, 8)) + 1j * rng.standard_normal((3, 8, 8))
    assert np.array_equal(x2c.merge(x2c.split(M, 4)), M)
    H = M + np.conj(np.swapaxes(M, 1, 2))
    assert np.array_equal(x2c.merge(x2c.split(H, 3)), H)


def test_gw_oracle_matches_reference_sigma_tau():
    # test/cu_solver_test.cpp:226-288 (solve_gw): one GW iteration on the H2 27 -> 4 k fixture
    # (space-group rotations U_k / U_q), compared with result/Sigma_tau at |a - b| < 1e-6
    # (:287).  The tau grid of the fixture's IR file is recovered from its mean-field G_tau
    # (tests/golden/gw_grid.py) and the transforms are built on it.
    import gw_grid
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hf_h2_27k.npz"))
    tau, mu, off = gw_grid.recover_tau(d["G_tau_gw"], d["Fock_k_full"], d["S_k_full"], d["k_ibz2bz"].astype(np.int64))
    assert off < 1e-13                       # G_tau is the mean-field G of HF/Fock-k: diagonal in the MO basis
    assert len(tau) == 110 and np.all(np.diff(tau) > 0)
    _, Ttn, Tnt = gw_grid.fixture_transforms()
    s, ref = fixture.load(gw=True)
    s.nw_b, s.Ttn_FB, s.Tnt_BF = Ttn.shape[1], Ttn, Tnt
    for solver in ("lu", "cholesky"):
        out = gw.gw_build(s, solver=solver)
        assert np.abs(out - ref["Sigma_tau_gw"]).max() < 1e-6
