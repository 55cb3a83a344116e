"""FP64 energy and chemical-potential reductions.

CPU: the library's chemical potential (gg_chemical_potential, host-only) against the oracle and
against the reference's H2 fixture, whose G_tau was built at the mu recovered from it
(tests/golden/gw_grid.py): both must agree to 1e-9 Ha.  The tau quadrature used by the GW
energy is exact (1e-12) for products of logistic-kernel functions.
GPU: gg_energy_hf / gg_energy_gw through the C ABI against the oracle (1e-12 relative), and the
split-precision E_GW of the cfg1 system within 1e-8 of FP64.
"""
import os

import numpy as np
import pytest

import fixture
from green_gpu_b200 import ir, native, synth
from oracle import energy as oen
from oracle import gw as ogw

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixture_mean_field():
    d = np.load(os.path.join(HERE, "golden", "hf_h2_27k.npz"))
    ibz = d["k_ibz2bz"].astype(np.int64)
    F = d["Fock_k_full"][:, ibz]
    S = d["S_k_full"][:, ibz]
    return d, F, S


def test_chemical_potential_reproduces_the_reference_fixture():
    import gw_grid
    d, F, S = _fixture_mean_field()
    s, _ = fixture.load(gw=True)
    w = oen.kweights(s)
    # H2: two electrons per cell, ns = 2 (spin factor 1), beta = 100
    mu, n = native.chemical_potential(F, S, w, 100.0, 2.0, 1.0)
    assert abs(n - 2.0) < 1e-12
    mu_ref = oen.chemical_potential(s, F, S, 100.0, 2.0)
    assert abs(mu - mu_ref) < 1e-9
    # the fixture's own mu (recovered from its G_tau) solves the same particle-number equation
    # to a search tolerance of ~1e-9 electrons; in the gap of this insulator dN/dmu ~ 1e-3, so
    # the two roots agree to ~1e-6 Ha
    _, mu_fixture, _ = gw_grid.recover_tau(d["G_tau_gw"], d["Fock_k_full"], d["S_k_full"], d["k_ibz2bz"].astype(np.int64))
    eps = oen.eigenvalues(F, S)
    assert abs(oen.particle_number(eps, w, mu_fixture, 100.0, 1.0) - 2.0) < 1e-8
    assert abs(mu - mu_fixture) < 1e-5


def test_chemical_potential_metal_and_errors():
    rng = np.random.default_rng(3)
    ns, ink, n = 1, 3, 6
    A = rng.standard_normal((ns, ink, n, n)) + 1j * rng.standard_normal((ns, ink, n, n))
    F = 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))
    B = rng.standard_normal((ns, ink, n, n)) + 1j * rng.standard_normal((ns, ink, n, n))
    S = np.eye(n)[None, None] + 0.05 * (B @ np.conj(np.swapaxes(B, -1, -2)))
    w = np.array([0.25, 0.25, 0.5])
    for nelec in (1.3, 5.0, 9.7):
        mu, nat = native.chemical_potential(F, S, w, 10.0, nelec, 2.0)
        assert abs(nat - nelec) < 1e-10
        eps = oen.eigenvalues(F, S)
        assert abs(oen.particle_number(eps, w, mu, 10.0, 2.0) - nelec) < 1e-10
    with pytest.raises(native.GreenError):
        native.chemical_potential(F, S, w, 10.0, 12.0, 2.0)  # as many electrons as states


def test_tau_quadrature_is_exact_for_logistic_functions():
    beta = 100.0
    s = synth.make_system(mesh=(1, 1, 1), nao=2, NQ=4, seed=0)
    M = ir.tau_quadrature(s.tau, beta, 1e4)

    def K(t, w):
        return np.exp(-t * w) / (1 + np.exp(-beta * w)) if w >= 0 else np.exp((beta - t) * w) / (1 + np.exp(beta * w))
    for a, b in [(0.3, -0.5), (-0.05, 0.1), (1.5, -2.0)]:
        f = np.array([K(x, a) for x in s.tau])
        g = np.array([K(x, b) for x in s.tau])
        # composite 20-point Gauss-Legendre on 2000 panels: exact to rounding for these exponentials
        x, wq = np.polynomial.legendre.leggauss(20)
        edges = np.linspace(0.0, beta, 2001)
        xs = (0.5 * (edges[1:] - edges[:-1])[:, None] * x[None, :] + 0.5 * (edges[1:] + edges[:-1])[:, None]).ravel()
        ws = (0.5 * (edges[1:] - edges[:-1])[:, None] * wq[None, :]).ravel()
        exact = float(sum(wi * K(xi, a) * K(beta - xi, b) for xi, wi in zip(xs, ws)))
        assert abs(f @ M @ g - exact) < 1e-12 * max(1.0, abs(exact))


@pytest.mark.gpu
def test_energies_match_oracle_and_split_within_1e8():
    s = synth.make_system(mesh=(2, 2, 2), nao=26, NQ=120, ns=1, seed=7, symmetry="tr")
    M = ir.tau_quadrature(s.tau, s.beta, 1e4)
    ctx = native.context_for(s)
    sig64 = ctx.gw_sigma(s.G_tskij, precision=native.PREC_FP64)
    sigsp = ctx.gw_sigma(s.G_tskij, precision=native.PREC_SPLIT)
    e64 = ctx.energy_gw(s.G_tskij, sig64, M)
    ref = oen.e_gw(s, s.G_tskij, ogw.gw_build(s), M)
    assert abs(e64 - ref) < 1e-12 * abs(ref)
    esp = ctx.energy_gw(s.G_tskij, sigsp, M)
    assert abs(esp - e64) < 1e-8 * abs(e64)
    H = s.S_k * 0.3  # any Hermitian one-body term
    F = ctx.hf_fock(s.dm, s.S_k, s.madelung)
    e1, ehf = ctx.energy_hf(s.dm, H, F)
    r1, rhf = oen.e_hf(s, s.dm, H, F)
    assert abs(e1 - r1) < 1e-12 * abs(r1) and abs(ehf - rhf) < 1e-12 * abs(rhf)
    ctx.close()
