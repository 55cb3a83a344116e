"""CPU FP64 oracle for the HF-exchange / GW self-energy path.

TEST INFRASTRUCTURE ONLY.  This package restates the reference's algorithm
(Green-Phys/green-gpu) in numpy so that the CUDA implementation can be checked
against it.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import it; the product path never does.

Every function cites the reference file:line whose arithmetic it restates.
Pinned against the reference's own golden vectors (``tests/golden/``):
HF ``result/Sigma1`` (test/cu_solver_test.cpp:34-96, tol 1e-8) and the
symmetry round trip of ``HF/Fock-k`` (test/cu_symmetry_test.cu:38-130).
The GW golden ``result/Sigma_tau`` needs green-grids' IR file, which the
reference does not ship, so the GW restatement is pinned through identities
(Hermiticity, P0(beta - tau) = P0(tau), symmetry-reduced == unreduced).
"""
