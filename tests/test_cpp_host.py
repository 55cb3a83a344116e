"""The C++17 host wrapper (include/green_b200.hpp) compiles, links against the library and
drives one GW + HF build whose results match the oracle."""
import os
import subprocess

import numpy as np
import pytest

from green_gpu_b200 import build, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "gw_hf_via_cpp.cpp")


def _compile(out):
    lib = build.build()
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", SRC,
           "-o", out, "-L", os.path.dirname(lib), "-lgreen_b200", "-Wl,-rpath," + os.path.dirname(lib)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_wrapper_compiles(tmp_path):
    _compile(str(tmp_path / "prog"))
    assert os.path.exists(tmp_path / "prog")


@pytest.mark.gpu
def test_cpp_wrapper_runs_gw_and_hf(tmp_path):
    from oracle import gw as ogw
    from oracle import hf as ohf
    prog = str(tmp_path / "prog")
    _compile(prog)
    s = synth.make_system(mesh=(3, 2, 1), nao=5, NQ=12, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=2,
                          symmetry="tr")
    d = str(tmp_path)
    dims = np.array([s.nk, s.ink, s.inq, s.nao, s.NQ, s.ns, s.nts, s.nw_b, s.num_kpair_stored], np.int64)
    files = {"dims": dims, "k_f2r": s.k_full_to_reduced, "k_r2f": s.k_reduced_to_full, "k_tr": s.k_tr_conj,
             "q_f2r": s.q_full_to_reduced, "q_r2f": s.q_reduced_to_full, "q_tr": s.q_tr_conj,
             "k1q": s.k1_from_k2q, "k2q": s.k2_from_k1q, "conj": s.conj_kpair_list, "trans": s.trans_kpair_list,
             "pos": s.irre_pos_kpair}
    for k, v in files.items():
        np.ascontiguousarray(v, np.int64).tofile(os.path.join(d, k + ".bin"))
    for k, v in {"V": s.V_stored, "Ttn": s.Ttn_FB, "Tnt": s.Tnt_BF, "G": s.G_tskij, "dm": s.dm}.items():
        np.ascontiguousarray(v, np.complex128).tofile(os.path.join(d, k + ".bin"))
    r = subprocess.run([prog, d], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    Sigma = np.fromfile(os.path.join(d, "Sigma.bin"), np.complex128).reshape(s.G_tskij.shape)
    K = np.fromfile(os.path.join(d, "K.bin"), np.complex128).reshape(s.dm.shape)
    ref = ogw.gw_build(s)
    assert np.abs(Sigma - ref).max() < 1e-10 * np.abs(ref).max()
    kref = ohf.exchange(s, s.dm)
    assert np.abs(K - kref).max() < 1e-10 * np.abs(kref).max()


def test_drop_in_header_compiles():
    # the green-mbpt drop-in (include/green/gpu/gpu_factory.h) against stand-ins of the green-*,
    # HDF5 and Eigen headers that declare what green-gpu's plugin code uses of them: every call
    # from the drop-in into the C++ wrapper is type-checked
    src = os.path.join(ROOT, "tests", "cpp", "drop_in_compile.cpp")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I",
           os.path.join(ROOT, "tests", "cpp", "stubs"), "-I", os.path.join(ROOT, "include"), src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
