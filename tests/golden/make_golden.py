"""Convert the reference's HF test fixtures into a small numpy golden file.

Run in a container where the reference tree is mounted read-only at
``/root/reference`` (it is not needed anywhere else):

    python tests/golden/make_golden.py [/root/reference]

Reads ``test/data/HF/{input.h5,data.h5,df_hf_int/*}``, ``test/data/GW/data.h5`` and
``test/data/HF_X2C/*`` (written to ``hf_x2c_gamma.npz``)
(the inputs of ``solve_hf`` / ``Symmetry_Transform`` in
test/cu_solver_test.cpp:34-96, 343-412) and writes ``hf_h2_27k.npz`` next to
this script.  The file holds the k/q symmetry tables, the stored
density-fitted integrals, G(tau), S_k, the madelung constant, the full-BZ
Fock matrix and the reference results ``result/Sigma1`` and
``result/Sigma_tau``.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from green_gpu_b200.h5lite import H5File  # noqa: E402


def main(ref_root="/root/reference"):
    base = os.path.join(ref_root, "test", "data")
    inp = H5File(os.path.join(base, "HF", "input.h5"))
    dat = H5File(os.path.join(base, "HF", "data.h5"))
    meta = H5File(os.path.join(base, "HF", "df_hf_int", "meta.h5"))
    chunk = int(meta["chunk_size"])
    vq = H5File(os.path.join(base, "HF", "df_hf_int", "VQ_0.h5"))
    raw = vq["/0"]
    V = raw[..., 0::2] + 1j * raw[..., 1::2]  # [kpair][Q][i][j]
    gwd = H5File(os.path.join(base, "GW", "data.h5"))
    gw_vq = H5File(os.path.join(base, "GW", "df_int", "VQ_0.h5"))["/0"]
    gw_V = gw_vq[..., 0::2] + 1j * gw_vq[..., 1::2]

    def cplx(a):
        a = np.asarray(a)
        return a[..., 0] + 1j * a[..., 1]

    out = {
        "nao": int(inp["params/nao"]), "nso": int(inp["params/nso"]), "ns": int(inp["params/ns"]),
        "nk": int(inp["params/nk"]), "NQ": int(inp["params/NQ"]), "ink": int(inp["symmetry/k/ink"]),
        "madelung": float(inp["HF/madelung"]), "chunk_size": chunk,
        "S_k_full": cplx(inp["HF/S-k"]), "Fock_k_full": cplx(inp["HF/Fock-k"]),
        "V_stored": V, "V_stored_gw": gw_V,
        "G_tau": dat["G_tau"], "Sigma1": dat["result/Sigma1"],
        "G_tau_gw": gwd["G_tau"], "Sigma_tau_gw": gwd["result/Sigma_tau"],
        "num_kpair_stored": int(inp["symmetry/pairs/num_kpair_stored"]),
        "conj_pairs_list": inp["symmetry/pairs/conj_pairs_list"],
        "trans_pairs_list": inp["symmetry/pairs/trans_pairs_list"],
        "kpair_irre_list": inp["symmetry/pairs/kpair_irre_list"],
        "kpair_idx": inp["symmetry/pairs/kpair_idx"],
    }
    for kq in ("k", "q"):
        out[f"{kq}_bz2ibz"] = inp[f"symmetry/{kq}/bz2ibz"]
        out[f"{kq}_ibz2bz"] = inp[f"symmetry/{kq}/ibz2bz"]
        out[f"{kq}_tr_conj"] = inp[f"symmetry/{kq}/tr_conj"]
        out[f"{kq}_mesh_scaled"] = inp[f"symmetry/{kq}/mesh_scaled"]
        nst = int(inp[f"symmetry/{kq}/n_stars"])
        stars = [inp[f"symmetry/{kq}/stars/{i}"] for i in range(nst)]
        out[f"{kq}_star_sizes"] = np.array([len(s) for s in stars], np.int64)
        out[f"{kq}_stars"] = np.concatenate(stars).astype(np.int64)
    out["U_k"] = inp["symmetry/k/k_sym_transform_ao"]
    out["U_q"] = inp["symmetry/q/k_sym_transform_p0"]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hf_h2_27k.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes")
    x2c(base)


def x2c(base):
    """HF_X2C fixture (test/cu_solver_test.cpp:335-337 -> solve_hf, :34-96): one k point,
    10 orbitals per spin (nso 20), NQ 154.  Stores the density dm = G_tau[last] (the only
    slice solve_hf reads), S_k, the stored integrals and result/Sigma1."""
    inp = H5File(os.path.join(base, "HF_X2C", "input.h5"))
    dat = H5File(os.path.join(base, "HF_X2C", "data.h5"))
    raw = H5File(os.path.join(base, "HF_X2C", "df_hf_int", "VQ_0.h5"))["/0"]

    def cplx(a):
        a = np.asarray(a)
        return a[..., 0] + 1j * a[..., 1]

    G = dat["G_tau"]
    out = {
        "nao": int(inp["params/nao"]), "nso": int(inp["params/nso"]), "ns": int(inp["params/ns"]),
        "nk": int(inp["params/nk"]), "NQ": int(inp["params/NQ"]), "ink": int(inp["symmetry/k/ink"]),
        "madelung": float(inp["HF/madelung"]), "S_k": cplx(inp["HF/S-k"]),
        "V_stored": raw[..., 0::2] + 1j * raw[..., 1::2], "dm": np.asarray(G[G.shape[0] - 1]),
        "Sigma1": dat["result/Sigma1"],
        "U_k": inp["symmetry/k/k_sym_transform_ao"], "U_q": inp["symmetry/q/k_sym_transform_p0"],
        "k_tr_conj": inp["symmetry/k/tr_conj"], "q_tr_conj": inp["symmetry/q/tr_conj"],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hf_x2c_gamma.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main(*sys.argv[1:])
