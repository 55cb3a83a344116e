"""Load ``hf_h2_27k.npz`` (made by ``make_golden.py``) as a ``green_gpu_b200.synth.System``."""
import os

import numpy as np

from green_gpu_b200.synth import System

HERE = os.path.dirname(os.path.abspath(__file__))


def _mesh_index(mesh_scaled):
    keys = {tuple(np.round(np.mod(m, 1.0) * 1e6).astype(np.int64) % 1000000): i for i, m in enumerate(mesh_scaled)}

    def find(v):
        return keys[tuple(np.round(np.mod(v, 1.0) * 1e6).astype(np.int64) % 1000000)]
    return find


def load(path=None, gw=False, nw_b=None):
    d = np.load(path or os.path.join(HERE, "hf_h2_27k.npz"))
    nk, ink, NQ, nao, ns = int(d["nk"]), int(d["ink"]), int(d["NQ"]), int(d["nao"]), int(d["ns"])
    ibz2bz = d["k_ibz2bz"].astype(np.int64)
    pos = {int(k): i for i, k in enumerate(ibz2bz)}
    f2r = np.array([pos[int(b)] for b in d["k_bz2ibz"]], np.int64)
    qibz2bz = d["q_ibz2bz"].astype(np.int64)
    qpos = {int(k): i for i, k in enumerate(qibz2bz)}
    qf2r = np.array([qpos[int(b)] for b in d["q_bz2ibz"]], np.int64)

    def stars(kq):
        sizes = d[f"{kq}_star_sizes"]
        flat = d[f"{kq}_stars"]
        out, o = [], 0
        for s in sizes:
            out.append(flat[o:o + s].astype(np.int64))
            o += s
        return out

    mesh = d["k_mesh_scaled"]
    find = _mesh_index(mesh)
    k1_from_k2q = np.array([find(mesh[k] + mesh[q]) for k in range(nk) for q in range(nk)], np.int64)
    k2_from_k1q = np.array([find(mesh[k] - mesh[q]) for k in range(nk) for q in range(nk)], np.int64)
    npairs = nk * (nk + 1) // 2
    irre_pos = -np.ones(npairs, np.int64)
    irre_pos[d["kpair_irre_list"]] = np.arange(len(d["kpair_irre_list"]))
    G = d["G_tau_gw"] if gw else d["G_tau"]
    nts = G.shape[0]
    S_ibz = d["S_k_full"][:, ibz2bz]
    sys_ = System(
        nk=nk, ink=ink, nq=nk, inq=len(qibz2bz), nao=nao, NQ=NQ, ns=ns, nts=nts,
        nw_b=int(nw_b or 0), beta=100.0,
        k_full_to_reduced=f2r, k_reduced_to_full=ibz2bz, k_tr_conj=d["k_tr_conj"].astype(np.int64),
        k_stars=stars("k"),
        q_full_to_reduced=qf2r, q_reduced_to_full=qibz2bz, q_tr_conj=d["q_tr_conj"].astype(np.int64),
        q_stars=stars("q"), k1_from_k2q=k1_from_k2q, k2_from_k1q=k2_from_k1q,
        U_k=d["U_k"].copy(), U_q=d["U_q"].copy(),
        conj_kpair_list=d["conj_pairs_list"].astype(np.int64),
        trans_kpair_list=d["trans_pairs_list"].astype(np.int64), irre_pos_kpair=irre_pos,
        V_stored=np.ascontiguousarray(d["V_stored_gw"] if gw else d["V_stored"]),
        G_tskij=np.ascontiguousarray(G), Ttn_FB=np.zeros((nts, 0), np.complex128),
        Tnt_BF=np.zeros((0, nts - 2), np.complex128), S_k=np.ascontiguousarray(S_ibz),
        madelung=float(d["madelung"]),
        meta={"fixture": "H2 3x3x3 (reference test/data/HF)"},
    )
    ref = {"Sigma1": d["Sigma1"], "Fock_k_full": d["Fock_k_full"], "Sigma_tau_gw": d["Sigma_tau_gw"]}
    return sys_, ref


def load_x2c(path=None):
    """``hf_x2c_gamma.npz``: the reference's HF_X2C fixture (one k point, identity symmetry) as a
    System with nao = orbitals per spin and ns = 1, plus dm [1][1][2n][2n] and Sigma1."""
    d = np.load(path or os.path.join(HERE, "hf_x2c_gamma.npz"))
    nk, NQ, nao = int(d["nk"]), int(d["NQ"]), int(d["nao"])
    assert nk == 1 and int(d["ink"]) == 1
    # the stored transforms are identities: the identity symmetry is used
    assert np.allclose(d["U_k"][0], np.eye(2 * nao)) and np.allclose(d["U_q"][0], np.eye(NQ))
    assert not np.any(d["k_tr_conj"]) and not np.any(d["q_tr_conj"])
    one = np.zeros(1, np.int64)
    sys_ = System(
        nk=1, ink=1, nq=1, inq=1, nao=nao, NQ=NQ, ns=1, nts=4, nw_b=0, beta=100.0,
        k_full_to_reduced=one, k_reduced_to_full=one, k_tr_conj=one, k_stars=[one],
        q_full_to_reduced=one, q_reduced_to_full=one, q_tr_conj=one, q_stars=[one],
        k1_from_k2q=one, k2_from_k1q=one, U_k=None, U_q=None,
        conj_kpair_list=one, trans_kpair_list=one, irre_pos_kpair=one,
        V_stored=np.ascontiguousarray(d["V_stored"]), G_tskij=np.zeros((4, 1, 1, 2 * nao, 2 * nao), np.complex128),
        Ttn_FB=np.zeros((4, 0), np.complex128), Tnt_BF=np.zeros((0, 2), np.complex128),
        S_k=np.ascontiguousarray(d["S_k"]), madelung=float(d["madelung"]),
        meta={"fixture": "X2C, one k point (reference test/data/HF_X2C)"},
    )
    return sys_, {"dm": np.ascontiguousarray(d["dm"]), "Sigma1": d["Sigma1"]}
