"""Density-fitted integral store in the reference's on-disk format.

green-mbpt writes V^Q_ij(k1,k2) for the irreducible k-pairs into HDF5 chunk files
(src/green/gpu/df_integral_t.h:41-258): ``<dir>/meta.h5`` holds ``chunk_size`` (and
``chunk_indices``), ``<dir>/VQ_<c>.h5`` holds dataset ``/<c>`` with shape
[chunk][NQ][nao][2*nao] (interleaved real/imaginary parts) for the pairs c..c+chunk-1 of
the store, in the order of the irreducible k-pair list.  ``read_stored`` returns the whole
store as complex128 [num_kpair_stored][NQ][nao][nao], the array gg_set_coulomb takes
(df_integral_t::read_entire, df_integral_t.h:96-129).
"""
from __future__ import annotations

import os

import numpy as np

from .h5lite import H5File


def read_stored(path: str, nao: int, NQ: int) -> np.ndarray:
    meta = H5File(os.path.join(path, "meta.h5"))
    chunk = int(meta["chunk_size"])
    try:
        starts = sorted(int(c) for c in np.atleast_1d(meta["chunk_indices"]))
    except KeyError:
        starts = sorted(int(f[3:-3]) for f in os.listdir(path) if f.startswith("VQ_") and f.endswith(".h5"))
    parts = []
    for c in starts:
        raw = H5File(os.path.join(path, f"VQ_{c}.h5"))[f"/{c}"]
        if raw.shape[1:] != (NQ, nao, 2 * nao):
            raise ValueError(f"VQ_{c}.h5: shape {raw.shape} does not match NQ={NQ}, nao={nao}")
        parts.append(raw[..., 0::2] + 1j * raw[..., 1::2])
    V = np.ascontiguousarray(np.concatenate(parts, axis=0))
    if chunk <= 0:
        raise ValueError("meta.h5: bad chunk_size")
    return V
