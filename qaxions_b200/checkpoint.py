"""Checkpoint / restart of a field's state.

The reference's IO::writeConf / readConf (src/io/io.cxx:276-369) store, in
HDF5, a Header group (N, dim, step, time, a, Lbox) and psi as real and
imaginary double datasets in reference site order.  HDF5 is not used here: a
checkpoint is `<path>.json` (the same header fields plus what a restart needs
to rebuild the field: dtype, pref, rho_mean, dt, k0, the cosmology mode and
the current time step ds) and `<path>.psi`
(interleaved complex128, little-endian, reference site order, x fastest).
"""
from __future__ import annotations

import json

import numpy as np

from . import Field

FORMAT = "qaxions_b200 checkpoint 1"


def save(field: Field, path: str, pref: float = 1.0, rho_mean: float = 1.0, k0: str = "reference") -> None:
    """Write `path`.json and `path`.psi.  The physical constants of the field
    (pref, rho_mean, k0) are not readable back from a Field, so the caller
    states them."""
    cosmo, a, ds = field.cosmology()
    hdr = {"format": FORMAT, "N": field.N_, "dim": field.dim_, "step": field.curr(), "time": field.time(),
           "a": a, "Lbox": field.L, "dtype": field.dtype, "pref": pref, "rho_mean": rho_mean,
           "dt": field.dt(), "k0": k0, "cosmo": cosmo, "ds": ds}
    psi = field.psi
    psi.astype("<c16").tofile(path + ".psi")
    with open(path + ".json", "w") as fh:
        json.dump(hdr, fh, indent=1)


def load(path: str, dtype: str | None = None) -> Field:
    """Rebuild the field of a checkpoint (optionally in another dtype)."""
    with open(path + ".json") as fh:
        hdr = json.load(fh)
    if hdr.get("format") != FORMAT:
        raise ValueError(f"{path}.json is not a {FORMAT} file")
    N, dim = int(hdr["N"]), int(hdr["dim"])
    f = Field(dim, N, L=float(hdr["Lbox"]), pref=float(hdr["pref"]), rho_mean=float(hdr["rho_mean"]),
              dtype=dtype or hdr["dtype"], k0=hdr["k0"], dt=float(hdr["dt"]))
    psi = np.fromfile(path + ".psi", dtype="<c16")
    if psi.size != N**dim:
        f.close()
        raise ValueError(f"{path}.psi holds {psi.size} values, expected {N**dim}")
    f.psi = psi.reshape((N,) * dim)
    if int(hdr.get("cosmo", 0)) == 1:
        # MRE: set_cosmology sets rho_mean and the Poisson prefactor's mode and
        # starts a afresh; then the checkpoint's a and ds are put back
        f.set_cosmology(1, float(hdr["a"]))
        f.restore_cosmology(float(hdr["a"]), float(hdr["ds"]))
    f.set_clock(int(hdr["step"]), float(hdr["time"]))
    return f
