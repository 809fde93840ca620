"""``pyqaxions.fieldtest`` on the B200 (src/examples/fieldtest.cxx:11-105).

Each function builds a field the way the reference does -- defaults()
(src/parse.cxx:7-29) with N, dim and norm = 1, i.e. pref = 4 pi norm a = 4 pi
(src/field.cxx:78,298) and rho_mean = 1 -- applies the Gaussian-soliton IC read
from ``solitons.txt`` in the current directory (src/ic/solitons.cxx:32), runs
one operation and returns Re psi[idx] (or V[idx]).  ``dtype`` selects the plain
FP64 ("c128", default) or fused FP32 ("c64") form; ``path`` overrides the
soliton file.
"""
from __future__ import annotations

import math

from .. import Field

_NORM = 1.0
_BKG = 1.0  # Params::sol_bkg default (src/parse.cxx:20)


def _field(n: int, N: int, dtype: str, path: str) -> Field:
    f = Field(n, N, L=1.0, pref=4.0 * math.pi * _NORM, rho_mean=1.0, dtype=dtype, dt=1e-4)
    f.ic_solitons_file(path, _BKG)
    return f


def test_kick(n: int, N: int, dt: float, idx: int, dtype: str = "c128", path: str = "solitons.txt") -> float:
    """updatePotential; kick(dt) -> Re psi[idx]   (src/examples/fieldtest.cxx:11-30)."""
    with _field(n, N, dtype, path) as f:
        f.updatePotential()
        f.kick(dt)
        return f.getPsiIdx(idx)


def test_drift(n: int, N: int, dt: float, idx: int, dtype: str = "c128", path: str = "solitons.txt") -> float:
    """drift(dt) -> Re psi[idx]   (src/examples/fieldtest.cxx:32-50)."""
    with _field(n, N, dtype, path) as f:
        f.drift(dt)
        return f.getPsiIdx(idx)


def test_potential(n: int, N: int, idx: int, dtype: str = "c128", path: str = "solitons.txt") -> float:
    """updatePotential -> V[idx]   (src/examples/fieldtest.cxx:53-71)."""
    with _field(n, N, dtype, path) as f:
        f.updatePotential()
        return f.getVIdx(idx)


def test_kick_drift_step(n: int, N: int, dt: float, idx: int, dtype: str = "c128",
                         path: str = "solitons.txt") -> float:
    """updatePotential; kick(dt/2); drift(dt); updatePotential; kick(dt/2)
    -> Re psi[idx]   (src/examples/fieldtest.cxx:73-96)."""
    with _field(n, N, dtype, path) as f:
        f.updatePotential()
        f.kick(0.5 * dt)
        f.drift(dt)
        f.updatePotential()
        f.kick(0.5 * dt)
        return f.getPsiIdx(idx)
