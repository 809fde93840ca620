"""``pyqaxions.ictest`` on the B200 (src/examples/ictest.cxx:8-50): the
Gaussian-soliton IC of src/ic/solitons.cxx:20-110 read from ``solitons.txt``
in the current directory, returning Re psi[idx]."""
from __future__ import annotations

from .fieldtest import _field


def test_solitons(N: int, idx: int, dtype: str = "c128", path: str = "solitons.txt") -> float:
    """2D IC -> Re psi[idx]   (src/examples/ictest.cxx:8-25)."""
    with _field(2, N, dtype, path) as f:
        return f.getPsiIdx(idx)


def test_solitons_3D(N: int, idx: int, dtype: str = "c128", path: str = "solitons.txt") -> float:
    """3D IC -> Re psi[idx]   (src/examples/ictest.cxx:27-42)."""
    with _field(3, N, dtype, path) as f:
        return f.getPsiIdx(idx)
