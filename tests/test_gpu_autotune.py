"""Autotuner: chooses a launch geometry without disturbing the state, caches
the choice per (dim, N, dtype, batch) in the process and in a file."""
import numpy as np
import pytest

import qaxions_b200 as qx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["c64", "c128"])
def test_autotune_keeps_state_and_caches(tmp_path, dtype):
    path = str(tmp_path / "tune.txt")
    f = qx.Field(3, 64, dtype=dtype, k0="zero", dt=0.2 / 64**2)
    f.ic_config(qx.IC_GRF, 3, 2, 0.01, 0.03)
    psi0 = f.psi
    ms, cached = f.autotune(2, cache=path)
    assert ms > 0 and not cached
    assert np.array_equal(f.psi, psi0)
    ms2, cached2 = f.autotune(2, cache=path)
    assert cached2 and ms2 == ms
    # the tuned geometry steps like the default one
    g = qx.Field(3, 64, dtype=dtype, k0="zero", dt=0.2 / 64**2)
    g.ic_config(qx.IC_GRF, 3, 2, 0.01, 0.03)
    f.step(5)
    g.step(5)
    tol = 1e-12 if dtype == "c128" else 1e-5
    assert np.linalg.norm(f.psi - g.psi) / np.linalg.norm(g.psi) < tol
    lines = open(path).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith(f"3 64 {dtype} 1 : ")
    f.close()
    g.close()
