"""Checkpoint / restart: a run split by a save and a load continues exactly
like the uninterrupted run."""
import numpy as np
import pytest

import qaxions_b200 as qx
from qaxions_b200 import checkpoint

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_checkpoint_restart_continues_exactly(tmp_path, dtype):
    dt = 0.2 / 32**2
    a = qx.Field(3, 32, dtype=dtype, k0="zero", dt=dt)
    a.ic_config(qx.IC_GRF, 9, 2, 0.01, 0.03)
    a.step(5)
    checkpoint.save(a, str(tmp_path / "c"), k0="zero")
    b = checkpoint.load(str(tmp_path / "c"))
    assert b.curr() == a.curr() and b.time() == a.time()
    a.step(7)
    b.step(7)
    assert np.array_equal(a.psi, b.psi)
    a.close()
    b.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_checkpoint_restart_continues_exactly_in_mre(tmp_path, dtype):
    """An MRE run (scale factor, time step and Poisson prefactor change every
    step) restarts with its cosmology: a, ds and the step/time clock."""
    dt = 0.2 / 32**2
    a = qx.Field(3, 32, dtype=dtype, k0="zero", dt=dt)
    a.set_cosmology(1, 0.1)
    a.ic_config(qx.IC_GRF, 9, 2, 0.01, 0.03)
    a.step(5)
    checkpoint.save(a, str(tmp_path / "m"), k0="zero")
    b = checkpoint.load(str(tmp_path / "m"))
    assert b.cosmology() == a.cosmology()
    assert b.curr() == a.curr() and b.time() == a.time() and b.a() == a.a()
    a.step(7)
    b.step(7)
    assert b.a() == a.a() and b.time() == a.time()
    assert np.array_equal(a.psi, b.psi)
    a.close()
    b.close()
