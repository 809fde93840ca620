"""Drift chain: the y forward, z drift and y inverse passes of a 3D complex64
field run as one kernel over x-slabs (qx_set_chain).  Each tile gets the same
arithmetic in the same element order as in the three separate passes, so the
state must match theirs bit for bit -- through the step's CUDA graph, the
reference-surface drift operator, and batched ensembles."""
import numpy as np
import pytest

import qaxions_b200 as qx

pytestmark = pytest.mark.gpu


def _run(N, chain, steps, seed=4321):
    f = qx.Field(3, N, dtype="c64", k0="zero", dt=0.2 / N**2)
    f.set_pencil_warp(0)  # the chain reproduces the 8-column passes bit for bit
    f.set_chain(chain)
    f.ic_config(qx.IC_GRF, seed, 4, 0.01, 0.03)
    f.step(steps)
    psi = f.psi.copy()
    f.drift(0.1 / N**2)
    psi_d = f.psi.copy()
    f.close()
    return psi, psi_d


@pytest.mark.parametrize("N", [16, 32, 64, 96, 128, 256, 512])
def test_chain_matches_separate_passes_bitwise(N):
    steps = 2 if N == 512 else 5
    b, bd = _run(N, 0, steps)
    for sw in (1, 2):  # slabs of 8 / 16 columns
        if N % (8 * sw):
            continue
        a, ad = _run(N, sw, steps)
        assert np.isfinite(a).all()
        assert np.array_equal(a, b), sw
        assert np.array_equal(ad, bd), sw


def test_chain_repeated_steps_and_toggle():
    """Counters are reset per launch: many graph replays in a row, and a field
    switched between the two paths mid-run, stay bit-identical."""
    N = 64
    f = qx.Field(3, N, dtype="c64", k0="zero", dt=0.2 / N**2)
    g = qx.Field(3, N, dtype="c64", k0="zero", dt=0.2 / N**2)
    g.set_chain(False)
    for h in (f, g):
        h.ic_config(qx.IC_GRF, 99, 3, 0.01, 0.03)
    # the same calls on both (each step() call has its own half-kick ends)
    f.step(40)
    f.set_chain(False)
    f.step(3)
    f.set_chain(1)
    f.step(7)
    for n in (40, 3, 7):
        g.step(n)
    assert np.array_equal(f.psi, g.psi)
    f.set_chain(2)
    g.step(9)
    f.step(9)
    assert np.array_equal(f.psi, g.psi)
    f.close()
    g.close()
