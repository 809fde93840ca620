"""One warp per pencil pair (qx_set_pencil_warp): the FP32 strided passes at
N = 256 and 512 in 16-column swizzled tiles with warp-local stage exchanges run
the same butterflies, twiddles and phase factors as the default passes, so the
state agrees with theirs to FP32 round-off (bit for bit where the compiler
fuses the same multiply-adds) -- through the step's graph, the reference-
surface drift and potential, the kinetic-energy pass and 2D fields (column-0
mirror in the last-axis Poisson pass)."""
import numpy as np
import pytest

import qaxions_b200 as qx
from oracle import sp_oracle as O

pytestmark = pytest.mark.gpu


def _run(dim, N, wp, steps, seed=77, row_stage=0):
    f = qx.Field(dim, N, pref=1.0, dtype="c64", k0="reference", dt=0.2 / N**2)
    f.set_pencil_warp(wp)
    f.set_row_stage(row_stage)
    assert f.get_tune()["pencil_warp"] == wp
    assert f.get_tune()["row_stage"] == row_stage
    f.ic_config(qx.IC_GRF, seed, 4, 0.02, 0.05)
    f.step(steps)
    psi = f.psi
    f.drift(0.1 / N**2)
    f.updatePotential()
    out = (psi, f.psi, f.V, f.mass_energy(), f.spectrum(0, qx.SPEC_REFERENCE)[1])
    f.close()
    return out


@pytest.mark.parametrize("wp", [1, 2])
@pytest.mark.parametrize("dim,N,steps", [(3, 256, 4), (3, 512, 2), (2, 256, 6), (2, 512, 6)])
def test_pencil_warp_matches_default_passes(dim, N, steps, wp):
    a = _run(dim, N, 0, steps)
    b = _run(dim, N, wp, steps)
    assert np.isfinite(b[0]).all()
    assert O.rel_l2(b[0], a[0]) < 2e-7
    assert O.rel_l2(b[1], a[1]) < 2e-7
    assert O.rel_l2(b[2] - b[2].mean(), a[2] - a[2].mean()) < 1e-6
    assert b[3][0] == pytest.approx(a[3][0], rel=1e-6)  # mass
    assert b[3][2] == pytest.approx(a[3][2], rel=1e-5)  # kinetic energy
    assert O.rel_l2(b[4], a[4]) < 1e-5


def test_pencil_warp_against_fp64_oracle():
    """3D 256^3, 5 merged steps with the warp passes against the FP64 form."""
    N, n = 256, 5
    dt = 0.2 / N**2
    with qx.Field(3, N, pref=1.0, dtype="c128", dt=dt) as g:
        g.ic_config(qx.IC_GRF, 3, 8, 0.02, 0.05)
        psi0 = g.psi
        g.step(n)
        ref = g.psi
    with qx.Field(3, N, pref=1.0, dtype="c64", dt=dt) as f:
        f.set_pencil_warp(2)
        f.psi = psi0
        f.step(n)
        assert O.rel_l2(f.psi, ref) < 1e-5


@pytest.mark.parametrize("wp", [3, 4])
@pytest.mark.parametrize("dim,N,steps", [(3, 512, 2), (2, 512, 6)])
def test_two_warps_per_pencil_pair_bitwise(dim, N, steps, wp):
    """wp 3 / 4: the drift pass / every wave-function pass with a pencil pair
    split over two warps (8 values of each pencil per thread, pair barriers):
    the same butterflies on the same operands, so bit for bit the one-warp
    passes."""
    a = _run(dim, N, 1, steps)
    b = _run(dim, N, wp, steps)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]


@pytest.mark.parametrize("dim,N,steps", [(3, 512, 2), (3, 256, 3), (2, 512, 6)])
def test_staged_row_pass_bitwise(dim, N, steps):
    """Row stage 1: the inverse x + density + r2c pass reads each row from a
    shared-memory copy made by cp.async one row ahead -- the same values in the
    same registers, so bit for bit the direct-load pass."""
    a = _run(dim, N, 3 if N == 512 else 1, steps, row_stage=0)
    b = _run(dim, N, 3 if N == 512 else 1, steps, row_stage=1)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]
