"""Ensemble of independent boxes (batched groups, one persistent launch per pass
over all boxes of a size): every box must evolve exactly as the same box run
alone through the single-box path, with the same seed."""
import numpy as np
import pytest

import qaxions_b200 as qx
from oracle import sp_oracle as O

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-13, "c64": 1e-6}


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("dim,groups,mixed", [(3, [(16, 2), (96, 2), (32, 3)], False),
                                              (3, [(16, 2), (96, 2), (32, 3)], True),
                                              (3, [(16, 2), (96, 2), (32, 3)], "passes"),
                                              (2, [(64, 3), (128, 2)], False)])
def test_ensemble_boxes_match_single_boxes(dim, groups, mixed, dtype):
    dt = 0.2 / max(n for n, _ in groups) ** 2
    ens = qx.Ensemble(groups, dim=dim, dtype=dtype, dt=dt, mixed=mixed)
    ens.ic_config(qx.IC_GRF, seed_base=1234, n_sol=2)
    ens.step(6)
    b = 0
    for n, c in groups:
        for _ in range(c):
            f = qx.Field(dim, n, dtype=dtype, k0="zero", dt=dt)
            f.ic_config(qx.IC_GRF, 1234 + b, 2, 0.01, 0.03)
            f.step(6)
            err = O.rel_l2(ens.psi(b), f.psi)
            assert err <= TOL[dtype], (n, b, err)
            f.close()
            b += 1
    m = ens.mass()
    assert m.shape == (b,)
    assert np.allclose(m, 1.0, rtol=1e-5 if dtype == "c64" else 1e-12)
    ens.close()


def test_ensemble_timing_and_errors():
    ens = qx.Ensemble([(32, 2), (64, 1)], dtype="c64")
    ens.ic_config(qx.IC_GRF, seed_base=7)
    ens.step(2)
    ms = ens.time_steps(4)
    assert ms > 0.0
    with pytest.raises(ValueError):
        ens.psi(3)
    with pytest.raises(ValueError):
        qx.Ensemble([(33, 1)])
    ens.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("mixed", [False, True, "passes"])
def test_ensemble_graph_replays_across_calls(dtype, mixed):
    """The loop bodies of all groups replay as one graph per step; calls of
    different lengths in a row (graph reused, and the 1- and 2-step calls that
    need no graph) leave every box as its single-box run with the same calls."""
    groups = [(32, 2), (96, 1), (64, 1)]
    dt = 0.2 / 96**2
    calls = (5, 1, 2, 7)
    ens = qx.Ensemble(groups, dtype=dtype, dt=dt, mixed=mixed)
    ens.ic_config(qx.IC_GRF, seed_base=40, n_sol=1)
    for n in calls:
        ens.step(n)
    b = 0
    for n, c in groups:
        for _ in range(c):
            f = qx.Field(3, n, dtype=dtype, k0="zero", dt=dt)
            f.ic_config(qx.IC_GRF, 40 + b, 1, 0.01, 0.03)
            for k in calls:
                f.step(k)
            assert O.rel_l2(ens.psi(b), f.psi) <= TOL[dtype], (n, b)
            f.close()
            b += 1
    ens.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("mixed", [True, "passes"])
def test_mixed_passes_match_per_size_passes(dtype, mixed):
    """The loop body as one launch per step (or per pass) over the boxes of all
    sizes against the per-size launches on concurrent graph branches: the C4
    sizes 64, 96 (radix 3) and 128, 16 boxes of 64^3 (the queue's cheap tail),
    and mode switches between calls."""
    groups = [(64, 16), (96, 2), (128, 2)]
    dt = 0.2 / 128**2
    a = qx.Ensemble(groups, dtype=dtype, dt=dt, mixed=False)
    b = qx.Ensemble(groups, dtype=dtype, dt=dt, mixed=mixed)
    for e in (a, b):
        e.ic_config(qx.IC_GRF, seed_base=500, n_sol=2)
    a.step(8)
    b.step(8)
    b.set_mixed(False)
    b.step(4)
    b.set_mixed("passes" if mixed is True else True)
    b.step(5)
    a.step(9)
    for box in range(a.nboxes):
        err = O.rel_l2(b.psi(box), a.psi(box))
        assert err <= TOL[dtype], (box, err)
    assert np.allclose(a.mass(), b.mass(), rtol=1e-13 if dtype == "c128" else 1e-6)
    a.close()
    b.close()


@pytest.mark.parametrize("window", [1, 20 << 20, 1 << 40])
def test_mixed_step_windows(window):
    """The one-launch step's queue windows: one box per window, a few boxes per
    window (windows that start and end inside a size group) and all boxes in
    one window (pass-by-pass order) advance the boxes as the per-size path."""
    groups = [(64, 5), (96, 3), (128, 2)]
    dt = 0.2 / 128**2
    a = qx.Ensemble(groups, dtype="c64", dt=dt, mixed=False)
    b = qx.Ensemble(groups, dtype="c64", dt=dt, mixed=True)
    b.set_mixed_window(window)
    for e in (a, b):
        e.ic_config(qx.IC_GRF, seed_base=900, n_sol=1)
        e.step(6)
    for box in range(a.nboxes):
        assert O.rel_l2(b.psi(box), a.psi(box)) <= TOL["c64"], box
    a.close()
    b.close()


def test_mixed_mode_rejects_what_it_does_not_cover():
    e2 = qx.Ensemble([(32, 1), (64, 1)], dim=2)
    with pytest.raises(ValueError):
        e2.set_mixed(True)
    e2.close()
    big = qx.Ensemble([(256, 1), (64, 1)])  # N = 256 has no mixed-size unit
    with pytest.raises(ValueError):
        big.set_mixed(True)
    big.close()
    many = qx.Ensemble([(16, 1), (32, 1), (64, 1), (96, 1), (128, 1)])
    with pytest.raises(ValueError):
        many.set_mixed(True)
    many.close()
