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
@pytest.mark.parametrize("dim,groups", [(3, [(16, 2), (96, 2), (32, 3)]), (2, [(64, 3), (128, 2)])])
def test_ensemble_boxes_match_single_boxes(dim, groups, dtype):
    dt = 0.2 / max(n for n, _ in groups) ** 2
    ens = qx.Ensemble(groups, dim=dim, dtype=dtype, dt=dt)
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
def test_ensemble_graph_replays_across_calls(dtype):
    """The loop bodies of all groups replay as one graph per step; calls of
    different lengths in a row (graph reused, and the 1- and 2-step calls that
    need no graph) leave every box as its single-box run with the same calls."""
    groups = [(32, 2), (96, 1), (64, 1)]
    dt = 0.2 / 96**2
    calls = (5, 1, 2, 7)
    ens = qx.Ensemble(groups, dtype=dtype, dt=dt)
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
