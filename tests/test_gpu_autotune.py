"""Autotuner: chooses a launch geometry -- including the radix plan of the
strided passes -- without disturbing the state, caches the choice per (dim,
N, dtype, batch) in the process and in a file, and fields created later start
from the cached choice."""
import numpy as np
import pytest

import qaxions_b200 as qx
from oracle import sp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fresh_tune_cache():
    """Tuned choices stay in this test: later tests' fields start from defaults."""
    qx.clear_tune_cache()
    yield
    qx.clear_tune_cache()


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
    chosen = f.get_tune()
    # a field created afterwards starts from the cached geometry
    g = qx.Field(3, 64, dtype=dtype, k0="zero", dt=0.2 / 64**2)
    t = g.get_tune()
    assert t["from_cache"] == 1
    assert {k: t[k] for k in t if k != "from_cache"} == {k: chosen[k] for k in chosen if k != "from_cache"}
    # the tuned geometry steps like the default one
    g.set_tune()
    g.set_plan(0)
    g.set_pencil_warp(False)
    g.ic_config(qx.IC_GRF, 3, 2, 0.01, 0.03)
    f.step(5)
    g.step(5)
    tol = 1e-12 if dtype == "c128" else 1e-5
    assert np.linalg.norm(f.psi - g.psi) / np.linalg.norm(g.psi) < tol
    lines = open(path).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith(f"v3 3 64 {dtype} 1 : ")
    assert len(lines[0].split(" : ")[1].split()) == 9  # x_rows y_tx la_tx tma nbuf pw plan wp ms
    f.close()
    g.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("dim,N", [(3, 64), (3, 96), (3, 128), (2, 256), (3, 256)])
def test_radix_plan1_steps_like_plan0(dim, N, dtype):
    """Radix plan 1 (the default plan's radices in reverse order) of the
    strided passes: same transforms, other rounding; the FP64 form also
    against the oracle."""
    dt = 0.2 / N**2
    n = 4 if N < 256 else 2
    psi0 = O.ic_config("grf+solitons", dim, N, seed=5, n_solitons=2, rc_lo=0.05, rc_hi=0.1)
    outs = []
    for plan in (0, 1):
        with qx.Field(dim, N, pref=1.0, dtype=dtype, dt=dt) as f:
            f.set_plan(plan)
            assert f.get_tune()["plan"] == plan
            f.psi = psi0
            f.step(n)
            outs.append((f.psi, f.spectrum(0, qx.SPEC_REFERENCE)[1], f.mass_energy()[0]))
    tol = 1e-13 if dtype == "c128" else 2e-6
    assert O.rel_l2(outs[1][0], outs[0][0]) < tol
    assert O.rel_l2(outs[1][1], outs[0][1]) < 100 * tol
    if dtype == "c128" and N <= 128:
        ref, _ = O.run(psi0, dt, n, 1.0)
        assert O.rel_l2(outs[1][0], ref) < 1e-12


def test_plan1_where_absent_runs_plan0():
    """512 = 8 x 8 x 8 has no other order: plan 1 runs as plan 0, bit for bit."""
    outs = []
    for plan in (0, 1):
        with qx.Field(3, 512, pref=1.0, dtype="c64", dt=0.2 / 512**2) as f:
            f.set_plan(plan)
            f.ic_config(qx.IC_GRF, 9, 0)
            f.step(1)
            outs.append(f.psi)
    assert np.array_equal(outs[0], outs[1])


def test_autotune_chooses_among_radix_plans(tmp_path):
    f = qx.Field(3, 96, dtype="c64", k0="zero", dt=0.2 / 96**2)
    f.ic_config(qx.IC_GRF, 3, 0)
    ms, cached = f.autotune(2, cache=str(tmp_path / "t96.txt"))
    assert ms > 0 and not cached
    assert f.get_tune()["plan"] in (0, 1)
    f.close()
