"""GPU: measure() and the measured time loop (src/meas.cxx:13-63,
src/main.cxx:60-85) against the reference build (oracle/_ref), whose loop
ref_run_measured spells out measure()'s computeEnergy + Spectrum dispatch.

The library measures without overwriting V; the reference's measure() leaves
V = |psi|^2 for the kick that follows (a hazard of the reference), which the
library reproduces only under MEAS_CLOBBER_V.  Both are checked against the
matching reference loop."""
import json
import math
import os

import numpy as np
import pytest

import qaxions_b200 as qx
from oracle import ref_lib as R
from oracle import sp_oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref (reference build) not built")]

N, NSTEPS, NMEAS = 32, 20, 5
DT = 0.2 / N**2


def _psi0():
    return O.ic_config("grf+solitons", 3, N, seed=41, n_solitons=3, rc_lo=0.05, rc_hi=0.1)


def _ref(clobber):
    ref = R.RefField(3, N, L=1.0, norm=1.0 / (4.0 * math.pi), dt=DT, nthr=os.cpu_count() or 1)
    ref.set_psi(_psi0())
    out = ref.run_measured(NSTEPS, NMEAS, clobber=clobber, spectrum=True)
    psi = ref.psi()
    ref.close()
    return out, psi


def _read_spec(path):
    with open(path) as fh:
        head = fh.readline()
        assert head.startswith("# a: ")
        assert fh.readline().startswith("# k_phys")
        rows = [ln.split() for ln in fh if ln.strip()]
    return np.array([[float(r[0]), float(r[1]), int(r[2])] for r in rows])


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_measured_run_matches_reference(tmp_path, dtype):
    (rm, curr, tm, P, cnt), psi_ref = _ref(clobber=False)
    tol = 1e-12 if dtype == "c128" else 1e-5
    with qx.Field(3, N, pref=1.0, dtype=dtype, k0="reference", dt=DT) as f:
        f.psi = _psi0()
        recs = f.run(NSTEPS, NMEAS, qx.MEAS_SPECTRUM | qx.MEAS_ENERGY, str(tmp_path))
        psi = f.psi
        assert [r["number"] for r in recs] == list(range(NMEAS + 1))
        assert [r["step"] for r in recs] == list(curr)
        assert [r["time"] for r in recs] == list(tm)
        for r, want in zip(recs, rm):
            assert r["rhomax"] == pytest.approx(want, rel=tol)
            assert math.isfinite(r["mass"]) and math.isfinite(r["energy"])
        # spec_NNNN.txt: the reference's shells and counts, its file layout
        nb = N // 2 + 1
        for m in range(NMEAS + 1):
            got = _read_spec(os.path.join(tmp_path, f"spec_{m:04d}.txt"))
            sel = cnt[m] > 0
            np.testing.assert_array_equal(got[:, 2].astype(np.int64), cnt[m][sel])
            np.testing.assert_allclose(got[:, 1], P[m][sel], rtol=2e-6 if dtype == "c128" else 1e-4,
                                       atol=1e-6 * P[m].max())  # 7 significant digits in the file
            assert len(got) == int(sel.sum()) <= nb
        lines = [json.loads(x) for x in open(os.path.join(tmp_path, "measurements.jsonl"))]
        assert [x["step"] for x in lines] == list(curr)
        assert all("mass" in x for x in lines)
    assert O.rel_l2(psi, psi_ref) < tol
    # measuring does not perturb the run: same state as the unmeasured loop
    with qx.Field(3, N, pref=1.0, dtype=dtype, k0="reference", dt=DT) as g:
        g.psi = _psi0()
        g.step(NSTEPS)
        assert O.rel_l2(psi, g.psi) < (1e-13 if dtype == "c128" else 1e-6)


def test_clobbering_measurements_match_reference_loop():
    """MEAS_CLOBBER_V reproduces the reference's loop bit for bit in
    behaviour: the kick after each measurement uses V = |psi|^2."""
    (rm, curr, tm, P, cnt), psi_ref = _ref(clobber=True)
    with qx.Field(3, N, pref=1.0, dtype="c128", k0="reference", dt=DT) as f:
        f.psi = _psi0()
        recs = f.run(NSTEPS, NMEAS, qx.MEAS_RHO_MAX | qx.MEAS_CLOBBER_V)
        assert [r["step"] for r in recs] == list(curr)
        for r, want in zip(recs, rm):
            assert r["rhomax"] == pytest.approx(want, rel=1e-12)
        assert O.rel_l2(f.psi, psi_ref) < 1e-12
        # the reference's hazard changes the trajectory: the unclobbered run differs
        g = qx.Field(3, N, pref=1.0, dtype="c128", k0="reference", dt=DT)
        g.psi = _psi0()
        g.step(NSTEPS)
        assert O.rel_l2(f.psi, g.psi) > 1e-9
        g.close()


def test_single_measure_and_mre_schedule(tmp_path):
    """measure() alone (number 7, density grid + header) and a measured MRE run
    whose times and scale factors follow updateTime (src/field.cxx:349-361)."""
    with qx.Field(3, 16, pref=1.0, dtype="c128", dt=DT) as f:
        f.psi = O.ic_config("grf", 3, 16, seed=3)
        r = f.measure(qx.MEAS_RHO_GRID | qx.MEAS_ENERGY, 7, str(tmp_path))
        rho = np.fromfile(os.path.join(tmp_path, "field_0007.rho"), dtype=np.float64).reshape((16,) * 3)
        np.testing.assert_allclose(rho, np.abs(f.psi) ** 2, rtol=1e-15)
        hdr = json.load(open(os.path.join(tmp_path, "field_0007.json")))
        assert hdr["N"] == 16 and hdr["dim"] == 3 and hdr["step"] == 0
        assert r["rhomax"] == pytest.approx(float(rho.max() / rho.mean()), rel=1e-13)
        assert r["mass"] == pytest.approx(O.mass(f.psi), rel=1e-12)
        f.set_cosmology(1, 0.1)
        recs = f.run(6, 3, qx.MEAS_RHO_MAX)
        assert [x["step"] for x in recs] == [0, 1, 3, 6]
        assert recs[-1]["a"] == f.a() and recs[-1]["time"] == f.time()
        assert recs[1]["a"] < recs[2]["a"] < recs[3]["a"]
