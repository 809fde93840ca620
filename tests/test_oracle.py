"""CPU: pin the NumPy oracle (oracle/sp_oracle.py) to the reference.

The fixtures in tests/golden/ were produced by the reference's own code
(tests/golden/make_golden.py drives oracle/_ref/libqx_ref.so and the
reference's pybind modules built from its sources).  Where that build exists
on this machine the oracle is also compared with it live.
"""
import math
import os

import numpy as np
import pytest

from oracle import ref_lib as R
from oracle import sp_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROWS = O.read_solitons_txt(os.path.join(GOLDEN, "ref_solitons.txt"))
REF = np.load(os.path.join(GOLDEN, "golden_ref.npz"))
PINS = np.load(os.path.join(GOLDEN, "golden_pins.npz"))
PREF = 4.0 * math.pi  # norm = 1 (src/field.cxx:78)
CASES = [(2, 16), (2, 32), (3, 8), (3, 16)]


def _pin_value(kind, n, N, dt, idx):
    """The reference test functions (src/examples/fieldtest.cxx, ictest.cxx)
    restated with the oracle."""
    psi = O.ic_solitons_reference(n, N, ROWS, 1.0)
    if kind in ("ic2d", "ic3d"):
        return psi.ravel()[idx].real
    if kind == "potential":
        return O.update_potential(psi, PREF)[0].ravel()[idx]
    if kind == "kick":
        V, _ = O.update_potential(psi, PREF)
        return O.kick(psi, V, dt).ravel()[idx].real
    if kind == "drift":
        return O.drift(psi, dt).ravel()[idx].real
    if kind == "kdk":
        return O.kdk_step(psi, dt, PREF)[0].ravel()[idx].real
    raise ValueError(kind)


def test_pins_match_reference_tests():
    """Every value the reference's pybind test functions return over the
    parameter grids of tests/test_field.py and tests/test_ic.py."""
    assert len(PINS["value"]) == 64
    for kind, n, N, dt, idx, val in zip(PINS["kind"], PINS["dim"], PINS["N"], PINS["dt"], PINS["idx"],
                                        PINS["value"]):
        got = _pin_value(str(kind), int(n), int(N), float(dt), int(idx))
        assert got == pytest.approx(val, rel=1e-12, abs=1e-13), (kind, n, N, dt, idx)


@pytest.mark.parametrize("dim,N", CASES)
def test_full_arrays_match_reference(dim, N):
    t = f"d{dim}_n{N}"
    psi0 = O.ic_solitons_reference(dim, N, ROWS, 1.0)
    assert O.rel_l2(psi0, REF[t + "_psi0"]) < 1e-14
    psi0 = REF[t + "_psi0"]
    V, vmax = O.update_potential(psi0, PREF)
    assert O.rel_l2(V, REF[t + "_V0"]) < 1e-13
    assert vmax == pytest.approx(float(REF[t + "_Vmax0"]), rel=1e-13)
    assert O.rel_l2(O.kick(psi0, V, 0.05), REF[t + "_psi_kick"]) < 1e-14
    assert O.rel_l2(O.drift(psi0, 0.05), REF[t + "_psi_drift"]) < 1e-14
    assert O.rel_l2(O.kdk_step(psi0, 0.05, PREF)[0], REF[t + "_psi_kdk"]) < 1e-14
    dt = float(REF[t + "_run_dt"])
    psi, Vr = O.run(psi0, dt, 10, PREF)
    assert O.rel_l2(psi, REF[t + "_psi_run"]) < 1e-13
    assert O.rel_l2(Vr, REF[t + "_V_run"]) < 1e-11
    rho, rhomax = O.compute_energy(REF[t + "_psi_run"])
    assert rhomax == pytest.approx(float(REF[t + "_rhomax_run"]), rel=1e-12)
    k, P, c = O.spectrum_reference(rho)
    np.testing.assert_array_equal(c, REF[t + "_spec_count"])
    np.testing.assert_allclose(P, REF[t + "_spec_P"], rtol=1e-11, atol=1e-300)
    np.testing.assert_allclose(k, REF[t + "_spec_k"], rtol=1e-15)


@pytest.mark.parametrize("dim,N", CASES)
def test_fft_conventions_match_reference(dim, N):
    t = f"d{dim}_n{N}"
    assert O.rel_l2(np.fft.fftn(REF[t + "_fft_in"]), REF[t + "_fft_fwd"]) < 1e-14
    assert O.rel_l2(np.fft.rfftn(REF[t + "_r2c_in"]), REF[t + "_r2c_out"]) < 1e-14


def test_spectrum_tables_exact_counts():
    """Binned counts equal the number of weighted half-spectrum modes."""
    for dim, N in [(2, 32), (3, 16)]:
        for mode, nb in [(O.SPEC_REFERENCE, 0), (O.SPEC_LINEAR, 8), (O.SPEC_LOG, 6)]:
            x = np.ones((N,) * dim)
            _, _, cnt = O.spectrum_binned(np.fft.rfftn(x), dim, N, mode, nb)
            tab = O.spectrum_bin_table(dim, N, mode, nb)
            M = O.k2_int(dim, N, half=True)
            ix = np.arange(N // 2 + 1)
            w = np.broadcast_to(np.where((ix == 0) | (ix == N // 2), 1, 2), M.shape)
            assert cnt.sum() == w[tab[M] >= 0].sum()


def test_ic_fixtures_reproducible():
    ic = np.load(os.path.join(GOLDEN, "golden_ic.npz"))
    for dim, N in [(2, 32), (3, 16)]:
        t = f"d{dim}_n{N}"
        np.testing.assert_allclose(
            O.ic_config("solitons", dim, N, 1234, n_solitons=8, rc_lo=0.02, rc_hi=0.05), ic[t + "_solitons"],
            rtol=0, atol=1e-13)
        np.testing.assert_allclose(O.ic_config("grf", dim, N, 1234), ic[t + "_grf"], rtol=0, atol=1e-13)
        psi = ic[t + "_grf"]
        assert np.mean(np.abs(psi) ** 2) == pytest.approx(1.0, rel=1e-13)


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors published with the Random123
    distribution (kat_vectors: counter/key all zero, and all ones)."""
    r = O.philox4x32(np.array([0], np.uint32), np.array([0], np.uint32), np.array([0], np.uint32),
                     np.array([0], np.uint32), 0, 0)
    assert [int(x[0]) for x in r] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    m = np.array([0xFFFFFFFF], np.uint32)
    r = O.philox4x32(m, m, m, m, 0xFFFFFFFF, 0xFFFFFFFF)
    assert [int(x[0]) for x in r] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


@pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")
def test_live_reference_matches_oracle(soliton_dir):
    for dim, N in [(2, 12), (3, 12), (2, 96)]:
        f = R.RefField(dim, N, 1.0, 1.0, 0.01)
        f.ic_solitons(1.0)
        psi0 = f.psi()
        f.run(5)
        psi, V = O.run(psi0, 0.01, 5, PREF)
        assert O.rel_l2(psi, f.psi()) < 1e-13
        f.close()


def test_mre_restatement_matches_reference_golden():
    """The MRE merged loop of the restatement against the reference's own run."""
    d = np.load(os.path.join(GOLDEN, "golden_mre.npz"))
    for tag in ("d2_n32", "d3_n16"):
        psi, a, n = O.run_mre(d[f"{tag}_psi0"], float(d[f"{tag}_dt"]), float(d[f"{tag}_ai"]), 10)
        assert abs(a - float(d[f"{tag}_a_run"])) <= 1e-15
        assert n == int(d[f"{tag}_curr_run"])
        assert O.rel_l2(psi, d[f"{tag}_psi_run"]) <= 1e-12
