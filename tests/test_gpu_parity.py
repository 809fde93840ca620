"""GPU parity: the sm_100a path (through the C ABI) against the reference.

Reference data: tests/golden/ (generated from the reference's own code) and
the NumPy oracle (oracle/sp_oracle.py, itself pinned by tests/test_oracle.py).
Tolerances (relative L2 unless stated):
  plain FP64 form (c128): <= 1e-12 against the FP64 reference/oracle
  fused FP32 form (c64):  <= 2e-6 for one operation, <= 1e-5 after a run,
                          and the reference tests' own abs 1e-5 / rel 1e-4 pins
"""
import math
import os

import numpy as np
import pytest

import pyqaxions.fieldtest as fieldtest  # the reference tests' own import (tests/test_field.py:8)
import pyqaxions.ictest as ictest  # (tests/test_ic.py:8)
import qaxions_b200 as qx
from oracle import sp_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF = np.load(os.path.join(GOLDEN, "golden_ref.npz"))
PINS = np.load(os.path.join(GOLDEN, "golden_pins.npz"))
ICS = np.load(os.path.join(GOLDEN, "golden_ic.npz"))
PREF = 4.0 * math.pi
CASES = [(2, 16), (2, 32), (3, 8), (3, 16)]
TOL1 = {"c128": 1e-12, "c64": 2e-6}


def v_err(Vg, Vr, dtype):
    """relL2 of a potential.  The reference divides the k = 0 Poisson mode by 1
    (src/field.cxx:253,282), which adds the constant -pref (<rho> - rho_mean)
    to V; in FP32 <rho> - 1 is a rounding residue (~1e-7), so the FP32 form is
    compared up to that constant (a global phase of psi)."""
    if dtype == "c128":
        return O.rel_l2(Vg, Vr)
    return O.rel_l2(Vg - Vg.mean(), Vr - Vr.mean())


def _call_pin(kind, n, N, dt, idx, dtype):
    if kind == "potential":
        return fieldtest.test_potential(n, N, idx, dtype=dtype)
    if kind == "kick":
        return fieldtest.test_kick(n, N, dt, idx, dtype=dtype)
    if kind == "drift":
        return fieldtest.test_drift(n, N, dt, idx, dtype=dtype)
    if kind == "kdk":
        return fieldtest.test_kick_drift_step(n, N, dt, idx, dtype=dtype)
    if kind == "ic2d":
        return ictest.test_solitons(N, idx, dtype=dtype)
    return ictest.test_solitons_3D(N, idx, dtype=dtype)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_reference_test_surface(soliton_dir, dtype):
    """The reference's own pybind test functions, same arguments, same values
    (tests/test_field.py:12-129, tests/test_ic.py:12-37): the pybind11 modules
    pyqaxions.fieldtest / pyqaxions.ictest of this library, imported under the
    reference's names, at every grid point of the reference's tests, against
    the values the reference's own modules return (tests/golden/golden_pins.npz)."""
    for kind, n, N, dt, idx, val in zip(PINS["kind"], PINS["dim"], PINS["N"], PINS["dt"], PINS["idx"],
                                        PINS["value"]):
        got = _call_pin(str(kind), int(n), int(N), float(dt), int(idx), dtype)
        if dtype == "c128":
            assert got == pytest.approx(val, rel=1e-11, abs=1e-12), (kind, n, N, dt, idx)
        else:
            assert got == pytest.approx(val, rel=1e-4, abs=1e-5), (kind, n, N, dt, idx)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("dim,N", CASES)
def test_full_arrays(soliton_dir, dim, N, dtype):
    t = f"d{dim}_n{N}"
    tol = TOL1[dtype]
    psi0 = REF[t + "_psi0"]
    with qx.Field(dim, N, pref=PREF, dtype=dtype, dt=0.05) as f:
        f.ic_solitons_file("solitons.txt", 1.0)
        assert O.rel_l2(f.psi, psi0) < (1e-14 if dtype == "c128" else 1e-7)
        f.psi = psi0
        f.updatePotential()
        assert v_err(f.V, REF[t + "_V0"], dtype) < 10 * tol
        assert f.Vmax() == pytest.approx(float(REF[t + "_Vmax0"]), rel=10 * tol)
        f.kick(0.05)
        assert O.rel_l2(f.psi, REF[t + "_psi_kick"]) < tol
        f.psi = psi0
        f.drift(0.05)
        assert O.rel_l2(f.psi, REF[t + "_psi_drift"]) < tol
        f.psi = psi0
        f.updatePotential()
        f.kick(0.025)
        f.drift(0.05)
        f.updatePotential()
        f.kick(0.025)
        assert O.rel_l2(f.psi, REF[t + "_psi_kdk"]) < tol
    dt = float(REF[t + "_run_dt"])
    with qx.Field(dim, N, pref=PREF, dtype=dtype, dt=dt) as g:
        g.psi = psi0
        g.step(10)
        assert O.rel_l2(g.psi, REF[t + "_psi_run"]) < (1e-12 if dtype == "c128" else 1e-5)
        assert v_err(g.V, REF[t + "_V_run"], dtype) < (1e-11 if dtype == "c128" else 1e-4)
        assert g.curr() == 10 and g.time() == pytest.approx(10 * dt)
        rhomax, _ = g.rho_stats()
        assert rhomax == pytest.approx(float(REF[t + "_rhomax_run"]), rel=1e-12 if dtype == "c128" else 1e-5)
        k, P, c = g.spectrum(source=0, mode=qx.SPEC_REFERENCE)
        np.testing.assert_array_equal(c, REF[t + "_spec_count"])
        np.testing.assert_allclose(k, REF[t + "_spec_k"], rtol=1e-15)
        sel = c > 0
        np.testing.assert_allclose(P[sel], REF[t + "_spec_P"][sel],
                                   rtol=1e-10 if dtype == "c128" else 1e-4, atol=1e-14 * P.max())


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("dim,N", [(2, 4), (2, 8), (2, 64), (2, 96), (2, 256), (2, 512), (3, 4), (3, 32),
                                   (3, 64), (3, 96)])
def test_fft_plugin(dim, N, dtype):
    rng = np.random.default_rng(7 + N + dim)
    x = rng.standard_normal((N,) * dim) + 1j * rng.standard_normal((N,) * dim)
    xr = rng.standard_normal((N,) * dim)
    tol = 1e-13 if dtype == "c128" else 1e-6
    with qx.Field(dim, N, dtype=dtype) as f:
        assert O.rel_l2(f.fft_c2c(x, -1), np.fft.fftn(x)) < tol
        assert O.rel_l2(f.fft_c2c(x, +1), np.fft.ifftn(x) * x.size) < tol
        h = np.fft.rfftn(xr)
        assert O.rel_l2(f.fft_r2c(xr), h) < tol
        assert O.rel_l2(f.fft_c2r(h), np.fft.irfftn(h, s=xr.shape, axes=tuple(range(dim))) * xr.size) < tol


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_step_matches_oracle_2d_solitons(dtype):
    """2D 256^2, 8 Schive solitons, dt = 0.2 dx^2, 50 merged KDK steps."""
    N = 256
    dt = 0.2 * (1.0 / N) ** 2
    psi0 = O.ic_config("solitons", 2, N, seed=1234, n_solitons=8, rc_lo=0.02, rc_hi=0.05)
    ref, Vref = O.run(psi0, dt, 50, 1.0)
    with qx.Field(2, N, pref=1.0, dtype=dtype, dt=dt) as f:
        f.ic_config(qx.IC_SOLITONS, 1234, 8, 0.02, 0.05)
        assert O.rel_l2(f.psi, psi0) < (1e-12 if dtype == "c128" else 1e-7)
        f.psi = psi0
        f.step(50)
        err = O.rel_l2(f.psi, ref)
        assert err < (1e-12 if dtype == "c128" else 1e-5), err


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_step_matches_oracle_3d_grf(dtype):
    """3D 64^3 GRF (sigma 0.3, kc = N/8 * 2 pi), 20 merged KDK steps."""
    N = 64
    dt = 0.2 * (1.0 / N) ** 2
    with qx.Field(3, N, pref=1.0, dtype="c128", dt=dt) as g:
        g.ic_config(qx.IC_GRF, 99, 0)
        psi0 = g.psi
    assert O.rel_l2(psi0, O.ic_config("grf", 3, N, seed=99)) < 1e-12
    ref, Vref = O.run(psi0, dt, 20, 1.0)
    with qx.Field(3, N, pref=1.0, dtype=dtype, dt=dt) as f:
        f.psi = psi0
        f.step(20)
        assert O.rel_l2(f.psi, ref) < (1e-12 if dtype == "c128" else 1e-5)
        assert v_err(f.V, Vref, dtype) < (1e-11 if dtype == "c128" else 1e-4)


def test_fused_step_equals_reference_call_sequence():
    """qx_step(n) == the reference's main loop spelled with the unfused calls
    (src/main.cxx:64-85)."""
    N, n = 32, 6
    dt = 0.2 * (1.0 / N) ** 2
    psi0 = O.ic_config("grf", 3, N, seed=5)
    with qx.Field(3, N, pref=1.0, dtype="c128", dt=dt) as a, qx.Field(3, N, pref=1.0, dtype="c128", dt=dt) as b:
        a.psi = psi0
        a.step(n)
        b.psi = psi0
        b.updatePotential()
        b.half_kick()
        for i in range(n):
            b.drift_update()
            if i != n - 1:
                b.full_kick()
        b.half_kick()
        assert O.rel_l2(a.psi, b.psi) < 1e-13
        assert a.curr() == b.curr() == n


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 16)])
def test_ic_generators(dim, N):
    t = f"d{dim}_n{N}"
    with qx.Field(dim, N, dtype="c128") as f:
        f.ic_config(qx.IC_SOLITONS, 1234, 8, 0.02, 0.05)
        assert O.rel_l2(f.psi, ICS[t + "_solitons"]) < 1e-12
        f.ic_config(qx.IC_GRF, 1234, 0)
        assert O.rel_l2(f.psi, ICS[t + "_grf"]) < 1e-12
        f.ic_config(qx.IC_GRF, 1234, 4, 0.1, 0.2)
        assert O.rel_l2(f.psi, ICS[t + "_grf_sol"]) < 1e-12
    with qx.Field(dim, N, dtype="c64") as f:
        f.ic_config(qx.IC_GRF, 1234, 0)
        assert O.rel_l2(f.psi, ICS[t + "_grf"]) < 1e-7


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("dim,N,mode,nb", [(2, 64, qx.SPEC_LINEAR, 64 // 2), (2, 256, qx.SPEC_LINEAR, 64),
                                           (3, 32, qx.SPEC_LOG, 12), (3, 64, qx.SPEC_LOG, 24),
                                           (3, 32, qx.SPEC_REFERENCE, 0)])
def test_spectrum_modes(dim, N, mode, nb, dtype):
    psi = O.ic_config("grf+solitons", dim, N, seed=3, n_solitons=3, rc_lo=0.05, rc_hi=0.1)
    with qx.Field(dim, N, dtype=dtype) as f:
        f.psi = psi
        k, P, c = f.spectrum(0, mode, nb)
        ko, Po, co = O.density_spectrum(psi, mode, nb)
        np.testing.assert_array_equal(c, co)
        np.testing.assert_allclose(k, ko, rtol=1e-14)
        sel = c > 0
        # FP32 FFT round-off is white with ~1e-7 of the field's norm, so a bin
        # holding power P carries an absolute error ~2 sqrt(P Pmax) 1e-7: bins
        # far below the peak are compared to that floor (atol) not to rtol.
        atol = 1e-13 if dtype == "c128" else 1e-9
        np.testing.assert_allclose(P[sel], Po[sel], rtol=1e-11 if dtype == "c128" else 2e-5,
                                   atol=atol * Po.max())
        V, _ = O.update_potential(psi, 1.0)
        f.V = V
        k, P, c = f.spectrum(1, mode, nb)
        kv, Pv, cv = O.spectrum_binned(np.fft.rfftn(V), dim, N, mode, nb)
        np.testing.assert_array_equal(c, cv)
        np.testing.assert_allclose(P[sel], Pv[sel], rtol=1e-10 if dtype == "c128" else 1e-4, atol=atol * Pv.max())


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_mass_energy(dtype):
    N = 32
    psi = O.ic_config("grf+solitons", 3, N, seed=11, n_solitons=2, rc_lo=0.08, rc_hi=0.12)
    V, _ = O.update_potential(psi, 1.0)
    E, K, W = O.energy(psi, V)
    with qx.Field(3, N, pref=1.0, dtype=dtype) as f:
        f.psi = psi
        M_, E_, K_, W_ = f.mass_energy()
        tol = 1e-12 if dtype == "c128" else 1e-5
        assert M_ == pytest.approx(O.mass(psi), rel=tol)
        assert K_ == pytest.approx(K, rel=tol)
        assert W_ == pytest.approx(W, rel=10 * tol)
        assert E_ == pytest.approx(E, rel=10 * tol)


def test_k0_policies_agree_when_mean_is_one():
    psi = O.ic_config("grf", 3, 32, seed=21)
    with qx.Field(3, 32, dtype="c128", k0="reference") as a, qx.Field(3, 32, dtype="c128", k0="zero") as b:
        a.psi = psi
        b.psi = psi
        a.updatePotential()
        b.updatePotential()
        Vz, _ = O.update_potential(psi, 1.0, k0="zero")
        assert O.rel_l2(b.V, Vz) < 1e-12
        assert np.max(np.abs(a.V - b.V)) < 1e-13


def test_deterministic_bitwise():
    psi = O.ic_config("grf", 3, 64, seed=8)
    outs = []
    for _ in range(2):
        with qx.Field(3, 64, dtype="c64", dt=1e-5) as f:
            f.psi = psi
            f.step(5)
            outs.append((f.psi, f.spectrum(0, qx.SPEC_LOG, 16)[1], f.mass_energy()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


def test_poisson_and_vhat_roundtrip():
    """Field::Poisson on the transformed V^ (src/field.cxx:230-291) and the
    FFTW-layout V^ accessor."""
    N = 16
    psi = O.ic_config("grf", 3, N, seed=4)
    src = 1.0 * (np.abs(psi) ** 2 - 1.0)
    with qx.Field(3, N, dtype="c128") as f:
        h = np.fft.rfftn(src)
        f.Vhat = h
        assert O.rel_l2(f.Vhat, h) < 1e-15
        f.Poisson()
        assert O.rel_l2(f.Vhat, h * O.poisson_factor(3, N, 1.0)) < 1e-14


def test_errors_are_reported():
    with pytest.raises(ValueError):
        qx.Field(3, 48)
    with qx.Field(2, 16) as f:
        with pytest.raises(ValueError):
            f.ic_solitons_file("/nonexistent/solitons.txt")
        with pytest.raises(ValueError):
            f.spectrum(0, 7, 4)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("dim,N", [(2, 64), (2, 512), (3, 16), (3, 96), (3, 128), (3, 512)])
def test_tma_and_direct_strided_kernels_agree(dim, N, dtype):
    """The TMA-fed persistent strided passes compute what the direct-load
    passes do: same butterflies and phase factors per element; only the
    compiler's fused multiply-add choices may differ between the two kernels,
    so the tolerance is a few units of round-off."""
    dt = 0.2 / N**2
    outs = []
    for tma in (0, 1):
        with qx.Field(dim, N, pref=1.0, dtype=dtype, dt=dt) as f:
            f.set_tune(tma=tma)
            f.ic_config(qx.IC_GRF, 17, 2, 0.05, 0.1)
            f.step(3)
            outs.append((f.psi, f.V, f.mass_energy(), f.spectrum(0, qx.SPEC_REFERENCE)[1]))
    tol = 1e-14 if dtype == "c128" else 1e-6
    # V = c2r(-pref (rho - 1)^/k^2): the cancellation in rho - 1 lifts its
    # relative round-off by ~100x over psi's
    tol_v = 1e-12 if dtype == "c128" else 1e-5
    errs = {"psi": O.rel_l2(outs[1][0], outs[0][0]), "P": O.rel_l2(outs[1][3], outs[0][3])}
    assert max(errs.values()) < tol, errs
    assert v_err(outs[1][1], outs[0][1], dtype) < tol_v
    assert outs[0][2][0] == pytest.approx(outs[1][2][0], rel=tol)
    assert outs[0][2][1] == pytest.approx(outs[1][2][1], rel=tol)


def test_fp32_kick_accuracy():
    """The FP32 kick psi exp(-i dt V) against FP64 on the same FP32 inputs, for
    phases across many quadrants and for small phases.  dt = 0.37 dx^2 is not
    representable in FP32, so the phase dt V must be formed and reduced mod
    2 pi in FP64 (an FP32 product would be off by up to |dt V| 6e-8, 3.6e-6 at
    |dt V| = 60); the bound is the FP32 rounding of the reduced phase, of
    sincosf's result and of the complex product."""
    rng = np.random.default_rng(7)
    N = 32
    f = qx.Field(3, N, dtype="c64")
    shape = f.shape
    psi = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64).astype(np.complex128)
    dt37 = 0.37 / N**2
    for dt, vmax in ((1.0, 60.0), (1.0, 3.0), (1e-3, 0.05), (dt37, 60.0 / dt37), (dt37, 3.0 / dt37),
                     (dt37, 1e-3 / dt37)):
        V = (rng.uniform(-vmax, vmax, size=shape)).astype(np.float32).astype(np.float64)
        f.psi = psi
        f.V = V
        f.kick(dt)
        got = f.psi
        ref = psi * np.exp(-1j * dt * V)
        err = np.abs(got - ref) / np.abs(psi)
        assert err.max() < 4e-7, (dt, vmax, err.max())
    f.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_mre_cosmology_matches_reference(dtype):
    """The merged loop in the MRE cosmology against the reference's own run
    (tests/golden/golden_mre.npz): psi, the scale factor and the step count."""
    d = np.load(os.path.join(GOLDEN, "golden_mre.npz"))
    for dim, N in ((2, 32), (3, 16)):
        tag = f"d{dim}_n{N}"
        f = qx.Field(dim, N, pref=1.0, dtype=dtype, k0="reference", dt=float(d[f"{tag}_dt"]))
        f.set_cosmology(1, float(d[f"{tag}_ai"]))
        f.psi = d[f"{tag}_psi0"]
        f.step(10)
        assert f.curr() == int(d[f"{tag}_curr_run"])
        assert abs(f.a() - float(d[f"{tag}_a_run"])) <= 1e-15
        err = O.rel_l2(f.psi, d[f"{tag}_psi_run"])
        assert err <= (1e-12 if dtype == "c128" else 1e-5), (tag, err)
        f.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_graph_replay_after_eager_drift_with_another_dt(dtype):
    """The captured loop body reads the drift factor tables of its time step;
    an eager drift with another step replaces them, and the next replay must
    see its own again: graph replays equal the same sequence run eagerly."""
    N = 32
    dt = 0.2 / N**2
    outs = []
    for use_graph in (True, False):
        with qx.Field(3, N, pref=1.0, dtype=dtype, dt=dt) as f:
            f.ic_config(qx.IC_GRF, 12, 2, 0.05, 0.1)
            f.time_steps(4, use_graph)
            f.drift(3.7 * dt)
            f.time_steps(4, use_graph)
            outs.append(f.psi)
    assert np.array_equal(outs[0], outs[1])
