"""Generate the committed golden fixtures from the REFERENCE solver itself.

Run here (where the reference sources exist) after ``make -C oracle``:

    python tests/golden/make_golden.py

It drives oracle/_ref/libqx_ref.so -- the reference's own src/field.cxx,
src/spectrum/spectrum.cxx and src/ic/*.cxx compiled unmodified against the
project FFTW shim -- from a directory holding the reference's solitons.txt
(the only fixture the reference ships, solitons.txt:1-2), and writes:

  ref_solitons.txt   the data rows of that solitons.txt (amp sigma x y z)
  golden_ref.npz     full-array outputs of the reference operations
  golden_pins.npz    the scalar pins of the reference's own tests
                     (tests/test_field.py:12-129, tests/test_ic.py:12-37):
                     each test's parameter grid with the value the reference
                     module returns
  golden_ic.npz      the synthetic benchmark ICs from the NumPy oracle
                     (no reference counterpart), small sizes
  golden_mre.npz     the merged loop in the MRE cosmology (make_mre)

Nothing at test time reads the reference tree.
"""
from __future__ import annotations

import math
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import REFERENCE_DIR  # noqa: E402
from oracle import ref_lib as R  # noqa: E402
from oracle import sp_oracle as O  # noqa: E402

REF_SOLITONS = os.path.join(REFERENCE_DIR, "solitons.txt")


def make_mre():
    """golden_mre.npz: the merged loop in the reference's MRE cosmology
    (src/field.cxx:82-88, 349-361), a_i = 0.1, 10 steps from the soliton IC."""
    work = tempfile.mkdtemp()
    shutil.copy(REF_SOLITONS, os.path.join(work, "solitons.txt"))
    cwd = os.getcwd()
    os.chdir(work)
    try:
        out = {}
        for dim, N in [(2, 32), (3, 16)]:
            tag = f"d{dim}_n{N}"
            f = R.RefField(dim, N, 1.0, 1.0, 0.05)
            f.ic_solitons(1.0)
            psi0 = f.psi()
            dt = 1e-3
            g = R.RefField(dim, N, 1.0, 1.0, dt, mre_ai=0.1)
            g.set_psi(psi0)
            g.run(10)
            out[f"{tag}_psi0"] = psi0
            out[f"{tag}_dt"] = np.float64(dt)
            out[f"{tag}_ai"] = np.float64(0.1)
            out[f"{tag}_psi_run"] = g.psi()
            out[f"{tag}_a_run"] = np.float64(R.lib().ref_a(g.h))
            out[f"{tag}_curr_run"] = np.int64(R.lib().ref_curr(g.h))
        np.savez_compressed(os.path.join(HERE, "golden_mre.npz"), **out)
    finally:
        os.chdir(cwd)


def main():
    if not R.available():
        raise SystemExit("build the oracle first: make -C oracle")
    rows = O.read_solitons_txt(REF_SOLITONS)
    with open(os.path.join(HERE, "ref_solitons.txt"), "w") as fh:
        for r in rows:
            fh.write(" ".join(repr(v) for v in r) + "\n")

    work = tempfile.mkdtemp()
    shutil.copy(REF_SOLITONS, os.path.join(work, "solitons.txt"))
    cwd = os.getcwd()
    os.chdir(work)
    try:
        out = {}
        pref = 4.0 * math.pi  # norm = 1
        for dim, N in [(2, 16), (2, 32), (3, 8), (3, 16)]:
            tag = f"d{dim}_n{N}"
            f = R.RefField(dim, N, 1.0, 1.0, 0.05)
            f.ic_solitons(1.0)
            psi0 = f.psi()
            out[f"{tag}_psi0"] = psi0
            f.update_potential()
            out[f"{tag}_V0"] = f.V()
            out[f"{tag}_Vmax0"] = np.float64(f.vmax())
            f.kick(0.05)
            out[f"{tag}_psi_kick"] = f.psi()
            f.set_psi(psi0)
            f.drift(0.05)
            out[f"{tag}_psi_drift"] = f.psi()
            # unmerged KDK (src/examples/fieldtest.cxx:73-96)
            f.set_psi(psi0)
            f.update_potential()
            f.kick(0.025)
            f.drift(0.05)
            f.update_potential()
            f.kick(0.025)
            out[f"{tag}_psi_kdk"] = f.psi()
            # merged loop (src/main.cxx:64-85), 10 steps at dt = 0.2 dx^2 * 50
            dt = 10.0 * (1.0 / N) ** 2
            g = R.RefField(dim, N, 1.0, 1.0, dt)
            g.set_psi(psi0)
            g.run(10)
            out[f"{tag}_run_dt"] = np.float64(dt)
            out[f"{tag}_psi_run"] = g.psi()
            out[f"{tag}_V_run"] = g.V()
            # computeEnergy + Spectrum of rho (src/meas.cxx:30-41)
            h = R.RefField(dim, N, 1.0, 1.0, dt)
            h.set_psi(g.psi())
            h.compute_energy()
            out[f"{tag}_rhomax_run"] = np.float64(h.rhomax())
            k, P, c = h.spectrum()
            out[f"{tag}_spec_k"], out[f"{tag}_spec_P"], out[f"{tag}_spec_count"] = k, P, c
            # FFT plugin on a seeded complex / real array
            rng = np.random.default_rng(100 + 10 * dim + N)
            x = rng.standard_normal((N,) * dim) + 1j * rng.standard_normal((N,) * dim)
            xr = rng.standard_normal((N,) * dim)
            y = x.copy()
            R.lib().ref_fft_forward_c2c(f.h, R._dp(y.view(np.float64)))
            out[f"{tag}_fft_in"], out[f"{tag}_fft_fwd"] = x, y
            hr = np.empty((N,) * (dim - 1) + (N // 2 + 1,), np.complex128)
            R.lib().ref_fft_forward_r2c(f.h, R._dp(xr), R._dp(hr.view(np.float64)))
            out[f"{tag}_r2c_in"], out[f"{tag}_r2c_out"] = xr, hr
        np.savez_compressed(os.path.join(HERE, "golden_ref.npz"), **out)

        # scalar pins of the reference's own pybind tests
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import pyqaxions.fieldtest as ft  # the reference's module built here
        import pyqaxions.ictest as it
        pins = []
        for n in (2, 3):
            for N in (4, 8):
                for idx in (1, 9):
                    pins.append(("potential", n, N, 0.0, idx, ft.test_potential(n, N, idx)))
                    for dt in (0.05, 0.1):
                        pins.append(("kick", n, N, dt, idx, ft.test_kick(n, N, dt, idx)))
                        pins.append(("drift", n, N, dt, idx, ft.test_drift(n, N, dt, idx)))
                        pins.append(("kdk", n, N, dt, idx, ft.test_kick_drift_step(n, N, dt, idx)))
        for N in (4, 8):
            for idx in (1, 9):
                pins.append(("ic2d", 2, N, 0.0, idx, it.test_solitons(N, idx)))
                pins.append(("ic3d", 3, N, 0.0, idx, it.test_solitons_3D(N, idx)))
        np.savez_compressed(
            os.path.join(HERE, "golden_pins.npz"),
            kind=np.array([p[0] for p in pins]), dim=np.array([p[1] for p in pins]),
            N=np.array([p[2] for p in pins]), dt=np.array([p[3] for p in pins]),
            idx=np.array([p[4] for p in pins]), value=np.array([p[5] for p in pins]))
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)

    ic = {}
    for dim, N in [(2, 32), (3, 16)]:
        ic[f"d{dim}_n{N}_solitons"] = O.ic_config("solitons", dim, N, seed=1234, n_solitons=8,
                                                  rc_lo=0.02, rc_hi=0.05)
        ic[f"d{dim}_n{N}_grf"] = O.ic_config("grf", dim, N, seed=1234)
        ic[f"d{dim}_n{N}_grf_sol"] = O.ic_config("grf+solitons", dim, N, seed=1234, n_solitons=4,
                                                 rc_lo=0.1, rc_hi=0.2)
    np.savez_compressed(os.path.join(HERE, "golden_ic.npz"), **ic)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    if sys.argv[1:] == ["mre"]:
        make_mre()
    else:
        main()
        make_mre()
