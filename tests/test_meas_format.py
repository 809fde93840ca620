"""Spectrum file format (reference Spectrum::write) read back the way the
reference's scripts/plot_spectrum.py reads it."""
import io

import numpy as np

from qaxions_b200.meas import format_profile, format_spectrum


def test_spectrum_file_round_trip():
    k = np.array([0.0, 6.283185307179586, 12.566370614359172, 18.84955592153876])
    P = np.array([1.5, 2.25e-3, 0.0, 7.0e-9])
    c = np.array([1, 6, 0, 24])
    txt = format_spectrum(1.0, k, P, c)
    fh = io.StringIO(txt)
    a = float(fh.readline().split(":")[1])
    kk, pp, cc = np.loadtxt(fh, unpack=True)
    assert a == 1.0
    assert len(kk) == 3  # the empty shell is skipped
    assert np.allclose(kk, k[c > 0], rtol=1e-6) and np.allclose(pp, P[c > 0], rtol=1e-6)
    assert np.array_equal(cc.astype(int), c[c > 0])
    assert txt.splitlines()[2] == "0.000000e+00  1.500000e+00  1"


def test_profile_summary():
    s = format_profile([("x_c2r_kick_fwd", 800.0, 10), ("z_drift", 830.0, 10)])
    assert "z_drift" in s and "50.9%" in s
