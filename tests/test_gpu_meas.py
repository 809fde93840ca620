"""spec_NNNN.txt written from a device field matches the field's spectrum."""
import numpy as np
import pytest

import qaxions_b200 as qx
from qaxions_b200.meas import write_spectrum

pytestmark = pytest.mark.gpu


def test_write_spectrum_file(tmp_path):
    f = qx.Field(3, 32, dtype="c64")
    f.ic_config(qx.IC_GRF, 5, 2, 0.01, 0.03)
    path = write_spectrum(f, str(tmp_path), 7)
    assert path.endswith("spec_0007.txt")
    with open(path) as fh:
        a = float(fh.readline().split(":")[1])
        k, P, c = np.loadtxt(fh, unpack=True)
    k0, P0, c0 = f.spectrum(0, qx.SPEC_REFERENCE)
    sel = c0 > 0
    assert a == 1.0
    assert np.allclose(k, k0[sel], rtol=1e-6) and np.allclose(P, P0[sel], rtol=1e-6)
    assert np.array_equal(c.astype(np.int64), c0[sel])
    f.close()
