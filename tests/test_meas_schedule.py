"""CPU: the measurement schedule of the library's time loop against the
reference's own generateMeasList (src/utils.cxx:8-28) from the reference build
(oracle/_ref), including the degenerate cases (no measurement, one, more
measurements than steps)."""
import pytest

import qaxions_b200 as qx
from oracle import ref_lib as R

CASES = [(0, 0), (0, 3), (5, 0), (1, 1), (10, 1), (10, 2), (10, 10), (3, 5), (1000, 50), (500, 11), (2000, 7),
         (7, 3), (100, 100), (101, 100)]


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (reference build) not built")
@pytest.mark.parametrize("nsteps,nmeas", CASES)
def test_meas_list_equals_reference(nsteps, nmeas):
    assert qx.meas_list(nsteps, nmeas) == R.meas_list(nsteps, nmeas)


def test_meas_list_formula():
    # k (n - 1) / (m - 1) in integer arithmetic; one measurement lands on the last step
    assert qx.meas_list(1000, 5) == [0, 249, 499, 749, 999]
    assert qx.meas_list(10, 1) == [9]
    assert qx.meas_list(0, 4) == []
    with pytest.raises(ValueError):
        qx.meas_list(-1, 2)
