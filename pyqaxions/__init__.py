"""``pyqaxions``: the reference's Python module name (its pybind11 test modules
``pyqaxions.fieldtest`` and ``pyqaxions.ictest``, src/examples/*.cxx), served
by this library's pybind11 modules of the same names in
qaxions_b200/pyqaxions/.  With the repository root on sys.path,
``import pyqaxions.fieldtest as field`` -- the import of the reference's
tests/test_field.py -- loads the B200 module.
"""
import os as _os

__path__ = [_os.path.join(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__))), "qaxions_b200",
                          "pyqaxions")]
