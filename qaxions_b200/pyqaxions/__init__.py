"""Reference-facing test surface: the functions of the reference's pybind11
modules ``pyqaxions.fieldtest`` and ``pyqaxions.ictest``
(src/examples/fieldtest.cxx:99-105, src/examples/ictest.cxx:46-50), with the
same names, arguments and return values, running on the B200 through the C ABI.
"""
