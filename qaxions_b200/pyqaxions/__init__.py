"""Reference-facing test surface: the pybind11 modules ``fieldtest`` and
``ictest`` (built from qaxions_b200/csrc/py/ into this directory), with the
names, arguments and return values of the reference's modules
``pyqaxions.fieldtest`` and ``pyqaxions.ictest``
(src/examples/fieldtest.cxx:99-105, src/examples/ictest.cxx:46-50), running on
the B200 through the C ABI.  The top-level package ``pyqaxions`` maps the
reference's import name onto this directory.
"""
