"""CPU: the pybind11 modules of the reference's Python test surface load under
the reference's import names and expose its functions (no GPU call here; the
GPU parity suite calls them)."""
import importlib.machinery
import inspect


def test_modules_are_pybind11_extensions_under_reference_names():
    import pyqaxions.fieldtest as field
    import pyqaxions.ictest as ic

    for mod in (field, ic):
        assert mod.__file__.endswith(tuple(importlib.machinery.EXTENSION_SUFFIXES)), mod.__file__
        assert "qaxions_b200" in mod.__file__
    for name in ("test_kick", "test_drift", "test_potential", "test_kick_drift_step"):
        assert callable(getattr(field, name))
    for name in ("test_solitons", "test_solitons_3D"):
        assert callable(getattr(ic, name))
    # the reference's positional arguments (src/examples/fieldtest.cxx:11-96,
    # src/examples/ictest.cxx:8-42), in order
    def params(f):
        sig = f.__doc__.split("(", 1)[1].split(")")[0]
        return [p.split(":")[0].strip() for p in sig.split(",") if p.strip()]
    assert params(field.test_kick)[:4] == ["n", "N", "dt", "idx"]
    assert params(field.test_potential)[:3] == ["n", "N", "idx"]
    assert params(ic.test_solitons)[:2] == ["N", "idx"]


def test_same_modules_through_the_package_path():
    from qaxions_b200.pyqaxions import fieldtest, ictest
    import pyqaxions.fieldtest as field

    assert fieldtest.__file__ == field.__file__
    assert inspect.isbuiltin(ictest.test_solitons_3D)
