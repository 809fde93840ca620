import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture
def soliton_dir(tmp_path, monkeypatch):
    """A working directory holding the reference's solitons.txt rows, since the
    soliton IC reads ./solitons.txt like the reference (src/ic/solitons.cxx:32)."""
    shutil.copy(os.path.join(GOLDEN, "ref_solitons.txt"), tmp_path / "solitons.txt")
    monkeypatch.chdir(tmp_path)
    return tmp_path
