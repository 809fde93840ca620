"""GPU: the allocation-free density-statistics entry point.

qx_rho_stats_noalloc serves callers that may not allocate device memory while
they run (their own pool owns the memory, or an allocation's implicit device
synchronisation would stall their time loop).  It works on a psi array the
caller already holds and keeps its scratch in a fixed array inside the
library.  This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import qaxions_b200 as qx
from oracle import sp_oracle as O

pytestmark = pytest.mark.gpu

_lib = qx.lib()
_lib.qx_rho_stats_noalloc.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p]
_lib.qx_rho_stats_noalloc.restype = C.c_int
_lib.qx_noalloc_last_error.argtypes = []
_lib.qx_noalloc_last_error.restype = C.c_char_p


@pytest.mark.parametrize("dtype,tol", [("c128", 1e-12), ("c64", 1e-12)])
def test_noalloc_rho_stats_matches_field_entry_point(dtype, tol):
    import torch

    N = 64
    psi = O.ic_config("grf+solitons", 3, N, seed=31, n_solitons=3, rc_lo=0.05, rc_hi=0.1)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    with qx.Field(3, N, dtype=dtype) as f:
        f.psi = psi
        rhomax_ref, _ = f.rho_stats()                  # existing entry point
        mass_ref = f.mass_energy()[0] / (1.0 / N) ** 3  # sum |psi|^2
        psi_dev, _ = f.device_pointers()
        code = qx.QX_C128 if dtype == "c128" else qx.QX_C64
        # the oracle's sum and max of |psi|^2 of the state the device holds
        rho = np.abs(f.psi) ** 2
        for _ in range(2):                              # two calls in a row share the scratch
            out.zero_()
            st = _lib.qx_rho_stats_noalloc(psi_dev, N**3, code, out.data_ptr(), None)
            assert st == qx.QX_OK, _lib.qx_noalloc_last_error()
            torch.cuda.synchronize()
            s, m, rhomax = out.cpu().tolist()
            assert rhomax == pytest.approx(rhomax_ref, rel=tol)
            assert s == pytest.approx(mass_ref, rel=tol)
            assert m == pytest.approx(rhomax_ref * s / N**3, rel=tol)
            assert s == pytest.approx(float(rho.sum()), rel=1e-13)
            assert m == pytest.approx(float(rho.max()), rel=1e-15)
            assert rhomax == pytest.approx(float(rho.max() / rho.mean()), rel=1e-13)


def test_noalloc_propagates_nan():
    import torch

    N = 16
    psi = np.ones((N,) * 3, np.complex128)
    psi[3, 4, 5] = np.nan
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    with qx.Field(3, N) as f:
        f.psi = psi
        psi_dev, _ = f.device_pointers()
        st = _lib.qx_rho_stats_noalloc(psi_dev, N**3, qx.QX_C128, out.data_ptr(), None)
        assert st == qx.QX_OK, _lib.qx_noalloc_last_error()
        torch.cuda.synchronize()
        assert all(np.isnan(v) for v in out.cpu().tolist())


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    with qx.Field(3, 16) as f:
        psi_dev, _ = f.device_pointers()
        st = _lib.qx_rho_stats_noalloc(psi_dev, (1 << 27) + 1, qx.QX_C128, out.data_ptr(), None)
        assert st == qx.QX_ERR_INVALID
        assert b"at most" in _lib.qx_noalloc_last_error()
        host = np.zeros(6)
        st = _lib.qx_rho_stats_noalloc(host.ctypes.data, 16**3, qx.QX_C128, out.data_ptr(), None)
        assert st == qx.QX_ERR_INVALID
        # an output in host memory is refused before any launch
        st = _lib.qx_rho_stats_noalloc(psi_dev, 16**3, qx.QX_C128, host.ctypes.data, None)
        assert st == qx.QX_ERR_INVALID
        assert b"out" in _lib.qx_noalloc_last_error()
        # more sites than psi's allocation holds (within the scratch limit)
        st = _lib.qx_rho_stats_noalloc(psi_dev, 64**3, qx.QX_C128, out.data_ptr(), None)
        assert st == qx.QX_ERR_INVALID
        assert b"past the end" in _lib.qx_noalloc_last_error()
