"""ctypes loader for oracle/_ref/libqx_ref.so -- the reference solver's own
translation units built against the project FFTW shim (oracle/Makefile).

TEST INFRASTRUCTURE (oracle and timed CPU baseline only).  ``available()`` is
False when the library was not built (it is built from the reference sources,
which exist only where those sources are present).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libqx_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, d, i, dp, ip = C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)
        sig = {
            "ref_create": ([i, i, d, d, d, i], vp),
            "ref_destroy": ([vp], None),
            "ref_sites": ([vp], C.c_size_t),
            "ref_ksites": ([vp], C.c_size_t),
            "ref_set_psi": ([vp, dp], None),
            "ref_get_psi": ([vp, dp], None),
            "ref_set_V": ([vp, dp], None),
            "ref_get_V": ([vp, dp], None),
            "ref_get_Vhat": ([vp, dp], None),
            "ref_ic_solitons": ([vp, d], None),
            "ref_kick": ([vp, d], None),
            "ref_drift": ([vp, d], None),
            "ref_update_potential": ([vp], None),
            "ref_poisson": ([vp], None),
            "ref_compute_energy": ([vp], None),
            "ref_half_kick": ([vp], None),
            "ref_full_kick": ([vp], None),
            "ref_drift_update": ([vp], None),
            "ref_propagate": ([vp], None),
            "ref_vmax": ([vp], d),
            "ref_rhomax": ([vp], d),
            "ref_time": ([vp], d),
            "ref_a": ([vp], d),
            "ref_create_mre": ([i, i, d, d, d, i], vp),
            "ref_curr": ([vp], i),
            "ref_run": ([vp, i], None),
            "ref_loop_body": ([vp, i], None),
            "ref_spectrum": ([vp, dp, ip, dp], None),
            "ref_meas_list": ([C.c_longlong, C.c_longlong, C.POINTER(C.c_longlong)], i),
            "ref_run_measured": ([vp, i, i, i, i, dp, ip, dp, dp, ip], i),
            "ref_fft_forward_c2c": ([vp, dp], None),
            "ref_fft_backward_c2c": ([vp, dp], None),
            "ref_fft_forward_r2c": ([vp, dp, dp], None),
            "ref_fft_backward_c2r": ([vp, dp, dp], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def meas_list(nsteps: int, nmeas: int):
    """The reference's own generateMeasList (src/utils.cxx:8-28)."""
    out = (C.c_longlong * max(nmeas, 1))()
    n = lib().ref_meas_list(nsteps, nmeas, out)
    return [int(out[k]) for k in range(n)]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RefField:
    """The reference ``Field`` (src/field.h:13-97) behind plain pointers.

    norm is the reference's --norm: pref = 4 pi norm (src/field.cxx:78)."""

    def __init__(self, dim: int, N: int, L: float = 1.0, norm: float = 1.0, dt: float = 1e-4,
                 nthr: int = 1, mre_ai: float | None = None):
        """mre_ai: build the MRE cosmology (src/field.cxx:82-88) starting at a = mre_ai."""
        self.dim, self.N = dim, N
        self.shape = (N,) * dim
        self.hshape = (N,) * (dim - 1) + (N // 2 + 1,)
        if mre_ai is None:
            self.h = lib().ref_create(dim, N, L, norm, dt, nthr)
        else:
            self.h = lib().ref_create_mre(dim, N, L, dt, mre_ai, nthr)

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_psi(self, psi: np.ndarray):
        a = np.ascontiguousarray(psi, dtype=np.complex128)
        lib().ref_set_psi(self.h, _dp(a.view(np.float64)))

    def psi(self) -> np.ndarray:
        a = np.empty(self.shape, np.complex128)
        lib().ref_get_psi(self.h, _dp(a.view(np.float64)))
        return a

    def set_V(self, V: np.ndarray):
        a = np.ascontiguousarray(V, dtype=np.float64)
        lib().ref_set_V(self.h, _dp(a))

    def V(self) -> np.ndarray:
        a = np.empty(self.shape, np.float64)
        lib().ref_get_V(self.h, _dp(a))
        return a

    def Vhat(self) -> np.ndarray:
        a = np.empty(self.hshape, np.complex128)
        lib().ref_get_Vhat(self.h, _dp(a.view(np.float64)))
        return a

    def spectrum(self):
        nb = self.N // 2 + 1
        P = np.empty(nb)
        k = np.empty(nb)
        c = np.empty(nb, np.int32)
        lib().ref_spectrum(self.h, _dp(P), c.ctypes.data_as(C.POINTER(C.c_int)), _dp(k))
        return k, P, c.astype(np.int64)

    def run_measured(self, nsteps: int, nmeas: int, clobber: bool, spectrum: bool):
        """The reference's main loop with measurements (ref_run_measured):
        (rhomax, curr, time, P[m, b], counts[m, b]) per measurement."""
        nb = self.N // 2 + 1
        cap = nmeas + 1
        rm, tm = np.zeros(cap), np.zeros(cap)
        cu = np.zeros(cap, np.int32)
        P = np.zeros((cap, nb))
        cnt = np.zeros((cap, nb), np.int32)
        m = lib().ref_run_measured(self.h, nsteps, nmeas, int(clobber), int(spectrum), _dp(rm),
                                   cu.ctypes.data_as(C.POINTER(C.c_int)), _dp(tm), _dp(P),
                                   cnt.ctypes.data_as(C.POINTER(C.c_int)))
        return rm[:m], cu[:m], tm[:m], P[:m], cnt[:m].astype(np.int64)

    def __getattr__(self, name):
        f = getattr(lib(), "ref_" + name)
        return lambda *a: f(self.h, *a)
