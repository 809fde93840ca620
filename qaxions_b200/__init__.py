"""qaxions_b200 -- B200-native Schroedinger-Poisson solver core.

Python face of the C ABI in include/qaxions_b200.h (libqaxions_b200.so, built
in-tree for sm_100a).  ``Field`` mirrors the reference's operator surface
(gpierobon/qaxions src/field.h:17-64): kick, drift, Poisson, updatePotential,
computeEnergy, updateTime, half_kick, full_kick, drift_update, propagate, plus
``step`` (the fused, graph-replayed KDK loop of src/main.cxx:64-85).

There is no CPU fallback: importing this package raises if the library is
missing, and constructing a Field raises if no CUDA device is usable.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqaxions_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "qaxions_b200.h")

QX_OK, QX_ERR_INVALID, QX_ERR_CUDA, QX_ERR_NOMEM, QX_ERR_STATE, QX_ERR_INTERNAL = range(6)
QX_C128, QX_C64 = 0, 1
QX_K0_REFERENCE, QX_K0_ZERO = 0, 1
SPEC_REFERENCE, SPEC_LINEAR, SPEC_LOG = 0, 1, 2
IC_SOLITONS, IC_GRF = 0, 1

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C qaxions_b200/csrc -j8` "
        "(or __graft_entry__.build()); there is no CPU fallback")

_lib = C.CDLL(LIB_PATH)
_vp, _d, _i = C.c_void_p, C.c_double, C.c_int
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_llp = C.POINTER(C.c_longlong)
_fp = C.POINTER(C.c_float)

# MeasureType bits (src/enum.h:39-47) and this library's own
MEAS_NONE, MEAS_SPECTRUM, MEAS_RHO_MAX, MEAS_RHO_SLICE, MEAS_RHO_GRID, MEAS_PSI_GRID = 0, 1, 2, 4, 8, 16
MEAS_ENERGY, MEAS_CLOBBER_V = 1 << 8, 1 << 9


class MeasRecord(C.Structure):
    """qx_meas_t: one measurement of measure() (src/meas.cxx:13-63)."""
    _fields_ = [("number", C.c_int), ("step", C.c_int), ("time", C.c_double), ("a", C.c_double),
                ("rhomax", C.c_double), ("vmax", C.c_double), ("mass", C.c_double), ("energy", C.c_double),
                ("kinetic", C.c_double), ("potential", C.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_SIGS = {
    "qx_version": ([], _i),
    "qx_last_error": ([_vp], C.c_char_p),
    "qx_set_device": ([_i], _i),
    "qx_create": ([_i, _i, _d, _d, _d, _i, _i, _d, C.POINTER(_vp)], _i),
    "qx_destroy": ([_vp], _i),
    "qx_set_dt": ([_vp, _d], _i),
    "qx_set_psi": ([_vp, _dp], _i),
    "qx_get_psi": ([_vp, _dp], _i),
    "qx_set_V": ([_vp, _dp], _i),
    "qx_get_V": ([_vp, _dp], _i),
    "qx_get_Vhat": ([_vp, _dp], _i),
    "qx_set_Vhat": ([_vp, _dp], _i),
    "qx_kick": ([_vp, _d], _i),
    "qx_drift": ([_vp, _d], _i),
    "qx_poisson": ([_vp], _i),
    "qx_update_potential": ([_vp], _i),
    "qx_compute_energy": ([_vp], _i),
    "qx_update_time": ([_vp], _i),
    "qx_half_kick": ([_vp], _i),
    "qx_full_kick": ([_vp], _i),
    "qx_drift_update": ([_vp], _i),
    "qx_propagate": ([_vp], _i),
    "qx_step": ([_vp, _i], _i),
    "qx_scalars": ([_vp, _dp, _dp, _dp, _dp, _ip], _i),
    "qx_rho_stats": ([_vp, _dp, _dp], _i),
    "qx_mass_energy": ([_vp, _dp, _dp, _dp, _dp], _i),
    "qx_spectrum": ([_vp, _i, _i, _i, _dp, _dp, _llp], _i),
    "qx_meas_list": ([C.c_longlong, C.c_longlong, _llp, _i, _ip], _i),
    "qx_measure": ([_vp, C.c_uint, _i, C.c_char_p, C.POINTER(MeasRecord)], _i),
    "qx_run": ([_vp, _i, _i, C.c_uint, C.c_char_p, C.POINTER(MeasRecord), _i, _ip], _i),
    "qx_fft_c2c": ([_vp, _dp, _i], _i),
    "qx_fft_r2c": ([_vp, _dp, _dp], _i),
    "qx_fft_c2r": ([_vp, _dp, _dp], _i),
    "qx_ic_solitons_file": ([_vp, C.c_char_p, _d], _i),
    "qx_ic_gaussian_solitons": ([_vp, _i, _dp, _d], _i),
    "qx_ic_config": ([_vp, _i, C.c_ulonglong, _i, _d, _d, _d, _d, _d, _d], _i),
    "qx_time_steps": ([_vp, _i, _i, _fp], _i),
    "qx_profile_step": ([_vp, _i, _i, C.c_char_p, _dp, _ip], _i),
    "qx_set_tune": ([_vp, _i, _i, _i, _i, _i, _i], _i),
    "qx_set_chain": ([_vp, _i], _i),
    "qx_set_plan": ([_vp, _i], _i),
    "qx_set_pencil_warp": ([_vp, _i], _i),
    "qx_set_row_stage": ([_vp, _i], _i),
    "qx_clear_tune_cache": ([], _i),
    "qx_get_tune": ([_vp, _ip, _i], _i),
    "qx_device_pointers": ([_vp, C.POINTER(_vp), C.POINTER(_vp)], _i),
    "qx_sync": ([_vp], _i),
    "qx_autotune": ([_vp, _i, C.c_char_p, _dp, _ip], _i),
    "qx_set_clock": ([_vp, _i, _d], _i),
    "qx_set_cosmology": ([_vp, _i, _d], _i),
    "qx_get_cosmology": ([_vp, _ip, _dp, _dp], _i),
    "qx_restore_cosmology": ([_vp, _d, _d], _i),
    "qx_ens_create": ([_i, _ip, _ip, _i, _d, _d, _i, _d, C.POINTER(_vp)], _i),
    "qx_ens_destroy": ([_vp], _i),
    "qx_ens_last_error": ([_vp], C.c_char_p),
    "qx_ens_size": ([_vp, _ip, _llp], _i),
    "qx_ens_box_n": ([_vp, _i, _ip], _i),
    "qx_ens_ic_config": ([_vp, _i, C.c_ulonglong, _i, _d, _d, _d, _d, _d, _d], _i),
    "qx_ens_ic_config_seeds": ([_vp, _i, C.POINTER(C.c_ulonglong), _i, _d, _d, _d, _d, _d, _d], _i),
    "qx_ens_set_psi": ([_vp, _i, _dp], _i),
    "qx_ens_get_psi": ([_vp, _i, _dp], _i),
    "qx_ens_step": ([_vp, _i], _i),
    "qx_ens_time_steps": ([_vp, _i, _fp], _i),
    "qx_ens_mass": ([_vp, _dp], _i),
    "qx_ens_set_mixed": ([_vp, _i], _i),
    "qx_ens_set_mixed_window": ([_vp, C.c_longlong], _i),
}
for _name, (_args, _res) in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.argtypes = _args
    _f.restype = _res


def lib():
    """The loaded ctypes library (C ABI of include/qaxions_b200.h)."""
    return _lib


class QxError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[qx status {status}] {msg}")
        self.status = status


def _check(status: int, h=None):
    if status != QX_OK:
        msg = (_lib.qx_last_error(h) or b"").decode(errors="replace")
        if status == QX_ERR_INVALID:
            raise ValueError(msg)
        if status == QX_ERR_NOMEM:
            raise MemoryError(msg)
        raise QxError(status, msg)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def meas_list(nsteps: int, nmeas: int):
    """generateMeasList (src/utils.cxx:8-28): the loop indices after whose
    drift_update the time loop measures."""
    out = (C.c_longlong * max(int(nmeas), 1))()
    n = C.c_int()
    _check(_lib.qx_meas_list(int(nsteps), int(nmeas), out, max(int(nmeas), 1), C.byref(n)))
    return [int(out[i]) for i in range(n.value)]


def clear_tune_cache():
    """Forget the autotuner's in-process choices (cache files are left alone)."""
    _check(_lib.qx_clear_tune_cache())


def set_device(device: int):
    """Place fields created afterwards by this thread on CUDA device `device`."""
    _check(_lib.qx_set_device(device))


class Field:
    """One periodic box (reference ``Field``, src/field.h:13-97).

    dtype "c128" is the plain FP64 form, "c64" the fused FP32 form.  Host
    arrays are complex128 / float64 in reference order ([z, y, x] / [y, x]).
    ``pref`` is the Poisson prefactor (the reference's 4 pi norm a,
    src/field.cxx:78,298)."""

    def __init__(self, dim: int, N: int, L: float = 1.0, pref: float = 1.0, rho_mean: float = 1.0,
                 dtype: str = "c128", k0: str = "reference", dt: float = 1e-4):
        if dtype not in ("c128", "c64"):
            raise ValueError("dtype must be 'c128' or 'c64'")
        if k0 not in ("reference", "zero"):
            raise ValueError("k0 must be 'reference' or 'zero'")
        self._h = _vp()
        _check(_lib.qx_create(dim, N, L, pref, rho_mean, QX_C128 if dtype == "c128" else QX_C64,
                              QX_K0_REFERENCE if k0 == "reference" else QX_K0_ZERO, dt, C.byref(self._h)))
        self.N_, self.dim_, self.L, self.dtype = N, dim, L, dtype
        self._dt = dt
        self.shape = (N,) * dim
        self.hshape = (N,) * (dim - 1) + (N // 2 + 1,)

    # -- lifetime --
    def close(self):
        if getattr(self, "_h", None):
            _lib.qx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, name, *args):
        _check(getattr(_lib, name)(self._h, *args), self._h)

    # -- reference operator surface --
    def kick(self, dt: float):
        self._c("qx_kick", dt)

    def drift(self, dt: float):
        self._c("qx_drift", dt)

    def Poisson(self):
        self._c("qx_poisson")

    def updatePotential(self):
        self._c("qx_update_potential")

    def computeEnergy(self):
        self._c("qx_compute_energy")

    def updateTime(self):
        self._c("qx_update_time")

    def half_kick(self):
        self._c("qx_half_kick")

    def full_kick(self):
        self._c("qx_full_kick")

    def drift_update(self):
        self._c("qx_drift_update")

    def propagate(self):
        self._c("qx_propagate")

    def step(self, nsteps: int):
        self._c("qx_step", nsteps)

    def set_dt(self, dt: float):
        self._c("qx_set_dt", dt)
        self._dt = dt

    def dt(self) -> float:
        return self._dt

    # -- buffers --
    @property
    def psi(self) -> np.ndarray:
        a = np.empty(self.shape, np.complex128)
        self._c("qx_get_psi", _ptr(a.view(np.float64)))
        return a

    @psi.setter
    def psi(self, value):
        a = np.ascontiguousarray(value, dtype=np.complex128).reshape(self.shape)
        self._c("qx_set_psi", _ptr(a.view(np.float64)))

    def set_psi_ptr(self, addr: int):
        """Upload psi from a host buffer at `addr` (2*sites float64, e.g. pinned)."""
        self._c("qx_set_psi", C.cast(C.c_void_p(addr), _dp))

    def get_psi_ptr(self, addr: int):
        """Download psi into a host buffer at `addr` (2*sites float64)."""
        self._c("qx_get_psi", C.cast(C.c_void_p(addr), _dp))

    @property
    def V(self) -> np.ndarray:
        a = np.empty(self.shape, np.float64)
        self._c("qx_get_V", _ptr(a))
        return a

    @V.setter
    def V(self, value):
        a = np.ascontiguousarray(value, dtype=np.float64).reshape(self.shape)
        self._c("qx_set_V", _ptr(a))

    @property
    def Vhat(self) -> np.ndarray:
        a = np.empty(self.hshape, np.complex128)
        self._c("qx_get_Vhat", _ptr(a.view(np.float64)))
        return a

    @Vhat.setter
    def Vhat(self, value):
        a = np.ascontiguousarray(value, dtype=np.complex128).reshape(self.hshape)
        self._c("qx_set_Vhat", _ptr(a.view(np.float64)))

    def getPsiIdx(self, idx: int) -> float:
        return float(self.psi.ravel()[idx].real)

    def getPsiImagIdx(self, idx: int) -> float:
        return float(self.psi.ravel()[idx].imag)

    def getVIdx(self, idx: int) -> float:
        return float(self.V.ravel()[idx])

    # -- scalars --
    def _scalars(self):
        v, r, t, a = (C.c_double() for _ in range(4))
        c = C.c_int()
        self._c("qx_scalars", C.byref(v), C.byref(r), C.byref(t), C.byref(a), C.byref(c))
        return v.value, r.value, t.value, a.value, c.value

    def size(self) -> int:
        return self.N_

    def dim(self) -> int:
        return self.dim_

    def sites(self) -> int:
        return self.N_ ** self.dim_

    def ksites(self) -> int:
        return self.N_ ** (self.dim_ - 1) * (self.N_ // 2 + 1)

    def Vmax(self) -> float:
        return self._scalars()[0]

    def rhomax(self) -> float:
        return self._scalars()[1]

    def time(self) -> float:
        return self._scalars()[2]

    def a(self) -> float:
        return self._scalars()[3]

    def curr(self) -> int:
        return self._scalars()[4]

    # -- measurements --
    def rho_stats(self):
        r, v = C.c_double(), C.c_double()
        self._c("qx_rho_stats", C.byref(r), C.byref(v))
        return r.value, v.value

    def mass_energy(self):
        """(M, E, K, W)."""
        out = [C.c_double() for _ in range(4)]
        self._c("qx_mass_energy", *(C.byref(o) for o in out))
        return tuple(o.value for o in out)

    def spectrum(self, source: int = 0, mode: int = SPEC_REFERENCE, nbins: int = 0):
        """(k, P, count) shell-binned spectrum of |psi|^2 (source 0) or V (1)."""
        nb = self.N_ // 2 + 1 if mode == SPEC_REFERENCE else nbins
        k, P = np.empty(nb), np.empty(nb)
        cnt = np.empty(nb, np.int64)
        self._c("qx_spectrum", source, mode, nbins, _ptr(k), _ptr(P), cnt.ctypes.data_as(_llp))
        return k, P, cnt

    def measure(self, mask: int = MEAS_RHO_MAX, number: int = 0, directory: str | None = None) -> dict:
        """measure() (src/meas.cxx:13-63) of the current state: rhomax and Vmax,
        the spectrum file (MEAS_SPECTRUM) and density grid (MEAS_RHO_GRID) in
        `directory`, mass and energy (MEAS_ENERGY).  V is left alone unless
        MEAS_CLOBBER_V."""
        r = MeasRecord()
        self._c("qx_measure", mask, number, directory.encode() if directory else None, C.byref(r))
        return r.as_dict()

    def run(self, nsteps: int, nmeas: int, mask: int = MEAS_RHO_MAX, directory: str | None = None):
        """The time loop of main() (src/main.cxx:60-85) with measure(0) and one
        measurement after each scheduled drift_update (meas_list); returns the
        records (dicts), also written to `directory`/measurements.jsonl."""
        recs = (MeasRecord * (nmeas + 1))()
        n = C.c_int()
        self._c("qx_run", nsteps, nmeas, mask, directory.encode() if directory else None, recs, nmeas + 1,
                C.byref(n))
        return [recs[i].as_dict() for i in range(n.value)]

    # -- FFT plugin on host buffers --
    def fft_c2c(self, data: np.ndarray, sign: int) -> np.ndarray:
        a = np.ascontiguousarray(data, dtype=np.complex128).reshape(self.shape).copy()
        self._c("qx_fft_c2c", _ptr(a.view(np.float64)), sign)
        return a

    def fft_r2c(self, data: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(data, dtype=np.float64).reshape(self.shape)
        out = np.empty(self.hshape, np.complex128)
        self._c("qx_fft_r2c", _ptr(a), _ptr(out.view(np.float64)))
        return out

    def fft_c2r(self, data: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(data, dtype=np.complex128).reshape(self.hshape)
        out = np.empty(self.shape, np.float64)
        self._c("qx_fft_c2r", _ptr(a.view(np.float64)), _ptr(out))
        return out

    # -- initial conditions --
    def ic_solitons_file(self, path: str = "solitons.txt", bkg: float = 1.0):
        self._c("qx_ic_solitons_file", path.encode(), bkg)

    def ic_gaussian_solitons(self, rows, bkg: float = 1.0):
        a = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(-1, 5))
        self._c("qx_ic_gaussian_solitons", a.shape[0], _ptr(a), bkg)

    def ic_config(self, kind: int, seed: int, n_solitons: int = 0, rc_lo: float = 0.02, rc_hi: float = 0.05,
                  sigma: float = 0.3, kc_factor: float = 0.125, clip: float = -0.9, rho0: float = 1.0e-6):
        self._c("qx_ic_config", kind, seed, n_solitons, rc_lo, rc_hi, sigma, kc_factor, clip, rho0)

    # -- timing --
    def time_steps(self, nsteps: int, use_graph: bool = True) -> float:
        ms = C.c_float()
        self._c("qx_time_steps", nsteps, int(use_graph), C.byref(ms))
        return ms.value

    def profile_step(self, nsteps: int):
        names = C.create_string_buffer(64 * 16)
        ms = np.zeros(16)
        n = C.c_int()
        self._c("qx_profile_step", nsteps, 16, names, _ptr(ms), C.byref(n))
        raw = names.raw
        return [(raw[64 * i:64 * i + 64].split(b"\0")[0].decode(), float(ms[i])) for i in range(n.value)]

    def set_tune(self, x_rows: int = 0, y_tx: int = 0, la_tx: int = 0, tma: int = -1, nbuf: int = 0, pw: int = 0):
        """Launch geometry overrides (0 = default); tma 1/0 selects the TMA-fed
        persistent or the direct-load strided kernels (-1 keeps the current);
        pw: pencils per thread of the TMA passes (0 default, 1 or 2)."""
        self._c("qx_set_tune", x_rows, y_tx, la_tx, tma, nbuf, pw)

    def set_plan(self, plan: int):
        """Radix plan of the strided passes: 0 default, 1 reversed radix order
        (grids N = 64, 96, 128, 256; elsewhere it runs as 0)."""
        self._c("qx_set_plan", int(plan))

    def get_tune(self) -> dict:
        """The launch geometry in use (and whether it came from the autotuner's
        cache when the field was created)."""
        v = (C.c_int * 11)()
        self._c("qx_get_tune", v, 11)
        keys = ("x_rows", "y_tx", "la_tx", "tma", "nbuf", "pw", "plan", "chain", "pencil_warp", "from_cache",
                "row_stage")
        return dict(zip(keys, list(v)))

    def set_pencil_warp(self, on):
        """FP32 strided passes at N = 256, 512: one warp per pencil pair in
        16-column swizzled tiles for the wave-function passes (1 / True), for
        every strided pass (2), or 8-column tiles everywhere (0 / False); at
        N = 512, 3 / 4 split each pencil pair over two warps in the drift pass /
        in every wave-function pass (bit for bit 1)."""
        self._c("qx_set_pencil_warp", int(on))

    def set_row_stage(self, on):
        """FP32 inverse x + density + r2c row pass (N >= 256): 1 copies each
        warp's next row into shared memory with cp.async while the current one
        is transformed, 0 loads rows directly (bit-identical)."""
        self._c("qx_set_row_stage", int(on))

    def set_chain(self, on):
        """Drift chain: the y, z-drift, y passes of a 3D complex64 field as
        three passes (False / 0, the default, fastest) or as one slab-ordered
        kernel over 16-column (True / 2) or 8-column (1) slabs; the results
        are bit-identical."""
        self._c("qx_set_chain", 2 if on is True else int(on))

    def set_cosmology(self, cosmo: int, ai: float = 1.0):
        """0: STATIC; 1: MRE from a = ai (the reference's --cosmo mre)."""
        self._c("qx_set_cosmology", cosmo, ai)

    def cosmology(self):
        """(mode, a, ds): 0 STATIC / 1 MRE, scale factor, current time step."""
        c, a, ds = C.c_int(), C.c_double(), C.c_double()
        self._c("qx_get_cosmology", C.byref(c), C.byref(a), C.byref(ds))
        return c.value, a.value, ds.value

    def restore_cosmology(self, a: float, ds: float):
        """Restore the scale factor and time step of a checkpoint (after
        set_cosmology, which starts the cosmology afresh)."""
        self._c("qx_restore_cosmology", a, ds)

    def set_clock(self, step: int, time: float):
        """Set the step counter and time (restoring a checkpoint)."""
        self._c("qx_set_clock", step, time)

    def autotune(self, nsteps: int = 3, cache: str | None = None):
        """Pick the fastest launch geometry for this grid (psi is left as it
        was).  Returns (ms per step of the choice, whether it came from the
        cache); `cache` names a text file shared between runs."""
        ms = C.c_double()
        fc = C.c_int()
        self._c("qx_autotune", nsteps, cache.encode() if cache else None, C.byref(ms), C.byref(fc))
        return ms.value, bool(fc.value)

    def device_pointers(self):
        p, v = _vp(), _vp()
        self._c("qx_device_pointers", C.byref(p), C.byref(v))
        return p.value, v.value

    def sync(self):
        self._c("qx_sync")


def _ens_check(status: int, h):
    if status != QX_OK:
        msg = (_lib.qx_ens_last_error(h) or b"").decode(errors="replace")
        if status == QX_ERR_INVALID:
            raise ValueError(msg)
        if status == QX_ERR_NOMEM:
            raise MemoryError(msg)
        raise QxError(status, msg)


class Ensemble:
    """Independent boxes of uneven sizes advanced together (no reference
    counterpart: the reference runs one box per process, src/main.cxx:34-53).

    ``groups`` is a list of (N, count): count boxes of N^dim sites each.  Boxes
    of one size share one batched device array, so each pass of a step is one
    persistent launch over all of their tiles; groups run concurrently, each
    replaying its loop body from a CUDA graph.  With ``mixed=True`` (3D, at
    most 4 sizes from 16, 32, 64, 96, 128) the loop body of every box is
    instead ONE persistent launch per step, fed by a work queue of (pass, box,
    tile) units in which a unit starts once its box has finished the previous
    pass; ``mixed="passes"`` runs the same queue as one launch per pass.  Boxes
    are numbered group by group; box b's initial condition is seeded with
    seed_base + b.
    """

    def __init__(self, groups, dim: int = 3, L: float = 1.0, pref: float = 1.0, dtype: str = "c64",
                 dt: float | None = None, mixed: bool = False):
        ns = [int(n) for n, _ in groups]
        cs = [int(c) for _, c in groups]
        if dt is None:
            dt = 0.2 / max(ns) ** 2
        NA = (C.c_int * len(ns))(*ns)
        CA = (C.c_int * len(cs))(*cs)
        h = _vp()
        st = _lib.qx_ens_create(len(ns), NA, CA, dim, L, pref, QX_C128 if dtype == "c128" else QX_C64, dt,
                                C.byref(h))
        _ens_check(st, None)
        self._h = h
        self.dim = dim
        self.dtype = dtype
        n = C.c_int()
        sites = C.c_longlong()
        _ens_check(_lib.qx_ens_size(self._h, C.byref(n), C.byref(sites)), self._h)
        self.nboxes = n.value
        self.sites = sites.value
        self.mixed = False
        if mixed:
            self.set_mixed(mixed)

    def set_mixed(self, mode=True):
        """Loop bodies as one launch per step over all sizes (True), one launch
        per pass over all sizes ("passes") or per-size launches on concurrent
        graph branches (False); every mode advances each box as its
        single-box run does."""
        code = 2 if mode == "passes" else (1 if mode else 0)
        self._c("qx_ens_set_mixed", code)
        self.mixed = mode if code else False

    def set_mixed_window(self, nbytes: int = 0):
        """Bytes of boxes (psi + half spectrum) whose passes the one-launch
        step runs together before the next window (0: default 48 MiB; more
        than the ensemble: pass-by-pass order)."""
        self._c("qx_ens_set_mixed_window", int(nbytes))

    def close(self):
        if getattr(self, "_h", None):
            _lib.qx_ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, name, *args):
        _ens_check(getattr(_lib, name)(self._h, *args), self._h)

    def box_n(self, box: int) -> int:
        n = C.c_int()
        self._c("qx_ens_box_n", box, C.byref(n))
        return n.value

    def box_shape(self, box: int):
        return (self.box_n(box),) * self.dim

    def ic_config(self, kind: int = IC_GRF, seed_base: int = 1234, n_sol: int = 0, rc_lo: float = 0.01,
                  rc_hi: float = 0.03, sigma: float = 0.3, kc_factor: float = 0.125, clip: float = -0.9,
                  rho0: float = 1e-6, seeds=None):
        """Initial conditions of every box: box b seeded with seed_base + b, or
        with seeds[b] when a per-box seed list is given (a sharded ensemble
        passes seed_base + its boxes' global indices)."""
        if seeds is None:
            self._c("qx_ens_ic_config", kind, seed_base, n_sol, rc_lo, rc_hi, sigma, kc_factor, clip, rho0)
            return
        seeds = [int(x) for x in seeds]
        if len(seeds) != self.nboxes:
            raise ValueError(f"seeds holds {len(seeds)} values for {self.nboxes} boxes")
        arr = (C.c_ulonglong * len(seeds))(*seeds)
        self._c("qx_ens_ic_config_seeds", kind, arr, n_sol, rc_lo, rc_hi, sigma, kc_factor, clip, rho0)

    def psi(self, box: int) -> np.ndarray:
        a = np.empty(self.box_shape(box), np.complex128)
        self._c("qx_ens_get_psi", box, _ptr(a.view(np.float64)))
        return a

    def set_psi(self, box: int, value):
        a = np.ascontiguousarray(value, dtype=np.complex128).reshape(self.box_shape(box))
        self._c("qx_ens_set_psi", box, _ptr(a.view(np.float64)))

    def step(self, nsteps: int):
        self._c("qx_ens_step", nsteps)

    def time_steps(self, nsteps: int) -> float:
        ms = C.c_float()
        self._c("qx_ens_time_steps", nsteps, C.byref(ms))
        return ms.value

    def mass(self) -> np.ndarray:
        m = np.empty(self.nboxes, np.float64)
        self._c("qx_ens_mass", _ptr(m))
        return m


def shard_groups(groups, world: int, rank: int):
    """Instance sharding of an ensemble over `world` ranks with no collective:
    the boxes, numbered group by group, are dealt out round-robin, so every
    rank gets a near-equal share of every size.  Returns (groups_of_rank,
    global box indices of rank) with groups_of_rank in the (N, count) form of
    Ensemble (groups with no box on this rank are left out) and the global
    indices in the rank's local box order (Ensemble numbers its boxes group
    by group): local box i of the rank's Ensemble is global box mine[i]."""
    out, mine = [], []
    start = 0
    for n, c in groups:
        local = [b for b in range(start, start + int(c)) if b % world == rank]
        if local:
            out.append((int(n), len(local)))
            mine += local
        start += int(c)
    return out, mine


def shard_seeds(groups, world: int, rank: int, seed_base: int):
    """Per-box seeds of rank `rank`'s Ensemble (in its local box order): box b
    of the whole ensemble is seeded with seed_base + b on whichever rank runs
    it, so a sharded run simulates exactly the boxes of the unsharded one."""
    _, mine = shard_groups(groups, world, rank)
    return [seed_base + b for b in mine]
