"""Learned corrector for coarse time steps (no counterpart in the reference).

One merged KDK step at 4 dt followed by a correction predicted by a small
periodic convolutional network replaces four KDK steps at dt.  The network
(C ABI qx_corr_*, kernels in qaxions_b200/csrc/qx_corrector.cu) is trained on
the GPU by the project's own forward and backward kernels on pairs the solver
generates itself: from a state psi_0, psi_c = one step at 4 dt, psi_f = four
steps at dt; the target is (psi_f - psi_c) / tau.

A corrected step keeps the mass exactly (the corrected state is rescaled to
the mass before the step, which the exact dynamics conserve) and is judged by
its energy drift: a step whose |dE/E| exceeds `tol` is discarded and redone as
four plain steps (the fallback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import Field, IC_GRF, QX_OK, QX_ERR_INVALID, QX_ERR_NOMEM, QxError, _lib, _vp

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_SIGS = {
    "qx_corr_create": ([C.c_int, C.c_ulonglong, C.POINTER(_vp)], C.c_int),
    "qx_corr_destroy": ([_vp], C.c_int),
    "qx_corr_last_error": ([_vp], C.c_char_p),
    "qx_corr_nparams": ([_vp, C.POINTER(C.c_int)], C.c_int),
    "qx_corr_set_scales": ([_vp, C.c_double, C.c_double], C.c_int),
    "qx_corr_set_tensor_path": ([_vp, C.c_int], C.c_int),
    "qx_corr_get_scales": ([_vp, _dp, _dp], C.c_int),
    "qx_corr_get_params": ([_vp, _fp], C.c_int),
    "qx_corr_set_params": ([_vp, _fp], C.c_int),
    "qx_corr_gradients": ([_vp, _vp, _vp, _vp, _fp, _dp], C.c_int),
    "qx_corr_train_pair": ([_vp, _vp, _vp, _vp, C.c_double, _dp], C.c_int),
    "qx_corr_apply": ([_vp, _vp, _vp, _vp], C.c_int),
    "qx_corr_output": ([_vp, _fp], C.c_int),
    "qx_copy_psi": ([_vp, _vp], C.c_int),
    "qx_psi_changed": ([_vp], C.c_int),
    "qx_scale_psi": ([_vp, C.c_double], C.c_int),
}
for _n, (_a, _r) in _SIGS.items():
    _f = getattr(_lib, _n)
    _f.argtypes = _a
    _f.restype = _r


def _check(st, h):
    if st != QX_OK:
        msg = (_lib.qx_corr_last_error(h) or b"").decode(errors="replace")
        if st == QX_ERR_INVALID:
            raise ValueError(msg)
        if st == QX_ERR_NOMEM:
            raise MemoryError(msg)
        raise QxError(st, msg)


def _fcheck(st, h):
    if st != QX_OK:
        msg = (_lib.qx_last_error(h) or b"").decode(errors="replace")
        if st == QX_ERR_INVALID:
            raise ValueError(msg)
        raise QxError(st, msg)


def _ptrs(f: Field):
    psi, V = f.device_pointers()
    return C.c_void_p(psi), C.c_void_p(V)


def copy_psi(dst: Field, src: Field):
    _fcheck(_lib.qx_copy_psi(dst._h, src._h), dst._h)


def psi_changed(f: Field):
    _fcheck(_lib.qx_psi_changed(f._h), f._h)


def scale_psi(f: Field, factor: float):
    _fcheck(_lib.qx_scale_psi(f._h, factor), f._h)


class Corrector:
    """Network for N^3 complex64 fields (N a multiple of 8)."""

    def __init__(self, N: int, seed: int = 0):
        h = _vp()
        _check(_lib.qx_corr_create(N, seed, C.byref(h)), None)
        self._h = h
        self.N = N
        n = C.c_int()
        _check(_lib.qx_corr_nparams(self._h, C.byref(n)), self._h)
        self.nparams = n.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.qx_corr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, name, *args):
        _check(getattr(_lib, name)(self._h, *args), self._h)

    @property
    def params(self) -> np.ndarray:
        p = np.empty(self.nparams, np.float32)
        self._c("qx_corr_get_params", p.ctypes.data_as(_fp))
        return p

    @params.setter
    def params(self, p):
        a = np.ascontiguousarray(p, dtype=np.float32)
        if a.size != self.nparams:
            raise ValueError(f"expected {self.nparams} parameters")
        self._c("qx_corr_set_params", a.ctypes.data_as(_fp))

    def set_tensor_path(self, tc: bool):
        """32 -> 32 convolutions on tcgen05 (True, default) or mma.sync (False)."""
        self._c("qx_corr_set_tensor_path", int(bool(tc)))

    def set_scales(self, v_scale: float, tau: float):
        self._c("qx_corr_set_scales", v_scale, tau)

    def scales(self):
        a, b = C.c_double(), C.c_double()
        self._c("qx_corr_get_scales", C.byref(a), C.byref(b))
        return a.value, b.value

    def gradients(self, coarse: Field, fine: Field):
        """Loss and parameter gradient of the pair (coarse result, fine result)."""
        pc, vc = _ptrs(coarse)
        pf, _ = _ptrs(fine)
        g = np.empty(self.nparams, np.float32)
        loss = C.c_double()
        self._c("qx_corr_gradients", pc, vc, pf, g.ctypes.data_as(_fp), C.byref(loss))
        return loss.value, g

    def train_pair(self, coarse: Field, fine: Field, lr: float) -> float:
        pc, vc = _ptrs(coarse)
        pf, _ = _ptrs(fine)
        loss = C.c_double()
        self._c("qx_corr_train_pair", pc, vc, pf, lr, C.byref(loss))
        return loss.value

    def apply(self, f: Field):
        """psi += tau * net(psi, V) in place (V must be the potential of psi)."""
        p, v = _ptrs(f)
        self._c("qx_corr_apply", p, v, C.c_void_p(0))
        f.sync()
        psi_changed(f)

    def output(self) -> np.ndarray:
        y = np.empty((self.N, self.N, self.N, 2), np.float32)
        self._c("qx_corr_output", y.ctypes.data_as(_fp))
        return y


def make_pair(state: Field, coarse: Field, dt: float):
    """coarse <- one step at 4 dt from state; state <- four steps at dt."""
    copy_psi(coarse, state)
    coarse.set_dt(4 * dt)
    coarse.step(1)
    state.set_dt(dt)
    state.step(4)


def train(corr: Corrector, seeds, pairs_per_seed: int, dt: float, lr: float = 1e-3, n_sol: int = 16,
          warm_steps: int = 8, log=None):
    """Online training on solver-generated pairs at the corrector's grid size:
    for each seed, a GRF + n_sol soliton state is advanced pair by pair (the
    fine result of one pair is the start of the next).  The scales (v_scale =
    rms V, tau = rms of the first target) are fixed from the first pair.
    Returns the per-pair losses."""
    N = corr.N
    losses = []
    first = True
    for seed in seeds:
        st = Field(3, N, dtype="c64", k0="zero", dt=dt)
        cs = Field(3, N, dtype="c64", k0="zero", dt=4 * dt)
        st.ic_config(IC_GRF, int(seed), n_sol, 0.01, 0.03)
        st.step(warm_steps)
        for _ in range(pairs_per_seed):
            make_pair(st, cs, dt)
            if first:
                d = st.psi - cs.psi
                tau = float(np.sqrt(np.mean(np.abs(d) ** 2)))
                v_scale = float(np.sqrt(np.mean(cs.V ** 2)))
                corr.set_scales(max(v_scale, 1e-30), max(tau, 1e-30))
                first = False
            losses.append(corr.train_pair(cs, st, lr))
            if log is not None:
                log(len(losses), losses[-1])
        st.close()
        cs.close()
    return losses


def corrected_steps(f: Field, corr: Corrector, n: int, dt: float, tol: float = 1e-6, backup: Field = None):
    """Advance f by n coarse steps of 4 dt, each corrected by the network, the
    mass restored exactly, and judged by |dE/E| <= tol; a step that fails is
    redone from its start as four plain steps of dt.  Returns the number of
    fallbacks."""
    own = backup is None
    if own:
        backup = Field(f.dim_, f.N_, dtype="c64", k0="zero", dt=dt)
    fallbacks = 0
    for _ in range(n):
        copy_psi(backup, f)
        M0, E0, _, _ = f.mass_energy()
        f.set_dt(4 * dt)
        f.step(1)
        corr.apply(f)
        M1 = f.mass_energy()[0]
        scale_psi(f, float(np.sqrt(M0 / M1)))
        E1 = f.mass_energy()[1]
        if not np.isfinite(E1) or abs(E1 - E0) > tol * abs(E0):
            copy_psi(f, backup)
            f.set_dt(dt)
            f.step(4)
            fallbacks += 1
    f.set_dt(dt)
    if own:
        backup.close()
    return fallbacks
