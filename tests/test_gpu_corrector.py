"""Learned corrector: the device forward/backward kernels against the CPU
oracle (oracle/corrector_oracle.py, BF16 rounding points emulated), training
on solver-generated pairs, and the plain-step fallback."""
import numpy as np
import pytest

import qaxions_b200 as qx
from qaxions_b200 import corrector as cr
from oracle import corrector_oracle as CO
from oracle import sp_oracle as O

pytestmark = pytest.mark.gpu


def _smooth(rng, N, amp):
    k = np.fft.fftfreq(N) * N
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    f = np.fft.ifftn(np.fft.fftn(rng.normal(size=(N, N, N))) * np.exp(-kk / 8.0)).real
    return amp * f / f.std()


@pytest.mark.parametrize("tc", [True, False])
def test_corrector_gradients_match_cpu_oracle(tc):
    """tc: the 32 -> 32 convolutions on tcgen05 (tensor memory) or mma.sync."""
    rng = np.random.default_rng(11)
    N = 16
    psi_c = (1.0 + _smooth(rng, N, 0.3) + 1j * _smooth(rng, N, 0.2)).astype(np.complex64).astype(np.complex128)
    V = _smooth(rng, N, 2.0).astype(np.float32).astype(np.float64)
    psi_f = (psi_c + 1e-3 * (_smooth(rng, N, 1.0) + 1j * _smooth(rng, N, 1.0))).astype(np.complex64).astype(np.complex128)
    fc = qx.Field(3, N, dtype="c64", k0="zero")
    ff = qx.Field(3, N, dtype="c64", k0="zero")
    fc.psi, fc.V, ff.psi = psi_c, V, psi_f
    corr = cr.Corrector(N, seed=3)
    corr.set_tensor_path(tc)
    v_scale, tau = float(np.sqrt(np.mean(V ** 2))), 1e-3
    corr.set_scales(v_scale, tau)
    loss, g = corr.gradients(fc, ff)
    y = corr.output()
    p = corr.params.astype(np.float64)
    lref, gref, yref = CO.loss_and_grads(p, psi_c.reshape(N, N, N), V.reshape(N, N, N), psi_f.reshape(N, N, N),
                                          v_scale, tau, bf=True)
    assert abs(loss - lref) <= 1e-3 * lref, (loss, lref)
    assert O.rel_l2(y.astype(np.float64), yref) <= 1e-3
    k = 0
    for ci, co in CO.DIMS:
        for n in (27 * ci * co, co):
            e = O.rel_l2(g[k:k + n].astype(np.float64), gref[k:k + n])
            assert e <= 1e-2, (ci, co, n, e)
            k += n
    # the same gradient without BF16 rounding differs only at BF16 level
    _, gfull, _ = CO.loss_and_grads(p, psi_c.reshape(N, N, N), V.reshape(N, N, N), psi_f.reshape(N, N, N),
                                    v_scale, tau, bf=False)
    assert O.rel_l2(g.astype(np.float64), gfull) <= 5e-2
    for f in (fc, ff):
        f.close()
    corr.close()


@pytest.mark.parametrize("N", [32, 96])
def test_tensor_paths_agree(N):
    """The tcgen05 kernels (convolutions on 8 x 16 x 2 bricks; weight gradients
    as im2col GEMMs; tensor-memory accumulators) and the mma.sync / CUDA-core
    kernels compute the same network: outputs agree to FP32 summation order and
    the BF16 rounding of the activations that follow, parameter gradients also
    to the BF16 rounding of dZ that the tensor-core weight gradient takes (two
    calls each, so a stale state would show)."""
    rng = np.random.default_rng(5 + N)
    psi_c = (1.0 + _smooth(rng, N, 0.3) + 1j * _smooth(rng, N, 0.2)).astype(np.complex64).astype(np.complex128)
    V = _smooth(rng, N, 2.0).astype(np.float32).astype(np.float64)
    psi_f = (psi_c + 1e-3 * (_smooth(rng, N, 1.0) + 1j * _smooth(rng, N, 1.0))).astype(np.complex64).astype(np.complex128)
    fc = qx.Field(3, N, dtype="c64", k0="zero")
    ff = qx.Field(3, N, dtype="c64", k0="zero")
    fc.psi, fc.V, ff.psi = psi_c, V, psi_f
    res = {}
    for tc in (True, False):
        corr = cr.Corrector(N, seed=9)
        corr.set_tensor_path(tc)
        corr.set_scales(float(np.sqrt(np.mean(V ** 2))), 1e-3)
        out = []
        for _ in range(2):
            loss, g = corr.gradients(fc, ff)
            out.append((loss, g.astype(np.float64), corr.output().astype(np.float64)))
        res[tc] = out
        corr.close()
    for (l1, g1, y1), (l0, g0, y0) in zip(res[True], res[False]):
        assert np.isfinite(g1).all() and np.isfinite(y1).all()
        assert abs(l1 - l0) <= 1e-4 * l0, (l1, l0)
        assert O.rel_l2(y1, y0) <= 1e-3
        assert O.rel_l2(g1, g0) <= 4e-3
    assert np.array_equal(res[True][0][1], res[True][1][1])  # deterministic
    for f in (fc, ff):
        f.close()


def test_training_reduces_the_coarse_step_error():
    # the coarse step must carry a learnable error: 32^3 with steps of 5 dx^2
    # (at 0.2 dx^2 one coarse step is within FP32 round-off of four fine ones)
    N = 32
    dt = 5.0 / N**2
    corr = cr.Corrector(N, seed=5)
    losses = cr.train(corr, seeds=[1, 2, 3, 4, 5, 6], pairs_per_seed=40, dt=dt, lr=3e-3, n_sol=4)
    assert np.mean(losses[-20:]) < 0.85 * np.mean(losses[:5]), (losses[:5], np.mean(losses[-20:]))
    # unseen seed: one coarse step (+ correction) against four fine steps
    st = qx.Field(3, N, dtype="c64", k0="zero", dt=dt)
    cs = qx.Field(3, N, dtype="c64", k0="zero", dt=4 * dt)
    st.ic_config(qx.IC_GRF, 99, 4, 0.01, 0.03)
    st.step(8)
    cr.make_pair(st, cs, dt)
    fine, coarse = st.psi, cs.psi
    corr.apply(cs)
    corrected = cs.psi
    e_coarse = O.rel_l2(coarse, fine)
    e_corr = O.rel_l2(corrected, fine)
    assert e_corr < 0.9 * e_coarse, (e_coarse, e_corr)
    for f in (st, cs):
        f.close()
    corr.close()


def test_fallback_redoes_failed_steps_as_plain_steps():
    N = 32
    dt = 0.2 / N**2
    corr = cr.Corrector(N, seed=1)
    corr.set_scales(1.0, 1e-3)
    a = qx.Field(3, N, dtype="c64", k0="zero", dt=dt)
    b = qx.Field(3, N, dtype="c64", k0="zero", dt=dt)
    a.ic_config(qx.IC_GRF, 4, 2, 0.01, 0.03)
    b.ic_config(qx.IC_GRF, 4, 2, 0.01, 0.03)
    nf = cr.corrected_steps(a, corr, 3, dt, tol=0.0)  # every corrected step rejected
    assert nf == 3
    for _ in range(3):
        b.step(4)
    assert O.rel_l2(a.psi, b.psi) == 0.0
    nf = cr.corrected_steps(a, corr, 2, dt, tol=np.inf)  # never rejected
    assert nf == 0
    for f in (a, b):
        f.close()
    corr.close()
