"""The corrector oracle's backward pass against central finite differences of
its own loss (FP64, no BF16 rounding), on a small periodic grid."""
import numpy as np

from oracle import corrector_oracle as CO


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    N = 4
    psi_c = 1.0 + 0.2 * (rng.normal(size=(N, N, N)) + 1j * rng.normal(size=(N, N, N)))
    V = rng.normal(size=(N, N, N))
    psi_f = psi_c + 1e-3 * (rng.normal(size=(N, N, N)) + 1j * rng.normal(size=(N, N, N)))
    p = 0.1 * rng.normal(size=CO.nparams())
    loss, g, _ = CO.loss_and_grads(p, psi_c, V, psi_f, 1.0, 1e-3, bf=False)
    idx = rng.choice(CO.nparams(), size=24, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = CO.loss_and_grads(pp, psi_c, V, psi_f, 1.0, 1e-3, bf=False)[0]
        lm = CO.loss_and_grads(pm, psi_c, V, psi_f, 1.0, 1e-3, bf=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-5 * abs(fd), (i, fd, g[i])
