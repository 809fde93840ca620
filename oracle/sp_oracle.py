"""FP64 CPU oracle for the Schroedinger-Poisson kick-drift-kick path.

TEST INFRASTRUCTURE.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg may import this module, and only as a checker; the product
path (qaxions_b200) never calls it.

Every function restates, with NumPy FP64 FFTs (pocketfft), the algorithm of the
reference file:line it cites.  Arrays use the reference's memory order: 3D
``psi[iz, iy, ix]`` and 2D ``psi[iy, ix]`` with x fastest
(src/ic/solitons.cxx:69-71), complex128, unnormalised FFT conventions as in
src/fft/fft.h:91-140.

Parity pins: this restatement is checked against the reference compiled here
from its own sources (oracle/Makefile -> oracle/_ref/libqx_ref.so) by
tests/test_oracle.py and against the committed fixtures in tests/golden/ that
tests/golden/make_golden.py generated from that build.

Pieces with no reference counterpart (mass, energy, Schive-profile solitons,
Gaussian random field, linear/log spectrum bins, Philox) are written from the
mathematics / the published algorithm named in each docstring.
"""
from __future__ import annotations

import math

import numpy as np

# ---------------------------------------------------------------------------
# k-grid helpers
# ---------------------------------------------------------------------------


def signed_modes(N: int) -> np.ndarray:
    """Integer wave number of FFT index i: i if i <= N/2 else i - N.

    src/field.cxx:151-153 (``(ix <= hN) ? ix : ix - N_``)."""
    i = np.arange(N)
    return np.where(i <= N // 2, i, i - N)


def k2_int(dim: int, N: int, half: bool = False) -> np.ndarray:
    """Integer |n|^2 on the full (or r2c half, last axis 0..N/2) grid, shaped
    like the reference arrays ([z,y,x] / [y,x])."""
    n = signed_modes(N)
    nx = np.arange(N // 2 + 1) if half else n
    if dim == 2:
        return (n[:, None] ** 2 + nx[None, :] ** 2).astype(np.int64)
    return (n[:, None, None] ** 2 + n[None, :, None] ** 2 + nx[None, None, :] ** 2).astype(np.int64)


# ---------------------------------------------------------------------------
# Field operations (src/field.cxx)
# ---------------------------------------------------------------------------


def kick(psi: np.ndarray, V: np.ndarray, dt: float) -> np.ndarray:
    """psi <- psi * exp(-i dt V).  src/field.cxx:93-116."""
    phase = -dt * V
    c, s = np.cos(phase), np.sin(phase)
    return (psi.real * c - psi.imag * s) + 1j * (psi.real * s + psi.imag * c)


def drift(psi: np.ndarray, dt: float, L: float = 1.0) -> np.ndarray:
    """psi <- IFFT[exp(-i dt k^2/2) FFT(psi)] with k = 2 pi n / L.

    src/field.cxx:119-198: forward c2c, multiply by the phase and 1/S, backward
    c2c (unnormalised), i.e. NumPy's normalised ifftn."""
    dim, N = psi.ndim, psi.shape[0]
    dk = 2.0 * math.pi / L
    k2 = k2_int(dim, N).astype(np.float64) * dk * dk
    phase = -0.5 * dt * k2
    h = np.fft.fftn(psi)
    h = (h.real * np.cos(phase) - h.imag * np.sin(phase)) + 1j * (h.real * np.sin(phase) + h.imag * np.cos(phase))
    return np.fft.ifftn(h)


def poisson_factor(dim: int, N: int, L: float, k0: str = "reference") -> np.ndarray:
    """Half-spectrum multiplier -1/(k^2 S) of src/field.cxx:230-291.

    k0="reference": the k=0 mode is divided by 1 (``k2 + (k2 == 0)``,
    src/field.cxx:253,282); k0="zero": the k=0 mode is set to exactly 0."""
    dk = 2.0 * math.pi / L
    S = float(N**dim)
    k2 = k2_int(dim, N, half=True).astype(np.float64) * dk * dk
    zero = k2 == 0.0
    f = -1.0 / (k2 + zero) / S
    if k0 == "zero":
        f = np.where(zero, 0.0, f)
    return f


def update_potential(psi: np.ndarray, pref: float, rho_mean: float = 1.0, L: float = 1.0,
                     k0: str = "reference"):
    """V = c2r(Poisson(r2c(pref (|psi|^2 - rho_mean)))) and Vmax = max |V|.

    src/field.cxx:294-346 (+ Poisson src/field.cxx:230-291).  Returns (V, Vmax)."""
    dim, N = psi.ndim, psi.shape[0]
    src = pref * (psi.real * psi.real + psi.imag * psi.imag - rho_mean)
    vh = np.fft.rfftn(src) * poisson_factor(dim, N, L, k0)
    V = np.fft.irfftn(vh, s=src.shape, axes=tuple(range(dim))) * float(N**dim)
    return V, float(np.max(np.abs(V)))


def compute_energy(psi: np.ndarray):
    """V <- |psi|^2 and rhomax = max|V| / mean|V|.  src/field.cxx:200-227.

    Returns (rho, rhomax)."""
    rho = psi.real * psi.real + psi.imag * psi.imag
    a = np.abs(rho)
    return rho, float(a.max() / (a.sum() / a.size))


def run(psi: np.ndarray, dt: float, nsteps: int, pref: float, rho_mean: float = 1.0,
        L: float = 1.0, k0: str = "reference"):
    """Merged KDK leapfrog of src/main.cxx:64-85 with measurements off:
    potential, half kick, nsteps x (drift, potential, full kick except after the
    last), final half kick.  Returns (psi, V)."""
    V, _ = update_potential(psi, pref, rho_mean, L, k0)
    psi = kick(psi, V, 0.5 * dt)
    for i in range(nsteps):
        psi = drift(psi, dt, L)
        V, _ = update_potential(psi, pref, rho_mean, L, k0)
        if i != nsteps - 1:
            psi = kick(psi, V, dt)
    psi = kick(psi, V, 0.5 * dt)
    return psi, V


MRE_RHO_MEAN = 1.5 * (2.0 * math.pi) ** 2 * 1.27 * 1.27


def run_mre(psi: np.ndarray, dt: float, ai: float, nsteps: int, L: float = 1.0):
    """Merged loop of src/main.cxx:64-85 in the MRE cosmology: a = ai,
    ds = dt / ai, pref = norm a with norm 1, rho_mean = 1.5 (2 pi)^2 1.27^2
    (src/field.cxx:82-88); updateTime after every drift sets ds = 0.00025 / a
    and a *= 1 + 1.27^2 sqrt(1 + a) ds (src/field.cxx:349-361); the kick after
    a drift uses the new ds.  Returns (psi, a, steps)."""
    a = ai
    ds = dt / ai
    V, _ = update_potential(psi, a, MRE_RHO_MEAN, L, "reference")
    psi = kick(psi, V, 0.5 * ds)
    for i in range(nsteps):
        psi = drift(psi, ds, L)
        ds = 0.00025 / a
        a = a * (1 + 1.27 * 1.27 * math.sqrt(1 + a) * ds)
        V, _ = update_potential(psi, a, MRE_RHO_MEAN, L, "reference")
        if i != nsteps - 1:
            psi = kick(psi, V, ds)
    psi = kick(psi, V, 0.5 * ds)
    return psi, a, nsteps


def kdk_step(psi: np.ndarray, dt: float, pref: float, rho_mean: float = 1.0, L: float = 1.0,
             k0: str = "reference"):
    """Unmerged step of src/examples/fieldtest.cxx:73-96 / Field::propagate
    (src/field.cxx:388-402): V(psi); kick dt/2; drift dt; V; kick dt/2."""
    V, _ = update_potential(psi, pref, rho_mean, L, k0)
    psi = kick(psi, V, 0.5 * dt)
    psi = drift(psi, dt, L)
    V, _ = update_potential(psi, pref, rho_mean, L, k0)
    return kick(psi, V, 0.5 * dt), V


# ---------------------------------------------------------------------------
# Spectrum (src/spectrum/spectrum.cxx)
# ---------------------------------------------------------------------------


def spectrum_reference(V: np.ndarray, L: float = 1.0):
    """Integer-shell power spectrum of a real field.

    src/spectrum/spectrum.cxx:32-164: r2c, bin b = round(|n|) < N/2+1 with
    weight 1 on the ix in {0, N/2} planes and 2 elsewhere, P += w |V^|^2 / S^2,
    count += w, P /= count, k_b = b 2pi/L.  Returns (k, P, count[int64])."""
    dim, N = V.ndim, V.shape[0]
    S = float(N**dim)
    vh = np.fft.rfftn(V)
    M = k2_int(dim, N, half=True)
    kb = np.rint(np.sqrt(M.astype(np.float64))).astype(np.int64)
    ix = np.arange(N // 2 + 1)
    w = np.where((ix == 0) | (ix == N // 2), 1, 2)
    w = np.broadcast_to(w, M.shape)
    nb = N // 2 + 1
    ok = kb < nb
    p2 = (vh.real**2 + vh.imag**2) / (S * S)
    P = np.bincount(kb[ok], weights=(w * p2)[ok], minlength=nb)
    cnt = np.bincount(kb[ok], weights=w[ok], minlength=nb).astype(np.int64)
    P = np.where(cnt > 0, P / np.maximum(cnt, 1), P)
    k = np.arange(nb) * (2.0 * math.pi / L)
    return k, P, cnt


SPEC_REFERENCE, SPEC_LINEAR, SPEC_LOG = 0, 1, 2


def spectrum_bin_table(dim: int, N: int, mode: int, nbins: int) -> np.ndarray:
    """Bin index for every integer |n|^2 = M in [0, dim (N/2)^2]; -1 = dropped.

    mode 0 (reference): round(sqrt(M)) if < N/2+1 (src/spectrum/spectrum.cxx:75-77).
    mode 1 (linear, nbins): floor(nbins |n| / (N/2)) for 0 < |n| < N/2.
    mode 2 (log, nbins): floor(nbins ln|n| / ln(N/2) + 1e-9) for 1 <= |n| < N/2.
    The 1e-9 guard makes exact bin edges (|n| = (N/2)^(b/nbins)) land in the
    upper bin regardless of the last ulp of the logarithm."""
    Mmax = dim * (N // 2) ** 2
    M = np.arange(Mmax + 1, dtype=np.float64)
    r = np.sqrt(M)
    nmax = N // 2
    if mode == SPEC_REFERENCE:
        b = np.rint(r).astype(np.int64)
        b[b >= nmax + 1] = -1
    elif mode == SPEC_LINEAR:
        b = np.floor(nbins * r / nmax).astype(np.int64)
        b[(M == 0) | (r >= nmax)] = -1
    elif mode == SPEC_LOG:
        lr = np.log(np.where(M > 0, r, 1.0))
        b = np.floor(nbins * lr / math.log(nmax) + 1e-9).astype(np.int64)
        b[(M == 0) | (r >= nmax)] = -1
    else:
        raise ValueError("unknown spectrum mode")
    b[b >= (nbins if mode != SPEC_REFERENCE else nmax + 1)] = -1
    return b


def spectrum_binned(field_hat_half: np.ndarray, dim: int, N: int, mode: int, nbins: int,
                    L: float = 1.0):
    """Shell-binned spectrum of an r2c half spectrum with the reference's
    Hermitian weights and 1/S^2 normalisation (src/spectrum/spectrum.cxx:63-155),
    using ``spectrum_bin_table`` for the bin of each mode.  Returns
    (k_centre, P, count[int64]) with P the shell average."""
    S = float(N**dim)
    tab = spectrum_bin_table(dim, N, mode, nbins)
    M = k2_int(dim, N, half=True)
    b = tab[M]
    ix = np.arange(N // 2 + 1)
    w = np.broadcast_to(np.where((ix == 0) | (ix == N // 2), 1, 2), M.shape)
    nb = (N // 2 + 1) if mode == SPEC_REFERENCE else nbins
    ok = b >= 0
    p2 = (field_hat_half.real**2 + field_hat_half.imag**2) / (S * S)
    P = np.bincount(b[ok], weights=(w * p2)[ok], minlength=nb)
    cnt = np.bincount(b[ok], weights=w[ok], minlength=nb).astype(np.int64)
    P = np.where(cnt > 0, P / np.maximum(cnt, 1), P)
    kc = spectrum_k_axis(N, mode, nbins, L)
    return kc, P, cnt


def spectrum_k_axis(N: int, mode: int, nbins: int, L: float = 1.0) -> np.ndarray:
    """Bin centres in physical k: reference b*dk (src/spectrum/spectrum.cxx:159-164);
    linear (b+1/2) (N/2)/nbins dk; log (N/2)^((b+1/2)/nbins) dk."""
    dk = 2.0 * math.pi / L
    nmax = N // 2
    if mode == SPEC_REFERENCE:
        return np.arange(nmax + 1) * dk
    b = np.arange(nbins) + 0.5
    if mode == SPEC_LINEAR:
        return b * nmax / nbins * dk
    return np.power(float(nmax), b / nbins) * dk


def density_spectrum(psi: np.ndarray, mode: int, nbins: int, L: float = 1.0):
    """Spectrum of rho = |psi|^2 -- what measure() bins after computeEnergy()
    overwrote V with rho (src/meas.cxx:30-41), computed without clobbering."""
    rho = psi.real**2 + psi.imag**2
    return spectrum_binned(np.fft.rfftn(rho), psi.ndim, psi.shape[0], mode, nbins, L)


# ---------------------------------------------------------------------------
# Diagnostics with no reference counterpart (from the mathematics)
# ---------------------------------------------------------------------------


def mass(psi: np.ndarray, L: float = 1.0) -> float:
    """M = sum |psi|^2 dV."""
    dV = (L / psi.shape[0]) ** psi.ndim
    return float(np.sum(psi.real**2 + psi.imag**2) * dV)


def energy(psi: np.ndarray, V: np.ndarray, L: float = 1.0):
    """E = K + W with K = 1/2 sum |grad psi|^2 dV evaluated spectrally
    (1/2 dV/S sum k^2 |FFT psi|^2, Parseval) and W = 1/2 sum V |psi|^2 dV.
    Returns (E, K, W)."""
    dim, N = psi.ndim, psi.shape[0]
    S = float(N**dim)
    dV = (L / N) ** dim
    dk = 2.0 * math.pi / L
    h = np.fft.fftn(psi)
    k2 = k2_int(dim, N).astype(np.float64) * dk * dk
    K = 0.5 * dV / S * float(np.sum(k2 * (h.real**2 + h.imag**2)))
    W = 0.5 * dV * float(np.sum(V * (psi.real**2 + psi.imag**2)))
    return K + W, K, W


# ---------------------------------------------------------------------------
# Initial conditions
# ---------------------------------------------------------------------------


def ic_solitons_reference(dim: int, N: int, rows, bkg: float = 1.0, L: float = 1.0) -> np.ndarray:
    """Gaussian 'solitons' IC of src/ic/solitons.cxx:20-110.

    rows: iterable of (amp, sigma, x, y, z) as in solitons.txt.  rho = bkg +
    sum amp/(2 pi sigma^3) exp(-r^2 / 2 sigma^2) with NON-periodic distances from
    (x L, y L, z L) to grid points (i dx); rho /= mean(rho); psi = sqrt(rho)."""
    dx = L / N
    c = np.arange(N) * dx
    if dim == 2:
        Y, X = np.meshgrid(c, c, indexing="ij")
        Z = np.zeros_like(X)
    else:
        Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    rho = np.full(X.shape, bkg, dtype=np.float64)
    for amp, sig, xs, ys, zs in rows:
        norm = 1.0 / (sig * sig * sig * 2.0 * math.pi)
        ddx = X - xs * L
        ddy = Y - ys * L
        ddz = (Z - zs * L) if dim == 3 else 0.0
        r2 = ddx * ddx + ddy * ddy + ddz * ddz
        rho += amp * norm * np.exp(-r2 / (2.0 * sig * sig))
    rho /= rho.sum() / rho.size
    return np.sqrt(rho).astype(np.complex128)


def read_solitons_txt(path: str):
    """Parse 'amp sigma x y z' rows as src/ic/solitons.cxx:32-50 does."""
    rows = []
    with open(path) as fh:
        for line in fh:
            v = line.split()
            if len(v) >= 5:
                rows.append(tuple(float(t) for t in v[:5]))
    return rows


# Philox4x32-10, Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy
# as 1, 2, 3", SC'11 (constants and round function as published there).
_PH_M0, _PH_M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_PH_W0, _PH_W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)


def philox4x32(c0, c1, c2, c3, k0, k1, rounds: int = 10):
    """Vectorised Philox4x32 over uint32 counter arrays; returns 4 uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint32) for x in (c0, c1, c2, c3))
    k0 = np.uint32(k0)
    k1 = np.uint32(k1)
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(rounds):
        p0 = _PH_M0 * c0.astype(np.uint64)
        p1 = _PH_M1 * c2.astype(np.uint64)
        hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & mask).astype(np.uint32)
        hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & mask).astype(np.uint32)
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = np.uint32((int(k0) + int(_PH_W0)) & 0xFFFFFFFF)
        k1 = np.uint32((int(k1) + int(_PH_W1)) & 0xFFFFFFFF)
    return c0, c1, c2, c3


def white_noise(S: int, seed: int, stream: int = 0) -> np.ndarray:
    """One standard normal per site: Philox4x32-10 with counter (site, 0,
    stream, 0) and key (seed lo, seed hi); Box-Muller cosine branch on the
    first two words, u = (w + 0.5) / 2^32."""
    idx = np.arange(S, dtype=np.uint64)
    lo = (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hi = (idx >> np.uint64(32)).astype(np.uint32)
    r0, r1, _, _ = philox4x32(lo, hi, np.full(S, stream, np.uint32), np.zeros(S, np.uint32),
                              seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u1 = (r0.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
    u2 = (r1.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def grf_delta(dim: int, N: int, seed: int, sigma: float = 0.3, kc_factor: float = 0.125,
              clip: float = -0.9, L: float = 1.0) -> np.ndarray:
    """Gaussian random density contrast: white noise filtered by sqrt(P(k)),
    P(k) = k^-2 exp(-(k/kc)^2), P(0) = 0, kc = kc_factor N (2 pi/L); rescaled to
    standard deviation sigma; clipped below at ``clip``."""
    S = N**dim
    shape = (N,) * dim
    noise = white_noise(S, seed).reshape(shape)
    dk = 2.0 * math.pi / L
    k2 = k2_int(dim, N).astype(np.float64) * dk * dk
    kc = kc_factor * N * dk
    with np.errstate(divide="ignore"):
        P = np.where(k2 > 0, np.exp(-k2 / (kc * kc)) / np.where(k2 > 0, k2, 1.0), 0.0)
    d = np.fft.ifftn(np.fft.fftn(noise) * np.sqrt(P)).real
    d *= sigma / np.sqrt(np.mean(d * d))
    return np.maximum(d, clip)


def schive_amplitude(r: np.ndarray, rc: float, rho0: float = 1.0e-6) -> np.ndarray:
    """sqrt(rho_c) / (1 + 0.091 (r/rc)^2)^4 with rho_c = rho0 rc^-4 (code units)."""
    rhoc = rho0 / rc**4
    return math.sqrt(rhoc) / (1.0 + 0.091 * (r / rc) ** 2) ** 4


def soliton_params(n: int, dim: int, seed: int, rc_lo: float, rc_hi: float):
    """Soliton list from Philox stream 1: per soliton j, counter (j, 0, 1, 0)
    gives rc ~ U[rc_lo, rc_hi) and phase ~ U[0, 2pi); counter (j, 1, 1, 0) gives
    the centre ~ U[0,1)^dim.  Returns arrays (rc, phase, centres[n,3])."""
    j = np.arange(n, dtype=np.uint32)
    a0, a1, _, _ = philox4x32(j, np.zeros(n, np.uint32), np.ones(n, np.uint32), np.zeros(n, np.uint32),
                              seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    b0, b1, b2, _ = philox4x32(j, np.ones(n, np.uint32), np.ones(n, np.uint32), np.zeros(n, np.uint32),
                               seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u = lambda w: (w.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)  # noqa: E731
    rc = rc_lo + (rc_hi - rc_lo) * u(a0)
    ph = 2.0 * math.pi * u(a1)
    cen = np.stack([u(b0), u(b1), u(b2) if dim == 3 else np.zeros(n)], axis=1)
    return rc, ph, cen


def add_schive_solitons(psi: np.ndarray, rc, phase, centres, L: float = 1.0,
                        rho0: float = 1.0e-6) -> np.ndarray:
    """psi += sum_j A(r_j; rc_j) exp(i phase_j), r_j the periodic minimum-image
    distance from grid point (i dx) to centre_j L."""
    dim, N = psi.ndim, psi.shape[0]
    dx = L / N
    c = np.arange(N) * dx
    out = psi.astype(np.complex128).copy()

    def mi(d):
        return d - L * np.rint(d / L)

    for j in range(len(rc)):
        # each axis' minimum-image term depends on that coordinate alone:
        # 1D terms broadcast over the grid (the same values, summed in the
        # same order, as full coordinate grids would give)
        ax = mi(c - centres[j, 0] * L) ** 2
        ay = mi(c - centres[j, 1] * L) ** 2
        if dim == 2:
            r2 = ax[None, :] + ay[:, None]
        else:
            az = mi(c - centres[j, 2] * L) ** 2
            r2 = (ax[None, None, :] + ay[None, :, None]) + az[:, None, None]
        out += schive_amplitude(np.sqrt(r2), rc[j], rho0) * np.exp(1j * phase[j])
    return out


def normalise_mean_density(psi: np.ndarray) -> np.ndarray:
    """Scale psi so that mean |psi|^2 = 1 (as src/ic/solitons.cxx:100-108 does
    for rho)."""
    m = np.mean(psi.real**2 + psi.imag**2)
    return psi / math.sqrt(m)


def ic_config(kind: str, dim: int, N: int, seed: int, n_solitons: int = 0,
              rc_lo: float = 0.02, rc_hi: float = 0.05, sigma: float = 0.3,
              L: float = 1.0) -> np.ndarray:
    """The synthetic initial conditions of the benchmark configurations:
    'solitons' (sum of Schive solitons, no background), 'grf' (sqrt(1+delta)),
    'grf+solitons'.  Always renormalised to mean |psi|^2 = 1."""
    if kind == "solitons":
        psi = np.zeros((N,) * dim, np.complex128)
    else:
        psi = np.sqrt(1.0 + grf_delta(dim, N, seed, sigma, L=L)).astype(np.complex128)
    if n_solitons:
        rc, ph, cen = soliton_params(n_solitons, dim, seed, rc_lo, rc_hi)
        psi = add_schive_solitons(psi, rc, ph, cen, L)
    return normalise_mean_density(psi)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b||_2 / ||b||_2."""
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))
