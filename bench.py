"""Benchmark: site-updates/s of the fused FP32 KDK step at 3D 512^3 on B200.

Workload (the 512^3 configuration): periodic box L = 1, psi = sqrt(1+delta)
with delta a Gaussian random field (P(k) ~ k^-2 exp(-(k/kc)^2), kc = N/8 * 2pi,
sigma 0.3, clipped at -0.9) plus 32 Schive-profile solitons (rc ~ U[0.01,
0.03)), mean |psi|^2 = 1, pref = 4 pi G = 1, dt = 0.2 dx^2.  Synthetic data,
seeded (Philox4x32-10), generated on the device in FP64.

A "step" is one merged kick-drift-kick step (Field::drift_update +
Field::full_kick of the reference's time loop) through qx_step: eight fused
HBM passes over the 1 GiB complex64 state (inputs larger than L2 -- no
flush needed).  The plain FP64 form (complex128) is measured the same way and
reported beside it.  Only one box per GPU: a single box does not shard, so N > 1
runs N independent replicas ("weak" scaling, no collective on the data path).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 512
DIM = 3
N_SOL = 32
SEED = 1234
METRIC = "site-updates/s @512^3 (fused FP32 KDK step, 1 B200)"
UNIT = "site-updates/s"
# algorithmic HBM bytes per site of one fused loop-body pass, w = bytes/real
PASS_BYTES_W = {
    "y_fwd(psi)": 4, "z_drift(psi)": 4, "y_inv(psi)": 4, "x_inv_r2c(psi->rho^)": 5,
    "y_fwd(rho^)": 2, "z_poisson(rho^)": 2, "y_inv(rho^)": 2, "x_c2r_kick_fwd": 5,
}
ROOFLINE_BYTES_W = 26  # graded per-site minimum of the whole step (26 w)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier_sync(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_field(qx, dtype, dt):
    f = qx.Field(DIM, N_GRID, L=1.0, pref=1.0, rho_mean=1.0, dtype=dtype, k0="zero" if dtype == "c64" else "reference",
                 dt=dt)
    f.ic_config(qx.IC_GRF, SEED, N_SOL, 0.01, 0.03)
    return f


def time_form(qx, dtype, dt, K, W, world, device, sample_clocks=False, autotune=True):
    f = make_field(qx, dtype, dt)
    tune = None
    if autotune:
        # the autotuner times each candidate launch geometry for a few steps and
        # keeps the fastest (state restored); later fields of this grid reuse it
        t_ms, cached = f.autotune(4)
        tune = dict(f.get_tune(), tuned_ms_per_step=t_ms)
    f.step(W)                     # warm-up (also captures the loop-body graph)
    barrier_sync(world)
    clocks = None
    if sample_clocks:
        with ClockSampler(device) as cs:
            ms = f.time_steps(K, True)
        clocks = cs.summary()
    else:
        ms = f.time_steps(K, True)
    barrier_sync(world)
    ms = max_over_ranks(ms, world)
    return f, ms, clocks, tune


def cpu_baseline(psi0, dt, budget_s=20.0):
    """The reference's own CPU path (oracle/_ref: its field/spectrum/IC sources
    + project FFTW shim, OpenMP on every host core): loop-body steps
    (Field::drift_update + Field::full_kick) of the same 512^3 state."""
    from oracle import ref_lib as R
    if not R.available():
        return None
    cores = os.cpu_count()
    f = R.RefField(DIM, N_GRID, 1.0, 1.0 / (4.0 * math.pi), dt, cores)
    f.set_psi(psi0)
    f.update_potential()
    f.half_kick()
    n, t = 0, 0.0
    while n < 1 or (t < budget_s and n < 3):
        t0 = time.perf_counter()
        f.loop_body(1)
        t += time.perf_counter() - t0
        n += 1
    cal = fft_calibration(f, cores)
    f.close()
    S = N_GRID ** DIM
    out = {"value": S * n / t, "unit": UNIT, "cores": cores, "kind": "reference",
           "sample": f"{n} KDK loop-body step(s) of the 512^3 state (complex128, reference loops + project FFTW shim)",
           "s_per_step": t / n, "fft_calibration": cal}
    if cal and cal.get("shim_over_scipy"):
        # a loop-body step runs 2 c2c + 1 r2c + 1 c2r (about 3 c2c of work): the
        # step time with an FFT as fast as scipy's instead of the shim's
        t_fast = max(t / n - 3.0 * (cal["shim_c2c_s"] - cal["scipy_c2c_s"]), 1e-9)
        out["value_if_fft_as_fast_as_scipy"] = S / t_fast
    return out


def fft_calibration(ref_field, cores):
    """How fast the project FFTW shim (the reference build's FFT) is: one
    forward 512^3 complex128 c2c through the reference's FFT plugin, beside
    scipy.fft.fftn (pocketfft, `cores` worker threads) on the same array."""
    try:
        import ctypes as C

        import scipy.fft as sf

        from oracle import ref_lib as R
    except ImportError:
        return None
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((N_GRID,) * DIM) + 1j * rng.standard_normal((N_GRID,) * DIM)).astype(np.complex128)
    y = x.copy()
    t0 = time.perf_counter()
    R.lib().ref_fft_forward_c2c(ref_field.h, y.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    t_shim = time.perf_counter() - t0
    sf.fftn(x[:64, :64, :64], workers=cores)  # warm the plan cache
    t0 = time.perf_counter()
    z = sf.fftn(x, workers=cores, overwrite_x=False)
    t_sc = time.perf_counter() - t0
    err = float(np.linalg.norm(z - y) / np.linalg.norm(z))
    del x, y, z
    return {"grid": N_GRID, "shim_c2c_s": t_shim, "scipy_c2c_s": t_sc, "shim_over_scipy": t_shim / t_sc,
            "relL2_shim_vs_scipy": err, "workers": cores}


def run_reference_arm(args, world, rank):
    """--impl reference: the reference's CPU implementation of the path on the
    host cores (oracle/_ref built from its sources)."""
    if rank != 0:
        return
    from oracle import ref_lib as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libqx_ref.so missing"}))
        return
    from oracle import sp_oracle as O
    cores = os.cpu_count()
    N = N_GRID
    dt = 0.2 / N**2
    # same workload; the IC is built with the oracle's FP64 generator at 512^3
    # would take minutes in NumPy, so the box state is a smooth GRF-like field
    # of the same size (the step's cost does not depend on the values)
    rng = np.random.default_rng(SEED)
    psi = (1.0 + 0.05 * rng.standard_normal((N,) * DIM)).astype(np.complex128)
    psi = O.normalise_mean_density(psi)
    f = R.RefField(DIM, N, 1.0, 1.0 / (4.0 * math.pi), dt, cores)
    f.set_psi(psi)
    del psi
    f.update_potential()
    f.half_kick()
    t0 = time.perf_counter()
    f.loop_body(1)
    t_one = time.perf_counter() - t0
    sample_n = N
    total = t_one * (args.steps + args.warmup)
    if total > 240.0:  # keep the arm within a few minutes: one 256^3 box per step
        f.close()
        sample_n = 256
        f = R.RefField(DIM, sample_n, 1.0, 1.0 / (4.0 * math.pi), 0.2 / sample_n**2, cores)
        f.set_psi(np.ones((sample_n,) * DIM, np.complex128))
        f.update_potential()
        f.half_kick()
    for _ in range(max(0, args.warmup - 1)):
        f.loop_body(1)
    t0 = time.perf_counter()
    f.loop_body(args.steps)
    t = time.perf_counter() - t0
    f.close()
    S = sample_n ** DIM
    value = S * args.steps / t
    sample = f"one KDK loop-body step of a {sample_n}^3 complex128 box per step"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "3D 512^3 Schroedinger-Poisson KDK step", "grid": N_GRID, "dim": DIM,
                   "sample_grid": sample_n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def e2e_run(qx, dt, K, host_in, host_out, world):
    """Through the C ABI with pinned host buffers: upload psi0, K steps,
    download psi (the copies are inside the timed region)."""
    f = qx.Field(DIM, N_GRID, L=1.0, pref=1.0, dtype="c64", k0="zero", dt=dt)
    f.set_psi_ptr(host_in)
    f.step(2)
    barrier_sync(world)
    t0 = time.perf_counter()
    f.set_psi_ptr(host_in)
    f.step(K)
    f.get_psi_ptr(host_out)
    t = time.perf_counter() - t0
    barrier_sync(world)
    f.close()
    return max_over_ranks(t, world)


ENSEMBLE = [(64, 16), (96, 16), (128, 16)]


def run_ensemble(args, world, rank, local):
    """Ensemble workload: 48 independent GRF boxes (16 x 64^3, 16 x 96^3 with
    radix 3, 16 x 128^3), box b seeded 1234 + b, dt = 0.2 dx^2 of the finest
    grid.  Boxes are dealt out to ranks (instance sharding, no collective in
    the step); value = all ranks' sites x steps / max-over-ranks device time."""
    import torch

    import qaxions_b200 as qx
    qx.set_device(local)
    groups, mine = qx.shard_groups(ENSEMBLE, world, rank)
    seeds = [1234 + b for b in mine]  # every box keeps its global seed on any rank
    dt = 0.2 / 128**2
    K, W = args.steps, args.warmup
    res = {}
    # mixed: one persistent launch per pass over the boxes of all sizes (work
    # queue); per_size: one launch per pass per size, sizes on graph branches
    for mixed in (True, "passes", False):
        for dtype in ("c64", "c128"):
            e = qx.Ensemble(groups, dtype=dtype, dt=dt, mixed=mixed)
            e.ic_config(qx.IC_GRF, seeds=seeds)
            e.step(W)
            barrier_sync(world)
            ms = e.time_steps(K)
            t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
            sites = torch.tensor([float(e.sites)], dtype=torch.float64, device=f"cuda:{local}")
            if world > 1:
                import torch.distributed as dist
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                dist.all_reduce(sites, op=dist.ReduceOp.SUM)
            res[(mixed, dtype)] = (float(t.item()), float(sites.item()))
            e.close()
    acc = None
    if rank == 0 and args.accuracy_steps > 0:
        a = qx.Ensemble(groups, dtype="c128", dt=dt, mixed=True)
        b = qx.Ensemble(groups, dtype="c64", dt=dt, mixed=True)
        a.ic_config(qx.IC_GRF, seeds=seeds)
        b.ic_config(qx.IC_GRF, seeds=seeds)
        a.step(args.accuracy_steps)
        b.step(args.accuracy_steps)
        errs = [float(np.linalg.norm(b.psi(i) - a.psi(i)) / np.linalg.norm(a.psi(i))) for i in range(a.nboxes)]
        ma, mb = a.mass(), b.mass()
        acc = {"steps": args.accuracy_steps, "relL2_psi_fp32_vs_fp64_max_over_boxes": max(errs),
               "relL2_psi_fp32_vs_fp64_mean": float(np.mean(errs)),
               "mass_drift_fp32_max": float(np.max(np.abs(mb - 1.0))), "mass_drift_fp64_max": float(np.max(np.abs(ma - 1.0)))}
        a.close()
        b.close()
    if rank == 0:
        ms32, sites = res[("passes", "c64")]
        ms64, _ = res[("passes", "c128")]
        ps32, _ = res[(False, "c64")]
        ps64, _ = res[(False, "c128")]
        st32, _ = res[(True, "c64")]
        st64, _ = res[(True, "c128")]
        value = sites * K / (ms32 / 1e3)
        print(json.dumps({
            "metric": "site-updates/s (ensemble 16x64^3 + 16x96^3 + 16x128^3, fused FP32 KDK)",
            "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms32 / K,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic",
            "config": {"workload": "ensemble of 48 GRF boxes (16x64^3, 16x96^3, 16x128^3), seeds 1234+b",
                       "sites": sites, "parallelism": f"instance sharding x{world}",
                       "passes": "one persistent launch per pass over the boxes of all sizes, driven by a work "
                                 "queue of (box, tile) units, costliest sizes first",
                       "l2": "state 415 MB complex64, larger than L2"},
            "plain_fp64": {"value": sites * K / (ms64 / 1e3), "ms_per_step": ms64 / K},
            "launch_per_step": {"value": sites * K / (st32 / 1e3), "ms_per_step": st32 / K,
                                "plain_fp64_value": sites * K / (st64 / 1e3), "plain_fp64_ms_per_step": st64 / K,
                                "what": "the loop body of every box as ONE persistent launch per step: a queue of "
                                        "(pass, box, tile) units, a unit waiting only for its box's previous pass"},
            "per_size_launches": {"value": sites * K / (ps32 / 1e3), "ms_per_step": ps32 / K,
                                  "plain_fp64_value": sites * K / (ps64 / 1e3), "plain_fp64_ms_per_step": ps64 / K,
                                  "what": "one launch per pass per size, the sizes on concurrent graph branches"},
            "accuracy": acc}), flush=True)


def run_corrector(args, world, rank, local):
    """Learned-corrector workload (3D 256^3 GRF + 16 solitons, complex64):
    the network is trained on pairs from 16 seeds at 128^3 (same dt / dx^2),
    then one coarse step at 4 dt + correction is compared with four fused fine
    steps and with the coarse step alone: errors against a plain FP64 fine run
    after the same simulated time, and simulated time per wall-second."""
    if rank != 0:
        return
    import time as _t

    import qaxions_b200 as qx
    from qaxions_b200 import corrector as cr
    qx.set_device(local)
    N, NT = 256, 128
    dt, dtt = 0.2 / N**2, 0.2 / NT**2
    ncoarse = max(args.steps, 4)
    corr_t = cr.Corrector(NT, seed=1)
    t0 = _t.time()
    losses = cr.train(corr_t, seeds=list(range(1, 17)), pairs_per_seed=args.corr_pairs, dt=dtt, lr=2e-3, n_sol=16)
    t_train = _t.time() - t0
    corr = cr.Corrector(N, seed=0)
    corr.params = corr_t.params
    corr.set_scales(*corr_t.scales())
    corr_t.close()

    def field(dtype, d):
        f = qx.Field(3, N, dtype=dtype, k0="zero", dt=d)
        f.ic_config(qx.IC_GRF, 1234, 16, 0.01, 0.03)
        return f

    ref = field("c128", dt)
    ref.step(4 * ncoarse)
    pref_ = ref.psi
    M0 = 1.0
    fine = field("c64", dt)
    fine.step(4 * ncoarse)
    coarse = field("c64", 4 * dt)
    coarse.step(ncoarse)
    corrd = field("c64", dt)
    fb = cr.corrected_steps(corrd, corr, ncoarse, dt, tol=1e-6)
    errs = {k: float(np.linalg.norm(f.psi - pref_) / np.linalg.norm(pref_)) for k, f in
            (("fine_fp32", fine), ("coarse_fp32", coarse), ("corrected_fp32", corrd))}
    mass = {k: abs(f.mass_energy()[0] - M0) for k, f in
            (("fine_fp32", fine), ("coarse_fp32", coarse), ("corrected_fp32", corrd))}
    # timing (device events for the plain forms; wall clock around the corrected loop)
    ms_fine = fine.time_steps(20, True) / 20
    coarse.set_dt(4 * dt)
    ms_coarse = coarse.time_steps(20, True) / 20
    corrd.sync()
    t0 = _t.time()
    for _ in range(5):
        corrd.set_dt(4 * dt)
        corrd.step(1)
        corr.apply(corrd)
    corrd.sync()
    ms_net_step = (_t.time() - t0) / 5 * 1e3
    t0 = _t.time()
    cr.corrected_steps(corrd, corr, 3, dt, tol=np.inf)
    ms_checked = (_t.time() - t0) / 3 * 1e3
    sim = {"fine_fp32": dt / (ms_fine * 1e-3), "coarse_fp32": 4 * dt / (ms_coarse * 1e-3),
           "corrected_fp32": 4 * dt / (ms_net_step * 1e-3),
           "corrected_fp32_with_checks": 4 * dt / (ms_checked * 1e-3)}
    print(json.dumps({
        "metric": "simulated time per wall-second, learned-corrector form vs fused form (256^3)",
        "value": sim["corrected_fp32"] / sim["fine_fp32"], "unit": "x fused form",
        "n_gpus": 1, "steps": ncoarse, "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 + bf16 network", "data": "synthetic",
        "config": {"workload": "3D 256^3 GRF + 16 Schive solitons, dt = 0.2 dx^2, coarse 4 dt",
                   "train": f"128^3, 16 seeds x {args.corr_pairs} pairs, Adam 2e-3, {t_train:.1f} s",
                   "loss_first": losses[0], "loss_last10": float(np.mean(losses[-10:]))},
        "errors_vs_fp64_fine": errs, "mass_drift": mass, "fallbacks": fb, "coarse_steps": ncoarse,
        "ms": {"fused_fine_step": ms_fine, "coarse_step": ms_coarse, "coarse_step_plus_network": ms_net_step,
               "corrected_step_with_mass_energy_checks": ms_checked},
        "sim_time_per_wall_s": sim}), flush=True)
    for f in (ref, fine, coarse, corrd):
        f.close()
    corr.close()


def run_report(args, world, rank, local):
    """Error report of the fused FP32 form against the plain FP64 form (which
    the GPU tests hold to <= 1e-12 of the CPU reference) for the 2D and 128^3
    configurations: psi, potential, mass, energy and P(k) errors."""
    if rank != 0:
        return
    import qaxions_b200 as qx
    qx.set_device(local)
    out = {}
    for name, dim, N, ic, nsteps, every, nbins in (
            ("2D 256^2, 8 Schive solitons, 500 steps, 64 linear P(k) bins every 50", 2, 256, qx.IC_SOLITONS, 500, 50, 64),
            ("3D 128^3 GRF, 2000 steps, 64 linear P(k) bins every 200", 3, 128, qx.IC_GRF, 2000, 200, 64)):
        dt = 0.2 / N**2
        f = {}
        for dtype in ("c128", "c64"):
            g = qx.Field(dim, N, pref=1.0, dtype=dtype, k0="zero", dt=dt)
            if ic == qx.IC_SOLITONS:
                g.ic_config(ic, 1234, 8, 0.02, 0.05)
            else:
                g.ic_config(ic, 1234, 0, 0.01, 0.03)
            f[dtype] = g
        M0, E0, _, _ = f["c128"].mass_energy()
        pk_err = 0.0
        done = 0
        while done < nsteps:
            for g in f.values():
                g.step(every)
            done += every
            _, pa, ca = f["c128"].spectrum(0, qx.SPEC_LINEAR, nbins)
            _, pb, _ = f["c64"].spectrum(0, qx.SPEC_LINEAR, nbins)
            sel = (ca > 0) & (pa > 1e-12 * pa.max())
            pk_err = max(pk_err, float(np.max(np.abs(pb[sel] - pa[sel]) / pa[sel])))
        a, b = f["c128"], f["c64"]
        Ma, Ea, _, _ = a.mass_energy()
        Mb, Eb, _, _ = b.mass_energy()
        Va, Vb = a.V, b.V
        out[name] = {
            "relL2_psi": float(np.linalg.norm(b.psi - a.psi) / np.linalg.norm(a.psi)),
            "relL2_V": float(np.linalg.norm((Vb - Vb.mean()) - (Va - Va.mean())) / np.linalg.norm(Va - Va.mean())),
            "mass_drift_fp32": abs(Mb - M0) / M0, "mass_drift_fp64": abs(Ma - M0) / M0,
            "energy_drift_fp32": abs(Eb - E0) / abs(E0), "energy_drift_fp64": abs(Ea - E0) / abs(E0),
            "Pk_max_rel_err": pk_err}
        for g in f.values():
            g.close()
    print(json.dumps({"metric": "FP32 (fused) vs FP64 (plain) error report", "configs": out}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--accuracy-steps", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="time the default launch geometry")
    ap.add_argument("--workload", default="kdk512", choices=["kdk512", "ensemble", "corrector", "report"],
                    help="kdk512: the 512^3 single-box step (default); ensemble: 16x64^3 + 16x96^3 + 16x128^3 "
                         "boxes; corrector: learned-corrector form at 256^3")
    ap.add_argument("--corr-pairs", type=int, default=8, help="training pairs per seed (corrector workload)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    if args.workload == "report" and args.impl == "ours":
        run_report(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "corrector" and args.impl == "ours":
        run_corrector(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "ensemble" and args.impl == "ours":
        run_ensemble(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch

    import qaxions_b200 as qx
    qx.set_device(local)
    K, W = args.steps, args.warmup
    S = N_GRID ** DIM
    dt = 0.2 / N_GRID**2
    hbm, peak_kind = peaks()

    # ---- fused FP32 form (the headline) ----
    f32, ms32, clocks, tune32 = time_form(qx, "c64", dt, K, W, world, local, sample_clocks=True,
                                          autotune=not args.no_autotune)
    prof = f32.profile_step(max(3, min(K, 10)))
    f32.close()
    # ---- plain FP64 form ----
    f64, ms64, _, tune64 = time_form(qx, "c128", dt, K, W, world, local, autotune=not args.no_autotune)
    f64.close()

    value = world * S * K / (ms32 / 1e3)
    value64 = world * S * K / (ms64 / 1e3)
    ms_step = ms32 / K

    # ---- roofline of the dominant pass ----
    w = 4
    top = max(prof, key=lambda p: p[1])
    per_pass = []
    for name, t in prof:
        b = PASS_BYTES_W.get(name, 0) * w * S
        per_pass.append({"pass": name, "us": 1e3 * t, "alg_bytes": b, "gbs": b / (t * 1e-3) / 1e9})
    top_b = PASS_BYTES_W[top[0]] * w * S
    achieved = top_b / (top[1] * 1e-3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_512.txt")
    if os.path.exists(tfile):
        for line in open(tfile):
            p = line.split()
            if len(p) >= 2 and p[0] == top[0]:
                traffic = float(p[1])
    step_bytes = sum(PASS_BYTES_W.values()) * w * S
    roofline = {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": top_b, "launch_us": 1e3 * top[1], "per_pass": per_pass,
                "step_alg_bytes": step_bytes, "step_gbs": step_bytes / (ms_step * 1e-3) / 1e9,
                "graded_roofline_26w": {
                    "bytes_per_site": ROOFLINE_BYTES_W * w,
                    "frac_of_8TBs": ROOFLINE_BYTES_W * w * S / (ms_step * 1e-3) / 8e12,
                    "frac_of_peak": ROOFLINE_BYTES_W * w * S / (ms_step * 1e-3) / (hbm * 1e9),
                    "peak_kind": peak_kind}}

    # ---- accuracy after --accuracy-steps (FP32 vs FP64 plain form, same IC) ----
    acc = None
    if rank == 0 and args.accuracy_steps > 0:
        a = make_field(qx, "c128", dt)
        b = make_field(qx, "c64", dt)
        M0, E0, _, _ = a.mass_energy()
        a.step(args.accuracy_steps)
        b.step(args.accuracy_steps)
        pa, pb = a.psi, b.psi
        Va, Vb = a.V, b.V
        Ma, Ea, _, _ = a.mass_energy()
        Mb, Eb, _, _ = b.mass_energy()
        ka, Pa, ca = a.spectrum(0, qx.SPEC_LOG, 256)
        kb, Pb, cb = b.spectrum(0, qx.SPEC_LOG, 256)
        sel = ca > 0
        acc = {"steps": args.accuracy_steps,
               "relL2_psi_fp32_vs_fp64": float(np.linalg.norm(pb - pa) / np.linalg.norm(pa)),
               "relL2_V_fp32_vs_fp64": float(np.linalg.norm((Vb - Vb.mean()) - (Va - Va.mean()))
                                             / np.linalg.norm(Va - Va.mean())),
               "mass_drift_fp64": abs(Ma - M0) / M0, "mass_drift_fp32": abs(Mb - M0) / M0,
               "energy_drift_fp64": abs(Ea - E0) / abs(E0), "energy_drift_fp32": abs(Eb - E0) / abs(E0),
               "Pk_log256_max_rel_err": float(np.max(np.abs(Pb[sel] - Pa[sel]) / np.abs(Pa[sel]))),
               "reference_form": "plain FP64 GPU form (validated against the CPU oracle at <=1e-12)"}
        del pa, pb, Va, Vb
        a.close()
        b.close()

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        g = make_field(qx, "c128", dt)
        psi0 = g.psi
        g.close()
        cpu = cpu_baseline(psi0, dt)
        del psi0

    # ---- end to end through the C ABI with pinned host buffers ----
    host_in = torch.empty(2 * S, dtype=torch.float64, pin_memory=True)
    host_out = torch.empty(2 * S, dtype=torch.float64, pin_memory=True)
    g = make_field(qx, "c64", dt)
    g.get_psi_ptr(host_in.data_ptr())
    g.close()
    t_e2e = e2e_run(qx, dt, K, host_in.data_ptr(), host_out.data_ptr(), world)
    e2e = {"value": world * S * K / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 16 * S / K,
           "d2h_bytes_per_step": 16 * S / K,
           "what": f"qx_set_psi (FP64 pinned host -> device) + qx_step({K}) + qx_get_psi (device -> pinned host)"}
    del host_in, host_out

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_step, "steps_per_s": 1e3 / ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c64 (fp32 complex; fp64 phase args, reductions, spectrum sums)", "data": "synthetic",
            "config": {"workload": "3D 512^3 GRF + 32 Schive solitons, merged KDK step (fused FP32 form)",
                       "grid": N_GRID, "dim": DIM, "dt": dt, "pref": 1.0, "seed": SEED,
                       "l2": "inputs larger than L2 (1 GiB complex64 state per pass)",
                       "parallelism": f"replicas x{world} (one box per GPU)",
                       "launch_geometry": tune32},
            "plain_fp64": {"value": value64, "ms_per_step": ms64 / K, "dtype": "c128", "launch_geometry": tune64},
            "fp32_over_fp64": value / value64,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            # qx_step(K) in 3D: a prologue of 6 launches (x r2c, y fwd, z Poisson
            # + its column-0 kernel, y inv, x c2r + half kick + x fwd), then K loop
            # bodies of 9 (y fwd, z drift, y inv, x inv + r2c, y fwd, z Poisson,
            # column 0, y inv, x c2r + kick + x fwd)
            "gpu_launches": 6 + 9 * K,
            "clocks": clocks,
            "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
