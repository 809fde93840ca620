// ref_runner.cpp -- C-ABI driver over the REFERENCE solver's own classes
// (TEST INFRASTRUCTURE: oracle and timed CPU baseline only).
//
// The reference translation units (src/field.cxx, src/spectrum/spectrum.cxx,
// src/ic/ic.cxx, src/ic/solitons.cxx, src/utils.cxx, src/parse.cxx) are compiled
// unmodified from the reference tree by oracle/Makefile and linked with the
// project FFTW-API shim (oracle/fftw_shim).  This file only drives them: it
// builds a Params/Field exactly as src/examples/fieldtest.cxx:11-23 does, exposes
// the Field methods (src/field.h:17-64) over plain pointers, and re-states the
// merged leapfrog loop of src/main.cxx:64-85 with measurements off.
#include <omp.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "field.h"
#include "ic/ic.h"
#include "parse.h"
#include "profiler.h"
#include "spectrum/spectrum.h"
#include "utils.h"

// src/meas.cxx:8-11 needs HDF5 for the rest of its file; this one cast is all
// src/parse.cxx uses from it.
MeasureType parseMeasureType(uint32_t value) { return static_cast<MeasureType>(value); }

namespace {
struct RefHandle {
    Params pars;
    std::unique_ptr<Field> field;
};
}  // namespace

extern "C" {

// norm is the reference's --norm (src/parse.cxx:19); STATIC cosmology sets
// pref = 4*pi*norm (src/field.cxx:78).  dt sets ds_ (src/field.cxx:77).
void* ref_create(int dim, int N, double L, double norm, double dt, int nthr) {
    auto* h = new RefHandle();
    defaults(h->pars);
    h->pars.N = N;
    h->pars.dim = dim;
    h->pars.Lbox = L;
    h->pars.norm = norm;
    h->pars.dt = dt;
    h->pars.nthr = nthr > 0 ? nthr : 1;
    h->pars.verb = false;
    h->pars.plan = FFTPlanType::ESTIMATE;
    h->pars.cosmotype = CosmoType::STATIC;
    h->pars.measinfo = MeasureType::NONE;
    omp_set_num_threads(h->pars.nthr);
    initProfilers();
    h->field = std::make_unique<Field>(h->pars);
    return h;
}

// MRE cosmology (src/field.cxx:82-88): a = ai, ds = dt / ai, norm 1,
// rho_mean = 1.5 (2 pi)^2 1.27^2; updateTime advances a (src/field.cxx:349-361)
void* ref_create_mre(int dim, int N, double L, double dt, double ai, int nthr) {
    auto* h = new RefHandle();
    defaults(h->pars);
    h->pars.N = N;
    h->pars.dim = dim;
    h->pars.Lbox = L;
    h->pars.norm = 1.0;
    h->pars.dt = dt;
    h->pars.ai = ai;
    h->pars.nthr = nthr > 0 ? nthr : 1;
    h->pars.verb = false;
    h->pars.plan = FFTPlanType::ESTIMATE;
    h->pars.cosmotype = CosmoType::MRE;
    h->pars.measinfo = MeasureType::NONE;
    omp_set_num_threads(h->pars.nthr);
    initProfilers();
    h->field = std::make_unique<Field>(h->pars);
    return h;
}

void ref_destroy(void* p) { delete static_cast<RefHandle*>(p); }

static Field& F(void* p) { return *static_cast<RefHandle*>(p)->field; }

size_t ref_sites(void* p) { return F(p).sites(); }
size_t ref_ksites(void* p) { return F(p).ksites(); }

void ref_set_psi(void* p, const double* src) {
    std::memcpy(F(p).psi(), src, sizeof(fftw_complex) * F(p).sites());
}
void ref_get_psi(void* p, double* dst) {
    std::memcpy(dst, F(p).psi(), sizeof(fftw_complex) * F(p).sites());
}
void ref_set_V(void* p, const double* src) {
    std::memcpy(F(p).V(), src, sizeof(double) * F(p).sites());
}
void ref_get_V(void* p, double* dst) {
    std::memcpy(dst, F(p).V(), sizeof(double) * F(p).sites());
}
void ref_get_Vhat(void* p, double* dst) {
    std::memcpy(dst, F(p).Vhat(), sizeof(fftw_complex) * F(p).ksites());
}

// SolitonsIC reads ./solitons.txt (src/ic/solitons.cxx:32).
void ref_ic_solitons(void* p, double bkg) {
    auto* h = static_cast<RefHandle*>(p);
    h->pars.sol_bkg = bkg;
    auto ic = createIC(ICType::SOLITONS, h->pars);
    ic->apply(*h->field);
}

void ref_kick(void* p, double dt) { F(p).kick(dt); }
void ref_drift(void* p, double dt) { F(p).drift(dt); }
void ref_update_potential(void* p) { F(p).updatePotential(); }
void ref_poisson(void* p) { F(p).Poisson(); }
void ref_compute_energy(void* p) { F(p).computeEnergy(); }
void ref_half_kick(void* p) { F(p).half_kick(); }
void ref_full_kick(void* p) { F(p).full_kick(); }
void ref_drift_update(void* p) { F(p).drift_update(); }
void ref_propagate(void* p) { F(p).propagate(); }
double ref_vmax(void* p) { return F(p).Vmax(); }
double ref_rhomax(void* p) { return F(p).rhomax(); }
double ref_time(void* p) { return F(p).time(); }
double ref_a(void* p) { return F(p).a(); }
int ref_curr(void* p) { return F(p).curr(); }

// src/main.cxx:64-85 with measinfo = NONE: potential, half kick, then
// nsteps x (drift_update, full kick except after the last), final half kick.
void ref_run(void* p, int nsteps) {
    Field& f = F(p);
    f.updatePotential();
    f.half_kick();
    for (int idx = 0; idx < nsteps; ++idx) {
        f.drift_update();
        if (idx != nsteps - 1) f.full_kick();
    }
    f.half_kick();
}

// generateMeasList (src/utils.cxx:8-28), the reference's own function; out
// holds at least nmeas entries; returns the number written.
int ref_meas_list(long long nsteps, long long nmeas, long long* out) {
    const auto v = generateMeasList((size_t)nsteps, (size_t)nmeas);
    for (size_t i = 0; i < v.size(); ++i) out[i] = (long long)v[i];
    return (int)v.size();
}

// src/main.cxx:60-85 with measurements.  measure() (src/meas.cxx:13-63) needs
// HDF5 for its file output, so its dispatch is spelled out here with what it
// computes: computeEnergy (rhomax; V <- rho) and, for the spectrum bit, the
// Spectrum of that V (src/meas.cxx:30-45).  clobber = 1 keeps the reference's
// behaviour (the kick after a measurement uses V = rho); clobber = 0 measures
// on a copy of V.  Per measurement m (0 .. returned count - 1): rhomax[m],
// curr[m], time[m], and (spectrum != 0) P[m*nb + b], counts[m*nb + b] with
// nb = N/2 + 1.
int ref_run_measured(void* p, int nsteps, int nmeas, int clobber, int spectrum, double* rhomax, int* curr,
                     double* time, double* P, int* counts) {
    Field& f = F(p);
    const auto mlist = generateMeasList((size_t)nsteps, (size_t)nmeas);
    int m = 0;
    std::vector<double> vsave;
    auto meas = [&]() {
        if (!clobber) vsave.assign(f.V(), f.V() + f.sites());
        f.computeEnergy();
        rhomax[m] = f.rhomax();
        curr[m] = f.curr();
        time[m] = f.time();
        if (spectrum) {
            Spectrum s(f);
            s.compute();
            const auto& pk = s.Pk();
            const auto& c = s.counts();
            for (size_t b = 0; b < pk.size(); ++b) {
                P[(size_t)m * pk.size() + b] = pk[b];
                counts[(size_t)m * pk.size() + b] = c[b];
            }
        }
        if (!clobber) std::memcpy(f.V(), vsave.data(), sizeof(double) * vsave.size());
        ++m;
    };
    meas();
    f.updatePotential();
    f.half_kick();
    size_t next = 0;
    for (int idx = 0; idx < nsteps; ++idx) {
        f.drift_update();
        if (next < mlist.size() && (size_t)idx == mlist[next]) {
            ++next;
            meas();
        }
        if (idx != nsteps - 1) f.full_kick();
    }
    f.half_kick();
    return m;
}

// Partial loop used to time a bounded CPU sample: `nsteps` iterations of the
// loop body of src/main.cxx:70-84 (drift_update + full_kick), no prologue.
void ref_loop_body(void* p, int nsteps) {
    Field& f = F(p);
    for (int idx = 0; idx < nsteps; ++idx) {
        f.drift_update();
        f.full_kick();
    }
}

// Spectrum of the current V_ (src/spectrum/spectrum.cxx:32-60).  Arrays hold
// N/2+1 entries.
void ref_spectrum(void* p, double* Pk, int* counts, double* k) {
    Spectrum s(F(p));
    s.compute();
    const auto& P = s.Pk();
    const auto& c = s.counts();
    const auto& kk = s.kmodes();
    for (size_t i = 0; i < P.size(); ++i) {
        Pk[i] = P[i];
        counts[i] = c[i];
        k[i] = kk[i];
    }
}

// Direct access to the reference's FFT backend (src/fft/fft.h:122-140).
void ref_fft_forward_c2c(void* p, double* data) {
    F(p).fftBackend()->forward_c2c(reinterpret_cast<fftw_complex*>(data));
}
void ref_fft_backward_c2c(void* p, double* data) {
    F(p).fftBackend()->backward_c2c(reinterpret_cast<fftw_complex*>(data));
}
void ref_fft_forward_r2c(void* p, double* in, double* out) {
    F(p).fftBackend()->forward_r2c(in, reinterpret_cast<fftw_complex*>(out));
}
void ref_fft_backward_c2r(void* p, double* in, double* out) {
    F(p).fftBackend()->backward_c2r(reinterpret_cast<fftw_complex*>(in), out);
}

}  // extern "C"
