// qx_capi.cpp -- extern "C" boundary over qx::Field (include/qaxions_b200.h).
// Exceptions are caught here and turned into status codes + messages.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qaxions_b200.h"
#include "qx_field.hpp"

struct qx_field_s {
    std::unique_ptr<qx::Field> f;
    std::string err;
};

namespace {
thread_local std::string g_err;

template <typename F>
int guarded(qx_field_t* h, F&& fn) {
    if (!h || !h->f) {
        g_err = "null or destroyed qx_field handle";
        return QX_ERR_INVALID;
    }
    try {
        fn(*h->f);
        h->err.clear();
        return QX_OK;
    } catch (const std::invalid_argument& e) {
        h->err = e.what();
        return QX_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        h->err = "device allocation failed";
        return QX_ERR_NOMEM;
    } catch (const std::logic_error& e) {
        h->err = e.what();
        return QX_ERR_STATE;
    } catch (const std::runtime_error& e) {
        h->err = e.what();
        return QX_ERR_CUDA;
    } catch (...) {
        h->err = "unknown error";
        return QX_ERR_INTERNAL;
    }
}

void need(bool ok, const char* msg) {
    if (!ok) throw std::invalid_argument(msg);
}
}  // namespace

extern "C" {

int qx_version(void) { return 100; }

const char* qx_last_error(const qx_field_t* h) {
    if (h && !h->err.empty()) return h->err.c_str();
    return g_err.c_str();
}

int qx_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return e == cudaErrorInvalidDevice ? QX_ERR_INVALID : QX_ERR_CUDA;
    }
    g_err.clear();
    return QX_OK;
}

int qx_create(int dim, int N, double L, double pref, double rho_mean, int dtype, int k0_policy, double dt,
              qx_field_t** out) {
    if (!out) {
        g_err = "out must not be NULL";
        return QX_ERR_INVALID;
    }
    *out = nullptr;
    if (dtype != QX_C128 && dtype != QX_C64) {
        g_err = "dtype must be QX_C128 or QX_C64";
        return QX_ERR_INVALID;
    }
    if (k0_policy != QX_K0_REFERENCE && k0_policy != QX_K0_ZERO) {
        g_err = "k0_policy must be QX_K0_REFERENCE or QX_K0_ZERO";
        return QX_ERR_INVALID;
    }
    qx::FieldConfig c;
    c.dim = dim;
    c.N = N;
    c.L = L;
    c.pref = pref;
    c.rho_mean = rho_mean;
    c.prec = dtype == QX_C128 ? qx::Prec::F64 : qx::Prec::F32;
    c.k0 = k0_policy == QX_K0_REFERENCE ? qx::K0::Reference : qx::K0::Zero;
    c.dt = dt;
    try {
        auto h = new qx_field_s();
        try {
            h->f = qx::make_field(c);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        g_err.clear();
        return QX_OK;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return QX_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        g_err = "device allocation failed";
        return QX_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_err = e.what();
        return QX_ERR_CUDA;
    }
}

int qx_destroy(qx_field_t* h) {
    if (!h) return QX_OK;
    try {
        h->f.reset();
    } catch (...) {
    }
    delete h;
    return QX_OK;
}

int qx_set_dt(qx_field_t* h, double dt) { return guarded(h, [&](qx::Field& f) { f.set_dt(dt); }); }

int qx_set_psi(qx_field_t* h, const double* p) {
    return guarded(h, [&](qx::Field& f) { need(p, "psi is NULL"); f.set_psi(p); });
}
int qx_get_psi(qx_field_t* h, double* p) {
    return guarded(h, [&](qx::Field& f) { need(p, "psi is NULL"); f.get_psi(p); });
}
int qx_set_V(qx_field_t* h, const double* v) {
    return guarded(h, [&](qx::Field& f) { need(v, "V is NULL"); f.set_V(v); });
}
int qx_get_V(qx_field_t* h, double* v) {
    return guarded(h, [&](qx::Field& f) { need(v, "V is NULL"); f.get_V(v); });
}
int qx_get_Vhat(qx_field_t* h, double* v) {
    return guarded(h, [&](qx::Field& f) { need(v, "Vhat is NULL"); f.get_Vhat(v); });
}
int qx_set_Vhat(qx_field_t* h, const double* v) {
    return guarded(h, [&](qx::Field& f) { need(v, "Vhat is NULL"); f.set_Vhat(v); });
}

int qx_kick(qx_field_t* h, double dt) { return guarded(h, [&](qx::Field& f) { f.kick(dt); f.sync(); }); }
int qx_drift(qx_field_t* h, double dt) { return guarded(h, [&](qx::Field& f) { f.drift(dt); f.sync(); }); }
int qx_poisson(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.Poisson(); f.sync(); }); }
int qx_update_potential(qx_field_t* h) {
    return guarded(h, [&](qx::Field& f) { f.updatePotential(); f.sync(); });
}
int qx_compute_energy(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.computeEnergy(); f.sync(); }); }
int qx_update_time(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.updateTime(); }); }
int qx_half_kick(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.half_kick(); f.sync(); }); }
int qx_full_kick(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.full_kick(); f.sync(); }); }
int qx_drift_update(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.drift_update(); f.sync(); }); }
int qx_propagate(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.propagate(); f.sync(); }); }
int qx_step(qx_field_t* h, int n) {
    return guarded(h, [&](qx::Field& f) {
        need(n >= 0, "nsteps must be >= 0");
        f.step(n);
        f.sync();
    });
}

int qx_scalars(qx_field_t* h, double* vmax, double* rhomax, double* time, double* a, int* curr) {
    return guarded(h, [&](qx::Field& f) {
        if (vmax) *vmax = f.Vmax();
        if (rhomax) *rhomax = f.rhomax();
        if (time) *time = f.time();
        if (a) *a = f.a();
        if (curr) *curr = f.curr();
    });
}
int qx_rho_stats(qx_field_t* h, double* rhomax, double* vmax) {
    return guarded(h, [&](qx::Field& f) { f.rho_stats(rhomax, vmax); });
}
int qx_mass_energy(qx_field_t* h, double* M, double* E, double* K, double* W) {
    return guarded(h, [&](qx::Field& f) { f.mass_energy(M, E, K, W); });
}
int qx_spectrum(qx_field_t* h, int source, int mode, int nbins, double* k, double* P, long long* count) {
    return guarded(h, [&](qx::Field& f) {
        need(source == 0 || source == 1, "source must be 0 (|psi|^2) or 1 (V)");
        f.spectrum(source, mode, nbins, k, P, count);
    });
}

int qx_fft_c2c(qx_field_t* h, double* data, int sign) {
    return guarded(h, [&](qx::Field& f) {
        need(data, "data is NULL");
        need(sign == -1 || sign == 1, "sign must be -1 or +1");
        f.host_c2c(data, sign);
    });
}
int qx_fft_r2c(qx_field_t* h, const double* in, double* out) {
    return guarded(h, [&](qx::Field& f) { need(in && out, "NULL buffer"); f.host_r2c(in, out); });
}
int qx_fft_c2r(qx_field_t* h, const double* in, double* out) {
    return guarded(h, [&](qx::Field& f) { need(in && out, "NULL buffer"); f.host_c2r(in, out); });
}

int qx_ic_gaussian_solitons(qx_field_t* h, int n, const double* rows5, double bkg) {
    return guarded(h, [&](qx::Field& f) {
        need(n >= 0 && (n == 0 || rows5), "bad soliton table");
        f.ic_gaussian_solitons(n, rows5, bkg);
    });
}

// src/ic/solitons.cxx:32-50: one soliton per parsable 'amp sigma x y z' line
int qx_ic_solitons_file(qx_field_t* h, const char* path, double bkg) {
    return guarded(h, [&](qx::Field& f) {
        need(path, "path is NULL");
        std::ifstream in(path);
        if (!in.is_open()) throw std::invalid_argument(std::string("Error opening file ") + path);
        std::vector<double> rows;
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream ss(line);
            double a, s, x, y, z;
            if (ss >> a >> s >> x >> y >> z) rows.insert(rows.end(), {a, s, x, y, z});
        }
        f.ic_gaussian_solitons((int)(rows.size() / 5), rows.data(), bkg);
    });
}

int qx_ic_config(qx_field_t* h, int kind, unsigned long long seed, int n_solitons, double rc_lo, double rc_hi,
                 double sigma, double kc_factor, double clip, double rho0) {
    return guarded(h, [&](qx::Field& f) {
        need(kind == QX_IC_SOLITONS || kind == QX_IC_GRF, "kind must be QX_IC_SOLITONS or QX_IC_GRF");
        need(n_solitons >= 0 && n_solitons <= 100000, "n_solitons out of range");
        need(kind == QX_IC_GRF || n_solitons > 0, "a soliton IC needs n_solitons > 0");
        f.ic_config(kind, seed, n_solitons, rc_lo, rc_hi, sigma, kc_factor, clip, rho0);
    });
}

int qx_time_steps(qx_field_t* h, int nsteps, int use_graph, float* ms) {
    return guarded(h, [&](qx::Field& f) {
        need(ms, "ms is NULL");
        *ms = f.time_steps(nsteps, use_graph);
    });
}

int qx_profile_step(qx_field_t* h, int nsteps, int max_entries, char* names, double* ms, int* n_out) {
    return guarded(h, [&](qx::Field& f) {
        need(nsteps > 0 && names && ms && n_out, "bad profile arguments");
        std::vector<std::pair<std::string, double>> r;
        f.profile_step(nsteps, r);
        const int n = (int)r.size() < max_entries ? (int)r.size() : max_entries;
        for (int i = 0; i < n; ++i) {
            std::strncpy(names + 64 * i, r[i].first.c_str(), 63);
            names[64 * i + 63] = 0;
            ms[i] = r[i].second;
        }
        *n_out = n;
    });
}

int qx_set_tune(qx_field_t* h, int x_rows, int y_tx, int la_tx, int tma, int nbuf, int pw) {
    return guarded(h, [&](qx::Field& f) {
        need(x_rows >= 0 && y_tx >= 0 && la_tx >= 0 && nbuf >= 0 && nbuf <= 8 && tma >= -1 && tma <= 1 &&
                 pw >= 0 && pw <= 2,
             "tune values out of range");
        f.tune().pw = pw;
        f.tune().x_rows = x_rows;
        f.tune().y_tx = y_tx;
        f.tune().la_tx = la_tx;
        if (tma >= 0) f.tune().tma = tma;
        f.tune().nbuf = nbuf;
        f.invalidate_graph();
    });
}

int qx_clear_tune_cache(void) {
    qx::clear_tune_cache();
    return QX_OK;
}

int qx_set_plan(qx_field_t* h, int plan) {
    return guarded(h, [&](qx::Field& f) {
        need(plan == 0 || plan == 1, "plan must be 0 or 1");
        f.tune().plan = plan;
        f.invalidate_graph();
    });
}

int qx_set_pencil_warp(qx_field_t* h, int on) {
    return guarded(h, [&](qx::Field& f) {
        need(on >= 0 && on <= 4, "on must be 0 ... 4");
        f.tune().wp = on;
        f.invalidate_graph();
    });
}

int qx_get_tune(qx_field_t* h, int* out, int n) {
    return guarded(h, [&](qx::Field& f) {
        need(out && n >= 10, "out must hold 10 ints");
        const qx::Tune& t = f.tune();
        const int v[11] = {t.x_rows, t.y_tx, t.la_tx, t.tma, t.nbuf, t.pw, t.plan, t.chain, t.wp,
                           f.tuned_from_cache() ? 1 : 0, t.xstage};
        for (int i = 0; i < (n < 11 ? n : 11); ++i) out[i] = v[i];
    });
}

int qx_set_row_stage(qx_field_t* h, int on) {
    return guarded(h, [&](qx::Field& f) {
        need(on == 0 || on == 1, "on must be 0 or 1");
        f.tune().xstage = on;
        f.invalidate_graph();
    });
}

int qx_set_chain(qx_field_t* h, int on) {
    return guarded(h, [&](qx::Field& f) {
        need(on >= 0 && on <= 2, "chain must be 0, 1 or 2");
        f.tune().chain = on;
        f.invalidate_graph();
    });
}

int qx_device_pointers(qx_field_t* h, void** psi, void** V) {
    return guarded(h, [&](qx::Field& f) {
        if (psi) *psi = f.psi_device();
        if (V) *V = f.V_device();
    });
}

int qx_sync(qx_field_t* h) { return guarded(h, [&](qx::Field& f) { f.sync(); }); }

}  // extern "C"

extern "C" {

int qx_copy_psi(qx_field_t* dst, qx_field_t* src) {
    return guarded(dst, [&](qx::Field& d) {
        need(src && src->f, "null source handle");
        qx::Field& s = *src->f;
        need(d.dim() == s.dim() && d.size() == s.size() && d.sites() == s.sites() &&
                 d.config().prec == s.config().prec,
             "fields differ in geometry or dtype");
        const size_t bytes = d.sites() * (d.config().prec == qx::Prec::F64 ? 16 : 8);
        s.sync();
        cudaError_t e = cudaMemcpyAsync(d.psi_device(), s.psi_device(), bytes, cudaMemcpyDeviceToDevice, d.stream());
        if (e == cudaSuccess) e = cudaStreamSynchronize(d.stream());
        if (e != cudaSuccess) throw std::runtime_error(std::string("psi copy: ") + cudaGetErrorString(e));
        d.psi_changed();
    });
}

int qx_autotune(qx_field_t* h, int nsteps, const char* cache_path, double* best_ms, int* from_cache) {
    return guarded(h, [&](qx::Field& f) {
        bool fc = false;
        const double ms = f.autotune(nsteps, cache_path, &fc);
        if (best_ms) *best_ms = ms;
        if (from_cache) *from_cache = fc ? 1 : 0;
    });
}

int qx_set_cosmology(qx_field_t* h, int cosmo, double ai) {
    return guarded(h, [&](qx::Field& f) { f.set_cosmology(cosmo, ai); });
}

static void to_c(const qx::MeasRecord& r, qx_meas_t* o) {
    o->number = r.number;
    o->step = r.step;
    o->time = r.time;
    o->a = r.a;
    o->rhomax = r.rhomax;
    o->vmax = r.vmax;
    o->mass = r.mass;
    o->energy = r.energy;
    o->kinetic = r.kinetic;
    o->potential = r.potential;
}

int qx_meas_list(long long nsteps, long long nmeas, long long* out, int max_out, int* n_out) {
    if (nsteps < 0 || nmeas < 0 || max_out < 0 || (max_out > 0 && !out)) {
        g_err = "nsteps, nmeas and max_out must be >= 0 and out not NULL";
        return QX_ERR_INVALID;
    }
    const auto ml = qx::meas_list((long)nsteps, (long)nmeas);
    if ((long long)ml.size() > max_out) {
        g_err = "out holds fewer than nmeas entries";
        return QX_ERR_INVALID;
    }
    for (size_t i = 0; i < ml.size(); ++i) out[i] = ml[i];
    if (n_out) *n_out = (int)ml.size();
    g_err.clear();
    return QX_OK;
}

int qx_measure(qx_field_t* h, unsigned mask, int number, const char* dir, qx_meas_t* rec) {
    return guarded(h, [&](qx::Field& f) {
        need(number >= 0, "number must be >= 0");
        qx::MeasRecord r;
        f.measure(mask, number, dir, &r);
        if (rec) to_c(r, rec);
    });
}

int qx_run(qx_field_t* h, int nsteps, int nmeas, unsigned mask, const char* dir, qx_meas_t* recs, int max_recs,
           int* n_out) {
    return guarded(h, [&](qx::Field& f) {
        need(nsteps >= 0 && nmeas >= 0, "nsteps and nmeas must be >= 0");
        need(max_recs >= 0 && (max_recs == 0 || recs), "recs must hold max_recs records");
        need(mask == QX_MEAS_NONE || max_recs >= nmeas + 1, "recs must hold nmeas + 1 records");
        std::vector<qx::MeasRecord> out;
        f.run(nsteps, nmeas, mask, dir, out);
        for (size_t i = 0; i < out.size() && (int)i < max_recs; ++i) to_c(out[i], &recs[i]);
        if (n_out) *n_out = (int)out.size();
    });
}

int qx_get_cosmology(qx_field_t* h, int* cosmo, double* a, double* ds) {
    return guarded(h, [&](qx::Field& f) {
        if (cosmo) *cosmo = f.cosmology();
        if (a) *a = f.a();
        if (ds) *ds = f.dt();
    });
}

int qx_restore_cosmology(qx_field_t* h, double a, double ds) {
    return guarded(h, [&](qx::Field& f) {
        need(std::isfinite(a) && a > 0 && std::isfinite(ds), "a must be finite and > 0, ds finite");
        need(f.cosmology() == 1 || a == 1.0, "a STATIC field keeps a = 1");
        f.restore_cosmology(a, ds);
    });
}

int qx_set_clock(qx_field_t* h, int step, double time) {
    return guarded(h, [&](qx::Field& f) {
        need(step >= 0 && std::isfinite(time), "step must be >= 0 and time finite");
        f.set_clock(step, time);
    });
}

int qx_psi_changed(qx_field_t* h) {
    return guarded(h, [&](qx::Field& f) { f.psi_changed(); });
}

int qx_scale_psi(qx_field_t* h, double factor) {
    return guarded(h, [&](qx::Field& f) {
        need(std::isfinite(factor), "factor must be finite");
        f.scale_psi(factor);
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// ensemble of independent boxes: one batched field per box size
// ---------------------------------------------------------------------------

struct qx_ens_s {
    std::vector<std::unique_ptr<qx::Field>> groups;
    std::vector<int> group_of;  // box -> group
    std::vector<int> index_in;  // box -> index within its group
    long long sites = 0;
    std::string err;
    // one loop body of every group as ONE graph (a branch per group on the
    // group's stream, forked from and joined into `s0`), replayed once per step
    cudaStream_t s0 = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<double> exec_dt;  // each group's ds when captured
    std::vector<cudaEvent_t> ev;  // per group: fork/join events
    cudaEvent_t ev0 = nullptr;
    // mixed-size modes: 1 = the loop body as one persistent launch over every
    // group, 2 = one launch per pass over every group.  Device counters: one
    // queue counter per pass, then the one-launch body's per-(pass, box)
    // completion counters, then its time-out flag
    int dtype = QX_C128;
    int mixed = 0;
    unsigned long long* ctr = nullptr;
    unsigned* done = nullptr;
    int* dflag = nullptr;
    size_t ctr_bytes = 0;
    long long mix_window = 48LL << 20;  // bytes of boxes whose passes run together (mode 1)  // bytes cleared before every body (all but the flag)
    ~qx_ens_s() {
        if (exec) cudaGraphExecDestroy(exec);
        if (ctr) cudaFree(ctr);
        for (auto e : ev) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (s0) cudaStreamDestroy(s0);
    }
};

namespace {
thread_local std::string g_ens_err;

template <typename F>
int ens_guarded(qx_ens_t* h, F&& fn) {
    if (!h) {
        g_ens_err = "null qx_ens handle";
        return QX_ERR_INVALID;
    }
    try {
        fn(*h);
        h->err.clear();
        return QX_OK;
    } catch (const std::invalid_argument& e) {
        h->err = e.what();
        return QX_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        h->err = "device allocation failed";
        return QX_ERR_NOMEM;
    } catch (const std::logic_error& e) {
        h->err = e.what();
        return QX_ERR_STATE;
    } catch (const std::runtime_error& e) {
        h->err = e.what();
        return QX_ERR_CUDA;
    } catch (...) {
        h->err = "unknown error";
        return QX_ERR_INTERNAL;
    }
}

void ens_box(const qx_ens_t& e, int box) {
    need(box >= 0 && box < (int)e.group_of.size(), "box index out of range");
}

#define QX_CU(call)                                                                            \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
}  // namespace

extern "C" {

int qx_ens_create(int ngroups, const int* N, const int* boxes, int dim, double L, double pref, int dtype,
                  double dt, qx_ens_t** out) {
    if (!out) {
        g_ens_err = "out must not be NULL";
        return QX_ERR_INVALID;
    }
    *out = nullptr;
    auto h = new qx_ens_s();
    const int rc = ens_guarded(h, [&](qx_ens_s& e) {
        need(ngroups > 0 && N && boxes, "need at least one group");
        need(dtype == QX_C128 || dtype == QX_C64, "dtype must be QX_C128 or QX_C64");
        e.dtype = dtype;
        for (int g = 0; g < ngroups; ++g) {
            need(boxes[g] > 0, "every group needs at least one box");
            qx::FieldConfig c;
            c.dim = dim;
            c.N = N[g];
            c.L = L;
            c.pref = pref;
            c.rho_mean = 1.0;
            c.prec = dtype == QX_C128 ? qx::Prec::F64 : qx::Prec::F32;
            c.k0 = qx::K0::Zero;
            c.dt = dt;
            c.batch = boxes[g];
            e.groups.push_back(qx::make_field(c));
            for (int b = 0; b < boxes[g]; ++b) {
                e.group_of.push_back(g);
                e.index_in.push_back(b);
            }
            e.sites += (long long)e.groups.back()->sites();
        }
    });
    if (rc != QX_OK) {
        g_ens_err = h->err;
        delete h;
        return rc;
    }
    *out = h;
    return QX_OK;
}

int qx_ens_destroy(qx_ens_t* h) {
    if (!h) return QX_OK;
    try {
        h->groups.clear();
    } catch (...) {
    }
    delete h;
    return QX_OK;
}

const char* qx_ens_last_error(const qx_ens_t* h) {
    if (h && !h->err.empty()) return h->err.c_str();
    return g_ens_err.c_str();
}

int qx_ens_size(qx_ens_t* h, int* nboxes, long long* sites) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        if (nboxes) *nboxes = (int)e.group_of.size();
        if (sites) *sites = e.sites;
    });
}

int qx_ens_box_n(qx_ens_t* h, int box, int* N) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        ens_box(e, box);
        need(N != nullptr, "N must not be NULL");
        *N = e.groups[e.group_of[box]]->size();
    });
}

int qx_ens_ic_config(qx_ens_t* h, int kind, unsigned long long seed_base, int n_sol, double rc_lo, double rc_hi,
                     double sigma, double kc_factor, double clip, double rho0) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(kind == QX_IC_GRF || kind == QX_IC_SOLITONS, "kind must be QX_IC_GRF or QX_IC_SOLITONS");
        need(n_sol >= 0, "n_sol must be >= 0");
        for (size_t i = 0; i < e.group_of.size(); ++i)
            e.groups[e.group_of[i]]->ic_config_box(e.index_in[i], kind, seed_base + i, n_sol, rc_lo, rc_hi, sigma,
                                                   kc_factor, clip, rho0);
    });
}

int qx_ens_ic_config_seeds(qx_ens_t* h, int kind, const unsigned long long* seeds, int n_sol, double rc_lo,
                           double rc_hi, double sigma, double kc_factor, double clip, double rho0) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(kind == QX_IC_GRF || kind == QX_IC_SOLITONS, "kind must be QX_IC_GRF or QX_IC_SOLITONS");
        need(n_sol >= 0, "n_sol must be >= 0");
        need(seeds != nullptr, "seeds must not be NULL");
        for (size_t i = 0; i < e.group_of.size(); ++i)
            e.groups[e.group_of[i]]->ic_config_box(e.index_in[i], kind, seeds[i], n_sol, rc_lo, rc_hi, sigma,
                                                   kc_factor, clip, rho0);
    });
}

int qx_ens_set_psi(qx_ens_t* h, int box, const double* psi) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        ens_box(e, box);
        need(psi != nullptr, "psi must not be NULL");
        e.groups[e.group_of[box]]->set_psi_box(e.index_in[box], psi);
    });
}

int qx_ens_get_psi(qx_ens_t* h, int box, double* psi) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        ens_box(e, box);
        need(psi != nullptr, "psi must not be NULL");
        e.groups[e.group_of[box]]->get_psi_box(e.index_in[box], psi);
    });
}

namespace {
// s0 waits for every group stream's work so far
void ens_join(qx_ens_s& e) {
    for (size_t i = 0; i < e.groups.size(); ++i) {
        QX_CU(cudaEventRecord(e.ev[i], e.groups[i]->stream()));
        QX_CU(cudaStreamWaitEvent(e.s0, e.ev[i], 0));
    }
}
// every group stream waits for s0's work so far
void ens_fork(qx_ens_s& e) {
    QX_CU(cudaEventRecord(e.ev0, e.s0));
    for (auto& g : e.groups) QX_CU(cudaStreamWaitEvent(g->stream(), e.ev0, 0));
}

// the loop body of every group on s0 with the mixed-size kernels: counters
// cleared, then one launch (mode 1) or one launch per pass (mode 2)
void ens_enqueue_mixed(qx_ens_s& e, const std::vector<qx::MixDesc>& d) {
    QX_CU(cudaMemsetAsync(e.ctr, 0, e.ctr_bytes, e.s0));
    const int ng = (int)d.size();
    if (e.mixed == 1) {
        if (e.dtype == QX_C64) qx::Mixed<float>::launch_step(d.data(), ng, e.ctr, e.done, e.dflag, (long)e.mix_window, e.s0);
        else qx::Mixed<double>::launch_step(d.data(), ng, e.ctr, e.done, e.dflag, (long)e.mix_window, e.s0);
        return;
    }
    for (int op = 0; op < qx::MX_NOPS; ++op) {
        if (e.dtype == QX_C64) qx::Mixed<float>::launch(op, d.data(), ng, e.ctr + op, e.dflag, e.s0);
        else qx::Mixed<double>::launch(op, d.data(), ng, e.ctr + op, e.dflag, e.s0);
    }
}

void ens_alloc_counters(qx_ens_s& e) {
    if (e.ctr) return;
    const size_t nbox = e.group_of.size();
    e.ctr_bytes = sizeof(unsigned long long) * qx::MX_NOPS + sizeof(unsigned) * qx::MX_NOPS * nbox;
    void* p = nullptr;
    QX_CU(cudaMalloc(&p, e.ctr_bytes + sizeof(int)));
    e.ctr = static_cast<unsigned long long*>(p);
    e.done = reinterpret_cast<unsigned*>(e.ctr + qx::MX_NOPS);
    e.dflag = reinterpret_cast<int*>(static_cast<char*>(p) + e.ctr_bytes);
    QX_CU(cudaMemset(p, 0, e.ctr_bytes + sizeof(int)));
}

// a time-out inside the one-launch body (a wait that gave up) -> error
void ens_check_flag(qx_ens_s& e) {
    if (!e.dflag) return;
    int f = 0;
    QX_CU(cudaMemcpy(&f, e.dflag, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) {
        QX_CU(cudaMemset(e.dflag, 0, sizeof(int)));
        throw std::runtime_error(f == 2 ? "mixed-size passes: the host's unit layout disagrees with the kernel's"
                                        : "mixed-size step: a wait for a box's previous pass timed out");
    }
}

void ens_capture(qx_ens_s& e) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    e.exec = nullptr;
    for (auto& g : e.groups) g->prepare_replay();
    for (auto& g : e.groups) g->sync();
    std::vector<qx::MixDesc> d;
    if (e.mixed) {
        ens_alloc_counters(e);
        d.resize(e.groups.size());
        for (size_t i = 0; i < e.groups.size(); ++i) e.groups[i]->mix_desc(d[i]);
        // kernel attributes are set outside the capture
        if (e.dtype == QX_C64) qx::Mixed<float>::prepare(d.data(), (int)d.size());
        else qx::Mixed<double>::prepare(d.data(), (int)d.size());
    }
    cudaGraph_t graph = nullptr;
    QX_CU(cudaStreamBeginCapture(e.s0, cudaStreamCaptureModeThreadLocal));
    try {
        if (e.mixed) {
            ens_enqueue_mixed(e, d);
        } else {
            ens_fork(e);  // the group streams join the capture
            for (auto& g : e.groups) g->enqueue_body(false);
            ens_join(e);
        }
    } catch (...) {
        cudaStreamEndCapture(e.s0, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    QX_CU(cudaStreamEndCapture(e.s0, &graph));
    const cudaError_t r = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    QX_CU(r);
    e.exec_dt.clear();
    for (auto& g : e.groups) e.exec_dt.push_back(g->dt());
}

// the merged loop of every box: prologues and the first and last bodies run
// eagerly on the group streams; the bodies in between are one graph replay
// per step over all groups
void ens_step(qx_ens_s& e, int nsteps) {
    if (nsteps <= 0) return;
    if (!e.s0) {
        QX_CU(cudaStreamCreateWithFlags(&e.s0, cudaStreamNonBlocking));
        QX_CU(cudaEventCreateWithFlags(&e.ev0, cudaEventDisableTiming));
        e.ev.resize(e.groups.size());
        for (auto& v : e.ev) QX_CU(cudaEventCreateWithFlags(&v, cudaEventDisableTiming));
    }
    for (auto& g : e.groups) g->step_begin();
    if (nsteps > 1) {
        for (auto& g : e.groups) g->enqueue_body(false);  // eager (also sets kernel attributes)
        if (nsteps > 2) {
            bool same = e.exec && e.exec_dt.size() == e.groups.size();
            for (size_t i = 0; same && i < e.groups.size(); ++i) same = e.exec_dt[i] == e.groups[i]->dt();
            if (!same) ens_capture(e);
            for (auto& g : e.groups) g->prepare_replay();
            ens_join(e);
            for (int i = 0; i < nsteps - 2; ++i) QX_CU(cudaGraphLaunch(e.exec, e.s0));
            ens_fork(e);
        }
    }
    for (auto& g : e.groups) g->enqueue_body(true);
    for (auto& g : e.groups) g->step_end(nsteps);
}
}  // namespace

int qx_ens_step(qx_ens_t* h, int nsteps) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(nsteps >= 0, "nsteps must be >= 0");
        ens_step(e, nsteps);
        for (auto& g : e.groups) g->sync();
        ens_check_flag(e);
    });
}

int qx_ens_time_steps(qx_ens_t* h, int nsteps, float* ms) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(nsteps > 0 && ms, "nsteps must be > 0 and ms not NULL");
        // first group's stream brackets the others: start event -> all wait,
        // every group's end event -> first stream waits -> stop event
        cudaStream_t s0 = e.groups[0]->stream();
        cudaEvent_t start, stop;
        std::vector<cudaEvent_t> ends(e.groups.size());
        QX_CU(cudaEventCreate(&start));
        QX_CU(cudaEventCreate(&stop));
        for (auto& ev : ends) QX_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        QX_CU(cudaEventRecord(start, s0));
        for (auto& g : e.groups) QX_CU(cudaStreamWaitEvent(g->stream(), start, 0));
        ens_step(e, nsteps);
        for (size_t i = 0; i < e.groups.size(); ++i) QX_CU(cudaEventRecord(ends[i], e.groups[i]->stream()));
        for (auto& ev : ends) QX_CU(cudaStreamWaitEvent(s0, ev, 0));
        QX_CU(cudaEventRecord(stop, s0));
        QX_CU(cudaEventSynchronize(stop));
        float t = 0.f;
        QX_CU(cudaEventElapsedTime(&t, start, stop));
        for (auto& g : e.groups) g->sync();
        for (auto& ev : ends) cudaEventDestroy(ev);
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        ens_check_flag(e);
        *ms = t;
    });
}

int qx_ens_set_mixed(qx_ens_t* h, int mixed) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(mixed >= 0 && mixed <= 2, "mixed must be 0, 1 or 2");
        if (mixed) {
            need((int)e.groups.size() <= qx::kMixMaxGroups, "mixed-size passes take at most 4 groups");
            for (auto& g : e.groups) {
                need(g->dim() == 3, "mixed-size passes are 3D only");
                need(g->cosmology() == 0, "mixed-size passes need the STATIC cosmology");
                const bool ok = e.dtype == QX_C64 ? qx::Mixed<float>::supports(g->size())
                                                  : qx::Mixed<double>::supports(g->size());
                need(ok, ("mixed-size passes: grid size N=" + std::to_string(g->size()) + " is not compiled in").c_str());
            }
        }
        if (mixed != e.mixed) {
            if (e.exec) cudaGraphExecDestroy(e.exec);
            e.exec = nullptr;
            e.mixed = mixed;
        }
    });
}

int qx_ens_set_mixed_window(qx_ens_t* h, long long bytes) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(bytes >= 0, "bytes must be >= 0");
        const long long w = bytes ? bytes : (48LL << 20);
        if (w != e.mix_window) {
            if (e.exec) cudaGraphExecDestroy(e.exec);
            e.exec = nullptr;
            e.mix_window = w;
        }
    });
}

int qx_ens_mass(qx_ens_t* h, double* M) {
    return ens_guarded(h, [&](qx_ens_s& e) {
        need(M != nullptr, "M must not be NULL");
        size_t off = 0;
        for (auto& g : e.groups) {
            g->box_mass(M + off);
            off += (size_t)g->batch();
        }
    });
}

}  // extern "C"
