// qx_field.cpp -- implementation of the host Field / FFT plugin mirror.
#include "qx_field.hpp"

#include <cmath>
#include <cstdlib>
#include <limits>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>

#include "qx_misc.hpp"
#include "qx_philox.h"

namespace qx {

#define QX_CUDA(call)                                                                               \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_));           \
    } while (0)

static const double kTwoPi = 6.283185307179586476925286766559005768;

// ---------------------------------------------------------------------------
// device buffer
// ---------------------------------------------------------------------------

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void alloc(size_t n) {
        if (n == bytes && p) return;
        release();
        cudaError_t e = cudaMalloc(&p, n ? n : 1);
        if (e != cudaSuccess) {
            p = nullptr;
            throw std::bad_alloc();
        }
        bytes = n;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// host helpers: twiddles, packing, spectrum tables
// ---------------------------------------------------------------------------

// Twiddles exp(-2 pi i j / L).  In FP32 each value is picked among the
// neighbours (+-2 ulp per component) of the correctly rounded pair to make
// |w|^2 as close to 1 as possible (angle error kept within 1.5 ulp): a
// forward/inverse transform pair cancels a twiddle's angle error but not its
// magnitude error, and the same table is applied every time step, so a
// magnitude bias would accumulate linearly with the number of steps.
template <typename C> static std::vector<C> twiddles(int L) {
    using R = decltype(C::x);
    std::vector<C> t(L);
    const long double tp = 6.283185307179586476925286766559005768L;
    for (int j = 0; j < L; ++j) {
        const long double a = -tp * (long double)j / (long double)L;
        const long double c = cosl(a), s = sinl(a);
        R bc = (R)c, bs = (R)s;
        if constexpr (sizeof(R) == 4) {
            const long double ulp = 1.0L / (1 << 24);
            long double best = fabsl((long double)bc * bc + (long double)bs * bs - 1.0L);
            for (int dc = -2; dc <= 2; ++dc) {
                for (int ds = -2; ds <= 2; ++ds) {
                    R cc = bc, ss = bs;
                    for (int k = 0; k < (dc < 0 ? -dc : dc); ++k) cc = nextafterf(cc, dc < 0 ? -2.0f : 2.0f);
                    for (int k = 0; k < (ds < 0 ? -ds : ds); ++k) ss = nextafterf(ss, ds < 0 ? -2.0f : 2.0f);
                    // angle error of the candidate, in units of 2^-24
                    const long double ang = fabsl(atan2l((long double)ss, (long double)cc) - atan2l(s, c));
                    const long double ang_w = (ang > 3.0L) ? fabsl(ang - tp) : ang;  // across +-pi
                    if (ang_w > 1.5L * ulp) continue;
                    const long double m = fabsl((long double)cc * cc + (long double)ss * ss - 1.0L);
                    if (m < best) {
                        best = m;
                        t[j].x = cc;
                        t[j].y = ss;
                    }
                }
            }
            if (best == fabsl((long double)bc * bc + (long double)bs * bs - 1.0L)) {
                t[j].x = bc;
                t[j].y = bs;
            }
        } else {
            t[j].x = bc;
            t[j].y = bs;
        }
    }
    return t;
}

// low parts exact - hi of a twiddle table (zero for FP64, which does not use them)
template <typename C> static std::vector<C> twiddles_lo(int L, const std::vector<C>& hi) {
    using R = decltype(C::x);
    std::vector<C> lo(L);
    const long double tp = 6.283185307179586476925286766559005768L;
    for (int j = 0; j < L; ++j) {
        const long double a = -tp * (long double)j / (long double)L;
        lo[j].x = sizeof(R) == 4 ? (R)(cosl(a) - (long double)hi[j].x) : (R)0;
        lo[j].y = sizeof(R) == 4 ? (R)(sinl(a) - (long double)hi[j].y) : (R)0;
    }
    return lo;
}

static inline long mirror_row(int dim, int N, long r) {
    if (dim == 2) return (N - r) % N;
    const long y = r % N, z = r / N;
    return ((N - z) % N) * N + (N - y) % N;
}

void pack_half(int dim, int N, const double* h, double* p) {
    const long rows = dim == 3 ? (long)N * N : N;
    const int X = N / 2, XH = N / 2 + 1;
    for (long r = 0; r < rows; ++r) {
        const double* hr = h + 2 * r * XH;
        double* pr = p + 2 * r * X;
        for (int k = 1; k < X; ++k) {
            pr[2 * k] = hr[2 * k];
            pr[2 * k + 1] = hr[2 * k + 1];
        }
        // col0 = A + i B, A = H[0], B = H[N/2]
        const double ax = hr[0], ay = hr[1], bx = hr[2 * X], by = hr[2 * X + 1];
        pr[0] = ax - by;
        pr[1] = ay + bx;
    }
}

void unpack_half(int dim, int N, const double* p, double* h) {
    const long rows = dim == 3 ? (long)N * N : N;
    const int X = N / 2, XH = N / 2 + 1;
    for (long r = 0; r < rows; ++r) {
        const double* pr = p + 2 * r * X;
        const double* pm = p + 2 * mirror_row(dim, N, r) * X;
        double* hr = h + 2 * r * XH;
        for (int k = 1; k < X; ++k) {
            hr[2 * k] = pr[2 * k];
            hr[2 * k + 1] = pr[2 * k + 1];
        }
        const double cx = pr[0], cy = pr[1], mx = pm[0], my = -pm[1];  // conj C(-k)
        hr[0] = 0.5 * (cx + mx);
        hr[1] = 0.5 * (cy + my);
        // B = (C - conj C(-k)) / (2i)
        const double dx = cx - mx, dy = cy - my;
        hr[2 * X] = 0.5 * dy;
        hr[2 * X + 1] = -0.5 * dx;
    }
}

std::vector<int> spectrum_bin_table(int dim, int N, int mode, int nbins) {
    const int nmax = N / 2;
    const long Mmax = (long)dim * nmax * nmax;
    std::vector<int> tab(Mmax + 1, -1);
    for (long M = 0; M <= Mmax; ++M) {
        const double r = std::sqrt((double)M);
        long b = -1;
        if (mode == 0) {
            b = std::lrint(r);
            if (b >= nmax + 1) b = -1;
        } else if (mode == 1) {
            if (M > 0 && r < nmax) b = (long)std::floor(nbins * r / nmax);
            if (b >= nbins) b = -1;
        } else {
            if (M > 0 && r < nmax) b = (long)std::floor(nbins * std::log(r) / std::log((double)nmax) + 1e-9);
            if (b >= nbins) b = -1;
        }
        tab[M] = (int)b;
    }
    return tab;
}

std::vector<double> spectrum_k_axis(int N, int mode, int nbins, double L) {
    const double dk = kTwoPi / L;
    const int nmax = N / 2;
    std::vector<double> k;
    if (mode == 0) {
        for (int b = 0; b <= nmax; ++b) k.push_back(b * dk);
    } else if (mode == 1) {
        for (int b = 0; b < nbins; ++b) k.push_back((b + 0.5) * nmax / nbins * dk);
    } else {
        for (int b = 0; b < nbins; ++b) k.push_back(std::pow((double)nmax, (b + 0.5) / nbins) * dk);
    }
    return k;
}

// ---------------------------------------------------------------------------
// FFT plugin
// ---------------------------------------------------------------------------

template <typename R>
static typename Ops<R>::XP xp0(const Geometry& g, const TwTables<typename Ops<R>::C>& tw) {
    typename Ops<R>::XP a{};
    a.twN = tw.N;
    a.twM = tw.M;
    a.twN_lo = tw.N_lo;
    a.twM_lo = tw.M_lo;
    a.twNn = tw.N_nat;
    a.rows = g.rows;
    a.scale = 1.0;
    a.pref = 1.0;
    a.rho_mean = 0.0;
    return a;
}

template <typename R>
static typename Ops<R>::SP sp0(int* err, const Geometry& g, typename Ops<R>::C* a,
                               const TwTables<typename Ops<R>::C>& tw, int X, const Tune& tu) {
    typename Ops<R>::SP s{};
    s.err = err;
    s.a = a;
    // radix plan 1 where the TMA passes run and the grid has it
    s.plan = (tu.tma && tu.plan == 1 && tw.N_p1) ? 1 : 0;
    s.tw = s.plan ? tw.N_p1 : tw.N;
    // double-float twiddles for wave-function arrays (X = N) only: the
    // half-spectrum (density / potential) transforms keep single twiddles
    s.tw_lo = X == g.N ? (s.plan ? tw.N_p1_lo : tw.N_lo) : nullptr;
    s.X = X;
    s.dim = g.dim;
    s.N = g.N;
    s.batch = g.B;
    s.scale = 1.0;
    return s;
}

template <typename R> void B200FFTBackend<R>::forward_c2c(void* data) {
    C* d = static_cast<C*>(data);
    auto a = xp0<R>(g_, tw_);
    a.in = d;
    a.out = d;
    Ops<R>::x_fwd(g_.N, a, false, *tune_, st_);
    if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp0<R>(err_, g_, d, tw_, g_.N, *tune_), -1, *tune_, st_);
    Ops<R>::la_pass(g_.N, sp0<R>(err_, g_, d, tw_, g_.N, *tune_), OP_FWD, *tune_, st_);
}

template <typename R> void B200FFTBackend<R>::forward_c2c_partial(const C* in, C* out) {
    auto a = xp0<R>(g_, tw_);
    a.in = in;
    a.out = out;
    Ops<R>::x_fwd(g_.N, a, false, *tune_, st_);
    if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp0<R>(err_, g_, out, tw_, g_.N, *tune_), -1, *tune_, st_);
}

template <typename R> void B200FFTBackend<R>::backward_c2c(void* data) {
    C* d = static_cast<C*>(data);
    Ops<R>::la_pass(g_.N, sp0<R>(err_, g_, d, tw_, g_.N, *tune_), OP_INV, *tune_, st_);
    if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp0<R>(err_, g_, d, tw_, g_.N, *tune_), +1, *tune_, st_);
    auto a = xp0<R>(g_, tw_);
    a.in = d;
    a.out = d;
    Ops<R>::x_inv(g_.N, a, false, *tune_, st_);
}

template <typename R> void B200FFTBackend<R>::forward_r2c(void* in_real, void* out_half) {
    C* h = static_cast<C*>(out_half);
    auto a = xp0<R>(g_, tw_);
    a.Vin = static_cast<const R*>(in_real);
    a.vh = h;
    Ops<R>::x_r2c(g_.N, a, true, *tune_, st_);
    if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp0<R>(err_, g_, h, tw_, g_.N / 2, *tune_), -1, *tune_, st_);
    Ops<R>::la_pass(g_.N, sp0<R>(err_, g_, h, tw_, g_.N / 2, *tune_), OP_FWD, *tune_, st_);
}

template <typename R> void B200FFTBackend<R>::backward_c2r(void* in_half, void* out_real) {
    C* h = static_cast<C*>(in_half);
    Ops<R>::la_pass(g_.N, sp0<R>(err_, g_, h, tw_, g_.N / 2, *tune_), OP_INV, *tune_, st_);
    if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp0<R>(err_, g_, h, tw_, g_.N / 2, *tune_), +1, *tune_, st_);
    auto a = xp0<R>(g_, tw_);
    a.vh = h;
    a.Vout = static_cast<R*>(out_real);
    Ops<R>::x_c2r(g_.N, a, C2R_WRITE_V, *tune_, st_);
}

template class B200FFTBackend<float>;
template class B200FFTBackend<double>;

// ---------------------------------------------------------------------------
// Field
// ---------------------------------------------------------------------------

void Field::updateTime() {  // src/field.cxx:349-361
    curr_ += 1;
    if (cosmo_ == 1) {  // MRE: the step follows a, then a advances
        ds_ = 0.00025 / a_;
        a_ = a_ * (1 + 1.27 * 1.27 * std::sqrt(1 + a_) * ds_);
    }
    s_ += ds_;
}

void Field::set_cosmology(int cosmo, double ai) {  // src/field.cxx:70-90
    if (cosmo == 0) {
        cosmo_ = 0;
        a_ = 1.0;
        ds_ = cfg_.dt;
    } else if (cosmo == 1) {
        if (!(ai > 0)) throw std::invalid_argument("MRE needs ai > 0");
        cosmo_ = 1;
        a_ = ai;
        ds_ = cfg_.dt / ai;
        s_ = 0.0;  // the reference leaves s unset here
        cfg_.rho_mean = 1.5 * kTwoPi * kTwoPi * 1.27 * 1.27;
    } else {
        throw std::invalid_argument("cosmology must be 0 (STATIC) or 1 (MRE)");
    }
    invalidate_graph();
}

void Field::drift_update() {  // src/field.cxx:378-386
    drift(ds_);
    updateTime();
    updatePotential();
}

void Field::propagate() {  // src/field.cxx:388-402
    kick(0.5 * ds_);
    drift(ds_);
    updateTime();
    updatePotential();
    kick(0.5 * ds_);
}

// ---------------------------------------------------------------------------
// autotuner cache: "v3 dim N dtype batch : x_rows y_tx la_tx tma nbuf pw plan wp ms"
// ---------------------------------------------------------------------------

static std::map<std::string, std::pair<Tune, double>>& tune_cache() {
    static std::map<std::string, std::pair<Tune, double>> c;
    return c;
}

void clear_tune_cache() { tune_cache().clear(); }

static bool tune_lookup(const std::string& key, const char* path, Tune& t, double& ms) {
    auto& c = tune_cache();
    auto it = c.find(key);
    if (it == c.end() && path && *path) {
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            const auto colon = line.find(" : ");
            if (colon == std::string::npos || line.compare(0, colon, key) != 0 || colon != key.size()) continue;
            std::istringstream vs(line.substr(colon + 3));
            Tune u;
            double m = 0.0;
            if (vs >> u.x_rows >> u.y_tx >> u.la_tx >> u.tma >> u.nbuf >> u.pw >> u.plan >> u.wp >> m) c[key] = {u, m};
        }
        it = c.find(key);
    }
    if (it == c.end()) return false;
    t = it->second.first;
    ms = it->second.second;
    return true;
}

static void tune_store(const std::string& key, const char* path, const Tune& t, double ms) {
    tune_cache()[key] = {t, ms};
    if (path && *path) {
        std::ofstream out(path, std::ios::app);
        out << key << " : " << t.x_rows << " " << t.y_tx << " " << t.la_tx << " " << t.tma << " " << t.nbuf << " "
            << t.pw << " " << t.plan << " " << t.wp << " " << ms << "\n";
    }
}

template <typename R>
class FieldT final : public Field {
  public:
    using C = typename Ops<R>::C;

    explicit FieldT(const FieldConfig& cfg) {
        cfg_ = cfg;
        if (cfg.dim != 2 && cfg.dim != 3) throw std::invalid_argument("Dimension must be 2 or 3");
        if (!supported_n(cfg.N)) throw std::invalid_argument("unsupported grid size N=" + std::to_string(cfg.N));
        if (!(cfg.L > 0.0)) throw std::invalid_argument("box size L must be positive");
        if (cfg.device >= 0) QX_CUDA(cudaSetDevice(cfg.device));
        QX_CUDA(cudaGetDevice(&device_));
        g_.dim = cfg.dim;
        g_.N = cfg.N;
        if (cfg.batch < 1) throw std::invalid_argument("batch must be >= 1");
        g_.B = cfg.batch;
        g_.rows = (long)cfg.batch * (cfg.dim == 3 ? (long)cfg.N * cfg.N : cfg.N);
        g_.S = g_.rows * cfg.N;
        g_.S1 = g_.S / cfg.batch;
        g_.hsites = g_.rows * (cfg.N / 2);
        ds_ = cfg.dt;
        QX_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
        psi_.alloc(sizeof(C) * g_.S);
        V_.alloc(sizeof(R) * g_.S);
        vh_.alloc(sizeof(C) * g_.hsites);
        red_.alloc(sizeof(double) * 2 * kRedBlocks);
        redout_.alloc(sizeof(double) * 4);
        errbuf_.alloc(sizeof(int));
        err_ = errbuf_.as<int>();
        QX_CUDA(cudaMemsetAsync(errbuf_.p, 0, sizeof(int), st_));
        auto tN = twiddles<C>(cfg.N), tM = twiddles<C>(cfg.N / 2);
        auto tNl = twiddles_lo<C>(cfg.N, tN), tMl = twiddles_lo<C>(cfg.N / 2, tM);
        // stage-major FFT tables (same values, reordered per stage)
        std::vector<C> sN(tN.size(), C{0, 0}), sM(tM.size(), C{0, 0}), sNl(tN.size(), C{0, 0}),
            sMl(tM.size(), C{0, 0});
        Ops<R>::stage_twiddles(tN.data(), cfg.N, sN.data());
        Ops<R>::stage_twiddles(tNl.data(), cfg.N, sNl.data());
        Ops<R>::stage_twiddles(tM.data(), cfg.N / 2, sM.data());
        Ops<R>::stage_twiddles(tMl.data(), cfg.N / 2, sMl.data());
        auto upload = [&](DevBuf& b, const std::vector<C>& h) {
            b.alloc(sizeof(C) * h.size());
            QX_CUDA(cudaMemcpy(b.p, h.data(), sizeof(C) * h.size(), cudaMemcpyHostToDevice));
        };
        upload(twN_, sN);
        upload(twM_, sM);
        upload(twNl_, sNl);
        upload(twMl_, sMl);
        upload(twNn_, tN);
        tw_ = TwTables<C>{twN_.as<C>(), twM_.as<C>(), twNl_.as<C>(), twMl_.as<C>(), twNn_.as<C>(), nullptr, nullptr};
        if (Ops<R>::has_plan1(cfg.N)) {
            std::vector<C> sP(tN.size(), C{0, 0}), sPl(tN.size(), C{0, 0});
            Ops<R>::stage_twiddles(tN.data(), plan_tagged(cfg.N, 1), sP.data());
            Ops<R>::stage_twiddles(tNl.data(), plan_tagged(cfg.N, 1), sPl.data());
            upload(twP_, sP);
            upload(twPl_, sPl);
            tw_.N_p1 = twP_.as<C>();
            tw_.N_p1_lo = twPl_.as<C>();
        }
        QX_CUDA(cudaMemsetAsync(psi_.p, 0, psi_.bytes, st_));
        QX_CUDA(cudaMemsetAsync(V_.p, 0, V_.bytes, st_));
        QX_CUDA(cudaMemsetAsync(vh_.p, 0, vh_.bytes, st_));
        fft_ = std::make_unique<B200FFTBackend<R>>(g_, tw_, &tune_, st_, err_);
        // measured default: at 512^3 FP32 the wave-function passes run faster with
        // one warp per pencil pair (the drift pass with two warps per pair), the
        // half-spectrum passes with the 8-column tiles
        if (sizeof(R) == 4 && cfg.dim == 3 && cfg.N == 512) tune_.wp = 3;
        consult_tune_cache();
        // drift chain: phase counters (as many as 8-column slabs need)
        chain_n_ = Ops<R>::chain_slabs(g_.N, g_.dim, g_.B, 1);
        if (chain_n_) chain_.alloc(sizeof(unsigned) * 3 * (size_t)chain_n_);
        QX_CUDA(cudaStreamSynchronize(st_));
    }

    ~FieldT() override {
        drop_graph();
        if (st_) {
            cudaStreamSynchronize(st_);
            cudaStreamDestroy(st_);
        }
    }

    // ---- derived constants ----
    double dk() const { return kTwoPi / cfg_.L; }
    // FFT normalisations are per box (S1 sites; S1 = S for a single box)
    double pois_c() const { return -1.0 / (dk() * dk() * (double)g_.S1); }
    double pois_g0() const { return cfg_.k0 == K0::Reference ? -1.0 / (double)g_.S1 : 0.0; }
    C* psi() { return psi_.as<C>(); }
    R* V() { return V_.as<R>(); }
    C* vh() { return vh_.as<C>(); }

    typename Ops<R>::XP xp() { return xp0<R>(g_, tw_); }
    typename Ops<R>::SP sp(C* a, int X) { return sp0<R>(err_, g_, a, tw_, X, tune_); }

    // ---- pass sequences ----
    void y_fwd(C* a, int X) {
        if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp(a, X), -1, tune_, st_);
    }
    void y_inv(C* a, int X) {
        if (g_.dim == 3) Ops<R>::y_pass(g_.N, g_.B * g_.N, sp(a, X), +1, tune_, st_);
    }
    // drift factor tables A(nx, ny), B(nz)/S for time step dt (recomputed only
    // when dt changes; capture_body computes them before a capture begins)
    const double2* ensure_axy(double dt) {
        const double fac = -0.5 * dt * dk() * dk();
        if (!axy_.p) axy_.alloc(sizeof(double2) * (size_t)g_.N * ((g_.dim == 3 ? g_.N : 1) + 1));
        if (!(axy_fac_ == fac)) {
            drift_tables(axy_.as<double2>(), g_.dim, g_.N, fac, 1.0 / (double)g_.S1, st_);
            axy_fac_ = fac;
        }
        return axy_.as<double2>();
    }
    void la_drift(double dt) {
        auto s = sp(psi(), g_.N);
        s.phase_fac = -0.5 * dt * dk() * dk();
        s.scale = 1.0 / (double)g_.S1;
        s.axy = ensure_axy(dt);
        Ops<R>::la_pass(g_.N, s, OP_DRIFT, tune_, st_);
    }
    // psi^_x -> y forward, z drift, y inverse: one slab-ordered kernel (FP32
    // 3D, tune_.chain) or three passes
    bool chain_on() const {
        return chain_n_ && tune_.tma && tune_.plan == 0 && Ops<R>::chain_slabs(g_.N, g_.dim, g_.B, tune_.chain);
    }
    void yz_drift(double dt) {
        if (chain_on()) {
            auto s = sp(psi(), g_.N);
            s.phase_fac = -0.5 * dt * dk() * dk();
            s.scale = 1.0 / (double)g_.S1;
            Ops<R>::drift_chain(g_.N, s, tune_.chain, chain_.as<unsigned>(), tune_, st_);
            return;
        }
        y_fwd(psi(), g_.N);
        la_drift(dt);
        y_inv(psi(), g_.N);
    }
    void la_poisson() {
        auto s = sp(vh(), g_.N / 2);
        s.pois_c = pois_c();
        s.pois_g0 = pois_g0();
        Ops<R>::la_pass(g_.N, s, OP_POISSON, tune_, st_);
    }
    // density source -> half spectrum, transformed along all axes but the
    // last (ready for the fused last-axis Poisson pass)
    void density_r2c_partial() {
        auto a = xp();
        a.in = psi();
        a.vh = vh();
        a.pref = pref_eff();
        a.rho_mean = cfg_.rho_mean;
        Ops<R>::x_r2c(g_.N, a, false, tune_, st_);
        y_fwd(vh(), g_.N / 2);
    }

    // ---- reference operator surface ----
    void kick(double dt) override { Misc<R>::kick(psi(), V(), dt, g_.S, st_); }

    void drift(double dt) override {  // src/field.cxx:119-198
        auto a = xp();
        a.in = psi();
        a.out = psi();
        Ops<R>::x_fwd(g_.N, a, false, tune_, st_);
        yz_drift(dt);
        Ops<R>::x_inv(g_.N, a, false, tune_, st_);
        v_current_ = false;
    }

    void Poisson() override {
        single_box("Poisson");
        Misc<R>::poisson_packed(vh(), g_.dim, g_.N, pois_c(), pois_g0(), st_);
    }

    void updatePotential() override {  // src/field.cxx:294-346
        density_r2c_partial();
        la_poisson();
        y_inv(vh(), g_.N / 2);
        auto a = xp();
        a.vh = vh();
        a.Vout = V();
        Ops<R>::x_c2r(g_.N, a, C2R_WRITE_V, tune_, st_);
        v_current_ = true;
        vmax_ = reduce(RED_VABS)[1];
    }

    void computeEnergy() override {  // src/field.cxx:200-227 (overwrites V with rho)
        Misc<R>::rho_to_V(psi(), V(), g_.S, st_);
        auto r = reduce(RED_RHO);
        rhomax_ = r[1] / (r[0] / (double)g_.S);
        v_current_ = false;
    }

    // prologue of the merged loop: potential of psi, half kick, forward x
    // transform (psi left transformed along x for the first drift)
    void prologue() {
        density_r2c_partial();
        la_poisson();
        y_inv(vh(), g_.N / 2);
        auto a = xp();
        a.in = psi();
        a.out = psi();
        a.vh = vh();
        a.Vout = V();
        a.dt = 0.5 * ds_;
        Ops<R>::x_c2r(g_.N, a, C2R_KICK | C2R_FWD, tune_, st_);
    }

    // fused merged leapfrog (src/main.cxx:64-85)
    void step(int nsteps) override {
        if (nsteps <= 0) return;
        prologue();
        if (cosmo_ == 1) {
            // MRE: every step has its own drift step, prefactor (norm a) and
            // kick step (after updateTime), so the body runs without the graph
            for (int i = 0; i < nsteps; ++i) {
                const double dt_drift = ds_;
                updateTime();
                body(dt_drift, ds_, pref_eff(), i == nsteps - 1);
            }
        } else {
            // body: psi^_x -> drift -> psi, rho^ -> Poisson -> kick -> psi^_x
            for (int i = 0; i < nsteps - 1; ++i) {
                if (graph_enabled_) {
                    if (!graph_exec_ || graph_dt_ != ds_) capture_body();
                    launch_graph();
                } else {
                    body(ds_, ds_, pref_eff(), false);
                }
            }
            body(ds_, ds_, pref_eff(), true);
            for (int i = 0; i < nsteps; ++i) updateTime();  // curr_ and s_ as the reference advances them
        }
        v_current_ = true;
        vmax_stale_ = true;
    }

    void step_begin() override {
        if (cosmo_ != 0) throw std::logic_error("stepping in pieces needs the STATIC cosmology");
        prologue();
    }
    void enqueue_body(bool last) override { body(ds_, ds_, pref_eff(), last); }
    void step_end(int nsteps) override {
        for (int i = 0; i < nsteps; ++i) updateTime();
        v_current_ = true;
        vmax_stale_ = true;
    }
    void prepare_replay() override { ensure_axy(ds_); }
    void mix_desc(MixDesc& d) override {
        if (g_.dim != 3) throw std::invalid_argument("mixed-size passes are 3D only");
        if (cosmo_ != 0) throw std::logic_error("mixed-size passes need the STATIC cosmology");
        d.psi = psi();
        d.vh = vh();
        d.twN = tw_.N;
        d.twN_lo = tw_.N_lo;
        d.twM = tw_.M;
        d.twNn = tw_.N_nat;
        d.axy = ensure_axy(ds_);
        d.N = g_.N;
        d.B = g_.B;
        d.pois_c = pois_c();
        d.pois_g0 = pois_g0();
        d.pref = pref_eff();
        d.rho_mean = cfg_.rho_mean;
        d.dt_kick = ds_;
    }

    // Poisson source prefactor: pref (STATIC) or norm a with norm = 1 (MRE,
    // src/field.cxx:84-86,298)
    double pref_eff() const { return cosmo_ == 1 ? a_ : cfg_.pref; }

    // one loop iteration; last = final half kick, psi in real space, V written
    void body(double dt, double dt_kick, double pref, bool last) {
        yz_drift(dt);
        auto a = xp();
        a.in = psi();
        a.out = psi();
        a.vh = vh();
        a.Vout = V();
        a.pref = pref;
        a.rho_mean = cfg_.rho_mean;
        Ops<R>::x_inv(g_.N, a, true, tune_, st_);
        y_fwd(vh(), g_.N / 2);
        la_poisson();
        y_inv(vh(), g_.N / 2);
        if (last) {
            a.dt = 0.5 * dt_kick;
            Ops<R>::x_c2r(g_.N, a, C2R_WRITE_V | C2R_KICK | C2R_WRITE_PSI, tune_, st_);
        } else {
            a.dt = dt_kick;
            Ops<R>::x_c2r(g_.N, a, C2R_KICK | C2R_FWD, tune_, st_);
        }
    }

    // ---- measured time loop (src/main.cxx:60-85, src/meas.cxx:13-63) ----

    // loop body up to the potential: drift, density, Poisson, c2r -> V; psi
    // stays in real space (the state measure() sees after drift_update)
    void body_to_potential(double dt, double pref) {
        yz_drift(dt);
        auto a = xp();
        a.in = psi();
        a.out = psi();
        a.vh = vh();
        a.Vout = V();
        a.pref = pref;
        a.rho_mean = cfg_.rho_mean;
        Ops<R>::x_inv(g_.N, a, true, tune_, st_);
        y_fwd(vh(), g_.N / 2);
        la_poisson();
        y_inv(vh(), g_.N / 2);
        Ops<R>::x_c2r(g_.N, a, C2R_WRITE_V, tune_, st_);
    }

    void measure(unsigned mask, int number, const char* dir, MeasRecord* rec) override {
        MeasRecord r;
        r.number = number;
        r.step = curr_;
        r.time = s_;
        r.a = a_;
        const double nan = std::numeric_limits<double>::quiet_NaN();
        r.mass = r.energy = r.kinetic = r.potential = nan;
        if (mask == MEAS_NONE) {  // src/meas.cxx:18-19
            if (rec) *rec = r;
            return;
        }
        single_box("measure");
        // computeEnergy's rhomax (src/meas.cxx:30), without overwriting V
        auto rr = reduce(RED_RHO);
        rhomax_ = rr[1] / (rr[0] / (double)g_.S);
        r.rhomax = rhomax_;
        ensure_V();
        vmax_ = reduce(RED_VABS)[1];
        vmax_stale_ = false;
        r.vmax = vmax_;
        if (mask & MEAS_ENERGY) mass_energy(&r.mass, &r.energy, &r.kinetic, &r.potential);
        const std::string d = dir ? dir : "";
        auto fname = [&](const char* stem, const char* ext) {
            std::ostringstream o;
            o << d << "/" << stem << "_" << std::setw(4) << std::setfill('0') << number << ext;
            return o.str();
        };
        if ((mask & MEAS_SPECTRUM) && dir) {
            // Spectrum of rho = |psi|^2 (the V_ that computeEnergy leaves), written
            // like Spectrum::write (src/spectrum/spectrum.cxx:167-183)
            const int nb = g_.N / 2 + 1;
            std::vector<double> k(nb), P(nb);
            std::vector<long long> c(nb);
            spectrum(0, 0, nb, k.data(), P.data(), c.data());
            std::ofstream out(fname("spec", ".txt"));
            if (!out) throw std::invalid_argument("cannot open " + fname("spec", ".txt"));
            out << "# a: " << a_ << "\n";
            out << "# k_phys      P(k)          count\n";
            out << std::scientific;
            for (int b = 0; b < nb; ++b)
                if (c[b] != 0) out << k[b] << "  " << P[b] << "  " << c[b] << "\n";
        }
        if ((mask & MEAS_RHO_GRID) && dir) {
            // the density grid of IO::writeConf (src/io/io.cxx:314-340) as raw
            // FP64 in reference order, with its Header fields in a JSON file
            std::vector<double> rho(g_.S);
            std::vector<double> hp(2 * (size_t)g_.S);
            get_psi(hp.data());
            for (long i = 0; i < g_.S; ++i) rho[i] = hp[2 * i] * hp[2 * i] + hp[2 * i + 1] * hp[2 * i + 1];
            std::ofstream out(fname("field", ".rho"), std::ios::binary);
            if (!out) throw std::invalid_argument("cannot open " + fname("field", ".rho"));
            out.write(reinterpret_cast<const char*>(rho.data()), sizeof(double) * rho.size());
            std::ofstream hdr(fname("field", ".json"));
            hdr << std::setprecision(17) << "{\"N\": " << g_.N << ", \"dim\": " << g_.dim << ", \"step\": " << curr_
                << ", \"time\": " << s_ << ", \"a\": " << a_ << ", \"Lbox\": " << cfg_.L << "}\n";
        }
        if (dir) {
            std::ofstream js(d + "/measurements.jsonl", number == 0 ? std::ios::trunc : std::ios::app);
            if (!js) throw std::invalid_argument("cannot open " + d + "/measurements.jsonl");
            js << std::setprecision(17) << "{\"number\": " << r.number << ", \"step\": " << r.step
               << ", \"time\": " << r.time << ", \"a\": " << r.a << ", \"rhomax\": " << r.rhomax
               << ", \"vmax\": " << r.vmax;
            if (mask & MEAS_ENERGY)
                js << ", \"mass\": " << r.mass << ", \"energy\": " << r.energy << ", \"kinetic\": " << r.kinetic
                   << ", \"potential\": " << r.potential;
            js << "}\n";
        }
        if (mask & MEAS_CLOBBER_V) computeEnergy();  // V <- |psi|^2 as the reference's measure leaves it
        if (rec) *rec = r;
    }

    void run(int nsteps, int nmeas, unsigned mask, const char* dir, std::vector<MeasRecord>& out) override {
        if (nsteps < 0 || nmeas < 0) throw std::invalid_argument("nsteps and nmeas must be >= 0");
        const auto ml = meas_list(nsteps, nmeas);
        out.clear();
        MeasRecord r;
        measure(mask, 0, dir, &r);  // src/main.cxx:64
        if (mask != MEAS_NONE) out.push_back(r);
        if (nsteps == 0) return;
        v_current_ = false;  // src/main.cxx:65: the loop starts from updatePotential
        prologue();          // updatePotential, half_kick (src/main.cxx:65-69), x forward
        size_t next = 0;
        int number = 0;
        for (int idx = 0; idx < nsteps; ++idx) {
            const bool last = idx == nsteps - 1;
            const bool meas = next < ml.size() && (long)idx == ml[next];
            const double dt_drift = ds_;
            if (!meas) {
                if (cosmo_ == 1) {
                    updateTime();
                    body(dt_drift, ds_, pref_eff(), last);
                } else {
                    if (!last && graph_enabled_) {
                        if (!graph_exec_ || graph_dt_ != ds_) capture_body();
                        launch_graph();
                    } else {
                        body(ds_, ds_, pref_eff(), last);
                    }
                    updateTime();
                }
                continue;
            }
            // drift_update (drift, updateTime, updatePotential), then measure
            if (cosmo_ == 1) updateTime();
            body_to_potential(dt_drift, pref_eff());
            if (cosmo_ != 1) updateTime();
            v_current_ = true;
            vmax_stale_ = true;
            ++next;
            measure(mask, ++number, dir, &r);  // src/main.cxx:75-79
            out.push_back(r);
            auto a = xp();
            a.in = psi();
            a.out = psi();
            a.Vin = V();
            if (!last) {  // full_kick, then x forward for the next drift
                a.dt = ds_;
                Ops<R>::x_fwd(g_.N, a, true, tune_, st_);
            } else {      // the final half_kick (src/main.cxx:82)
                Misc<R>::kick(psi(), V(), 0.5 * ds_, g_.S, st_);
            }
        }
        // V is the potential of psi unless the last step was measured with
        // MEAS_CLOBBER_V (then it holds rho, as the reference leaves it)
        const bool last_measured = next > 0 && ml[next - 1] == (long)nsteps - 1;
        v_current_ = !(last_measured && (mask & MEAS_CLOBBER_V));
        vmax_stale_ = true;
        QX_CUDA(cudaStreamSynchronize(st_));
    }

    // replay the captured loop body; its drift pass reads the factor tables
    // of ds_, which an eager pass with another time step may have replaced
    void launch_graph() {
        ensure_axy(ds_);
        QX_CUDA(cudaGraphLaunch(graph_exec_, st_));
    }

    void capture_body() {
        drop_graph();
        ensure_axy(ds_);  // the drift table is an input of the graph, not part of it
        // one eager launch first so kernel attributes are set outside capture
        QX_CUDA(cudaStreamSynchronize(st_));
        cudaGraph_t g;
        QX_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        try {
            body(ds_, ds_, pref_eff(), false);
        } catch (...) {
            cudaStreamEndCapture(st_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        QX_CUDA(cudaStreamEndCapture(st_, &g));
        QX_CUDA(cudaGraphInstantiate(&graph_exec_, g, 0));
        cudaGraphDestroy(g);
        graph_dt_ = ds_;
    }

    void drop_graph() {
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    void invalidate_graph() override { drop_graph(); }

    // ---- reductions ----
    std::vector<double> reduce(int kind) {
        Misc<R>::reduce(kind, psi(), V(), g_.S, red_.as<double>(), redout_.as<double>(), st_);
        double h[2];
        QX_CUDA(cudaMemcpyAsync(h, redout_.p, sizeof(h), cudaMemcpyDeviceToHost, st_));
        QX_CUDA(cudaStreamSynchronize(st_));
        return {h[0], h[1]};
    }

    void rho_stats(double* rhomax, double* vmax) override {
        auto r = reduce(RED_RHO);
        rhomax_ = r[1] / (r[0] / (double)g_.S);
        if (vmax_stale_) {
            vmax_ = reduce(RED_VABS)[1];
            vmax_stale_ = false;
        }
        if (rhomax) *rhomax = rhomax_;
        if (vmax) *vmax = vmax_;
    }

    void ensure_V() {
        if (!v_current_) updatePotential();
    }

    void mass_energy(double* M, double* E, double* K, double* W) override {
        const double dV = std::pow(cfg_.L / g_.N, g_.dim);
        const double m = reduce(RED_RHO)[0] * dV;
        ensure_V();
        const double w = 0.5 * dV * reduce(RED_VRHO)[0];
        // kinetic: 1/2 dV/S sum k^2 |psi^|^2 with the last axis fused into the reduction
        mpsi_.alloc(sizeof(C) * g_.S);
        fft_->forward_c2c_partial(psi(), mpsi_.as<C>());
        auto s = sp(mpsi_.as<C>(), g_.N);
        const long cap = Ops<R>::la_blocks(g_.N, g_.N, g_.dim, OP_KIN, tune_);
        kin_.alloc(sizeof(double) * (cap + 1));
        s.partial = kin_.as<double>();
        const long nblk = Ops<R>::la_pass(g_.N, s, OP_KIN, tune_, st_);
        Misc<R>::fold_sum(kin_.as<double>(), nblk, redout_.as<double>(), st_);
        double ks = 0.0;
        QX_CUDA(cudaMemcpyAsync(&ks, redout_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
        QX_CUDA(cudaStreamSynchronize(st_));
        const double kin = 0.5 * dV / (double)g_.S1 * dk() * dk() * ks;
        if (M) *M = m;
        if (K) *K = kin;
        if (W) *W = w;
        if (E) *E = kin + w;
    }

    void spectrum(int source, int mode, int nbins, double* k, double* P, long long* count) override {
        single_box("spectrum");
        if (mode < 0 || mode > 2) throw std::invalid_argument("spectrum mode must be 0, 1 or 2");
        if (mode == 0) nbins = g_.N / 2 + 1;
        if (nbins <= 0 || nbins > 4096) throw std::invalid_argument("nbins out of range");
        const long key = ((long)mode << 20) | nbins;
        auto it = bintab_.find(key);
        if (it == bintab_.end()) {
            auto tab = spectrum_bin_table(g_.dim, g_.N, mode, nbins);
            auto buf = std::make_unique<DevBuf>();
            buf->alloc(sizeof(int) * tab.size());
            QX_CUDA(cudaMemcpy(buf->p, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice));
            it = bintab_.emplace(key, std::move(buf)).first;
        }
        mvh_.alloc(sizeof(C) * g_.hsites);
        auto a = xp();
        a.vh = mvh_.as<C>();
        if (source == 0) {
            a.in = psi();
            a.pref = 1.0;
            a.rho_mean = 0.0;
            Ops<R>::x_r2c(g_.N, a, false, tune_, st_);
        } else {
            a.Vin = V();
            Ops<R>::x_r2c(g_.N, a, true, tune_, st_);
        }
        y_fwd(mvh_.as<C>(), g_.N / 2);
        Ops<R>::la_pass(g_.N, sp(mvh_.as<C>(), g_.N / 2), OP_FWD, tune_, st_);
        const int nblk_max = 296;
        specP_.alloc(sizeof(double) * (size_t)nblk_max * nbins + sizeof(double) * nbins);
        specC_.alloc(sizeof(long long) * (size_t)nblk_max * nbins + sizeof(long long) * nbins);
        double* partP = specP_.as<double>();
        long long* partC = specC_.as<long long>();
        const int nblk = Misc<R>::spectrum_bin(mvh_.as<C>(), g_.dim, g_.N, it->second->as<int>(), nbins, partP,
                                               partC, st_);
        double* outP = partP + (size_t)nblk_max * nbins;
        long long* outC = partC + (size_t)nblk_max * nbins;
        Misc<R>::spectrum_fold(partP, partC, nblk, nbins, outP, outC, st_);
        std::vector<double> hp(nbins);
        std::vector<long long> hc(nbins);
        QX_CUDA(cudaMemcpyAsync(hp.data(), outP, sizeof(double) * nbins, cudaMemcpyDeviceToHost, st_));
        QX_CUDA(cudaMemcpyAsync(hc.data(), outC, sizeof(long long) * nbins, cudaMemcpyDeviceToHost, st_));
        QX_CUDA(cudaStreamSynchronize(st_));
        const double S2 = (double)g_.S * (double)g_.S;
        auto kax = spectrum_k_axis(g_.N, mode, nbins, cfg_.L);
        for (int b = 0; b < nbins; ++b) {
            const double p = hp[b] / S2;
            if (P) P[b] = hc[b] > 0 ? p / (double)hc[b] : p;
            if (count) count[b] = hc[b];
            if (k) k[b] = kax[b];
        }
    }

    // ---- host buffers ----
    void stage_alloc(size_t bytes) { stage_.alloc(bytes); }

    void upload_psi(const double* h, C* dst, long n_el) {
        if constexpr (sizeof(R) == 8) {
            QX_CUDA(cudaMemcpyAsync(dst, h, sizeof(C) * n_el, cudaMemcpyHostToDevice, st_));
        } else {
            const long chunk = 1L << 22;
            stage_alloc(sizeof(double2) * chunk);
            for (long o = 0; o < n_el; o += chunk) {
                const long n = std::min(chunk, n_el - o);
                QX_CUDA(cudaMemcpyAsync(stage_.p, h + 2 * o, sizeof(double2) * n, cudaMemcpyHostToDevice, st_));
                Misc<R>::from_f64(stage_.as<double2>(), dst + o, n, st_);
            }
        }
        QX_CUDA(cudaStreamSynchronize(st_));
        v_current_ = false;
        vmax_stale_ = true;
    }

    void set_psi(const double* h) override { upload_psi(h, psi(), g_.S); }

    void psi_changed() override {
        v_current_ = false;
        vmax_stale_ = true;
    }

    void scale_psi(double factor) override {
        Misc<R>::scale(psi(), factor, g_.S, st_);
        QX_CUDA(cudaStreamSynchronize(st_));
        psi_changed();
    }

    void get_psi(double* h) override { download_c(psi(), g_.S, h); }

    // ---- boxes of a batched field ----
    void check_box(int box) const {
        if (box < 0 || box >= g_.B) throw std::invalid_argument("box index out of range");
    }
    void single_box(const char* what) const {
        if (g_.B != 1) throw std::invalid_argument(std::string(what) + " needs a single-box field (batch 1)");
    }
    void set_psi_box(int box, const double* h) override {
        check_box(box);
        upload_psi(h, psi() + (long)box * g_.S1, g_.S1);
    }
    void get_psi_box(int box, double* h) override {
        check_box(box);
        download_c(psi() + (long)box * g_.S1, g_.S1, h);
    }
    void box_mass(double* M) override {
        const double dV = std::pow(cfg_.L / g_.N, g_.dim);
        std::vector<double> h(2 * g_.B);
        for (int b = 0; b < g_.B; ++b) {
            Misc<R>::reduce(RED_RHO, psi() + (long)b * g_.S1, V() + (long)b * g_.S1, g_.S1, red_.as<double>(),
                            redout_.as<double>(), st_);
            QX_CUDA(cudaMemcpyAsync(&h[2 * b], redout_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
            QX_CUDA(cudaStreamSynchronize(st_));
        }
        for (int b = 0; b < g_.B; ++b) M[b] = h[2 * b] * dV;
    }
    void ic_config_box(int box, int kind, uint64_t seed, int n_sol, double rc_lo, double rc_hi, double sigma,
                       double kc_factor, double clip, double rho0) override {
        check_box(box);
        FieldConfig c = cfg_;
        c.prec = Prec::F64;
        c.batch = 1;
        FieldT<double> tmp(c);
        tmp.ic_config(kind, seed, n_sol, rc_lo, rc_hi, sigma, kc_factor, clip, rho0);
        QX_CUDA(cudaStreamSynchronize(tmp.stream()));
        const double2* src = reinterpret_cast<const double2*>(tmp.psi_device());
        C* dst = psi() + (long)box * g_.S1;
        if constexpr (sizeof(R) == 8) {
            QX_CUDA(cudaMemcpyAsync(dst, src, sizeof(C) * g_.S1, cudaMemcpyDeviceToDevice, st_));
        } else {
            Misc<R>::from_f64(src, dst, g_.S1, st_);
        }
        QX_CUDA(cudaStreamSynchronize(st_));
        v_current_ = false;
        vmax_stale_ = true;
    }

    void download_c(const C* d, long n_el, double* h) {
        if constexpr (sizeof(R) == 8) {
            QX_CUDA(cudaMemcpyAsync(h, d, sizeof(C) * n_el, cudaMemcpyDeviceToHost, st_));
        } else {
            const long chunk = 1L << 22;
            stage_alloc(sizeof(double2) * chunk);
            for (long o = 0; o < n_el; o += chunk) {
                const long n = std::min(chunk, n_el - o);
                Misc<R>::to_f64(d + o, stage_.as<double2>(), n, st_);
                QX_CUDA(cudaMemcpyAsync(h + 2 * o, stage_.p, sizeof(double2) * n, cudaMemcpyDeviceToHost, st_));
            }
        }
        QX_CUDA(cudaStreamSynchronize(st_));
    }

    void upload_c(const double* h, C* d, long n_el) {
        if constexpr (sizeof(R) == 8) {
            QX_CUDA(cudaMemcpyAsync(d, h, sizeof(C) * n_el, cudaMemcpyHostToDevice, st_));
        } else {
            const long chunk = 1L << 22;
            stage_alloc(sizeof(double2) * chunk);
            for (long o = 0; o < n_el; o += chunk) {
                const long n = std::min(chunk, n_el - o);
                QX_CUDA(cudaMemcpyAsync(stage_.p, h + 2 * o, sizeof(double2) * n, cudaMemcpyHostToDevice, st_));
                Misc<R>::from_f64(stage_.as<double2>(), d + o, n, st_);
            }
        }
        QX_CUDA(cudaStreamSynchronize(st_));
    }

    void upload_r(const double* h, R* d, long n_el) {
        if constexpr (sizeof(R) == 8) {
            QX_CUDA(cudaMemcpyAsync(d, h, sizeof(R) * n_el, cudaMemcpyHostToDevice, st_));
        } else {
            const long chunk = 1L << 23;
            stage_alloc(sizeof(double) * chunk);
            for (long o = 0; o < n_el; o += chunk) {
                const long n = std::min(chunk, n_el - o);
                QX_CUDA(cudaMemcpyAsync(stage_.p, h + o, sizeof(double) * n, cudaMemcpyHostToDevice, st_));
                Misc<R>::real_from_f64(stage_.as<double>(), d + o, n, st_);
            }
        }
        QX_CUDA(cudaStreamSynchronize(st_));
    }

    void download_r(const R* d, long n_el, double* h) {
        if constexpr (sizeof(R) == 8) {
            QX_CUDA(cudaMemcpyAsync(h, d, sizeof(R) * n_el, cudaMemcpyDeviceToHost, st_));
        } else {
            const long chunk = 1L << 23;
            stage_alloc(sizeof(double) * chunk);
            for (long o = 0; o < n_el; o += chunk) {
                const long n = std::min(chunk, n_el - o);
                Misc<R>::real_to_f64(d + o, stage_.as<double>(), n, st_);
                QX_CUDA(cudaMemcpyAsync(h + o, stage_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st_));
            }
        }
        QX_CUDA(cudaStreamSynchronize(st_));
    }

    void set_V(const double* h) override {
        upload_r(h, V(), g_.S);
        vmax_stale_ = true;
    }
    void get_V(double* h) override { download_r(V(), g_.S, h); }

    void get_Vhat(double* h) override {
        single_box("get_Vhat");
        std::vector<double> packed(2 * g_.hsites);
        download_c(vh(), g_.hsites, packed.data());
        unpack_half(g_.dim, g_.N, packed.data(), h);
    }
    void set_Vhat(const double* h) override {
        single_box("set_Vhat");
        std::vector<double> packed(2 * g_.hsites);
        pack_half(g_.dim, g_.N, h, packed.data());
        upload_c(packed.data(), vh(), g_.hsites);
    }

    // ---- FFT plugin on host buffers (uses the measurement scratch) ----
    void host_c2c(double* data, int sign) override {
        single_box("host_c2c");
        mpsi_.alloc(sizeof(C) * g_.S);
        upload_c(data, mpsi_.as<C>(), g_.S);
        if (sign < 0) fft_->forward_c2c(mpsi_.p);
        else fft_->backward_c2c(mpsi_.p);
        download_c(mpsi_.as<C>(), g_.S, data);
    }
    void host_r2c(const double* in, double* out) override {
        single_box("host_r2c");
        mpsi_.alloc(sizeof(C) * g_.S);  // real staging inside the complex scratch
        mvh_.alloc(sizeof(C) * g_.hsites);
        upload_r(in, reinterpret_cast<R*>(mpsi_.p), g_.S);
        fft_->forward_r2c(mpsi_.p, mvh_.p);
        std::vector<double> packed(2 * g_.hsites);
        download_c(mvh_.as<C>(), g_.hsites, packed.data());
        unpack_half(g_.dim, g_.N, packed.data(), out);
    }
    void host_c2r(const double* in, double* out) override {
        single_box("host_c2r");
        mpsi_.alloc(sizeof(C) * g_.S);
        mvh_.alloc(sizeof(C) * g_.hsites);
        std::vector<double> packed(2 * g_.hsites);
        pack_half(g_.dim, g_.N, in, packed.data());
        upload_c(packed.data(), mvh_.as<C>(), g_.hsites);
        fft_->backward_c2r(mvh_.p, mpsi_.p);
        download_r(reinterpret_cast<R*>(mpsi_.p), g_.S, out);
    }
    FFTBackend* fftBackend() override { return fft_.get(); }

    // ---- initial conditions ----
    void ic_gaussian_solitons(int n, const double* rows5, double bkg) override {
        single_box("ic_gaussian_solitons");
        if constexpr (sizeof(R) == 8) {
            DevBuf rows;
            rows.alloc(sizeof(double) * 5 * (n > 0 ? n : 1));
            if (n > 0) QX_CUDA(cudaMemcpy(rows.p, rows5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice));
            IC::gauss_rho(reinterpret_cast<double2*>(psi()), g_.dim, g_.N, cfg_.L, bkg, n, rows.as<double>(), st_);
            const double mean = reduce(RED_RE)[0] / (double)g_.S;
            IC::sqrt_div(reinterpret_cast<double2*>(psi()), g_.S, mean, st_);
            QX_CUDA(cudaStreamSynchronize(st_));
            v_current_ = false;
            vmax_stale_ = true;
        } else {
            FieldConfig c = cfg_;
            c.prec = Prec::F64;
            FieldT<double> tmp(c);
            tmp.ic_gaussian_solitons(n, rows5, bkg);
            adopt_f64(tmp);
        }
    }

    void ic_config(int kind, uint64_t seed, int n_sol, double rc_lo, double rc_hi, double sigma,
                   double kc_factor, double clip, double rho0) override {
        if (g_.B > 1) {  // an ensemble group: box b gets seed + b
            for (int b = 0; b < g_.B; ++b)
                ic_config_box(b, kind, seed + (uint64_t)b, n_sol, rc_lo, rc_hi, sigma, kc_factor, clip, rho0);
            return;
        }
        if constexpr (sizeof(R) == 8) {
            double2* p = reinterpret_cast<double2*>(psi());
            if (kind == 0) {
                QX_CUDA(cudaMemsetAsync(psi_.p, 0, psi_.bytes, st_));
            } else {
                IC::noise(p, g_.S, seed, st_);
                fft_->forward_c2c(psi_.p);
                IC::grf_filter(p, g_.dim, g_.N, dk(), kc_factor * g_.N * dk(), st_);
                fft_->backward_c2c(psi_.p);
                auto r = reduce(RED_RE2);
                const double sd = std::sqrt(r[0] / (double)g_.S);
                IC::grf_finish(p, g_.S, sigma / sd, clip, st_);
            }
            if (n_sol > 0) {
                std::vector<double> par(7 * n_sol);
                for (int j = 0; j < n_sol; ++j) {
                    const U4 a = philox4x32_10((uint32_t)j, 0u, 1u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
                    const U4 b = philox4x32_10((uint32_t)j, 1u, 1u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
                    const double rc = rc_lo + (rc_hi - rc_lo) * u01(a.v[0]);
                    const double ph = kTwoPi * u01(a.v[1]);
                    par[7 * j] = rc * rc;
                    par[7 * j + 1] = std::sqrt(rho0 / (rc * rc * rc * rc));
                    par[7 * j + 2] = std::cos(ph);
                    par[7 * j + 3] = std::sin(ph);
                    par[7 * j + 4] = u01(b.v[0]);
                    par[7 * j + 5] = u01(b.v[1]);
                    par[7 * j + 6] = g_.dim == 3 ? u01(b.v[2]) : 0.0;
                }
                DevBuf dpar;
                dpar.alloc(sizeof(double) * par.size());
                QX_CUDA(cudaMemcpy(dpar.p, par.data(), sizeof(double) * par.size(), cudaMemcpyHostToDevice));
                IC::add_schive(p, g_.dim, g_.N, cfg_.L, n_sol, dpar.as<double>(), st_);
                QX_CUDA(cudaStreamSynchronize(st_));
            }
            auto r = reduce(RED_RHO);
            Misc<double>::scale(psi(), 1.0 / std::sqrt(r[0] / (double)g_.S), g_.S, st_);
            QX_CUDA(cudaStreamSynchronize(st_));
            v_current_ = false;
            vmax_stale_ = true;
        } else {
            FieldConfig c = cfg_;
            c.prec = Prec::F64;
            FieldT<double> tmp(c);
            tmp.ic_config(kind, seed, n_sol, rc_lo, rc_hi, sigma, kc_factor, clip, rho0);
            adopt_f64(tmp);
        }
    }

    void adopt_f64(FieldT<double>& src) {
        QX_CUDA(cudaStreamSynchronize(src.stream()));
        Misc<R>::from_f64(reinterpret_cast<const double2*>(src.psi_device()), psi(), g_.S, st_);
        QX_CUDA(cudaStreamSynchronize(st_));
        v_current_ = false;
        vmax_stale_ = true;
    }

    // ---- timing ----
    float time_steps(int nsteps, int use_graph) override {
        graph_enabled_ = use_graph != 0;
        if (graph_enabled_ && nsteps > 1 && (!graph_exec_ || graph_dt_ != ds_)) capture_body();
        cudaEvent_t e0, e1;
        QX_CUDA(cudaEventCreate(&e0));
        QX_CUDA(cudaEventCreate(&e1));
        QX_CUDA(cudaEventRecord(e0, st_));
        step(nsteps);
        QX_CUDA(cudaEventRecord(e1, st_));
        QX_CUDA(cudaEventSynchronize(e1));
        check_device_error();
        float ms = 0.f;
        QX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        graph_enabled_ = true;
        return ms;
    }

    double autotune(int nsteps, const char* cache_path, bool* from_cache) override {
        if (nsteps < 1) throw std::invalid_argument("autotune needs nsteps >= 1");
        const std::string key = tune_key();
        Tune cached;
        double cached_ms = 0.0;
        if (tune_lookup(key, cache_path, cached, cached_ms)) {
            tune_ = cached;
            invalidate_graph();
            if (from_cache) *from_cache = true;
            return cached_ms;
        }
        // candidates: radix plan of the strided passes, pencils per thread, ring
        // depth, y / last-axis tile widths, rows per x block (plan 1 runs 8-column tiles)
        std::vector<Tune> cands;
        const int pws[2] = {sizeof(R) == 4 ? 2 : 1, 1};
        const int nplans = Ops<R>::has_plan1(g_.N) ? 2 : 1;
        for (int plan = 0; plan < nplans; ++plan)
            for (int ip = 0; ip < (sizeof(R) == 4 ? 2 : 1); ++ip)
                for (int nb : {0, 2, 4})
                    for (int ytx : {8, 16})
                        for (int latx : {8, 16})
                            for (int xr : {0, 4}) {
                                if (plan == 1 && (ytx != 8 || latx != 8)) continue;
                                Tune t;
                                t.plan = plan;
                                t.pw = pws[ip];
                                t.nbuf = nb;
                                t.y_tx = ytx;
                                t.la_tx = latx;
                                t.x_rows = xr;
                                t.tma = 1;
                                cands.push_back(t);
                            }
        // one warp per pencil pair (FP32 N = 256, 512) for the wave-function passes
        // (wp 1, the half-spectrum passes on the default tiles) or all (wp 2); at
        // N = 512 also two warps per pair in the drift pass (3) or in every
        // wave-function pass (4)
        if (sizeof(R) == 4 && (g_.N == 256 || g_.N == 512))
            for (int wp : {1, 2, 3, 4}) {
                if (wp > 2 && g_.N != 512) continue;
                for (int nb : {0, 2})
                    for (int xr : {0, 4}) {
                        Tune t;
                        t.wp = wp;
                        t.pw = 2;
                        t.nbuf = nb;
                        t.x_rows = xr;
                        t.tma = 1;
                        cands.push_back(t);
                    }
            }
        // keep the state: tuning advances it
        DevBuf save;
        save.alloc(sizeof(C) * g_.S);
        QX_CUDA(cudaMemcpyAsync(save.p, psi_.p, sizeof(C) * g_.S, cudaMemcpyDeviceToDevice, st_));
        const Tune orig = tune_;
        double best = 1e300;
        Tune best_t = orig;
        for (const Tune& t : cands) {
            tune_ = t;
            invalidate_graph();
            try {
                time_steps(1, 1);  // warm-up, capture
                const double ms = time_steps(nsteps, 1) / nsteps;
                if (ms < best) {
                    best = ms;
                    best_t = t;
                }
            } catch (const std::exception&) {
                // a geometry this grid cannot launch (shared memory, tile width): skip it
                cudaGetLastError();
                QX_CUDA(cudaStreamSynchronize(st_));
            }
            QX_CUDA(cudaMemcpyAsync(psi_.p, save.p, sizeof(C) * g_.S, cudaMemcpyDeviceToDevice, st_));
        }
        QX_CUDA(cudaStreamSynchronize(st_));
        if (best == 1e300) {
            tune_ = orig;
            invalidate_graph();
            throw std::runtime_error("autotune: no candidate launch geometry ran");
        }
        tune_ = best_t;
        invalidate_graph();
        psi_changed();
        tune_store(key, cache_path, best_t, best);
        if (from_cache) *from_cache = false;
        return best;
    }

    std::string tune_key() const {
        return "v3 " + std::to_string(g_.dim) + " " + std::to_string(g_.N) + " " + (sizeof(R) == 4 ? "c64" : "c128") +
               " " + std::to_string(g_.B);
    }

    // apply a tuned geometry for this grid if the process cache or the file
    // named by QX_TUNE_CACHE holds one (called at construction)
    void consult_tune_cache() {
        Tune t;
        double ms = 0.0;
        if (tune_lookup(tune_key(), std::getenv("QX_TUNE_CACHE"), t, ms)) {
            tune_ = t;
            tuned_from_cache_ = true;
        }
    }
    bool tuned_from_cache() const override { return tuned_from_cache_; }

    // per-pass device time of the loop body, averaged over nsteps bodies
    void profile_step(int nsteps, std::vector<std::pair<std::string, double>>& out) override {
        const bool d3 = g_.dim == 3;
        const bool chain = chain_on();
        std::vector<std::string> names;
        if (chain) {
            names.push_back("yzy_drift_chain(psi)");
        } else {
            if (d3) names.push_back("y_fwd(psi)");
            names.push_back(d3 ? "z_drift(psi)" : "y_drift(psi)");
            if (d3) names.push_back("y_inv(psi)");
        }
        names.push_back("x_inv_r2c(psi->rho^)");
        if (d3) names.push_back("y_fwd(rho^)");
        names.push_back(d3 ? "z_poisson(rho^)" : "y_poisson(rho^)");
        if (d3) names.push_back("y_inv(rho^)");
        names.push_back("x_c2r_kick_fwd");
        const size_t np = names.size();
        std::vector<cudaEvent_t> ev(np + 1);
        for (auto& e : ev) QX_CUDA(cudaEventCreate(&e));
        std::vector<double> acc(np, 0.0);
        {  // the loop body expects the x-transformed state
            auto a = xp();
            a.in = psi();
            a.out = psi();
            Ops<R>::x_fwd(g_.N, a, false, tune_, st_);
        }
        for (int it = 0; it < nsteps; ++it) {
            size_t k = 0;
            QX_CUDA(cudaEventRecord(ev[0], st_));
            auto mark = [&]() { QX_CUDA(cudaEventRecord(ev[++k], st_)); };
            if (chain) {
                yz_drift(ds_); mark();
            } else {
                if (d3) { y_fwd(psi(), g_.N); mark(); }
                la_drift(ds_); mark();
                if (d3) { y_inv(psi(), g_.N); mark(); }
            }
            auto a = xp();
            a.in = psi(); a.out = psi(); a.vh = vh(); a.Vout = V();
            a.pref = pref_eff(); a.rho_mean = cfg_.rho_mean; a.dt = ds_;
            Ops<R>::x_inv(g_.N, a, true, tune_, st_); mark();
            if (d3) { y_fwd(vh(), g_.N / 2); mark(); }
            la_poisson(); mark();
            if (d3) { y_inv(vh(), g_.N / 2); mark(); }
            Ops<R>::x_c2r(g_.N, a, C2R_KICK | C2R_FWD, tune_, st_); mark();
            QX_CUDA(cudaEventSynchronize(ev[np]));
            for (size_t j = 0; j < np; ++j) {
                float ms = 0.f;
                QX_CUDA(cudaEventElapsedTime(&ms, ev[j], ev[j + 1]));
                acc[j] += ms;
            }
        }
        for (auto& e : ev) cudaEventDestroy(e);
        out.clear();
        for (size_t j = 0; j < np; ++j) out.emplace_back(names[j], acc[j] / nsteps);
        // back to real space (the profiled steps advanced the state by nsteps
        // full kicks and drifts)
        restore_after_profile();
    }

    void restore_after_profile() {
        // psi holds the x-transformed state after a full kick; undo the x
        // transform (1/N) so the field is back in real space.
        auto a = xp();
        a.in = psi();
        a.out = psi();
        a.scale = 1.0 / (double)g_.N;
        Ops<R>::x_inv(g_.N, a, false, tune_, st_);
        QX_CUDA(cudaStreamSynchronize(st_));
        v_current_ = false;
        vmax_stale_ = true;
    }

    void* psi_device() override { return psi_.p; }
    void* V_device() override { return V_.p; }
    void sync() override {
        QX_CUDA(cudaStreamSynchronize(st_));
        check_device_error();
    }

    // A pass kernel whose bounded wait for a tile load timed out raised the
    // flag and returned early; report it (and clear it) as an error.
    void check_device_error() {
        int h = 0;
        QX_CUDA(cudaMemcpy(&h, errbuf_.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            QX_CUDA(cudaMemset(errbuf_.p, 0, sizeof(int)));
            throw std::runtime_error("a pass kernel timed out waiting for a tile load; results are invalid");
        }
    }

  private:
    int device_ = 0;
    DevBuf psi_, V_, vh_, twN_, twM_, twNl_, twMl_, twNn_, twP_, twPl_, red_, redout_, errbuf_;
    TwTables<C> tw_{};
    int* err_ = nullptr;
    bool tuned_from_cache_ = false;
    DevBuf axy_;       // drift factor tables A(nx, ny), B(nz)/S (ensure_axy)
    double axy_fac_ = std::numeric_limits<double>::quiet_NaN();
    DevBuf chain_;     // drift chain: [3n] phase counters
    int chain_n_ = 0;  // 8-column slabs of the drift chain (0: three separate passes)
    DevBuf mpsi_, mvh_, kin_, specP_, specC_, stage_;
    std::map<long, std::unique_ptr<DevBuf>> bintab_;
    std::unique_ptr<B200FFTBackend<R>> fft_;
    bool v_current_ = false;
    bool vmax_stale_ = true;
    bool graph_enabled_ = true;
    cudaGraphExec_t graph_exec_ = nullptr;
    double graph_dt_ = 0.0;
};

std::vector<long> meas_list(long nsteps, long nmeas) {  // src/utils.cxx:8-28
    std::vector<long> out;
    if (nmeas <= 0 || nsteps <= 0) return out;
    if (nmeas == 1) return {nsteps - 1};
    out.reserve(nmeas);
    for (long k = 0; k < nmeas; ++k) out.push_back(k * (nsteps - 1) / (nmeas - 1));
    return out;
}

std::unique_ptr<Field> make_field(const FieldConfig& cfg) {
    if (cfg.prec == Prec::F64) return std::make_unique<FieldT<double>>(cfg);
    return std::make_unique<FieldT<float>>(cfg);
}

}  // namespace qx
