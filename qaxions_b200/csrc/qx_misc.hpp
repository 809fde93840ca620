// qx_misc.hpp -- host launchers of the pointwise, reduction, spectrum and
// initial-condition kernels (qx_misc.cu).  Nothing here allocates; callers
// pass device scratch.  Reductions are deterministic: a fixed grid writes
// per-block FP64 partials that one block folds in a fixed order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace qx {

constexpr int kRedBlocks = 592;   // 4 x 148 SMs: per-block partials of reductions
constexpr int kRedThreads = 256;

enum RedKind {
    RED_RHO = 0,      // out[0] = sum |psi|^2, out[1] = max |psi|^2
    RED_VABS = 1,     // out[0] = max |V|
    RED_VRHO = 2,     // out[0] = sum V |psi|^2
    RED_RE2 = 3,      // out[0] = sum (Re psi)^2  (GRF normalisation)
    RED_RE = 4,       // out[0] = sum Re psi        (IC density mean)
};

template <typename R> struct Misc {
    using C = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
    // psi <- psi exp(-i dt V)   (Field::kick, src/field.cxx:93-116)
    static void kick(C* psi, const R* V, double dt, long S, cudaStream_t st);
    // V <- |psi|^2   (Field::computeEnergy, src/field.cxx:205-211)
    static void rho_to_V(const C* psi, R* V, long S, cudaStream_t st);
    // reductions; partial must hold 2*kRedBlocks doubles, out 2 doubles
    static void reduce(int kind, const C* psi, const R* V, long S, double* partial, double* out, cudaStream_t st);
    // fold n per-block sums in order: out[0] = sum partial[0..n)
    static void fold_sum(const double* partial, long n, double* out, cudaStream_t st);
    // Poisson multiplier on a fully transformed packed half spectrum
    // (Field::Poisson, src/field.cxx:230-291)
    static void poisson_packed(C* vh, int dim, int N, double pois_c, double pois_g0, cudaStream_t st);
    // shell binning of a fully transformed packed half spectrum; part_P and
    // part_c hold nblk*nbins entries; returns nblk (the fold size)
    static int spectrum_bin(const C* vh, int dim, int N, const int* bin_of_m2, int nbins, double* part_P,
                            long long* part_c, cudaStream_t st);
    static void spectrum_fold(const double* part_P, const long long* part_c, int nblk, int nbins, double* P,
                              long long* cnt, cudaStream_t st);
    // FP64 host layout <-> device storage (device-side conversion)
    static void from_f64(const double2* src, C* dst, long n, cudaStream_t st);
    static void to_f64(const C* src, double2* dst, long n, cudaStream_t st);
    static void real_from_f64(const double* src, R* dst, long n, cudaStream_t st);
    static void real_to_f64(const R* src, double* dst, long n, cudaStream_t st);
    static void scale(C* psi, double s, long n, cudaStream_t st);
};

// drift factor tables of exp(i fac |n|^2) / S = A(nx, ny) B(nz) (FP64,
// arguments reduced mod 2 pi): A = exp(i fac (nx^2 + ny^2)) at t[y * N + x]
// for x < N and y < N (3D) or y = 0 (2D), then B = exp(i fac n^2) * scale at
// t[rowsA * N + i] for i < N (rowsA = N in 3D, 1 in 2D)
void drift_tables(double2* t, int dim, int N, double fac, double scale, cudaStream_t st);

// initial-condition kernels (FP64 only)
struct IC {
    // psi = (g, 0), g standard normal from Philox (counter (i, 0, stream, 0))
    static void noise(double2* psi, long S, uint64_t seed, cudaStream_t st);
    // multiply a natural-order full spectrum by sqrt(P(k)), P = exp(-k^2/kc^2)/k^2, P(0)=0
    static void grf_filter(double2* h, int dim, int N, double dk, double kc, cudaStream_t st);
    // psi = sqrt(1 + max(Re psi * s, clip)) + 0 i
    static void grf_finish(double2* psi, long S, double s, double clip, cudaStream_t st);
    // psi += sum_j A(r_j) exp(i phase_j), A = sqrt(rho_c)/(1 + 0.091 r^2/rc^2)^4
    // (Schive profile, periodic minimum-image r);
    // par: n x {rc^2, sqrt(rho_c), cos phase, sin phase, cx, cy, cz}
    static void add_schive(double2* psi, int dim, int N, double L, int n, const double* par, cudaStream_t st);
    // rho = bkg + sum amp/(2 pi s^3) exp(-r^2/2s^2) (non-periodic), stored as (rho, 0);
    // rows: n x {amp, sigma, x, y, z}   (SolitonsIC, src/ic/solitons.cxx:63-95)
    static void gauss_rho(double2* psi, int dim, int N, double L, double bkg, int n, const double* rows,
                          cudaStream_t st);
    // psi = sqrt(Re psi / mean) + 0 i  (src/ic/solitons.cxx:102-109)
    static void sqrt_div(double2* psi, long S, double mean, cudaStream_t st);
};

}  // namespace qx
