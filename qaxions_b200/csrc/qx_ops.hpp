// qx_ops.hpp -- host-side launchers of the pass kernels (no CUDA templates
// exposed).  One instantiation per precision lives in qx_ops_f32.cu /
// qx_ops_f64.cu.  All launches go to the caller's stream; nothing allocates.
#pragma once

#include <cuda_runtime.h>

namespace qx {

// supported grid sizes N (per axis)
bool supported_n(int N);

// transform length n tagged with a radix plan (the encoding of qx_with_plan in
// qx_fft.cuh: the plan index in the bits above 16)
constexpr int plan_tagged(int n, int plan) { return n | (plan << 16); }

enum XC2R { C2R_WRITE_V = 1, C2R_KICK = 2, C2R_WRITE_PSI = 4, C2R_FWD = 8 };
enum LaOp { OP_FWD = 0, OP_INV = 1, OP_DRIFT = 2, OP_POISSON = 3, OP_KIN = 4 };

// Launch geometry knobs (autotuned per (N, dim, precision); 0 = default).
struct Tune {
    int x_rows = 0;   // rows per block in x passes
    int y_tx = 0;     // columns per tile in y passes
    int la_tx = 0;    // columns per tile in last-axis passes
    int tma = 1;      // strided passes: 1 = persistent TMA-fed kernels, 0 = direct-load kernels
    int nbuf = 0;     // TMA ring depth (0 = as many 64 KB-class tiles as fit in ~200 KB)
    int pw = 0;       // pencils per thread of TMA passes (0 = default: 2 in FP32, 1 in FP64)
    int wp = 0;       // FP32 strided passes at N = 256 / 512 with one warp per pencil pair
                      // (16-column swizzled tiles, warp-local stage exchanges): 1 for the
                      // wave-function arrays' passes, 2 for every strided pass, 0 none
    int plan = 0;     // radix plan of the TMA strided passes: 0 default order, 1 reversed
                      // (grids whose plan has radices of different sizes: 64, 96, 128, 256)
    int chain = 0;    // FP32 3D drift's y / z / y passes: 0 three passes; 1 / 2 one slab-ordered
                      // kernel over slabs of `chain` 8-column tiles (bit-identical, measured slower)
    int xstage = 0;   // FP32 x inverse + density + r2c pass (N >= 256): 1 = each warp copies its
                      // next row into shared memory with cp.async while it transforms the
                      // current one; 0 = direct loads (bit-identical)
};

template <typename R> struct Ops {
    using C = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
    struct XP {
        const C* in; C* out; C* vh; const R* Vin; R* Vout;
        const C* twN; const C* twM;        // stage-major FFT twiddles (N- and N/2-point)
        const C* twN_lo; const C* twM_lo;  // low parts (exact - table), FP32 double-float twiddles
        const C* twNn;                     // natural-order exp(-2 pi i k/N), k < N/2 (r2c/c2r)
        long rows; double dt, pref, rho_mean, scale;
    };
    struct SP {
        C* a; const C* tw; const C* tw_lo; int X, dim, N;
        int batch;  // boxes stacked in the array (0 or 1: a single box)
        double phase_fac, scale, pois_c, pois_g0; double* partial;
        int* err;  // device flag set when a bounded wait times out
        // drift: the factor tables A(nx, ny), B(nz) of drift_tables (qx_misc.hpp);
        // the TMA drift pass reads them
        const double2* axy;
        int plan;  // radix plan of the TMA passes; tw / tw_lo are that plan's tables
    };
    static void x_fwd(int N, const XP& a, bool kick, const Tune& tu, cudaStream_t st);
    static void x_inv(int N, const XP& a, bool r2c, const Tune& tu, cudaStream_t st);
    static void x_r2c(int N, const XP& a, bool real_src, const Tune& tu, cudaStream_t st);
    static void x_c2r(int N, const XP& a, int flags, const Tune& tu, cudaStream_t st);
    // y pass of an [outer][N][X] array (3D only)
    static void y_pass(int N, int outer, const SP& s, int sign, const Tune& tu, cudaStream_t st);
    // last-axis pass; returns the number of blocks (partials written for OP_KIN)
    static long la_pass(int N, const SP& s, int op, const Tune& tu, cudaStream_t st);
    static long la_blocks(int N, int X, int dim, int op, const Tune& tu);
    // The drift chain (y forward, z forward + drift + z inverse, y inverse) of a
    // 3D wave-function array as one kernel over x-slabs of sw 8-column tiles
    // (FP32, N >= 16, sw = 1 or 2).  chain_slabs: slabs of the array (0: the
    // chain does not apply); drift_chain: runs it with `cnt` (3 * slabs
    // counters, zeroed here) on stream st.
    static int chain_slabs(int N, int dim, int batch, int sw);
    static void drift_chain(int N, const SP& a, int sw, unsigned* cnt, const Tune& tu, cudaStream_t st);
    // stage-major FFT twiddle table of a (plan-tagged, qx_with_plan) length L
    // from the natural-order table nat[j] = exp(-2 pi i j/n), n = qx_len(L)
    // (entries beyond n - r0 are left as they are)
    static void stage_twiddles(const C* nat, int L, C* out);
    // whether the strided passes of grid size N offer radix plan 1
    static bool has_plan1(int N);
};

}  // namespace qx
