// qx_ops_impl.cuh -- definitions of Ops<R> (included by qx_ops_f32.cu and
// qx_ops_f64.cu).
#pragma once

#include <stdexcept>
#include <string>
#include <type_traits>

#include <cudaTypedefs.h>

#include "qx_kernels.cuh"
#include "qx_ops.hpp"
#include "qx_tma.cuh"
#include "qx_yzy.cuh"

namespace qx {

#define QX_LAUNCH_CHECK()                                                                 \
    do {                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// Dispatch a template functor over the supported N.
#define QX_FOR_N(N, ...)                      \
    switch (N) {                               \
        case 4: { constexpr int NN = 4; __VA_ARGS__; break; }     \
        case 8: { constexpr int NN = 8; __VA_ARGS__; break; }     \
        case 16: { constexpr int NN = 16; __VA_ARGS__; break; }   \
        case 32: { constexpr int NN = 32; __VA_ARGS__; break; }   \
        case 64: { constexpr int NN = 64; __VA_ARGS__; break; }   \
        case 96: { constexpr int NN = 96; __VA_ARGS__; break; }   \
        case 128: { constexpr int NN = 128; __VA_ARGS__; break; } \
        case 256: { constexpr int NN = 256; __VA_ARGS__; break; } \
        case 512: { constexpr int NN = 512; __VA_ARGS__; break; } \
        default: throw std::invalid_argument("unsupported grid size N=" + std::to_string(N)); \
    }

template <typename K>
static void set_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) throw std::runtime_error(std::string("smem attribute: ") + cudaGetErrorString(e));
    }
}

template <typename R> static XArgs<R> to_x(const typename Ops<R>::XP& a) {
    XArgs<R> x;
    x.in = a.in; x.out = a.out; x.vh = a.vh; x.Vin = a.Vin; x.Vout = a.Vout;
    x.twN = a.twN; x.twM = a.twM; x.twN_lo = a.twN_lo; x.twM_lo = a.twM_lo; x.twNn = a.twNn;
    x.rows = a.rows; x.dt = a.dt; x.pref = a.pref;
    x.rho_mean = a.rho_mean; x.scale = a.scale;
    return x;
}
template <typename R> static SArgs<R> to_s(const typename Ops<R>::SP& a) {
    SArgs<R> s;
    s.a = a.a; s.tw = a.tw; s.tw_lo = a.tw_lo; s.X = a.X; s.dim = a.dim; s.N = a.N; s.phase_fac = a.phase_fac;
    s.scale = a.scale; s.pois_c = a.pois_c; s.pois_g0 = a.pois_g0; s.partial = a.partial;
    return s;
}

template <typename R>
void Ops<R>::stage_twiddles(const C* nat, int L, C* out) {
    const int S = qx_nstages(L), n = qx_len(L);
    for (int s = 1; s < S; ++s) {
        const int r = qx_radix(L, s), Ns = qx_span(L, s), stw = n / (Ns * r);
        for (int m = 1; m < r; ++m)
            for (int k = 0; k < Ns; ++k) out[qx_tw_index(L, Ns, m, k)] = nat[(k * m * stw) % n];
    }
}


// rows per block for x passes: T*P ~ 256 threads, P | rows
static int x_rows_per_block(int N, long rows, int want) {
    QX_FOR_N(N, {
        const int T = qx_row_threads(NN);
        int P = want > 0 ? want : (256 / T > 0 ? 256 / T : 1);
        while (P > 1 && (rows % P)) P >>= 1;
        return P;
    });
    return 1;
}

static int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cache[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 1;
    }
    return cache[dev];
}

template <typename R, int NN, typename K>
static void launch_x(K kernel, const XArgs<R>& x, int P, cudaStream_t st, int stage_elems = 0) {
    using C = cx_t<R>;
    const int T = qx_row_threads(NN);
    // tables + P row buffers (+ P staging buffers and alignment slack)
    const size_t smem = ((size_t)x_table_elems<NN, R>() + (size_t)P * row_smem_elems(NN) +
                         (stage_elems ? (size_t)P * stage_elems + 2 : 0)) * sizeof(C);
    set_smem(kernel, smem);
    // persistent grid: as many blocks as fit on the device at once (the
    // twiddle tables are staged once per block), at most one per P rows
    static const void* cache_k[32] = {nullptr};
    static int cache_bps[32] = {0};
    int bps = 0;
    for (int i = 0; i < 32 && cache_k[i]; ++i)
        if (cache_k[i] == (const void*)kernel) bps = cache_bps[i];
    if (!bps) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, T * P, smem) != cudaSuccess || bps < 1) bps = 1;
        for (int i = 0; i < 32; ++i)
            if (!cache_k[i]) {
                cache_k[i] = (const void*)kernel;
                cache_bps[i] = bps;
                break;
            }
    }
    const long blocks = x.rows / P;
    long grid = (long)sm_count() * bps;
    if (grid > blocks) grid = blocks;
    dim3 blk(T, P);
    kernel<<<(unsigned)grid, blk, smem, st>>>(x);
    QX_LAUNCH_CHECK();
}

template <typename R>
void Ops<R>::x_fwd(int N, const XP& a, bool kick, const Tune& tu, cudaStream_t st) {
    const XArgs<R> x = to_x<R>(a);
    const int P = x_rows_per_block(N, a.rows, tu.x_rows);
    QX_FOR_N(N, {
        if (kick) launch_x<R, NN>(k_x_fwd<NN, R, XF_KICK>, x, P, st);
        else launch_x<R, NN>(k_x_fwd<NN, R, XF_PLAIN>, x, P, st);
    });
}

template <typename R>
void Ops<R>::x_inv(int N, const XP& a, bool r2c, const Tune& tu, cudaStream_t st) {
    const XArgs<R> x = to_x<R>(a);
    const int P = x_rows_per_block(N, a.rows, tu.x_rows);
    QX_FOR_N(N, {
        if constexpr (sizeof(R) == 4 && NN >= 256) {
            // software-pipelined density + r2c pass (tu.xstage)
            if (r2c && tu.xstage == 1) {
                launch_x<R, NN>(k_x_inv<NN, R, XI_R2C | XI_STAGE>, x, P, st,
                                x_inv_stage_elems<NN, R, XI_R2C | XI_STAGE>());
                return;
            }
        }
        if (r2c) launch_x<R, NN>(k_x_inv<NN, R, XI_R2C>, x, P, st);
        else launch_x<R, NN>(k_x_inv<NN, R, XI_PLAIN>, x, P, st);
    });
}

template <typename R>
void Ops<R>::x_r2c(int N, const XP& a, bool real_src, const Tune& tu, cudaStream_t st) {
    const XArgs<R> x = to_x<R>(a);
    const int P = x_rows_per_block(N, a.rows, tu.x_rows);
    QX_FOR_N(N, {
        if (real_src) launch_x<R, NN>(k_x_r2c<NN, R, XR_REAL>, x, P, st);
        else launch_x<R, NN>(k_x_r2c<NN, R, XR_DENSITY>, x, P, st);
    });
}

template <typename R>
void Ops<R>::x_c2r(int N, const XP& a, int flags, const Tune& tu, cudaStream_t st) {
    const XArgs<R> x = to_x<R>(a);
    const int P = x_rows_per_block(N, a.rows, tu.x_rows);
    QX_FOR_N(N, {
        switch (flags) {
            case C2R_WRITE_V: launch_x<R, NN>(k_x_c2r<NN, R, XC_WRITE_V>, x, P, st); break;
            case C2R_KICK | C2R_FWD:
                launch_x<R, NN>(k_x_c2r<NN, R, XC_KICK | XC_FWD>, x, P, st,
                                x_c2r_stage_elems<NN, R, XC_KICK | XC_FWD>());
                break;
            case C2R_WRITE_V | C2R_KICK | C2R_FWD:
                launch_x<R, NN>(k_x_c2r<NN, R, XC_WRITE_V | XC_KICK | XC_FWD>, x, P, st,
                                x_c2r_stage_elems<NN, R, XC_WRITE_V | XC_KICK | XC_FWD>());
                break;
            case C2R_WRITE_V | C2R_KICK | C2R_WRITE_PSI:
                launch_x<R, NN>(k_x_c2r<NN, R, XC_WRITE_V | XC_KICK | XC_WRITE_PSI>, x, P, st,
                                x_c2r_stage_elems<NN, R, XC_WRITE_V | XC_KICK | XC_WRITE_PSI>());
                break;
            default: throw std::invalid_argument("x_c2r: unsupported flag combination");
        }
    });
}

// max threads per block the kernel can launch with (registers included)
template <typename K>
static int max_threads(K kernel) {
    cudaFuncAttributes at;
    if (cudaFuncGetAttributes(&at, kernel) != cudaSuccess) return 256;
    return at.maxThreadsPerBlock;
}

// columns per strided tile: largest power of two <= want (default 16) that
// divides X, fits the kernel's thread limit and ~100 KB of shared memory
static int pick_tx(int X, int T, int G, int want, size_t elem, int N, int maxthr) {
    int tx = want > 0 ? want : 16;
    while (tx > 1 && ((long)tx * T * G > maxthr || (X % tx) || (size_t)G * N * (tx + 1) * elem > 100 * 1024)) tx >>= 1;
    return tx;
}

// ---------------------------------------------------------------------------
// TMA-fed persistent strided passes
// ---------------------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
            throw std::runtime_error("cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Tensor map over a complex [NZ][N][X] array viewed as reals [NZ][N][2X];
// box = 2TX reals x `box` positions along dim 1 (pencil_dim 1) or dim 2.
template <typename R>
static CUtensorMap make_tmap(const void* base, int X, int N, int NZ, int TX, int box, int pencil_dim, bool swz = false) {
    CUtensorMap tm;
    cuuint64_t dims[3] = {(cuuint64_t)2 * X, (cuuint64_t)N, (cuuint64_t)NZ};
    cuuint64_t strides[2] = {(cuuint64_t)2 * X * sizeof(R), (cuuint64_t)2 * X * (cuuint64_t)N * sizeof(R)};
    cuuint32_t boxd[3] = {(cuuint32_t)(2 * TX), (cuuint32_t)(pencil_dim == 1 ? box : 1),
                          (cuuint32_t)(pencil_dim == 2 ? box : 1)};
    cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = tmap_encoder()(&tm, sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                                      3, const_cast<void*>(base), dims, strides, boxd, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      swz ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return tm;
}


// Launch geometry of a TMA pencil pass.
struct TmaGeom {
    int TX, T, nbuf, box, nbox;
    size_t tile_bytes;
};

template <int NN, typename R, int PW, int TXF>
static TmaGeom tma_geom(int X, int want_tx, int op, const Tune& tu) {
    using C = cx_t<R>;
    TmaGeom g;
    g.T = NN / tma_e<NN, R, PW>();
    // default tile: 8 columns (64-byte rows for c64, 128-byte rows for c128) and
    // a 3-deep ring, which lets two FP32 blocks share an SM (measured best at
    // 512^3 against 16 columns / deeper rings)
    int tx = want_tx > 0 ? want_tx : 8;
    if (tx > kTmaMaxTX) tx = kTmaMaxTX;
    while (tx > PW && ((X % tx) || (tx / PW) * g.T > tma_max_threads<PW>())) tx >>= 1;
    if (TXF > 0) {  // compiled-in tile width
        tx = TXF;
        if ((X % tx) || (tx / PW) * g.T > 512) throw std::logic_error("TMA tile width does not fit");
    }
    g.TX = tx;
    g.box = NN <= 256 ? NN : 256;
    g.nbox = NN / g.box;
    g.tile_bytes = ((size_t)NN * tx * sizeof(C) + 1023) & ~(size_t)1023;  // 1 KB-aligned buffer stride
    if (sizeof(R) == 4 && tx < 2) throw std::logic_error("TMA tile narrower than 16 bytes");
    // ring depth: 3, or as many tiles as fit beside the tables in ~210 KB
    const size_t tables = tma_smem_bytes<R>(NN, tx, 0, op);
    int nb = tu.nbuf > 0 ? tu.nbuf : (int)((210 * 1024 - tables) / g.tile_bytes);
    if (tu.nbuf == 0 && nb > 3) nb = 3;
    g.nbuf = nb < 2 ? 2 : (nb > 4 ? 4 : nb);
    return g;
}

// Double-float twiddles: FP32 passes given a low-part table (the host passes
// one for wave-function arrays only).  The drift and kinetic passes always act
// on psi, the Poisson pass never does.
template <typename R, int OP> constexpr bool df_only() { return sizeof(R) == 4 && (OP == OP_DRIFT || OP == OP_KIN); }
template <typename R, int OP> constexpr bool df_never() { return sizeof(R) != 4 || OP == OP_POISSON; }
template <typename R, int OP> static bool use_df(const typename Ops<R>::SP& a) {
    if constexpr (df_never<R, OP>()) return false;
    else if constexpr (df_only<R, OP>()) {
        if (!a.tw_lo) throw std::logic_error("pass needs the low twiddle table");
        return true;
    } else {
        return a.tw_lo != nullptr;
    }
}

static_assert(plan_tagged(96, 1) == qx_with_plan(96, 1), "one plan encoding for host and device");

// grids whose strided passes are also compiled with radix plan 1 (reversed
// order; only where it differs from the default)
template <int NN> constexpr bool strided_plan1() { return NN >= 64 && qx_plan1_differs(NN); }

template <typename R>
bool Ops<R>::has_plan1(int N) {
    QX_FOR_N(N, { return strided_plan1<NN>(); });
    return false;
}

// Run one TMA pencil pass over `a` ([NZ][N][X]) with radix plan PLAN (the SP's
// twiddle tables are that plan's).  Returns the grid size.
template <int NN, typename R, int OP, int PW, bool DF, int TXF, int PLAN = 0>
static long launch_tma_e(const typename Ops<R>::SP& a, int NZ, int outer, int pencil_dim, int la3d, int col0_ext,
                         const Tune& tu, cudaStream_t st) {
    const TmaGeom g = tma_geom<NN, R, PW, TXF>(a.X, pencil_dim == 2 || outer == 1 ? tu.la_tx : tu.y_tx, OP, tu);
    TArgs<R> s;
    s.tw = a.tw;
    s.tw_lo = a.tw_lo;
    s.X = a.X;
    s.N = NN;
    s.outer = outer;
    s.pencil_dim = pencil_dim;
    s.la3d = la3d;
    s.TX = g.TX;
    s.tiles_x = a.X / g.TX;
    s.nbuf = g.nbuf;
    s.nbox = g.nbox;
    s.box = g.box;
    s.n_tiles = (long)s.tiles_x * outer;
    s.phase_fac = a.phase_fac;
    s.scale = a.scale;
    s.pois_c = a.pois_c;
    s.pois_g0 = a.pois_g0;
    s.col0_external = col0_ext;
    s.axy = a.axy;
    if (OP == OP_DRIFT && !a.axy) throw std::logic_error("drift pass needs the A(nx, ny) table");
    s.partial = a.partial;
    s.err = a.err;
    constexpr bool SWZ = tma_swizzled<NN, R, PW, TXF>();
    const CUtensorMap tm = make_tmap<R>(a.a, a.X, NN, NZ, g.TX, g.box, pencil_dim, SWZ);
    auto kern = k_pencil_tma<NN, R, OP, PW, DF, TXF, PLAN>;
    const size_t smem = tma_smem_bytes<R>(NN, g.TX, g.nbuf, OP, SWZ);
    set_smem(kern, smem);
    static int bps_cache[64] = {0};
    const int key = g.nbuf * 8 + (g.TX == 16 ? 4 : g.TX == 8 ? 3 : g.TX == 4 ? 2 : g.TX == 2 ? 1 : 0);
    int& bps = bps_cache[key & 63];
    if (!bps) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, (g.TX / PW) * g.T, smem) != cudaSuccess || bps < 1)
            bps = 1;
    }
    long grid = (long)sm_count() * bps;
    if (grid > s.n_tiles) grid = s.n_tiles;
    dim3 blk(SWZ ? g.TX / PW / 2 : g.TX / PW, g.T, SWZ ? 2 : 1);
    kern<<<(unsigned)grid, blk, smem, st>>>(tm, s);
    QX_LAUNCH_CHECK();
    return grid;
}

// Warp-per-pencil-pair pass (k_pencil_wp): FP32, N = 256 / 512, paired
// pencils, 16-column swizzled tiles, a 3-deep ring, one block per SM of 8 warps
// (WPP = 1) or 16 warps, two per pencil pair (WPP = 2).
template <int NN, typename R, int OP, bool DF, int WPP = 1>
static long launch_wp(const typename Ops<R>::SP& a, int NZ, int outer, int pencil_dim, int la3d, int col0_ext,
                      cudaStream_t st) {
    if constexpr (sizeof(R) == 4 && wp_supported(NN)) {
        constexpr int TX = kWpTX;
        if (a.X % TX) throw std::logic_error("warp-pencil pass: columns not a multiple of 16");
        TArgs<R> s;
        s.tw = a.tw;
        s.tw_lo = a.tw_lo;
        s.X = a.X;
        s.N = NN;
        s.outer = outer;
        s.pencil_dim = pencil_dim;
        s.la3d = la3d;
        s.TX = TX;
        s.tiles_x = a.X / TX;
        s.nbuf = 3;
        s.box = NN <= 256 ? NN : 256;
        s.nbox = NN / s.box;
        s.n_tiles = (long)s.tiles_x * outer;
        s.phase_fac = a.phase_fac;
        s.scale = a.scale;
        s.pois_c = a.pois_c;
        s.pois_g0 = a.pois_g0;
        s.col0_external = col0_ext;
        s.axy = a.axy;
        if (OP == OP_DRIFT && !a.axy) throw std::logic_error("drift pass needs the A(nx, ny) table");
        s.partial = a.partial;
        s.err = a.err;
        const CUtensorMap tm = make_tmap<R>(a.a, a.X, NN, NZ, TX, s.box, pencil_dim, true);
        auto kern = k_pencil_wp<NN, OP, DF, 0, WPP>;
        const size_t smem = tma_smem_bytes<R>(NN, TX, s.nbuf, OP, true);
        set_smem(kern, smem);
        long grid = (long)sm_count();
        if (grid > s.n_tiles) grid = s.n_tiles;
        kern<<<(unsigned)grid, dim3(32 * WPP, kWpThreads / 32), smem, st>>>(tm, s);
        QX_LAUNCH_CHECK();
        return grid;
    } else {
        (void)a, (void)NZ, (void)outer, (void)pencil_dim, (void)la3d, (void)col0_ext, (void)st;
        throw std::logic_error("warp-pencil pass not compiled for this grid / precision");
    }
}

// tile columns: tu.la_tx (last axis) / tu.y_tx (y passes) when 8 or 16, else 8
// (FP32 16 is compiled for N >= 64: it streams z pencils faster, but at 512^3
// the FP32 passes are compute-bound and one 512-thread block per SM loses
// more than the wider rows gain).  Grids N < 16 choose at run time.
template <int NN, typename R, int OP, int PW, bool DF>
static long launch_tma_tx(const typename Ops<R>::SP& a, int NZ, int outer, int pencil_dim, int la3d, int col0_ext,
                          const Tune& tu, cudaStream_t st) {
    if constexpr (NN < 16) {
        return launch_tma_e<NN, R, OP, PW, DF, 0>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
    } else {
        const int want = (pencil_dim == 2 || outer == 1) ? tu.la_tx : tu.y_tx;
        const int tx = want == 8 || want == 16 ? want : 8;
        if constexpr (sizeof(R) == 4 && PW == 2 && wp_supported(NN)) {
            // wp 1: the wave-function arrays' passes (X = N), wp 2: every strided
            // pass; wp 3 / 4: as wp 1 with two warps per pencil pair in the z drift
            // pass / in every wave-function pass (N = 512)
            if (a.plan == 0 && (tu.wp == 2 || (tu.wp != 0 && a.X == NN))) {
                if constexpr (NN == 512 && DF && (OP == OP_FWD || OP == OP_INV || OP == OP_DRIFT)) {
                    if (tu.wp == 4 || (tu.wp == 3 && OP == OP_DRIFT))
                        return launch_wp<NN, R, OP, DF, 2>(a, NZ, outer, pencil_dim, la3d, col0_ext, st);
                }
                return launch_wp<NN, R, OP, DF>(a, NZ, outer, pencil_dim, la3d, col0_ext, st);
            }
        }
        if constexpr (strided_plan1<NN>()) {
            if (a.plan == 1) return launch_tma_e<NN, R, OP, PW, DF, 8, 1>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
        }
        if (a.plan != 0) throw std::logic_error("radix plan not compiled for this grid");
        if constexpr (sizeof(R) == 4 && NN >= 64) {
            if (tx == 16) return launch_tma_e<NN, R, OP, PW, DF, 16>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
        }
        return launch_tma_e<NN, R, OP, PW, DF, 8>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
    }
}

// pencils per thread: tu.pw, default 2 in the FP32 form (paired columns), 1 in FP64
template <int NN, typename R, int OP, bool DF>
static long launch_tma_df(const typename Ops<R>::SP& a, int NZ, int outer, int pencil_dim, int la3d, int col0_ext,
                          const Tune& tu, cudaStream_t st) {
    if constexpr (sizeof(R) == 4) {
        if (tu.pw != 1) return launch_tma_tx<NN, R, OP, 2, DF>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
    }
    return launch_tma_tx<NN, R, OP, 1, DF>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
}

template <int NN, typename R, int OP>
static long launch_tma(const typename Ops<R>::SP& a, int NZ, int outer, int pencil_dim, int la3d, int col0_ext,
                       const Tune& tu, cudaStream_t st) {
    const bool df = use_df<R, OP>(a);
    if constexpr (!df_never<R, OP>()) {
        if (df) return launch_tma_df<NN, R, OP, true>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
    }
    if constexpr (!df_only<R, OP>()) return launch_tma_df<NN, R, OP, false>(a, NZ, outer, pencil_dim, la3d, col0_ext, tu, st);
    throw std::logic_error("launch_tma: unreachable twiddle mode");
}

template <typename R>
void Ops<R>::y_pass(int N, int outer, const SP& a, int sign, const Tune& tu, cudaStream_t st) {
    using C = cx_t<R>;
    const SArgs<R> s = to_s<R>(a);
    if (tu.tma) {
        QX_FOR_N(N, {
            if (sign < 0) launch_tma<NN, R, OP_FWD>(a, outer, outer, 1, 0, 0, tu, st);
            else launch_tma<NN, R, OP_INV>(a, outer, outer, 1, 0, 0, tu, st);
        });
        return;
    }
    const bool df = use_df<R, OP_FWD>(a);
    QX_FOR_N(N, {
        constexpr int E = qx_col_e(NN);
        const int T = NN / E;
        auto kern = sign < 0 ? (df ? k_y_pass<NN, R, -1, true> : k_y_pass<NN, R, -1, false>)
                             : (df ? k_y_pass<NN, R, +1, true> : k_y_pass<NN, R, +1, false>);
        static int mt_cache[4] = {0, 0, 0, 0};
        int& mt = mt_cache[(sign < 0 ? 0 : 1) + (df ? 2 : 0)];
        if (!mt) mt = max_threads(kern);
        const int tx = pick_tx(a.X, T, 1, tu.y_tx, sizeof(C), NN, mt);
        const int pitch = (tx * (int)sizeof(C) < 128) ? tx + 1 : tx;
        const size_t smem = (size_t)NN * pitch * sizeof(C);
        dim3 blk(tx, T, 1), grd(a.X / tx, outer);
        set_smem(kern, smem);
        kern<<<grd, blk, smem, st>>>(s);
        QX_LAUNCH_CHECK();
    });
}

// direct-load last-axis kernel of an op; the FP32 drift and kinetic passes
// always take double-float twiddles, the Poisson pass never, the plain
// transforms when `df` (a wave-function array)
template <int NN, typename R>
static void (*la_kernel(int op, bool df))(SArgs<R>) {
    constexpr bool f32 = sizeof(R) == 4;
    switch (op) {
        case OP_FWD: return df ? k_la_pass<NN, R, LA_FWD, f32> : k_la_pass<NN, R, LA_FWD, false>;
        case OP_INV: return df ? k_la_pass<NN, R, LA_INV, f32> : k_la_pass<NN, R, LA_INV, false>;
        case OP_DRIFT: return k_la_pass<NN, R, LA_DRIFT, f32>;
        case OP_POISSON: return k_la_pass<NN, R, LA_POISSON, false>;
        case OP_KIN: return k_la_pass<NN, R, LA_KIN, f32>;
    }
    throw std::invalid_argument("la_pass: bad op");
}

template <int NN, typename R>
static int la_max_threads(int op, bool df) {
    static int cache[10] = {0};
    const int key = op + (df ? 5 : 0);
    if (!cache[key]) cache[key] = max_threads(la_kernel<NN, R>(op, df));
    return cache[key];
}

template <typename R>
long Ops<R>::la_blocks(int N, int X, int dim, int op, const Tune& tu) {
    using C = cx_t<R>;
    if (tu.tma) return (long)sm_count() * 32;  // upper bound of the persistent grid
    QX_FOR_N(N, {
        constexpr int E = qx_col_e(NN);
        const int T = NN / E;
        const int G = (dim == 3 && op == OP_POISSON) ? 2 : 1;
        const int tx = pick_tx(X, T, G, tu.la_tx, sizeof(C), NN, la_max_threads<NN, R>(op, X == NN));
        const long gy = dim == 3 ? (G == 2 ? NN / 2 : NN) : 1;
        return (long)(X / tx) * gy;
    });
    return 0;
}

template <int NN, typename R>
static void launch_col0(const typename Ops<R>::SP& a, cudaStream_t st) {
    using C = cx_t<R>;
    constexpr int E0 = qx_lcm_radices(NN);
    dim3 blk(2, NN / E0, 1);
    dim3 grd(NN / 2, a.batch > 0 ? a.batch : 1);
    if constexpr (strided_plan1<NN>()) {
        if (a.plan == 1) {
            k_poisson_col0<NN, R, 1><<<grd, blk, 2 * NN * sizeof(C), st>>>(a.a, a.tw, a.tw_lo, a.pois_c, a.pois_g0);
            QX_LAUNCH_CHECK();
            return;
        }
    }
    k_poisson_col0<NN, R><<<grd, blk, 2 * NN * sizeof(C), st>>>(a.a, a.tw, a.tw_lo, a.pois_c, a.pois_g0);
    QX_LAUNCH_CHECK();
}

template <typename R>
long Ops<R>::la_pass(int N, const SP& a, int op, const Tune& tu, cudaStream_t st) {
    using C = cx_t<R>;
    const SArgs<R> s = to_s<R>(a);
    const bool df = sizeof(R) == 4 && a.tw_lo != nullptr;
    if (tu.tma) {
        QX_FOR_N(N, {
            const int d3 = a.dim == 3 ? 1 : 0;
            const int nb = a.batch > 0 ? a.batch : 1;
            const int NZ = d3 ? nb * NN : nb, outer = d3 ? nb * NN : nb, pdim = d3 ? 2 : 1;
            long grid = 0;
            switch (op) {
                case OP_FWD: grid = launch_tma<NN, R, OP_FWD>(a, NZ, outer, pdim, d3, 0, tu, st); break;
                case OP_INV: grid = launch_tma<NN, R, OP_INV>(a, NZ, outer, pdim, d3, 0, tu, st); break;
                case OP_DRIFT: grid = launch_tma<NN, R, OP_DRIFT>(a, NZ, outer, pdim, d3, 0, tu, st); break;
                case OP_POISSON:
                    grid = launch_tma<NN, R, OP_POISSON>(a, NZ, outer, pdim, d3, d3, tu, st);
                    if (d3) launch_col0<NN, R>(a, st);
                    break;
                case OP_KIN: grid = launch_tma<NN, R, OP_KIN>(a, NZ, outer, pdim, d3, 0, tu, st); break;
                default: throw std::invalid_argument("la_pass: bad op");
            }
            return grid;
        });
    }
    if (a.batch > 1) throw std::invalid_argument("batched arrays need the TMA-fed strided passes");
    QX_FOR_N(N, {
        constexpr int E = qx_col_e(NN);
        const int T = NN / E;
        const int G = (a.dim == 3 && op == OP_POISSON) ? 2 : 1;
        const int tx = pick_tx(a.X, T, G, tu.la_tx, sizeof(C), NN, la_max_threads<NN, R>(op, df));
        const int pitch = (tx * (int)sizeof(C) < 128) ? tx + 1 : tx;
        const size_t smem = (size_t)G * NN * pitch * sizeof(C);
        const unsigned gy = a.dim == 3 ? (G == 2 ? NN / 2 : NN) : 1;
        dim3 blk(tx, T, G), grd(a.X / tx, gy);
        auto kern = la_kernel<NN, R>(op, df);
        set_smem(kern, smem);
        kern<<<grd, blk, smem, st>>>(s);
        QX_LAUNCH_CHECK();
        return (long)grd.x * grd.y;
    });
    return 0;
}

// ---------------------------------------------------------------------------
// drift chain: y forward / z drift / y inverse as one slab-ordered kernel
// ---------------------------------------------------------------------------

constexpr int kChainTX = 8;  // tile columns of the chain (one slab = 8 columns)

template <typename R>
int Ops<R>::chain_slabs(int N, int dim, int batch, int sw) {
    if (sizeof(R) != 4 || dim != 3 || N < 16 || sw < 1 || sw > 2 || N % (sw * kChainTX)) return 0;
    bool fits = false;
    QX_FOR_N(N, {
        if constexpr (NN >= 16) fits = yzy_fits<NN, float, 2, kChainTX>();
    });
    return fits ? (batch > 0 ? batch : 1) * (N / (sw * kChainTX)) : 0;
}

template <typename R>
void Ops<R>::drift_chain(int N, const SP& a, int sw, unsigned* cnt, const Tune& tu, cudaStream_t st) {
    const int n_slabs = chain_slabs(N, a.dim, a.batch, sw);
    if (!n_slabs || a.X != N || !a.tw_lo) throw std::logic_error("drift chain: not a 3D FP32 wave-function array");
    if constexpr (sizeof(R) == 4) {
        QX_FOR_N(N, {
            if constexpr (NN >= 16 && yzy_fits<NN, R, 2, kChainTX>()) {
                constexpr int PW = 2, TXF = kChainTX;
                const TmaGeom g = tma_geom<NN, R, PW, TXF>(a.X, TXF, OP_DRIFT, tu);
                const int nb = a.batch > 0 ? a.batch : 1;
                YZYArgs<R> s;
                s.tw = a.tw;
                s.tw_lo = a.tw_lo;
                // ring: as many tiles as fit beside the tables (at most 8)
                const size_t tile = align1k((size_t)NN * TXF * sizeof(cx_t<R>));
                int nbuf = (int)((227 * 1024 - yzy_smem_bytes<R>(NN, TXF, 0)) / tile);
                if (nbuf > 8) nbuf = 8;
                if (tu.nbuf >= 3 && tu.nbuf < nbuf) nbuf = tu.nbuf;
                if (nbuf < 3) throw std::logic_error("drift chain: ring of fewer than 3 tiles");
                s.sw = sw;
                s.slabs_x = a.X / (sw * TXF);
                s.nbuf = nbuf;
                s.nbox = g.nbox;
                s.box = g.box;
                s.n_slabs = n_slabs;
                s.n_items = 3L * n_slabs * sw * NN;
                s.cnt = cnt;
                s.phase_fac = a.phase_fac;
                s.scale = a.scale;
                s.err = a.err;
                const CUtensorMap tmy = make_tmap<R>(a.a, a.X, NN, nb * NN, TXF, g.box, 1);
                const CUtensorMap tmz = make_tmap<R>(a.a, a.X, NN, nb * NN, TXF, g.box, 2);
                auto kern = k_yzy_tma<NN, R, PW, TXF>;
                const size_t smem = yzy_smem_bytes<R>(NN, TXF, nbuf);
                set_smem(kern, smem);
                const int threads = yzy_block_threads<NN, R, PW, TXF>();
                static int bps_cache[9] = {0};
                int& bps = bps_cache[nbuf];
                if (!bps) {
                    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, threads, smem) != cudaSuccess || bps < 1)
                        throw std::runtime_error("drift chain: kernel does not fit an SM");
                }
                long grid = (long)sm_count() * bps;
                if (grid > s.n_items) grid = s.n_items;
                cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned) * 3 * (size_t)n_slabs, st);
                if (e != cudaSuccess) throw std::runtime_error(std::string("drift chain: ") + cudaGetErrorString(e));
                // cooperative: all blocks resident at once (they wait on one another's tiles)
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)grid);
                cfg.blockDim = dim3(threads, 1, 1);
                cfg.dynamicSmemBytes = smem;
                cfg.stream = st;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeCooperative;
                at[0].val.cooperative = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                e = cudaLaunchKernelEx(&cfg, kern, tmy, tmz, s);
                if (e != cudaSuccess) throw std::runtime_error(std::string("drift chain launch: ") + cudaGetErrorString(e));
            }
        });
    }
}

}  // namespace qx
