// qx_ops_impl.cuh -- definitions of Ops<R> (included by qx_ops_f32.cu and
// qx_ops_f64.cu).
#pragma once

#include <stdexcept>
#include <string>
#include <type_traits>

#include "qx_kernels.cuh"
#include "qx_ops.hpp"

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
    x.twN = a.twN; x.twM = a.twM; x.rows = a.rows; x.dt = a.dt; x.pref = a.pref;
    x.rho_mean = a.rho_mean; x.scale = a.scale;
    return x;
}
template <typename R> static SArgs<R> to_s(const typename Ops<R>::SP& a) {
    SArgs<R> s;
    s.a = a.a; s.tw = a.tw; s.X = a.X; s.dim = a.dim; s.N = a.N; s.phase_fac = a.phase_fac;
    s.scale = a.scale; s.pois_c = a.pois_c; s.pois_g0 = a.pois_g0; s.partial = a.partial;
    return s;
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

template <typename R, int NN, typename K>
static void launch_x(K kernel, const XArgs<R>& x, int P, cudaStream_t st) {
    using C = cx_t<R>;
    const int T = qx_row_threads(NN);
    const size_t smem = (size_t)P * row_smem_elems(NN) * sizeof(C);
    set_smem(kernel, smem);
    dim3 blk(T, P);
    dim3 grd((unsigned)(x.rows / P));
    kernel<<<grd, blk, smem, st>>>(x);
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
            case C2R_KICK | C2R_FWD: launch_x<R, NN>(k_x_c2r<NN, R, XC_KICK | XC_FWD>, x, P, st); break;
            case C2R_WRITE_V | C2R_KICK | C2R_FWD:
                launch_x<R, NN>(k_x_c2r<NN, R, XC_WRITE_V | XC_KICK | XC_FWD>, x, P, st); break;
            case C2R_WRITE_V | C2R_KICK | C2R_WRITE_PSI:
                launch_x<R, NN>(k_x_c2r<NN, R, XC_WRITE_V | XC_KICK | XC_WRITE_PSI>, x, P, st); break;
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

template <typename R>
void Ops<R>::y_pass(int N, int outer, const SP& a, int sign, const Tune& tu, cudaStream_t st) {
    using C = cx_t<R>;
    const SArgs<R> s = to_s<R>(a);
    QX_FOR_N(N, {
        constexpr int E = qx_col_e(NN);
        const int T = NN / E;
        auto kern = sign < 0 ? k_y_pass<NN, R, -1> : k_y_pass<NN, R, +1>;
        static int mt_cache[2] = {0, 0};
        int& mt = mt_cache[sign < 0 ? 0 : 1];
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

template <int NN, typename R>
static void (*la_kernel(int op))(SArgs<R>) {
    switch (op) {
        case OP_FWD: return k_la_pass<NN, R, LA_FWD>;
        case OP_INV: return k_la_pass<NN, R, LA_INV>;
        case OP_DRIFT: return k_la_pass<NN, R, LA_DRIFT>;
        case OP_POISSON: return k_la_pass<NN, R, LA_POISSON>;
        case OP_KIN: return k_la_pass<NN, R, LA_KIN>;
    }
    throw std::invalid_argument("la_pass: bad op");
}

template <int NN, typename R>
static int la_max_threads(int op) {
    static int cache[5] = {0, 0, 0, 0, 0};
    if (!cache[op]) cache[op] = max_threads(la_kernel<NN, R>(op));
    return cache[op];
}

template <typename R>
long Ops<R>::la_blocks(int N, int X, int dim, int op, const Tune& tu) {
    using C = cx_t<R>;
    QX_FOR_N(N, {
        constexpr int E = qx_col_e(NN);
        const int T = NN / E;
        const int G = (dim == 3 && op == OP_POISSON) ? 2 : 1;
        const int tx = pick_tx(X, T, G, tu.la_tx, sizeof(C), NN, la_max_threads<NN, R>(op));
        const long gy = dim == 3 ? (G == 2 ? NN / 2 : NN) : 1;
        return (long)(X / tx) * gy;
    });
    return 0;
}

template <typename R>
long Ops<R>::la_pass(int N, const SP& a, int op, const Tune& tu, cudaStream_t st) {
    using C = cx_t<R>;
    const SArgs<R> s = to_s<R>(a);
    QX_FOR_N(N, {
        constexpr int E = qx_col_e(NN);
        const int T = NN / E;
        const int G = (a.dim == 3 && op == OP_POISSON) ? 2 : 1;
        const int tx = pick_tx(a.X, T, G, tu.la_tx, sizeof(C), NN, la_max_threads<NN, R>(op));
        const int pitch = (tx * (int)sizeof(C) < 128) ? tx + 1 : tx;
        const size_t smem = (size_t)G * NN * pitch * sizeof(C);
        const unsigned gy = a.dim == 3 ? (G == 2 ? NN / 2 : NN) : 1;
        dim3 blk(tx, T, G), grd(a.X / tx, gy);
        auto kern = la_kernel<NN, R>(op);
        set_smem(kern, smem);
        kern<<<grd, blk, smem, st>>>(s);
        QX_LAUNCH_CHECK();
        return (long)grd.x * grd.y;
    });
    return 0;
}

}  // namespace qx
