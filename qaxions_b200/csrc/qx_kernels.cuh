// qx_kernels.cuh -- pass kernels of the Schroedinger-Poisson step on sm_100a.
//
// Data layout in HBM (reference order, x fastest; src/ic/solitons.cxx:69-71):
//   psi  [N^d]       complex (float2 for the fused FP32 form, double2 for FP64)
//   vh   [N^(d-1) N/2] complex: r2c half spectrum with the self-conjugate
//        kx = N/2 plane packed into column 0 (col0 = X[kx=0] + i X[kx=N/2]
//        after the x transform; linear through the y/z transforms)
//   V    [N^d]       real potential
// A 3D transform is three passes over HBM: an x pass over contiguous rows, a
// y pass over tiles of TX columns x N rows, and a last-axis (z) pass over tiles
// of TX columns x N planes.  In 2D the y pass is the last axis.  Pointwise
// work is fused into the passes:
//   x passes    kick exp(-i dt V) before the forward x FFT; |psi|^2 density
//               and the real-to-complex x FFT after the inverse x FFT; the
//               complex-to-real x FFT, the kick and the next forward x FFT
//   last axis   drift phase exp(-i dt k^2/2)/S between the forward and inverse
//               transforms; Poisson divide -1/(k^2 S) between them on vh
// Reference operations replaced: Field::kick/drift/Poisson/updatePotential
// (src/field.cxx:93-346) and the FFTW plugin transforms (src/fft/fft.h:122-140).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "qx_fft.cuh"

namespace qx {

// ---------------------------------------------------------------------------
// shared-memory accessors
// ---------------------------------------------------------------------------

// contiguous row, one padding element per 16: with radix-8-first plans every
// Stockham exchange, the even/odd staging and contiguous reads of a row touch
// each 4-byte bank word at most as often as a conflict-free 8-byte access does
// (checked for the 512- and 256-point plans with a 32-lane bank model).  A
// row's threads all sit in one warp (qx_row_threads(N) divides 32), so its
// exchanges only need a warp barrier; `mask` names the warp's existing lanes.
template <typename C> struct RowAcc {
    C* base;
    unsigned mask;
    __device__ __forceinline__ C& operator()(int p) const { return base[p + (p >> 4)]; }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// lanes of the calling thread's warp that exist in this block
__device__ __forceinline__ unsigned warp_lanes_mask() {
    const int n = blockDim.x * blockDim.y * blockDim.z;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int left = n - (tid & ~31);
    return left >= 32 ? 0xffffffffu : ((1u << left) - 1u);
}
__host__ __device__ constexpr int row_smem_elems(int n) { return n + (n >> 4) + 1; }

// Row passes chain an N-point c2c transform with the N/2-point core of an
// r2c/c2r transform.  When both plans start with the same radix, the N-point
// transform runs with paired stage-0 columns (stage_j, J0 = 1): thread t then
// holds positions 2q and 2q+1 for every q = in_pos<N/2, E/2, 0>(e, t), the
// pairs the half-length transform consumes or produces, in registers
// v[row_pair_idx<N>(e, h)] (h = 0, 1).
template <int N> __host__ __device__ constexpr bool row_paired() {
    return N >= 16 && qx_radix(N, 0) == qx_radix(N / 2, 0) && (qx_row_efull(N) / qx_radix(N, 0)) % 2 == 0;
}
template <int N> __host__ __device__ constexpr int row_pair_idx(int e, int h) {
    constexpr int r0 = qx_radix(N, 0);
    return row_paired<N>() ? (2 * (e / r0) + h) * r0 + e % r0 : 2 * e + h;
}

// column of a strided tile: element p of this pencil at base[p * pitch]
template <typename C> struct ColAcc {
    C* base;
    int pitch;
    __device__ __forceinline__ C& operator()(int p) const { return base[p * pitch]; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// ---------------------------------------------------------------------------
// phase helpers: arguments in FP64, reduced mod 2 pi, then sin/cos in R
// ---------------------------------------------------------------------------

__device__ __forceinline__ double reduce_2pi(double phi) {
    const double inv2pi = 0.15915494309189533576888376337251436;
    const double twopi = 6.283185307179586476925286766559005768;
    return fma(-twopi, rint(phi * inv2pi), phi);
}

template <typename R> __device__ __forceinline__ cx_t<R> cis(double phi);
template <> __device__ __forceinline__ float2 cis<float>(double phi) {
    float s, c;
    sincosf((float)reduce_2pi(phi), &s, &c);
    return make_float2(c, s);
}
template <> __device__ __forceinline__ double2 cis<double>(double phi) {
    double s, c;
    sincos(reduce_2pi(phi), &s, &c);
    return make_double2(c, s);
}

// exp(i phi) in FP64 with the argument reduced mod 2 pi
__device__ __forceinline__ double2 cis_d(double phi) {
    double s, c;
    sincos(reduce_2pi(phi), &s, &c);
    return make_double2(c, s);
}
__device__ __forceinline__ double2 dcmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// v * w with w in FP64 and one rounding of the product.  A unit factor that is
// applied every step with the same value (the drift phase of each mode) must
// not be rounded to FP32 first: its fixed rounding error would compound
// linearly over the steps instead of averaging out.
template <typename C> __device__ __forceinline__ C cmul_d(C v, double2 w) {
    const double vx = v.x, vy = v.y;
    return mk<C>((decltype(C::x))fma(vx, w.x, -vy * w.y), (decltype(C::x))fma(vx, w.y, vy * w.x));
}

// exp(i phi) for the FP32 kick.  phi (FP64) is reduced in FP64 to
// r in [-pi/4, pi/4] and a quadrant q (Cody-Waite reduction with pi/2 split
// into its double and the remainder), r is rounded once to FP32, and sin r,
// cos r come from polynomials in r^2 fitted on that interval
// (fit_kick_poly.py: largest error 4.7e-8 for sin, 6.5e-8 for cos), then
// rotated by i^q.
__device__ __forceinline__ float2 cis_kick(double phi) {
    const double two_over_pi = 0.636619772367581343075535053490057448;
    const double pio2_hi = 1.57079632679489655800;   // the double nearest pi/2
    const double pio2_lo = 6.12323399573676588613e-17;  // pi/2 - pio2_hi
    const double qd = rint(phi * two_over_pi);
    const int k = (int)(__double2ll_rn(qd) & 3);
    const float r = (float)fma(-qd, pio2_lo, fma(-qd, pio2_hi, phi));
    const float r2 = r * r;
    const float sn = fmaf(r * r2, fmaf(r2, fmaf(r2, -0x1.9aca00p-13f, 0x1.110c2ap-7f), -0x1.555552p-3f), r);
    const float cs =
        fmaf(r2, fmaf(r2, fmaf(r2, fmaf(r2, 0x1.9a6fb4p-16f, -0x1.6c0e0ap-10f), 0x1.55554cp-5f), -0.5f), 1.0f);
    float re = (k & 1) ? sn : cs, im = (k & 1) ? cs : sn;
    if ((k + 1) & 2) re = -re;  // k = 1, 2
    if (k & 2) im = -im;        // k = 2, 3
    return make_float2(re, im);
}

// psi * exp(-i dt V)   (src/field.cxx:100-112).  Both forms form the phase
// -dt V in FP64 and reduce it there (FP64: mod 2 pi, then sincos; FP32: to
// [-pi/4, pi/4] and a quadrant, cis_kick).  Forming dt V in FP32 instead
// would round dt itself (a fixed relative error applied at every step) and
// lose |dt V| 6e-8 of absolute phase to the product.
template <typename R> __device__ __forceinline__ cx_t<R> kick1(cx_t<R> p, R v, double dt);
template <> __device__ __forceinline__ double2 kick1<double>(double2 p, double v, double dt) {
    return cmul(p, cis<double>(-dt * v));
}
template <> __device__ __forceinline__ float2 kick1<float>(float2 p, float v, double dt) {
    return cmul(p, cis_kick(-dt * (double)v));
}

__device__ __forceinline__ int signed_mode(int i, int N) { return i <= (N >> 1) ? i : i - N; }

// elements 2q and 2q+1 of a complex row: one 16-byte access per lane in the
// FP32 form (a lane-contiguous q then reads whole lines), two in FP64
template <typename C> __device__ __forceinline__ void load_pair(const C* row, int q, C& a, C& b) {
    if constexpr (sizeof(C) == 8) {
        const float4 v = reinterpret_cast<const float4*>(row)[q];
        a = mk<C>(v.x, v.y);
        b = mk<C>(v.z, v.w);
    } else {
        a = row[2 * q];
        b = row[2 * q + 1];
    }
}
template <typename C> __device__ __forceinline__ void store_pair(C* row, int q, C a, C b) {
    if constexpr (sizeof(C) == 8) {
        reinterpret_cast<float4*>(row)[q] = make_float4(a.x, a.y, b.x, b.y);
    } else {
        row[2 * q] = a;
        row[2 * q + 1] = b;
    }
}

// ---------------------------------------------------------------------------
// deterministic block reductions (fixed tree, FP64)
// ---------------------------------------------------------------------------

// max that keeps a NaN from either side: a NaN density or potential must show
// up in the diagnostics instead of being hidden behind a finite maximum
__device__ __forceinline__ double fmax_nan(double a, double b) { return (a > b || a != a) ? a : b; }

template <int OP>  // 0 sum, 1 max (NaN-propagating)
__device__ __forceinline__ double red_op(double a, double b) { return OP == 0 ? a + b : fmax_nan(a, b); }

template <int OP>
__device__ double block_reduce(double v, double* red) {
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if ((nthr & 31) == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = red_op<OP>(v, __shfl_xor_sync(0xffffffffu, v, o));
        __syncthreads();
        if ((tid & 31) == 0) red[tid >> 5] = v;
        __syncthreads();
        double r = red[0];
        for (int w = 1; w < (nthr >> 5); ++w) r = red_op<OP>(r, red[w]);
        __syncthreads();
        return r;
    }
    __syncthreads();
    red[tid] = v;
    __syncthreads();
    double r = red[0];
    for (int w = 1; w < nthr; ++w) r = red_op<OP>(r, red[w]);
    __syncthreads();
    return r;
}

// One warp folds n per-block partials in a fixed order (deterministic): lane l
// takes l, l + 32, ... in turn, then a fixed shuffle tree; every lane returns
// the result.  Call with all 32 lanes of the warp.
template <int OP>
__device__ __forceinline__ double warp_fold(const double* p, long n) {
    double v = OP == 0 ? 0.0 : -CUDART_INF;
    for (long i = threadIdx.x & 31; i < n; i += 32) v = red_op<OP>(v, p[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = red_op<OP>(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// x passes (contiguous rows).  blockDim = (T, P): T = qx_row_threads(N)
// threads per row, P rows per block; persistent grid, each warp loops over its
// rows.  Dynamic smem: twiddle tables (x_table_elems) + P * row_smem_elems(N) C.
// ---------------------------------------------------------------------------

template <typename R> struct XArgs {
    const cx_t<R>* in;      // complex rows of N (psi or psi^_x)
    cx_t<R>* out;           // complex rows of N
    cx_t<R>* vh;            // packed half rows of N/2
    const R* Vin;           // real rows of N (potential for the kick / r2c source)
    R* Vout;                // real rows of N
    const cx_t<R>* twN;     // stage-major N-point FFT twiddles (qx_tw_index)
    const cx_t<R>* twM;     // stage-major N/2-point FFT twiddles
    const cx_t<R>* twN_lo;  // exact - twN (double-float twiddles of the FP32 form)
    const cx_t<R>* twM_lo;
    const cx_t<R>* twNn;    // natural-order exp(-2 pi i k/N), k < N/2 (r2c/c2r)
    long rows;
    double dt;              // kick time step
    double pref, rho_mean;  // r2c source pref*(|psi|^2 - rho_mean)
    double scale;           // applied after an inverse c2c (1/S when requested)
};

// shared twiddle tables of a row pass (complex elements): N-point FFT table,
// its low part (FP32 only), N/2-point FFT table, natural-order k < N/2 table
template <int N, typename R> __host__ __device__ constexpr int x_table_elems() {
    return N + (sizeof(R) == 4 ? N : 0) + N / 2 + N / 2;
}

template <typename C> struct XTabs {
    const C* N;
    const C* N_lo;
    const C* M;
    const C* Nn;
};

// Copy the twiddle tables into shared memory once per (persistent) block and
// return the row buffer of the calling thread's row slot.
template <int N, typename R>
__device__ __forceinline__ cx_t<R>* x_setup(const XArgs<R>& a, unsigned char* smem, XTabs<cx_t<R>>& tb) {
    using C = cx_t<R>;
    C* tN = reinterpret_cast<C*>(smem);
    C* tNl = tN + N;
    C* tM = tNl + (sizeof(R) == 4 ? N : 0);
    C* tNn = tM + N / 2;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    for (int i = tid; i < N; i += nthr) {
        tN[i] = a.twN[i];
        if constexpr (sizeof(R) == 4) tNl[i] = a.twN_lo[i];
    }
    for (int i = tid; i < N / 2; i += nthr) {
        tM[i] = a.twM[i];
        tNn[i] = a.twNn[i];
    }
    __syncthreads();
    tb = XTabs<C>{tN, sizeof(R) == 4 ? tNl : tN, tM, tNn};
    return tN + x_table_elems<N, R>() + threadIdx.y * row_smem_elems(N);
}

// first row of this thread's row slot and the row stride of the grid
__device__ __forceinline__ long x_row0() { return (long)blockIdx.x * blockDim.y + threadIdx.y; }
__device__ __forceinline__ long x_row_step() { return (long)gridDim.x * blockDim.y; }

// cp.async 16-byte copy global -> shared (no register round trip) and its groups
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
                 "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }


// per-warp staging buffer after the P row buffers (16-byte aligned for cp.async)
template <int N, typename C> __device__ __forceinline__ C* x_stage_ptr(C* row_buf, int stage_elems) {
    C* end = row_buf - threadIdx.y * row_smem_elems(N) + blockDim.y * row_smem_elems(N);
    return reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(end) + 15) & ~(uintptr_t)15) + threadIdx.y * stage_elems;
}

enum XFwdMode { XF_PLAIN = 0, XF_KICK = 1 };

// forward c2c along x; optional kick by V first.  (Field::kick + first FFT pass)
template <int N, typename R, int MODE>
__global__ void __launch_bounds__(256, 3) k_x_fwd(XArgs<R> a) {
    using C = cx_t<R>;
    constexpr int E = qx_row_efull(N);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    XTabs<C> tb;
    C* sm = x_setup<N, R>(a, smem_raw, tb);
    const int t = threadIdx.x;
    RowAcc<C> acc{sm, warp_lanes_mask()};
    for (long row = x_row0(); row < a.rows; row += x_row_step()) {
        acc.sync();  // this slot's previous row is done with the buffer
        const C* src = a.in + row * N;
        C v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int p = in_pos<N, E, 0>(e, t);
            v[e] = src[p];
            if constexpr (MODE == XF_KICK) v[e] = kick1<R>(v[e], a.Vin[row * N + p], a.dt);
        }
        fft_pencil<N, E, -1>(v, acc, t, tw_src<true>(tb.N, tb.N_lo));
        C* dst = a.out + row * N;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[out_pos<N, E>(e, t)] = v[e];
    }
}

// r2c post-processing of one row held in smem (Z[k], k < M) -> packed X row.
// X[k] = (A + B)/2 - i W_N^k (A - B)/2, A = Z[k], B = conj(Z[M-k]);
// col 0 = (Re Z0 + Im Z0) + i (Re Z0 - Im Z0) = X[0] + i X[N/2].
template <int N, typename R>
__device__ __forceinline__ void r2c_post_store(RowAcc<cx_t<R>>& acc, int t, cx_t<R>* dst, const cx_t<R>* twN) {
    using C = cx_t<R>;
    constexpr int M = N / 2;
    constexpr int T = qx_row_threads(N);
#pragma unroll
    for (int i = 0; i < M / T; ++i) {
        const int k = t + i * T;
        const C A = acc(k);
        C x;
        if (k == 0) {
            x = mk<C>(A.x + A.y, A.x - A.y);
        } else {
            const C B = cconj(acc(M - k));
            const C s = cadd(A, B), d = csub(A, B);
            const C w = twN[k];
            // -i * w * d
            const C wd = cmul(w, d);
            x = mk<C>(R(0.5) * (s.x + wd.y), R(0.5) * (s.y - wd.x));
        }
        dst[k] = x;
    }
}

enum XInvMode { XI_PLAIN = 0, XI_R2C = 1, XI_STAGE = 2 };

// staging buffer of an x inverse row pass with XI_STAGE (FP32): the next row (N)
template <int N, typename R, int MODE> __host__ __device__ constexpr int x_inv_stage_elems() {
    return (sizeof(R) == 4 && (MODE & XI_STAGE)) ? N : 0;
}

// inverse c2c along x (psi^_x -> psi, times scale); optionally (XI_R2C) the
// density source pref(|psi|^2 - rho_mean) and its r2c x transform into vh.
// XI_STAGE (FP32): software-pipelined like the kicking c2r pass -- once every
// lane has read its row from the staging buffer, the warp copies its next row
// there with cp.async, so that row arrives while the current one is transformed.
template <int N, typename R, int MODE>
__global__ void __launch_bounds__(256, 2) k_x_inv(XArgs<R> a) {
    using C = cx_t<R>;
    constexpr int E = qx_row_efull(N);
    constexpr int M = N / 2;
    constexpr int EH = E / 2;
    constexpr int T = qx_row_threads(N);
    constexpr bool PAIRED = row_paired<N>();
    constexpr int SE = x_inv_stage_elems<N, R, MODE>();
    constexpr bool STAGE = SE > 0;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    XTabs<C> tb;
    C* sm = x_setup<N, R>(a, smem_raw, tb);
    const int t = threadIdx.x;
    RowAcc<C> acc{sm, warp_lanes_mask()};
    C* stg = x_stage_ptr<N>(sm, SE);
    auto prefetch = [&](long r) {
        if constexpr (STAGE) {
            const char* gp = reinterpret_cast<const char*>(a.in + r * N);
            char* sp = reinterpret_cast<char*>(stg);
            for (int i = t; i < (int)(N * sizeof(C) / 16); i += T) cp_async16(sp + 16 * i, gp + 16 * i);
            cp_async_commit();
        }
    };
    if (STAGE && x_row0() < a.rows) prefetch(x_row0());
    for (long row = x_row0(); row < a.rows; row += x_row_step()) {
        acc.sync();
        C v[E];
        if constexpr (STAGE) {
            cp_async_wait_all();
            acc.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = stg[out_pos<N, E>(e, t)];
            // every lane has its values: fetch the next row
            acc.sync();
            const long nrow = row + x_row_step();
            if (nrow < a.rows) prefetch(nrow);
        } else {
            const C* src = a.in + row * N;
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = src[out_pos<N, E>(e, t)];
        }
        ifft_pencil_rev<N, E, PAIRED ? 1 : 0>(v, acc, t, tw_src<true>(tb.N, tb.N_lo));
        const R sc = (R)a.scale;
        C* dst = a.out + row * N;
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = cscale(v[e], sc);
        if constexpr (PAIRED) {
#pragma unroll
            for (int e = 0; e < EH; ++e)
                store_pair(dst, in_pos<M, EH, 0>(e, t), v[row_pair_idx<N>(e, 0)], v[row_pair_idx<N>(e, 1)]);
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) dst[in_pos<N, E, 0>(e, t)] = v[e];
        }
        if constexpr ((MODE & XI_R2C) != 0) {
            const R pr = (R)a.pref, rm = (R)a.rho_mean;
            auto src_of = [&](const C& u) { return pr * (u.x * u.x + u.y * u.y - rm); };
            C z[EH];  // (rho[2q], rho[2q+1]), q = in_pos<M, EH, 0>(e, t)
            if constexpr (PAIRED) {
#pragma unroll
                for (int e = 0; e < EH; ++e)
                    z[e] = mk<C>(src_of(v[row_pair_idx<N>(e, 0)]), src_of(v[row_pair_idx<N>(e, 1)]));
            } else {
                // stage the real source in smem (as R[N] over the same buffer)
                R* rs = reinterpret_cast<R*>(sm);
                acc.sync();
#pragma unroll
                for (int e = 0; e < E; ++e) rs[in_pos<N, E, 0>(e, t)] = src_of(v[e]);
                acc.sync();
#pragma unroll
                for (int e = 0; e < EH; ++e) z[e] = reinterpret_cast<const C*>(rs)[in_pos<M, EH, 0>(e, t)];
            }
            fft_pencil<M, EH, -1>(z, acc, t, tw_src<false>(tb.M, tb.M));
            acc.sync();
#pragma unroll
            for (int e = 0; e < EH; ++e) acc(out_pos<M, EH>(e, t)) = z[e];
            acc.sync();
            r2c_post_store<N, R>(acc, t, a.vh + row * M, tb.Nn);
        }
    }
}

enum XR2CSrc { XR_DENSITY = 0, XR_REAL = 1 };

// r2c along x of a real source: the density pref(|psi|^2 - rho_mean) of psi
// (XR_DENSITY) or a real array Vin (XR_REAL), into the packed vh rows.
template <int N, typename R, int SRC>
__global__ void __launch_bounds__(256, 3) k_x_r2c(XArgs<R> a) {
    using C = cx_t<R>;
    constexpr int E = qx_row_efull(N);
    constexpr int M = N / 2;
    constexpr int EH = E / 2;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    XTabs<C> tb;
    C* sm = x_setup<N, R>(a, smem_raw, tb);
    const int t = threadIdx.x;
    RowAcc<C> acc{sm, warp_lanes_mask()};
    const R pr = (R)a.pref, rm = (R)a.rho_mean;
    for (long row = x_row0(); row < a.rows; row += x_row_step()) {
        acc.sync();
        C z[EH];
#pragma unroll
        for (int e = 0; e < EH; ++e) {
            const int q = in_pos<M, EH, 0>(e, t);
            if constexpr (SRC == XR_DENSITY) {
                C p0, p1;
                load_pair(a.in + row * N, q, p0, p1);
                z[e] = mk<C>(pr * (p0.x * p0.x + p0.y * p0.y - rm), pr * (p1.x * p1.x + p1.y * p1.y - rm));
            } else {
                z[e] = reinterpret_cast<const C*>(a.Vin + row * N)[q];
            }
        }
        fft_pencil<M, EH, -1>(z, acc, t, tw_src<false>(tb.M, tb.M));
        acc.sync();
#pragma unroll
        for (int e = 0; e < EH; ++e) acc(out_pos<M, EH>(e, t)) = z[e];
        acc.sync();
        r2c_post_store<N, R>(acc, t, a.vh + row * M, tb.Nn);
    }
}

enum XC2RFlags {
    XC_WRITE_V = 1,    // store the potential row
    XC_KICK = 2,       // kick psi (real space) by the potential
    XC_WRITE_PSI = 4,  // store the kicked psi in real space
    XC_FWD = 8,        // forward x FFT of the kicked psi -> out
};

// staging buffer of a kicking c2r row pass (FP32): next row's vh (N/2) and psi (N)
template <int N, typename R, int FLAGS> __host__ __device__ constexpr int x_c2r_stage_elems() {
    return (sizeof(R) == 4 && (FLAGS & 2)) ? N / 2 + N : 0;
}

// c2r along x of the packed vh rows -> V (unnormalised, FFTW convention);
// then optionally kick psi by V (dt), store psi, or forward-transform it.
// FP32 kicking passes are software-pipelined: after its kick, a warp copies
// its next row's vh and psi into a per-warp staging buffer with cp.async, so
// they arrive while the forward transform and stores of the current row run.
template <int N, typename R, int FLAGS>
__global__ void __launch_bounds__(256, 2) k_x_c2r(XArgs<R> a) {
    using C = cx_t<R>;
    constexpr int E = qx_row_efull(N);
    constexpr int M = N / 2;
    constexpr int EH = E / 2;
    constexpr int T = qx_row_threads(N);
    constexpr int SE = x_c2r_stage_elems<N, R, FLAGS>();
    constexpr bool STAGE = SE > 0;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    XTabs<C> tb;
    C* sm = x_setup<N, R>(a, smem_raw, tb);
    const int t = threadIdx.x;
    RowAcc<C> acc{sm, warp_lanes_mask()};
    C* stg = x_stage_ptr<N>(sm, SE);
    auto prefetch = [&](long r) {
        if constexpr (STAGE) {
            const char* gv = reinterpret_cast<const char*>(a.vh + r * M);
            const char* gp = reinterpret_cast<const char*>(a.in + r * N);
            char* sv = reinterpret_cast<char*>(stg);
            char* sp = reinterpret_cast<char*>(stg + M);
            for (int i = t; i < (int)(M * sizeof(C) / 16); i += T) cp_async16(sv + 16 * i, gv + 16 * i);
            for (int i = t; i < (int)(N * sizeof(C) / 16); i += T) cp_async16(sp + 16 * i, gp + 16 * i);
            cp_async_commit();
        }
    };
    if (x_row0() < a.rows) prefetch(x_row0());
    for (long row = x_row0(); row < a.rows; row += x_row_step()) {
        acc.sync();
        if constexpr (STAGE) {
            cp_async_wait_all();
            acc.sync();
        } else {
            const C* hrow = a.vh + row * M;
#pragma unroll
            for (int i = 0; i < M / T; ++i) acc(t + i * T) = hrow[t + i * T];
            acc.sync();
        }
        // the vh row: staged copy (FP32 kicking passes) or the row buffer
        auto hv = [&](int k) -> C { return STAGE ? stg[k] : acc(k); };
        C z[EH];
#pragma unroll
        for (int e = 0; e < EH; ++e) {
            const int k = out_pos<M, EH>(e, t);
            const C X = hv(k);
            if (k == 0) {
                // X[0] = Re col0, X[N/2] = Im col0
                z[e] = mk<C>(X.x + X.y, X.x - X.y);
            } else {
                const C B = cconj(hv(M - k));
                const C s = cadd(X, B), d = csub(X, B);
                const C w = cconj(tb.Nn[k]);  // W_N^{-k}
                const C wd = cmul(w, d);
                z[e] = mk<C>(s.x - wd.y, s.y + wd.x);  // s + i*wd
            }
        }
        ifft_pencil_rev<M, EH>(z, acc, t, tw_src<false>(tb.M, tb.M));
        // z at in_pos<M, EH, 0> q holds (V[2q], V[2q+1])
        if constexpr (FLAGS & XC_WRITE_V) {
            C* vrow = reinterpret_cast<C*>(a.Vout + row * N);
#pragma unroll
            for (int e = 0; e < EH; ++e) vrow[in_pos<M, EH, 0>(e, t)] = z[e];
        }
        if constexpr (FLAGS & XC_KICK) {
            constexpr bool PAIRED = row_paired<N>();
            C ps[E];  // kicked psi: position 2q+h in ps[row_pair_idx<N>(e, h)]
#pragma unroll
            for (int e = 0; e < EH; ++e) {
                C p0, p1;
                load_pair(STAGE ? stg + M : a.in + row * N, in_pos<M, EH, 0>(e, t), p0, p1);
                ps[row_pair_idx<N>(e, 0)] = kick1<R>(p0, z[e].x, a.dt);
                ps[row_pair_idx<N>(e, 1)] = kick1<R>(p1, z[e].y, a.dt);
            }
            if constexpr (STAGE) {
                // every lane is done with the staged row: fetch the next one
                acc.sync();
                const long nrow = row + x_row_step();
                if (nrow < a.rows) prefetch(nrow);
            }
            if constexpr (FLAGS & XC_WRITE_PSI) {
#pragma unroll
                for (int e = 0; e < EH; ++e) {
                    store_pair(a.out + row * N, in_pos<M, EH, 0>(e, t), ps[row_pair_idx<N>(e, 0)],
                               ps[row_pair_idx<N>(e, 1)]);
                }
            }
            if constexpr (FLAGS & XC_FWD) {
                C v[E];
                if constexpr (PAIRED) {
                    // already in the paired stage-0 input order
#pragma unroll
                    for (int e = 0; e < E; ++e) v[e] = ps[e];
                } else {
                    acc.sync();
#pragma unroll
                    for (int e = 0; e < EH; ++e) {
                        const int q = in_pos<M, EH, 0>(e, t);
                        acc(2 * q) = ps[2 * e];
                        acc(2 * q + 1) = ps[2 * e + 1];
                    }
                    acc.sync();
#pragma unroll
                    for (int e = 0; e < E; ++e) v[e] = acc(in_pos<N, E, 0>(e, t));
                }
                fft_pencil<N, E, -1, PAIRED ? 1 : 0>(v, acc, t, tw_src<true>(tb.N, tb.N_lo));
                C* dst = a.out + row * N;
#pragma unroll
                for (int e = 0; e < E; ++e) dst[out_pos<N, E>(e, t)] = v[e];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// strided passes.  Array A of shape [outer][N][X] (y pass) or, for the last
// axis, [N][rows][X] (3D, pencil along z with rows = N y-rows) / [N][X] (2D).
// Tile: G groups x TX columns x N; blockDim = (TX, T, G), T = N / E.
// Dynamic smem: G * N * pitch C with pitch = TX (+1 if TX*sizeof(C) < 128).
// ---------------------------------------------------------------------------

__host__ __device__ constexpr int qx_col_e(int N) { return qx_lcm_radices(N) < 8 && N >= 8 ? 8 : qx_lcm_radices(N); }

template <typename R> struct SArgs {
    cx_t<R>* a;
    const cx_t<R>* tw;   // exp(-2 pi i j/N)
    const cx_t<R>* tw_lo;  // exact - tw (FP32 double-float twiddles)
    int X;               // columns of the array (N or N/2)
    int dim;
    int N;
    double phase_fac;    // drift: -dt/2 * dk^2  (phase = fac * |n|^2)
    double scale;        // drift: 1/S
    double pois_c;       // Poisson: -1/(dk^2 S) (times 1/|n|^2)
    double pois_g0;      // Poisson multiplier of the k = 0 mode
    double* partial;     // per-block reduction output (kinetic)
};

template <typename C> __device__ __forceinline__ int col_pitch(int TX) {
    return TX * (int)sizeof(C) < 128 ? TX + 1 : TX;
}

// y pass (3D): pencils along y of an [outer][N][X] array; blockIdx = (x tile, outer).
// DF: double-float twiddles (wave-function arrays of the FP32 form).
template <int N, typename R, int SIGN, bool DF>
__global__ void k_y_pass(SArgs<R> s) {
    using C = cx_t<R>;
    constexpr int E = qx_col_e(N);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int TX = blockDim.x;
    const int c = threadIdx.x, t = threadIdx.y;
    const int pitch = col_pitch<C>(TX);
    C* sm = reinterpret_cast<C*>(smem_raw) + c;
    ColAcc<C> acc{sm, pitch};
    const long base = (long)blockIdx.y * N * s.X + (long)blockIdx.x * TX + c;
    C v[E];
    if constexpr (SIGN < 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = s.a[base + (long)in_pos<N, E, 0>(e, t) * s.X];
        fft_pencil<N, E, -1>(v, acc, t, tw_src<DF>(s.tw, s.tw_lo));
#pragma unroll
        for (int e = 0; e < E; ++e) s.a[base + (long)out_pos<N, E>(e, t) * s.X] = v[e];
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = s.a[base + (long)out_pos<N, E>(e, t) * s.X];
        ifft_pencil_rev<N, E>(v, acc, t, tw_src<DF>(s.tw, s.tw_lo));
#pragma unroll
        for (int e = 0; e < E; ++e) s.a[base + (long)in_pos<N, E, 0>(e, t) * s.X] = v[e];
    }
}

enum LAOp { LA_FWD = 0, LA_INV = 1, LA_DRIFT = 2, LA_POISSON = 3, LA_KIN = 4 };

// Poisson multiplier of integer |n|^2 (src/field.cxx:250-256,279-285)
template <typename R> __device__ __forceinline__ R pois_mult(long M2, const SArgs<R>& s);
template <> __device__ __forceinline__ float pois_mult<float>(long M2, const SArgs<float>& s) {
    return M2 == 0 ? (float)s.pois_g0 : (float)s.pois_c * __frcp_rn((float)M2);
}
template <> __device__ __forceinline__ double pois_mult<double>(long M2, const SArgs<double>& s) {
    return M2 == 0 ? s.pois_g0 : s.pois_c / (double)M2;
}

// Last-axis pass.  3D: pencils along z of [N][N][X]; blockIdx = (x tile,
// y group); G = 1: y = blockIdx.y; G = 2: rows {g, N-g} (g = 0 pairs 0 with
// N/2) so the mirror -k_y of every row is in the block.  2D: pencils along y
// of [N][X]; blockIdx = (x tile).  DF as for k_y_pass.
template <int N, typename R, int OP, bool DF>
__global__ void k_la_pass(SArgs<R> s) {
    using C = cx_t<R>;
    constexpr int E = qx_col_e(N);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int TX = blockDim.x, G = blockDim.z;
    const int c = threadIdx.x, t = threadIdx.y, g = threadIdx.z;
    const int pitch = col_pitch<C>(TX);
    C* sm0 = reinterpret_cast<C*>(smem_raw);
    ColAcc<C> acc{sm0 + (long)g * N * pitch + c, pitch};
    const int x0 = blockIdx.x * TX;
    const int x = x0 + c;
    int y = 0;
    long base, pstride;
    if (s.dim == 3) {
        const int gi = blockIdx.y;
        if (G == 1) y = gi;
        else y = (g == 0) ? gi : (gi == 0 ? N / 2 : N - gi);
        base = (long)y * s.X + x;
        pstride = (long)N * s.X;
    } else {
        base = x;
        pstride = s.X;
    }
    // forward transforms load in stage-0 order and store in natural order; the
    // inverse runs the other way round
    auto load_pos = [&](int e) { return OP == LA_INV ? out_pos<N, E>(e, t) : in_pos<N, E, 0>(e, t); };
    auto store_pos = [&](int e) { return OP == LA_INV ? in_pos<N, E, 0>(e, t) : out_pos<N, E>(e, t); };
    C v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = s.a[base + (long)load_pos(e) * pstride];
    if constexpr (OP == LA_INV) {
        ifft_pencil_rev<N, E>(v, acc, t, tw_src<DF>(s.tw, s.tw_lo));
    } else {
        fft_pencil<N, E, -1>(v, acc, t, tw_src<DF>(s.tw, s.tw_lo));
    }
    if constexpr (OP == LA_FWD || OP == LA_INV) {
#pragma unroll
        for (int e = 0; e < E; ++e) s.a[base + (long)store_pos(e) * pstride] = v[e];
        return;
    }
    // |n|^2 contribution of x (and y in 3D)
    const int nx = (s.X == N) ? signed_mode(x, N) : x;  // half arrays: x < N/2
    const int ny = (s.dim == 3) ? signed_mode(y, N) : 0;
    const long mxy = (long)nx * nx + (long)ny * ny;
    if constexpr (OP == LA_KIN) {
        double acc_k = 0.0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int nz = signed_mode(out_pos<N, E>(e, t), N);
            const double m2 = (double)(mxy + (long)nz * nz);
            acc_k += m2 * ((double)v[e].x * (double)v[e].x + (double)v[e].y * (double)v[e].y);
        }
        __shared__ double red[32];
        const double tot = block_reduce<0>(acc_k, red);
        if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0)
            s.partial[blockIdx.x + (long)gridDim.x * blockIdx.y] = tot;
        return;
    }
    if constexpr (OP == LA_DRIFT) {
        // exp(-i dt/2 dk^2 |n|^2)/S = A(nx, ny) B(nz), both in FP64 (same
        // arithmetic as the TMA-fed pass, which tabulates B)
        const double2 A = cis_d(s.phase_fac * (double)mxy);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long nz = signed_mode(out_pos<N, E>(e, t), N);
            const double2 b = cis_d(s.phase_fac * (double)(nz * nz));
            const double2 w = dcmul(A, make_double2(b.x * s.scale, b.y * s.scale));
            v[e] = cmul_d(v[e], w);
        }
    }
    if constexpr (OP == LA_POISSON) {
        if (x0 == 0) {
            // stage the forward result so column 0 can read its mirror mode
            __syncthreads();
#pragma unroll
            for (int e = 0; e < E; ++e) acc(out_pos<N, E>(e, t)) = v[e];
            __syncthreads();
            if (c == 0) {
                const int gm = (s.dim == 3 && G == 2) ? ((y == 0 || y == N / 2) ? g : 1 - g) : g;
                ColAcc<C> macc{sm0 + (long)gm * N * pitch, pitch};
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int p = out_pos<N, E>(e, t);
                    const int nz = signed_mode(p, N);
                    const long mA = (long)ny * ny + (long)nz * nz;
                    const long mB = mA + (long)(N / 2) * (N / 2);
                    const R gA = pois_mult<R>(mA, s), gB = pois_mult<R>(mB, s);
                    const R al = R(0.5) * (gA + gB), be = R(0.5) * (gA - gB);
                    const C cm = cconj(macc((N - p) % N));
                    v[e] = cadd(cscale(v[e], al), cscale(cm, be));
                }
            }
        }
        if (!(x0 == 0 && c == 0)) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int nz = signed_mode(out_pos<N, E>(e, t), N);
                v[e] = cscale(v[e], pois_mult<R>(mxy + (long)nz * nz, s));
            }
        }
    }
    // the inverse transform undoes the forward stages in reverse order straight
    // from the forward output order and ends in the load order
    ifft_pencil_rev<N, E>(v, acc, t, tw_src<DF>(s.tw, s.tw_lo));
#pragma unroll
    for (int e = 0; e < E; ++e) s.a[base + (long)in_pos<N, E, 0>(e, t) * pstride] = v[e];
}

}  // namespace qx
