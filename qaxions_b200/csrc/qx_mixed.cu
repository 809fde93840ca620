// qx_mixed.cu -- mixed-size ensemble passes (sm_100a).
//
// An ensemble holds boxes of several grid sizes, one batched array per size.
// Here every pass of the loop body is ONE persistent launch over the boxes of
// all sizes: the work of a pass is a queue of units (a tile of pencils, or a
// set of rows, of one box), listed size group by size group with the
// costliest units first, and each unit executor -- 64 threads, four per block
// -- takes the next unit from a global atomic counter until the queue is
// empty.  A unit executor runs the pass's transform for whichever grid size its
// unit has (the unit code is compiled for N = 16, 32, 64, 96, 128) on a
// shared-memory buffer of its own, synchronising its two warps with a named
// barrier; the twiddle and drift-factor tables of every size are staged in
// shared memory once per block.  Units never wait for one another, so the
// launch needs no inter-block synchronisation, and the queue balances the
// sizes' uneven costs at run time.
//
// The arithmetic is that of the per-size passes (same radix plan 0 butterflies,
// double-float twiddles on the wave-function transforms in FP32, drift factor
// A(nx, ny) B(nz) in FP64 with one rounding, Poisson column 0 paired with its
// mirror row), so a box advances as it does alone.
//
// Reference operations replaced: the loop body of src/main.cxx:64-85 (drift,
// updatePotential, kick of src/field.cxx:93-346) for an ensemble of boxes
// that the reference runs one per process.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "qx_kernels.cuh"
#include "qx_mixed.hpp"

namespace qx {
namespace {

constexpr int kUnitThreads = 64;   // one unit executor: two warps
constexpr int kUnitsPerBlock = 4;  // executors per block (256 threads)

__device__ __forceinline__ void unit_sync(int bar) {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(kUnitThreads) : "memory");
}

// pencil values of a strided unit: two adjacent columns (16 bytes) in FP32,
// one column in FP64
template <typename R> using mx_val_t = typename std::conditional<sizeof(R) == 4, CPair<cx_t<R>>, cx_t<R>>::type;
template <typename R> __host__ __device__ constexpr int mx_pw() { return sizeof(R) == 4 ? 2 : 1; }
// resident blocks per SM the kernels are compiled for: FP64 units hold twice
// the register state (and their shared buffers allow one block), so one
template <typename R> __host__ __device__ constexpr int mx_min_blocks() { return sizeof(R) == 4 ? 2 : 1; }

// strided units: E values per pencil and thread, T threads per pencil, S
// pencil slots per unit, shared-memory row pitch (in 16-byte values)
template <int N> __host__ __device__ constexpr int mx_e() { return qx_col_e(N); }
template <int N> __host__ __device__ constexpr int mx_t() { return N / qx_col_e(N); }
template <int N> __host__ __device__ constexpr int mx_slots() { return kUnitThreads / mx_t<N>(); }
// Unpadded: a warp's 8-lane phase of a 16-byte access covers 8 / S positions of
// S slots each, and with S = 4 the two positions of a phase are consecutive
// Stockham positions (an odd difference), so their 64-byte rows fall in
// opposite halves of the 128-byte bank window; a padded pitch of S + 1 made
// them overlap (ncu: 33 % of shared wavefronts were conflicts).
template <int N> __host__ __device__ constexpr int mx_pitch() { return mx_slots<N>(); }
// rows of an x-pass unit
template <int N> __host__ __device__ constexpr int mx_rows() { return kUnitThreads / qx_row_threads(N); }

__host__ __device__ constexpr bool mx_is_row(int op) { return op == MX_X_INV_R2C || op == MX_X_C2R_KICK; }
__host__ __device__ constexpr bool mx_is_psi(int op) {
    return op == MX_Y_FWD_PSI || op == MX_Z_DRIFT || op == MX_Y_INV_PSI;
}
__host__ __device__ constexpr bool mx_is_y(int op) {
    return op == MX_Y_FWD_PSI || op == MX_Y_INV_PSI || op == MX_Y_FWD_VH || op == MX_Y_INV_VH;
}

// columns of a strided unit (per row: a Poisson unit holds two rows) and the
// unit tiles across the X columns of its array
template <int N, typename R> __host__ __device__ constexpr int mx_txu(int op) {
    return (op == MX_Z_POISSON ? mx_slots<N>() / 2 : mx_slots<N>()) * mx_pw<R>();
}
template <int N, typename R> __host__ __device__ constexpr int mx_tiles_x(int op) {
    return ((mx_is_psi(op) ? N : N / 2) + mx_txu<N, R>(op) - 1) / mx_txu<N, R>(op);
}
// work units of one box in pass op
template <int N, typename R> __host__ __device__ constexpr long mx_units_box(int op) {
    return mx_is_row(op) ? (long)N * N / mx_rows<N>()
           : op == MX_Z_POISSON ? (long)(N / 2) * mx_tiles_x<N, R>(op)
                                : (long)N * mx_tiles_x<N, R>(op);
}
// The same counts computed at run time from (op, N, values per slot) for the
// host's queue layout.  The host does not evaluate the templates above: nvcc
// -O3 was found to fold mx_units_box<N, double> of the wave-function passes to
// the half-spectrum count in a host loop over the passes (checked with a
// host-only probe: -O0 and -O2 give the right count).  Every kernel compares
// the host's counts with its compile-time ones and refuses to run on a
// mismatch.
inline long mx_units_rt(int op, int N, int pw) {
    const int S = kUnitThreads / (N / qx_col_e(N));
    if (op == MX_X_INV_R2C || op == MX_X_C2R_KICK) return (long)N * N / (kUnitThreads / qx_row_threads(N));
    const int txu = (op == MX_Z_POISSON ? S / 2 : S) * pw;
    const int X = (op == MX_Y_FWD_PSI || op == MX_Z_DRIFT || op == MX_Y_INV_PSI) ? N : N / 2;
    const long tiles = (X + txu - 1) / txu;
    return (op == MX_Z_POISSON ? (long)(N / 2) : (long)N) * tiles;
}
inline int mx_unit_bytes_rt(int N, int csize) {
    const int S = kUnitThreads / (N / qx_col_e(N));
    const int pitch = S;
    const int pencil = N * pitch * 16;
    const int rows = (kUnitThreads / qx_row_threads(N)) * row_smem_elems(N) * csize;
    return ((pencil > rows ? pencil : rows) + 15) & ~15;
}

// shared-memory bytes of one unit executor for grid size N
template <int N, typename R> __host__ __device__ constexpr int mx_unit_bytes() {
    const int pencil = N * mx_pitch<N>() * 16;
    const int rows = mx_rows<N>() * row_smem_elems(N) * (int)sizeof(cx_t<R>);
    return ((pencil > rows ? pencil : rows) + 15) & ~15;
}

template <typename R> struct MGroup {
    cx_t<R>* psi;
    cx_t<R>* vh;
    const cx_t<R>* twN;
    const cx_t<R>* twN_lo;
    const cx_t<R>* twM;
    const cx_t<R>* twNn;
    const double2* axy;
    int N, B;
    double pois_c, pois_g0, pref, rho_mean, dt;
    int tab_off;  // this group's twiddle tables in shared memory (complex elements)
    int bz_off;   // its B(nz) drift factors in shared memory (double2 elements)
};

template <typename R> struct MArgs {
    MGroup<R> g[kMixMaxGroups];
    long off[kMixMaxGroups + 1];  // queue index of each group's first unit (queue order)
    long ub[kMixMaxGroups];       // units of one box of each group (checked by the kernel)
    int ng;
    int tab_elems, bz_elems, unit_bytes;
    unsigned long long* ctr;
    int* err;                     // set to 2 when the host's layout disagrees with the kernel's
};

// a group's tables in shared memory: N-point twiddles (and their low parts),
// N/2-point twiddles, natural-order exp(-2 pi i k/N) (k < N/2), B(nz)/S
template <typename R> struct MTabs {
    const cx_t<R>* N;
    const cx_t<R>* N_lo;
    const cx_t<R>* M;
    const cx_t<R>* Nn;
    const double2* bz;
};

// Loads of psi / vh go through L2 only (ld.global.cg): in the one-launch step
// a unit reads data that units on other SMs wrote earlier in the same launch,
// which a stale L1 line must not shadow.
__device__ __forceinline__ float2 ld_cg(const float2* p) { return __ldcg(p); }
__device__ __forceinline__ double2 ld_cg(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ CPair<float2> ld_cg(const CPair<float2>* p) {
    const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
    return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
// elements 2q and 2q+1 of a complex row (as load_pair), through L2 only
template <typename C> __device__ __forceinline__ void ld_cg_pair(const C* row, int q, C& a, C& b) {
    if constexpr (sizeof(C) == 8) {
        const float4 v = __ldcg(reinterpret_cast<const float4*>(row) + q);
        a = mk<C>(v.x, v.y);
        b = mk<C>(v.z, v.w);
    } else {
        a = ld_cg(row + 2 * q);
        b = ld_cg(row + 2 * q + 1);
    }
}

// column of a strided unit: element p of slot c at base[p * pitch]
template <typename P> struct UnitColAcc {
    P* base;
    int pitch, bar;
    __device__ __forceinline__ P& operator()(int p) const { return base[p * pitch]; }
    __device__ __forceinline__ void sync() const { unit_sync(bar); }
};

// One strided unit: a tile of columns x N positions of one box (y passes: one
// z plane; z passes: one y row, or for the Poisson pass the rows y and -y,
// so column 0 finds its mirror mode in the unit).  Thread tu is pencil thread
// t of slot c (c fastest: a warp's loads cover whole row segments).
template <int N, typename R, int OP>
__device__ __forceinline__ void mx_pencil_unit(const MGroup<R>& G, long l, int tu, int bar, unsigned char* ubuf,
                                               const MTabs<R>& tb) {
    using C = cx_t<R>;
    using P = mx_val_t<R>;
    constexpr int PW = mx_pw<R>();
    constexpr int E = mx_e<N>(), S = mx_slots<N>(), PITCH = mx_pitch<N>();
    constexpr bool PSI = mx_is_psi(OP), YP = mx_is_y(OP), POIS = OP == MX_Z_POISSON;
    constexpr bool INV = OP == MX_Y_INV_PSI || OP == MX_Y_INV_VH;
    constexpr int X = PSI ? N : N / 2;
    constexpr int SR = POIS ? S / 2 : S;  // slots per row
    constexpr int TXU = SR * PW;
    constexpr int TILES_X = mx_tiles_x<N, R>(OP);
    const int c = tu % S, t = tu / S;
    const int half = POIS ? c / SR : 0;
    const int cc = c - half * SR;
    const int xt = (int)(l % TILES_X);
    const long rest = l / TILES_X;
    const int x = xt * TXU + cc * PW;
    const bool valid = x < X;
    int y = 0;
    long base, pstride;
    if constexpr (YP) {  // rest = z plane of the batched [B N][N][X] array
        base = rest * N * X + x;
        pstride = X;
    } else if constexpr (POIS) {  // rows g and N - g (0 pairs with N/2)
        const int gi = (int)(rest % (N / 2));
        const long b = rest / (N / 2);
        y = half == 0 ? gi : (gi == 0 ? N / 2 : N - gi);
        base = b * N * N * X + (long)y * X + x;
        pstride = (long)N * X;
    } else {
        y = (int)(rest % N);
        const long b = rest / N;
        base = b * N * N * X + (long)y * X + x;
        pstride = (long)N * X;
    }
    C* arr = PSI ? G.psi : G.vh;
    auto at = [&](int p) -> P* { return reinterpret_cast<P*>(arr + base + (long)p * pstride); };
    P* buf = reinterpret_cast<P*>(ubuf);
    UnitColAcc<P> acc{buf + c, PITCH, bar};
    const auto tw = tw_src<PSI>(tb.N, tb.N_lo);
    P v[E];
    if constexpr (INV) {
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = valid ? ld_cg(at(out_pos<N, E>(e, t))) : P{};
        ifft_pencil_rev<N, E>(v, acc, t, tw);
        if (valid) {
#pragma unroll
            for (int e = 0; e < E; ++e) *at(in_pos<N, E, 0>(e, t)) = v[e];
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = valid ? ld_cg(at(in_pos<N, E, 0>(e, t))) : P{};
    fft_pencil<N, E, -1>(v, acc, t, tw);
    if constexpr (YP) {
        if (valid) {
#pragma unroll
            for (int e = 0; e < E; ++e) *at(out_pos<N, E>(e, t)) = v[e];
        }
        return;
    }
    if constexpr (OP == MX_Z_DRIFT) {
        // exp(-i dt/2 dk^2 |n|^2)/S = A(nx, ny) B(nz), multiplied in FP64, one rounding
#pragma unroll
        for (int h = 0; h < PW; ++h) {
            const double2 A = valid ? G.axy[(long)y * N + x + h] : make_double2(0.0, 0.0);
#pragma unroll
            for (int e = 0; e < E; ++e) pen(v[e], h) = cmul_d(pen(v[e], h), dcmul(A, tb.bz[out_pos<N, E>(e, t)]));
        }
    } else {
        SArgs<R> sa;
        sa.pois_c = G.pois_c;
        sa.pois_g0 = G.pois_g0;
        const long ny = signed_mode(y, N);
        const bool col0 = xt == 0 && cc == 0;  // pencil 0 of this slot is column 0 (kx = 0 and N/2)
        if (xt == 0) {
            // C'(k) = a C(k) + b conj C(-k): stage the forward result, read the mirror row's column 0
            acc.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) acc(out_pos<N, E>(e, t)) = v[e];
            acc.sync();
            if (col0) {
                const int gm = (y == 0 || y == N / 2) ? half : 1 - half;
                const P* mb = buf + gm * SR;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int p = out_pos<N, E>(e, t);
                    const long nz = signed_mode(p, N);
                    const long mA = ny * ny + nz * nz;
                    const long mB = mA + (long)(N / 2) * (N / 2);
                    const R gA = pois_mult<R>(mA, sa), gB = pois_mult<R>(mB, sa);
                    const R al = R(0.5) * (gA + gB), be = R(0.5) * (gA - gB);
                    P mv = mb[((N - p) % N) * PITCH];
                    const C cm = cconj(pen(mv, 0));
                    pen(v[e], 0) = cadd(cscale(pen(v[e], 0), al), cscale(cm, be));
                }
            }
        }
#pragma unroll
        for (int h = 0; h < PW; ++h) {
            if (h == 0 && col0) continue;
            const long nx = x + h;
            const long mxy = nx * nx + ny * ny;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const long nz = signed_mode(out_pos<N, E>(e, t), N);
                pen(v[e], h) = cscale(pen(v[e], h), pois_mult<R>(mxy + nz * nz, sa));
            }
        }
    }
    ifft_pencil_rev<N, E>(v, acc, t, tw);
    if (valid) {
#pragma unroll
        for (int e = 0; e < E; ++e) *at(in_pos<N, E, 0>(e, t)) = v[e];
    }
}

// One row of the x inverse pass: inverse x transform of psi^_x -> psi, the
// density source pref(|psi|^2 - rho_mean) and its r2c x transform -> vh.
template <int N, typename R>
__device__ __forceinline__ void mx_x_inv_row(const MGroup<R>& G, long row, int t, cx_t<R>* rb, const MTabs<R>& tb) {
    using C = cx_t<R>;
    constexpr int E = qx_row_efull(N), M = N / 2, EH = E / 2;
    constexpr bool PAIRED = row_paired<N>();
    RowAcc<C> acc{rb, 0xffffffffu};
    acc.sync();
    C* prow = G.psi + row * N;
    C v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = ld_cg(prow + out_pos<N, E>(e, t));
    ifft_pencil_rev<N, E, PAIRED ? 1 : 0>(v, acc, t, tw_src<true>(tb.N, tb.N_lo));
    if constexpr (PAIRED) {
#pragma unroll
        for (int e = 0; e < EH; ++e)
            store_pair(prow, in_pos<M, EH, 0>(e, t), v[row_pair_idx<N>(e, 0)], v[row_pair_idx<N>(e, 1)]);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) prow[in_pos<N, E, 0>(e, t)] = v[e];
    }
    const R pr = (R)G.pref, rm = (R)G.rho_mean;
    auto src_of = [&](const C& u) { return pr * (u.x * u.x + u.y * u.y - rm); };
    C z[EH];
    if constexpr (PAIRED) {
#pragma unroll
        for (int e = 0; e < EH; ++e) z[e] = mk<C>(src_of(v[row_pair_idx<N>(e, 0)]), src_of(v[row_pair_idx<N>(e, 1)]));
    } else {
        R* rs = reinterpret_cast<R*>(rb);
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
    r2c_post_store<N, R>(acc, t, G.vh + row * M, tb.Nn);
}

// One row of the c2r pass: c2r x of the packed vh row -> V, kick psi by V,
// forward x transform of the kicked psi -> psi^_x.
template <int N, typename R>
__device__ __forceinline__ void mx_x_c2r_row(const MGroup<R>& G, long row, int t, cx_t<R>* rb, const MTabs<R>& tb) {
    using C = cx_t<R>;
    constexpr int E = qx_row_efull(N), M = N / 2, EH = E / 2, T = qx_row_threads(N);
    constexpr bool PAIRED = row_paired<N>();
    RowAcc<C> acc{rb, 0xffffffffu};
    acc.sync();
    const C* hrow = G.vh + row * M;
#pragma unroll
    for (int i = 0; i < M / T; ++i) acc(t + i * T) = ld_cg(hrow + t + i * T);
    acc.sync();
    C z[EH];
#pragma unroll
    for (int e = 0; e < EH; ++e) {
        const int k = out_pos<M, EH>(e, t);
        const C Xk = acc(k);
        if (k == 0) {
            z[e] = mk<C>(Xk.x + Xk.y, Xk.x - Xk.y);  // X[0] = Re col0, X[N/2] = Im col0
        } else {
            const C Bk = cconj(acc(M - k));
            const C s = cadd(Xk, Bk), d = csub(Xk, Bk);
            const C w = cconj(tb.Nn[k]);
            const C wd = cmul(w, d);
            z[e] = mk<C>(s.x - wd.y, s.y + wd.x);
        }
    }
    ifft_pencil_rev<M, EH>(z, acc, t, tw_src<false>(tb.M, tb.M));
    C* prow = G.psi + row * N;
    C ps[E];
#pragma unroll
    for (int e = 0; e < EH; ++e) {
        C p0, p1;
        ld_cg_pair(prow, in_pos<M, EH, 0>(e, t), p0, p1);
        ps[row_pair_idx<N>(e, 0)] = kick1<R>(p0, z[e].x, G.dt);
        ps[row_pair_idx<N>(e, 1)] = kick1<R>(p1, z[e].y, G.dt);
    }
    C v[E];
    if constexpr (PAIRED) {
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
#pragma unroll
    for (int e = 0; e < E; ++e) prow[out_pos<N, E>(e, t)] = v[e];
}

template <int N, typename R, int OP>
__device__ __forceinline__ void mx_unit(const MGroup<R>& G, long l, int tu, int bar, unsigned char* ubuf,
                                        const MTabs<R>& tb) {
    if constexpr (mx_is_row(OP)) {
        constexpr int T = qx_row_threads(N);
        const int r = tu / T, t = tu % T;
        const long row = l * mx_rows<N>() + r;
        cx_t<R>* rb = reinterpret_cast<cx_t<R>*>(ubuf) + r * row_smem_elems(N);
        if constexpr (OP == MX_X_INV_R2C) mx_x_inv_row<N, R>(G, row, t, rb, tb);
        else mx_x_c2r_row<N, R>(G, row, t, rb, tb);
    } else {
        mx_pencil_unit<N, R, OP>(G, l, tu, bar, ubuf, tb);
    }
}

template <typename R, int OP>
__device__ __forceinline__ void mx_dispatch(const MGroup<R>& G, long l, int tu, int bar, unsigned char* ubuf,
                                            const MTabs<R>& tb) {
    switch (G.N) {
        case 16: mx_unit<16, R, OP>(G, l, tu, bar, ubuf, tb); break;
        case 32: mx_unit<32, R, OP>(G, l, tu, bar, ubuf, tb); break;
        case 64: mx_unit<64, R, OP>(G, l, tu, bar, ubuf, tb); break;
        case 96: mx_unit<96, R, OP>(G, l, tu, bar, ubuf, tb); break;
        case 128: mx_unit<128, R, OP>(G, l, tu, bar, ubuf, tb); break;
        default: break;
    }
}

// stage every group's twiddle tables (and, if `bz`, its B(nz) drift factors)
// in shared memory; returns after a block barrier
template <typename R>
__device__ __forceinline__ void mx_stage_tables(const MGroup<R>* gs, int ng, cx_t<R>* tabs, double2* bzs, bool bz) {
    for (int g = 0; g < ng; ++g) {
        const MGroup<R>& G = gs[g];
        const int n = G.N;
        cx_t<R>* t0 = tabs + G.tab_off;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            t0[i] = G.twN[i];
            t0[n + i] = G.twN_lo[i];
            if (bz) bzs[G.bz_off + i] = G.axy[(long)n * n + i];
        }
        for (int i = threadIdx.x; i < n / 2; i += blockDim.x) {
            t0[2 * n + i] = G.twM[i];
            t0[2 * n + n / 2 + i] = G.twNn[i];
        }
    }
    __syncthreads();
}

// the kernel's own (compile-time) units per box and unit bytes of grid size n
template <typename R> __device__ long mx_ub_dev(int op, int n) {
    switch (n) {
        case 16: return mx_units_box<16, R>(op);
        case 32: return mx_units_box<32, R>(op);
        case 64: return mx_units_box<64, R>(op);
        case 96: return mx_units_box<96, R>(op);
        case 128: return mx_units_box<128, R>(op);
        default: return -1;
    }
}
template <typename R> __device__ int mx_bytes_dev(int n) {
    switch (n) {
        case 16: return mx_unit_bytes<16, R>();
        case 32: return mx_unit_bytes<32, R>();
        case 64: return mx_unit_bytes<64, R>();
        case 96: return mx_unit_bytes<96, R>();
        case 128: return mx_unit_bytes<128, R>();
        default: return 1 << 30;
    }
}

// Persistent launch of pass OP over every group: each 64-thread unit executor
// takes units from the queue (*a.ctr, zero at the start) until it is empty.
template <typename R, int OP>
__global__ void __launch_bounds__(kUnitThreads * kUnitsPerBlock, mx_min_blocks<R>()) k_mixed(const __grid_constant__ MArgs<R> a) {
    using C = cx_t<R>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ long long s_idx[kUnitsPerBlock];
    C* tabs = reinterpret_cast<C*>(smem_raw);
    double2* bzs = reinterpret_cast<double2*>(smem_raw + (((size_t)a.tab_elems * sizeof(C) + 15) & ~(size_t)15));
    unsigned char* units = reinterpret_cast<unsigned char*>(bzs + a.bz_elems);
    mx_stage_tables<R>(a.g, a.ng, tabs, bzs, OP == MX_Z_DRIFT);
    __shared__ int s_bad;
    if (threadIdx.x == 0) {
        int bad = 0;
        for (int g = 0; g < a.ng; ++g)
            bad |= a.ub[g] != mx_ub_dev<R>(OP, a.g[g].N) || a.unit_bytes < mx_bytes_dev<R>(a.g[g].N);
        s_bad = bad;
        if (bad) atomicExch(a.err, 2);
    }
    __syncthreads();
    if (s_bad) return;
    const int u = threadIdx.x / kUnitThreads, tu = threadIdx.x % kUnitThreads, bar = 1 + u;
    unsigned char* ubuf = units + (size_t)u * a.unit_bytes;
    const long total = a.off[a.ng];
    for (;;) {
        unit_sync(bar);  // every thread has read the previous unit index
        if (tu == 0) s_idx[u] = (long long)atomicAdd(a.ctr, 1ULL);
        unit_sync(bar);
        const long idx = (long)s_idx[u];
        if (idx >= total) break;
        int g = 0;
        while (g + 1 < a.ng && idx >= a.off[g + 1]) ++g;
        const MGroup<R>& G = a.g[g];
        const C* t0 = tabs + G.tab_off;
        const MTabs<R> tb{t0, t0 + G.N, t0 + 2 * G.N, t0 + 2 * G.N + G.N / 2, bzs + G.bz_off};
        mx_dispatch<R, OP>(G, idx - a.off[g], tu, bar, ubuf, tb);
    }
}

// ---------------------------------------------------------------------------
// The whole loop body as ONE persistent launch.  The queue lists the units of
// pass 0 (every box), then pass 1, ... pass 7.  A unit of pass p > 0 of box b
// starts once every unit of pass p - 1 of box b has finished (per-box
// completion counters: barrier, then one thread's release add after the
// unit's stores; acquire before its loads), so the passes of different boxes
// overlap and no pass ends in a
// device-wide drain.  A unit only waits for units earlier in the queue, which
// executors that are running have claimed and finish without waiting for any
// later unit, so the launch always completes; every wait is bounded (~1 s of
// SM clock) and a time-out sets *err (the host reports it) instead of hanging.
// ---------------------------------------------------------------------------

// A segment of the queue: units q0, q0 + 1, ... are units l0, l0 + 1, ... of
// pass `op` of group `g` (box-major within the group); segments are sorted by q0.
struct MSeg {
    int q0, l0, op, g;
};
constexpr int kMixMaxSeg = 512;  // 8 KB of the kernel's parameters

template <typename R> struct MStepArgs {
    MGroup<R> g[kMixMaxGroups];
    long ub[MX_NOPS][kMixMaxGroups];  // units of one box of group k in pass op
    int box0[kMixMaxGroups];          // counter index of group k's first box
    int ng, nbox, nseg, total;
    int tab_elems, bz_elems, unit_bytes;
    unsigned long long* ctr;  // queue counter (zero at the start)
    unsigned* done;           // [MX_NOPS][nbox] finished units (zero at the start)
    int* err;
    MSeg seg[kMixMaxSeg];
};

__device__ __forceinline__ unsigned mx_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void mx_red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename R>
__global__ void __launch_bounds__(kUnitThreads * kUnitsPerBlock, mx_min_blocks<R>())
    k_mixed_step(const __grid_constant__ MStepArgs<R> a) {
    using C = cx_t<R>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ long long s_idx[kUnitsPerBlock];
    C* tabs = reinterpret_cast<C*>(smem_raw);
    double2* bzs = reinterpret_cast<double2*>(smem_raw + (((size_t)a.tab_elems * sizeof(C) + 15) & ~(size_t)15));
    unsigned char* units = reinterpret_cast<unsigned char*>(bzs + a.bz_elems);
    mx_stage_tables<R>(a.g, a.ng, tabs, bzs, true);
    __shared__ int s_bad;
    if (threadIdx.x == 0) {
        int bad = 0;
        for (int g = 0; g < a.ng; ++g) {
            bad |= a.unit_bytes < mx_bytes_dev<R>(a.g[g].N);
            for (int op = 0; op < MX_NOPS; ++op) bad |= a.ub[op][g] != mx_ub_dev<R>(op, a.g[g].N);
        }
        s_bad = bad;
        if (bad) atomicExch(a.err, 2);
    }
    __syncthreads();
    if (s_bad) return;
    const int u = threadIdx.x / kUnitThreads, tu = threadIdx.x % kUnitThreads, bar = 1 + u;
    unsigned char* ubuf = units + (size_t)u * a.unit_bytes;
    const long total = a.total;
    for (;;) {
        unit_sync(bar);
        if (tu == 0) s_idx[u] = (long long)atomicAdd(a.ctr, 1ULL);
        unit_sync(bar);
        const long idx = (long)s_idx[u];
        if (idx >= total) break;
        int lo = 0, hi = a.nseg - 1;  // the last segment starting at or before idx
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.seg[mid].q0 <= idx) lo = mid;
            else hi = mid - 1;
        }
        const int op = a.seg[lo].op, g = a.seg[lo].g;
        const long l = a.seg[lo].l0 + (idx - a.seg[lo].q0);
        const long box = a.box0[g] + l / a.ub[op][g];
        if (op > 0) {
            if (tu == 0) {
                const unsigned* c = a.done + (long)(op - 1) * a.nbox + box;
                const unsigned target = (unsigned)a.ub[op - 1][g];
                const long long t0 = clock64();
                while (mx_ld_acquire(c) < target) {
                    if (clock64() - t0 > (1LL << 31)) {
                        atomicExch(a.err, 1);
                        break;
                    }
                    __nanosleep(64);
                }
            }
            unit_sync(bar);
        }
        const MGroup<R>& G = a.g[g];
        const C* t0 = tabs + G.tab_off;
        const MTabs<R> tb{t0, t0 + G.N, t0 + 2 * G.N, t0 + 2 * G.N + G.N / 2, bzs + G.bz_off};
        switch (op) {
            case MX_Y_FWD_PSI: mx_dispatch<R, MX_Y_FWD_PSI>(G, l, tu, bar, ubuf, tb); break;
            case MX_Z_DRIFT: mx_dispatch<R, MX_Z_DRIFT>(G, l, tu, bar, ubuf, tb); break;
            case MX_Y_INV_PSI: mx_dispatch<R, MX_Y_INV_PSI>(G, l, tu, bar, ubuf, tb); break;
            case MX_X_INV_R2C: mx_dispatch<R, MX_X_INV_R2C>(G, l, tu, bar, ubuf, tb); break;
            case MX_Y_FWD_VH: mx_dispatch<R, MX_Y_FWD_VH>(G, l, tu, bar, ubuf, tb); break;
            case MX_Z_POISSON: mx_dispatch<R, MX_Z_POISSON>(G, l, tu, bar, ubuf, tb); break;
            case MX_Y_INV_VH: mx_dispatch<R, MX_Y_INV_VH>(G, l, tu, bar, ubuf, tb); break;
            default: mx_dispatch<R, MX_X_C2R_KICK>(G, l, tu, bar, ubuf, tb); break;
        }
        // publish: the unit's stores are ordered before thread 0's release add
        // by the barrier, and a release is cumulative, so a unit that acquires
        // the counter sees them (a separate fence before the add measured 5 %
        // slower: 1.827 against 1.743 ms per C4 step)
        unit_sync(bar);
        if (tu == 0) mx_red_release_add(a.done + (long)op * a.nbox + box, 1u);
    }
}

#define MX_FOR_N(N, ...)                                               \
    switch (N) {                                                        \
        case 16: { constexpr int NN = 16; __VA_ARGS__; break; }         \
        case 32: { constexpr int NN = 32; __VA_ARGS__; break; }         \
        case 64: { constexpr int NN = 64; __VA_ARGS__; break; }         \
        case 96: { constexpr int NN = 96; __VA_ARGS__; break; }         \
        case 128: { constexpr int NN = 128; __VA_ARGS__; break; }       \
        default: throw std::invalid_argument("mixed-size passes: unsupported grid size N=" + std::to_string(N)); \
    }

int sm_count_dev() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

// groups in queue order (costliest units of pass `cost_op` first) with their
// shared-memory table offsets; returns the order and the table / unit sizes
template <typename R>
std::vector<int> fill_groups(const MixDesc* d, int ng, int cost_op, MGroup<R>* out, int& tab, int& bz, int& ub) {
    using C = cx_t<R>;
    if (ng < 1 || ng > kMixMaxGroups) throw std::invalid_argument("mixed-size passes take 1 to 4 groups");
    std::vector<int> order(ng);
    std::vector<double> cost(ng);
    for (int g = 0; g < ng; ++g) {
        order[g] = g;
        MX_FOR_N(d[g].N, {
            const double units = (double)mx_units_rt(cost_op, NN, mx_pw<R>());
            const double sites = (double)NN * NN * (mx_is_psi(cost_op) || mx_is_row(cost_op) ? NN : NN / 2);
            cost[g] = sites / units * std::log2((double)NN);
        });
    }
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return cost[i] > cost[j]; });
    tab = bz = ub = 0;
    for (int k = 0; k < ng; ++k) {
        const MixDesc& s = d[order[k]];
        if (!s.psi || !s.vh || !s.twN || !s.twN_lo || !s.twM || !s.twNn || !s.axy || s.B < 1)
            throw std::invalid_argument("mixed-size passes: incomplete group description");
        MGroup<R>& G = out[k];
        G.psi = static_cast<C*>(s.psi);
        G.vh = static_cast<C*>(s.vh);
        G.twN = static_cast<const C*>(s.twN);
        G.twN_lo = static_cast<const C*>(s.twN_lo);
        G.twM = static_cast<const C*>(s.twM);
        G.twNn = static_cast<const C*>(s.twNn);
        G.axy = s.axy;
        G.N = s.N;
        G.B = s.B;
        G.pois_c = s.pois_c;
        G.pois_g0 = s.pois_g0;
        G.pref = s.pref;
        G.rho_mean = s.rho_mean;
        G.dt = s.dt_kick;
        G.tab_off = tab;
        G.bz_off = bz;
        tab += 3 * s.N;
        bz += s.N;
        MX_FOR_N(s.N, { ub = std::max(ub, mx_unit_bytes_rt(NN, (int)sizeof(C))); });
    }
    return order;
}

template <typename R> size_t mx_smem(int tab, int bz, int ub) {
    return (((size_t)tab * sizeof(cx_t<R>) + 15) & ~(size_t)15) + (size_t)bz * sizeof(double2) +
           (size_t)kUnitsPerBlock * ub;
}

// set the kernel's shared-memory limit; returns the persistent grid size
template <typename K> long mx_grid(K kern, size_t smem, long units, bool attr_only) {
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) throw std::runtime_error(std::string("mixed-size smem attribute: ") + cudaGetErrorString(e));
    }
    if (attr_only) return 0;
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, kUnitThreads * kUnitsPerBlock, smem) != cudaSuccess ||
        bps < 1)
        bps = 1;
    long grid = (long)sm_count_dev() * bps;
    const long need = (units + kUnitsPerBlock - 1) / kUnitsPerBlock;
    if (grid > need) grid = need;
    return grid < 1 ? 1 : grid;
}

template <typename R, int OP>
void launch_op(const MixDesc* d, int ng, unsigned long long* ctr, int* err, cudaStream_t st, bool attr_only = false) {
    MArgs<R> a{};
    int tab, bz, ub;
    const auto order = fill_groups<R>(d, ng, OP, a.g, tab, bz, ub);
    a.ng = ng;
    a.ctr = ctr;
    a.err = err;
    long off = 0;
    for (int k = 0; k < ng; ++k) {
        a.off[k] = off;
        a.ub[k] = mx_units_rt(OP, a.g[k].N, mx_pw<R>());
        off += a.ub[k] * a.g[k].B;
    }
    a.off[ng] = off;
    a.tab_elems = tab;
    a.bz_elems = bz;
    a.unit_bytes = ub;
    const size_t smem = mx_smem<R>(tab, bz, ub);
    auto kern = k_mixed<R, OP>;
    const long grid = mx_grid(kern, smem, off, attr_only);
    if (attr_only) return;
    kern<<<(unsigned)grid, kUnitThreads * kUnitsPerBlock, smem, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string("mixed-size launch: ") + cudaGetErrorString(e));
}

template <typename R>
void launch_step(const MixDesc* d, int ng, unsigned long long* ctr, unsigned* done, int* err, long window_bytes,
                 cudaStream_t st, bool attr_only) {
    using C = cx_t<R>;
    MStepArgs<R> a{};
    int tab, bz, ub;
    (void)fill_groups<R>(d, ng, MX_Z_DRIFT, a.g, tab, bz, ub);
    a.ng = ng;
    a.ctr = ctr;
    a.done = done;
    a.err = err;
    int nbox = 0;
    for (int k = 0; k < ng; ++k) {
        a.box0[k] = nbox;
        nbox += a.g[k].B;
        for (int op = 0; op < MX_NOPS; ++op) a.ub[op][k] = mx_units_rt(op, a.g[k].N, mx_pw<R>());
    }
    a.nbox = nbox;
    // Windows of boxes (queue order of the groups, box by box) whose psi and
    // half spectrum fit in `window_bytes`: the queue runs all passes of one
    // window (pass by pass, box-major within a pass) before the next, so a
    // box's arrays can stay in L2 from one pass to the next.
    long q = 0;
    int nseg = 0;
    int k0 = 0, b0 = 0;  // first box of the window: group k0, box b0
    while (k0 < ng) {
        int k1 = k0, b1 = b0;  // one past the window's last box
        long bytes = 0;
        while (k1 < ng) {
            const long n3 = (long)a.g[k1].N * a.g[k1].N * a.g[k1].N;
            const long box_bytes = n3 * (long)sizeof(C) * 3 / 2;
            if (bytes > 0 && bytes + box_bytes > window_bytes) break;
            bytes += box_bytes;
            if (++b1 == a.g[k1].B) {
                ++k1;
                b1 = 0;
            }
        }
        for (int op = 0; op < MX_NOPS; ++op)
            for (int k = k0; k <= k1 && k < ng; ++k) {
                const int first = k == k0 ? b0 : 0;
                const int last = k == k1 ? b1 : a.g[k].B;  // one past
                if (last <= first) continue;
                if (nseg == kMixMaxSeg) throw std::invalid_argument("mixed-size step: too many queue segments");
                MSeg& sg = a.seg[nseg++];
                sg.q0 = (int)q;
                sg.l0 = (int)(first * a.ub[op][k]);
                sg.op = op;
                sg.g = k;
                q += (long)(last - first) * a.ub[op][k];
            }
        k0 = k1;
        b0 = b1;
    }
    if (q >= (1L << 31)) throw std::invalid_argument("mixed-size step: queue too long");
    a.nseg = nseg;
    a.total = (int)q;
    a.tab_elems = tab;
    a.bz_elems = bz;
    a.unit_bytes = ub;
    const size_t smem = mx_smem<R>(tab, bz, ub);
    auto kern = k_mixed_step<R>;
    const long grid = mx_grid(kern, smem, q, attr_only);
    if (attr_only) return;
    kern<<<(unsigned)grid, kUnitThreads * kUnitsPerBlock, smem, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string("mixed-size step launch: ") + cudaGetErrorString(e));
}

}  // namespace

template <typename R> bool Mixed<R>::supports(int N) {
    return N == 16 || N == 32 || N == 64 || N == 96 || N == 128;
}

template <typename R> long Mixed<R>::units(int op, const MixDesc& d) {
    if (!supports(d.N)) throw std::invalid_argument("mixed-size passes: unsupported grid size N=" + std::to_string(d.N));
    return mx_units_rt(op, d.N, mx_pw<R>()) * d.B;
}

template <typename R>
void Mixed<R>::launch(int op, const MixDesc* d, int ng, unsigned long long* ctr, int* err, cudaStream_t st) {
    switch (op) {
        case MX_Y_FWD_PSI: launch_op<R, MX_Y_FWD_PSI>(d, ng, ctr, err, st); break;
        case MX_Z_DRIFT: launch_op<R, MX_Z_DRIFT>(d, ng, ctr, err, st); break;
        case MX_Y_INV_PSI: launch_op<R, MX_Y_INV_PSI>(d, ng, ctr, err, st); break;
        case MX_X_INV_R2C: launch_op<R, MX_X_INV_R2C>(d, ng, ctr, err, st); break;
        case MX_Y_FWD_VH: launch_op<R, MX_Y_FWD_VH>(d, ng, ctr, err, st); break;
        case MX_Z_POISSON: launch_op<R, MX_Z_POISSON>(d, ng, ctr, err, st); break;
        case MX_Y_INV_VH: launch_op<R, MX_Y_INV_VH>(d, ng, ctr, err, st); break;
        case MX_X_C2R_KICK: launch_op<R, MX_X_C2R_KICK>(d, ng, ctr, err, st); break;
        default: throw std::invalid_argument("mixed-size passes: unknown pass");
    }
}

template <typename R>
void Mixed<R>::launch_step(const MixDesc* d, int ng, unsigned long long* ctr, unsigned* done, int* err,
                           long window_bytes, cudaStream_t st) {
    qx::launch_step<R>(d, ng, ctr, done, err, window_bytes, st, false);
}

template <typename R> void Mixed<R>::prepare(const MixDesc* d, int ng) {
    qx::launch_step<R>(d, ng, nullptr, nullptr, nullptr, 1L << 40, nullptr, true);
    launch_op<R, MX_Y_FWD_PSI>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_Z_DRIFT>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_Y_INV_PSI>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_X_INV_R2C>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_Y_FWD_VH>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_Z_POISSON>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_Y_INV_VH>(d, ng, nullptr, nullptr, nullptr, true);
    launch_op<R, MX_X_C2R_KICK>(d, ng, nullptr, nullptr, nullptr, true);
}

template struct Mixed<float>;
template struct Mixed<double>;

}  // namespace qx
