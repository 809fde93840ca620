// qx_fft.cuh -- device-side pencil FFT for sm_100a.
//
// One pencil (a 1D transform of length L) is processed by T = L/E threads,
// each holding E complex values in registers.  The transform is a mixed-radix
// Stockham autosort FFT (radices 2, 3, 4, 8): every stage applies twiddles and
// E/r radix-r butterflies in registers, and consecutive stages exchange data
// through shared memory.  Stage s with radix r and span Ns reads inputs
// x[j + m L/r] and writes outputs y[(j/Ns) Ns r + j%Ns + m Ns]
// (j = t + b T, m = 0..r-1), so the result comes out in natural order.
//
// The first stage's inputs (positions t + b T + m L/r0) and the last stage's
// outputs (positions t + b T + m L/r_last) are both lane-contiguous, so the
// callers load the first stage straight from HBM and store the last stage
// straight to HBM with coalesced accesses; only the S-1 inner exchanges touch
// shared memory.
//
// Twiddles come from a table tw[i] = exp(-2 pi i i / L) evaluated in long
// double on the host and rounded once to the storage precision.
//
// This replaces the FFTW c2c/r2c/c2r transforms of the reference's FFT plugin
// (src/fft/fft.h:122-140): same unnormalised definitions, FORWARD = exp(-i..).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qx {

template <typename R> struct Cx;
template <> struct Cx<float> { using T = float2; };
template <> struct Cx<double> { using T = double2; };

template <typename R> using cx_t = typename Cx<R>::T;

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) { C c; c.x = a; c.y = b; return c; }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
// multiply by sign*i: sign=-1 -> -i, sign=+1 -> +i
template <int SIGN, typename C> __device__ __forceinline__ C cmul_si(C a) {
    return SIGN < 0 ? mk<C>(a.y, -a.x) : mk<C>(-a.y, a.x);
}

// Two pencils at the same position (adjacent columns of a strided tile),
// transformed together: one 16-byte shared-memory access moves both values,
// and every twiddle is loaded and indexed once for the two.  The codelets and
// stage drivers below are written over a generic value type (C or CPair<C>).
template <typename C> struct __align__(2 * sizeof(C)) CPair {
    C a, b;
};
template <typename T> struct real_of { using type = decltype(T::x); };
template <typename C> struct real_of<CPair<C>> { using type = decltype(C::x); };
template <typename T> using real_t = typename real_of<T>::type;

template <typename C> __device__ __forceinline__ CPair<C> cadd(CPair<C> u, CPair<C> v) {
    return {cadd(u.a, v.a), cadd(u.b, v.b)};
}
template <typename C> __device__ __forceinline__ CPair<C> csub(CPair<C> u, CPair<C> v) {
    return {csub(u.a, v.a), csub(u.b, v.b)};
}
template <typename C> __device__ __forceinline__ CPair<C> cscale(CPair<C> u, decltype(C::x) s) {
    return {cscale(u.a, s), cscale(u.b, s)};
}
template <int SIGN, typename C> __device__ __forceinline__ CPair<C> cmul_si(CPair<C> u) {
    return {cmul_si<SIGN>(u.a), cmul_si<SIGN>(u.b)};
}
// pencil h (0 or 1) of a value
template <typename C> __device__ __forceinline__ C& pen(C& v, int) { return v; }
template <typename C> __device__ __forceinline__ C& pen(CPair<C>& v, int h) { return h ? v.b : v.a; }

// ---------------------------------------------------------------------------
// Radix plans (compile time).  Default plan of a length n: n = 2^e:
// [8]*(e/3) + [2^(e%3) if e%3] (e <= 3: one stage of radix n) -- the radix-8
// stages come first so that every shared-memory exchange of a one-warp-per-row
// transform is bank-conflict free under RowAcc's padding.  n = 3*2^k:
// [4]*(k/2) + [2]*(k%2) + [3].
//
// A transform length L may carry a plan index in its high bits,
// L = n | (plan << 16) (qx_with_plan): plan 0 is the default order above, plan
// 1 the same radices in reverse order (same elements per thread, other stage
// spans, twiddles and exchange patterns; the strided passes offer it to the
// autotuner).  Everything below takes such an L; qx_len(L) is the length.
// ---------------------------------------------------------------------------

__host__ __device__ constexpr int qx_len(int L) { return L & 0xFFFF; }
__host__ __device__ constexpr int qx_plan(int L) { return L >> 16; }
__host__ __device__ constexpr int qx_with_plan(int n, int plan) { return n | (plan << 16); }

__host__ __device__ constexpr bool qx_is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
__host__ __device__ constexpr int qx_log2(int n) { return n <= 1 ? 0 : 1 + qx_log2(n / 2); }

__host__ __device__ constexpr int qx_nstages0(int n) {
    return qx_is_pow2(n) ? (qx_log2(n) <= 3 ? 1 : (qx_log2(n) / 3 + (qx_log2(n) % 3 ? 1 : 0)))
                         : (qx_log2(n / 3) / 2 + qx_log2(n / 3) % 2 + 1);
}
__host__ __device__ constexpr int qx_nstages(int L) { return qx_nstages0(qx_len(L)); }

// radix of stage s of the default plan of length n
__host__ __device__ constexpr int qx_radix0(int n, int s) {
    if (qx_is_pow2(n)) {
        const int e = qx_log2(n);
        if (e <= 3) return n;
        const int rem = e % 3;
        if (rem) return s == e / 3 ? (1 << rem) : 8;
        return 8;
    }
    const int k = qx_log2(n / 3);
    const int n4 = k / 2, n2 = k % 2;
    if (s < n4) return 4;
    if (s < n4 + n2) return 2;
    return 3;
}

__host__ __device__ constexpr int qx_radix(int L, int s) {
    return qx_radix0(qx_len(L), qx_plan(L) == 1 ? qx_nstages(L) - 1 - s : s);
}

// does plan 1 differ from plan 0 for length n (radices not all equal)?
__host__ __device__ constexpr bool qx_plan1_differs(int n, int s = 1) {
    return s >= qx_nstages0(n) ? false : (qx_radix0(n, s) != qx_radix0(n, 0) || qx_plan1_differs(n, s + 1));
}

__host__ __device__ constexpr int qx_span(int L, int s) {  // product of radices before stage s
    return s == 0 ? 1 : qx_span(L, s - 1) * qx_radix(L, s - 1);
}

__host__ __device__ constexpr int qx_gcd(int a, int b) { return b == 0 ? a : qx_gcd(b, a % b); }
__host__ __device__ constexpr int qx_lcm(int a, int b) { return a / qx_gcd(a, b) * b; }
__host__ __device__ constexpr int qx_lcm_radices(int L, int s = 0) {
    return s >= qx_nstages(L) ? 1 : qx_lcm(qx_radix(L, s), qx_lcm_radices(L, s + 1));
}

// Elements per thread for a row pass that holds both an N-point c2c and the
// N/2-point core of an r2c/c2r: E_half = lcm(radices(N/2)), E_full = 2 E_half.
__host__ __device__ constexpr int qx_row_efull(int N) { return 2 * qx_lcm_radices(N / 2); }
__host__ __device__ constexpr int qx_row_threads(int N) { return N / qx_row_efull(N); }

// ---------------------------------------------------------------------------
// Small DFT codelets (SIGN = -1 forward, +1 backward), in place on a[0..r-1].
// ---------------------------------------------------------------------------

template <typename R> struct Consts {
    static constexpr R rsqrt2 = R(0.70710678118654752440084436210484903928);
    // rsqrt2 - R(rsqrt2): with it, x * (rsqrt2 + rsqrt2_lo) has an unbiased
    // magnitude (|(1 +- i) h| = 1 to O(eps^2)) instead of 1 - 1.7e-8 in FP32,
    // a bias every radix-8 stage would otherwise apply to the same modes at
    // every time step
    static constexpr R rsqrt2_lo = R(0.70710678118654752440084436210484903928L - (long double)R(0.70710678118654752440084436210484903928L));
    static constexpr R sqrt3_2 = R(0.86602540378443864676372317075293618347);
};

// x * 1/sqrt(2) with the constant carried to twice the working precision
template <typename C> __device__ __forceinline__ C cscale_rsqrt2(C a) {
    using R = decltype(C::x);
    return mk<C>(fma(a.x, Consts<R>::rsqrt2, a.x * Consts<R>::rsqrt2_lo),
                 fma(a.y, Consts<R>::rsqrt2, a.y * Consts<R>::rsqrt2_lo));
}
template <typename C> __device__ __forceinline__ CPair<C> cscale_rsqrt2(CPair<C> u) {
    return {cscale_rsqrt2(u.a), cscale_rsqrt2(u.b)};
}

template <int SIGN, typename C> __device__ __forceinline__ void dft2(C* a) {
    C t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft4(C* a) {
    C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    C t2 = cadd(a[1], a[3]), t3 = cmul_si<SIGN>(csub(a[1], a[3]));
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, t3);
    a[3] = csub(t1, t3);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft3(C* a) {
    using R = real_t<C>;
    const C s = cadd(a[1], a[2]);
    const C d = csub(a[1], a[2]);
    const C m = csub(a[0], cscale(s, R(0.5)));
    const C rot = cmul_si<SIGN>(cscale(d, Consts<R>::sqrt3_2));
    a[0] = cadd(a[0], s);
    a[1] = cadd(m, rot);
    a[2] = csub(m, rot);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft8(C* a) {
    C e[4] = {a[0], a[2], a[4], a[6]};
    C o[4] = {a[1], a[3], a[5], a[7]};
    dft4<SIGN>(e);
    dft4<SIGN>(o);
    // o[q] *= W8^q (sign SIGN): W8^1 = h(1 + SIGN i), W8^2 = SIGN i, W8^3 = h(-1 + SIGN i)
    const C o1 = o[1], o3 = o[3];
    o[1] = cscale_rsqrt2(cadd(o1, cmul_si<SIGN>(o1)));
    o[2] = cmul_si<SIGN>(o[2]);
    o[3] = cscale_rsqrt2(csub(cmul_si<SIGN>(o3), o3));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        a[q] = cadd(e[q], o[q]);
        a[q + 4] = csub(e[q], o[q]);
    }
}

template <int r, int SIGN, typename C> __device__ __forceinline__ void dft(C* a) {
    if constexpr (r == 2) dft2<SIGN>(a);
    else if constexpr (r == 3) dft3<SIGN>(a);
    else if constexpr (r == 4) dft4<SIGN>(a);
    else if constexpr (r == 8) dft8<SIGN>(a);
    else static_assert(r == 2 || r == 3 || r == 4 || r == 8, "unsupported radix");
}

// ---------------------------------------------------------------------------
// Stage driver.
// Acc: shared-memory accessor with `C& operator()(int pos)` for this pencil and
// a `sync()` that is a barrier over every thread sharing the buffer.
// ---------------------------------------------------------------------------

// Butterfly column j of block b of thread t at stage s.  J0 = 1 pairs the
// stage-0 columns, j = 2t + 2T (b/2) + (b%2), so that a thread holds the
// adjacent positions 2q and 2q+1 of its inputs: the layout in which an r2c
// transform of length L/2 leaves its real output and a c2r transform takes
// its real input, so a row pass can chain them without a shared-memory copy.
template <int L, int E, int s, int J0> __device__ __forceinline__ int stage_j(int b, int t) {
    constexpr int T = qx_len(L) / E;
    if constexpr (s == 0 && J0 == 1) {
        static_assert((E / qx_radix(L, 0)) % 2 == 0, "paired stage-0 columns need an even number of blocks");
        return 2 * t + 2 * T * (b >> 1) + (b & 1);
    } else {
        return t + b * T;
    }
}

// position held in v[e] before stage s (stage-s input order)
template <int L, int E, int s, int J0 = 0> __device__ __forceinline__ int in_pos(int e, int t) {
    constexpr int r = qx_radix(L, s);
    return stage_j<L, E, s, J0>(e / r, t) + (e % r) * (qx_len(L) / r);
}
// position held in v[e] after the last stage (natural-order output)
template <int L, int E> __device__ __forceinline__ int out_pos(int e, int t) {
    constexpr int r = qx_radix(L, qx_nstages(L) - 1);
    constexpr int T = qx_len(L) / E;
    return t + (e / r) * T + (e % r) * (qx_len(L) / r);
}

// Twiddle tables are stage-major: stage s >= 1 (span Ns, radix r) keeps its
// (r-1) Ns twiddles w_L^(k m L/(Ns r)) at (Ns - r0) + (m-1) Ns + k, so lanes
// with consecutive butterfly columns k read consecutive words (no bank
// conflicts when staged in shared memory); a table has L - r0 entries.
__host__ __device__ constexpr int qx_tw_index(int L, int Ns, int m, int k) {
    return (Ns - qx_radix(L, 0)) + (m - 1) * Ns + k;
}

// Twiddle sources: a stage-major table (global or a shared-memory copy), or a
// double-float pair of such tables hi + lo (lo = exact - hi), which
// applies each twiddle to twice the working precision.  A twiddle table is
// applied with the same values at every time step, so its rounding error
// would otherwise compound over the steps for modes whose forward and
// inverse transforms do not cancel it (those with a drift phase).
template <typename C> struct TwPair {
    const C* hi;
    const C* lo;
};

template <int SIGN, typename C> __device__ __forceinline__ C tw_mul(C v, const C* tw, int i) {
    C w = tw[i];
    if (SIGN > 0) w.y = -w.y;
    return cmul(v, w);
}
// v (w + l) with the small correction v l added before the final rounding
template <typename C> __device__ __forceinline__ C df_mul(C v, C w, C l) {
    const auto cx = v.x * l.x - v.y * l.y;
    const auto cy = v.x * l.y + v.y * l.x;
    return mk<C>(fma(v.x, w.x, fma(-v.y, w.y, cx)), fma(v.x, w.y, fma(v.y, w.x, cy)));
}
template <int SIGN, typename C> __device__ __forceinline__ C tw_mul(C v, const TwPair<C>& tw, int i) {
    C w = tw.hi[i], l = tw.lo[i];
    if (SIGN > 0) {
        w.y = -w.y;
        l.y = -l.y;
    }
    return df_mul(v, w, l);
}
template <int SIGN, typename C> __device__ __forceinline__ CPair<C> tw_mul(CPair<C> v, const C* tw, int i) {
    C w = tw[i];
    if (SIGN > 0) w.y = -w.y;
    return {cmul(v.a, w), cmul(v.b, w)};
}
template <int SIGN, typename C> __device__ __forceinline__ CPair<C> tw_mul(CPair<C> v, const TwPair<C>& tw, int i) {
    C w = tw.hi[i], l = tw.lo[i];
    if (SIGN > 0) {
        w.y = -w.y;
        l.y = -l.y;
    }
    return {df_mul(v.a, w, l), df_mul(v.b, w, l)};
}

template <int L, int E, int SIGN, int s, int J0, typename C, typename Acc, typename TW>
__device__ __forceinline__ void fft_stages(C (&v)[E], Acc& acc, int t, const TW& tw) {
    constexpr int S = qx_nstages(L);
    if constexpr (s < S) {
        constexpr int r = qx_radix(L, s);
        constexpr int Ns = qx_span(L, s);
        static_assert(E % r == 0, "radix must divide elements per thread");
        constexpr int nb = E / r;
#pragma unroll
        for (int b = 0; b < nb; ++b) {
            const int j = stage_j<L, E, s, J0>(b, t);
            if constexpr (Ns > 1) {
                const int k = j % Ns;
#pragma unroll
                for (int m = 1; m < r; ++m) v[b * r + m] = tw_mul<SIGN>(v[b * r + m], tw, qx_tw_index(L, Ns, m, k));
            }
            dft<r, SIGN>(&v[b * r]);
        }
        if constexpr (s + 1 < S) {
            constexpr int r2 = qx_radix(L, s + 1);
            acc.sync();
#pragma unroll
            for (int b = 0; b < nb; ++b) {
                const int j = stage_j<L, E, s, J0>(b, t);
                const int idxD = (j / Ns) * Ns * r + (j % Ns);
#pragma unroll
                for (int m = 0; m < r; ++m) acc(idxD + m * Ns) = v[b * r + m];
            }
            acc.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = acc(in_pos<L, E, s + 1>(e, t));
            fft_stages<L, E, SIGN, s + 1, J0>(v, acc, t, tw);
        }
    }
}

// Full transform: v in stage-0 input order on entry (see in_pos<L,E,0,J0>),
// natural-order outputs at out_pos<L,E> on exit.
template <int L, int E, int SIGN, int J0 = 0, typename C, typename Acc, typename TW>
__device__ __forceinline__ void fft_pencil(C (&v)[E], Acc& acc, int t, const TW& tw) {
    fft_stages<L, E, SIGN, 0, J0>(v, acc, t, tw);
}

// Twiddle source of a transform: DF = true selects double-float twiddles in
// the FP32 form (FP64 always uses the single table).  The wave-function
// transforms of the time step use them: the inverse transforms below undo the
// forward stages exactly, so a forward/phase/inverse sequence alone would not
// accumulate the twiddles' rounding, but the kick between steps does not
// commute with it and the rounded twiddles' magnitudes are not exactly 1, so
// with single FP32 twiddles the phase and norm errors of psi grow linearly
// with the number of steps.  The density/potential transforms keep single
// twiddles: V is rebuilt from psi every step and its errors do not compound.
template <bool DF, typename C>
__device__ __forceinline__ auto tw_src(const C* hi, const C* lo) {
    if constexpr (DF && sizeof(C) == 8) {
        return TwPair<C>{hi, lo};
    } else {
        (void)lo;
        return hi;
    }
}

// Position held by v[e] in the OUTPUT order of forward stage s (where stage s
// writes its results); for the last stage this is out_pos.
template <int L, int E, int s, int J0 = 0> __device__ __forceinline__ int stage_out_pos(int e, int t) {
    constexpr int r = qx_radix(L, s);
    constexpr int Ns = qx_span(L, s);
    const int j = stage_j<L, E, s, J0>(e / r, t);
    return (j / Ns) * Ns * r + (j % Ns) + (e % r) * Ns;
}

// Undo forward stage s (inverse butterfly, then conjugate twiddles), then
// move on to stage s-1.  Entry: v in stage_out_pos<s> order; exit of the
// whole chain: v in stage-0 input order (in_pos<L,E,0,J0>).
template <int L, int E, int s, int J0, typename C, typename Acc, typename TW>
__device__ __forceinline__ void ifft_rev_stages(C (&v)[E], Acc& acc, int t, const TW& tw) {
    constexpr int r = qx_radix(L, s);
    constexpr int Ns = qx_span(L, s);
    constexpr int nb = E / r;
#pragma unroll
    for (int b = 0; b < nb; ++b) {
        dft<r, +1>(&v[b * r]);
        if constexpr (Ns > 1) {
            const int k = stage_j<L, E, s, J0>(b, t) % Ns;
#pragma unroll
            for (int m = 1; m < r; ++m) v[b * r + m] = tw_mul<+1>(v[b * r + m], tw, qx_tw_index(L, Ns, m, k));
        }
    }
    if constexpr (s > 0) {
        acc.sync();
#pragma unroll
        for (int e = 0; e < E; ++e) acc(in_pos<L, E, s>(e, t)) = v[e];
        acc.sync();
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = acc(stage_out_pos<L, E, s - 1, J0>(e, t));
        ifft_rev_stages<L, E, s - 1, J0>(v, acc, t, tw);
    }
}

// Unnormalised inverse transform (x L) that exactly undoes fft_pencil<L,E,-1>:
// v in natural output order (out_pos<L,E>) on entry, in stage-0 input order
// (in_pos<L,E,0,J0>) on exit.
template <int L, int E, int J0 = 0, typename C, typename Acc, typename TW>
__device__ __forceinline__ void ifft_pencil_rev(C (&v)[E], Acc& acc, int t, const TW& tw) {
    ifft_rev_stages<L, E, qx_nstages(L) - 1, J0>(v, acc, t, tw);
}

}  // namespace qx
