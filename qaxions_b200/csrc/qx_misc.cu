// qx_misc.cu -- pointwise, reduction, spectrum-binning and initial-condition
// kernels (sm_100a).  See qx_misc.hpp for the contracts.
#include <stdexcept>
#include <string>

#include "qx_kernels.cuh"
#include "qx_misc.hpp"
#include "qx_philox.h"

namespace qx {

#define QX_CHECK_LAUNCH()                                                                              \
    do {                                                                                               \
        cudaError_t e_ = cudaGetLastError();                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

static unsigned grid_for(long n, int threads, long cap = 148L * 16) {
    long g = (n + threads - 1) / threads;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (unsigned)g;
}

// ---------------------------------------------------------------------------
// pointwise
// ---------------------------------------------------------------------------

template <typename R>
__global__ void k_kick(cx_t<R>* psi, const R* V, double dt, long S) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x)
        psi[i] = kick1<R>(psi[i], V[i], dt);
}

template <typename R>
__global__ void k_rho_to_V(const cx_t<R>* psi, R* V, long S) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        const cx_t<R> p = psi[i];
        V[i] = p.x * p.x + p.y * p.y;
    }
}

template <typename R>
__global__ void k_scale(cx_t<R>* psi, double s, long n) {
    const R sc = (R)s;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        psi[i] = cscale(psi[i], sc);
}

template <typename R>
__global__ void k_from_f64(const double2* src, cx_t<R>* dst, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double2 a = src[i];
        dst[i] = mk<cx_t<R>>((R)a.x, (R)a.y);
    }
}
template <typename R>
__global__ void k_to_f64(const cx_t<R>* src, double2* dst, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const cx_t<R> a = src[i];
        dst[i] = make_double2((double)a.x, (double)a.y);
    }
}
template <typename R>
__global__ void k_real_from_f64(const double* src, R* dst, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = (R)src[i];
}
template <typename R>
__global__ void k_real_to_f64(const R* src, double* dst, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

// ---------------------------------------------------------------------------
// reductions: fixed grid kRedBlocks x kRedThreads, per-block partials
// ---------------------------------------------------------------------------

template <typename R>
__global__ void __launch_bounds__(kRedThreads) k_reduce(int kind, const cx_t<R>* psi, const R* V, long S,
                                                        double* partial) {
    __shared__ double red[32];
    double a0 = 0.0, a1 = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        if (kind == RED_RHO) {
            const cx_t<R> p = psi[i];
            const double r = (double)p.x * p.x + (double)p.y * p.y;
            a0 += r;
            a1 = fmax_nan(a1, r);
        } else if (kind == RED_VABS) {
            a1 = fmax_nan(a1, fabs((double)V[i]));
        } else if (kind == RED_VRHO) {
            const cx_t<R> p = psi[i];
            a0 += (double)V[i] * ((double)p.x * p.x + (double)p.y * p.y);
        } else if (kind == RED_RE2) {
            const double r = (double)psi[i].x;
            a0 += r * r;
        } else {
            a0 += (double)psi[i].x;
        }
    }
    const double s0 = block_reduce<0>(a0, red);
    const double s1 = block_reduce<1>(a1, red);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = s0;
        partial[gridDim.x + blockIdx.x] = s1;
    }
}

// one warp (launched <<<1, 32>>>) folds the per-block partials
__global__ void k_fold(const double* partial, int n, double* out) {
    const double s = warp_fold<0>(partial, n);
    const double m = warp_fold<1>(partial + n, n);
    if (threadIdx.x == 0) {
        out[0] = s;
        out[1] = m;
    }
}

__global__ void k_fold_sum(const double* partial, long n, double* out) {
    const double s = warp_fold<0>(partial, n);
    if (threadIdx.x == 0) out[0] = s;
}

// drift factor tables (qx_misc.hpp)
__global__ void k_drift_tables(double2* t, int dim, int N, double fac, double scale) {
    const long na = dim == 3 ? (long)N * N : N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < na + N; i += (long)gridDim.x * blockDim.x) {
        if (i < na) {
            const long nx = signed_mode((int)(i % N), N);
            const long ny = dim == 3 ? signed_mode((int)(i / N), N) : 0;
            t[i] = cis_d(fac * (double)(nx * nx + ny * ny));
        } else {
            const long n = signed_mode((int)(i - na), N);
            const double2 w = cis_d(fac * (double)(n * n));
            t[i] = make_double2(w.x * scale, w.y * scale);
        }
    }
}

void drift_tables(double2* t, int dim, int N, double fac, double scale, cudaStream_t st) {
    const long n = (dim == 3 ? (long)N * N : N) + N;
    k_drift_tables<<<grid_for(n, 256), 256, 0, st>>>(t, dim, N, fac, scale);
    QX_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// packed half spectrum helpers.  Element (z, y, x) of [N][N][N/2] (3D) or
// (y, x) of [N][N/2] (2D); column 0 holds A + i B with A the kx = 0 mode and
// B the kx = N/2 mode, A(k) = (C(k) + conj C(-k))/2, B(k) = (C(k) - conj C(-k))/(2i).
// ---------------------------------------------------------------------------

__device__ __forceinline__ long mirror0(long i, int dim, int N) {  // index of (-ky,-kz) in column 0
    const int X = N / 2;
    const long rest = i / X;
    if (dim == 3) {
        const int y = (int)(rest % N), z = (int)(rest / N);
        return ((long)((N - z) % N) * N + (N - y) % N) * X;
    }
    const int y = (int)rest;
    return (long)((N - y) % N) * X;
}

template <typename R>
__global__ void k_poisson_packed(cx_t<R>* vh, int dim, int N, double pc, double g0) {
    using C = cx_t<R>;
    const int X = N / 2;
    const long total = (dim == 3 ? (long)N * N : (long)N) * X;
    auto g = [&](long m2) -> double { return m2 == 0 ? g0 : pc / (double)m2; };
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % X);
        const long rest = i / X;
        const int y = dim == 3 ? (int)(rest % N) : (int)rest;
        const int z = dim == 3 ? (int)(rest / N) : 0;
        const long ny = signed_mode(y, N), nz = dim == 3 ? signed_mode(z, N) : 0;
        if (x > 0) {
            vh[i] = cscale(vh[i], (R)g((long)x * x + ny * ny + nz * nz));
            continue;
        }
        const long im = mirror0(i, dim, N);
        if (im < i) continue;  // the pair is handled by its lower index
        const long mA = ny * ny + nz * nz, mB = mA + (long)X * X;
        const double al = 0.5 * (g(mA) + g(mB)), be = 0.5 * (g(mA) - g(mB));
        const C c = vh[i], cm = vh[im];
        // C'(k) = al C(k) + be conj C(-k); both modes share |k|^2 so al, be agree
        const C o = mk<C>((R)(al * c.x + be * cm.x), (R)(al * c.y - be * cm.y));
        const C om = mk<C>((R)(al * cm.x + be * c.x), (R)(al * cm.y - be * c.y));
        vh[i] = o;
        if (im != i) vh[im] = om;
    }
}

// deterministic per-warp aggregation of (bin, value, weight) into warp histograms
__device__ __forceinline__ void spec_agg(int b, double v, int w, double* hP, long long* hC) {
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    double s = 0.0;
    long long cnt = 0;
#pragma unroll 4
    for (int l = 0; l < 32; ++l) {
        const double vl = __shfl_sync(0xffffffffu, v, l);
        const int wl = __shfl_sync(0xffffffffu, w, l);
        if ((peers >> l) & 1u) {
            s += vl;
            cnt += wl;
        }
    }
    const int lane = threadIdx.x & 31;
    if (b >= 0 && lane == __ffs(peers) - 1) {
        hP[b] += s;
        hC[b] += cnt;
    }
    __syncwarp();
}

// Shell binning with the reference's Hermitian weights
// (src/spectrum/spectrum.cxx:63-155): weight 2 for 0 < kx < N/2, 1 for the
// kx = 0 and kx = N/2 modes (both unpacked from column 0).  Sums w |X|^2
// (the 1/S^2 factor is applied by the caller); counts are exact integers.
template <typename R>
__global__ void k_spec_bin(const cx_t<R>* vh, int dim, int N, const int* __restrict__ tab, int nbins,
                           double* part_P, long long* part_c) {
    using C = cx_t<R>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5;
    double* hPall = reinterpret_cast<double*>(smem_raw);
    long long* hCall = reinterpret_cast<long long*>(hPall + nw * nbins);
    for (int i = threadIdx.x; i < nw * nbins; i += blockDim.x) {
        hPall[i] = 0.0;
        hCall[i] = 0;
    }
    __syncthreads();
    double* hP = hPall + warp * nbins;
    long long* hC = hCall + warp * nbins;
    const int X = N / 2;
    const long total = (dim == 3 ? (long)N * N : (long)N) * X;
    const long stride = (long)gridDim.x * blockDim.x;
    const long iters = (total + stride - 1) / stride;
    for (long it = 0; it < iters; ++it) {
        const long i = it * stride + blockIdx.x * (long)blockDim.x + threadIdx.x;
        int b1 = -1, b2 = -1, w1 = 0, w2 = 0;
        double v1 = 0.0, v2 = 0.0;
        if (i < total) {
            const int x = (int)(i % X);
            const long rest = i / X;
            const int y = dim == 3 ? (int)(rest % N) : (int)rest;
            const int z = dim == 3 ? (int)(rest / N) : 0;
            const long ny = signed_mode(y, N), nz = dim == 3 ? signed_mode(z, N) : 0;
            const C c = vh[i];
            if (x > 0) {
                b1 = tab[(long)x * x + ny * ny + nz * nz];
                w1 = 2;
                v1 = 2.0 * ((double)c.x * c.x + (double)c.y * c.y);
            } else {
                const C cm = vh[mirror0(i, dim, N)];
                const double ax = 0.5 * ((double)c.x + cm.x), ay = 0.5 * ((double)c.y - cm.y);
                const double bx = 0.5 * ((double)c.x - cm.x), by = 0.5 * ((double)c.y + cm.y);
                const long mA = ny * ny + nz * nz;
                b1 = tab[mA];
                w1 = 1;
                v1 = ax * ax + ay * ay;
                b2 = tab[mA + (long)X * X];
                w2 = 1;
                v2 = bx * bx + by * by;
            }
            if (b1 < 0) w1 = 0;
            if (b2 < 0) w2 = 0;
        }
        spec_agg(b1, v1, w1, hP, hC);
        spec_agg(b2, v2, w2, hP, hC);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
        double s = 0.0;
        long long c = 0;
        for (int w = 0; w < nw; ++w) {
            s += hPall[w * nbins + b];
            c += hCall[w * nbins + b];
        }
        part_P[(long)blockIdx.x * nbins + b] = s;
        part_c[(long)blockIdx.x * nbins + b] = c;
    }
}

__global__ void k_spec_fold(const double* part_P, const long long* part_c, int nblk, int nbins, double* P,
                            long long* cnt) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) {
        double s = 0.0;
        long long c = 0;
        for (int k = 0; k < nblk; ++k) {
            s += part_P[(long)k * nbins + b];
            c += part_c[(long)k * nbins + b];
        }
        P[b] = s;
        cnt[b] = c;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

template <typename R>
void Misc<R>::kick(C* psi, const R* V, double dt, long S, cudaStream_t st) {
    k_kick<R><<<grid_for(S, 256), 256, 0, st>>>(psi, V, dt, S);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::rho_to_V(const C* psi, R* V, long S, cudaStream_t st) {
    k_rho_to_V<R><<<grid_for(S, 256), 256, 0, st>>>(psi, V, S);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::reduce(int kind, const C* psi, const R* V, long S, double* partial, double* out, cudaStream_t st) {
    k_reduce<R><<<kRedBlocks, kRedThreads, 0, st>>>(kind, psi, V, S, partial);
    QX_CHECK_LAUNCH();
    k_fold<<<1, 32, 0, st>>>(partial, kRedBlocks, out);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::fold_sum(const double* partial, long n, double* out, cudaStream_t st) {
    k_fold_sum<<<1, 32, 0, st>>>(partial, n, out);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::poisson_packed(C* vh, int dim, int N, double pc, double g0, cudaStream_t st) {
    const long total = (dim == 3 ? (long)N * N : (long)N) * (N / 2);
    k_poisson_packed<R><<<grid_for(total, 256), 256, 0, st>>>(vh, dim, N, pc, g0);
    QX_CHECK_LAUNCH();
}
template <typename R>
int Misc<R>::spectrum_bin(const C* vh, int dim, int N, const int* tab, int nbins, double* part_P,
                          long long* part_c, cudaStream_t st) {
    const int threads = 256, nblk = 296;
    const size_t smem = (size_t)(threads / 32) * nbins * (sizeof(double) + sizeof(long long));
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_spec_bin<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) throw std::runtime_error(std::string("smem attribute: ") + cudaGetErrorString(e));
    }
    k_spec_bin<R><<<nblk, threads, smem, st>>>(vh, dim, N, tab, nbins, part_P, part_c);
    QX_CHECK_LAUNCH();
    return nblk;
}
template <typename R>
void Misc<R>::spectrum_fold(const double* part_P, const long long* part_c, int nblk, int nbins, double* P,
                            long long* cnt, cudaStream_t st) {
    k_spec_fold<<<(nbins + 127) / 128, 128, 0, st>>>(part_P, part_c, nblk, nbins, P, cnt);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::from_f64(const double2* src, C* dst, long n, cudaStream_t st) {
    k_from_f64<R><<<grid_for(n, 256), 256, 0, st>>>(src, dst, n);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::to_f64(const C* src, double2* dst, long n, cudaStream_t st) {
    k_to_f64<R><<<grid_for(n, 256), 256, 0, st>>>(src, dst, n);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::real_from_f64(const double* src, R* dst, long n, cudaStream_t st) {
    k_real_from_f64<R><<<grid_for(n, 256), 256, 0, st>>>(src, dst, n);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::real_to_f64(const R* src, double* dst, long n, cudaStream_t st) {
    k_real_to_f64<R><<<grid_for(n, 256), 256, 0, st>>>(src, dst, n);
    QX_CHECK_LAUNCH();
}
template <typename R>
void Misc<R>::scale(C* psi, double s, long n, cudaStream_t st) {
    k_scale<R><<<grid_for(n, 256), 256, 0, st>>>(psi, s, n);
    QX_CHECK_LAUNCH();
}

template struct Misc<float>;
template struct Misc<double>;

// ---------------------------------------------------------------------------
// initial conditions (FP64)
// ---------------------------------------------------------------------------

__global__ void k_noise(double2* psi, long S, uint32_t k0, uint32_t k1) {
    const double twopi = 6.283185307179586476925286766559005768;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        const U4 r = philox4x32_10((uint32_t)i, (uint32_t)((uint64_t)i >> 32), 0u, 0u, k0, k1);
        const double u1 = u01(r.v[0]), u2 = u01(r.v[1]);
        psi[i] = make_double2(sqrt(-2.0 * log(u1)) * cos(twopi * u2), 0.0);
    }
}

__global__ void k_grf_filter(double2* h, int dim, int N, double dk, double kc) {
    const long S = dim == 3 ? (long)N * N * N : (long)N * N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        const long x = i % N, rest = i / N;
        const long y = rest % N, z = dim == 3 ? rest / N : 0;
        const long nx = signed_mode((int)x, N), ny = signed_mode((int)y, N), nz = signed_mode((int)z, N);
        const double k2 = (double)(nx * nx + ny * ny + nz * nz) * dk * dk;
        const double P = k2 > 0.0 ? exp(-k2 / (kc * kc)) / k2 : 0.0;
        const double a = sqrt(P);
        h[i] = make_double2(h[i].x * a, h[i].y * a);
    }
}

__global__ void k_grf_finish(double2* psi, long S, double s, double clip) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        const double d = fmax(psi[i].x * s, clip);
        psi[i] = make_double2(sqrt(1.0 + d), 0.0);
    }
}

__global__ void k_add_schive(double2* psi, int dim, int N, double L, int n, const double* par) {
    const long S = dim == 3 ? (long)N * N * N : (long)N * N;
    const double dx = L / N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        const long xi = i % N, rest = i / N;
        const long yi = rest % N, zi = dim == 3 ? rest / N : 0;
        const double x = xi * dx, y = yi * dx, z = zi * dx;
        double re = 0.0, im = 0.0;
        for (int j = 0; j < n; ++j) {
            const double* q = par + 7 * j;  // rc^2, sqrt(rho_c), cos ph, sin ph, cx, cy, cz
            double ddx = x - q[4] * L, ddy = y - q[5] * L;
            ddx -= L * rint(ddx / L);
            ddy -= L * rint(ddy / L);
            double r2 = ddx * ddx + ddy * ddy;
            if (dim == 3) {
                double ddz = z - q[6] * L;
                ddz -= L * rint(ddz / L);
                r2 += ddz * ddz;
            }
            const double u = 1.0 + 0.091 * (r2 / q[0]);
            const double u2 = u * u;
            const double amp = q[1] / (u2 * u2);
            re += amp * q[2];
            im += amp * q[3];
        }
        psi[i] = make_double2(psi[i].x + re, psi[i].y + im);
    }
}

__global__ void k_gauss_rho(double2* psi, int dim, int N, double L, double bkg, int n, const double* rows) {
    const long S = dim == 3 ? (long)N * N * N : (long)N * N;
    const double dx = L / N;
    const double twopi = 6.283185307179586476925286766559005768;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x) {
        const long xi = i % N, rest = i / N;
        const long yi = rest % N, zi = dim == 3 ? rest / N : 0;
        const double x = xi * dx, y = yi * dx, z = zi * dx;
        double rho = bkg;
        for (int j = 0; j < n; ++j) {
            const double amp = rows[5 * j], sg = rows[5 * j + 1];
            const double nrm = 1.0 / (sg * sg * sg * twopi);
            const double ddx = x - rows[5 * j + 2] * L, ddy = y - rows[5 * j + 3] * L;
            const double ddz = dim == 3 ? z - rows[5 * j + 4] * L : 0.0;
            const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
            rho += amp * nrm * exp(-r2 / (2.0 * sg * sg));
        }
        psi[i] = make_double2(rho, 0.0);
    }
}

__global__ void k_sqrt_div(double2* psi, long S, double mean) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < S; i += (long)gridDim.x * blockDim.x)
        psi[i] = make_double2(sqrt(psi[i].x / mean), 0.0);
}

void IC::noise(double2* psi, long S, uint64_t seed, cudaStream_t st) {
    k_noise<<<grid_for(S, 256), 256, 0, st>>>(psi, S, (uint32_t)seed, (uint32_t)(seed >> 32));
    QX_CHECK_LAUNCH();
}
void IC::grf_filter(double2* h, int dim, int N, double dk, double kc, cudaStream_t st) {
    const long S = dim == 3 ? (long)N * N * N : (long)N * N;
    k_grf_filter<<<grid_for(S, 256), 256, 0, st>>>(h, dim, N, dk, kc);
    QX_CHECK_LAUNCH();
}
void IC::grf_finish(double2* psi, long S, double s, double clip, cudaStream_t st) {
    k_grf_finish<<<grid_for(S, 256), 256, 0, st>>>(psi, S, s, clip);
    QX_CHECK_LAUNCH();
}
void IC::add_schive(double2* psi, int dim, int N, double L, int n, const double* par, cudaStream_t st) {
    const long S = dim == 3 ? (long)N * N * N : (long)N * N;
    k_add_schive<<<grid_for(S, 256), 256, 0, st>>>(psi, dim, N, L, n, par);
    QX_CHECK_LAUNCH();
}
void IC::gauss_rho(double2* psi, int dim, int N, double L, double bkg, int n, const double* rows,
                   cudaStream_t st) {
    const long S = dim == 3 ? (long)N * N * N : (long)N * N;
    k_gauss_rho<<<grid_for(S, 256), 256, 0, st>>>(psi, dim, N, L, bkg, n, rows);
    QX_CHECK_LAUNCH();
}
void IC::sqrt_div(double2* psi, long S, double mean, cudaStream_t st) {
    k_sqrt_div<<<grid_for(S, 256), 256, 0, st>>>(psi, S, mean);
    QX_CHECK_LAUNCH();
}

}  // namespace qx
