// qx_corrector.cu -- learned corrector for coarse time steps (no counterpart in
// the reference).
//
// A small periodic convolutional network maps the state after one coarse step
// (dt_c = 4 dt) to the difference between four fine steps and that coarse
// step: psi_fine - psi_coarse ~ tau * net(features(psi_coarse, V_coarse)).
//
//   features (4 channels): Re psi, Im psi, V / v_scale, |psi|^2 - 1
//   layer 1: 3^3 periodic conv 4 -> 32, GELU
//   layer 2: 3^3 periodic conv 32 -> 32, GELU
//   layer 3: 3^3 periodic conv 32 -> 2 (the correction / tau)
//
// Weights are kept in FP32 (master copy, Adam moments) and rounded to BF16 for
// the tensor cores; activations between layers are BF16, every accumulation is
// FP32.  Activations are channel-last [site][C] in reference site order
// (x fastest).
//
// Convolutions (forward, and the data gradient as the same convolution with
// spatially flipped, channel-transposed weights) are implicit GEMMs on the
// tensor cores with mma.sync m16n8k16 (BF16 in, FP32 accumulate): a block owns
// an 8 x 8 x 4 brick of sites, stages the brick's periodic halo and the layer's
// weights in shared memory, and each warp accumulates 32 sites x all output
// channels over K = 27 offsets x input channels.  Weight gradients are summed
// over sites with CUDA-core FMAs, 4 x 4 register blocks per thread, per-block
// partial sums folded in a fixed order (deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qaxions_b200.h"

namespace qx {
namespace nn {

constexpr int KOFF = 27;
constexpr int BX = 8, BY = 8, BZ = 4;          // brick of sites per block
constexpr int HX = BX + 2, HY = BY + 2, HZ = BZ + 2;
constexpr int HALO = HX * HY * HZ;             // 600 halo sites
constexpr int BSITES = BX * BY * BZ;           // 256 sites

#define NN_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// offset index o = (dz+1)*9 + (dy+1)*3 + (dx+1)
__host__ __device__ constexpr int off_dx(int o) { return o % 3 - 1; }
__host__ __device__ constexpr int off_dy(int o) { return (o / 3) % 3 - 1; }
__host__ __device__ constexpr int off_dz(int o) { return o / 9 - 1; }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---------------------------------------------------------------------------
// tensor-core periodic 3^3 convolution
//   X:  [S][CINP] bf16 input (channel-last, padded with zeros)
//   W:  [27][COUTP][CINP + 8] bf16 (k contiguous; pitch padded against bank conflicts)
//   out: zf [S][cout] FP32 (pre-activation, optional), ab [S][COUTP] bf16 GELU(z) (optional)
// ---------------------------------------------------------------------------
template <int CINP, int COUTP>
struct ConvSmem {
    static constexpr int XP = CINP + 8;  // halo pitch (bf16)
    static constexpr int WP = CINP + 8;  // weight pitch (bf16)
    static constexpr size_t bytes() { return (size_t)HALO * XP * 2 + (size_t)KOFF * COUTP * WP * 2 + COUTP * 4; }
};

template <int CINP, int COUTP>
__global__ void __launch_bounds__(256) k_conv(const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ W,
                                              const float* __restrict__ bias, int N, int cout, float* zf,
                                              __nv_bfloat16* ab, float* out2, int gelu_ab) {
    using SM = ConvSmem<CINP, COUTP>;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* ws = xs + HALO * SM::XP;
    float* bs = reinterpret_cast<float*>(ws + KOFF * COUTP * SM::WP);
    const int tid = threadIdx.x;
    const int nbx = N / BX, nby = N / BY;
    const int bxi = blockIdx.x % nbx, byi = (blockIdx.x / nbx) % nby, bzi = blockIdx.x / (nbx * nby);
    const int x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;

    // weights and bias
    {
        const uint4* src = reinterpret_cast<const uint4*>(W);
        uint4* dst = reinterpret_cast<uint4*>(ws);
        const int n16 = KOFF * COUTP * SM::WP * 2 / 16;
        for (int i = tid; i < n16; i += blockDim.x) dst[i] = src[i];
        for (int i = tid; i < COUTP; i += blockDim.x) bs[i] = (bias && i < cout) ? bias[i] : 0.f;
    }
    // periodic halo of the brick (16-byte chunks of a site's channels)
    {
        constexpr int CH = CINP / 8;  // 16-byte chunks per site
        for (int i = tid; i < HALO * CH; i += blockDim.x) {
            const int h = i / CH, c = i % CH;
            const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
            const long gs = ((long)wrapi(z0 + hz - 1, N) * N + wrapi(y0 + hy - 1, N)) * N + wrapi(x0 + hx - 1, N);
            *reinterpret_cast<uint4*>(xs + h * SM::XP + c * 8) = *reinterpret_cast<const uint4*>(X + gs * CINP + c * 8);
        }
    }
    __syncthreads();

    const int warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, tg = lane & 3;
    constexpr int NT = COUTP / 8;
    // two m-tiles of 16 sites per warp: brick sites s = 32 warp + 16 mt + r, s = x + 8 y + 64 z
    float acc[2][NT][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[mt][nt][q] = 0.f;
    int hbase[2][2];  // halo index of rows g and g+8 of each m-tile at offset 0
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int s = 32 * warp + 16 * mt + g + 8 * rr;
            const int x = s % BX, y = (s / BX) % BY, z = s / (BX * BY);
            hbase[mt][rr] = (x + 1) + HX * ((y + 1) + HY * (z + 1));
        }
#pragma unroll 1
    for (int o = 0; o < KOFF; ++o) {
        const int doff = off_dx(o) + HX * (off_dy(o) + HY * off_dz(o));
        const __nv_bfloat16* wo = ws + o * COUTP * SM::WP;
#pragma unroll
        for (int kc = 0; kc < CINP / 16; ++kc) {
            uint32_t b[NT][2];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const __nv_bfloat16* wr = wo + (nt * 8 + g) * SM::WP + kc * 16 + tg * 2;
                b[nt][0] = *reinterpret_cast<const uint32_t*>(wr);
                b[nt][1] = *reinterpret_cast<const uint32_t*>(wr + 8);
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const __nv_bfloat16* r0 = xs + (hbase[mt][0] + doff) * SM::XP + kc * 16 + tg * 2;
                const __nv_bfloat16* r1 = xs + (hbase[mt][1] + doff) * SM::XP + kc * 16 + tg * 2;
                uint32_t a[4];
                a[0] = *reinterpret_cast<const uint32_t*>(r0);
                a[1] = *reinterpret_cast<const uint32_t*>(r1);
                a[2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
                a[3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], a, b[nt]);
            }
        }
    }
    // epilogue: rows g, g+8; columns nt*8 + 2tg, +1
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int s = 32 * warp + 16 * mt + g + 8 * rr;
            const int x = s % BX, y = (s / BX) % BY, z = s / (BX * BY);
            const long gs = ((long)(z0 + z) * N + (y0 + y)) * N + (x0 + x);
#pragma unroll
            for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int co = nt * 8 + 2 * tg + cc;
                    const float zv = acc[mt][nt][2 * rr + cc] + bs[co];
                    if (co < cout) {
                        if (zf) zf[gs * cout + co] = zv;
                        if (out2) out2[gs * cout + co] = zv;
                    }
                    if (ab) ab[gs * COUTP + co] = __float2bfloat16(co < cout ? (gelu_ab ? gelu(zv) : zv) : 0.f);
                }
        }
}

// ---------------------------------------------------------------------------
// CIN -> 32 periodic 3^3 convolutions (CIN = 16 or 32) on the 5th-generation
// tensor cores (tcgen05.mma kind::f16: BF16 operands read from shared memory
// through matrix descriptors, FP32 accumulators in tensor memory).
//
// Persistent blocks (two per SM) keep all 27 offsets' weights in shared memory
// and walk bricks of 8 x 16 x 2 sites.  A brick is two M = 128 tiles (one per
// z), each the GEMM [128 sites] x [K = 27 offsets x CIN channels] x [32
// outputs]: 27 CIN / 16 MMAs of K = 16.  (A one-block-per-SM version with a
// dedicated MMA warp, triple-buffered halos and double-buffered accumulators
// measured slower: with N = 32 the two independent blocks overlap each other's
// halo loads and epilogues better.)  Both operands use the canonical no-swizzle K-major
// layout, whose unit is a "core matrix" of 8 rows x 16 bytes (8 BF16 channels)
// stored contiguously:
//   weights  W[o]: core matrix (n-group g, channel chunk c) at ((o*4 + g)*KC + c)*128 B
//            (K step LBO = 128 B, N step SBO = KC*128 B; KC = CIN / 8)
//   halo     [hz][hy][c][hx][8 ch]: 16 B per (site, chunk), so the 8 sites
//            x..x+7 of one (y, z) row of any offset are one contiguous core
//            matrix, and an offset is just a shifted start address
//            (K step LBO = HX*16 B, M step = next y, SBO = KC*HX*16 B)
// One thread issues the MMAs and commits them to an mbarrier; then all eight
// warps read the accumulators back (tcgen05.ld, warp w: tile w/4, lanes
// 32*(w%4) ..) for the bias / GELU epilogue.  Waits are bounded; tensor memory
// is freed on every exit path.
// ---------------------------------------------------------------------------
namespace tc {
constexpr int BX = 8, BY = 16, BZ = 2;  // brick: BZ tiles of 128 sites
constexpr int HX = BX + 2, HY = BY + 2, HZ = BZ + 2;
constexpr int COUT = 32;
constexpr int TMEM_COLS = 64;  // BZ x 32 FP32 columns
template <int CIN> struct Geo {
    static constexpr int KC = CIN / 8;                                 // 16-byte channel chunks
    static constexpr int HALO_BYTES = HZ * HY * KC * HX * 16;          // 46,080 for CIN = 32
    static constexpr int W_BYTES = KOFF * (COUT / 8) * KC * 128;       // 55,296 for CIN = 32
    static constexpr size_t SMEM = (size_t)HALO_BYTES + W_BYTES + 128;  // + alignment slack
    static constexpr uint32_t LBO_A = HX * 16, SBO_A = KC * HX * 16;
    static constexpr uint32_t LBO_B = 128, SBO_B = KC * 128;
};
// instruction descriptor: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(COUT >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    // start >> 4 (bits 0-13), LBO >> 4 (16-29), SBO >> 4 (32-45), version 1
    // (bits 46-47), base offset 0, no swizzle (bits 61-63 = 0)
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(accumulate), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred q;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
    }
}
// 32 lanes x 32 consecutive FP32 columns: thread t of the warp gets lane base + t
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
}  // namespace tc

// X: [S][CIN] bf16; W: [27][32][CIN + 8] bf16 (the packed layer weights);
// outputs as k_conv.  blockDim 256; grid <= number of bricks.
template <int CIN>
__global__ void __launch_bounds__(256, 2) k_conv_tc(const __nv_bfloat16* __restrict__ X,
                                                    const __nv_bfloat16* __restrict__ W,
                                                    const float* __restrict__ bias, int N, int cout, float* zf,
                                                    __nv_bfloat16* ab, float* out2, int gelu_ab, int* err) {
    // the brick of this kernel (the names shadow the mma.sync kernels' brick)
    constexpr int BX = tc::BX, BY = tc::BY, BZ = tc::BZ, HX = tc::HX, HY = tc::HY, HZ = tc::HZ;
    using G = tc::Geo<CIN>;
    constexpr int COUT = tc::COUT, KC = G::KC, HALO_BYTES = G::HALO_BYTES;
    constexpr uint32_t TMEM_COLS = tc::TMEM_COLS;
    using tc::commit;
    using tc::fence_after;
    using tc::fence_before;
    using tc::mbar_init;
    using tc::mbar_wait;
    using tc::mma;
    using tc::proxy_fence;
    using tc::smem_addr;
    using tc::smem_desc;
    extern __shared__ __align__(128) unsigned char smem_tc[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ float bs[COUT];
    __shared__ int s_fail;
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_tc) + 127) & ~(uintptr_t)127);
    unsigned char* halo = base;
    unsigned char* wsm = base + HALO_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // weights -> canonical K-major core matrices; bias
    for (int i = tid; i < KOFF * COUT * KC; i += blockDim.x) {
        const int o = i / (COUT * KC), co = (i / KC) % COUT, c = i % KC;
        const uint4 v = *reinterpret_cast<const uint4*>(W + ((size_t)o * COUT + co) * (CIN + 8) + c * 8);
        *reinterpret_cast<uint4*>(wsm + ((o * (COUT / 8) + co / 8) * KC + c) * 128 + (co % 8) * 16) = v;
    }
    if (tid < COUT) bs[tid] = (bias && tid < cout) ? bias[tid] : 0.f;
    if (tid == 0) {
        s_fail = 0;
        mbar_init(smem_addr(&mbar));
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"((uint32_t)TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    const int nbx = N / BX, nby = N / BY;
    const long nbricks = (long)nbx * nby * (N / BZ);
    uint32_t phase = 0;
    for (long br = blockIdx.x; br < nbricks; br += gridDim.x) {
        const int bxi = (int)(br % nbx), byi = (int)((br / nbx) % nby), bzi = (int)(br / ((long)nbx * nby));
        const int x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;
        // periodic halo, 16-byte chunks: [hz][hy][c][hx], all copies in flight at once
        for (int i = tid; i < HZ * HY * KC * HX; i += blockDim.x) {
            const int hx = i % HX, c = (i / HX) % KC, hy = (i / (HX * KC)) % HY, hz = i / (HX * KC * HY);
            const long gs = ((long)wrapi(z0 + hz - 1, N) * N + wrapi(y0 + hy - 1, N)) * N + wrapi(x0 + hx - 1, N);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(halo + (size_t)i * 16)),
                         "l"(X + gs * CIN + c * 8)
                         : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        proxy_fence();  // shared-memory writes -> visible to the tensor cores' reads
        __syncthreads();
        if (tid == 0) {
            fence_after();
            const uint32_t h0 = smem_addr(halo), w0 = smem_addr(wsm);
#pragma unroll 1
            for (int zt = 0; zt < BZ; ++zt)
#pragma unroll 1
                for (int o = 0; o < KOFF; ++o) {
                    const int hz = zt + 1 + off_dz(o), hy = 1 + off_dy(o), hx = 1 + off_dx(o);
#pragma unroll
                    for (int kk = 0; kk < KC / 2; ++kk) {
                        const uint32_t a = h0 + (uint32_t)((((hz * HY + hy) * KC + 2 * kk) * HX + hx) * 16);
                        const uint32_t b = w0 + (uint32_t)(((o * (COUT / 8)) * KC + 2 * kk) * 128);
                        mma(tmem + (uint32_t)(zt * COUT), smem_desc(a, G::LBO_A, G::SBO_A),
                            smem_desc(b, G::LBO_B, G::SBO_B), (o | kk) != 0);
                    }
                }
            commit(smem_addr(&mbar));
        }
        __syncwarp();
        if (!mbar_wait(smem_addr(&mbar), phase, 1LL << 31)) s_fail = 1;
        phase ^= 1u;
        fence_after();
        // epilogue: warp w reads tile w / 4, rows 32 (w % 4) + lane (row r = site x + 8 y)
        {
            const int zt = warp >> 2, q = warp & 3;
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(zt * COUT), v);
            const int r = 32 * q + lane;
            const int x = r % BX, y = r / BX;
            const long gs = ((long)(z0 + zt) * N + (y0 + y)) * N + (x0 + x);
#pragma unroll
            for (int co = 0; co < COUT; ++co) v[co] += bs[co];
            if (cout == COUT) {  // 16-byte stores of the site's 32 channels
                if (zf) {
#pragma unroll
                    for (int j = 0; j < COUT / 4; ++j)
                        reinterpret_cast<float4*>(zf + gs * COUT)[j] =
                            make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                }
                if (out2) {
#pragma unroll
                    for (int j = 0; j < COUT / 4; ++j)
                        reinterpret_cast<float4*>(out2 + gs * COUT)[j] =
                            make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                }
            } else {
#pragma unroll
                for (int co = 0; co < COUT; ++co)
                    if (co < cout) {
                        if (zf) zf[gs * cout + co] = v[co];
                        if (out2) out2[gs * cout + co] = v[co];
                    }
            }
            if (ab) {
#pragma unroll
                for (int j = 0; j < COUT / 8; ++j) {
                    union {
                        __nv_bfloat162 h[4];
                        uint4 u;
                    } pk;
#pragma unroll
                    for (int q2 = 0; q2 < 4; ++q2) {
                        const int co = 8 * j + 2 * q2;
                        const float a0 = co < cout ? (gelu_ab ? gelu(v[co]) : v[co]) : 0.f;
                        const float a1 = co + 1 < cout ? (gelu_ab ? gelu(v[co + 1]) : v[co + 1]) : 0.f;
                        pk.h[q2] = __floats2bfloat162_rn(a0, a1);
                    }
                    reinterpret_cast<uint4*>(ab + gs * COUT)[j] = pk.u;
                }
            }
        }
        fence_before();
        __syncthreads();  // accumulators read and halo consumed before the next brick
        if (s_fail) break;
    }
    if (s_fail && tid == 0) {
        atomicExch(err, 1);
        mbar_wait(smem_addr(&mbar), phase ^ 1u, 1LL << 32);  // let the timed-out MMAs drain before freeing
    }
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TMEM_COLS)
                     : "memory");
}

// weight gradient: dW[o][ci][co] = sum_s A[s + o][ci] dZ[s][co]; db[co] = sum_s dZ[s][co]
// A: [S][CINP] bf16 (forward input of the layer), dZ: [S][cout] FP32.
// Persistent blocks over bricks; thread t owns 4x4 (ci, co) blocks of offsets.
// partial: [gridDim.x][27 * cin * cout + cout]
template <int CINP>
__global__ void __launch_bounds__(256) k_wgrad(const __nv_bfloat16* __restrict__ A, const float* __restrict__ dZ, int N,
                                               int cin, int cout, float* partial) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* as = reinterpret_cast<float*>(smem);              // [HALO][CINP]
    float* zs = as + HALO * CINP;                            // [BSITES][cout]
    const int tid = threadIdx.x;
    const int nbx = N / BX, nby = N / BY, nbz = N / BZ;
    const int nbricks = nbx * nby * nbz;
    const int cib = (cin + 3) / 4, cob = (cout + 3) / 4;
    const int ngroups = KOFF * cib * cob;
    constexpr int GMAX = 8;  // groups per thread (27 * 8 * 8 = 1728 <= 256 * 8)
    float acc[GMAX][16];
    float bacc = 0.f;
#pragma unroll
    for (int j = 0; j < GMAX; ++j)
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[j][q] = 0.f;
    for (int br = blockIdx.x; br < nbricks; br += gridDim.x) {
        const int bxi = br % nbx, byi = (br / nbx) % nby, bzi = br / (nbx * nby);
        const int x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;
        __syncthreads();
        for (int i = tid; i < HALO * CINP; i += blockDim.x) {
            const int h = i / CINP, c = i % CINP;
            const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
            const long gs = ((long)wrapi(z0 + hz - 1, N) * N + wrapi(y0 + hy - 1, N)) * N + wrapi(x0 + hx - 1, N);
            as[i] = __bfloat162float(A[gs * CINP + c]);
        }
        for (int i = tid; i < BSITES * cout; i += blockDim.x) {
            const int s = i / cout, c = i % cout;
            const int x = s % BX, y = (s / BX) % BY, z = s / (BX * BY);
            const long gs = ((long)(z0 + z) * N + (y0 + y)) * N + (x0 + x);
            zs[i] = dZ[gs * cout + c];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < GMAX; ++j) {
            const int gidx = tid + j * blockDim.x;
            if (gidx >= ngroups) break;
            const int o = gidx / (cib * cob), cb = (gidx / cob) % cib, ob = gidx % cob;
            const int doff = off_dx(o) + HX * (off_dy(o) + HY * off_dz(o));
            for (int s = 0; s < BSITES; ++s) {
                const int x = s % BX, y = (s / BX) % BY, z = s / (BX * BY);
                const int h = (x + 1) + HX * ((y + 1) + HY * (z + 1)) + doff;
                float av[4], zv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int ci = 4 * cb + q, co = 4 * ob + q;
                    av[q] = ci < cin ? as[h * CINP + ci] : 0.f;
                    zv[q] = co < cout ? zs[s * cout + co] : 0.f;
                }
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[j][4 * p + q] = fmaf(av[p], zv[q], acc[j][4 * p + q]);
            }
        }
        if (tid < cout)
            for (int s = 0; s < BSITES; ++s) bacc += zs[s * cout + tid];
    }
    const int nw = KOFF * cin * cout;
    float* outp = partial + (long)blockIdx.x * (nw + cout);
#pragma unroll
    for (int j = 0; j < GMAX; ++j) {
        const int gidx = tid + j * blockDim.x;
        if (gidx >= ngroups) break;
        const int o = gidx / (cib * cob), cb = (gidx / cob) % cib, ob = gidx % cob;
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ci = 4 * cb + p, co = 4 * ob + q;
                if (ci < cin && co < cout) outp[(o * cin + ci) * cout + co] = acc[j][4 * p + q];
            }
    }
    if (tid < cout) outp[nw + tid] = bacc;
}

// Weight gradient on the tensor cores (tcgen05), the same sums as k_wgrad:
//   dW[o][ci][co] = sum_s A[s + o][ci] dZ[s][co],  db[co] = sum_s dZ[s][co].
// Per 8 x 8 x 4 brick (K = 256 sites) and per group of OPG = 128 / CINP
// offsets, the block builds the group's shifted activations as the A operand
// [128 rows (offset j, channel ci)] x [256 sites] in the canonical no-swizzle
// K-major layout (core matrix (row group, 8-site chunk) at (rg * 32 + chunk) *
// 128 B), and dZ of the brick once as the B operand [32 outputs] x [256 sites]
// (BF16, the same layout); one thread issues 16 MMAs of M = 128, N = 32, K = 16
// into the group's 32 tensor-memory columns, accumulating over every brick the
// block processes.  Two group buffers alternate, so the next group is built
// while the previous group's MMAs run; an mbarrier per buffer orders reuse.
// dZ is rounded to BF16 for the tensor cores (the activations already are);
// the bias gradient stays an FP32 sum.  Waits are bounded; tensor memory is
// freed on every path.  partial: as k_wgrad.
namespace wtc {
constexpr int K = BSITES;            // 256 sites per brick
constexpr int KCH = K / 8;           // 32 chunks of 8 sites
constexpr int OPER_BYTES = 128 * K * 2;  // one A operand: 64 KB
constexpr int DZ_BYTES = 32 * K * 2;     // B operand: 16 KB
constexpr uint32_t LBO = 128, SBO = KCH * 128;
template <int CINP> struct Geo {
    static constexpr int OPG = 128 / CINP;                    // offsets per group
    static constexpr int NGROUPS = (KOFF + OPG - 1) / OPG;    // 7 (CINP 32) or 4 (CINP 16)
    static constexpr int HALO_BYTES = HALO * CINP * 2;
    static constexpr size_t SMEM = 2 * (size_t)OPER_BYTES + DZ_BYTES + HALO_BYTES + 128;
    static constexpr uint32_t TMEM_COLS = NGROUPS * 32 <= 128 ? 128 : 256;
};
}  // namespace wtc

template <int CINP>
__global__ void __launch_bounds__(256, 1) k_wgrad_tc(const __nv_bfloat16* __restrict__ A, const float* __restrict__ dZ,
                                                     int N, int cin, int cout, float* partial, int* err) {
    using G = wtc::Geo<CINP>;
    constexpr int OPG = G::OPG, NG = G::NGROUPS;
    using tc::commit;
    using tc::fence_after;
    using tc::fence_before;
    using tc::mbar_init;
    using tc::mbar_wait;
    using tc::mma;
    using tc::proxy_fence;
    using tc::smem_addr;
    using tc::smem_desc;
    extern __shared__ __align__(128) unsigned char smem_w[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ float bred[8][32];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_w) + 127) & ~(uintptr_t)127);
    unsigned char* oper[2] = {base, base + wtc::OPER_BYTES};
    unsigned char* dzb = base + 2 * wtc::OPER_BYTES;
    __nv_bfloat16* halo = reinterpret_cast<__nv_bfloat16*>(dzb + wtc::DZ_BYTES);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mbar_init(smem_addr(&mbar[0]));
        mbar_init(smem_addr(&mbar[1]));
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(G::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;

    const int nbx = N / BX, nby = N / BY, nbz = N / BZ;
    const int nbricks = nbx * nby * nbz;
    int ncommit[2] = {0, 0};  // commits issued on each buffer (the same in every thread)
    int last = -1;            // buffer of the latest commit
    float bsum = 0.f;         // bias partial of output tid % 32
    bool first = true;
    int fail = 0;             // this thread's wait timed out; combined at block barriers
    auto wait_buf = [&](int b, long long limit) {
        if (ncommit[b] > 0 && !mbar_wait(smem_addr(&mbar[b]), (uint32_t)((ncommit[b] - 1) & 1), limit)) fail = 1;
    };
    bool abort = false;
    for (int br = blockIdx.x; br < nbricks && !abort; br += gridDim.x) {
        const int bxi = br % nbx, byi = (br / nbx) % nby, bzi = br / (nbx * nby);
        const int x0 = bxi * BX, y0 = byi * BY, z0 = bzi * BZ;
        // the previous brick's MMAs read the halo, dZ and both buffers: wait for the last commit
        if (last >= 0) wait_buf(last, 1LL << 31);
        fence_after();
        // periodic halo [hz][hy][hx][CINP] (16-byte copies)
        for (int i = tid; i < HALO * (CINP / 8); i += blockDim.x) {
            const int h = i / (CINP / 8), c = i % (CINP / 8);
            const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
            const long gs = ((long)wrapi(z0 + hz - 1, N) * N + wrapi(y0 + hy - 1, N)) * N + wrapi(x0 + hx - 1, N);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(halo + (size_t)h * CINP + c * 8)),
                         "l"(A + gs * CINP + c * 8)
                         : "memory");
        }
        // dZ of the brick -> B operand: output co, chunk r = y + 8 z of 8 sites x = 0..7
        for (int q = tid; q < 32 * wtc::KCH; q += blockDim.x) {
            const int co = q % 32, r = q / 32;
            const int y = r % BY, z = r / BY;
            union {
                __nv_bfloat162 h[4];
                uint4 u;
            } pk;
#pragma unroll
            for (int x2 = 0; x2 < 4; ++x2) {
                float v0 = 0.f, v1 = 0.f;
                if (co < cout) {
                    const long g0 = ((long)(z0 + z) * N + (y0 + y)) * N + (x0 + 2 * x2);
                    v0 = dZ[g0 * cout + co];
                    v1 = dZ[(g0 + 1) * cout + co];
                    bsum += v0 + v1;
                }
                pk.h[x2] = __floats2bfloat162_rn(v0, v1);
            }
            *reinterpret_cast<uint4*>(dzb + (size_t)((co / 8) * wtc::KCH + r) * 128 + (co % 8) * 16) = pk.u;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (__syncthreads_or(fail)) {
            abort = true;
            break;
        }
        for (int g = 0; g < NG; ++g) {
            const int b = (ncommit[0] + ncommit[1]) & 1;
            wait_buf(b, 1LL << 31);  // this buffer's previous MMAs are done
            fence_after();
            unsigned char* op = oper[b];
            // rows m = j CINP + ci (offset o = g OPG + j), chunk r: the 8 sites
            // x = 0..7 of row (y, z) shifted by the offset
            for (int q = tid; q < 128 * wtc::KCH; q += blockDim.x) {
                const int ci = q % CINP, rest = q / CINP;
                const int r = rest % wtc::KCH, j = rest / wtc::KCH;
                const int o = g * OPG + j;
                const int y = r % BY, z = r / BY;
                union {
                    __nv_bfloat16 h[8];
                    uint4 u;
                } pk;
                if (o < KOFF) {
                    const int hb = (1 + off_dx(o)) + HX * ((1 + y + off_dy(o)) + HY * (1 + z + off_dz(o)));
#pragma unroll
                    for (int x = 0; x < 8; ++x) pk.h[x] = halo[(size_t)(hb + x) * CINP + ci];
                } else {
                    pk.u = make_uint4(0u, 0u, 0u, 0u);
                }
                const int m = j * CINP + ci;
                *reinterpret_cast<uint4*>(op + (size_t)((m / 8) * wtc::KCH + r) * 128 + (m % 8) * 16) = pk.u;
            }
            proxy_fence();  // generic-proxy shared writes -> visible to the tensor cores
            if (__syncthreads_or(fail)) {  // the same decision in every thread
                abort = true;
                break;
            }
            if (tid == 0) {
                fence_after();
                const uint32_t a0 = smem_addr(op), b0 = smem_addr(dzb);
#pragma unroll 1
                for (int kk = 0; kk < wtc::KCH / 2; ++kk)
                    mma(tmem + (uint32_t)(g * 32), smem_desc(a0 + (uint32_t)(2 * kk * 128), wtc::LBO, wtc::SBO),
                        smem_desc(b0 + (uint32_t)(2 * kk * 128), wtc::LBO, wtc::SBO), (!first || kk > 0) ? 1u : 0u);
                commit(smem_addr(&mbar[b]));
            }
            ++ncommit[b];
            last = b;
        }
        first = false;
    }
    // every MMA done before the accumulators are read (after a time-out: a
    // longer bounded wait, so the MMAs in flight drain before tensor memory
    // is freed)
    if (last >= 0) wait_buf(last, abort ? (1LL << 32) : (1LL << 31));
    if (last >= 0) wait_buf(last ^ 1, abort ? (1LL << 32) : (1LL << 31));
    fence_after();
    if (__syncthreads_or(fail)) abort = true;
    const int nw = KOFF * cin * cout;
    float* outp = partial + (long)blockIdx.x * (nw + cout);
    if (!abort) {
        // warp w reads lanes 32 (w % 4) .. of groups w / 4, w / 4 + 2, ...
        for (int g = warp >> 2; g < NG; g += 2) {
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(g * 32), v);
            const int m = 32 * (warp & 3) + lane;
            const int o = g * OPG + m / CINP, ci = m % CINP;
            if (o < KOFF && ci < cin && !first) {
                for (int co = 0; co < cout; ++co) outp[(o * cin + ci) * cout + co] = v[co];
            } else if (o < KOFF && ci < cin) {  // no brick: zero partial
                for (int co = 0; co < cout; ++co) outp[(o * cin + ci) * cout + co] = 0.f;
            }
        }
    }
    bred[warp][lane] = bsum;
    fence_before();
    __syncthreads();
    if (tid < cout) {
        float s = 0.f;
        for (int w = 0; w < 8; ++w) s += bred[w][tid];
        outp[nw + tid] = s;
    }
    if (abort && tid == 0) atomicExch(err, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G::TMEM_COLS) : "memory");
}

// fixed-order fold of per-block partials: out[i] = sum_b partial[b][i] (FP64 sum)
__global__ void k_fold(const float* partial, int nblk, int n, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += partial[(long)b * n + i];
    out[i] = (float)s;
}

// input features [S][16] bf16: Re psi, Im psi, V / v_scale, |psi|^2 - 1, zeros
__global__ void k_features(const float2* psi, const float* V, long S, float v_inv, __nv_bfloat16* X) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= S) return;
    const float2 p = psi[i];
    union {
        __nv_bfloat162 h[4];
        uint4 u;
    } w;
    w.h[0] = __floats2bfloat162_rn(p.x, p.y);
    w.h[1] = __floats2bfloat162_rn(V[i] * v_inv, p.x * p.x + p.y * p.y - 1.0f);
    w.h[2] = __floats2bfloat162_rn(0.f, 0.f);
    w.h[3] = w.h[2];
    uint4* dst = reinterpret_cast<uint4*>(X + i * 16);
    dst[0] = w.u;
    dst[1] = make_uint4(0u, 0u, 0u, 0u);
}

// target (psi_f - psi_c) / tau as [S][2]
__global__ void k_target(const float2* pf, const float2* pc, long S, float tau_inv, float* T) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= S) return;
    T[2 * i] = (pf[i].x - pc[i].x) * tau_inv;
    T[2 * i + 1] = (pf[i].y - pc[i].y) * tau_inv;
}

// MSE loss gradient: dY = 2 (Y - T) / (2 S); loss partials per block
__global__ void k_mse(const float* Y, const float* T, long n, float scale, float* dY, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = 2.0f * d * scale;
        s += (double)d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// dZ_prev = dA * gelu'(Z_prev): FP32 [S][c] and bf16 [S][CP] (padded) copies
__global__ void k_gelu_back(const float* dA, const float* Z, long S, int c, int CP, float* dZ, __nv_bfloat16* dZb) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= S * CP) return;
    const long s = i / CP;
    const int ch = (int)(i % CP);
    float v = 0.f;
    if (ch < c) {
        v = dA[s * c + ch] * gelu_grad(Z[s * c + ch]);
        dZ[s * c + ch] = v;
    }
    dZb[i] = __float2bfloat16(v);
}

// dY [S][2] FP32 -> bf16 [S][16] (the data-gradient conv input)
__global__ void k_pad16(const float* dY, long S, int c, __nv_bfloat16* out) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= S * 16) return;
    const long s = i / 16;
    const int ch = (int)(i % 16);
    out[i] = __float2bfloat16(ch < c ? dY[s * c + ch] : 0.f);
}

// psi += tau * Y
__global__ void k_apply(float2* psi, const float* Y, long S, float tau) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= S) return;
    float2 p = psi[i];
    p.x = fmaf(tau, Y[2 * i], p.x);
    p.y = fmaf(tau, Y[2 * i + 1], p.y);
    psi[i] = p;
}

// Adam on FP32 master parameters
__global__ void k_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float c1,
                       float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// master [27][cin][cout] -> forward tensor-core layout [27][COUTP][CINP+8] bf16
// (flip = 1: data-gradient layout [27][CINP_out = cin pad][COUTP_in + 8] with o -> 26 - o,
//  i.e. input channels are the layer's outputs, output channels its inputs)
__global__ void k_pack(const float* Wm, int cin, int cout, int kp_in, int np_out, int pitch, int flip, __nv_bfloat16* Wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int tot = KOFF * np_out * pitch;
    if (i >= tot) return;
    const int o = i / (np_out * pitch), n = (i / pitch) % np_out, k = i % pitch;
    float v = 0.f;
    if (!flip) {
        if (n < cout && k < cin) v = Wm[(o * cin + k) * cout + n];
    } else {
        const int of = KOFF - 1 - o;
        if (n < cin && k < cout) v = Wm[(of * cin + n) * cout + k];
    }
    (void)kp_in;
    Wt[i] = __float2bfloat16(v);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct DBuf {
    void* p = nullptr;
    size_t n = 0;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t bytes) {
        if (bytes <= n && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) throw std::bad_alloc();
        n = bytes;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct Layer {
    int cin, cout, cinp, coutp;
    std::vector<float> w, b;  // master (host mirror)
    DBuf dw, db, gw, gb, mw, vw, mb, vb;  // device master, grads, Adam moments
    DBuf fwd, bwd;                        // packed bf16
};

class Corrector {
  public:
    Corrector(int N, uint64_t seed) : N_(N) {
        if (N % 8 || N < 8) throw std::invalid_argument("corrector grids need N divisible by 8");
        S_ = (long)N * N * N;
        const int dims[3][4] = {{4, 32, 16, 32}, {32, 32, 32, 32}, {32, 2, 32, 8}};
        uint64_t st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
        auto urand = [&]() {  // PCG-style LCG stream in [0, 1)
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            return (double)(st >> 11) * (1.0 / 9007199254740992.0);
        };
        for (int l = 0; l < 3; ++l) {
            Layer& L = layers_[l];
            L.cin = dims[l][0];
            L.cout = dims[l][1];
            L.cinp = dims[l][2];
            L.coutp = dims[l][3];
            const int nw = KOFF * L.cin * L.cout;
            L.w.resize(nw);
            L.b.assign(L.cout, 0.f);
            const double a = std::sqrt(3.0 / (KOFF * L.cin)) * (l == 2 ? 0.1 : 1.0);  // uniform fan-in init
            for (auto& x : L.w) x = (float)(a * (2.0 * urand() - 1.0));
        }
        for (auto& L : layers_) {
            const int nw = KOFF * L.cin * L.cout;
            L.dw.alloc(4 * nw);
            L.db.alloc(4 * L.cout);
            L.gw.alloc(4 * nw);
            L.gb.alloc(4 * L.cout);
            for (DBuf* b : {&L.mw, &L.vw}) {
                b->alloc(4 * nw);
                NN_CUDA(cudaMemset(b->p, 0, 4 * nw));
            }
            for (DBuf* b : {&L.mb, &L.vb}) {
                b->alloc(4 * L.cout);
                NN_CUDA(cudaMemset(b->p, 0, 4 * L.cout));
            }
        }
        upload();  // creates the stream
        NN_CUDA(cudaFuncSetAttribute(k_conv<16, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ConvSmem<16, 32>::bytes()));
        NN_CUDA(cudaFuncSetAttribute(k_conv<32, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ConvSmem<32, 32>::bytes()));
        NN_CUDA(cudaFuncSetAttribute(k_conv<32, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ConvSmem<32, 8>::bytes()));
        NN_CUDA(cudaFuncSetAttribute(k_conv_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::Geo<32>::SMEM));
        NN_CUDA(cudaFuncSetAttribute(k_conv_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::Geo<16>::SMEM));
        errb_.alloc(sizeof(int));
        NN_CUDA(cudaMemset(errb_.p, 0, sizeof(int)));
        NN_CUDA(cudaFuncSetAttribute(k_wgrad<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wgrad_smem(16, 32)));
        NN_CUDA(cudaFuncSetAttribute(k_wgrad<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wgrad_smem(32, 32)));
        NN_CUDA(cudaFuncSetAttribute(k_wgrad_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)wtc::Geo<32>::SMEM));
        NN_CUDA(cudaFuncSetAttribute(k_wgrad_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)wtc::Geo<16>::SMEM));
    }
    ~Corrector() {
        if (st_) {
            cudaStreamSynchronize(st_);
            cudaStreamDestroy(st_);
        }
    }

    int N() const { return N_; }
    int nparams() const {
        int n = 0;
        for (auto& L : layers_) n += KOFF * L.cin * L.cout + L.cout;
        return n;
    }
    void set_scales(double v_scale, double tau) {
        if (!(v_scale > 0) || !(tau > 0)) throw std::invalid_argument("scales must be positive");
        v_scale_ = v_scale;
        tau_ = tau;
    }
    void get_scales(double* v_scale, double* tau) const {
        if (v_scale) *v_scale = v_scale_;
        if (tau) *tau = tau_;
    }

    // parameters in layer order: w1 [27][4][32], b1, w2, b2, w3 [27][32][2], b3
    void get_params(float* out) {
        download();
        for (auto& L : layers_) {
            std::memcpy(out, L.w.data(), 4 * L.w.size());
            out += L.w.size();
            std::memcpy(out, L.b.data(), 4 * L.b.size());
            out += L.b.size();
        }
    }
    void set_params(const float* in) {
        for (auto& L : layers_) {
            std::memcpy(L.w.data(), in, 4 * L.w.size());
            in += L.w.size();
            std::memcpy(L.b.data(), in, 4 * L.b.size());
            in += L.b.size();
        }
        upload();
    }
    void get_grads(float* out) {
        NN_CUDA(cudaStreamSynchronize(st_));
        for (auto& L : layers_) {
            const int nw = KOFF * L.cin * L.cout;
            NN_CUDA(cudaMemcpy(out, L.gw.p, 4 * nw, cudaMemcpyDeviceToHost));
            out += nw;
            NN_CUDA(cudaMemcpy(out, L.gb.p, 4 * L.cout, cudaMemcpyDeviceToHost));
            out += L.cout;
        }
    }

    // forward on (psi, V) of this grid; Y = net output [S][2] (device, owned)
    void forward(const float2* psi, const float* V, bool keep) {
        alloc_acts(keep);
        const long S = S_;
        k_features<<<(unsigned)((S + 255) / 256), 256, 0, st_>>>(psi, V, S, (float)(1.0 / v_scale_), X0_.as<__nv_bfloat16>());
        conv<16, 32>(X0_.as<__nv_bfloat16>(), layers_[0], keep ? Z1_.as<float>() : nullptr, A1_.as<__nv_bfloat16>(),
                     nullptr, true);
        conv<32, 32>(A1_.as<__nv_bfloat16>(), layers_[1], keep ? Z2_.as<float>() : nullptr, A2_.as<__nv_bfloat16>(),
                     nullptr, true);
        conv<32, 8>(A2_.as<__nv_bfloat16>(), layers_[2], nullptr, nullptr, Y_.as<float>(), false);
        NN_CUDA(cudaGetLastError());
    }

    // loss and gradients of one pair (coarse state, fine result); no update
    double gradients(const float2* psi_c, const float* V_c, const float2* psi_f) {
        const long S = S_;
        forward(psi_c, V_c, true);
        T_.alloc(sizeof(float) * 2 * S);
        dY_.alloc(sizeof(float) * 2 * S);
        k_target<<<(unsigned)((S + 255) / 256), 256, 0, st_>>>(psi_f, psi_c, S, (float)(1.0 / tau_), T_.as<float>());
        const int nb = 592;
        lossp_.alloc(sizeof(double) * nb);
        k_mse<<<nb, 256, 0, st_>>>(Y_.as<float>(), T_.as<float>(), 2 * S, (float)(1.0 / (2.0 * S)), dY_.as<float>(),
                                   lossp_.as<double>());
        // layer 3: dZ3 = dY (linear)
        wgrad<32>(A2_.as<__nv_bfloat16>(), dY_.as<float>(), layers_[2]);
        dYb_.alloc(sizeof(__nv_bfloat16) * 16 * S);
        k_pad16<<<(unsigned)((S * 16 + 255) / 256), 256, 0, st_>>>(dY_.as<float>(), S, 2, dYb_.as<__nv_bfloat16>());
        dA_.alloc(sizeof(float) * 32 * S);
        conv_bwd<16, 32>(dYb_.as<__nv_bfloat16>(), layers_[2], dA_.as<float>());  // dA2 = conv^T(dZ3)
        dZ_.alloc(sizeof(float) * 32 * S);
        dZb_.alloc(sizeof(__nv_bfloat16) * 32 * S);
        k_gelu_back<<<(unsigned)((S * 32 + 255) / 256), 256, 0, st_>>>(dA_.as<float>(), Z2_.as<float>(), S, 32, 32,
                                                                         dZ_.as<float>(), dZb_.as<__nv_bfloat16>());
        wgrad<32>(A1_.as<__nv_bfloat16>(), dZ_.as<float>(), layers_[1]);
        conv_bwd<32, 32>(dZb_.as<__nv_bfloat16>(), layers_[1], dA_.as<float>());  // dA1 = conv^T(dZ2)
        k_gelu_back<<<(unsigned)((S * 32 + 255) / 256), 256, 0, st_>>>(dA_.as<float>(), Z1_.as<float>(), S, 32, 32,
                                                                         dZ_.as<float>(), dZb_.as<__nv_bfloat16>());
        wgrad<16>(X0_.as<__nv_bfloat16>(), dZ_.as<float>(), layers_[0]);
        NN_CUDA(cudaGetLastError());
        std::vector<double> lp(nb);
        NN_CUDA(cudaMemcpyAsync(lp.data(), lossp_.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st_));
        NN_CUDA(cudaStreamSynchronize(st_));
        check_err();
        double loss = 0.0;
        for (double x : lp) loss += x;
        return loss / (2.0 * S);
    }

    double train_pair(const float2* psi_c, const float* V_c, const float2* psi_f, double lr) {
        const double loss = gradients(psi_c, V_c, psi_f);
        ++t_;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)t_), c2 = 1.f - std::pow(b2, (float)t_);
        for (auto& L : layers_) {
            const int nw = KOFF * L.cin * L.cout;
            k_adam<<<(nw + 255) / 256, 256, 0, st_>>>(L.dw.as<float>(), L.gw.as<float>(), L.mw.as<float>(),
                                                      L.vw.as<float>(), nw, (float)lr, b1, b2, c1, c2, 1e-8f);
            k_adam<<<1, 256, 0, st_>>>(L.db.as<float>(), L.gb.as<float>(), L.mb.as<float>(), L.vb.as<float>(), L.cout,
                                       (float)lr, b1, b2, c1, c2, 1e-8f);
        }
        pack_all();
        NN_CUDA(cudaStreamSynchronize(st_));
        return loss;
    }

    // psi += tau * net(psi, V) on `stream` (the field's stream)
    void apply(float2* psi, const float* V, cudaStream_t stream) {
        cudaEvent_t ev;
        NN_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        NN_CUDA(cudaEventRecord(ev, stream));
        NN_CUDA(cudaStreamWaitEvent(st_, ev, 0));
        forward(psi, V, false);
        k_apply<<<(unsigned)((S_ + 255) / 256), 256, 0, st_>>>(psi, Y_.as<float>(), S_, (float)tau_);
        NN_CUDA(cudaEventRecord(ev, st_));
        NN_CUDA(cudaStreamWaitEvent(stream, ev, 0));
        NN_CUDA(cudaEventDestroy(ev));
        NN_CUDA(cudaGetLastError());
    }
    void output(float* host) {
        NN_CUDA(cudaStreamSynchronize(st_));
        check_err();
        NN_CUDA(cudaMemcpy(host, Y_.p, sizeof(float) * 2 * S_, cudaMemcpyDeviceToHost));
    }
    void sync() {
        NN_CUDA(cudaStreamSynchronize(st_));
        check_err();
    }
    // 1: 32-output convolutions and the weight gradients on the tcgen05 kernels
    // (default), 0: convolutions on mma.sync, weight gradients on CUDA cores
    void set_tensor_path(int tc) { use_tc_ = tc != 0; }
    void check_err() {
        int e = 0;
        NN_CUDA(cudaMemcpy(&e, errb_.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) throw std::runtime_error("corrector: a tensor-core wait timed out");
    }

  private:
    static size_t wgrad_smem(int cinp, int cout) { return sizeof(float) * ((size_t)HALO * cinp + (size_t)BSITES * cout); }

    void alloc_acts(bool keep) {
        const long S = S_;
        X0_.alloc(sizeof(__nv_bfloat16) * 16 * S);
        A1_.alloc(sizeof(__nv_bfloat16) * 32 * S);
        A2_.alloc(sizeof(__nv_bfloat16) * 32 * S);
        Y_.alloc(sizeof(float) * 2 * S);
        if (keep) {
            Z1_.alloc(sizeof(float) * 32 * S);
            Z2_.alloc(sizeof(float) * 32 * S);
        }
    }
    // CIN -> 32 layers on the tcgen05 kernel (grids N % 16 == 0), the others on mma.sync
    bool tc_ok() const { return use_tc_ && N_ % tc::BY == 0; }
    template <int CIN>
    void conv_tc(const __nv_bfloat16* X, const __nv_bfloat16* W, const float* bias, int cout, float* zf,
                 __nv_bfloat16* ab, float* out2, bool gelu_ab) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // two blocks per SM (the kernel's launch bounds; the shared-memory carve-out is
        // set at launch), so one block's MMAs overlap the other's halo loads and epilogue
        const long nbricks = S_ / (tc::BX * tc::BY * tc::BZ);
        const unsigned blocks = (unsigned)std::min<long>(nbricks, 2L * sms);
        k_conv_tc<CIN><<<blocks, 256, tc::Geo<CIN>::SMEM, st_>>>(X, W, bias, N_, cout, zf, ab, out2, gelu_ab ? 1 : 0,
                                                                 errb_.as<int>());
    }
    template <int CINP, int COUTP>
    void conv(const __nv_bfloat16* X, Layer& L, float* zf, __nv_bfloat16* ab, float* out2, bool gelu_ab) {
        if constexpr ((CINP == 32 || CINP == 16) && COUTP == 32) {
            if (tc_ok()) {
                conv_tc<CINP>(X, L.fwd.as<__nv_bfloat16>(), L.db.as<float>(), L.cout, zf, ab, out2, gelu_ab);
                return;
            }
        }
        const unsigned blocks = (unsigned)(S_ / BSITES);
        k_conv<CINP, COUTP><<<blocks, 256, ConvSmem<CINP, COUTP>::bytes(), st_>>>(
            X, L.fwd.as<__nv_bfloat16>(), L.db.as<float>(), N_, L.cout, zf, ab, out2, gelu_ab ? 1 : 0);
    }
    // data gradient: input channels = the layer's outputs (padded to CINP), outputs = its inputs
    template <int CINP, int COUTP>
    void conv_bwd(const __nv_bfloat16* dZb, Layer& L, float* dA) {
        if constexpr ((CINP == 32 || CINP == 16) && COUTP == 32) {
            if (tc_ok()) {
                conv_tc<CINP>(dZb, L.bwd.as<__nv_bfloat16>(), nullptr, L.cin, dA, nullptr, nullptr, false);
                return;
            }
        }
        const unsigned blocks = (unsigned)(S_ / BSITES);
        k_conv<CINP, COUTP><<<blocks, 256, ConvSmem<CINP, COUTP>::bytes(), st_>>>(
            dZb, L.bwd.as<__nv_bfloat16>(), nullptr, N_, L.cin, dA, nullptr, nullptr, 0);
    }
    template <int CINP>
    void wgrad(const __nv_bfloat16* A, const float* dZ, Layer& L) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int nbricks = (int)(S_ / BSITES);
        const int nw = KOFF * L.cin * L.cout;
        // tensor cores (one block per SM, shared memory for two operand buffers),
        // or the CUDA-core sums (set_tensor_path(0))
        const int nblk = use_tc_ ? std::min(nbricks, sms) : std::min(nbricks, 2 * sms);
        part_.alloc(sizeof(float) * (size_t)nblk * (nw + L.cout));
        if (use_tc_)
            k_wgrad_tc<CINP><<<nblk, 256, wtc::Geo<CINP>::SMEM, st_>>>(A, dZ, N_, L.cin, L.cout, part_.as<float>(),
                                                                       errb_.as<int>());
        else
            k_wgrad<CINP><<<nblk, 256, wgrad_smem(CINP, L.cout), st_>>>(A, dZ, N_, L.cin, L.cout, part_.as<float>());
        fold_.alloc(sizeof(float) * (nw + L.cout));
        k_fold<<<(nw + L.cout + 255) / 256, 256, 0, st_>>>(part_.as<float>(), nblk, nw + L.cout, fold_.as<float>());
        NN_CUDA(cudaMemcpyAsync(L.gw.p, fold_.p, sizeof(float) * nw, cudaMemcpyDeviceToDevice, st_));
        NN_CUDA(cudaMemcpyAsync(L.gb.p, fold_.as<float>() + nw, sizeof(float) * L.cout, cudaMemcpyDeviceToDevice, st_));
    }
    void pack_all() {
        for (auto& L : layers_) {
            const int fpitch = L.cinp + 8;
            const int ftot = KOFF * L.coutp * fpitch;
            L.fwd.alloc(2 * ftot);
            k_pack<<<(ftot + 255) / 256, 256, 0, st_>>>(L.dw.as<float>(), L.cin, L.cout, L.cinp, L.coutp, fpitch, 0,
                                                         L.fwd.as<__nv_bfloat16>());
            // data gradient: K = layer outputs padded (16 for 2 outputs, else coutp), N = layer inputs (32)
            const int kin = L.cout <= 16 ? 16 : L.coutp;
            const int bpitch = kin + 8;
            const int btot = KOFF * 32 * bpitch;
            L.bwd.alloc(2 * btot);
            k_pack<<<(btot + 255) / 256, 256, 0, st_>>>(L.dw.as<float>(), L.cin, L.cout, kin, 32, bpitch, 1,
                                                         L.bwd.as<__nv_bfloat16>());
        }
    }
    void upload() {
        for (auto& L : layers_) {
            NN_CUDA(cudaMemcpy(L.dw.p, L.w.data(), 4 * L.w.size(), cudaMemcpyHostToDevice));
            NN_CUDA(cudaMemcpy(L.db.p, L.b.data(), 4 * L.b.size(), cudaMemcpyHostToDevice));
        }
        if (!st_) NN_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
        pack_all();
        NN_CUDA(cudaStreamSynchronize(st_));
    }
    void download() {
        NN_CUDA(cudaStreamSynchronize(st_));
        for (auto& L : layers_) {
            NN_CUDA(cudaMemcpy(L.w.data(), L.dw.p, 4 * L.w.size(), cudaMemcpyDeviceToHost));
            NN_CUDA(cudaMemcpy(L.b.data(), L.db.p, 4 * L.b.size(), cudaMemcpyDeviceToHost));
        }
    }

    int N_;
    long S_;
    cudaStream_t st_ = nullptr;
    Layer layers_[3];
    double v_scale_ = 1.0, tau_ = 1.0;
    long t_ = 0;
    DBuf X0_, A1_, A2_, Z1_, Z2_, Y_, T_, dY_, dYb_, dA_, dZ_, dZb_, lossp_, part_, fold_;
    DBuf errb_;           // device flag: a bounded wait of the tcgen05 kernel timed out
    bool use_tc_ = true;
};

}  // namespace nn
}  // namespace qx

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

struct qx_corr_s {
    std::unique_ptr<qx::nn::Corrector> c;
    std::string err;
};

namespace {
thread_local std::string g_corr_err;

template <typename F>
int corr_guarded(qx_corr_t* h, F&& fn) {
    if (!h || !h->c) {
        g_corr_err = "null qx_corr handle";
        return QX_ERR_INVALID;
    }
    try {
        fn(*h->c);
        h->err.clear();
        return QX_OK;
    } catch (const std::invalid_argument& e) {
        h->err = e.what();
        return QX_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        h->err = "device allocation failed";
        return QX_ERR_NOMEM;
    } catch (const std::exception& e) {
        h->err = e.what();
        return QX_ERR_CUDA;
    } catch (...) {
        h->err = "unknown error";
        return QX_ERR_INTERNAL;
    }
}
}  // namespace

extern "C" {

int qx_corr_create(int N, unsigned long long seed, qx_corr_t** out) {
    if (!out) {
        g_corr_err = "out must not be NULL";
        return QX_ERR_INVALID;
    }
    *out = nullptr;
    try {
        auto h = new qx_corr_s();
        try {
            h->c = std::make_unique<qx::nn::Corrector>(N, seed);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return QX_OK;
    } catch (const std::invalid_argument& e) {
        g_corr_err = e.what();
        return QX_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        g_corr_err = "device allocation failed";
        return QX_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_corr_err = e.what();
        return QX_ERR_CUDA;
    }
}

int qx_corr_destroy(qx_corr_t* h) {
    if (!h) return QX_OK;
    try {
        h->c.reset();
    } catch (...) {
    }
    delete h;
    return QX_OK;
}

const char* qx_corr_last_error(const qx_corr_t* h) {
    if (h && !h->err.empty()) return h->err.c_str();
    return g_corr_err.c_str();
}

int qx_corr_nparams(qx_corr_t* h, int* n) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) { *n = c.nparams(); });
}

int qx_corr_set_tensor_path(qx_corr_t* h, int tc) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) { c.set_tensor_path(tc); });
}

int qx_corr_set_scales(qx_corr_t* h, double v_scale, double tau) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) { c.set_scales(v_scale, tau); });
}

int qx_corr_get_scales(qx_corr_t* h, double* v_scale, double* tau) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) { c.get_scales(v_scale, tau); });
}

int qx_corr_get_params(qx_corr_t* h, float* p) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) {
        if (!p) throw std::invalid_argument("params must not be NULL");
        c.get_params(p);
    });
}

int qx_corr_set_params(qx_corr_t* h, const float* p) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) {
        if (!p) throw std::invalid_argument("params must not be NULL");
        c.set_params(p);
    });
}

int qx_corr_gradients(qx_corr_t* h, const void* psi_c, const void* V_c, const void* psi_f, float* grads,
                      double* loss) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) {
        if (!psi_c || !V_c || !psi_f) throw std::invalid_argument("state pointers must not be NULL");
        const double l = c.gradients(static_cast<const float2*>(psi_c), static_cast<const float*>(V_c),
                                     static_cast<const float2*>(psi_f));
        if (grads) c.get_grads(grads);
        if (loss) *loss = l;
    });
}

int qx_corr_train_pair(qx_corr_t* h, const void* psi_c, const void* V_c, const void* psi_f, double lr, double* loss) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) {
        if (!psi_c || !V_c || !psi_f) throw std::invalid_argument("state pointers must not be NULL");
        const double l = c.train_pair(static_cast<const float2*>(psi_c), static_cast<const float*>(V_c),
                                      static_cast<const float2*>(psi_f), lr);
        if (loss) *loss = l;
    });
}

int qx_corr_apply(qx_corr_t* h, void* psi, const void* V, void* stream) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) {
        if (!psi || !V) throw std::invalid_argument("state pointers must not be NULL");
        c.apply(static_cast<float2*>(psi), static_cast<const float*>(V), static_cast<cudaStream_t>(stream));
    });
}

int qx_corr_output(qx_corr_t* h, float* out) {
    return corr_guarded(h, [&](qx::nn::Corrector& c) {
        if (!out) throw std::invalid_argument("out must not be NULL");
        c.output(out);
    });
}

}  // extern "C"
