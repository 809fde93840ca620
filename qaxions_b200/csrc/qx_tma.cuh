// qx_tma.cuh -- TMA-fed persistent pencil passes (sm_100a).
//
// A strided pass streams tiles of TX columns x N pencil positions through a
// ring of NBUF shared-memory buffers.  One elected thread moves every tile with
// the Tensor Memory Accelerator: a tensor load (cp.async.bulk.tensor, completion
// counted on one mbarrier per buffer) brings the tile in, all threads run the
// pencil FFT in place in the tile, and a tensor store (bulk group) writes the
// finished tile back from the same buffer.  The buffer of tile k-1 is refilled
// with tile k+NBUF-1 once its store has been read out, so loads, the FFT and
// stores of neighbouring tiles overlap and the threads issue no global
// loads/stores of their own.
//
// Twiddles (and, for the drift pass, the z-dependent phase factors) are staged
// in shared memory once per launch.  The drift phase exp(-i dt/2 dk^2 |n|^2)/S
// is factored exactly as A(nx, ny) * B(nz); both factors are evaluated in FP64
// with the argument reduced mod 2 pi, multiplied in FP64 and rounded once.
// Both come from per-grid tables (drift_tables, computed once per time step
// size); B is staged in shared memory once per launch.
//
// Every mbarrier wait is bounded (~1 s of SM clock); on time-out the kernel
// sets *err, waits (bounded) for its own loads still in flight and for its
// stores, and returns.  No clusters, no multicast: a block only loads what it
// transforms.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

#include "qx_kernels.cuh"
#include "qx_ops.hpp"

namespace qx {

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: gives up after `limit` SM cycles (default 2^31, ~1 s)
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit = (1LL << 31)) {
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* tm, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* tm, int c0, int c1, int c2, uint32_t src) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
        ::"l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(src)
        : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// wait until at most one bulk group still reads its shared-memory source
__device__ __forceinline__ void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------------------
// persistent TMA pencil pass
// ---------------------------------------------------------------------------

// Pencils per thread of a strided pass: PW = 2 (FP32 only) gives every thread
// two adjacent columns, transformed together as CPair values, so each shared-
// memory access moves 16 bytes and each twiddle is loaded once for both.
template <int PW, typename C> using pencil_val_t = typename std::conditional<PW == 2, CPair<C>, C>::type;

// elements per thread (per pencil) of a strided pass
template <int N, typename R, int PW> __host__ __device__ constexpr int tma_e() {
    return PW == 2 ? qx_lcm_radices(N) : ((N >= 256 && sizeof(R) == 4) ? 16 : qx_lcm_radices(N));
}
// launch bounds: one-pencil blocks take up to 512 threads (one per SM), paired
// blocks up to 256 threads with two blocks per SM
template <int PW> __host__ __device__ constexpr int tma_max_threads() { return PW == 2 ? 256 : 512; }
template <int PW> __host__ __device__ constexpr int tma_min_blocks() { return PW == 2 ? 2 : 1; }
// Tile columns TXF: 8 or 16, fixed at compile time so shared-memory addresses
// fold to constants (0: chosen at run time, grids N < 16).  Rows of a tile
// are TXF * sizeof(complex) bytes of one HBM row; at the 2 MB stride of a z
// pencil, 128-byte rows (FP32 TXF = 16, FP64 TXF = 8) stream at nearly the
// rate of contiguous copies, 64-byte rows at about half of it.
template <int N, typename R, int PW, int TXF> __host__ __device__ constexpr int tma_block_threads() {
    return TXF > 0 ? (TXF / PW) * (N / tma_e<N, R, PW>()) : tma_max_threads<PW>();
}
template <int N, typename R, int PW, int TXF> __host__ __device__ constexpr int tma_block_min() {
    return TXF > 0 ? (tma_block_threads<N, R, PW, TXF>() <= 256 ? 2 : 1) : tma_min_blocks<PW>();
}

__host__ __device__ constexpr size_t align1k(size_t b) { return (b + 1023) & ~(size_t)1023; }

// widest tile (columns) of a strided pass: the drift pass keeps one A(nx, ny)
// slot of this many double2 per ring buffer
constexpr int kTmaMaxTX = 16;

// dynamic shared memory of a pass: NBUF tiles + twiddles + drift factors
// (drift only) + column-0 stash (Poisson only) + 128-byte base-alignment slack (the
// tensor-copy alignment of unswizzled tiles; tiles are 1 KB multiples)
template <typename R> __host__ __device__ constexpr size_t tma_smem_bytes(int N, int TX, int nbuf, int op,
                                                                          bool swz = false) {
    return (size_t)nbuf * align1k((size_t)N * TX * 2 * sizeof(R)) + (size_t)N * 4 * sizeof(R) +
           (op == OP_DRIFT ? (size_t)N * 16 + (size_t)nbuf * kTmaMaxTX * 16 : 0) +
           (op == OP_POISSON ? (size_t)N * 2 * sizeof(R) : 0) + (swz ? 1024 : 128);
}

template <typename R> struct TArgs {
    const cx_t<R>* tw;   // exp(-2 pi i j/N), global
    const cx_t<R>* tw_lo;  // exact - tw (FP32 double-float twiddles), global
    int X;               // columns (N for psi, N/2 for the packed half spectrum)
    int N;
    int outer;           // tiles along the non-pencil axis (z planes for y passes, box * N + y for
                         // 3D z passes, boxes in 2D; batched arrays stack boxes along z)
    int pencil_dim;      // 1: pencil along tensor dim 1 (y passes, 2D last axis); 2: along dim 2 (3D z)
    int la3d;            // last-axis pass of a 3D array (pencil = z, outer = y)
    int TX, tiles_x, nbuf, nbox, box;
    long n_tiles;
    double phase_fac, scale, pois_c, pois_g0;
    int col0_external;   // 3D Poisson: column 0 is finished by k_poisson_col0
    const double2* axy;  // drift: A(nx, ny) table [y][x] (x < N; y < N in 3D), then B(nz) / S
    double* partial;     // OP_KIN per-block sums
    int* err;            // set to 1 when a wait timed out
};

// 128-byte-row tiles of paired pencils (FP32, TX = 16, PW = 2): the tile is
// stored with TMA's 128-byte swizzle (16-byte chunk index XOR row mod 8), so
// the 16-byte pencil-pair accesses of a warp stay bank-conflict free, and the
// block runs as two groups of 8 warps that synchronise their FFT exchanges
// with named barriers (a group owns 4 of the 8 pencil pairs of every row).
template <int N, typename R, int PW, int TXF> __host__ __device__ constexpr bool tma_swizzled() {
    return sizeof(R) == 4 && PW == 2 && TXF == 16;
}

__device__ __forceinline__ void named_barrier(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// pencil group c of a tile: element p at base[p * pitch + c] (plain) or at
// base[p * 8 + (c ^ (p & 7))] (swizzled 128-byte rows of 8 pairs)
template <typename P, bool SWZ> struct TileAcc {
    P* base;
    int c, pitch;
    __device__ __forceinline__ P& operator()(int p) const {
        if constexpr (SWZ) return base[p * 8 + (c ^ (p & 7))];
        else return base[p * pitch + c];
    }
    __device__ __forceinline__ void sync() const {
        if constexpr (SWZ) named_barrier(1 + (int)threadIdx.z, (int)(blockDim.x * blockDim.y));
        else __syncthreads();
    }
};

// blockDim = (TX / PW, N / E, 1), or (TX / PW / 2, N / E, 2) when swizzled:
// thread (c, t) owns columns x0 + PW c + h (h < PW), c = x + blockDim.x z;
// TX = TXF when TXF > 0
// PLAN: radix plan of the pencil transforms (qx_with_plan); the twiddle tables
// passed in TArgs are the stage-major tables of that plan.
template <int N, typename R, int OP, int PW, bool DF, int TXF, int PLAN = 0>
__global__ void __launch_bounds__((tma_block_threads<N, R, PW, TXF>()), (tma_block_min<N, R, PW, TXF>()))
    k_pencil_tma(const __grid_constant__ CUtensorMap tm, TArgs<R> s) {
    using C = cx_t<R>;
    using P = pencil_val_t<PW, C>;
    static_assert(PW == 1 || sizeof(R) == 4, "paired pencils are an FP32 layout");
    constexpr int NL = qx_with_plan(N, PLAN);
    constexpr int E = tma_e<N, R, PW>();
    static_assert(qx_lcm_radices(NL) == qx_lcm_radices(N), "a plan keeps the elements per thread");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar[8];
    __shared__ int s_abort;
    __shared__ double red[32];
    const int TX = TXF > 0 ? TXF : s.TX;
    constexpr bool SWZ = tma_swizzled<N, R, PW, TXF>();
    const int TG = TX / PW;  // pencil groups per tile row
    const int c = threadIdx.x + blockDim.x * threadIdx.z, t = threadIdx.y;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const uint32_t tile_bytes = (uint32_t)((size_t)N * TX * sizeof(C));
    const long tile_elems = (long)(align1k(tile_bytes) / sizeof(C));
    // tiles on 128-byte boundaries, 1024 for the 128-byte swizzle
    constexpr uintptr_t BA = SWZ ? 1023 : 127;
    C* bufs = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smem_raw) + BA) & ~BA);
    C* tws = bufs + s.nbuf * tile_elems;
    C* tws_lo = tws + N;
    double2* bz = reinterpret_cast<double2*>(tws_lo + N);
    double2* aslot = bz + N;  // drift: A(nx, ny) of each ring buffer's tile columns
    C* col0 = reinterpret_cast<C*>(bz + (OP == OP_DRIFT ? N + s.nbuf * kTmaMaxTX : 0));
    // drift: address of A(nx, ny) of column j of tile `id` in the per-grid table
    auto a_of_tile = [&](long id, int j) {
        const int ox = (int)(id / s.tiles_x);
        return s.axy + (s.la3d ? (long)(ox % N) * N : 0L) + (id % s.tiles_x) * TX + j;
    };

    auto coords = [&](long id, int j, int& c0, int& c1, int& c2) {
        const int x0 = (int)(id % s.tiles_x) * TX;
        const int o = (int)(id / s.tiles_x);
        c0 = 2 * x0;
        if (s.pencil_dim == 1) { c1 = j * s.box; c2 = o; }
        else { c1 = o % N; c2 = (o / N) * N + j * s.box; }  // o = box * N + y
    };
    auto issue_load = [&](long id, int b) {
        const uint32_t bar = smem_u32(&mbar[b]);
        mbar_expect_tx(bar, tile_bytes);
        for (int j = 0; j < s.nbox; ++j) {
            int c0, c1, c2;
            coords(id, j, c0, c1, c2);
            tma_load_3d(smem_u32(bufs + b * tile_elems + (long)j * s.box * TX), &tm, c0, c1, c2, bar);
        }
    };

    // per-launch tables and barriers
    for (int i = tid; i < N; i += nthr) {
        tws[i] = s.tw[i];
        if constexpr (DF) tws_lo[i] = s.tw_lo[i];
    }
    if constexpr (OP == OP_DRIFT) {
        const double2* gbz = s.axy + (s.la3d ? (long)N * N : (long)N);
        for (int i = tid; i < N; i += nthr) bz[i] = gbz[i];
        if (blockIdx.x < s.n_tiles)
            for (int j = tid; j < TX; j += nthr) aslot[j] = *a_of_tile(blockIdx.x, j);
    }
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < s.nbuf; ++b) mbar_init(smem_u32(&mbar[b]), 1);
        fence_mbar_init();
        for (int k = 0; k < s.nbuf - 1; ++k) {
            const long id = blockIdx.x + (long)k * gridDim.x;
            if (id < s.n_tiles) issue_load(id, k);
        }
    }
    __syncthreads();

    double kin = 0.0;
    int k = 0;
    for (;; ++k) {
        const long id = blockIdx.x + (long)k * gridDim.x;
        if (id >= s.n_tiles) break;
        const int b = k % s.nbuf;
        const uint32_t parity = (uint32_t)((k / s.nbuf) & 1);
        // every thread waits for (and acquires) the tile itself; a time-out is
        // recorded and acted on at the tile's last barrier, where all threads
        // read the same flag
        if (!mbar_wait_bounded(smem_u32(&mbar[b]), parity)) s_abort = 1;
        C* tile = bufs + b * tile_elems;
        const int x0 = (int)(id % s.tiles_x) * TX;
        const int o = (int)(id / s.tiles_x);
        const int xb = x0 + PW * c;  // column of pencil 0 of this thread
        TileAcc<P, SWZ> acc{reinterpret_cast<P*>(tile), c, TG};
        // drift: the next tile's A(nx, ny) is copied into its ring slot now
        // (asynchronously, no registers held) and waited for before this
        // tile's store barrier, so its latency stays hidden
        const long id_next = id + gridDim.x;
        const bool a_copy = OP == OP_DRIFT && tid < TX && id_next < s.n_tiles;
        if (a_copy) {  // (a block of fewer than TX threads copies several columns each)
            for (int j = tid; j < TX; j += nthr)
                cp_async16(&aslot[((k + 1) % s.nbuf) * kTmaMaxTX + j], a_of_tile(id_next, j));
            cp_async_commit();
        }
        P v[E];
        if constexpr (OP == OP_INV) {
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = acc(out_pos<NL, E>(e, t));
            ifft_pencil_rev<NL, E>(v, acc, t, tw_src<DF>(tws, tws_lo));
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = acc(in_pos<NL, E, 0>(e, t));
            fft_pencil<NL, E, -1>(v, acc, t, tw_src<DF>(tws, tws_lo));
        }

        // |n|^2 contribution of x (and y in 3D) of pencil h
        auto mxy_of = [&](int h) {
            const int x = xb + h;
            const int nx = (s.X == N) ? signed_mode(x, N) : x;
            const int ny = s.la3d ? signed_mode(o % N, N) : 0;
            return (long)nx * nx + (long)ny * ny;
        };
        bool store = true;
        if constexpr (OP == OP_KIN) {
#pragma unroll
            for (int h = 0; h < PW; ++h) {
                const long mxy = mxy_of(h);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int nz = signed_mode(out_pos<NL, E>(e, t), N);
                    const C u = pen(v[e], h);
                    kin += (double)(mxy + (long)nz * nz) * ((double)u.x * (double)u.x + (double)u.y * (double)u.y);
                }
            }
            store = false;
        } else if constexpr (OP == OP_DRIFT || OP == OP_POISSON) {
            // column 0 of the tile row (pencil 0 of thread group 0)
            const bool has_col0 = x0 == 0 && c == 0;
            const bool c0ext = (OP == OP_POISSON) && s.col0_external && has_col0;
            if constexpr (OP == OP_DRIFT) {
                // A(nx, ny) of the thread's columns from the tile's ring slot
                // (staged before the previous tile's store barrier; a multi-stage
                // forward transform has synchronised the block since)
                if constexpr (qx_nstages(NL) == 1) __syncthreads();
#pragma unroll
                for (int h = 0; h < PW; ++h) {
                    const double2 A = aslot[b * kTmaMaxTX + PW * c + h];
#pragma unroll
                    for (int e = 0; e < E; ++e)
                        pen(v[e], h) = cmul_d(pen(v[e], h), dcmul(A, bz[out_pos<NL, E>(e, t)]));
                }
            } else {
                SArgs<R> sa;
                sa.pois_c = s.pois_c;
                sa.pois_g0 = s.pois_g0;
                if (c0ext) {
                    // 3D: column 0 (kx = 0 and N/2 packed) is paired with its mirror
                    // row by k_poisson_col0; keep the forward result for it
#pragma unroll
                    for (int e = 0; e < E; ++e) col0[out_pos<NL, E>(e, t)] = pen(v[e], 0);
                } else if (x0 == 0 && !s.col0_external) {
                    // 2D: the mirror -k_y of column 0 lies in the same pencil
                    __syncthreads();
#pragma unroll
                    for (int e = 0; e < E; ++e) acc(out_pos<NL, E>(e, t)) = v[e];
                    __syncthreads();
                    if (c == 0) {
#pragma unroll
                        for (int e = 0; e < E; ++e) {
                            const int p = out_pos<NL, E>(e, t);
                            const long np = signed_mode(p, N);
                            const long mA = np * np, mB = mA + (long)(N / 2) * (N / 2);
                            const R gA = pois_mult<R>(mA, sa), gB = pois_mult<R>(mB, sa);
                            const C cm = cconj(pen(acc((N - p) % N), 0));
                            pen(v[e], 0) = cadd(cscale(pen(v[e], 0), R(0.5) * (gA + gB)), cscale(cm, R(0.5) * (gA - gB)));
                        }
                    }
                }
#pragma unroll
                for (int h = 0; h < PW; ++h) {
                    if (h == 0 && has_col0) continue;
                    const long mxy = mxy_of(h);
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int nz = signed_mode(out_pos<NL, E>(e, t), N);
                        pen(v[e], h) = cscale(pen(v[e], h), pois_mult<R>(mxy + (long)nz * nz, sa));
                    }
                }
            }
            // inverse transform: the forward stages undone in reverse order,
            // from the forward output order back to the load order
            ifft_pencil_rev<NL, E>(v, acc, t, tw_src<DF>(tws, tws_lo));
            if (OP == OP_POISSON && s.col0_external && x0 == 0) {
                // the stash was written in another order by other threads; a
                // multi-stage inverse already synchronised the block
                if constexpr (qx_nstages(NL) == 1) __syncthreads();
                if (c0ext) {
#pragma unroll
                    for (int e = 0; e < E; ++e) pen(v[e], 0) = col0[in_pos<NL, E, 0>(e, t)];
                }
            }
        }

        if (a_copy) cp_async_wait_all();
        if (store) {
            // finished tile -> buffer (natural order) -> tensor store
            __syncthreads();
            if constexpr (OP == OP_FWD) {
#pragma unroll
                for (int e = 0; e < E; ++e) acc(out_pos<NL, E>(e, t)) = v[e];
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) acc(in_pos<NL, E, 0>(e, t)) = v[e];
            }
            fence_proxy_async();
            __syncthreads();
            if (s_abort) break;
            if (tid == 0) {
                for (int j = 0; j < s.nbox; ++j) {
                    int c0, c1, c2;
                    coords(id, j, c0, c1, c2);
                    tma_store_3d(&tm, c0, c1, c2, smem_u32(tile + (long)j * s.box * TX));
                }
                bulk_commit();
            }
        } else {
            __syncthreads();
            if (s_abort) break;
        }
        // refill the buffer of tile k-1 (its store has been read out) with tile k+NBUF-1
        if (tid == 0) {
            const long nid = id + (long)(s.nbuf - 1) * gridDim.x;
            if (nid < s.n_tiles) {
                bulk_wait_read_1();
                fence_proxy_async();
                issue_load(nid, (k + s.nbuf - 1) % s.nbuf);
            }
        }
    }
    if (s_abort) {
        // a tile did not arrive in time: flag it, wait (bounded) for this
        // block's loads still in flight and for its stores, and leave
        if (tid == 0) {
            atomicExch(s.err, 1);
            for (int j = 0; j < s.nbuf - 1; ++j) {  // tiles k .. k+NBUF-2 were requested
                const long jd = blockIdx.x + (long)(k + j) * gridDim.x;
                if (jd < s.n_tiles)
                    mbar_wait_bounded(smem_u32(&mbar[(k + j) % s.nbuf]), (uint32_t)(((k + j) / s.nbuf) & 1),
                                      1LL << 28);
            }
            bulk_wait_all();
        }
        return;
    }
    if (tid == 0) bulk_wait_all();
    if constexpr (OP == OP_KIN) {
        const double tot = block_reduce<0>(kin, red);
        if (tid == 0) s.partial[blockIdx.x] = tot;
    }
}

// ---------------------------------------------------------------------------
// Warp-per-pencil-pair strided pass (FP32, N = 256 or 512).
//
// Tiles of 16 columns x N positions (128-byte rows, TMA 128-byte swizzle: the
// 16-byte pencil pair q of row r sits in chunk q ^ (r & 7)) stream through a
// 3-deep ring; one block of 8 warps per SM; warp w transforms the pencil pair
// of columns x0 + 2w, x0 + 2w + 1 with E = N/32 values of each pencil per lane.
// A pencil pair lives in its warp's own 16-byte slots of the tile, so the FFT
// stage exchanges need only __syncwarp: the block synchronises once per tile,
// before the tensor store.  The exchanges address element p at row
// sigma(p) = p ^ ((p >> 3) & 7) of those slots, which keeps every exchange of
// the 512- and 256-point plans and the tile's own (identity) rows free of
// bank conflicts (checked on the CPU with a model of the banks); loads from and
// stores to the tensor copy use the identity rows.
// ---------------------------------------------------------------------------

// barrier over the WPP warps that share pencil pair c (named barrier 1 + c)
template <int WPP> __device__ __forceinline__ void pair_sync(int c) {
    if constexpr (WPP == 1) __syncwarp();
    else named_barrier(1 + c, 32 * WPP);
}
// a pencil pair's element p in the tensor copy's row p of a swizzled tile
template <typename P, int WPP = 1> struct SwzRowAcc {
    P* base;
    int c;
    __device__ __forceinline__ P& operator()(int p) const { return base[p * 8 + (c ^ (p & 7))]; }
    __device__ __forceinline__ void sync() const { pair_sync<WPP>(c); }
};
// the same slots with the exchange rows sigma(p)
template <typename P, int WPP = 1> struct WarpXAcc {
    P* base;
    int c;
    __device__ __forceinline__ P& operator()(int p) const {
        const int r = p ^ ((p >> 3) & 7);
        return base[r * 8 + (c ^ (r & 7))];
    }
    __device__ __forceinline__ void sync() const { pair_sync<WPP>(c); }
};

constexpr int kWpTX = 16;        // tile columns
constexpr int kWpThreads = 256;  // 8 warps, one pencil pair each

__host__ __device__ constexpr bool wp_supported(int N) { return N == 256 || N == 512; }

// WPP warps per pencil pair: WPP = 1 keeps E = N/32 values of each pencil per
// lane (exchanges under __syncwarp); WPP = 2 (N = 512, the wave-function
// passes) splits a pair over two warps with E = N/64, halving the registers so
// that 16 warps fit on an SM, and synchronises the pair's exchanges with a
// 64-thread named barrier.  The exchange rows are the same; with 64 threads
// and radix-8 stages every exchange stays conflict-free (each 8-lane phase of
// an access meets 8 distinct rows mod 8 after sigma).
// blockDim = (32 WPP, 8): thread t = threadIdx.x of pencil pair c = threadIdx.y
template <int N, int OP, bool DF, int PLAN = 0, int WPP = 1>
__global__ void __launch_bounds__(kWpThreads * WPP, 1) k_pencil_wp(const __grid_constant__ CUtensorMap tm, TArgs<float> s) {
    using R = float;
    using C = float2;
    using P = CPair<C>;
    static_assert(wp_supported(N), "warp-per-pencil passes are compiled for N = 256, 512");
    static_assert(WPP == 1 || (WPP == 2 && N == 512 && (OP == OP_FWD || OP == OP_INV || OP == OP_DRIFT)),
                  "two warps per pencil pair: N = 512 wave-function passes only");
    constexpr int NL = qx_with_plan(N, PLAN);
    constexpr int TPP = 32 * WPP;
    constexpr int E = N / TPP;
    static_assert(E % qx_lcm_radices(NL) == 0, "values per thread must hold whole butterflies");
    constexpr int TX = kWpTX;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar[8];
    __shared__ int s_abort;
    __shared__ double red[32];
    const int t = threadIdx.x, c = threadIdx.y;
    const int tid = threadIdx.x + TPP * threadIdx.y;
    const int nthr = kWpThreads * WPP;
    const uint32_t tile_bytes = (uint32_t)((size_t)N * TX * sizeof(C));
    const long tile_elems = (long)(align1k(tile_bytes) / sizeof(C));
    C* bufs = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    C* tws = bufs + s.nbuf * tile_elems;
    C* tws_lo = tws + N;
    double2* bz = reinterpret_cast<double2*>(tws_lo + N);
    double2* aslot = bz + N;
    C* col0 = reinterpret_cast<C*>(bz + (OP == OP_DRIFT ? N + s.nbuf * kTmaMaxTX : 0));
    auto a_of_tile = [&](long id, int j) {
        const int ox = (int)(id / s.tiles_x);
        return s.axy + (s.la3d ? (long)(ox % N) * N : 0L) + (id % s.tiles_x) * TX + j;
    };
    auto coords = [&](long id, int j, int& c0, int& c1, int& c2) {
        const int x0 = (int)(id % s.tiles_x) * TX;
        const int o = (int)(id / s.tiles_x);
        c0 = 2 * x0;
        if (s.pencil_dim == 1) { c1 = j * s.box; c2 = o; }
        else { c1 = o % N; c2 = (o / N) * N + j * s.box; }
    };
    auto issue_load = [&](long id, int b) {
        const uint32_t bar = smem_u32(&mbar[b]);
        mbar_expect_tx(bar, tile_bytes);
        for (int j = 0; j < s.nbox; ++j) {
            int c0, c1, c2;
            coords(id, j, c0, c1, c2);
            tma_load_3d(smem_u32(bufs + b * tile_elems + (long)j * s.box * TX), &tm, c0, c1, c2, bar);
        }
    };

    for (int i = tid; i < N; i += nthr) {
        tws[i] = s.tw[i];
        if constexpr (DF) tws_lo[i] = s.tw_lo[i];
    }
    if constexpr (OP == OP_DRIFT) {
        const double2* gbz = s.axy + (s.la3d ? (long)N * N : (long)N);
        for (int i = tid; i < N; i += nthr) bz[i] = gbz[i];
        if (blockIdx.x < s.n_tiles && tid < TX) aslot[tid] = *a_of_tile(blockIdx.x, tid);
    }
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < s.nbuf; ++b) mbar_init(smem_u32(&mbar[b]), 1);
        fence_mbar_init();
        for (int k = 0; k < s.nbuf - 1; ++k) {
            const long id = blockIdx.x + (long)k * gridDim.x;
            if (id < s.n_tiles) issue_load(id, k);
        }
    }
    __syncthreads();

    double kin = 0.0;
    int k = 0;
    for (;; ++k) {
        const long id = blockIdx.x + (long)k * gridDim.x;
        if (id >= s.n_tiles) break;
        const int b = k % s.nbuf;
        const uint32_t parity = (uint32_t)((k / s.nbuf) & 1);
        if (!mbar_wait_bounded(smem_u32(&mbar[b]), parity)) s_abort = 1;
        C* tile = bufs + b * tile_elems;
        const int x0 = (int)(id % s.tiles_x) * TX;
        const int o = (int)(id / s.tiles_x);
        const int xb = x0 + 2 * c;
        SwzRowAcc<P, WPP> io{reinterpret_cast<P*>(tile), c};
        WarpXAcc<P, WPP> acc{reinterpret_cast<P*>(tile), c};
        const long id_next = id + gridDim.x;
        const bool a_copy = OP == OP_DRIFT && tid < TX && id_next < s.n_tiles;
        if (a_copy) {
            cp_async16(&aslot[((k + 1) % s.nbuf) * kTmaMaxTX + tid], a_of_tile(id_next, tid));
            cp_async_commit();
        }
        P v[E];
        if constexpr (OP == OP_INV) {
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = io(out_pos<NL, E>(e, t));
            ifft_pencil_rev<NL, E>(v, acc, t, tw_src<DF>(tws, tws_lo));
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = io(in_pos<NL, E, 0>(e, t));
            fft_pencil<NL, E, -1>(v, acc, t, tw_src<DF>(tws, tws_lo));
        }
        auto mxy_of = [&](int h) {
            const int x = xb + h;
            const int nx = (s.X == N) ? signed_mode(x, N) : x;
            const int ny = s.la3d ? signed_mode(o % N, N) : 0;
            return (long)nx * nx + (long)ny * ny;
        };
        bool store = true;
        if constexpr (OP == OP_KIN) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long mxy = mxy_of(h);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int nz = signed_mode(out_pos<NL, E>(e, t), N);
                    const C u = pen(v[e], h);
                    kin += (double)(mxy + (long)nz * nz) * ((double)u.x * (double)u.x + (double)u.y * (double)u.y);
                }
            }
            store = false;
        } else if constexpr (OP == OP_DRIFT || OP == OP_POISSON) {
            const bool has_col0 = x0 == 0 && c == 0;
            const bool c0ext = (OP == OP_POISSON) && s.col0_external && has_col0;
            if constexpr (OP == OP_DRIFT) {
                // A(nx, ny) from the tile's ring slot, written before the previous
                // tile's block barrier
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const double2 A = aslot[b * kTmaMaxTX + 2 * c + h];
#pragma unroll
                    for (int e = 0; e < E; ++e)
                        pen(v[e], h) = cmul_d(pen(v[e], h), dcmul(A, bz[out_pos<NL, E>(e, t)]));
                }
            } else {
                SArgs<R> sa;
                sa.pois_c = s.pois_c;
                sa.pois_g0 = s.pois_g0;
                if (c0ext) {
                    // 3D: column 0 is finished by k_poisson_col0; keep its forward result
#pragma unroll
                    for (int e = 0; e < E; ++e) col0[out_pos<NL, E>(e, t)] = pen(v[e], 0);
                } else if (has_col0 && !s.col0_external) {
                    // 2D: the mirror -k_y of column 0 lies in the same pencil (this pair's)
                    pair_sync<WPP>(c);
#pragma unroll
                    for (int e = 0; e < E; ++e) acc(out_pos<NL, E>(e, t)) = v[e];
                    pair_sync<WPP>(c);
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int p = out_pos<NL, E>(e, t);
                        const long np = signed_mode(p, N);
                        const long mA = np * np, mB = mA + (long)(N / 2) * (N / 2);
                        const R gA = pois_mult<R>(mA, sa), gB = pois_mult<R>(mB, sa);
                        const C cm = cconj(pen(acc((N - p) % N), 0));
                        pen(v[e], 0) = cadd(cscale(pen(v[e], 0), R(0.5) * (gA + gB)), cscale(cm, R(0.5) * (gA - gB)));
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (h == 0 && has_col0) continue;
                    const long mxy = mxy_of(h);
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int nz = signed_mode(out_pos<NL, E>(e, t), N);
                        pen(v[e], h) = cscale(pen(v[e], h), pois_mult<R>(mxy + (long)nz * nz, sa));
                    }
                }
            }
            ifft_pencil_rev<NL, E>(v, acc, t, tw_src<DF>(tws, tws_lo));
            if (c0ext) {
                // the stash was written by other threads of this pencil pair in another
                // order; the inverse's exchanges synchronised the pair since
#pragma unroll
                for (int e = 0; e < E; ++e) pen(v[e], 0) = col0[in_pos<NL, E, 0>(e, t)];
            }
        }

        if (a_copy) cp_async_wait_all();
        if (store) {
            // the finished pencil pair -> its slots (identity rows) -> tensor store
            pair_sync<WPP>(c);
            if constexpr (OP == OP_FWD) {
#pragma unroll
                for (int e = 0; e < E; ++e) io(out_pos<NL, E>(e, t)) = v[e];
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) io(in_pos<NL, E, 0>(e, t)) = v[e];
            }
            fence_proxy_async();
            __syncthreads();
            if (s_abort) break;
            if (tid == 0) {
                for (int j = 0; j < s.nbox; ++j) {
                    int c0, c1, c2;
                    coords(id, j, c0, c1, c2);
                    tma_store_3d(&tm, c0, c1, c2, smem_u32(tile + (long)j * s.box * TX));
                }
                bulk_commit();
            }
        } else {
            __syncthreads();
            if (s_abort) break;
        }
        if (tid == 0) {
            const long nid = id + (long)(s.nbuf - 1) * gridDim.x;
            if (nid < s.n_tiles) {
                bulk_wait_read_1();
                fence_proxy_async();
                issue_load(nid, (k + s.nbuf - 1) % s.nbuf);
            }
        }
    }
    if (s_abort) {
        if (tid == 0) {
            atomicExch(s.err, 1);
            for (int j = 0; j < s.nbuf - 1; ++j) {
                const long jd = blockIdx.x + (long)(k + j) * gridDim.x;
                if (jd < s.n_tiles)
                    mbar_wait_bounded(smem_u32(&mbar[(k + j) % s.nbuf]), (uint32_t)(((k + j) / s.nbuf) & 1),
                                      1LL << 28);
            }
            bulk_wait_all();
        }
        return;
    }
    if (tid == 0) bulk_wait_all();
    if constexpr (OP == OP_KIN) {
        const double tot = block_reduce<0>(kin, red);
        if (tid == 0) s.partial[blockIdx.x] = tot;
    }
}

// 3D Poisson, column 0: rows y and N-y (0 pairs with N/2) of the packed
// kx = {0, N/2} column, already transformed along x, y and z, get
// C'(k) = a C(k) + b conj C(-k) with a, b from the kx = 0 and kx = N/2
// multipliers, then the inverse z transform.  blockDim = (2, N/E); grid
// (N/2, boxes of a batched array).
template <int N, typename R, int PLAN = 0>
__global__ void k_poisson_col0(cx_t<R>* vh, const cx_t<R>* tw, const cx_t<R>* tw_lo, double pois_c,
                               double pois_g0) {
    using C = cx_t<R>;
    constexpr int NL = qx_with_plan(N, PLAN);
    constexpr int E = qx_lcm_radices(N);
    constexpr int X = N / 2;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    const int g = threadIdx.x, t = threadIdx.y;
    const int gi = blockIdx.x;
    vh += (long)blockIdx.y * N * N * X;  // box of a batched array
    const int ya = gi == 0 ? 0 : gi, yb = gi == 0 ? N / 2 : N - gi;
    const int y = g == 0 ? ya : yb;
    const int gm = (gi == 0) ? g : 1 - g;
    ColAcc<C> acc{sm + g, 2};
    ColAcc<C> macc{sm + gm, 2};
    const long pstride = (long)N * X;
    const long base = (long)y * X;
    for (int p = t; p < N; p += blockDim.y) acc(p) = vh[base + (long)p * pstride];
    __syncthreads();
    SArgs<R> sa;
    sa.pois_c = pois_c;
    sa.pois_g0 = pois_g0;
    const long ny = signed_mode(y, N);
    C v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int p = out_pos<NL, E>(e, t);
        const long nz = signed_mode(p, N);
        const long mA = ny * ny + nz * nz, mB = mA + (long)X * X;
        const R gA = pois_mult<R>(mA, sa), gB = pois_mult<R>(mB, sa);
        const C cm = cconj(macc((N - p) % N));
        v[e] = cadd(cscale(acc(p), R(0.5) * (gA + gB)), cscale(cm, R(0.5) * (gA - gB)));
    }
    ifft_pencil_rev<NL, E>(v, acc, t, tw_src<false>(tw, tw_lo));
#pragma unroll
    for (int e = 0; e < E; ++e) vh[base + (long)in_pos<NL, E, 0>(e, t) * pstride] = v[e];
}

}  // namespace qx
