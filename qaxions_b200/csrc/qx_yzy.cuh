// qx_yzy.cuh -- the wave-function drift chain (y forward, z forward + drift +
// z inverse, y inverse) as ONE persistent TMA kernel that walks the array in
// x-slabs held in L2 (sm_100a).
//
// The three strided passes of the drift each stream the whole array through
// HBM.  A slab -- sw tiles of TX = 8 columns of x over all y and z of one box,
// 32 MB for sw = 2 and a 512^3 complex64 array -- is closed under the chain:
// its y pencils and its z pencils lie inside it.  So the kernel processes the
// work as units (phase, slab), phase 0 = y forward, 1 = z drift, 2 = y
// inverse, each unit sw N tiles (the N z-planes of the slab for the y phases,
// its N y-rows for the z phase; the sw tiles of one plane or row next to each
// other, so each 128-byte line is read and written whole), in the order
//
//     y(0) | y(1) z(0) | y(2) z(1) y(-0) | y(3) z(2) y(-1) | ...
//
// (unit r of the interleave: y(r), z(r-1), y^-1(r-2)).  About three slabs are
// live at a time, which the 126 MB L2 is meant to hold, so a slab's z and
// inverse-y phases read what the previous phase wrote from L2, and HBM sees
// one read and one write of the array instead of three of each.
//
// Ordering.  Tile g of the global order goes to block g mod G (G = grid, one
// block per SM), and every block walks its tiles in increasing g.  When a tile's tensor store has
// completed, the block adds 1 to the counter of its (phase, slab) with release
// semantics; a z tile may load once its slab's y-forward counter reads sw N, a
// y-inverse tile once the z counter reads sw N (acquire).  The loads of the TMA
// ring are issued ahead, in order, only when their counter is already
// complete; a tile whose load had to be deferred is waited for when its turn
// comes, after the block has completed and published all of its own stores.  Then the
// unpublished tile with the smallest index always belongs to a block that can
// run it (its dependencies have smaller indices), so the walk finishes when
// all blocks are resident -- which the cooperative launch guarantees.
//
// Every wait (mbarrier, counter) is bounded (~1 s of SM clock); a block that
// gives up sets *err, waits (bounded) for its own loads in flight and its
// stores, and returns; blocks waiting for its tiles then give up in turn.
// The work of a block is split between warps: two compute groups transform
// alternate tiles, and one producer warp moves the tiles and keeps the
// counters, so the bookkeeping never holds up the transforms.
//
// The arithmetic of each tile is that of the three separate passes
// (k_pencil_tma with OP_FWD, OP_DRIFT, OP_INV, double-float twiddles), in the
// same element orders, so the chain's result is bit-identical to theirs.
#pragma once

#include "qx_tma.cuh"

namespace qx {

template <typename R> struct YZYArgs {
    const cx_t<R>* tw;     // exp(-2 pi i j/N), stage-major, global
    const cx_t<R>* tw_lo;  // exact - tw
    int sw;                // tiles per slab row: the slab is sw * TX columns wide
    int slabs_x;           // slabs per box (X / (sw TX))
    int nbuf, nbox, box;   // ring depth; TMA boxes per tile and their length
    int n_slabs;           // boxes * slabs_x
    long n_items;          // 3 * n_slabs * sw * N tiles
    unsigned* cnt;         // [3 n_slabs] completed tiles per (phase, slab); zero at launch
    double phase_fac, scale;
    int* err;              // set to 1 when a wait timed out
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// orders this thread's generic-proxy and async-proxy (TMA) accesses to global memory
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}
// wait until at most two bulk groups of this thread are incomplete (writes performed)
__device__ __forceinline__ void bulk_wait_2() { asm volatile("cp.async.bulk.wait_group 2;" ::: "memory"); }

// L2 policy: lines touched through it are the first to be evicted
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void tma_load_3d_hint(uint32_t dst, const CUtensorMap* tm, int c0, int c1, int c2,
                                                 uint32_t bar, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4}], [%5], %6;"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(bar), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void tma_store_3d_hint(const CUtensorMap* tm, int c0, int c1, int c2, uint32_t src,
                                                  uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group.L2::cache_hint [%0, {%1, %2, %3}], [%4], %5;"
        ::"l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(src), "l"(pol)
        : "memory");
}

// Unit u of the processing order of n slabs, as phase * n + slab: unit r of
// the interleave holds y(r), z(r-1), y^-1(r-2), those with a slab in [0, n).
__host__ __device__ constexpr int chain_unit(int u, int n) {
    if (n == 1) return u;  // y(0) z(0) y^-1(0)
    if (u == 0) return 0;
    if (u <= 2) return (u - 1) * n + (2 - u);  // y(1), z(0)
    if (u <= 3 * n - 4) {
        const int r = 2 + (u - 3) / 3, p = (u - 3) % 3;
        return p * n + (r - p);
    }
    if (u == 3 * n - 3) return n + (n - 1);  // z(n-1)
    if (u == 3 * n - 2) return 2 * n + (n - 2);  // y^-1(n-2)
    return 2 * n + (n - 1);  // y^-1(n-1)
}

// dynamic shared memory: NBUF tiles + twiddles (hi, lo) + z drift factors + alignment slack
template <typename R> __host__ __device__ constexpr size_t yzy_smem_bytes(int N, int TX, int nbuf) {
    return (size_t)nbuf * align1k((size_t)N * TX * 2 * sizeof(R)) + (size_t)N * 4 * sizeof(R) + (size_t)N * 16 + 128;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// threads of one compute group (TX / PW pencil groups x N / E threads per
// pencil) and of the block (two groups and the producer warp)
template <int N, typename R, int PW, int TXF> __host__ __device__ constexpr int yzy_group_threads() {
    return (TXF / PW) * (N / tma_e<N, R, PW>());
}
template <int N, typename R, int PW, int TXF> __host__ __device__ constexpr int yzy_block_threads() {
    return 2 * yzy_group_threads<N, R, PW, TXF>() + 32;
}
// compute groups synchronise with named barriers: whole warps only
template <int N, typename R, int PW, int TXF> __host__ __device__ constexpr bool yzy_fits() {
    return yzy_group_threads<N, R, PW, TXF>() % 32 == 0 && yzy_block_threads<N, R, PW, TXF>() <= 1024;
}

// tile accessor of a compute group: plain indexing, FFT exchanges
// synchronised by the group's own named barrier
template <typename P> struct GroupAcc {
    P* base;
    int c, pitch, bar_id, nthr;
    __device__ __forceinline__ P& operator()(int p) const { return base[p * pitch + c]; }
    __device__ __forceinline__ void sync() const { named_barrier(bar_id, nthr); }
};

// One block per SM: compute groups 0 and 1 (threads [0, GT) and [GT, 2 GT))
// transform the block's tiles k = 0, 2, 4, ... and 1, 3, 5, ...; the last
// warp is the producer, whose lane 0 moves every tile with the TMA, checks the
// dependencies and publishes the counters, off the compute warps' path.  Ring
// slot of tile k: k mod NBUF, with mbarriers full[] (tile loaded, TMA
// transaction count) and done[] (tile transformed and written back).  Within
// a group thread (c, t) owns columns x0 + PW c + h.
template <int N, typename R, int PW, int TXF>
__global__ void __launch_bounds__((yzy_block_threads<N, R, PW, TXF>()), 1)
    k_yzy_tma(const __grid_constant__ CUtensorMap tmy, const __grid_constant__ CUtensorMap tmz, YZYArgs<R> s) {
    using C = cx_t<R>;
    using P = pencil_val_t<PW, C>;
    static_assert(TXF > 0 && !tma_swizzled<N, R, PW, TXF>(), "plain tiles of a compiled-in width");
    static_assert(PW == 1 || sizeof(R) == 4, "paired pencils are an FP32 layout");
    static_assert(yzy_fits<N, R, PW, TXF>(), "compute groups of whole warps");
    constexpr int E = tma_e<N, R, PW>();
    constexpr int TX = TXF;
    constexpr int TG = TX / PW;
    constexpr int GT = yzy_group_threads<N, R, PW, TXF>();
    constexpr uint32_t tile_bytes = (uint32_t)(N * TX * sizeof(C));
    constexpr long tile_elems = (long)(align1k(tile_bytes) / sizeof(C));
    constexpr long long kLimit = 1LL << 31;  // ~1 s of SM clock
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[8];
    __shared__ __align__(8) uint64_t done[8];
    __shared__ int s_abort[2];  // per compute group, written by its own threads only
    const int tid = threadIdx.x;
    const long G = gridDim.x;
    C* bufs = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    C* tws = bufs + s.nbuf * tile_elems;
    C* tws_lo = tws + N;
    double2* bz = reinterpret_cast<double2*>(tws_lo + N);

    // tile id: unit id / (sw N); within it, plane / row q and the slab's
    // x-tile (fastest, so the sw tiles of one 128-byte row run together)
    const int upt = s.sw * N;  // tiles per unit
    auto unit_of = [&](long id) { return chain_unit((int)(id / upt), s.n_slabs); };
    auto tile_pos = [&](long id, int& ph, int& q, int& c0, int& zb) {
        const int u = unit_of(id);
        const int w = (int)(id % upt);
        const int sl = u % s.n_slabs;
        ph = u / s.n_slabs;
        q = w / s.sw;
        c0 = 2 * ((sl % s.slabs_x) * s.sw + w % s.sw) * TX;
        zb = (sl / s.slabs_x) * N;
    };

    for (int i = tid; i < N; i += blockDim.x) {
        tws[i] = s.tw[i];
        tws_lo[i] = s.tw_lo[i];
        const long n = signed_mode(i, N);
        const double2 w = cis_d(s.phase_fac * (double)(n * n));
        bz[i] = make_double2(w.x * s.scale, w.y * s.scale);
    }
    if (tid == 0) {
        s_abort[0] = s_abort[1] = 0;
        for (int b = 0; b < s.nbuf; ++b) {
            mbar_init(smem_u32(&full[b]), 1);
            mbar_init(smem_u32(&done[b]), 1);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (tid >= 2 * GT) {
        // ------------------------------------------------------------ producer
        if (tid == 2 * GT) {
            const uint64_t pol_first = l2_evict_first();
            const int ntiles = blockIdx.x < s.n_items ? (int)((s.n_items - blockIdx.x + G - 1) / G) : 0;
            auto tile_id = [&](int k) { return blockIdx.x + k * G; };
            auto issue_load = [&](int k) {
                int ph, q, c0, zb;
                tile_pos(tile_id(k), ph, q, c0, zb);
                const int b = k % s.nbuf;
                const uint32_t bar = smem_u32(&full[b]);
                mbar_expect_tx(bar, tile_bytes);
                for (int j = 0; j < s.nbox; ++j) {
                    const uint32_t dst = smem_u32(bufs + b * tile_elems + (long)j * s.box * TX);
                    if (ph == 1) tma_load_3d(dst, &tmz, c0, q, zb + j * s.box, bar);  // z pencils of y-row q
                    else if (ph == 2) tma_load_3d(dst, &tmy, c0, j * s.box, zb + q, bar);  // y pencils of z-plane q
                    else tma_load_3d_hint(dst, &tmy, c0, j * s.box, zb + q, bar, pol_first);  // read once from HBM
                }
            };
            auto issue_store = [&](int k) {
                int ph, q, c0, zb;
                tile_pos(tile_id(k), ph, q, c0, zb);
                const C* tile = bufs + (k % s.nbuf) * tile_elems;
                for (int j = 0; j < s.nbox; ++j) {
                    const uint32_t src = smem_u32(tile + (long)j * s.box * TX);
                    if (ph == 1) tma_store_3d(&tmz, c0, q, zb + j * s.box, src);
                    else if (ph == 0) tma_store_3d(&tmy, c0, j * s.box, zb + q, src);
                    else tma_store_3d_hint(&tmy, c0, j * s.box, zb + q, src, pol_first);  // final: no reuse in L2
                }
                bulk_commit();
            };
            // a tile's input is final: y forward reads the previous kernel's
            // output, the later phases wait for all sw N tiles of the previous
            // phase of the slab.  A complete counter is acquired once per unit;
            // the proxy fence after it orders all later tensor loads behind it.
            int ok_unit = -1;
            auto dep_ok = [&](int k) -> bool {
                const int u = unit_of(tile_id(k));
                if (u < s.n_slabs || u == ok_unit) return true;
                if (ld_acquire_u32(&s.cnt[u - s.n_slabs]) < (unsigned)upt) return false;
                fence_proxy_async_global();
                ok_unit = u;
                return true;
            };
            // completed own tiles are counted per unit, once the block's last
            // tile of the unit is among them (or before a wait, or at the end)
            int pub = 0, pend_u = -1;
            unsigned pend_c = 0;
            auto flush = [&]() {
                if (!pend_c) return;
                fence_proxy_async_global();
                red_release_add_u32(&s.cnt[pend_u], pend_c);
                pend_c = 0;
            };
            auto publish_upto = [&](int kend, bool force) {  // own tiles pub .. kend-1 (stores complete)
                for (; pub < kend; ++pub) {
                    const long id = tile_id(pub);
                    const int u = unit_of(id);
                    if (u != pend_u) {
                        flush();
                        pend_u = u;
                    }
                    ++pend_c;
                    if (id + G >= s.n_items || unit_of(id + G) != u) flush();
                }
                if (force) flush();
            };

            int kl = 0;  // next tile to load (loads are issued in order)
            int ks = 0;  // next tile to store
            bool abort = false;
            // tile kl may load once the store of tile kl - NBUF (its slot) was read out
            auto try_loads = [&](int limit) {
                while (kl < ntiles && kl < limit && dep_ok(kl)) {
                    issue_load(kl);
                    ++kl;
                }
            };
            try_loads(s.nbuf);
            while (ks < ntiles) {
                if (kl == ks) {
                    // the next tile's input is not final yet: complete and
                    // publish every own store, then wait (bounded) for it
                    bulk_wait_all();
                    publish_upto(ks, true);
                    const long long t0 = clock64();
                    bool ok = dep_ok(ks);
                    while (!ok && clock64() - t0 < kLimit / 2) {
                        __nanosleep(128);
                        ok = dep_ok(ks);
                    }
                    if (!ok) {
                        abort = true;
                        break;
                    }
                    issue_load(ks);
                    ++kl;
                }
                if (!mbar_wait_bounded(smem_u32(&done[ks % s.nbuf]), (uint32_t)((ks / s.nbuf) & 1), kLimit)) {
                    abort = true;
                    break;
                }
                issue_store(ks);
                ++ks;
                bulk_wait_read_1();  // stores of tiles <= ks-2 read out
                try_loads(ks - 1 + s.nbuf);
                bulk_wait_2();  // stores of tiles <= ks-3 complete
                publish_upto(ks - 2, false);
            }
            if (abort) {
                // flag it; wait (bounded) for the loads this block still has in
                // flight, then for its stores
                atomicExch(s.err, 1);
                for (int k = ks; k < kl; ++k)
                    mbar_wait_bounded(smem_u32(&full[k % s.nbuf]), (uint32_t)((k / s.nbuf) & 1), 1LL << 28);
                bulk_wait_all();
            } else {
                bulk_wait_all();
                publish_upto(ks, true);
            }
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- compute groups
        const int grp = tid / GT, lt = tid % GT;
        const int c = lt % TG, t = lt / TG;
        const auto tw = tw_src<true>(tws, tws_lo);
        for (int k = grp;; k += 2) {
            const long id = blockIdx.x + k * G;
            if (id >= s.n_items) break;
            const int b = k % s.nbuf;
            // a time-out is acted on at the tile's last group barrier, where
            // all threads of the group read the same flag
            if (!mbar_wait_bounded(smem_u32(&full[b]), (uint32_t)((k / s.nbuf) & 1), kLimit)) s_abort[grp] = 1;
            int ph, q, c0, zb;
            tile_pos(id, ph, q, c0, zb);
            const int x0 = c0 / 2;
            GroupAcc<P> acc{reinterpret_cast<P*>(bufs + b * tile_elems), c, TG, 1 + grp, GT};
            P v[E];
            if (ph == 2) {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = acc(out_pos<N, E>(e, t));
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = acc(in_pos<N, E, 0>(e, t));
                fft_pencil<N, E, -1>(v, acc, t, tw);
            }
            if (ph == 1) {
                // exp(-i dt/2 dk^2 (nx^2 + ny^2 + nz^2)) / S = A(nx, ny) B(nz), FP64
                const long ny = signed_mode(q, N);
                double2 A[PW];
#pragma unroll
                for (int h = 0; h < PW; ++h) {
                    const long nx = signed_mode(x0 + PW * c + h, N);
                    A[h] = cis_d(s.phase_fac * (double)(nx * nx + ny * ny));
                }
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const double2 bze = bz[out_pos<N, E>(e, t)];
#pragma unroll
                    for (int h = 0; h < PW; ++h) pen(v[e], h) = cmul_d(pen(v[e], h), dcmul(A[h], bze));
                }
            }
            if (ph != 0) ifft_pencil_rev<N, E>(v, acc, t, tw);

            // finished tile -> buffer (natural order); the producer stores it
            acc.sync();
            if (ph == 0) {
#pragma unroll
                for (int e = 0; e < E; ++e) acc(out_pos<N, E>(e, t)) = v[e];
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) acc(in_pos<N, E, 0>(e, t)) = v[e];
            }
            fence_proxy_async();
            acc.sync();
            if (s_abort[grp]) break;
            if (lt == 0) mbar_arrive(smem_u32(&done[b]));
        }
    }
    __syncthreads();
}

}  // namespace qx
