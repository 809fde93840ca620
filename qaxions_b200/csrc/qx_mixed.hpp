// qx_mixed.hpp -- host side of the mixed-size ensemble passes: one persistent
// launch per pass over the boxes of every grid size of an ensemble, fed by a
// work queue (qx_mixed.cu).  No CUDA templates are exposed here.
#pragma once

#include <cuda_runtime.h>

namespace qx {

// the passes of one merged-KDK loop body, in the order they run
enum MixOp {
    MX_Y_FWD_PSI = 0,   // forward y transform of psi^_x (double-float twiddles in FP32)
    MX_Z_DRIFT = 1,     // forward z, drift phase A(nx, ny) B(nz), inverse z
    MX_Y_INV_PSI = 2,   // inverse y transform of psi
    MX_X_INV_R2C = 3,   // inverse x -> psi; density pref(|psi|^2 - rho_mean); r2c x -> vh
    MX_Y_FWD_VH = 4,    // forward y transform of the half spectrum
    MX_Z_POISSON = 5,   // forward z, -1/(k^2 S) (column 0 with its mirror), inverse z
    MX_Y_INV_VH = 6,    // inverse y transform of the half spectrum
    MX_X_C2R_KICK = 7,  // c2r x -> V; kick psi by V; forward x -> psi^_x
    MX_NOPS = 8
};

constexpr int kMixMaxGroups = 4;

// One box size of an ensemble: a batched array of `B` boxes of N^3 sites and
// the device tables the passes read (plain pointers; complex arrays are
// interleaved in the field's precision).
struct MixDesc {
    void* psi = nullptr;         // [B][N][N][N] complex
    void* vh = nullptr;          // [B][N][N][N/2] packed half spectrum
    const void* twN = nullptr;   // stage-major N-point twiddles (radix plan 0)
    const void* twN_lo = nullptr;  // their low parts (FP32 double-float twiddles)
    const void* twM = nullptr;   // stage-major N/2-point twiddles
    const void* twNn = nullptr;  // natural-order exp(-2 pi i k/N), k < N/2
    const double2* axy = nullptr;  // drift factors: A(nx, ny) [N][N], then B(nz)/S [N]
    int N = 0, B = 0;
    double pois_c = 0, pois_g0 = 0;   // Poisson -1/(dk^2 S) and the k = 0 multiplier
    double pref = 1, rho_mean = 1;    // density source pref (|psi|^2 - rho_mean)
    double dt_kick = 0;               // kick step of the loop body
};

template <typename R> struct Mixed {
    // whether grid size N (3D) has a compiled mixed-size unit
    static bool supports(int N);
    // work units of group d in pass op (the queue length is their sum)
    static long units(int op, const MixDesc& d);
    // launch pass `op` over the groups d[0..ng) on stream st; `ctr` is the
    // pass's queue counter, which must be zero when the launch starts; *err is
    // set to 2 (and no unit runs) if the kernel's unit layout disagrees with
    // the host's
    static void launch(int op, const MixDesc* d, int ng, unsigned long long* ctr, int* err, cudaStream_t st);
    // the whole loop body (the 8 passes) as ONE persistent launch over a queue
    // of every pass's units, a unit starting once its box has finished the
    // previous pass.  The queue runs windows of boxes whose psi and half
    // spectrum fit in window_bytes (every pass of a window before the next
    // window), so a box's arrays can stay in L2 between its passes; a window
    // as large as the ensemble gives pass-by-pass order.  ctr (1 counter) and
    // done (MX_NOPS * boxes counters) must be zero when the launch starts;
    // *err is set to 1 if a wait timed out, 2 if the kernel's unit layout
    // disagrees with the host's (then no unit runs).
    static void launch_step(const MixDesc* d, int ng, unsigned long long* ctr, unsigned* done, int* err,
                            long window_bytes, cudaStream_t st);
    // set the kernels' shared-memory attributes for these groups (before a
    // stream capture of launch() / launch_step())
    static void prepare(const MixDesc* d, int ng);
};

}  // namespace qx
