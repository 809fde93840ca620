/*
 * qaxions_b200.h -- C ABI of the B200-native Schroedinger-Poisson solver core.
 *
 * One opaque handle per periodic 2D/3D box.  Every entry point returns an int
 * status (QX_OK = 0); on failure qx_last_error(handle) gives the message
 * (qx_last_error(NULL) for failures of qx_create).  No C++ exception crosses
 * this boundary.  Host arrays are FP64 in the reference's memory order
 * (3D: idx = iz*N*N + iy*N + ix, x fastest; complex interleaved re,im), whatever
 * the device precision.  A handle owns its device buffers and one CUDA stream;
 * it is not thread-safe.
 *
 * Each declaration names the reference interface it replaces
 * (gpierobon/qaxions, path:line).
 */
#ifndef QAXIONS_B200_H
#define QAXIONS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define QX_OK 0
#define QX_ERR_INVALID 1     /* bad argument / unsupported shape        */
#define QX_ERR_CUDA 2        /* CUDA runtime or launch failure          */
#define QX_ERR_NOMEM 3       /* device allocation failed                */
#define QX_ERR_STATE 4       /* call not valid in the handle's state    */
#define QX_ERR_INTERNAL 5

#define QX_C128 0            /* plain FP64 form (complex128)            */
#define QX_C64 1             /* fused FP32 form (complex64)             */

#define QX_K0_REFERENCE 0    /* k=0 Poisson mode divided by 1 (src/field.cxx:253,282) */
#define QX_K0_ZERO 1         /* k=0 Poisson mode set to exactly 0       */

#define QX_SPEC_REFERENCE 0  /* integer shells round(|n|), N/2+1 bins (src/spectrum/spectrum.cxx:63-155) */
#define QX_SPEC_LINEAR 1     /* nbins linear bins over 0 < |n| < N/2    */
#define QX_SPEC_LOG 2        /* nbins log bins over 1 <= |n| < N/2      */

#define QX_IC_SOLITONS 0     /* sum of Schive-profile solitons          */
#define QX_IC_GRF 1          /* sqrt(1 + delta), delta a Gaussian random field (+ solitons if n > 0) */

typedef struct qx_field_s qx_field_t;

int qx_version(void);
const char *qx_last_error(const qx_field_t *h);
/* select the CUDA device for handles created afterwards by this thread
 * (one process per GPU: the reference's --nthr thread setting,
 * src/parse.cxx:162, has no GPU counterpart; this is its placement knob) */
int qx_set_device(int device);

/* Field construction: Field::Field(Params&) / Field::init / setCosmo
 * (src/field.cxx:13-46,68-91), STATIC cosmology.  pref = norm_*a_
 * (src/field.cxx:78,298), rho_mean = rho_mean_ (src/field.cxx:77),
 * dt = ds_ (src/field.cxx:77).  Supported N: 4, 8, 16, 32, 64, 96, 128, 256, 512. */
int qx_create(int dim, int N, double L, double pref, double rho_mean, int dtype, int k0_policy,
              double dt, qx_field_t **out);
/* Field::~Field (src/field.cxx:58-66) */
int qx_destroy(qx_field_t *h);
/* ds_ (src/field.h:82) */
int qx_set_dt(qx_field_t *h, double dt);

/* Field::psi() / getPsiIdx / getPsiImagIdx (src/field.h:36-39): 2*sites doubles */
int qx_set_psi(qx_field_t *h, const double *psi);
int qx_get_psi(qx_field_t *h, double *psi);
/* Field::V() / getVIdx (src/field.h:41-43): sites doubles */
int qx_set_V(qx_field_t *h, const double *V);
int qx_get_V(qx_field_t *h, double *V);
/* Field::Vhat() (src/field.h:45): 2*ksites doubles in FFTW r2c layout
 * [..][N/2+1] (the device keeps a packed N/2-column form) */
int qx_get_Vhat(qx_field_t *h, double *vhat);
int qx_set_Vhat(qx_field_t *h, const double *vhat);

/* Field::kick (src/field.cxx:93-116) */
int qx_kick(qx_field_t *h, double dt);
/* Field::drift (src/field.cxx:119-198) */
int qx_drift(qx_field_t *h, double dt);
/* Field::Poisson (src/field.cxx:230-291), on the transformed V^ */
int qx_poisson(qx_field_t *h);
/* Field::updatePotential (src/field.cxx:294-346) */
int qx_update_potential(qx_field_t *h);
/* Field::computeEnergy (src/field.cxx:200-227): V <- |psi|^2, rhomax */
int qx_compute_energy(qx_field_t *h);
/* Field::updateTime / half_kick / full_kick / drift_update / propagate
 * (src/field.cxx:349-402) */
int qx_update_time(qx_field_t *h);
int qx_half_kick(qx_field_t *h);
int qx_full_kick(qx_field_t *h);
int qx_drift_update(qx_field_t *h);
int qx_propagate(qx_field_t *h);
/* The KDK time loop of main() (src/main.cxx:64-85) with measurements off:
 * updatePotential, half_kick, nsteps x (drift_update, full_kick but the last),
 * half_kick -- fused passes, loop body replayed from a CUDA graph. */
int qx_step(qx_field_t *h, int nsteps);

/* Field::Vmax / rhomax / time / a / curr (src/field.h:56-62) */
int qx_scalars(qx_field_t *h, double *vmax, double *rhomax, double *time, double *a, int *curr);
/* computeEnergy's rhomax and updatePotential's Vmax without overwriting V
 * (src/field.cxx:216-226,338-345) */
int qx_rho_stats(qx_field_t *h, double *rhomax, double *vmax);
/* mass and energy diagnostics (no reference counterpart; M = sum |psi|^2 dV,
 * E = K + W, K spectral, W = 1/2 sum V |psi|^2 dV) */
int qx_mass_energy(qx_field_t *h, double *M, double *E, double *K, double *W);
/* Spectrum::compute + Pk/counts/kmodes (src/spectrum/spectrum.cxx:32-164,
 * src/spectrum/spectrum.h:21-32).  source 0: |psi|^2 (what measure() bins
 * after computeEnergy, src/meas.cxx:30-41), 1: V.  Arrays hold nbins entries
 * (N/2+1 for QX_SPEC_REFERENCE, nbins ignored). */
int qx_spectrum(qx_field_t *h, int source, int mode, int nbins, double *k, double *P, long long *count);

/* ---- measurements (src/meas.h, src/meas.cxx:13-63, src/enum.h:39-47) ----
 * MeasureType bits of the reference, and two of this library's own. */
#define QX_MEAS_NONE 0u
#define QX_MEAS_SPECTRUM (1u << 0)   /* spec_NNNN.txt: reference shells of |psi|^2 */
#define QX_MEAS_RHO_MAX (1u << 1)    /* rhomax (taken whenever the mask is not NONE) */
#define QX_MEAS_RHO_SLICE (1u << 2)  /* enumerated by the reference; its measure() ignores it */
#define QX_MEAS_RHO_GRID (1u << 3)   /* field_NNNN.rho (raw FP64 rho) + field_NNNN.json Header */
#define QX_MEAS_PSI_GRID (1u << 4)   /* enumerated by the reference; its measure() ignores it */
#define QX_MEAS_ENERGY (1u << 8)     /* mass and energy (no reference counterpart) */
#define QX_MEAS_CLOBBER_V (1u << 9)  /* leave V = |psi|^2 afterwards, as the reference's
                                        computeEnergy does (src/field.cxx:205-211) */
/* one measurement: the values measure()/printStatus report (src/utils.cxx:64-85)
 * plus this library's diagnostics; mass/energy/kinetic/potential are NaN
 * unless QX_MEAS_ENERGY */
typedef struct {
    int number;        /* measurement number, 0 = before the loop */
    int step;          /* Field::curr() */
    double time;       /* Field::time() */
    double a;          /* Field::a() */
    double rhomax;     /* max |psi|^2 / mean |psi|^2 (computeEnergy) */
    double vmax;       /* max |V| of the potential of this psi */
    double mass, energy, kinetic, potential;
} qx_meas_t;
/* generateMeasList (src/utils.cxx:8-28): the loop indices after whose
 * drift_update main() measures; *n_out = number written (<= max_out) */
int qx_meas_list(long long nsteps, long long nmeas, long long *out, int max_out, int *n_out);
/* measure(Field&, Params&, measNumber, ...) (src/meas.cxx:13-63) of the current
 * state.  Unlike the reference it leaves V alone unless mask has
 * QX_MEAS_CLOBBER_V.  Files (spec_NNNN.txt, field_NNNN.*, measurements.jsonl)
 * go to directory `dir` when it is not NULL.  rec may be NULL. */
int qx_measure(qx_field_t *h, unsigned mask, int number, const char *dir, qx_meas_t *rec);
/* The time loop of main() (src/main.cxx:60-85) with its measurements:
 * measure(0), updatePotential, half_kick, then for every loop index idx
 * drift_update, measure(k) if idx is the k-th entry of
 * qx_meas_list(nsteps, nmeas), full_kick but the last; final half_kick.
 * Unmeasured loop bodies are the fused, graph-replayed passes of qx_step.
 * recs holds max_recs records (nmeas + 1 suffice); *n_out = records taken. */
int qx_run(qx_field_t *h, int nsteps, int nmeas, unsigned mask, const char *dir, qx_meas_t *recs, int max_recs,
           int *n_out);

/* FFTBackend::forward_c2c / backward_c2c / forward_r2c / backward_c2r
 * (src/fft/fft.h:14-17) on host buffers; sign -1 forward, +1 backward;
 * r2c/c2r halves use FFTW's [..][N/2+1] layout; all unnormalised. */
int qx_fft_c2c(qx_field_t *h, double *data, int sign);
int qx_fft_r2c(qx_field_t *h, const double *in, double *out);
int qx_fft_c2r(qx_field_t *h, const double *in, double *out);

/* SolitonsIC::apply (src/ic/solitons.cxx:20-110): Gaussian 'solitons' from a
 * solitons.txt-format file (rows: amp sigma x y z) over background bkg. */
int qx_ic_solitons_file(qx_field_t *h, const char *path, double bkg);
/* the same from an in-memory table of n rows {amp, sigma, x, y, z} */
int qx_ic_gaussian_solitons(qx_field_t *h, int n, const double *rows5, double bkg);
/* synthetic benchmark initial conditions (no reference counterpart):
 * kind QX_IC_SOLITONS (psi = sum of n Schive solitons) or QX_IC_GRF
 * (psi = sqrt(1+delta) + n solitons), delta ~ P(k) = k^-2 exp(-(k/kc)^2),
 * kc = kc_factor*N*2pi/L, std sigma, clipped at clip; soliton rc ~ U[rc_lo,
 * rc_hi), rho_c = rho0 rc^-4, centres ~ U[0,1)^d, phases ~ U[0,2pi) from
 * Philox4x32-10 keyed by seed; finally mean |psi|^2 = 1. */
int qx_ic_config(qx_field_t *h, int kind, unsigned long long seed, int n_solitons, double rc_lo,
                 double rc_hi, double sigma, double kc_factor, double clip, double rho0);

/* device time (CUDA events on the handle's stream) of qx_step(nsteps) */
int qx_time_steps(qx_field_t *h, int nsteps, int use_graph, float *ms);
/* per-pass average device time of the fused loop body over nsteps bodies;
 * names: max_entries x 64 chars.  Advances the state. */
int qx_profile_step(qx_field_t *h, int nsteps, int max_entries, char *names, double *ms, int *n_out);
/* launch geometry overrides (0 = default): rows per x-pass block, tile columns
 * of y / last-axis passes, strided-pass kernel family (1 = TMA-fed persistent,
 * 0 = direct loads; -1 = keep), TMA ring depth, pencils per thread of the TMA
 * passes (1 or 2; 0 = default: 2 in the FP32 form, FP64 always 1) */
int qx_set_tune(qx_field_t *h, int x_rows, int y_tx, int la_tx, int tma, int nbuf, int pw);
/* Radix plan of the TMA strided (y / last-axis) passes, no counterpart in the
 * reference (FFTW plans its own): 0 default, 1 the same radices in reverse
 * order, for grids whose default plan mixes radix sizes (N = 64, 96, 128,
 * 256); elsewhere plan 1 runs as plan 0.  Results agree to round-off. */
int qx_set_plan(qx_field_t *h, int plan);
/* Pencil-to-thread mapping of the FP32 strided passes at N = 256 and 512 (no
 * counterpart in the reference): 8-column tiles with a pencil pair per 64
 * (N = 512) threads and block-wide stage exchanges, or 16-column swizzled tiles
 * with one warp per pencil pair, warp-local exchanges and one block barrier
 * per tile.  on = 0: the 8-column passes everywhere; 1: the warp passes for
 * the wave-function arrays; 2: the warp passes everywhere; 3 / 4 (N = 512):
 * as 1, with each pencil pair split over two warps (16 warps per SM, pair
 * barriers) in the drift pass / in every wave-function pass, bit for bit the
 * one-warp form.  The 3D 512^3 default is 3 (measured fastest).  Results
 * agree to round-off. */
int qx_set_pencil_warp(qx_field_t *h, int on);
/* the launch geometry in use: out[10] = {x_rows, y_tx, la_tx, tma, nbuf, pw,
 * plan, chain, pencil_warp, from_cache}, and out[10] = row_stage when n >= 11;
 * from_cache = 1 when the field took it from the autotuner's cache at creation
 * (the process cache, or the file named by the environment variable
 * QX_TUNE_CACHE) */
int qx_get_tune(qx_field_t *h, int *out, int n);
/* Row pass of the inverse x transform, density and r2c (the FP32 form, N >= 256;
 * no counterpart in the reference, whose drift/updatePotential call library
 * FFTs, src/field.cxx:119-198, 294-346): on = 1 copies each warp's next row
 * into shared memory with cp.async while the current row is transformed, on = 0
 * loads rows directly.  Bit-identical results. */
int qx_set_row_stage(qx_field_t *h, int on);
/* Drift chain (no counterpart in the reference: the reference's drift,
 * src/field.cxx:119-198, is three library FFT calls around a multiply).  on = 0
 * (default): the y forward, z drift and y inverse passes of a 3D complex64
 * field run as three persistent passes; on = 2 / 1: as one cooperative kernel
 * that walks the array in x-slabs of 16 / 8 columns, so the later phases of a
 * slab can read the earlier ones' output from L2.  Results are bit-identical
 * in all three modes; on B200 the three passes are faster at every size
 * measured (64^3 .. 512^3). */
int qx_set_chain(qx_field_t *h, int on);
/* Autotuner: time nsteps steps under each candidate launch geometry (radix
 * plan of the strided passes, pencils per thread, TMA ring depth, tile widths,
 * rows per x block), keep the fastest; psi is restored afterwards.  Cached per
 * (dim, N, dtype, batch) in the process and in the text file cache_path if not
 * NULL (read first, appended after); fields created later with the same key
 * start with the cached geometry (qx_get_tune).  best_ms: ms per step of the
 * choice; from_cache: 1 if nothing was timed. */
int qx_autotune(qx_field_t *h, int nsteps, const char *cache_path, double *best_ms, int *from_cache);
/* forget the autotuner's in-process choices (cache files are not touched) */
int qx_clear_tune_cache(void);
int qx_device_pointers(qx_field_t *h, void **psi, void **V);
/* dst psi <- src psi on the device (same dim, N, batch and dtype) */
int qx_copy_psi(qx_field_t *dst, qx_field_t *src);
/* psi was written through qx_device_pointers: recompute V before it is used */
int qx_psi_changed(qx_field_t *h);
/* cosmology: 0 STATIC (a = 1, the default); 1 MRE starting at a = ai:
 * ds = dt / ai, norm 1 (Poisson prefactor a), rho_mean = 1.5 (2 pi)^2 1.27^2,
 * and every step ds = 0.00025 / a, a *= 1 + 1.27^2 sqrt(1 + a) ds
 * (src/field.cxx:70-90, 349-361).  MRE steps run without the loop-body graph. */
int qx_set_cosmology(qx_field_t *h, int cosmo, double ai);
/* cosmology state Field::a_ / ds_ (src/field.h:80-82): mode (0 STATIC, 1
 * MRE), scale factor and current time step */
int qx_get_cosmology(qx_field_t *h, int *cosmo, double *a, double *ds);
/* restore a and ds of a checkpoint after qx_set_cosmology (which starts the
 * cosmology afresh); the reference's checkpoint header stores a
 * (IO::writeConf, src/io/io.cxx:362-367) but its reader does not restore it */
int qx_restore_cosmology(qx_field_t *h, double a, double ds);
/* set the step counter and time (restoring a checkpoint) */
int qx_set_clock(qx_field_t *h, int step, double time);
/* psi *= factor (real) */
int qx_scale_psi(qx_field_t *h, double factor);
int qx_sync(qx_field_t *h);

/* ---- ensemble of independent boxes (no counterpart in the reference, which
 * runs one box per process, src/main.cxx:34-53) ----
 * ngroups groups of boxes; group g holds boxes[g] boxes of size N[g]^dim, all
 * with the same L, pref, dtype and dt.  The boxes of a group are stacked in one
 * device array, so every pass of a step is one persistent launch over the
 * tiles of all of the group's boxes; each group's loop body is replayed from a
 * CUDA graph on its own stream and the groups run concurrently.  Boxes are
 * numbered group by group.  Single-box operations (spectrum, Vhat, FFT plugin)
 * are not available on ensemble boxes.  Errors: qx_ens_last_error(h). */
typedef struct qx_ens_s qx_ens_t;
int qx_ens_create(int ngroups, const int *N, const int *boxes, int dim, double L, double pref, int dtype,
                  double dt, qx_ens_t **out);
int qx_ens_destroy(qx_ens_t *h);
const char *qx_ens_last_error(const qx_ens_t *h);
/* number of boxes and total sites */
int qx_ens_size(qx_ens_t *h, int *nboxes, long long *sites);
/* grid size of one box */
int qx_ens_box_n(qx_ens_t *h, int box, int *N);
/* initial conditions as qx_ic_config, box b seeded with seed_base + b */
int qx_ens_ic_config(qx_ens_t *h, int kind, unsigned long long seed_base, int n_sol, double rc_lo,
                     double rc_hi, double sigma, double kc_factor, double clip, double rho0);
/* the same with one seed per box (nboxes values): an ensemble sharded over
 * several processes seeds each local box by its global box index */
int qx_ens_ic_config_seeds(qx_ens_t *h, int kind, const unsigned long long *seeds, int n_sol, double rc_lo,
                           double rc_hi, double sigma, double kc_factor, double clip, double rho0);
int qx_ens_set_psi(qx_ens_t *h, int box, const double *psi);
int qx_ens_get_psi(qx_ens_t *h, int box, double *psi);
/* nsteps merged KDK steps of every box (returns when all are done) */
int qx_ens_step(qx_ens_t *h, int nsteps);
/* device time of qx_ens_step(nsteps) over all groups (events on the groups' streams) */
int qx_ens_time_steps(qx_ens_t *h, int nsteps, float *ms);
/* mass sum |psi|^2 dV of every box (nboxes doubles) */
int qx_ens_mass(qx_ens_t *h, double *M);
/* Loop-body mode of the steps in between the first and the last of a call.
 * mixed = 0 (default): each group's body replayed on its own stream (a graph
 * branch per group, one launch per pass per group).  mixed = 1: the whole
 * loop body of every box as ONE persistent launch per step, driven by a work
 * queue of (pass, box, tile-or-rows) units (pass by pass, the costliest sizes
 * first); a unit starts once its box has finished the previous pass, so the
 * passes of different boxes overlap.  mixed = 2: one persistent launch per
 * pass over the boxes of every size (the same queue, one pass at a time).
 * Modes 1 and 2: 3D, STATIC cosmology, at most 4 groups, every N in
 * {16, 32, 64, 96, 128} (QX_ERR_INVALID otherwise).  Every mode advances each
 * box as its single-box run does. */
int qx_ens_set_mixed(qx_ens_t *h, int mixed);
/* Mode 1's queue runs the passes of windows of boxes whose psi and half
 * spectrum together take at most `bytes` (at least one box per window) before
 * moving to the next window, so a box's arrays can stay in the 126 MB L2 from
 * one pass to the next.  0 = the default, 48 MiB; a value above the whole
 * ensemble's size gives pass-by-pass order over all boxes. */
int qx_ens_set_mixed_window(qx_ens_t *h, long long bytes);

/* ---- learned corrector for coarse steps (no counterpart in the reference) ----
 * A periodic 3^3 convolutional network (4 -> 32 -> 32 -> 2 channels, GELU,
 * BF16 weights on the tensor cores, FP32 accumulation) on N^3 grids (N a
 * multiple of 8) predicts psi(4 fine steps) - psi(1 coarse step of 4 dt) from
 * the coarse result: features Re psi, Im psi, V / v_scale, |psi|^2 - 1; output
 * scaled by tau.  State arguments are device pointers to complex64 psi and
 * float32 V of an N^3 field (qx_device_pointers of a QX_C64 field).
 * Parameters (qx_corr_get/set_params, FP32): w1 [27][4][32], b1 [32],
 * w2 [27][32][32], b2 [32], w3 [27][32][2], b3 [2]; offset index
 * o = (dz+1)*9 + (dy+1)*3 + (dx+1).  Errors: qx_corr_last_error(h). */
typedef struct qx_corr_s qx_corr_t;
int qx_corr_create(int N, unsigned long long seed, qx_corr_t **out);
int qx_corr_destroy(qx_corr_t *h);
const char *qx_corr_last_error(const qx_corr_t *h);
int qx_corr_nparams(qx_corr_t *h, int *n);
int qx_corr_set_scales(qx_corr_t *h, double v_scale, double tau);
/* Tensor path of the convolutions with 32 outputs (forward of the first and
 * middle layers, data gradients of the middle and last layers): 1 (default)
 * tcgen05.mma with tensor-memory accumulators, for grids with N % 16 == 0; 0
 * the mma.sync kernel that the last layer's forward always uses. */
int qx_corr_set_tensor_path(qx_corr_t *h, int tc);
int qx_corr_get_scales(qx_corr_t *h, double *v_scale, double *tau);
int qx_corr_get_params(qx_corr_t *h, float *params);
int qx_corr_set_params(qx_corr_t *h, const float *params);
/* loss (mean square of net - (psi_f - psi_c)/tau) and its gradient (nparams
 * floats, layout of the parameters) for one pair, without updating */
int qx_corr_gradients(qx_corr_t *h, const void *psi_c, const void *V_c, const void *psi_f, float *grads,
                      double *loss);
/* one Adam step (learning rate lr) on one pair; returns the loss before it */
int qx_corr_train_pair(qx_corr_t *h, const void *psi_c, const void *V_c, const void *psi_f, double lr,
                       double *loss);
/* psi += tau * net(psi, V), ordered after prior work on `stream` (a
 * cudaStream_t, e.g. the field's) and before later work on it */
int qx_corr_apply(qx_corr_t *h, void *psi, const void *V, void *stream);
/* the last forward's raw output [N^3][2] (host copy) */
int qx_corr_output(qx_corr_t *h, float *out);

/* Allocation-free density statistics of a psi array in the CALLER's device
 * memory.  This entry point has no counterpart in the reference.  It is for
 * callers that may not allocate device memory while they run: an application
 * whose own pool or caching allocator owns the device memory, a time loop that
 * cannot take the implicit synchronisation of cudaMalloc/cudaFree, a fixed
 * memory budget.  Computes out[0] = sum |psi|^2, out[1] = max |psi|^2 and
 * out[2] = out[1] / (out[0]/sites) (max density over mean density; a NaN in
 * psi gives NaN) into `out`, 3 doubles of device memory, asynchronously on
 * `stream` (a cudaStream_t, NULL for the default stream).  psi: `sites`
 * complex values (dtype QX_C128 double2 or QX_C64 float2) inside one device
 * allocation of the current device; `out` likewise.  Scratch is a fixed
 * per-device array inside the library sized for at most QX_NOALLOC_MAX_SITES
 * sites; larger sizes are rejected.  The first call on a device looks up that
 * array's device address -- make it before any stream capture.  Calls that
 * overlap on the GPU share the scratch and race.
 * Errors: qx_noalloc_last_error(). */
#define QX_NOALLOC_MAX_SITES 134217728LL /* 512^3 */
int qx_rho_stats_noalloc(const void *psi, long long sites, int dtype, double *out, void *stream);
const char *qx_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
