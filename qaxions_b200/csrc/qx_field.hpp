// qx_field.hpp -- C++ host mirror of the reference's Field / FFTBackend
// operator surface, driving the sm_100a kernels on one CUDA stream.
//
//   reference                                  here
//   FFTBackend (src/fft/fft.h:9-26)            qx::FFTBackend (device buffers)
//   FFTWOpenMPBackend (src/fft/fft.h:28-149)   qx::B200FFTBackend<R>
//   Field (src/field.h:13-97)                  qx::Field (abstract) / qx::FieldT<R>
//
// R = double is the plain FP64 (complex128) form; R = float is the fused FP32
// (complex64) form, whose phase arguments, reductions and spectrum sums stay
// FP64.  Device buffers are owned by the field; host data moves only through
// set_*/get_* copies.  A field is bound to one stream and is not thread-safe.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "qx_mixed.hpp"
#include "qx_ops.hpp"

namespace qx {

enum class Prec { F64 = 0, F32 = 1 };
enum class K0 { Reference = 0, Zero = 1 };

struct FieldConfig {
    int dim = 3;
    int N = 64;
    double L = 1.0;
    double pref = 1.0;      // Poisson source prefactor (reference: norm_ * a_, src/field.cxx:298)
    double rho_mean = 1.0;  // background density (src/field.cxx:77)
    Prec prec = Prec::F64;
    K0 k0 = K0::Reference;
    double dt = 1e-4;       // ds_ used by half_kick/full_kick/drift_update/step
    int device = -1;        // CUDA device (-1: current)
    int batch = 1;          // boxes of this size stacked in one array (an ensemble group)
};

// Device-side FFT plugin: in-place c2c, r2c into the packed half spectrum,
// c2r from it (input overwritten), all unnormalised with FFTW's sign
// conventions.  ksites() is the packed size N^(d-1) N/2: column 0 carries the
// kx = 0 and kx = N/2 planes as A + iB.
class FFTBackend {
  public:
    virtual ~FFTBackend() = default;
    virtual void forward_c2c(void* data) = 0;
    virtual void backward_c2c(void* data) = 0;
    virtual void forward_r2c(void* in_real, void* out_half) = 0;
    virtual void backward_c2r(void* in_half, void* out_real) = 0;
    virtual size_t sites() const = 0;
    virtual size_t ksites() const = 0;
    virtual bool owns_zero_mode() const { return true; }
    virtual bool owns_zero_mode_k() const { return true; }
    virtual ptrdiff_t global_N() const = 0;
};

// S, rows and hsites count every box of a batched field; S1 is one box
struct Geometry {
    int dim, N;
    long S, rows, hsites;
    int B = 1;
    long S1 = 0;
    long fftw_ksites() const { return rows * (N / 2 + 1); }
};

// device twiddle tables for L = N and N/2: the FFT passes read stage-major
// tables (Ops::stage_twiddles), with the low parts (exact - table) used by the
// FP32 form's double-float twiddles; the r2c/c2r pre/post-processing reads the
// natural-order table exp(-2 pi i k/N)
template <typename C> struct TwTables {
    const C* N;
    const C* M;
    const C* N_lo;
    const C* M_lo;
    const C* N_nat;
    // N-point stage-major tables of radix plan 1 (qx_with_plan) for the TMA
    // strided passes, where the grid has that plan (else null)
    const C* N_p1;
    const C* N_p1_lo;
};

template <typename R>
class B200FFTBackend : public FFTBackend {
  public:
    using C = typename Ops<R>::C;
    B200FFTBackend(const Geometry& g, const TwTables<C>& tw, const Tune* tune, cudaStream_t st, int* err)
        : g_(g), tw_(tw), tune_(tune), st_(st), err_(err) {}
    void forward_c2c(void* data) override;
    void backward_c2c(void* data) override;
    void forward_r2c(void* in_real, void* out_half) override;
    void backward_c2r(void* in_half, void* out_real) override;
    size_t sites() const override { return (size_t)g_.S; }
    size_t ksites() const override { return (size_t)g_.hsites; }
    ptrdiff_t global_N() const override { return g_.N; }
    // out-of-place forward c2c along all axes except the last, used by the
    // kinetic-energy measurement (last axis fused with the reduction)
    void forward_c2c_partial(const C* in, C* out);

  private:
    Geometry g_;
    TwTables<C> tw_;
    const Tune* tune_;
    cudaStream_t st_;
    int* err_;  // device flag raised by a timed-out wait in a pass kernel
};

// MeasureType bits (src/enum.h:39-47) plus this library's own
enum MeasBits : unsigned {
    MEAS_NONE = 0,
    MEAS_SPECTRUM = 1u << 0,   // spec_NNNN.txt of |psi|^2, reference shells
    MEAS_RHO_MAX = 1u << 1,    // (rhomax is measured whenever the mask is not NONE)
    MEAS_RHO_SLICE = 1u << 2,  // enumerated by the reference, not acted on by its measure()
    MEAS_RHO_GRID = 1u << 3,   // field_NNNN.rho (raw FP64 density) + field_NNNN.json header
    MEAS_PSI_GRID = 1u << 4,   // enumerated by the reference, not acted on by its measure()
    MEAS_ENERGY = 1u << 8,     // mass, kinetic and potential energy (no reference counterpart)
    MEAS_CLOBBER_V = 1u << 9,  // reproduce the reference's V <- |psi|^2 before the next kick
};

// one measurement (the quantities measure()/printStatus report, plus ours)
struct MeasRecord {
    int number = 0;      // measurement number (0: before the time loop)
    int step = 0;        // Field::curr()
    double time = 0.0;   // Field::time()
    double a = 1.0;      // Field::a()
    double rhomax = 0.0; // computeEnergy: max |psi|^2 / mean |psi|^2
    double vmax = 0.0;   // max |V| of the potential of this psi
    double mass = 0.0, energy = 0.0, kinetic = 0.0, potential = 0.0;  // MEAS_ENERGY, else NaN
};

// generateMeasList (src/utils.cxx:8-28): the loop indices after whose
// drift_update a measurement is taken
std::vector<long> meas_list(long nsteps, long nmeas);

class Field {
  public:
    virtual ~Field() = default;

    // ---- reference operator surface (src/field.h:24-34) ----
    virtual void kick(double dt) = 0;
    virtual void drift(double dt) = 0;
    virtual void Poisson() = 0;           // on the transformed packed V^ (after forward_r2c)
    virtual void updatePotential() = 0;
    virtual void computeEnergy() = 0;     // reference semantics: V <- |psi|^2, rhomax
    void updateTime();
    // 0: STATIC (a = 1); 1: MRE from a = ai (src/field.cxx:70-90, 349-361)
    void set_cosmology(int cosmo, double ai);
    int cosmology() const { return cosmo_; }
    void half_kick() { kick(0.5 * ds_); }
    void full_kick() { kick(ds_); }
    void drift_update();
    void propagate();
    // merged leapfrog of src/main.cxx:64-85 (measurements off), fused passes,
    // loop body replayed from a CUDA graph
    virtual void step(int nsteps) = 0;
    // step() in pieces, for a caller that replays several fields' loop bodies
    // in one CUDA graph of its own (an ensemble; STATIC cosmology): the
    // prologue, one loop body on the field's stream (last: the final body,
    // ending in the half kick), the clock advance of nsteps, and what a
    // replay of a captured body needs first (the drift factor tables of ds)
    virtual void step_begin() = 0;
    virtual void enqueue_body(bool last) = 0;
    virtual void step_end(int nsteps) = 0;
    virtual void prepare_replay() = 0;
    // the device arrays, tables and loop-body constants one pass launch over
    // several fields of different sizes needs (3D; after prepare_replay)
    virtual void mix_desc(MixDesc& d) = 0;
    // measure() (src/meas.cxx:13-63) without overwriting V (unless the mask
    // has MEAS_CLOBBER_V); files go to `dir` when it is not null
    virtual void measure(unsigned mask, int number, const char* dir, MeasRecord* rec) = 0;
    // the time loop of main() (src/main.cxx:64-85) with its measurements:
    // measure(0), then one measurement after the drift_update of every loop
    // index of meas_list(nsteps, nmeas); records in `out`
    virtual void run(int nsteps, int nmeas, unsigned mask, const char* dir, std::vector<MeasRecord>& out) = 0;

    // ---- buffers (host FP64, reference index order) ----
    virtual void set_psi(const double* interleaved) = 0;
    virtual void get_psi(double* interleaved) = 0;
    virtual void set_V(const double* v) = 0;
    virtual void get_V(double* v) = 0;
    virtual void get_Vhat(double* fftw_half) = 0;   // unpacked to FFTW's N/2+1 layout
    virtual void set_Vhat(const double* fftw_half) = 0;

    // ---- FFT plugin on host buffers ----
    virtual void host_c2c(double* data, int sign) = 0;
    virtual void host_r2c(const double* in, double* out_fftw_half) = 0;
    virtual void host_c2r(const double* in_fftw_half, double* out) = 0;
    virtual FFTBackend* fftBackend() = 0;

    // ---- measurements (non-destructive) ----
    virtual void rho_stats(double* rhomax, double* vmax) = 0;
    virtual void mass_energy(double* M, double* E, double* K, double* W) = 0;
    // shell-binned spectrum; source 0 = |psi|^2, 1 = V
    virtual void spectrum(int source, int mode, int nbins, double* k, double* P, long long* count) = 0;

    // ---- initial conditions (generated in FP64 on the device) ----
    virtual void ic_gaussian_solitons(int n, const double* rows5, double bkg) = 0;
    virtual void ic_config(int kind, uint64_t seed, int n_sol, double rc_lo, double rc_hi, double sigma,
                           double kc_factor, double clip, double rho0) = 0;

    // ---- boxes of a batched field (batch > 1: an ensemble group) ----
    int batch() const { return g_.B; }
    virtual void ic_config_box(int box, int kind, uint64_t seed, int n_sol, double rc_lo, double rc_hi,
                               double sigma, double kc_factor, double clip, double rho0) = 0;
    virtual void set_psi_box(int box, const double* interleaved) = 0;
    virtual void get_psi_box(int box, double* interleaved) = 0;
    virtual void box_mass(double* M) = 0;  // per-box sum |psi|^2 dV

    // ---- timing / device access ----
    virtual float time_steps(int nsteps, int use_graph) = 0;  // device ms of step(nsteps)
    // Autotuner: time `nsteps` steps under each candidate launch geometry, keep
    // the fastest (psi is restored afterwards).  Results are cached per (dim,
    // N, precision, batch) in the process and, if `cache_path` is given, in
    // that text file (read before tuning, appended after).  Returns the best
    // ms per step; `from_cache` tells whether no timing was needed.
    virtual double autotune(int nsteps, const char* cache_path, bool* from_cache) = 0;
    virtual void profile_step(int nsteps, std::vector<std::pair<std::string, double>>& per_kernel_ms) = 0;
    virtual void* psi_device() = 0;
    // psi was changed in place through psi_device(): drop derived state (V)
    virtual void psi_changed() = 0;
    virtual void scale_psi(double factor) = 0;
    virtual void* V_device() = 0;
    virtual void sync() = 0;
    cudaStream_t stream() const { return st_; }

    // ---- scalars ----
    const FieldConfig& config() const { return cfg_; }
    const Geometry& geom() const { return g_; }
    int size() const { return cfg_.N; }
    int dim() const { return cfg_.dim; }
    double Lbox() const { return cfg_.L; }
    size_t sites() const { return (size_t)g_.S; }
    size_t ksites() const { return (size_t)g_.fftw_ksites(); }
    double Vmax() { return vmax_; }
    double rhomax() const { return rhomax_; }
    double rho_mean() const { return cfg_.rho_mean; }
    int curr() const { return curr_; }
    double time() const { return s_; }
    double a() const { return a_; }
    double dt() const { return ds_; }
    void set_dt(double dt) { ds_ = dt; }
    // restore the scale factor and time step of a checkpoint (after
    // set_cosmology, which resets them to the start of the cosmology)
    void restore_cosmology(double a, double ds) {
        a_ = a;
        ds_ = ds;
        invalidate_graph();
    }
    // restore the step counter and time of a checkpoint
    void set_clock(int step, double time) {
        curr_ = step;
        s_ = time;
    }
    Tune& tune() { return tune_; }
    // whether construction applied a geometry from the autotuner's cache
    virtual bool tuned_from_cache() const = 0;
    // drop the captured loop-body graph (after launch geometry changes)
    virtual void invalidate_graph() = 0;

  protected:
    FieldConfig cfg_;
    Geometry g_{};
    cudaStream_t st_ = nullptr;
    Tune tune_;
    int curr_ = 0;
    double s_ = 0.0, a_ = 1.0, ds_ = 0.0;
    double vmax_ = 0.0, rhomax_ = 0.0;
    int cosmo_ = 0;
};

std::unique_ptr<Field> make_field(const FieldConfig& cfg);

// forget the autotuner's in-process choices (files are left alone)
void clear_tune_cache();

// host-side conversion between FFTW's r2c layout and the packed layout
void pack_half(int dim, int N, const double* fftw_half, double* packed);
void unpack_half(int dim, int N, const double* packed, double* fftw_half);

// spectrum bin of every integer |n|^2 (mode 0 reference shells, 1 linear, 2 log)
std::vector<int> spectrum_bin_table(int dim, int N, int mode, int nbins);
std::vector<double> spectrum_k_axis(int N, int mode, int nbins, double L);

}  // namespace qx
