// Host-side interface of the device solver (one simulation on one GPU).
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace hydft {

struct Phys;  // kernels.cuh

// Everything the solver needs, computed by the host setup (setup.cpp).
struct SolverSetup {
    Grid g;
    int nm = 1;                       // momentum components evolved (= ndim)
    // physics constants (mirrors Phys in kernels.cuh)
    double beta = 3, mass = 1, n0 = 0;
    int term_order[8] = {0};
    int nterms_local = 0;
    double cn = 0, cg = 0, alpha_ref = 0;
    int evolve = 0, newtonian = 0;
    double eta = 0, xi = 0, tau = 0;
    int ext_active = 0, ext_kind = 0, ext_td = 0;
    double ext_k[3] = {0, 0, 0}, ext_amp = 0, ext_omega = 0, ext_ramp = 0;
    int drive_in_band = 0, drive_idx = 0, drive_conj = 0;
    double volume = 1;
    std::vector<double> klin;         // compact band, sum of hartree/ry mu kernels
    std::vector<double> fdtab;        // 6*6601, electrons only
    std::vector<std::complex<double>> ex, ey, ez;
    std::vector<double> gauss_v;      // gaussian external potential on the grid (ext_kind 3)
    // free energy (functional_t%energy): term ids in input order (1 ideal,
    // 2 tf, 3 gradient, 4 hartree, 5 ry), hartree v(k) and RY c_cor(k) on
    // the compact band, and both at k = 0
    int eterm_order[8] = {0};
    int neterms = 0;
    std::vector<double> kh, kr;
    double vk0 = 0, ck0 = 0;
};

struct KernelStat {
    std::string name;
    double ms = 0.0;      // total device time of the launches (CUDA events)
    double bytes = 0.0;   // total algorithmic bytes of the launches
    int64_t n = 0;        // launches
};

// One kernel launch of a step in the form an ensemble replays it: the
// kernel (kind identifies its pack type), its launch shape for one
// simulation, and the launch arguments (the pack) as bytes.  An ensemble
// groups simulations whose steps record the same kinds and shapes, copies
// their packs into one device table per launch and runs each launch once
// for the whole group (ensemble_kernel in common.cuh).
struct LaunchRec {
    const void *kind = nullptr;
    const char *name = nullptr;
    double bytes = 0.0;
    dim3 grid, block;
    size_t smem = 0;
    std::vector<unsigned char> pack;
    unsigned per_launch = 1;          // simulations one launch of the ensemble form carries
    // the ensemble form for n simulations whose packs lie back to back at
    // `packs` (host memory; they travel as kernel parameters)
    void (*launch)(const void *packs, unsigned n, dim3 grid, dim3 block, size_t smem, cudaStream_t st) = nullptr;
    // raises the ensemble form's dynamic shared-memory limit to smem
    cudaError_t (*prepare)(size_t smem) = nullptr;
};

class SolverBase {
public:
    virtual ~SolverBase() {}
    virtual int set_state(const double *n, const double *mom, const double *pi) = 0;
    virtual int get_state(double *n, double *mom, double *pi) = 0;
    virtual int advance(int nsteps) = 0;
    virtual int rhs(double t, double *dn, double *dmom, double *dpi) = 0;
    // FP64 compensated sums over the grid
    virtual int reductions(double *sum_n, double sum_m[3], double *sum_m2n, double *nmin,
                           double *nmax, double *umax) = 0;
    virtual int mode(int field, int mx, int my, int mz, double *re, double *im) = 0;
    // functional_t%energy plus the external-potential energy of the current
    // state (diagnostics.f90:41-60), FP64
    virtual int energy(double *fe) = 0;
    virtual void set_time(double t, double dt) = 0;
    virtual void get_time(double *t, double *dt, int64_t *step) = 0;
    virtual void *stream() = 0;
    virtual int precision_bits() const = 0;
    // drive frequency of the external potential (model_t%ext%omega); the
    // captured step graph is rebuilt on the next advance
    virtual void set_ext_omega(double w) = 0;
    // nsteps uncaptured steps with CUDA events around every launch
    virtual int profile(int nsteps, std::vector<KernelStat> &out) = 0;
    // the host-side setup constants in use
    virtual const SolverSetup &setup() const = 0;
    // Enqueues k RK3 steps on this solver's stream without capturing,
    // launching a graph or synchronising (an ensemble captures the steps of
    // many solvers into one graph through this call).
    virtual void enqueue_steps(int k) = 0;
    // picks the tile shapes (autotuner) if not done yet; must precede a
    // capture of enqueue_steps
    virtual int prepare() = 0;
    // tile shapes in use: kx columns and threads per y/z block of the
    // inverse passes, the same of the forward passes, threads per x block
    virtual void tiles(int *t5) const = 0;
    // radix plan of axis 0/1/2 as decimal digits (843: radix 8, 4, 3),
    // negative when the autotuner did not choose it
    virtual int radix_code(int axis) const = 0;
    // axes whose passes classify band elements at compile time (x 1, y 2, z 4)
    virtual int band_axes() const = 0;
    // Records the launches of one RK3 step (after tuning) without running
    // them.  Returns HYDFT_ERR_UNSUPPORTED, with out empty, when a launch of
    // the step has no ensemble form (that simulation then steps on its own).
    virtual int record_step(std::vector<LaunchRec> &out) = 0;
    // records that steps enqueued earlier (a replayed ensemble graph) ran
    virtual void mark_advanced() = 0;
    // k replays of the captured step graph on this solver's stream, without
    // waiting for them or reading the status word (poll_status does that)
    virtual int launch_steps(int k) = 0;
    // waits for this solver's stream and turns its status word into a code
    virtual int poll_status() = 0;
    // bytes of device memory this solver allocated
    virtual size_t device_bytes() const = 0;
    virtual void set_step(int64_t step) = 0;
    // Probes (diag_t%probe, diagnostics.f90:70-77) recorded on the device:
    // probe_setup picks the Fourier mode; launch_steps_probed runs k steps
    // (graph replays) and after every step whose number is a multiple of
    // `every` stores t and the n and mom_x coefficients of the mode (5
    // doubles) in a device ring of probe_capacity() entries, read back and
    // cleared by read_probes.
    virtual int probe_setup(int mx, int my, int mz) = 0;
    virtual int probe_capacity() const = 0;
    virtual int launch_steps_probed(int k, int every) = 0;
    virtual int read_probes(std::vector<double> &out) = 0;
    // device address of the status word the step kernels set (ST_* bits)
    virtual const unsigned *status_word() const = 0;
    // turns status bits read from status_word() into an error code and
    // message, and clears the device word; 0 if stv is 0
    virtual int take_status(unsigned stv) = 0;
    int64_t launches = 0;
    int64_t graph_gen = 0;   // bumped when values baked into captured steps change
    std::string err;
};

// precision: 64 or 32.  Returns nullptr and fills err on failure.
SolverBase *make_solver(const SolverSetup &s, int precision, int device, std::string &err);

}  // namespace hydft
