// Common interface of the simulations the C ABI drives (Cartesian FIT and the
// tetrahedral dga / gfdtd paths).
#pragma once
#include <cstddef>
#include <cstdint>

#include "script.hpp"

namespace tf {

struct RunOptions {
  int precision = 0;        // 0 fp64, 1 fp32
  int device = 0;
  int graph_steps = 0;      // 0: automatic
  bool verbose = false;
  bool consistent_mass = false;  // gfdtd: corrected eps-mass (see tet.cpp)
  int warm_start = 0;       // gfdtd CG initial guess: 0 previous solution, 1 zero, 2 extrapolation, 3 learned
  int cg_criterion = 0;     // 0 ||r||/||r0|| <= tol (reference), 1 ||r|| <= tol ||b||
  int cg_maxiter = 100;
  // run the stability estimate even when the script pins the step (batches
  // turn it off: with a pinned step it only sets the possibly-unstable flag)
  bool estimate_pinned = true;
  // learned warm start (warm_start 3)
  int fit_variant = 0;        // fdtd: 0 autotune, k > 0 force kernel variant k - 1
  int learn_steps = 500;      // steps whose solutions train the network
  int learn_samples = 32768;  // sampled rows per training step
  int learn_inner = 2;        // Adam steps per training step
  float learn_rate = 1e-3f;
  int setup_threads = 0;      // host threads of one simulation's set-up (0: all)
};

class Sim {
 public:
  virtual ~Sim() = default;
  virtual int method() const = 0;  // 0 fdtd, 1 dga, 2 gfdtd
  virtual uint64_t step(uint64_t n) = 0;
  virtual uint64_t n_edges() const = 0;
  virtual uint64_t n_faces() const = 0;
  virtual uint64_t n_cells() const = 0;
  virtual uint64_t n_probes() const = 0;
  virtual uint64_t n_steps() const = 0;
  virtual uint64_t step_index() const = 0;
  virtual int nx() const { return 0; }
  virtual int ny() const { return 0; }
  virtual int nz() const { return 0; }
  virtual double dt() const = 0;
  virtual double dt_estimate() const = 0;
  virtual bool possibly_unstable() const = 0;
  virtual int precision() const = 0;
  virtual uint64_t device_bytes() const = 0;
  virtual double last_step_ms() const = 0;
  virtual const Output& output() const = 0;
  virtual const Simulation& simulation() const = 0;
  virtual size_t n_samples() const = 0;
  virtual double sample_time_shift() const = 0;  // H-column time offset in the probe files
  virtual void get_probes(double* times, double* values, size_t cap) const = 0;
  virtual void probe_points(double* xyz, uint64_t* cells, size_t cap) const = 0;
  virtual void get_state(double* U, double* B, double* F) = 0;
  virtual void set_state(const double* U, const double* F) = 0;
  virtual void get_flux(double* flux, size_t cap, size_t* n) const = 0;
  // Joule loss per step (Discretization.hpp:895, :1519, :1902).  Zero unless
  // the simulation conducts: dga accepts lossless materials only, gfdtd and
  // fem form it from SigMat, and the FIT path's conductance vector is
  // non-zero only for l2norm outputs, as in the reference.
  virtual void get_losses(double* loss, size_t cap, size_t* n) const {
    const uint64_t s = step_index();
    const size_t m = s < cap ? (size_t)s : cap;
    if (loss)
      for (size_t q = 0; q < m; q++) loss[q] = 0.0;
    if (n) *n = (size_t)s;
  }
  virtual double energy() = 0;
  virtual uint64_t phase_times(uint64_t n, double* ms5) = 0;
  virtual uint64_t step_io(const double* carrier_in, double* probe_out) = 0;
  virtual int kernels_per_step() const = 0;
  virtual size_t n_sources() const = 0;
  virtual uint64_t n_free() const { return 0; }
  virtual uint64_t nnz_system() const { return 0; }
  virtual uint64_t nnz_operators() const { return 0; }
  // kernel variant in use (see tf_info.cg_variant)
  virtual int kernel_variant() const { return 0; }
  // iterative solver statistics (gfdtd): iterations and final residual per step
  virtual size_t solver_stats(int32_t* iters, double* resid, size_t cap) const {
    (void)iters; (void)resid; (void)cap;
    return 0;
  }
  // learned warm start: per step 1 when the network's guess was kept
  virtual size_t guess_stats(int8_t* kept, size_t cap) const {
    (void)kept; (void)cap;
    return 0;
  }
  // learned warm start: training loss of every Adam step so far
  virtual size_t training_loss(float* loss, size_t cap) const {
    (void)loss; (void)cap;
    return 0;
  }
  // Tetrahedral mesh of the silo-mode field dumps: node coordinates and the
  // tets' node ids (0-based), each tet ordered as the reference's ExportMesh
  // writes it (Discretization.hpp:2354-2376).  False without a tet mesh.
  virtual bool mesh_arrays(std::vector<double>* xyz, std::vector<int32_t>* tets) const {
    (void)xyz; (void)tets;
    return false;
  }
};

}  // namespace tf
