// Tetrahedral DGA simulations ("method dga" explicit, "method gfdtd" with the
// conjugate-gradient eps-mass solve): host set-up of the complex and operators
// and the device runtime driving tet_kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "host_parallel.hpp"
#include "script.hpp"
#include "sim.hpp"
#include "tet_kernels.cuh"

namespace tf {

class TetGroup;

// CSR on the host (int32 columns, double values), duplicates summed in
// insertion order.
struct HostCsr {
  uint32_t nrows = 0, ncols = 0;
  std::vector<int64_t> ptr;
  std::vector<int32_t> col;
  std::vector<double> val;
  struct Trip {
    uint32_t r, c;
    double v;
  };
  using Trips = std::vector<Trip, default_init_allocator<Trip>>;
  // threads: host threads for the per-row work (<= 0: all); t is consumed
  static HostCsr build(uint32_t nr, uint32_t nc, Trips& t, int threads = 1);
  void mul(const double* x, double* y, int threads = 1) const;
};

class TetSim : public Sim {
 public:
  // device = false builds the complex, operators, probes and source tables on
  // the host only (a batch lays several of them out in one device image)
  TetSim(Script& sc, uint32_t label, const RunOptions& opt, bool device = true);
  ~TetSim() override;
  int method() const override { return method_; }
  uint64_t step(uint64_t n) override;
  uint64_t n_edges() const override { return edges_.size(); }
  uint64_t n_faces() const override { return faces_.size(); }
  uint64_t n_cells() const override { return vols_.size(); }
  uint64_t n_probes() const override { return probe_tet_.size(); }
  uint64_t n_steps() const override { return nsteps_; }
  uint64_t step_index() const override { return step_; }
  double dt() const override { return dt_; }
  double dt_estimate() const override { return dt_est_; }
  bool possibly_unstable() const override { return unstable_; }
  int precision() const override { return opt_.precision; }
  uint64_t device_bytes() const override;
  double last_step_ms() const override;
  const Output& output() const override { return out_; }
  const Simulation& simulation() const override { return sim_; }
  size_t n_samples() const override;
  double sample_time_shift() const override { return method_ >= 2 ? 0.5 * dt_ : -0.5 * dt_; }
  void get_probes(double* times, double* values, size_t cap) const override;
  void probe_points(double* xyz, uint64_t* cells, size_t cap) const override;
  void get_state(double* U, double* B, double* F) override;
  void set_state(const double* U, const double* F) override;
  void get_flux(double* flux, size_t cap, size_t* n) const override;
  double energy() override;
  uint64_t phase_times(uint64_t n, double* ms5) override;
  uint64_t step_io(const double* carrier_in, double* probe_out) override;
  int kernels_per_step() const override;
  size_t n_sources() const override { return src_labels_.size(); }
  size_t solver_stats(int32_t* iters, double* resid, size_t cap) const override;
  size_t guess_stats(int8_t* kept, size_t cap) const override;
  int kernel_variant() const override;
  size_t training_loss(float* loss, size_t cap) const override;
  bool mesh_arrays(std::vector<double>* xyz, std::vector<int32_t>* tets) const override;
  void get_losses(double* loss, size_t cap, size_t* n) const override;
  uint64_t n_free() const override { return free_edges_.size(); }
  uint64_t nnz_system() const override { return A_.val.size(); }
  // nonzeros of the step's main operator: H (dga) or E (gfdtd)
  uint64_t nnz_operators() const override { return method_ == 1 ? H_.val.size() : E_.val.size(); }
  // frees the complex and operator arrays once a group has laid them out
  void release_host();

 private:
  void read_mesh();
  void classify();
  void build_ops();
  void split_system(double scale, double sig_coef = 0.0);
  bool dt_estimate_needed() const;
  double estimate_dt(const HostCsr& Minv_or_E, bool generalized);
  void locate_probes();
  void build_sources();
  void alloc_and_upload();
  friend class TetGroup;
  void launch_steps(int n, cudaEvent_t* ev);
  std::array<int32_t, 6> vol_edges(uint32_t v) const;

  Script& sc_;
  Simulation sim_;
  Output out_;
  RunOptions opt_;
  uint32_t label_;
  int method_ = 2;
  // complex
  std::vector<std::array<double, 3>> pts_;
  std::vector<std::array<int32_t, 4>> vols_;
  std::vector<uint32_t> vol_mat_;
  std::vector<double> cell_vol_;
  std::vector<std::array<int32_t, 3>> faces_;      // sorted node triples
  std::vector<std::array<int32_t, 2>> edges_;      // sorted node pairs
  std::vector<std::array<int32_t, 4>> vtf_;        // faces opposite nodes 0..3 (bcd, acd, abd, abc)
  std::vector<std::array<int32_t, 2>> ftv_;        // tets of a face (-1 if none)
  std::vector<std::array<int32_t, 3>> fte_;        // edges p0p1, p0p2, p1p2 (signs +, -, +)
  std::vector<int64_t> star_ptr_;                  // node -> incident edges (ascending)
  std::vector<int32_t> star_edge_;
  std::vector<int64_t> nvol_ptr_;                  // node -> incident tets (ascending)
  std::vector<int32_t> nvol_;
  std::vector<int32_t> bnd_edge_;                  // edge -> boundary dual index or -1
  std::vector<std::array<double, 3>> bnd_dual_;
  std::vector<uint8_t> cls_;                       // 1 interior dof, 4 Dirichlet; dga with
                                                   // conducting tets: 2 uniformly conducting,
                                                   // 3 fractured
  // dga with conducting tets: class-1 and class-2 rows share H_ (U = P U +
  // dt H cf, P = 1 on class 1); fractured edges sum two node-star fractions
  // U_c, which step as U_c = Q U_c_old + dt Mq cf
  bool dga_frac_ = false;                          // some edge of class 2 or 3
  std::vector<double> hp_;                         // P per edge (dga_frac_ only)
  HostCsr Q_, Mq_;                                 // U_c rows
  std::vector<int64_t> frac_off_;                  // node -> U_c offset, -1 if not fractured
  uint32_t q_size_ = 0;
  std::vector<int32_t> fe_edge_, fe_a_, fe_b_;     // fractured edges and their two U_c entries
  std::vector<double> nr_;                         // dga with chi: R per face (F = R F - dt N cu)
  // dga energy (tf_energy), set up on the first call: the class-1 edges, the
  // class-1 block of H in FP64 with its PCG work, and the partial sums
  DevPtrs en_cg_;
  int en_blocks_ = 0, en_n_ = 0;
  int32_t* en_edges_ = nullptr;
  double *en_part_ = nullptr, *en_out_ = nullptr;
  double dga_energy();
  std::vector<uint8_t> pec_;
  std::vector<std::vector<uint32_t>> edge_src_;
  // operators
  HostCsr Ct_;                                     // E x F, +-1 (C transposed)
  HostCsr N_, H_, E_, A_, R_;                      // R_: SysMat, free rows x Dirichlet cols
  HostCsr Sig_;                                    // conductivity mass SigMat (gfdtd, fem; lossy_ only)
  bool lossy_ = false;                             // some tet conducts
  std::vector<int32_t> free_edges_, dir_edges_;
  std::vector<double> jacobi_;
  // sources
  std::vector<uint32_t> src_labels_;
  std::vector<int32_t> src_edge_;                  // source-driven edges
  std::vector<int8_t> src_kind_e_;                 // 1 e, 2 h, 3 j
  std::vector<int> src_begin_;
  std::vector<int> pair_src_;
  std::vector<double> pair_fac_;
  std::vector<int8_t> pair_dir_;
  std::vector<double> src_vec_, src_post_;
  std::vector<double> carrier_, src_amp_;
  std::vector<int8_t> src_kind_;
  std::vector<double> init_U_, init_I_, init_src_;  // state at t = 0
  // probes
  std::vector<int32_t> probe_tet_;
  std::vector<std::array<double, 3>> probe_pts_;
  std::vector<double> probe_we_, probe_hf_;        // [p][6][3] Whitney weights, [p][4][3] flux weights
  std::vector<int> slot_of_step_;
  std::vector<double> sample_times_;
  int nslots_ = 0;
  double dt_ = 0, dt_est_ = 0;
  bool unstable_ = false;
  uint64_t nsteps_ = 0, step_ = 0;
  double last_ms_ = 0;
  uint64_t dev_bytes_ = 0;
  // device
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::vector<void*> allocs_;
  DevPtrs dp_{};
  double* pinned_ = nullptr;
  // gfdtd runs on the group engine (a group of one simulation)
  std::unique_ptr<TetGroup> group_;
};

}  // namespace tf
