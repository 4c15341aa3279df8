// A group of gfdtd simulations stepped together on one GPU (one set of
// launches and one persistent CG kernel per step for all of them).  A single
// simulation is a group of one.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "sim.hpp"
#include "tet.hpp"
#include "mlp.hpp"
#include "tet_group_kernels.cuh"

namespace tf {

class TetGroup {
 public:
  // sims: gfdtd simulations built on the host (TetSim(..., device = false)).
  // release_host frees their operator and complex arrays once laid out.
  TetGroup(std::vector<TetSim*> sims, const RunOptions& opt, bool release_host);
  ~TetGroup();
  TetGroup(const TetGroup&) = delete;
  TetGroup& operator=(const TetGroup&) = delete;

  int size() const { return (int)meta_.size(); }
  // advance every unfinished simulation by up to n steps; returns the steps
  // taken by the simulation that moved furthest
  uint64_t step(uint64_t n);
  // same, with CUDA events between the phases (ms5: H update + probes,
  // sources + rhs, CG, scatter, step end)
  uint64_t phase_times(uint64_t n, double* ms5);
  // one step of every member driven from host memory: car_in holds n_sources
  // values per member, probe_out n_probes * 6 per member (members in order);
  // members without a sample this step leave their slots untouched
  uint64_t step_io(const double* car_in, double* probe_out);
  size_t io_sources() const { return io_src_; }
  size_t io_probes() const { return io_probe_; }
  double last_step_ms() const { return last_ms_; }
  uint64_t step_index(int s) const { return meta_[s].step; }
  uint64_t n_steps(int s) const { return meta_[s].nsteps; }
  uint64_t nnz_A(int s) const { return meta_[s].nnz_a; }
  void get_state(int s, double* U, double* B, double* F);
  void set_state(int s, const double* U, const double* F);
  size_t n_samples(int s) const;
  void get_probes(int s, double* times, double* values, size_t cap) const;
  size_t solver_stats(int s, int32_t* iters, double* resid, size_t cap) const;
  size_t guess_stats(int s, int8_t* kept, size_t cap) const;
  size_t training_loss(float* loss, size_t cap) const;
  // current network parameters (kNParam floats); false without warm_start 3
  bool mlp_params(float* out) const;
  void get_flux(int s, double* flux, size_t cap, size_t* n) const;
  void get_losses(int s, double* loss, size_t cap, size_t* n) const;
  // leapfrog energy of member s on the GPU (see grp_energy)
  double energy(int s);
  uint64_t device_bytes() const { return dev_bytes_; }
  int kernels_per_step() const {
    return 7 + (dev_.np ? 1 : 0) + (opt_.warm_start == 3 ? 2 : 0) + (dev_.nsa ? 2 : 0);
  }
  int cg_blocks() const { return cg_blocks_; }
  int cg_variant() const { return cg_variant_; }
  uint64_t total_dofs() const { return dofs_; }
  uint64_t total_rows() const { return (uint64_t)dev_.nrow; }
  uint64_t nnz_A_stored() const { return nnz_a_; }
  uint64_t nnz_A() const { return nnz_a_real_; }
  const std::vector<int64_t>& seg_layout() const { return blk_seg_; }

 private:
  struct Meta {
    uint64_t nE = 0, nF = 0, nsteps = 0, step = 0, np = 0, nsrc = 0, nnz_a = 0;
    int64_t eoff = 0, foff = 0, roff = 0, stat_off = 0, samp_off = 0, car_off = 0;
    int64_t nrow_pad = 0, nface_pad = 0;  // the member's free rows and faces, padded to 32
    int nslots = 0;
    std::vector<int> slot_of_step;
    std::vector<double> sample_times;
  };
  template <typename T>
  void build(std::vector<TetSim*>& sims, bool release_host);
  void partition();
  void check_err();
  void launch(int n, cudaEvent_t* ev);
  void capture_graph(int len);
  void* dalloc(size_t bytes);
  template <typename V, typename A>
  void* upload(const std::vector<V, A>& v);

  RunOptions opt_;
  std::vector<Meta> meta_;
  GroupDev dev_{};
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::vector<void*> allocs_;
  std::vector<int64_t> blk_seg_;
  uint64_t dev_bytes_ = 0, dofs_ = 0, nnz_a_ = 0, nnz_a_real_ = 0;
  int cg_blocks_ = 0, cg_variant_ = 0;
  size_t cg_smem_ = 0;
  int tune_pos_ = 0;
  double tune_ms_[2] = {0, 0};
  double last_ms_ = 0;
  double* pinned_ = nullptr;
  double *dio_in_ = nullptr, *dio_out_ = nullptr;  // step_io staging on the device
  size_t pinned_len_ = 0, io_src_ = 0, io_probe_ = 0;
  std::vector<double> carrier_host_;
  std::vector<uint8_t> lossy_host_;  // member has conducting tets
  // learned warm start
  MlpTrain mlp_{};
  int64_t launched_ = 0;     // steps launched so far (group clock of the training schedule)
  int adam_step_ = 0;
  int64_t samp_n_ = 0, samp_stride_ = 1;
  float* loss_hist_ = nullptr;
  double* energy_part_ = nullptr;  // partial sums of grp_energy (allocated on first use)
  // captured step loop (see step())
  cudaGraphExec_t graph_exec_ = nullptr;
  int graph_len_ = 0;
  bool graph_failed_ = false;
 public:
  bool graph_active() const { return graph_exec_ != nullptr; }
 private:
  int64_t loss_cap_ = 0;  // per-simulation carrier tables (for step_io overrides)
};

}  // namespace tf
