// Cartesian FIT simulation: host setup in Yee index space and the device
// runtime that drives the kernels of fit_kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "fit_kernels.cuh"
#include "script.hpp"
#include "sim.hpp"

namespace tf {

// One special edge as built on the host (see SpecialEdges for the device form).
struct HostSpecial {
  int comp;
  int64_t slot;
  int op, kind;  // op: 0 hold, 1 explicit faces, 2 stencil with current; kind: 0 none 1 e 2 h 3 j
  int nface = 0;
  int fcomp[4] = {0, 0, 0, 0};
  int64_t fslot[4] = {0, 0, 0, 0};
  int fsign[4] = {0, 0, 0, 0};
  double mh = 0, mq = 0, post = 1.0;
  std::array<double, 3> vec{0, 0, 0};
  std::vector<uint32_t> srcs;  // source labels in the reference's edge_src order
};

class FitSim : public Sim {
 public:
  FitSim(Script& sc, uint32_t label, const RunOptions& opt);
  ~FitSim() override;
  int method() const override { return 0; }
  uint64_t step(uint64_t n) override;
  // accessors
  uint64_t n_edges() const override { return nE_; }
  uint64_t n_faces() const override { return nF_; }
  uint64_t n_cells() const override { return (uint64_t)Nx_ * Ny_ * Nz_; }
  uint64_t n_probes() const override { return probe_cell_.size(); }
  uint64_t n_steps() const override { return nsteps_; }
  uint64_t step_index() const override { return step_; }
  int nx() const override { return Nx_; }
  int ny() const override { return Ny_; }
  int nz() const override { return Nz_; }
  double dt() const override { return dt_; }
  double dt_estimate() const override { return dt_est_; }
  bool possibly_unstable() const override { return unstable_; }
  int precision() const override { return opt_.precision; }
  uint64_t device_bytes() const override { return dev_bytes_; }
  double last_step_ms() const override { return last_ms_; }
  const Output& output() const override { return out_; }
  size_t n_samples() const override;
  double sample_time_shift() const override { return -0.5 * dt_; }
  void get_probes(double* times, double* values, size_t cap) const override;
  void probe_points(double* xyz, uint64_t* cells, size_t cap) const override;
  void get_state(double* U, double* B, double* F) override;
  void set_state(const double* U, const double* F) override;
  void get_flux(double* flux, size_t cap, size_t* n) const override;
  void get_losses(double* loss, size_t cap, size_t* n) const override;
  double energy() override;
  uint64_t phase_times(uint64_t n, double* ms5) override;
  uint64_t step_io(const double* carrier_in, double* probe_out) override;
  int kernels_per_step() const override;
  int e_variant() const { return e_var_; }
  int h_variant() const { return h_var_; }
  size_t n_sources() const override { return src_labels_.size(); }
  const Simulation& simulation() const override { return sim_; }

 private:
  void setup_grid();
  void classify_edges();
  void locate_probes_and_dipoles();
  void build_tables();
  double estimate_dt();
  void alloc_device();
  void upload();
  void build_ref_maps();
  void launch_steps(int n, cudaEvent_t* ev = nullptr);
  void autotune(uint64_t& n);
  void check_tma();
  template <typename T>
  void fill_grid(FitGrid<T>& g, SpecialEdges<T>& s);

  Script& sc_;
  Simulation sim_;
  Output out_;
  RunOptions opt_;
  uint32_t label_;
  std::map<uint32_t, Solid> solids_;
  int Nx_ = 0, Ny_ = 0, Nz_ = 0;
  double L_[3] = {0, 0, 0}, lo_[3] = {0, 0, 0};
  std::vector<double> xs_[3];  // node coordinates by axis, accumulated as the reference sweeps
  int64_t sx_ = 0, sxy_ = 0, nslot_ = 0;
  uint64_t nE_ = 0, nF_ = 0;
  std::vector<uint8_t> mat_;            // compact material per cell
  std::vector<uint32_t> mat_label_;     // compact index -> material label
  uint32_t maxmat_ = 0;
  // per material tables, [m][3]
  std::vector<double> P_, S_, R_, X_, mh_pure_, mq_pure_, mnu_pure_, mmu_pure_, inv_mu_;
  std::vector<uint8_t> live_;
  std::vector<HostSpecial> special_;
  std::vector<uint32_t> src_labels_;    // simulation sources in order
  std::vector<std::array<int, 3>> probe_cell_;
  std::vector<std::array<double, 3>> probe_pts_;
  std::vector<int> slot_of_step_;
  int nslots_ = 0;
  std::vector<double> sample_times_;
  double dt_ = 0, dt_est_ = 0;
  bool unstable_ = false;
  uint64_t nsteps_ = 0, step_ = 0;
  double last_ms_ = 0;
  uint64_t dev_bytes_ = 0;
  // device
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::vector<void*> allocs_;
  void* dU_[3] = {nullptr, nullptr, nullptr};
  void* dF_[3] = {nullptr, nullptr, nullptr};
  uint8_t* dmat_ = nullptr;
  double *dP_ = nullptr, *dS_ = nullptr, *dR_ = nullptr, *dX_ = nullptr;
  void *dmh_ = nullptr, *dmq_ = nullptr, *dmnu_ = nullptr, *dmmu_ = nullptr;
  uint8_t* dlive_ = nullptr;
  int* dstep_ = nullptr;
  double* dflux_ = nullptr;
  double* dflux_part_ = nullptr;
  int nflux_part_ = 0;
  // Joule losses (l2norm outputs with conducting materials only)
  bool losses_on_ = false;
  void* dUold_[3] = {nullptr, nullptr, nullptr};
  double* dloss_ = nullptr;
  double* dloss_part_ = nullptr;
  int nloss_part_ = 0;
  // special edges (device SoA)
  int64_t* dsp_slot_ = nullptr;
  int8_t *dsp_comp_ = nullptr, *dsp_op_ = nullptr, *dsp_nface_ = nullptr, *dsp_fcomp_ = nullptr, *dsp_fsign_ = nullptr;
  int64_t* dsp_fslot_ = nullptr;
  double *dsp_mh_ = nullptr, *dsp_mq_ = nullptr, *dsp_vec_ = nullptr, *dsp_post_ = nullptr;
  int *dsp_begin_ = nullptr, *dsp_psrc_ = nullptr;
  double* dsp_pfac_ = nullptr;
  int8_t* dsp_pdir_ = nullptr;
  double *dsrc_amp_ = nullptr, *dcarrier_ = nullptr;
  int8_t* dsrc_kind_ = nullptr;
  void* dsp_out_ = nullptr;
  // probes
  int *dpi_ = nullptr, *dpj_ = nullptr, *dpk_ = nullptr, *dslot_ = nullptr;
  double *dinvmu_ = nullptr, *dsamples_ = nullptr;
  double* pinned_ = nullptr;  // host staging for step_io
  int e_var_ = 2, h_var_ = 2; // kernel variants (see fit_launch_step)
  bool tuned_ = false;
  int tune_pos_ = 0;
  double tune_e_[6] = {0, 0, 0, 0, 0, 0}, tune_h_[6] = {0, 0, 0, 0, 0, 0};
  FitTmaMaps tma_{};
  bool tma_ok_ = false;
  int* dtma_err_ = nullptr;
  void* dC_[12] = {};  // per-dof coefficients M_h, M_q, M_nu, M_mu x 3 axes (autotuned grids)
  uint16_t* dK_[6] = {};  // coefficient classes of the x, y, z edges, then faces
  void* dlut_[2] = {};    // class tables (edges, faces)
  bool cls_ok_ = false;
  int ncls_[2] = {0, 0};  // edge and face classes (-1: more than the tables hold)
  void build_coefficients();

 public:
  int kernel_variant() const override { return e_var_ + 8 * h_var_; }

 private:
  // graphs
  cudaGraphExec_t graph_ = nullptr;
  int graph_len_ = 0;
  // reference numbering maps (built on demand): comp << 60 | slot
  std::vector<int64_t> edge_map_, face_map_;
};

}  // namespace tf
