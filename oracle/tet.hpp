// ORACLE — test infrastructure only.  FP64 CPU restatement of TetFIT's
// tetrahedral DGA paths ("method dga" explicit, "method gfdtd" and "method
// fem" with the Jacobi-PCG solve); see tet.cpp for the reference lines
// followed.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "script.hpp"

namespace orc {

// Compressed sparse rows with duplicates summed in insertion order, the way
// Eigen's setFromTriplets(..., add) assembles (columns ascending per row).
struct Csr {
  uint32_t nrows = 0, ncols = 0;
  std::vector<uint64_t> ptr;
  std::vector<uint32_t> col;
  std::vector<double> val;
  struct Trip {
    uint32_t r, c;
    double v;
  };
  static Csr build(uint32_t nr, uint32_t nc, const std::vector<Trip>& t);
  void mul(const double* x, double* y) const;          // y = A x
  void mul_t(const double* x, double* y) const;        // y = A^T x (A^T built on the fly)
  double diag(uint32_t i) const;
};

struct TetOracle {
  Script sc;
  Simulation sim;
  Output out;
  uint32_t sim_label = 0;
  int method = 1;  // 1 dga, 2 gfdtd, 3 fem
  // mesh and complex (reference numbering: sorted unique faces/edges)
  std::vector<std::array<double, 3>> pts;
  std::vector<std::array<uint32_t, 4>> vols;
  std::vector<uint32_t> vol_mat;
  std::vector<double> cell_vol;
  std::vector<std::array<uint32_t, 3>> faces;
  std::vector<std::array<uint32_t, 2>> edges;
  std::vector<std::array<std::pair<uint32_t, int>, 4>> vtf;
  std::vector<std::vector<std::pair<uint32_t, int>>> ftv;
  std::vector<std::array<std::pair<uint32_t, int>, 3>> fte;
  std::vector<std::vector<std::pair<uint32_t, int>>> nte;
  std::vector<std::vector<uint32_t>> node_vols;
  std::vector<uint64_t> boundary_face;
  std::vector<int32_t> bnd_edges;
  std::vector<std::array<double, 3>> bnd_dual;
  std::vector<uint32_t> edge_bcs;
  std::vector<std::vector<uint32_t>> edge_src;
  std::vector<uint8_t> is_pec, cls;  // cls: 1 interior dof, 4 Dirichlet (PEC or e-source); dga
                                     // also 2 (uniformly conducting) and 3 (fractured)
  Csr C;                               // F x E, +-1
  // operators
  Csr N;                               // F x F
  Csr H;                               // E x E, rows of class-1 and class-2 edges (dga; view of Ha, Mp)
  // dga with conductivity (Discretization.hpp:6776-6903, 9262-9475): U is M
  // times U_frac = [U_a (class 1), U_b (class 2), U_c (node-star fractions)]
  std::vector<uint32_t> h_index, p_index;  // edge -> row of Ha / Mp (0 when not of that class)
  std::vector<uint32_t> dual_frac;         // node -> U_c offset + 1 (0: not fractured)
  std::vector<std::array<uint32_t, 2>> frac_cols;  // class-3 edge -> its two U_c entries
  uint32_t H_size = 0, P_size = 0, Q_size = 0;
  Csr Ha, Mp, Q, Mq;                   // H_size x E, P_size x E, Q_size x Q_size, Q_size x E
  std::vector<double> P_p, U_a, U_b, U_c, U_c_old;
  // dga with magnetic losses (face classes, :6357-6542, 9128-9205): F is T
  // times F_frac = [F_a (class-1 faces, rows of Na), F_b (class-2, rows of Tr)]
  std::vector<uint8_t> fcls;               // face -> 1 (chi = 0) or 2 (chi, uniform across it)
  std::vector<uint32_t> n_index, r_index;  // face -> row of Na / Tr
  uint32_t N_size = 0, R_size = 0;
  Csr Na, Tr;                              // N_size x F, R_size x F
  Csr Nv;                                  // F x F view: the Na or Tr row of each face
  std::vector<double> R_r, F_a, F_b;
  Csr E;                               // E x E eps mass (gfdtd: node-star dual basis; fem: Whitney)
  Csr Sig;                             // E x E conductivity mass (SigMat), same construction with sigma
  bool lossy = false;                  // some tet conducts (sigma with non-zero determinant)
  std::vector<double> losses;          // poynting.dat third column entries (gfdtd, fem)
  Csr A, RHS1;                         // free x free system; E(free rows, Dirichlet cols)
  std::vector<int64_t> free_index;     // edge -> compressed free index or -1
  std::vector<uint32_t> free_edges;
  std::vector<double> jacobi;
  double dt = 0, dt_estimate = 0;
  bool possibly_unstable = false;
  // state
  std::vector<double> U, I, F, B, Fb, Fb_old, U_old, U_older, SrcFld, solution;
  uint32_t root = 0;
  std::vector<uint32_t> probe_elem;
  std::vector<std::array<double, 3>> probe_pts;
  std::vector<double> times, samples, flux;
  std::vector<int> cg_iters;
  std::vector<double> cg_err;
  uint64_t step_index = 0, nsteps_total = 0;
  int cg_maxiter = 100;
  bool consistent_mass = false;  // gfdtd: corrected eps-mass (see tet.cpp)

  void prepare(uint32_t label);
  uint64_t step(uint64_t n);
  // helpers shared with the C ABI
  std::array<double, 3> edge_bar(uint32_t e) const;
  std::array<double, 3> face_bar(uint32_t f) const;
  std::array<double, 3> vol_bar(uint32_t v) const;

 private:
  void read_mesh();
  void build_dga();
  void classify_dga();
  void build_gfdtd();
  void build_fem();
  void split_system(double scale, double sig_coef = 0.0);
  void push_loss_pre(const std::vector<double>& su);
  void push_loss_post();
  std::array<uint32_t, 6> vol_edges(uint32_t v) const;
  std::array<std::array<double, 3>, 6> dual_area_vectors(uint32_t v) const;
  std::array<std::array<double, 3>, 4> primal_area_vectors(uint32_t v) const;
  void local_M(uint32_t v, double M[4][4], const Mat3* mat = nullptr) const;  // mat: mu by default
  Csr assemble_N() const;
  uint32_t find_probe(const std::array<double, 3>& pv);
  double efield_source(uint32_t e, double t);
  double current_source(uint32_t e, double t);
  double hfield_source(uint32_t e, double t);
  void apply_K(const double* x, double* y, std::vector<double>& tf) const;
  int cg_solve(const Csr& M, const std::vector<double>& pre, const double* b, double* x, double tol, int maxit,
               double* err) const;
  void export_probes(double t);
  void dga_step(double t);
  void gfdtd_step(double t, double t_prev);
  void fem_step(double t, double t_prev);
  void estimate_dt_pencil();
  std::vector<std::array<double, 16>> whitney_;
};

}  // namespace orc
