// ORACLE — test infrastructure only.  FP64 CPU restatement of the Cartesian
// FIT path; see fit.cpp for the reference lines followed.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "script.hpp"

namespace orc {

struct FitOracle {
  Script sc;
  Simulation sim;
  Output out;
  uint32_t sim_label = 0;
  std::map<uint32_t, Solid> solids;
  // grid
  uint32_t Nx = 0, Ny = 0, Nz = 0;
  double xmin = 0, ymin = 0, zmin = 0, xmax = 0, ymax = 0, zmax = 0, Lx = 0, Ly = 0, Lz = 0;
  uint32_t nE = 0, nF = 0, nV = 0;
  std::vector<uint64_t> matad;
  // complex, in the reference's numbering
  std::vector<std::array<uint32_t, 6>> D;                  // cube -> faces
  std::vector<std::vector<std::pair<uint32_t, int>>> Dt;   // face -> cubes (sign)
  std::vector<std::array<uint32_t, 12>> Ecl;               // cube -> edges
  std::vector<std::array<uint32_t, 8>> Pcl;                // cube -> nodes
  std::vector<std::array<double, 3>> pts;
  std::vector<std::array<uint32_t, 2>> G;                  // edge -> nodes
  std::vector<std::array<uint32_t, 4>> C;                  // face -> edges
  std::vector<std::vector<std::pair<uint32_t, int8_t>>> Ct; // edge -> signed faces
  std::vector<int> curl, dual_curl;
  std::vector<uint64_t> boundary_face;
  std::vector<uint8_t> tbc_flag;
  std::vector<uint32_t> tbc, vol_material;
  std::vector<uint32_t> bc_edges, src_edges, uncommon_edges, common_edges;
  std::vector<std::vector<uint32_t>> edge_src;
  std::vector<double> M_nu, M_mu, M_h, M_q;
  // Si_vec (Discretization.hpp:5374, :5594-5597): sigma-bar / length of each
  // edge, filled only when the output mode is l2norm (store_E, :5368); zero
  // otherwise, so the loss column is zero for every other output mode
  std::vector<double> Si;
  std::vector<std::array<double, 3>> bnd_dual;
  double dt = 0, dt_estimate = 0;
  bool possibly_unstable = false;
  // state
  std::vector<double> U, I, F, B, curl_fb;
  uint32_t root = 0;
  std::vector<uint32_t> probe_elem;
  std::vector<std::array<double, 3>> probe_pts;
  std::vector<double> times, samples, flux;  // samples: [time][probe][Ex Ey Ez Hx Hy Hz]
  std::vector<double> losses;               // Joule loss per step (Discretization.hpp:1902)
  uint64_t step_index = 0, nsteps_total = 0;

  void prepare(uint32_t label);
  uint64_t step(uint64_t n);

 private:
  void build_mesh();
  uint32_t which_solid(double x, double y, double z);
  double fdtd_time_step(const std::vector<double>& Nvec, const std::vector<double>& Hvec);
  uint32_t find_probe(const std::array<double, 3>& pv);
  std::array<double, 3> edge_bar(uint32_t e) const;
  std::array<double, 3> face_bar(uint32_t f) const;
  std::array<double, 3> vol_bar(uint32_t v) const;
  double efield_source(uint32_t e, double t);
  double current_source(uint32_t e, double t);
  double hfield_source(uint32_t e, double t);
  void export_probes(double t);
};

}  // namespace orc
