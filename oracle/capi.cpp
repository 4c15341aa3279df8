// ORACLE — test infrastructure only.  extern "C" surface of the CPU oracle,
// loaded with ctypes by tests/ and by bench.py's cpu_baseline leg.
#include <cstring>
#include <exception>
#include <string>

#include "fit.hpp"

using orc::FitOracle;

static void put_err(char* err, int len, const char* m) {
  if (err && len > 0) {
    std::strncpy(err, m, (size_t)len - 1);
    err[len - 1] = 0;
  }
}

extern "C" {

void* orc_fit_open(const char* script, unsigned label, char* err, int errlen) {
  auto* o = new FitOracle();
  try {
    o->sc.parse(script);
    o->prepare(label);
    return o;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    delete o;
    return nullptr;
  }
}

void orc_fit_close(void* h) { delete static_cast<FitOracle*>(h); }

// ints: nE nF nV nprobes nsteps_total Nx Ny Nz possibly_unstable
// dbls: dt dt_estimate Lx Ly Lz xmin ymin zmin
int orc_fit_info(void* h, long long* iv, double* dv) {
  auto* o = static_cast<FitOracle*>(h);
  iv[0] = o->nE; iv[1] = o->nF; iv[2] = o->nV; iv[3] = (long long)o->probe_elem.size();
  iv[4] = (long long)o->nsteps_total; iv[5] = o->Nx; iv[6] = o->Ny; iv[7] = o->Nz;
  iv[8] = o->possibly_unstable;
  dv[0] = o->dt; dv[1] = o->dt_estimate; dv[2] = o->Lx; dv[3] = o->Ly; dv[4] = o->Lz;
  dv[5] = o->xmin; dv[6] = o->ymin; dv[7] = o->zmin;
  return 0;
}

long long orc_fit_step(void* h, long long n) { return (long long)static_cast<FitOracle*>(h)->step((uint64_t)n); }

long long orc_fit_nsamples(void* h) { return (long long)static_cast<FitOracle*>(h)->times.size(); }

int orc_fit_probes(void* h, double* times, double* samples, double* points, long long* elems) {
  auto* o = static_cast<FitOracle*>(h);
  if (times) std::memcpy(times, o->times.data(), o->times.size() * sizeof(double));
  if (samples) std::memcpy(samples, o->samples.data(), o->samples.size() * sizeof(double));
  for (size_t p = 0; p < o->probe_elem.size(); p++) {
    if (points)
      for (int a = 0; a < 3; a++) points[3 * p + a] = o->probe_pts[p][a];
    if (elems) elems[p] = o->probe_elem[p];
  }
  return 0;
}

int orc_fit_state(void* h, double* U, double* F, double* B) {
  auto* o = static_cast<FitOracle*>(h);
  if (U) std::memcpy(U, o->U.data(), o->U.size() * sizeof(double));
  if (F) std::memcpy(F, o->F.data(), o->F.size() * sizeof(double));
  if (B) std::memcpy(B, o->B.data(), o->B.size() * sizeof(double));
  return 0;
}

int orc_fit_flux(void* h, double* flux) {
  auto* o = static_cast<FitOracle*>(h);
  std::memcpy(flux, o->flux.data(), o->flux.size() * sizeof(double));
  return 0;
}

// Edge nodes (2 per edge) and node coordinates, to relate orderings by geometry.
int orc_fit_topology(void* h, unsigned* edge_nodes, double* node_xyz, unsigned* face_edges, unsigned* classes) {
  auto* o = static_cast<FitOracle*>(h);
  if (edge_nodes)
    for (uint32_t e = 0; e < o->nE; e++) { edge_nodes[2 * e] = o->G[e][0]; edge_nodes[2 * e + 1] = o->G[e][1]; }
  if (node_xyz)
    for (size_t p = 0; p < o->pts.size(); p++)
      for (int a = 0; a < 3; a++) node_xyz[3 * p + a] = o->pts[p][a];
  if (face_edges)
    for (uint32_t f = 0; f < o->nF; f++)
      for (int r = 0; r < 4; r++) face_edges[4 * f + r] = o->C[f][r];
  if (classes) {  // 0 common, 1 pec, 2 e/j source, 3 uncommon
    for (uint32_t e = 0; e < o->nE; e++) classes[e] = 255;
    for (auto e : o->common_edges) classes[e] = 0;
    for (auto e : o->bc_edges) classes[e] = 1;
    for (auto e : o->src_edges) classes[e] = 2;
    for (auto e : o->uncommon_edges) classes[e] = 3;
  }
  return (int)o->pts.size();
}

}  // extern "C"
