// ORACLE — test infrastructure only.  extern "C" surface of the CPU oracle,
// loaded with ctypes by tests/ and by bench.py's cpu_baseline leg.
#include <cstring>
#include <exception>
#include <string>

#include "fit.hpp"
#include "tet.hpp"

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

// Material coefficients in the reference numbering: M_h, M_q (edges), M_nu, M_mu (faces).
int orc_fit_coeffs(void* h, double* mh, double* mq, double* mnu, double* mmu) {
  auto* o = static_cast<FitOracle*>(h);
  for (uint32_t e = 0; e < o->nE; e++) { if (mh) mh[e] = o->M_h[e]; if (mq) mq[e] = o->M_q[e]; }
  for (uint32_t f = 0; f < o->nF; f++) { if (mnu) mnu[f] = o->M_nu[f]; if (mmu) mmu[f] = o->M_mu[f]; }
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

// ---------------------------------------------------------------- tets
void* orc_tet_open(const char* script, unsigned label, int flags, char* err, int errlen) {
  auto* o = new orc::TetOracle();
  o->consistent_mass = (flags & 1) != 0;
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

void orc_tet_close(void* h) { delete static_cast<orc::TetOracle*>(h); }

// ints: nE nF nV(tets) nNodes nprobes nsteps method nfree nbnd possibly_unstable
// dbls: dt dt_estimate
int orc_tet_info(void* h, long long* iv, double* dv) {
  auto* o = static_cast<orc::TetOracle*>(h);
  iv[0] = (long long)o->edges.size(); iv[1] = (long long)o->faces.size(); iv[2] = (long long)o->vols.size();
  iv[3] = (long long)o->pts.size(); iv[4] = (long long)o->probe_elem.size(); iv[5] = (long long)o->nsteps_total;
  iv[6] = o->method; iv[7] = (long long)o->free_edges.size(); iv[8] = (long long)o->bnd_dual.size();
  iv[9] = o->possibly_unstable;
  dv[0] = o->dt; dv[1] = o->dt_estimate;
  return 0;
}

long long orc_tet_step(void* h, long long n) { return (long long)static_cast<orc::TetOracle*>(h)->step((uint64_t)n); }
long long orc_tet_nsamples(void* h) { return (long long)static_cast<orc::TetOracle*>(h)->times.size(); }

int orc_tet_probes(void* h, double* times, double* samples, double* points, long long* elems) {
  auto* o = static_cast<orc::TetOracle*>(h);
  if (times) std::memcpy(times, o->times.data(), o->times.size() * sizeof(double));
  if (samples) std::memcpy(samples, o->samples.data(), o->samples.size() * sizeof(double));
  for (size_t p = 0; p < o->probe_elem.size(); p++) {
    if (points) for (int a = 0; a < 3; a++) points[3 * p + a] = o->probe_pts[p][a];
    if (elems) elems[p] = o->probe_elem[p];
  }
  return 0;
}

int orc_tet_state(void* h, double* U, double* F, double* B) {
  auto* o = static_cast<orc::TetOracle*>(h);
  if (U) std::memcpy(U, o->U.data(), o->U.size() * sizeof(double));
  if (F) std::memcpy(F, o->F.data(), o->F.size() * sizeof(double));
  if (B) std::memcpy(B, o->B.data(), o->B.size() * sizeof(double));
  return 0;
}

int orc_tet_flux(void* h, double* flux) {
  auto* o = static_cast<orc::TetOracle*>(h);
  std::memcpy(flux, o->flux.data(), o->flux.size() * sizeof(double));
  return (int)o->flux.size();
}

int orc_tet_cg(void* h, int* iters, double* errs) {
  auto* o = static_cast<orc::TetOracle*>(h);
  for (size_t k = 0; k < o->cg_iters.size(); k++) {
    if (iters) iters[k] = o->cg_iters[k];
    if (errs) errs[k] = o->cg_err[k];
  }
  return (int)o->cg_iters.size();
}

// topology: edges [nE][2] (node ids), faces [nF][3], classes [nE], bnd index [nE]
int orc_tet_topology(void* h, unsigned* edges, unsigned* faces, unsigned char* cls, int* bnd) {
  auto* o = static_cast<orc::TetOracle*>(h);
  for (size_t e = 0; e < o->edges.size(); e++) {
    if (edges) { edges[2 * e] = o->edges[e][0]; edges[2 * e + 1] = o->edges[e][1]; }
    if (cls) cls[e] = o->cls[e];
    if (bnd) bnd[e] = o->bnd_edges[e];
  }
  if (faces)
    for (size_t f = 0; f < o->faces.size(); f++)
      for (int a = 0; a < 3; a++) faces[3 * f + a] = o->faces[f][a];
  return 0;
}

// CSR export of an operator: which 0 C, 1 N, 2 H, 3 E, 4 A; returns nnz
long long orc_tet_matrix(void* h, int which, unsigned long long* ptr, unsigned* col, double* val) {
  auto* o = static_cast<orc::TetOracle*>(h);
  const orc::Csr* m = which == 0 ? &o->C : which == 1 ? &o->N : which == 2 ? &o->H : which == 3 ? &o->E : &o->A;
  if (ptr) for (size_t i = 0; i < m->ptr.size(); i++) ptr[i] = m->ptr[i];
  if (col) std::memcpy(col, m->col.data(), m->col.size() * sizeof(unsigned));
  if (val) std::memcpy(val, m->val.data(), m->val.size() * sizeof(double));
  return (long long)m->val.size();
}

}  // extern "C"
