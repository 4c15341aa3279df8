// ORACLE — test infrastructure only.  extern "C" surface of the CPU oracle,
// loaded with ctypes by tests/ and by bench.py's cpu_baseline leg.
#include <array>
#include <cstdio>
#include <cstring>
#include <exception>
#include <iomanip>
#include <sstream>
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


// ---------------------------------------------------------------- script dump
// Canonical JSON of a parsed script: every primitive by ascending label, with
// doubles printed to 17 significant digits (exact round trip).  The solids of
// each cartesian mesh are read from its file.
namespace {

void js_str(std::ostringstream& o, const std::string& s) {
  o << '"';
  for (char ch : s) {
    if (ch == '"' || ch == '\\') o << '\\' << ch;
    else if ((unsigned char)ch < 0x20) o << "\\u" << std::hex << std::setw(4) << std::setfill('0') << (int)ch
                                          << std::dec << std::setfill(' ');
    else o << ch;
  }
  o << '"';
}
void js_num(std::ostringstream& o, double v) {
  char b[40];
  std::snprintf(b, sizeof b, "%.17g", v);
  o << b;
}
template <class V>
void js_vec(std::ostringstream& o, const V& v) {
  o << '[';
  bool first = true;
  for (const auto& x : v) {
    if (!first) o << ", ";
    first = false;
    js_num(o, (double)x);
  }
  o << ']';
}
void js_strs(std::ostringstream& o, const std::array<std::string, 3>& v) {
  o << '[';
  for (int k = 0; k < 3; k++) {
    if (k) o << ", ";
    js_str(o, v[k]);
  }
  o << ']';
}
void js_mat(std::ostringstream& o, const orc::Mat3& m) {
  o << '[';
  for (int r = 0; r < 3; r++) {
    if (r) o << ", ";
    o << '[';
    for (int c = 0; c < 3; c++) {
      if (c) o << ", ";
      js_num(o, m.m[r][c]);
    }
    o << ']';
  }
  o << ']';
}
struct Obj {  // comma bookkeeping for one JSON object
  std::ostringstream& o;
  bool first = true;
  explicit Obj(std::ostringstream& os) : o(os) { o << '{'; }
  std::ostringstream& key(const char* k) {
    if (!first) o << ", ";
    first = false;
    js_str(o, k);
    o << ": ";
    return o;
  }
  void num(const char* k, double v) { key(k); js_num(o, v); }
  void str(const char* k, const std::string& v) { key(k); js_str(o, v); }
  void end() { o << '}'; }
};
template <class MapT, class F>
void js_map(Obj& top, const char* name, const MapT& m, F&& each) {
  std::ostringstream& o = top.key(name);
  Obj inner(o);
  for (const auto& kv : m) {
    inner.key(std::to_string(kv.first).c_str());
    each(kv.second);
  }
  inner.end();
}

std::string script_json(const orc::Script& sc) {
  std::ostringstream o;
  Obj top(o);
  js_map(top, "materials", sc.materials, [&](const orc::Material& m) {
    Obj x(o);
    x.key("eps"); js_mat(o, m.eps);
    x.key("mu"); js_mat(o, m.mu);
    x.key("sigma"); js_mat(o, m.sigma);
    x.key("chi"); js_mat(o, m.chi);
    x.end();
  });
  js_map(top, "bcs", sc.bcs, [&](const orc::BoundaryCondition& b) {
    Obj x(o);
    x.str("type", b.type); x.str("dir", b.dir); x.num("width", b.width); x.num("val", b.val);
    x.key("surfs"); js_vec(o, b.surfs);
    x.end();
  });
  js_map(top, "meshes", sc.meshes, [&](const orc::Mesh& m) {
    Obj x(o);
    x.str("file", m.file); x.str("name", m.name); x.str("type", m.type); x.str("mesher", m.mesher);
    x.num("scale", m.scale);
    x.num("xmin", m.xmin); x.num("xstep", m.xstep); x.num("xmax", m.xmax);
    x.num("ymin", m.ymin); x.num("ystep", m.ystep); x.num("ymax", m.ymax);
    x.num("zmin", m.zmin); x.num("zstep", m.zstep); x.num("zmax", m.zmax);
    x.end();
  });
  js_map(top, "sources", sc.sources, [&](const orc::Source& s) {
    Obj x(o);
    x.str("st", s.st); x.str("prof", s.prof); x.str("carrier", s.carrier); x.str("dir", s.dir);
    x.num("amp", s.amp); x.num("freq", s.freq); x.num("radius", s.radius); x.num("decay", s.decay);
    x.num("width", s.width); x.num("delay", s.delay); x.num("impedance", s.impedance);
    x.key("kvec"); js_vec(o, s.kvec);
    x.key("center"); js_vec(o, s.center);
    x.key("location"); js_vec(o, s.location);
    x.key("bfuncs"); js_strs(o, s.bfuncs);
    x.key("surfaces"); js_vec(o, s.surfaces);
    x.end();
  });
  js_map(top, "simulations", sc.simulations, [&](const orc::Simulation& s) {
    Obj x(o);
    x.num("duration", s.duration); x.num("courant", s.courant); x.num("step", s.step); x.num("tol", s.tol);
    x.str("method", s.method); x.str("solver", s.solver); x.str("analytic", s.analytic);
    x.key("debug") << (s.debug ? "true" : "false");
    x.key("sources"); js_vec(o, s.sources);
    x.num("mesh", s.mesh); x.num("output", s.output);
    x.end();
  });
  js_map(top, "outputs", sc.outputs, [&](const orc::Output& p) {
    Obj x(o);
    x.str("mode", p.mode); x.str("name", p.name); x.num("period", p.period); x.num("nextprint", p.nextprint);
    x.num("delay", p.delay); x.num("ref_sys", p.ref_sys);
    x.num("xstart", p.xstart); x.num("xstep", p.xstep); x.num("xstop", p.xstop);
    x.num("ystart", p.ystart); x.num("ystep", p.ystep); x.num("ystop", p.ystop);
    x.num("zstart", p.zstart); x.num("zstep", p.zstep); x.num("zstop", p.zstop);
    x.key("probes");
    o << '[';
    for (size_t q = 0; q < p.probes.size(); q++) {
      if (q) o << ", ";
      js_vec(o, p.probes[q]);
    }
    o << ']';
    x.end();
  });
  top.key("bnd_to_bc"); js_vec(o, sc.bnd_to_bc);
  // solids of the cartesian meshes (solids-file reader)
  {
    std::ostringstream& os = top.key("solids");
    Obj meshes(os);
    for (const auto& kv : sc.meshes) {
      if (kv.second.type != "cartesian" || kv.second.file == "none") continue;
      meshes.key(std::to_string(kv.first).c_str());
      Obj sol(o);
      for (const auto& s : orc::read_solids(kv.second.file)) {
        sol.key(std::to_string(s.first).c_str());
        Obj x(o);
        x.str("type", s.second.type); x.num("material", s.second.material); x.num("sqr", s.second.sqr);
        x.key("center"); js_vec(o, s.second.center);
        x.key("corner"); js_vec(o, s.second.corner);
        x.key("size"); js_vec(o, s.second.size);
        x.end();
      }
      sol.end();
    }
    meshes.end();
  }
  top.end();
  return o.str();
}

}  // namespace

extern "C" {

// Parses a script with the oracle's front end and writes its canonical JSON
// into buf (cap bytes); returns the length needed including the terminator,
// or -1 with the error text in buf.
long orc_script_dump(const char* script, char* buf, long cap) {
  std::string out;
  long rc;
  try {
    orc::Script sc;
    sc.parse(script);
    out = script_json(sc);
    rc = (long)out.size() + 1;
  } catch (const std::exception& e) {
    out = e.what();
    rc = -1;
  }
  if (buf && cap > 0) {
    const size_t m = out.size() < (size_t)cap - 1 ? out.size() : (size_t)cap - 1;
    std::memcpy(buf, out.data(), m);
    buf[m] = 0;
  }
  return rc;
}

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

int orc_fit_losses(void* h, double* loss) {
  auto* o = static_cast<FitOracle*>(h);
  std::memcpy(loss, o->losses.data(), o->losses.size() * sizeof(double));
  return (int)o->losses.size();
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

// poynting.dat's third column: the first n entries of the losses list, one
// per step taken (gfdtd, fem; dga returns zeros)
int orc_tet_losses(void* h, double* loss) {
  auto* o = static_cast<orc::TetOracle*>(h);
  const size_t n = o->flux.size();
  for (size_t k = 0; k < n; k++) loss[k] = k < o->losses.size() ? o->losses[k] : 0.0;
  return (int)n;
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

// dga: P per edge (1 on class-1 edges, P_p on class-2 edges, 0 elsewhere)
int orc_tet_dga_p(void* h, double* P) {
  auto* o = static_cast<orc::TetOracle*>(h);
  for (size_t e = 0; e < o->edges.size(); e++)
    P[e] = o->cls[e] == 1 ? 1.0 : o->cls[e] == 2 ? o->P_p[o->p_index[e]] : 0.0;
  return (int)o->Q_size;
}

// dga: R per face (1 on class-1 faces, R_r on class-2 faces)
int orc_tet_dga_r(void* h, double* R) {
  auto* o = static_cast<orc::TetOracle*>(h);
  for (size_t f = 0; f < o->faces.size(); f++) R[f] = o->fcls[f] == 1 ? 1.0 : o->R_r[o->r_index[f]];
  return (int)o->R_size;
}

// CSR export of an operator: which 0 C, 1 N, 2 H, 3 E, 4 A, 5 Sig, 6 the dga F-update
// operator (Na / Tr rows by face); returns nnz
long long orc_tet_matrix(void* h, int which, unsigned long long* ptr, unsigned* col, double* val) {
  auto* o = static_cast<orc::TetOracle*>(h);
  const orc::Csr* m = which == 0 ? &o->C : which == 1 ? &o->N : which == 2 ? &o->H : which == 3 ? &o->E
                     : which == 5 ? &o->Sig : which == 6 ? &o->Nv : &o->A;
  if (ptr) for (size_t i = 0; i < m->ptr.size(); i++) ptr[i] = m->ptr[i];
  if (col) std::memcpy(col, m->col.data(), m->col.size() * sizeof(unsigned));
  if (val) std::memcpy(val, m->val.data(), m->val.size() * sizeof(double));
  return (long long)m->val.size();
}

}  // extern "C"
