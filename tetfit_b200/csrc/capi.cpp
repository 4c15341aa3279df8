// extern "C" boundary (include/tetfit.h).  Maps C++ exceptions to status
// codes; nothing throws across the ABI.
#include <array>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>

#include "../../include/tetfit.h"
#include "cuda_util.hpp"
#include "fit.hpp"
#include "script.hpp"
#include "sim.hpp"
#include "tet.hpp"

struct tf_ctx {
  tf::Script sc;
  std::string path, err;
  std::unique_ptr<tf::Sim> fit;
  uint32_t label = 0;
  tf_opts opts{};
};

namespace tf {
// message of the last context-free call on this host thread
static thread_local std::string g_thread_error;
void set_thread_error(const std::string& m) { g_thread_error = m; }
}  // namespace tf

namespace {

int fail(tf_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

template <typename F>
int guarded(tf_ctx* c, F&& f) {
  try {
    return f();
  } catch (const tf::ScriptError& e) {
    return fail(c, TF_E_SCRIPT, e.what());
  } catch (const tf::CudaError& e) {
    return fail(c, TF_E_CUDA, e.what());
  } catch (const tf::UnsupportedError& e) {
    return fail(c, TF_E_UNSUPPORTED, e.what());
  } catch (const tf::SolverError& e) {
    return fail(c, TF_E_SOLVER, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(c, TF_E_ARG, e.what());
  } catch (const std::exception& e) {
    return fail(c, TF_E_ARG, e.what());
  }
}

// Output files of Discretization.hpp:1948-2010 (probe series) and :1936-1941
// (poynting.dat): std::setw(15), default stream precision.
void write_outputs(tf_ctx* c) {
  tf::Sim& f = *c->fit;
  const tf::Output& o = f.output();
  if (o.mode == "probepoint") {
    size_t ns = f.n_samples(), np = f.n_probes();
    std::vector<double> t(ns), v(ns * np * 6), xyz(np * 3);
    f.get_probes(t.data(), v.data(), ns);
    f.probe_points(xyz.data(), nullptr, np);
    std::stringstream se, sh;
    se << o.name << std::setw(5) << std::setfill('0') << c->label << "_probe_E.dat";
    sh << o.name << std::setw(5) << std::setfill('0') << c->label << "_probe_H.dat";
    std::ofstream os(se.str()), osh(sh.str());
    if (c->opts.file_digits > 0) {  // more digits than the reference's default 6 (an extension)
      os.precision(c->opts.file_digits);
      osh.precision(c->opts.file_digits);
    }
    for (size_t k = 0; k < ns; k++)
      for (size_t p = 0; p < np; p++) {
        const double* s = &v[(k * np + p) * 6];
        os << std::setw(15) << xyz[3 * p] << " " << std::setw(15) << xyz[3 * p + 1] << " " << std::setw(15)
           << xyz[3 * p + 2] << " " << std::setw(15) << t[k] << " " << std::setw(15) << s[0] << " "
           << std::setw(15) << s[1] << " " << std::setw(15) << s[2] << std::endl;
        osh << std::setw(15) << xyz[3 * p] << " " << std::setw(15) << xyz[3 * p + 1] << " " << std::setw(15)
            << xyz[3 * p + 2] << " " << std::setw(15) << t[k] + f.sample_time_shift() << " " << std::setw(15) << s[3]
            << " " << std::setw(15) << s[4] << " " << std::setw(15) << s[5] << std::endl;
      }
  }
  if (o.mode == "silo") {
    // In place of the Silo files (Discretization.hpp:2601-2677): one binary
    // dump per print time, <output name><simulation, 5 digits>_<dump, 5
    // digits>.tfd, little endian:
    //   char[8] "TFDUMP1", int32 n_nodes, n_tets, simulation, dump; double t;
    //   double xyz[n_nodes][3]; int32 tet[n_tets][4] (0-based, ExportMesh's
    //   orientation); double E[n_tets][3] (Whitney, barycentre); double H[n_tets][3]
    std::vector<double> xyz;
    std::vector<int32_t> tets;
    if (f.mesh_arrays(&xyz, &tets)) {
      const size_t ns = f.n_samples(), np = f.n_probes();
      std::vector<double> t(ns), v(ns * np * 6), e(np * 3), h(np * 3);
      f.get_probes(t.data(), v.data(), ns);
      for (size_t k = 0; k < ns; k++) {
        std::stringstream sn;
        sn << o.name << std::setw(5) << std::setfill('0') << c->label << "_" << std::setw(5) << std::setfill('0')
           << k << ".tfd";
        std::ofstream os(sn.str(), std::ios::binary);
        const char magic[8] = {'T', 'F', 'D', 'U', 'M', 'P', '1', 0};
        const int32_t head[4] = {(int32_t)(xyz.size() / 3), (int32_t)(tets.size() / 4), (int32_t)c->label,
                                 (int32_t)k};
        for (size_t p = 0; p < np; p++)
          for (int a = 0; a < 3; a++) {
            e[3 * p + a] = v[(k * np + p) * 6 + a];
            h[3 * p + a] = v[(k * np + p) * 6 + 3 + a];
          }
        os.write(magic, 8);
        os.write(reinterpret_cast<const char*>(head), sizeof head);
        os.write(reinterpret_cast<const char*>(&t[k]), sizeof(double));
        os.write(reinterpret_cast<const char*>(xyz.data()), (std::streamsize)(xyz.size() * sizeof(double)));
        os.write(reinterpret_cast<const char*>(tets.data()), (std::streamsize)(tets.size() * sizeof(int32_t)));
        os.write(reinterpret_cast<const char*>(e.data()), (std::streamsize)(e.size() * sizeof(double)));
        os.write(reinterpret_cast<const char*>(h.data()), (std::streamsize)(h.size() * sizeof(double)));
      }
    }
  }
  size_t n = 0;
  f.get_flux(nullptr, 0, &n);
  std::vector<double> fl(n), lo(n);
  f.get_flux(fl.data(), n, &n);
  f.get_losses(lo.data(), n, nullptr);
  // poynting.dat: times (k + 1/2) dt for fdtd/dga (:1936-1941, :945-950),
  // (k + 1) dt for gfdtd (:1570-1574)
  std::ofstream pf("poynting.dat");
  const double off = f.method() >= 2 ? 1.0 : 0.5;
  for (size_t k = 0; k < n; k++) pf << double(k + off) * f.dt() << "\t" << fl[k] << "\t" << lo[k] << std::endl;
}

void banner(tf_ctx* c) {
  tf::Sim& f = *c->fit;
  static const char* kNames[4] = {"fdtd", "dga", "gfdtd", "fem"};
  std::cout << std::endl << "Simulation parameters:" << std::endl;
  std::cout << std::setw(20) << "Method: " << std::setw(20) << kNames[f.method()] << std::endl;
  std::cout << std::setw(20) << "Simulation time: " << std::setw(20) << f.simulation().duration << " sec"
            << std::endl;
  std::cout << std::setw(20) << "Time step: " << std::setw(20) << f.dt() << " sec" << std::endl;
  std::cout << std::setw(20) << "Elements: " << std::setw(20) << f.n_cells() << std::endl;
  std::cout << std::setw(20) << "Surfaces: " << std::setw(20) << f.n_faces() << std::endl;
  std::cout << std::setw(20) << "Edges:    " << std::setw(20) << f.n_edges() << std::endl;
  std::cout << std::setw(20) << "Unknowns: " << std::setw(20) << f.n_edges() + f.n_faces() << std::endl;
  if (f.possibly_unstable())
    std::cout << "WARNING: the time step size chosen by the user is possibly unstable! (Upper stable limit will "
                 "be used instead...)"
              << std::endl;
}

}  // namespace


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
void js_mat(std::ostringstream& o, const tf::Mat3& m) {
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

std::string script_json(const tf::Script& sc) {
  std::ostringstream o;
  Obj top(o);
  js_map(top, "materials", sc.materials, [&](const tf::Material& m) {
    Obj x(o);
    x.key("eps"); js_mat(o, m.eps);
    x.key("mu"); js_mat(o, m.mu);
    x.key("sigma"); js_mat(o, m.sigma);
    x.key("chi"); js_mat(o, m.chi);
    x.end();
  });
  js_map(top, "bcs", sc.bcs, [&](const tf::BoundaryCondition& b) {
    Obj x(o);
    x.str("type", b.type); x.str("dir", b.dir); x.num("width", b.width); x.num("val", b.val);
    x.key("surfs"); js_vec(o, b.surfs);
    x.end();
  });
  js_map(top, "meshes", sc.meshes, [&](const tf::Mesh& m) {
    Obj x(o);
    x.str("file", m.file); x.str("name", m.name); x.str("type", m.type); x.str("mesher", m.mesher);
    x.num("scale", m.scale);
    x.num("xmin", m.xmin); x.num("xstep", m.xstep); x.num("xmax", m.xmax);
    x.num("ymin", m.ymin); x.num("ystep", m.ystep); x.num("ymax", m.ymax);
    x.num("zmin", m.zmin); x.num("zstep", m.zstep); x.num("zmax", m.zmax);
    x.end();
  });
  js_map(top, "sources", sc.sources, [&](const tf::Source& s) {
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
  js_map(top, "simulations", sc.simulations, [&](const tf::Simulation& s) {
    Obj x(o);
    x.num("duration", s.duration); x.num("courant", s.courant); x.num("step", s.step); x.num("tol", s.tol);
    x.str("method", s.method); x.str("solver", s.solver); x.str("analytic", s.analytic);
    x.key("debug") << (s.debug ? "true" : "false");
    x.key("sources"); js_vec(o, s.sources);
    x.num("mesh", s.mesh); x.num("output", s.output);
    x.end();
  });
  js_map(top, "outputs", sc.outputs, [&](const tf::Output& p) {
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
      for (const auto& s : tf::read_solids(kv.second.file)) {
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

void tf_default_opts(tf_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = TF_FP64;
}

int tf_open(const char* path, tf_ctx** out) {
  if (!out || !path) return TF_E_ARG;
  *out = nullptr;
  auto* c = new tf_ctx();
  c->path = path;
  tf_default_opts(&c->opts);
  int rc = guarded(c, [&]() -> int {
    c->sc.parse(path);
    return TF_OK;
  });
  *out = c;  // the context carries the error message even on failure
  return rc;
}

int tf_script_dump(tf_ctx* c, char* buf, size_t cap, size_t* len) {
  if (!c) return TF_E_ARG;
  return guarded(c, [&]() -> int {
    const std::string js = script_json(c->sc);
    if (len) *len = js.size() + 1;
    if (buf && cap) {
      const size_t m = js.size() < cap - 1 ? js.size() : cap - 1;
      std::memcpy(buf, js.data(), m);
      buf[m] = 0;
      if (m < js.size()) return fail(c, TF_E_ARG, "tf_script_dump: buffer too small");
    }
    return TF_OK;
  });
}

int tf_simulations(tf_ctx* c, uint32_t* labels, uint32_t cap, uint32_t* n) {
  if (!c) return TF_E_ARG;
  uint32_t k = 0;
  for (auto& kv : c->sc.simulations) {
    if (labels && k < cap) labels[k] = kv.first;
    k++;
  }
  if (n) *n = k;
  return TF_OK;
}

int tf_prepare(tf_ctx* c, uint32_t label, const tf_opts* opts) {
  if (!c) return TF_E_ARG;
  return guarded(c, [&]() -> int {
    c->fit.reset();
    if (opts) c->opts = *opts;
    auto it = c->sc.simulations.find(label);
    if (it == c->sc.simulations.end()) return fail(c, TF_E_ARG, "unknown simulation label " + std::to_string(label));
    const std::string& meth = it->second.method;
    const std::string mtype = c->sc.meshes[it->second.mesh].type;
    // Discretization.hpp:313-316
    if ((mtype == "tetrahedral" && meth == "fdtd") || (mtype == "cartesian" && meth != "fdtd" && meth != "fdtdo2"))
      throw tf::ScriptError("Input file error at line 0: If mesh type is tetrahedral, method must be fem or dga. If "
                            "mesh type is cartesian, method must be fdtd");
    tf::RunOptions ro;
    ro.precision = c->opts.precision;
    ro.device = c->opts.device;
    ro.graph_steps = c->opts.graph_steps;
    ro.verbose = c->opts.verbose != 0;
    ro.consistent_mass = c->opts.mass_model == 1;
    ro.warm_start = c->opts.warm_start;
    ro.cg_criterion = c->opts.cg_criterion;
    if (c->opts.cg_maxiter > 0) ro.cg_maxiter = c->opts.cg_maxiter;
    if (c->opts.learn_steps > 0) ro.learn_steps = c->opts.learn_steps;
    ro.fit_variant = c->opts.fit_variant;
    ro.setup_threads = c->opts.host_threads > 0 ? c->opts.host_threads : 0;
    if (ro.fit_variant < 0 || ro.fit_variant > 6) return fail(c, TF_E_ARG, "fit_variant must be 0..6");
    if (c->opts.file_digits < 0 || c->opts.file_digits > 17) return fail(c, TF_E_ARG, "file_digits must be 0..17");
    if (meth == "fdtd") {
      c->fit.reset(new tf::FitSim(c->sc, label, ro));
    } else if (meth == "dga" || meth == "gfdtd" || meth == "fem") {
      c->fit.reset(new tf::TetSim(c->sc, label, ro));
    } else {
      return fail(c, TF_E_UNSUPPORTED, "method " + meth + " is outside the time-stepping path (fdtd, dga, gfdtd, fem)");
    }
    c->label = label;
    if (ro.verbose) banner(c);
    return TF_OK;
  });
}

int tf_get_info(tf_ctx* c, tf_info* info) {
  if (!c || !info) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_get_info before tf_prepare");
  std::memset(info, 0, sizeof(*info));
  tf::Sim& f = *c->fit;
  info->n_edges = f.n_edges();
  info->n_faces = f.n_faces();
  info->n_cells = f.n_cells();
  info->n_probes = f.n_probes();
  info->n_steps = f.n_steps();
  info->step_index = f.step_index();
  info->nx = f.nx(); info->ny = f.ny(); info->nz = f.nz();
  info->method = f.method();
  info->dt = f.dt();
  info->dt_estimate = f.dt_estimate();
  info->possibly_unstable = f.possibly_unstable();
  info->precision = f.precision();
  info->device_bytes = f.device_bytes();
  info->kernels_per_step = (uint32_t)f.kernels_per_step();
  info->n_sources = (uint32_t)f.n_sources();
  info->n_free = f.n_free();
  info->nnz_system = f.nnz_system();
  info->nnz_operators = f.nnz_operators();
  info->cg_variant = f.kernel_variant();
  return TF_OK;
}

int tf_step(tf_ctx* c, uint64_t n, uint64_t* done) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_step before tf_prepare");
  return guarded(c, [&]() -> int {
    uint64_t d = c->fit->step(n);
    if (done) *done = d;
    return TF_OK;
  });
}

int tf_step_io(tf_ctx* c, const double* carrier_in, double* probe_out, uint64_t* done) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_step_io before tf_prepare");
  return guarded(c, [&]() -> int {
    uint64_t d = c->fit->step_io(carrier_in, probe_out);
    if (done) *done = d;
    return TF_OK;
  });
}

int tf_phase_times(tf_ctx* c, uint64_t n, double* ms5, uint64_t* done) {
  if (!c || !ms5) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_phase_times before tf_prepare");
  return guarded(c, [&]() -> int {
    uint64_t d = c->fit->phase_times(n, ms5);
    if (done) *done = d;
    return TF_OK;
  });
}

int tf_get_probes(tf_ctx* c, double* times, double* values, size_t cap, size_t* n) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_get_probes before tf_prepare");
  return guarded(c, [&]() -> int {
    size_t ns = c->fit->n_samples();
    if (n) *n = ns;
    c->fit->get_probes(times, values, cap);
    return TF_OK;
  });
}

int tf_get_probe_points(tf_ctx* c, double* xyz, uint64_t* cells, size_t cap) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_get_probe_points before tf_prepare");
  c->fit->probe_points(xyz, cells, cap);
  return TF_OK;
}

int tf_get_state(tf_ctx* c, double* U, size_t nU, double* B, size_t nB, double* F, size_t nF) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_get_state before tf_prepare");
  if ((U && nU < c->fit->n_edges()) || (B && nB < c->fit->n_faces()) || (F && nF < c->fit->n_faces()))
    return fail(c, TF_E_ARG, "state buffer too small");
  return guarded(c, [&]() -> int {
    c->fit->get_state(U, B, F);
    return TF_OK;
  });
}

int tf_set_state(tf_ctx* c, const double* U, size_t nU, const double* F, size_t nF) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_set_state before tf_prepare");
  if ((U && nU < c->fit->n_edges()) || (F && nF < c->fit->n_faces()))
    return fail(c, TF_E_ARG, "state buffer too small");
  return guarded(c, [&]() -> int {
    c->fit->set_state(U, F);
    return TF_OK;
  });
}

int tf_get_flux(tf_ctx* c, double* flux, size_t cap, size_t* n) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_get_flux before tf_prepare");
  return guarded(c, [&]() -> int {
    c->fit->get_flux(flux, cap, n);
    return TF_OK;
  });
}

int tf_get_losses(tf_ctx* c, double* loss, size_t cap, size_t* n) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_get_losses before tf_prepare");
  return guarded(c, [&]() -> int {
    c->fit->get_losses(loss, cap, n);
    return TF_OK;
  });
}

int tf_energy(tf_ctx* c, double* e) {
  if (!c || !e) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_energy before tf_prepare");
  return guarded(c, [&]() -> int {
    *e = c->fit->energy();
    return TF_OK;
  });
}

int tf_run(tf_ctx* c, uint32_t label, const tf_opts* opts) {
  int rc = tf_prepare(c, label, opts);
  if (rc) return rc;
  return guarded(c, [&]() -> int {
    while (c->fit->step_index() < c->fit->n_steps()) c->fit->step(c->fit->n_steps() - c->fit->step_index());
    if (c->opts.write_files) write_outputs(c);
    return TF_OK;
  });
}

int tf_solver_stats(tf_ctx* c, int32_t* iters, double* resid, size_t cap, size_t* n) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "no simulation prepared");
  return guarded(c, [&]() -> int {
    size_t k = c->fit->solver_stats(iters, resid, cap);
    if (n) *n = k;
    return TF_OK;
  });
}

int tf_guess_stats(tf_ctx* c, int8_t* kept, size_t cap, size_t* n) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_guess_stats before tf_prepare");
  return guarded(c, [&]() -> int {
    const size_t k = c->fit->guess_stats(kept, cap);
    if (n) *n = k;
    return TF_OK;
  });
}

int tf_training_loss(tf_ctx* c, float* loss, size_t cap, size_t* n) {
  if (!c) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "tf_training_loss before tf_prepare");
  return guarded(c, [&]() -> int {
    const size_t k = c->fit->training_loss(loss, cap);
    if (n) *n = k;
    return TF_OK;
  });
}

int tf_last_step_ms(tf_ctx* c, double* ms) {
  if (!c || !ms) return TF_E_ARG;
  if (!c->fit) return fail(c, TF_E_STATE, "no simulation prepared");
  *ms = c->fit->last_step_ms();
  return TF_OK;
}

const char* tf_last_error(tf_ctx* c) { return c ? c->err.c_str() : tf::g_thread_error.c_str(); }

void tf_close(tf_ctx* c) { delete c; }

}  // extern "C"
