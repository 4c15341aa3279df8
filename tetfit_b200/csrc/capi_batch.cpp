// extern "C" batch entry points (include/tetfit.h, tf_batch_*): many gfdtd
// simulations built on the host in parallel and advanced together on one GPU.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tetfit.h"
#include "cuda_util.hpp"
#include "script.hpp"
#include "tet.hpp"
#include "tet_group.hpp"

struct tf_batch {
  std::vector<std::unique_ptr<tf::Script>> scripts;
  std::vector<std::unique_ptr<tf::TetSim>> sims;
  std::vector<std::unique_ptr<tf::TetGroup>> groups;
  std::vector<std::pair<int, int>> where;  // member -> (group, index in group)
  std::string err;
  double last_ms = 0;
  int mode = 0;
};

namespace {

int bfail(tf_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return code;
}

template <typename F>
int bguarded(tf_batch* b, F&& f) {
  try {
    return f();
  } catch (const tf::ScriptError& e) {
    return bfail(b, TF_E_SCRIPT, e.what());
  } catch (const tf::CudaError& e) {
    return bfail(b, TF_E_CUDA, e.what());
  } catch (const tf::UnsupportedError& e) {
    return bfail(b, TF_E_UNSUPPORTED, e.what());
  } catch (const tf::SolverError& e) {
    return bfail(b, TF_E_SOLVER, e.what());
  } catch (const std::exception& e) {
    return bfail(b, TF_E_ARG, e.what());
  }
}

int member_ok(tf_batch* b, uint32_t m) {
  if (!b) return TF_E_ARG;
  if (m >= b->where.size()) return bfail(b, TF_E_ARG, "batch member " + std::to_string(m) + " out of range");
  return TF_OK;
}

}  // namespace

extern "C" {

int tf_batch_open(const char* const* scripts, const uint32_t* labels, uint32_t n, const tf_opts* opts,
                  tf_batch** out) {
  if (!out) return TF_E_ARG;
  *out = nullptr;
  auto* b = new tf_batch();
  *out = b;
  if (!scripts || !labels || n == 0) return bfail(b, TF_E_ARG, "a batch needs at least one script and label");
  return bguarded(b, [&]() -> int {
    tf_opts o;
    tf_default_opts(&o);
    if (opts) o = *opts;
    tf::RunOptions ro;
    ro.precision = o.precision;
    ro.device = o.device;
    ro.graph_steps = o.graph_steps;
    ro.verbose = o.verbose != 0;
    ro.consistent_mass = o.mass_model == 1;
    ro.warm_start = o.warm_start;
    ro.cg_criterion = o.cg_criterion;
    if (o.cg_maxiter > 0) ro.cg_maxiter = o.cg_maxiter;
    if (o.learn_steps > 0) ro.learn_steps = o.learn_steps;
    ro.estimate_pinned = false;
    b->mode = o.batch_mode;
    if (b->mode != 0 && b->mode != 1) return bfail(b, TF_E_ARG, "batch_mode must be 0 or 1");
    b->scripts.resize(n);
    b->sims.resize(n);
    std::vector<std::string> errs(n);
    std::vector<int> codes(n, TF_OK);
    std::atomic<uint32_t> next{0};
    const unsigned limit =
        o.host_threads > 0 ? (unsigned)o.host_threads : std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = std::min<unsigned>(limit, n);
    // members are built nt at a time; each takes its share of the host threads
    ro.setup_threads = (int)std::max(1u, limit / nt);
    // host build of every member (mesh, operators, probes, source tables)
    auto work = [&]() {
      for (uint32_t i = next++; i < n; i = next++) {
        try {
          auto sc = std::make_unique<tf::Script>();
          sc->parse(scripts[i]);
          auto it = sc->simulations.find(labels[i]);
          if (it == sc->simulations.end()) throw std::invalid_argument("unknown simulation label " +
                                                                       std::to_string(labels[i]));
          if ((it->second.method != "gfdtd" && it->second.method != "fem") ||
              sc->meshes[it->second.mesh].type != "tetrahedral")
            throw std::invalid_argument("batches run tetrahedral method gfdtd or fem simulations");
          b->sims[i].reset(new tf::TetSim(*sc, labels[i], ro, false));
          b->scripts[i] = std::move(sc);
        } catch (const tf::ScriptError& e) {
          codes[i] = TF_E_SCRIPT;
          errs[i] = e.what();
        } catch (const std::exception& e) {
          codes[i] = TF_E_ARG;
          errs[i] = e.what();
        }
      }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (uint32_t i = 0; i < n; i++)
      if (codes[i] != TF_OK) return bfail(b, codes[i], "batch member " + std::to_string(i) + ": " + errs[i]);
    // the device image is laid out by this thread alone: all host threads
    tf::RunOptions rg = ro;
    rg.setup_threads = (int)limit;
    if (b->mode == 0) {
      std::vector<tf::TetSim*> v;
      for (auto& s : b->sims) v.push_back(s.get());
      b->groups.emplace_back(new tf::TetGroup(v, rg, true));
      for (uint32_t i = 0; i < n; i++) b->where.push_back({0, (int)i});
    } else {
      for (uint32_t i = 0; i < n; i++) {
        b->groups.emplace_back(new tf::TetGroup({b->sims[i].get()}, rg, true));
        b->where.push_back({(int)i, 0});
      }
    }
    return TF_OK;
  });
}

int tf_batch_info(tf_batch* b, uint32_t m, tf_info* info) {
  if (int rc = member_ok(b, m)) return rc;
  if (!info) return bfail(b, TF_E_ARG, "info is NULL");
  std::memset(info, 0, sizeof(*info));
  const tf::TetSim& t = *b->sims[m];
  const auto [g, k] = b->where[m];
  const tf::TetGroup& grp = *b->groups[g];
  info->n_edges = t.n_edges();
  info->n_faces = t.n_faces();
  info->n_cells = t.n_cells();
  info->n_probes = t.n_probes();
  info->n_steps = grp.n_steps(k);
  info->step_index = grp.step_index(k);
  info->method = 2;
  info->dt = t.dt();
  info->dt_estimate = t.dt_estimate();
  info->possibly_unstable = t.possibly_unstable();
  info->precision = t.precision();
  info->device_bytes = grp.device_bytes();
  info->kernels_per_step = (uint32_t)grp.kernels_per_step();
  info->n_sources = (uint32_t)t.n_sources();
  info->n_free = t.n_free();
  info->nnz_system = grp.nnz_A(k);
  info->cg_blocks = (uint32_t)grp.cg_blocks();
  info->cg_variant = grp.cg_variant();
  return TF_OK;
}

int tf_batch_step(tf_batch* b, uint64_t n, uint64_t* done) {
  if (!b) return TF_E_ARG;
  return bguarded(b, [&]() -> int {
    uint64_t most = 0;
    double ms = 0;
    for (auto& g : b->groups) {
      most = std::max(most, g->step(n));
      ms += g->last_step_ms();
    }
    b->last_ms = ms;
    if (done) *done = most;
    return TF_OK;
  });
}

int tf_batch_phase_times(tf_batch* b, uint64_t n, double* ms5, uint64_t* done) {
  if (!b || !ms5) return TF_E_ARG;
  return bguarded(b, [&]() -> int {
    uint64_t most = 0;
    double acc[5] = {0, 0, 0, 0, 0};
    for (auto& g : b->groups) {
      double t[5];
      most = std::max(most, g->phase_times(n, t));
      for (int q = 0; q < 5; q++) acc[q] += t[q];
    }
    for (int q = 0; q < 5; q++) ms5[q] = acc[q];
    if (done) *done = most;
    return TF_OK;
  });
}

int tf_batch_step_io(tf_batch* b, const double* carriers_in, double* probes_out, uint64_t* done) {
  if (!b) return TF_E_ARG;
  return bguarded(b, [&]() -> int {
    uint64_t most = 0;
    size_t ci = 0, po = 0;
    for (auto& g : b->groups) {
      most = std::max(most, g->step_io(carriers_in ? carriers_in + ci : nullptr, probes_out ? probes_out + po : nullptr));
      ci += g->io_sources();
      po += g->io_probes();
    }
    if (done) *done = most;
    return TF_OK;
  });
}

int tf_batch_get_probes(tf_batch* b, uint32_t m, double* times, double* values, size_t cap, size_t* n) {
  if (int rc = member_ok(b, m)) return rc;
  return bguarded(b, [&]() -> int {
    const auto [g, k] = b->where[m];
    const size_t ns = b->groups[g]->n_samples(k);
    if (n) *n = ns;
    b->groups[g]->get_probes(k, times, values, cap);
    return TF_OK;
  });
}

int tf_batch_get_probe_points(tf_batch* b, uint32_t m, double* xyz, uint64_t* cells, size_t cap) {
  if (int rc = member_ok(b, m)) return rc;
  b->sims[m]->probe_points(xyz, cells, cap);
  return TF_OK;
}

int tf_batch_get_state(tf_batch* b, uint32_t m, double* U, size_t nU, double* B, size_t nB, double* F, size_t nF) {
  if (int rc = member_ok(b, m)) return rc;
  const tf::TetSim& t = *b->sims[m];
  if ((U && nU < t.n_edges()) || (B && nB < t.n_faces()) || (F && nF < t.n_faces()))
    return bfail(b, TF_E_ARG, "state buffer too small");
  return bguarded(b, [&]() -> int {
    const auto [g, k] = b->where[m];
    b->groups[g]->get_state(k, U, B, F);
    return TF_OK;
  });
}

int tf_batch_get_flux(tf_batch* b, uint32_t m, double* flux, size_t cap, size_t* n) {
  if (int rc = member_ok(b, m)) return rc;
  return bguarded(b, [&]() -> int {
    const auto [g, k] = b->where[m];
    b->groups[g]->get_flux(k, flux, cap, n);
    return TF_OK;
  });
}

int tf_batch_energy(tf_batch* b, uint32_t m, double* energy) {
  if (int rc = member_ok(b, m)) return rc;
  if (!energy) return bfail(b, TF_E_ARG, "tf_batch_energy: null output");
  return bguarded(b, [&]() -> int {
    const auto [g, k] = b->where[m];
    *energy = b->groups[g]->energy(k);
    return TF_OK;
  });
}

int tf_batch_solver_stats(tf_batch* b, uint32_t m, int32_t* iters, double* resid, size_t cap, size_t* n) {
  if (int rc = member_ok(b, m)) return rc;
  return bguarded(b, [&]() -> int {
    const auto [g, k] = b->where[m];
    const size_t s = b->groups[g]->solver_stats(k, iters, resid, cap);
    if (n) *n = s;
    return TF_OK;
  });
}

int tf_batch_guess_stats(tf_batch* b, uint32_t m, int8_t* kept, size_t cap, size_t* n) {
  if (int rc = member_ok(b, m)) return rc;
  return bguarded(b, [&]() -> int {
    const auto [g, k] = b->where[m];
    const size_t s = b->groups[g]->guess_stats(k, kept, cap);
    if (n) *n = s;
    return TF_OK;
  });
}

int tf_batch_training_loss(tf_batch* b, uint32_t m, float* loss, size_t cap, size_t* n) {
  if (int rc = member_ok(b, m)) return rc;
  return bguarded(b, [&]() -> int {
    const size_t s = b->groups[b->where[m].first]->training_loss(loss, cap);
    if (n) *n = s;
    return TF_OK;
  });
}

int tf_batch_mlp_params(tf_batch* b, uint32_t m, float* params) {
  if (int rc = member_ok(b, m)) return rc;
  if (!params) return bfail(b, TF_E_ARG, "params is NULL");
  return bguarded(b, [&]() -> int {
    if (!b->groups[b->where[m].first]->mlp_params(params))
      return bfail(b, TF_E_STATE, "the batch was not opened with the learned warm start (warm_start 3)");
    return TF_OK;
  });
}

int tf_batch_last_step_ms(tf_batch* b, double* ms) {
  if (!b || !ms) return TF_E_ARG;
  *ms = b->last_ms;
  return TF_OK;
}

const char* tf_batch_last_error(tf_batch* b) { return b ? b->err.c_str() : ""; }

void tf_batch_close(tf_batch* b) { delete b; }

}  // extern "C"
