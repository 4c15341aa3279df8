// Tetrahedral DGA simulations: host set-up and device runtime.
//
// The complex is numbered as TetFIT numbers it (Discretization.hpp:5868-6926):
// tets, faces and edges sorted lexicographically by their sorted node tuples,
// so every state vector is already in the reference's order.  Numbering is
// done with packed 64-bit keys and one sort per entity kind.  The material
// operators follow ConstructCodecasaMaterialMatrices (Discretization.hpp
// :8694-9513, dga) and ConstructGFDTDMaterialMatrices (:8132-8692, gfdtd) and
// are uploaded as CSR; the time loop runs entirely on the device
// (tet_kernels.cu).  Lossless materials only (sigma = chi = 0).
#include "tet.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <numeric>
#include <sstream>
#include <stdexcept>

#include "cuda_util.hpp"
#include "dt_gpu.hpp"
#include "host_parallel.hpp"
#include "tet_group.hpp"

namespace tf {

template <typename T>
cudaError_t tet_launch_step(const DevPtrs& d, cudaStream_t st, cudaEvent_t* ev);
template <typename T>
void tet_launch_initial_probes(const DevPtrs& d, cudaStream_t st);
template <typename T>
cudaError_t tet_launch_energy(const DevPtrs& d, DevPtrs d_cg, int cg_blocks, const int32_t* ie, int ni,
                              double* part, double* out, cudaStream_t st);
template <typename T>
int tet_cg_blocks(int device);

namespace {
using V3 = std::array<double, 3>;
V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
V3 cross(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
V3 scale(const V3& a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
V3 mv(const Mat3& m, const V3& v) {
  V3 r;
  for (int i = 0; i < 3; i++) r[i] = m.m[i][0] * v[0] + m.m[i][1] * v[1] + m.m[i][2] * v[2];
  return r;
}
// ConvertFromGMSH (Discretization.hpp:5692-5866, element parser
// Utilities.hpp:159-223): an ASCII gmsh 2.x mesh becomes the netgen text the
// reader takes, as the reference writes it to a temporary .mesh file.  Layout
// read: four header lines, the node count, one "id x y z" line per node, two
// lines, the element count, one "id type ntags tag1 tag2 nodes..." line per
// element (two tags assumed, as the reference does).  Written: the node
// count and coordinates with 6 significant digits (the reference prints
// them through a default ostream, so they are rounded), the tetrahedra (type
// 4, material = first tag) with sorted 1-based nodes in sorted order, then
// the triangles (type 2, boundary id = first tag) in file order.
std::string gmsh_to_netgen(const std::string& text) {
  std::vector<const char*> line;
  line.push_back(text.c_str());
  for (size_t i = 0; i < text.size(); i++)
    if (text[i] == '\n' && i + 1 < text.size()) line.push_back(text.c_str() + i + 1);
  auto at = [&](size_t k) -> const char* {
    if (k >= line.size()) throw ScriptError("gmsh mesh file ends early");
    return line[k];
  };
  char* end;
  size_t k = 4;
  const uint32_t np = (uint32_t)std::strtoul(at(k), &end, 10);
  std::string out = std::to_string(np) + "\n";
  char num[64];
  for (uint32_t i = 0; i < np; i++) {
    const char* q = at(k + 1 + i);
    std::strtod(q, &end);  // node id
    for (int a = 0; a < 3; a++) {
      std::snprintf(num, sizeof(num), a < 2 ? "%g " : "%g\n", std::strtod(end, &end));
      out += num;
    }
  }
  k += 1 + np + 2;
  const uint32_t ne = (uint32_t)std::strtoul(at(k), &end, 10);
  std::vector<std::array<uint32_t, 5>> tets;  // sorted nodes (0-based), material
  std::vector<std::array<uint32_t, 4>> tris;  // boundary id, nodes (0-based)
  for (uint32_t i = 0; i < ne; i++) {
    const char* q = at(k + 1 + i);
    std::strtoul(q, &end, 10);  // element id
    const uint32_t type = (uint32_t)std::strtoul(end, &end, 10);
    if (type != 4 && type != 2) continue;
    std::strtoul(end, &end, 10);  // number of tags
    const uint32_t tag = (uint32_t)std::strtoul(end, &end, 10);
    std::strtoul(end, &end, 10);  // second tag
    uint32_t n[4] = {0, 0, 0, 0};
    for (uint32_t j = 0; j < (type == 4 ? 4u : 3u); j++) n[j] = (uint32_t)std::strtoul(end, &end, 10) - 1;
    if (type == 4) {
      std::sort(n, n + 4);
      tets.push_back({n[0], n[1], n[2], n[3], tag});
    } else {
      tris.push_back({tag, n[0], n[1], n[2]});
    }
  }
  std::stable_sort(tets.begin(), tets.end(), [](const auto& a, const auto& b) {
    return std::lexicographical_compare(a.begin(), a.begin() + 4, b.begin(), b.begin() + 4);
  });
  out += std::to_string(tets.size()) + "\n";
  for (const auto& t : tets)
    out += std::to_string(t[4]) + " " + std::to_string(t[0] + 1) + " " + std::to_string(t[1] + 1) + " " +
           std::to_string(t[2] + 1) + " " + std::to_string(t[3] + 1) + "\n";
  out += std::to_string(tris.size()) + "\n";
  for (const auto& t : tris)
    out += std::to_string(t[0]) + " " + std::to_string(t[1] + 1) + " " + std::to_string(t[2] + 1) + " " +
           std::to_string(t[3] + 1) + "\n";
  return out;
}

bool is_zero(const Mat3& m) {
  for (auto& r : m.m)
    for (double x : r)
      if (x != 0) return false;
  return true;
}

// 3x3 determinant by cofactor expansion along the first row: the reference's
// zero test on sigma (Discretization.hpp:8604, 8041, 8897)
double mat_det(const Mat3& a) {
  const auto& m = a.m;
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// inverse of a small SPD matrix by Cholesky
void spd_inv(std::vector<double>& a, int n) {
  std::vector<double> L(n * n, 0.0), inv(n * n), y(n);
  for (int k = 0; k < n; k++) {
    double x = a[k * n + k];
    for (int j = 0; j < k; j++) x -= L[k * n + j] * L[k * n + j];
    if (!(x > 0)) throw std::runtime_error("local mass matrix is not positive definite (degenerate element?)");
    L[k * n + k] = std::sqrt(x);
    for (int i = k + 1; i < n; i++) {
      double v = a[i * n + k];
      for (int j = 0; j < k; j++) v -= L[i * n + j] * L[k * n + j];
      L[i * n + k] = v / L[k * n + k];
    }
  }
  for (int c = 0; c < n; c++) {
    for (int i = 0; i < n; i++) {
      double s = i == c ? 1.0 : 0.0;
      for (int j = 0; j < i; j++) s -= L[i * n + j] * y[j];
      y[i] = s / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
      double s = y[i];
      for (int j = i + 1; j < n; j++) s -= L[j * n + i] * inv[j * n + c];
      inv[i * n + c] = s / L[i * n + i];
    }
  }
  a.swap(inv);
}

double tridiag_max(const std::vector<double>& a, const std::vector<double>& bf) {
  const size_t m = a.size();
  double lo = a[0], hi = a[0];
  for (size_t i = 0; i < m; i++) {
    double r = (i > 0 ? std::fabs(bf[i - 1]) : 0) + (i + 1 < m ? std::fabs(bf[i]) : 0);
    lo = std::fmin(lo, a[i] - r);
    hi = std::fmax(hi, a[i] + r);
  }
  for (int it = 0; it < 200 && hi - lo > 1e-15 * std::fabs(hi); it++) {
    double x = 0.5 * (lo + hi), d = 1;
    int below = 0;
    for (size_t i = 0; i < m; i++) {
      d = a[i] - x - (i > 0 ? bf[i - 1] * bf[i - 1] / d : 0);
      if (d == 0) d = 1e-300;
      if (d < 0) below++;
    }
    if (below >= (int)m) hi = x;
    else lo = x;
  }
  return hi;
}
}  // namespace

// Triplets to CSR with duplicates summed.  Entries are bucketed by row in
// their given order (a counting sort), then each row is sorted by column with
// a stable sort: the same order as one stable sort by (row, column), so
// duplicates are summed in the order they were given, for any thread count.
HostCsr HostCsr::build(uint32_t nr, uint32_t nc, Trips& t, int threads) {
  HostCsr m;
  m.nrows = nr;
  m.ncols = nc;
  struct CV {
    int32_t c;
    double v;
  };
  // Stable bucketing in two levels: contiguous chunks of the triplets are
  // counted into row ranges and placed range by range in chunk order, then
  // each row range is bucketed by row; every row keeps the order its entries
  // were given in.
  const int64_t nt_ = (int64_t)t.size();
  const int64_t P = std::max<int64_t>(1, std::min<int64_t>(host_threads(threads), nt_ / 65536));
  const int64_t R = P;  // row ranges
  auto range_of = [&](uint32_t r) { return (int64_t)r * R / std::max<int64_t>(nr, 1); };
  std::vector<int64_t> rcut(R + 1);
  for (int64_t q = 0; q <= R; q++) {  // first row of each range
    int64_t lo = 0, hi = nr;
    while (lo < hi) {
      const int64_t mid = (lo + hi) / 2;
      if (range_of((uint32_t)mid) >= q) hi = mid;
      else lo = mid + 1;
    }
    rcut[q] = lo;
  }
  std::vector<int64_t> cc((size_t)P * R, 0);  // [chunk][range] counts, then offsets
  parallel_for(P, (int)P, [&](int64_t c0, int64_t c1) {
    for (int64_t c = c0; c < c1; c++)
      for (int64_t k = nt_ * c / P; k < nt_ * (c + 1) / P; k++) cc[c * R + range_of(t[k].r)]++;
  }, 1);
  std::vector<int64_t> rbeg(R + 1, 0);
  {
    int64_t o = 0;
    for (int64_t q = 0; q < R; q++) {
      rbeg[q] = o;
      for (int64_t c = 0; c < P; c++) {
        const int64_t x = cc[c * R + q];
        cc[c * R + q] = o;
        o += x;
      }
    }
    rbeg[R] = o;
  }
  Trips tmp(t.size());
  parallel_for(P, (int)P, [&](int64_t c0, int64_t c1) {
    for (int64_t c = c0; c < c1; c++) {
      int64_t* pos = &cc[c * R];
      for (int64_t k = nt_ * c / P; k < nt_ * (c + 1) / P; k++) tmp[pos[range_of(t[k].r)]++] = t[k];
    }
  }, 1);
  Trips().swap(t);
  std::vector<int64_t> start(nr + 1, 0);
  std::vector<CV, default_init_allocator<CV>> b(tmp.size());
  parallel_for(R, (int)R, [&](int64_t q0, int64_t q1) {
    for (int64_t q = q0; q < q1; q++) {
      const int64_t r0 = rcut[q], r1 = rcut[q + 1];
      std::vector<int64_t> pos(r1 - r0, 0);
      for (int64_t k = rbeg[q]; k < rbeg[q + 1]; k++) pos[tmp[k].r - r0]++;
      int64_t o = rbeg[q];
      for (int64_t r = r0; r < r1; r++) {  // each range writes the starts of its own rows only
        const int64_t x = pos[r - r0];
        start[r] = pos[r - r0] = o;
        o += x;
      }
      for (int64_t k = rbeg[q]; k < rbeg[q + 1]; k++) {
        const Trip& x = tmp[k];
        b[pos[x.r - r0]++] = {(int32_t)x.c, x.v};
      }
    }
  }, 1);
  start[nr] = (int64_t)b.size();
  Trips().swap(tmp);
  std::vector<int64_t> cnt(nr + 1, 0);
  parallel_for(nr, threads, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; r++) {
      const int64_t lo = start[r], hi = start[r + 1];
      if (hi - lo <= 32) {
        for (int64_t k = lo + 1; k < hi; k++) {  // insertion sort: stable
          const CV e = b[k];
          int64_t j = k;
          while (j > lo && b[j - 1].c > e.c) {
            b[j] = b[j - 1];
            j--;
          }
          b[j] = e;
        }
      } else {
        std::stable_sort(b.begin() + lo, b.begin() + hi, [](const CV& x, const CV& y) { return x.c < y.c; });
      }
      int64_t w = lo;
      for (int64_t k = lo; k < hi; k++) {
        if (w > lo && b[w - 1].c == b[k].c) b[w - 1].v += b[k].v;
        else b[w++] = b[k];
      }
      cnt[r + 1] = w - lo;
    }
  });
  m.ptr.assign(nr + 1, 0);
  for (uint32_t r = 0; r < nr; r++) m.ptr[r + 1] = m.ptr[r] + cnt[r + 1];
  m.col.resize(m.ptr[nr]);
  m.val.resize(m.ptr[nr]);
  parallel_for(nr, threads, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; r++)
      for (int64_t k = 0; k < cnt[r + 1]; k++) {
        m.col[m.ptr[r] + k] = b[start[r] + k].c;
        m.val[m.ptr[r] + k] = b[start[r] + k].v;
      }
  });
  return m;
}

void HostCsr::mul(const double* x, double* y, int threads) const {
  parallel_for(nrows, threads, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; r++) {
      double s = 0;
      for (int64_t k = ptr[r]; k < ptr[r + 1]; k++) s += val[k] * x[col[k]];
      y[r] = s;
    }
  });
}

// ------------------------------------------------------------------ set-up
TetSim::TetSim(Script& sc, uint32_t label, const RunOptions& opt, bool device)
    : sc_(sc), opt_(opt), label_(label) {
  sim_ = sc_.simulations.at(label);
  out_ = sc_.outputs[sim_.output];
  out_.initialize();
  method_ = sim_.method == "dga" ? 1 : (sim_.method == "fem" ? 3 : 2);
  src_labels_ = sim_.sources;
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char* what) {
    auto t1 = std::chrono::steady_clock::now();
    if (opt_.verbose) std::printf("  set-up %-14s %8.3f s\n", what, std::chrono::duration<double>(t1 - t0).count());
    t0 = t1;
  };
  read_mesh();
  lap("mesh");
  classify();
  lap("classes");
  build_ops();
  lap("operators");
  locate_probes();
  lap("probes");
  // loop length: i = 1 .. while i dt <= duration (Discretization.hpp:810, 1459)
  nsteps_ = 0;
  while ((double)(nsteps_ + 1) * dt_ <= sim_.duration) nsteps_++;
  // print schedule: dga exports t = 0 and after every step (index i <-> i dt),
  // gfdtd exports U^{i-1} inside step i (index i-1 <-> (i-1) dt)
  const uint64_t nsched = method_ == 1 ? nsteps_ + 1 : nsteps_;
  slot_of_step_.assign(nsched + 1, -1);
  if (out_.mode == "probepoint" || out_.mode == "silo") {
    Output o = out_;
    for (uint64_t i = 0; i < nsched; i++) {
      // gfdtd stamps the export of loop step i+1 as current_time - t_step
      // (Discretization.hpp:1470-1471), which is not always (double)i * dt
      double t = method_ == 1 ? (double)i * dt_ : (double)(i + 1) * dt_ - dt_;
      if (o.allow_print(t)) {
        slot_of_step_[i] = nslots_++;
        sample_times_.push_back(t);
      }
    }
  }
  build_sources();
  if (!device) return;
  if (method_ >= 2) group_.reset(new TetGroup({this}, opt_, false));
  else alloc_and_upload();
}

uint64_t TetSim::device_bytes() const { return group_ ? group_->device_bytes() : dev_bytes_; }
double TetSim::last_step_ms() const { return group_ ? group_->last_step_ms() : last_ms_; }
int TetSim::kernels_per_step() const {
  if (group_) return group_->kernels_per_step();
  const int np = probe_tet_.empty() ? 0 : 1;
  return 6 + np + (src_edge_.empty() ? 0 : 1) + (dp_.nq > 0 ? 1 : 0) + (dp_.nfe > 0 ? 1 : 0);
}

void TetSim::release_host() {
  auto drop = [](auto& v) { std::remove_reference_t<decltype(v)>().swap(v); };
  for (HostCsr* m : {&Ct_, &N_, &H_, &E_, &A_, &R_, &Sig_, &Q_, &Mq_}) {
    drop(m->ptr);
    drop(m->col);
    drop(m->val);
  }
  drop(vtf_); drop(ftv_); drop(fte_); drop(star_ptr_); drop(star_edge_); drop(nvol_ptr_); drop(nvol_);
  drop(bnd_edge_); drop(bnd_dual_); drop(edge_src_); drop(carrier_); drop(init_U_); drop(init_I_);
  drop(init_src_); drop(jacobi_); drop(cls_); drop(pec_);
  drop(hp_); drop(nr_); drop(frac_off_); drop(fe_edge_); drop(fe_a_); drop(fe_b_);
}

TetSim::~TetSim() {
  group_.reset();
  if (pinned_) cudaFreeHost(pinned_);
  for (void* p : allocs_) cudaFree(p);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

void TetSim::read_mesh() {
  // netgen neutral reader (Discretization.hpp:5924-6101); gmsh files are
  // converted to the same text first (Discretization.hpp:5890-5895)
  const Mesh& msh = sc_.meshes[sim_.mesh];
  std::ifstream fin(msh.file.c_str(), std::ios::binary);
  if (!fin.is_open()) throw ScriptError("Invalid mesh file name");
  std::stringstream ss;
  ss << fin.rdbuf();
  const std::string buf = msh.mesher == "gmsh" ? gmsh_to_netgen(ss.str()) : ss.str();
  const char* p = buf.c_str();
  if (*p < '0' || *p > '9') my_throw(0, "Undefined mesh type! Available: tetrahedral, cartesian");
  char* end;
  const uint32_t np = (uint32_t)std::strtoul(p, &end, 10);
  pts_.resize(np);
  for (uint32_t i = 0; i < np; i++) {
    double x = std::strtod(end, &end), y = std::strtod(end, &end), z = std::strtod(end, &end);
    pts_[i] = {msh.scale * x, msh.scale * y, msh.scale * z};
  }
  const uint32_t nt = (uint32_t)std::strtoul(end, &end, 10);
  std::vector<std::array<int32_t, 5>> tt;  // 4 sorted nodes + material
  tt.reserve(nt);
  for (uint32_t i = 0; i < nt; i++) {
    int32_t m = (int32_t)std::strtoul(end, &end, 10);
    std::array<int32_t, 4> q;
    for (int k = 0; k < 4; k++) q[k] = (int32_t)std::strtoul(end, &end, 10) - 1;
    std::sort(q.begin(), q.end());
    if (m != 7) tt.push_back({q[0], q[1], q[2], q[3], m});
  }
  const int nth = opt_.setup_threads;
  parallel_stable_sort(tt.begin(), tt.end(), nth, [](const auto& a, const auto& b) {
    return std::lexicographical_compare(a.begin(), a.begin() + 4, b.begin(), b.begin() + 4);
  });
  const uint32_t L = (uint32_t)tt.size();
  vols_.resize(L);
  vol_mat_.resize(L);
  cell_vol_.resize(L);
  for (uint32_t k = 0; k < L; k++) {
    vols_[k] = {tt[k][0], tt[k][1], tt[k][2], tt[k][3]};
    vol_mat_[k] = (uint32_t)tt[k][4];
    const auto& t = vols_[k];
    V3 v1 = sub(pts_[t[1]], pts_[t[0]]), v2 = sub(pts_[t[2]], pts_[t[0]]), v3 = sub(pts_[t[3]], pts_[t[0]]);
    cell_vol_[k] = dot(v1, cross(v2, v3)) / 6.0;
    const Material& mt = sc_.materials[vol_mat_[k]];
    // conductivity enters gfdtd and fem through SigMat and dga through its
    // edge classes; magnetic losses (chi) enter dga through its face classes
    if (!is_zero(mt.chi) && method_ != 1)
      throw UnsupportedError("magnetic losses (chi) on tetrahedra are supported with method dga only");
  }
  // faces: packed keys when node ids fit in 21 bits, else tuple order
  const bool packed = np < (1u << 21);
  auto fkey = [](int32_t a, int32_t b, int32_t c) {
    return ((uint64_t)a << 42) | ((uint64_t)b << 21) | (uint64_t)c;
  };
  std::vector<std::pair<uint64_t, uint32_t>> fk(4 * (size_t)L);
  std::vector<std::array<int32_t, 3>> ftup;
  if (!packed) ftup.resize(4 * (size_t)L);
  parallel_for(L, nth, [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; k++) {
      const auto& t = vols_[k];
      const int32_t tri[4][3] = {{t[0], t[1], t[2]}, {t[0], t[1], t[3]}, {t[0], t[2], t[3]}, {t[1], t[2], t[3]}};
      for (int q = 0; q < 4; q++) {
        size_t slot = k + (size_t)q * L;
        fk[slot] = {packed ? fkey(tri[q][0], tri[q][1], tri[q][2]) : slot, (uint32_t)slot};
        if (!packed) ftup[slot] = {tri[q][0], tri[q][1], tri[q][2]};
      }
    }
  });
  // (key, slot) pairs are distinct: any sort gives this order
  if (packed) parallel_stable_sort(fk.begin(), fk.end(), nth, std::less<std::pair<uint64_t, uint32_t>>());
  else
    parallel_stable_sort(fk.begin(), fk.end(), nth,
                         [&](const auto& a, const auto& b) { return ftup[a.first] < ftup[b.first]; });
  std::vector<int32_t> flab(4 * (size_t)L);
  auto face_tuple = [&](size_t slot) -> std::array<int32_t, 3> {
    uint32_t k = (uint32_t)(slot % L);
    int q = (int)(slot / L);
    const auto& t = vols_[k];
    const int32_t tri[4][3] = {{t[0], t[1], t[2]}, {t[0], t[1], t[3]}, {t[0], t[2], t[3]}, {t[1], t[2], t[3]}};
    return {tri[q][0], tri[q][1], tri[q][2]};
  };
  // a new face starts wherever the sorted tuple changes: mark, number by a
  // prefix, then place (the numbering of one sequential pass)
  const int64_t nk = (int64_t)fk.size();
  std::vector<int32_t> fid(nk);
  parallel_for(nk, nth, [&](int64_t q0, int64_t q1) {
    for (int64_t q = q0; q < q1; q++)
      fid[q] = q == 0 || face_tuple(fk[q].second) != face_tuple(fk[q - 1].second) ? 1 : 0;
  });
  for (int64_t q = 1; q < nk; q++) fid[q] += fid[q - 1];  // 1-based face number
  faces_.resize(nk ? (size_t)fid[nk - 1] : 0);
  parallel_for(nk, nth, [&](int64_t q0, int64_t q1) {
    for (int64_t q = q0; q < q1; q++) {
      const int32_t f = fid[q] - 1;
      if (q == 0 || fid[q] != fid[q - 1]) faces_[f] = face_tuple(fk[q].second);
      flab[fk[q].second] = f;
    }
  });
  fk.clear();
  fk.shrink_to_fit();
  const uint32_t NF = (uint32_t)faces_.size();
  ftv_.assign(NF, {-1, -1});
  vtf_.resize(L);
  for (uint32_t k = 0; k < L; k++) {
    const int32_t f0 = flab[k], f1 = flab[k + L], f2 = flab[k + 2 * (size_t)L], f3 = flab[k + 3 * (size_t)L];
    for (int32_t f : {f0, f1, f2, f3}) {
      if (ftv_[f][0] < 0) ftv_[f][0] = (int32_t)k;
      else ftv_[f][1] = (int32_t)k;
    }
    vtf_[k] = {f3, f2, f1, f0};  // opposite nodes 0..3 (Discretization.hpp:6239-6267)
  }
  // edges
  std::vector<uint64_t, default_init_allocator<uint64_t>> ek(3 * (size_t)NF);
  parallel_for(NF, nth, [&](int64_t f0, int64_t f1) {
    for (int64_t f = f0; f < f1; f++) {
      const auto& s = faces_[f];
      ek[f] = ((uint64_t)s[0] << 32) | (uint32_t)s[1];
      ek[f + NF] = ((uint64_t)s[0] << 32) | (uint32_t)s[2];
      ek[f + 2 * (size_t)NF] = ((uint64_t)s[1] << 32) | (uint32_t)s[2];
    }
  });
  std::vector<uint64_t> eu(ek.begin(), ek.end());
  parallel_stable_sort(eu.begin(), eu.end(), nth, std::less<uint64_t>());
  eu.erase(std::unique(eu.begin(), eu.end()), eu.end());
  edges_.resize(eu.size());
  for (size_t e = 0; e < eu.size(); e++) edges_[e] = {(int32_t)(eu[e] >> 32), (int32_t)(eu[e] & 0xffffffffu)};
  auto eid = [&](uint64_t key) { return (int32_t)(std::lower_bound(eu.begin(), eu.end(), key) - eu.begin()); };
  fte_.resize(NF);
  parallel_for(NF, nth, [&](int64_t f0, int64_t f1) {
    for (int64_t f = f0; f < f1; f++) fte_[f] = {eid(ek[f]), eid(ek[f + NF]), eid(ek[f + 2 * (size_t)NF])};
  });
  const uint32_t NE = (uint32_t)edges_.size();
  // node stars (edges ascending) and node -> tets (ascending)
  star_ptr_.assign(np + 1, 0);
  for (auto& e : edges_) { star_ptr_[e[0] + 1]++; star_ptr_[e[1] + 1]++; }
  for (uint32_t i = 0; i < np; i++) star_ptr_[i + 1] += star_ptr_[i];
  star_edge_.resize(star_ptr_[np]);
  {
    std::vector<int64_t> pos(star_ptr_.begin(), star_ptr_.end() - 1);
    for (uint32_t e = 0; e < NE; e++) {
      star_edge_[pos[edges_[e][0]]++] = (int32_t)e;
      star_edge_[pos[edges_[e][1]]++] = (int32_t)e;
    }
  }
  nvol_ptr_.assign(np + 1, 0);
  for (auto& t : vols_)
    for (int32_t n : t) nvol_ptr_[n + 1]++;
  for (uint32_t i = 0; i < np; i++) nvol_ptr_[i + 1] += nvol_ptr_[i];
  nvol_.resize(nvol_ptr_[np]);
  {
    std::vector<int64_t> pos(nvol_ptr_.begin(), nvol_ptr_.end() - 1);
    for (uint32_t k = 0; k < L; k++)
      for (int32_t n : vols_[k]) nvol_[pos[n]++] = (int32_t)k;
  }
  // C^T: edge -> faces ascending, sign in bit 31
  {
    HostCsr::Trips t(3 * (size_t)NF);
    parallel_for(NF, nth, [&](int64_t f0, int64_t f1) {
      for (int64_t f = f0; f < f1; f++) {
        t[3 * f] = {(uint32_t)fte_[f][0], (uint32_t)f, 1.0};
        t[3 * f + 1] = {(uint32_t)fte_[f][1], (uint32_t)f, -1.0};
        t[3 * f + 2] = {(uint32_t)fte_[f][2], (uint32_t)f, 1.0};
      }
    });
    Ct_ = HostCsr::build(NE, NF, t, nth);
  }
  // boundary faces and their dual edges (Discretization.hpp:6380-6489)
  bnd_edge_.assign(NE, -1);
  auto fbar = [&](uint32_t f) {
    const auto &a = pts_[faces_[f][0]], &b = pts_[faces_[f][1]], &c = pts_[faces_[f][2]];
    return V3{(a[0] + b[0] + c[0]) / 3.0, (a[1] + b[1] + c[1]) / 3.0, (a[2] + b[2] + c[2]) / 3.0};
  };
  auto vbar = [&](int32_t v) {
    V3 r{0, 0, 0};
    for (int q = 0; q < 4; q++)
      for (int a = 0; a < 3; a++) r[a] += pts_[vols_[v][q]][a];
    return V3{r[0] / 4.0, r[1] / 4.0, r[2] / 4.0};
  };
  for (uint32_t f = 0; f < NF; f++) {
    if (ftv_[f][0] < 0) throw std::invalid_argument("Conductor boundary cannot be on mesh boundary!");
    if (ftv_[f][1] >= 0) continue;
    for (int32_t e : fte_[f]) {
      if (bnd_edge_[e] < 0) {
        bnd_edge_[e] = (int32_t)bnd_dual_.size();
        bnd_dual_.push_back(fbar(f));
      } else {
        V3& bd = bnd_dual_[bnd_edge_[e]];
        bd = sub(fbar(f), bd);
        V3 ev = sub(pts_[edges_[e][1]], pts_[edges_[e][0]]);
        V3 fv = cross(sub(pts_[faces_[f][1]], pts_[faces_[f][0]]), sub(pts_[faces_[f][2]], pts_[faces_[f][0]]));
        if (dot(fv, sub(vbar(ftv_[f][0]), fbar(f))) >= 0) fv = scale(fv, -1);
        if (dot(cross(ev, fv), bd) > 0) bd = scale(bd, -1);
        bd = scale(bd, -1);
      }
    }
  }
  // boundary triangles: PEC and source surfaces (Discretization.hpp:6612-6754)
  const uint32_t ntri = (uint32_t)std::strtoul(end, &end, 10);
  std::vector<uint32_t> edge_bc(NE, 0);
  pec_.assign(NE, 0);
  edge_src_.assign(NE, {});
  for (uint32_t i = 0; i < ntri; i++) {
    uint32_t bid = (uint32_t)std::strtoul(end, &end, 10);
    std::array<int32_t, 3> s;
    for (int k = 0; k < 3; k++) s[k] = (int32_t)std::strtoul(end, &end, 10) - 1;
    std::sort(s.begin(), s.end());
    auto it = std::lower_bound(faces_.begin(), faces_.end(), s);
    if (it == faces_.end() || *it != s) continue;
    const uint32_t f = (uint32_t)(it - faces_.begin());
    const uint32_t which = bid < 100 ? sc_.bnd_to_bc[bid] : 0;
    if (which != 0) {
      auto bc = sc_.bcs.find(which);
      if (bc != sc_.bcs.end() && bc->second.type == "pec")
        for (int32_t e : fte_[f]) {
          edge_bc[e] = which;
          edge_src_[e].clear();
          pec_[e] = 1;
          if (bnd_edge_[e] >= 0) {
            bnd_dual_[bnd_edge_[e]] = {0, 0, 0};
            bnd_edge_[e] = -1;
          }
        }
    } else {
      for (uint32_t sl : src_labels_) {
        Source& src = sc_.sources[sl];
        if (std::find(src.surfaces.begin(), src.surfaces.end(), bid) == src.surfaces.end() || src.st == "b") continue;
        for (int32_t e : fte_[f])
          if (!pec_[e] && std::find(edge_src_[e].begin(), edge_src_[e].end(), sl) == edge_src_[e].end())
            edge_src_[e].push_back(sl);
      }
    }
  }
}

void TetSim::classify() {
  // source consistency filter and edge classes (Discretization.hpp:6758-6859)
  const uint32_t NE = (uint32_t)edges_.size();
  cls_.assign(NE, 1);
  for (uint32_t e = 0; e < NE; e++) {
    auto& es = edge_src_[e];
    if (!es.empty()) {
      const Source& f = sc_.sources[es[0]];
      uint32_t fs = f.surfaces.empty() ? 0 : f.surfaces[0];
      std::vector<uint32_t> keep;
      for (uint32_t s : es) {
        const Source& x = sc_.sources[s];
        if (x.st == f.st && (x.surfaces.empty() ? 0 : x.surfaces[0]) == fs) keep.push_back(s);
      }
      es.swap(keep);
    }
    bool dir = pec_[e] != 0;
    for (uint32_t s : es)
      if (sc_.sources[s].st == "e") dir = true;
    if (dir) cls_[e] = 4;
  }
  if (method_ != 1) return;
  // dga with conducting tets (Discretization.hpp:6186-6215, 6776-6903).  A
  // node holds the eps and sigma of its first tet; its class bits: 1 that
  // sigma is non-zero, 2 that a later tet differs in eps, 4 in sigma.
  const uint32_t NP = (uint32_t)pts_.size();
  std::vector<uint8_t> nb(NP, 0);
  std::vector<int32_t> first(NP, -1);  // material of the node's first tet
  auto same = [](const Mat3& a, const Mat3& b) {  // element-wise ==, as Eigen compares
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        if (a.m[i][j] != b.m[i][j]) return false;
    return true;
  };
  for (size_t v = 0; v < vols_.size(); v++) {
    const Material& mt = sc_.materials.at(vol_mat_[v]);
    for (int32_t p : vols_[v]) {
      // a node counts as seen once it holds a non-zero eps (the reference's test)
      if (first[p] >= 0 && !is_zero(sc_.materials.at(first[p]).eps)) {
        const Material& f = sc_.materials.at(first[p]);
        if (!same(mt.sigma, f.sigma)) nb[p] |= 4;
        if (!same(mt.eps, f.eps)) nb[p] |= 2;
        if (!is_zero(f.sigma)) nb[p] |= 1;
      } else {
        first[p] = (int32_t)vol_mat_[v];
        if (!is_zero(mt.sigma)) nb[p] |= 1;
      }
    }
  }
  // free edges: fractured (3) if an end's class exceeds 2, the classes sum to
  // 1 or 3, or the ends' first sigmas differ; lossless (1) if an end has
  // class 0 or 2; else uniformly conducting (2).  A fractured edge's ends get
  // a block of U_c as long as their star.
  frac_off_.assign(NP, -1);
  q_size_ = 0;
  dga_frac_ = false;
  for (uint32_t e = 0; e < NE; e++) {
    if (cls_[e] == 4) continue;
    const int32_t p0 = edges_[e][0], p1 = edges_[e][1];
    const int r0 = nb[p0], r1 = nb[p1];
    const bool sig_eq = same(sc_.materials.at(first[p0]).sigma, sc_.materials.at(first[p1]).sigma);
    if (r0 > 2 || r1 > 2 || r0 + r1 == 1 || r0 + r1 == 3 || !sig_eq) {
      cls_[e] = 3;
      for (int32_t p : {p0, p1})
        if (frac_off_[p] < 0) {
          frac_off_[p] = q_size_;
          q_size_ += (uint32_t)(star_ptr_[p + 1] - star_ptr_[p]);
        }
    } else if (!(r0 == 2 || r1 == 2 || r0 == 0 || r1 == 0)) {
      cls_[e] = 2;
    }
    dga_frac_ = dga_frac_ || cls_[e] != 1;
  }
  fe_edge_.clear(); fe_a_.clear(); fe_b_.clear();
  for (uint32_t e = 0; e < NE; e++) {
    if (cls_[e] != 3) continue;
    int32_t at[2];
    for (int a = 0; a < 2; a++) {
      const int32_t p = edges_[e][a];
      const int64_t b0 = star_ptr_[p];
      const int64_t pos = std::lower_bound(star_edge_.begin() + b0, star_edge_.begin() + star_ptr_[p + 1], (int32_t)e) -
                          (star_edge_.begin() + b0);
      at[a] = (int32_t)(frac_off_[p] + pos);
    }
    fe_edge_.push_back((int32_t)e);
    fe_a_.push_back(at[0]);
    fe_b_.push_back(at[1]);
  }
}

std::array<int32_t, 6> TetSim::vol_edges(uint32_t v) const {
  // local order ab, bc, ac, ad, bd, cd: the sorted edges of the tet after
  // the reference's two swaps (Discretization.hpp:10309-10314)
  std::array<int32_t, 6> es;
  int n = 0;
  for (int q = 0; q < 4; q++)
    for (int32_t e : fte_[vtf_[v][q]]) {
      bool seen = false;
      for (int k = 0; k < n; k++) seen = seen || es[k] == e;
      if (!seen) es[n++] = e;
    }
  std::sort(es.begin(), es.end());
  std::swap(es[1], es[2]);
  std::swap(es[1], es[3]);
  return es;
}

void TetSim::build_ops() {
  const uint32_t NE = (uint32_t)edges_.size(), NF = (uint32_t)faces_.size(), L = (uint32_t)vols_.size();
  auto ebar = [&](int32_t e) {
    const auto &a = pts_[edges_[e][0]], &b = pts_[edges_[e][1]];
    return V3{0.5 * (a[0] + b[0]), 0.5 * (a[1] + b[1]), 0.5 * (a[2] + b[2])};
  };
  auto fbar = [&](int32_t f) {
    const auto &a = pts_[faces_[f][0]], &b = pts_[faces_[f][1]], &c = pts_[faces_[f][2]];
    return V3{(a[0] + b[0] + c[0]) / 3.0, (a[1] + b[1] + c[1]) / 3.0, (a[2] + b[2] + c[2]) / 3.0};
  };
  const int nth = opt_.setup_threads;
  // conducting tets (gfdtd, fem): sigma with a non-zero determinant, the
  // reference's test (Discretization.hpp:8604, 8041), by cofactor expansion
  // along the first row
  std::vector<uint8_t> sig_tet(L, 0);
  lossy_ = false;
  if (method_ >= 2)
    for (uint32_t v = 0; v < L; v++)
      if (mat_det(sc_.materials.at(vol_mat_[v]).sigma) != 0) sig_tet[v] = 1, lossy_ = true;
  // N = sum of per-tet inverse magnetic blocks (Discretization.hpp:8754-8807, 9158-9255);
  // the blocks are formed in parallel, then listed in tet order.  mag_mass is
  // the per-tet magnetic mass M from the dual area vectors, or with chi in
  // place of mu the magnetic-loss matrix Z (:8778-8802).
  auto mag_mass = [&](uint32_t v, const Mat3& mat, double* M) {
    auto es = vol_edges(v);
    V3 eb[6], fb[4];
    for (int i = 0; i < 6; i++) eb[i] = ebar(es[i]);
    for (int i = 0; i < 4; i++) fb[i] = fbar(vtf_[v][i]);
    V3 vb{0, 0, 0};
    for (int q = 0; q < 4; q++)
      for (int a = 0; a < 3; a++) vb[a] += pts_[vols_[v][q]][a];
    vb = {vb[0] / 4.0, vb[1] / 4.0, vb[2] / 4.0};
    const double sgn = cell_vol_[v] < 0 ? -0.5 : 0.5;
    const V3 fv[6] = {scale(cross(sub(vb, eb[0]), sub(fb[2], fb[3])), sgn),
                      scale(cross(sub(vb, eb[1]), sub(fb[0], fb[3])), sgn),
                      scale(cross(sub(vb, eb[2]), sub(fb[3], fb[1])), sgn),
                      scale(cross(sub(vb, eb[3]), sub(fb[1], fb[2])), sgn),
                      scale(cross(sub(vb, eb[4]), sub(fb[2], fb[0])), sgn),
                      scale(cross(sub(vb, eb[5]), sub(fb[0], fb[1])), sgn)};
    auto d = [&](int a, int b) { return dot(fv[a], mv(mat, fv[b])); };
    const double c = 36.0 / std::fabs(cell_vol_[v]);
    const double m[16] = {(d(0, 0) + d(2, 2) + d(3, 3)) * c, (-d(1, 2) - d(3, 4)) * c,
                          (-d(0, 1) + d(3, 5)) * c,          (d(0, 4) + d(2, 5)) * c,
                          0, (d(0, 0) + d(1, 1) + d(4, 4)) * c, (-d(0, 2) - d(4, 5)) * c, (d(0, 3) - d(1, 5)) * c,
                          0, 0, (d(1, 1) + d(2, 2) + d(5, 5)) * c, (-d(2, 3) - d(1, 4)) * c,
                          0, 0, 0, (d(3, 3) + d(4, 4) + d(5, 5)) * c};
    for (int i = 0; i < 16; i++) M[i] = m[i];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < i; j++) M[4 * i + j] = M[4 * j + i];
  };
  std::vector<double> blk(16 * (size_t)L);
  auto build_N = [&]() {
    // nonzero entries in tet order, at positions from a prefix of the counts
    std::vector<int64_t> off(L + 1, 0);
    parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
      for (int64_t v = v0; v < v1; v++)
        for (int k = 0; k < 16; k++) off[v + 1] += blk[16 * v + k] != 0;
    });
    for (uint32_t v = 0; v < L; v++) off[v + 1] += off[v];
    HostCsr::Trips t(off[L]);
    parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
      for (int64_t v = v0; v < v1; v++) {
        int64_t w = off[v];
        for (int j = 0; j < 4; j++)
          for (int k = 0; k < 4; k++) {
            const double x = blk[16 * v + 4 * j + k];
            if (x != 0) t[w++] = {(uint32_t)vtf_[v][j], (uint32_t)vtf_[v][k], x};
          }
      }
    });
    N_ = HostCsr::build(NF, NF, t, nth);
  };
  parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
    std::vector<double> M(16);
    for (uint32_t v = (uint32_t)v0; v < (uint32_t)v1; v++) {
      mag_mass(v, sc_.materials.at(vol_mat_[v]).mu, M.data());
      spd_inv(M, 4);
      std::copy(M.begin(), M.end(), blk.begin() + 16 * (size_t)v);
    }
  });
  build_N();
  auto primal_area = [&](uint32_t v) {
    const auto& n = vols_[v];
    V3 e[6] = {sub(pts_[n[1]], pts_[n[0]]), sub(pts_[n[2]], pts_[n[1]]), sub(pts_[n[2]], pts_[n[0]]),
               sub(pts_[n[3]], pts_[n[0]]), sub(pts_[n[3]], pts_[n[1]]), sub(pts_[n[3]], pts_[n[2]])};
    return std::array<V3, 4>{scale(cross(e[1], e[4]), 0.5), scale(cross(e[2], e[3]), 0.5),
                             scale(cross(e[0], e[3]), 0.5), scale(cross(e[0], e[2]), 0.5)};
  };
  // node -> local position of the three incident tet edges
  static const int kEd[4][3] = {{0, 2, 3}, {0, 1, 4}, {1, 2, 5}, {3, 4, 5}};
  if (method_ == 1) {
    // node-star eps-matrices (Discretization.hpp:8856-9123) and their inverses
    static const int kFv[4][3] = {{1, 2, 3}, {0, 2, 3}, {1, 0, 3}, {0, 1, 2}};
    static const double kSg[4][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {1, 1, 1}};
    static const int kVtfSign[4] = {1, -1, 1, -1};  // vtf signs (Discretization.hpp:6239-6267)
    // star matrix of eps, or of sigma over the star's tets whose sigma has a
    // non-zero determinant (:8897); returns whether such a tet exists
    auto star_mass = [&](uint32_t nid, bool sigma, std::vector<double>& E) {
      const int64_t b0 = star_ptr_[nid];
      const int n = (int)(star_ptr_[nid + 1] - b0);
      E.assign((size_t)n * n, 0.0);
      bool any = false;
      for (int64_t q = nvol_ptr_[nid]; q < nvol_ptr_[nid + 1]; q++) {
        const int32_t vv = nvol_[q];
        const Mat3& mat = sigma ? sc_.materials.at(vol_mat_[vv]).sigma : sc_.materials.at(vol_mat_[vv]).eps;
        if (sigma && mat_det(mat) == 0) continue;
        any = true;
        auto el = vol_edges(vv);
        auto fv = primal_area(vv);
        const double V = std::fabs(cell_vol_[vv]);
        int k = 0;
        while (vols_[vv][k] != (int32_t)nid) k++;
        int li[3];
        V3 w[3];
        for (int a = 0; a < 3; a++) {
          li[a] = (int)(std::lower_bound(star_edge_.begin() + b0, star_edge_.begin() + b0 + n, el[kEd[k][a]]) -
                        (star_edge_.begin() + b0));
          w[a] = scale(fv[kFv[k][a]], kSg[k][a] * 2.0 / 3.0 / V * kVtfSign[kFv[k][a]]);
        }
        for (int a = 0; a < 3; a++)
          for (int b = a; b < 3; b++) {
            double val = dot(w[a], mv(mat, w[b])) * V / 4;
            E[li[a] * n + li[b]] += val;
            if (a != b) E[li[b] * n + li[a]] = E[li[a] * n + li[b]];
          }
      }
      return any;
    };
    // node stars in parallel, each into its own lists, then concatenated in
    // node order (the order a sequential pass would list them)
    // the unmasked inverses Einv only feed the dt estimate
    const bool want_einv = dt_estimate_needed();
    const size_t NP = pts_.size();
    std::vector<HostCsr::Trips> ein_n(NP), h_n(NP);
    parallel_for((int64_t)NP, nth, [&](int64_t n0, int64_t n1) {
      std::vector<double> E;
      for (uint32_t nid = (uint32_t)n0; nid < (uint32_t)n1; nid++) {
        HostCsr::Trips& einv_t = ein_n[nid];
        HostCsr::Trips& h_t = h_n[nid];
        const int64_t b0 = star_ptr_[nid];
        const int n = (int)(star_ptr_[nid + 1] - b0);
        star_mass(nid, false, E);
        if (want_einv) {
          std::vector<double> Hl = E;
          spd_inv(Hl, n);
          for (int j = 0; j < n; j++)
            for (int k = j; k < n; k++)
              if (Hl[j * n + k] != 0) {
                einv_t.push_back({(uint32_t)star_edge_[b0 + j], (uint32_t)star_edge_[b0 + k], Hl[j * n + k]});
                if (j != k) einv_t.push_back({(uint32_t)star_edge_[b0 + k], (uint32_t)star_edge_[b0 + j], Hl[j * n + k]});
              }
        }
        if (dga_frac_) continue;  // the masked inverses need dt (below)
        // masked inverse (Discretization.hpp:9263-9333)
        for (int j = 0; j < n; j++)
          if (cls_[star_edge_[b0 + j]] == 4) {
            for (int k = 0; k < n; k++) E[j * n + k] = E[k * n + j] = 0;
            E[j * n + j] = 1;
          }
        spd_inv(E, n);
        for (int j = 0; j < n; j++) {
          const int32_t ej = star_edge_[b0 + j];
          if (cls_[ej] != 1) continue;
          for (int k = j; k < n; k++) {
            const int32_t ek = star_edge_[b0 + k];
            if (cls_[ek] == 4 || E[j * n + k] == 0) continue;
            h_t.push_back({(uint32_t)ej, (uint32_t)ek, E[j * n + k]});
            if (j != k) h_t.push_back({(uint32_t)ek, (uint32_t)ej, E[j * n + k]});
          }
        }
      }
    });
    HostCsr::Trips einv_t;
    for (size_t nid = 0; nid < NP; nid++) {
      einv_t.insert(einv_t.end(), ein_n[nid].begin(), ein_n[nid].end());
      HostCsr::Trips().swap(ein_n[nid]);
    }
    HostCsr Einv;
    if (want_einv) Einv = HostCsr::build(NE, NE, einv_t, nth);
    dt_est_ = sim_.courant * estimate_dt(Einv, false);
    // magnetic losses (Discretization.hpp:6357-6542, 9128-9205), with the
    // run's dt: a face is class 1 when its tets have chi = 0, class 2 when
    // they share one chi (and mu); a face whose tets differ is fractured in
    // the reference, which then reads its old values from the electric state
    // (Old_F_c, :586), so it is refused.  A tet whose chi has a non-zero
    // determinant gets the block N = (M + dt/2 Z)^-1 and RS = N (M - dt/2 Z);
    // R of a class-2 face is the diagonal of RS in its last tet.  dt above
    // comes from the lossless N, as in the reference.
    bool chi_any = false;
    for (uint32_t v = 0; v < L; v++) chi_any = chi_any || !is_zero(sc_.materials.at(vol_mat_[v]).chi);
    if (chi_any) {
      auto same = [](const Mat3& a, const Mat3& b) {
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++)
            if (a.m[i][j] != b.m[i][j]) return false;
        return true;
      };
      for (uint32_t f = 0; f < NF; f++) {
        if (ftv_[f][1] < 0) continue;
        const Material& m0 = sc_.materials.at(vol_mat_[ftv_[f][0]]);
        const Material& m1 = sc_.materials.at(vol_mat_[ftv_[f][1]]);
        if ((!is_zero(m0.chi) || !is_zero(m1.chi)) && (!same(m0.chi, m1.chi) || !same(m0.mu, m1.mu)))
          throw UnsupportedError("fractured magnetic-loss faces (chi, or mu where chi is set, changing across a face) "
                                 "are outside the supported path: the reference reads their old values from the "
                                 "electric state");
      }
      double dt = dt_est_;
      if (sim_.step != 0 && !(sim_.step > dt)) dt = sim_.step;
      nr_.assign(NF, 1.0);
      parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
        double M[16], Z[16];
        std::vector<double> Nl(16);
        for (uint32_t v = (uint32_t)v0; v < (uint32_t)v1; v++) {
          const Mat3& chi = sc_.materials.at(vol_mat_[v]).chi;
          if (mat_det(chi) == 0) continue;
          mag_mass(v, sc_.materials.at(vol_mat_[v]).mu, M);
          mag_mass(v, chi, Z);
          for (int q = 0; q < 16; q++) Nl[q] = M[q] + 0.5 * dt * Z[q];
          spd_inv(Nl, 4);
          std::copy(Nl.begin(), Nl.end(), blk.begin() + 16 * (size_t)v);
          for (int j = 0; j < 4; j++) {
            const int32_t f = vtf_[v][j];
            if ((int32_t)v != std::max(ftv_[f][0], ftv_[f][1])) continue;  // the face's last tet writes R
            double acc = 0;
            for (int m = 0; m < 4; m++) acc += Nl[4 * j + m] * (M[4 * m + j] - 0.5 * dt * Z[4 * m + j]);
            nr_[f] = acc;
          }
        }
      });
      build_N();
    }
    if (dga_frac_) {
      // conducting tets (Discretization.hpp:9262-9475) with the run's dt: a
      // star with a conducting tet gets H = (E + dt/2 S)^-1 and PQ =
      // H (E - dt/2 S), else H = E^-1 and PQ = I, Dirichlet rows and
      // columns masked.  Class-1 and class-2 rows (never in one star) are
      // filled from the upper triangle and its mirror; the mirror's row is
      // the column edge's own when it has the row's class, else that of the
      // class's first edge (the reference indexes the mirror through
      // zero-filled h_index / p_index vectors, :6546-6547).  P of a class-2
      // edge is the diagonal of PQ in the star of its higher node (the star
      // the reference writes last).  A fractured star's rows go to Q and Mq.
      double dt = dt_est_;
      if (sim_.step != 0 && !(sim_.step > dt)) dt = sim_.step;
      int32_t first_of[5] = {-1, -1, -1, -1, -1};
      for (uint32_t e = 0; e < NE; e++)
        if (first_of[cls_[e]] < 0) first_of[cls_[e]] = (int32_t)e;
      hp_.assign(NE, 1.0);
      std::vector<HostCsr::Trips> q_n(NP), mq_n(NP);
      parallel_for((int64_t)NP, nth, [&](int64_t n0, int64_t n1) {
        std::vector<double> E, S;
        for (uint32_t nid = (uint32_t)n0; nid < (uint32_t)n1; nid++) {
          const int64_t b0 = star_ptr_[nid];
          const int n = (int)(star_ptr_[nid + 1] - b0);
          const int32_t* gi = star_edge_.data() + b0;
          star_mass(nid, false, E);
          const bool sig_node = star_mass(nid, true, S);
          for (int j = 0; j < n; j++)
            if (cls_[gi[j]] == 4) {
              for (int k = 0; k < n; k++) E[j * n + k] = E[k * n + j] = S[j * n + k] = S[k * n + j] = 0;
              E[j * n + j] = 1;
            }
          std::vector<double> Hl(E), PQ((size_t)n * n, 0.0);
          if (sig_node) {
            for (size_t q = 0; q < Hl.size(); q++) Hl[q] += 0.5 * dt * S[q];
            spd_inv(Hl, n);
            for (int j = 0; j < n; j++)
              for (int k = 0; k < n; k++) {
                double acc = 0;
                for (int m = 0; m < n; m++) acc += Hl[j * n + m] * (E[m * n + k] - 0.5 * dt * S[m * n + k]);
                PQ[j * n + k] = acc;
              }
          } else {
            spd_inv(Hl, n);
            for (int j = 0; j < n; j++) PQ[j * n + j] = 1;
          }
          HostCsr::Trips& h_t = h_n[nid];
          const int64_t off = frac_off_[nid];
          for (int j = 0; j < n; j++) {
            const int32_t ej = gi[j];
            const int c = cls_[ej];
            if (c == 4) continue;
            if (c == 1 || c == 2) {
              if (c == 2 && (int32_t)nid == std::max(edges_[ej][0], edges_[ej][1])) hp_[ej] = PQ[j * n + j];
              for (int k = j; k < n; k++) {
                const int32_t ek = gi[k];
                if (cls_[ek] == 4 || Hl[j * n + k] == 0) continue;
                h_t.push_back({(uint32_t)ej, (uint32_t)ek, Hl[j * n + k]});
                if (j != k) h_t.push_back({(uint32_t)(cls_[ek] == c ? ek : first_of[c]), (uint32_t)ej, Hl[j * n + k]});
              }
            }
            if (off >= 0)
              for (int k = 0; k < n; k++) {
                if (cls_[gi[k]] == 4) continue;
                const uint32_t r = (uint32_t)(off + j);
                if (PQ[j * n + k] != 0) q_n[nid].push_back({r, (uint32_t)(off + k), PQ[j * n + k]});
                if (Hl[j * n + k] != 0) mq_n[nid].push_back({r, (uint32_t)gi[k], Hl[j * n + k]});
              }
          }
        }
      });
      HostCsr::Trips q_t, mq_t;
      for (size_t nid = 0; nid < NP; nid++) {
        q_t.insert(q_t.end(), q_n[nid].begin(), q_n[nid].end());
        mq_t.insert(mq_t.end(), mq_n[nid].begin(), mq_n[nid].end());
      }
      Q_ = HostCsr::build(q_size_, q_size_, q_t, nth);
      Mq_ = HostCsr::build(q_size_, NE, mq_t, nth);
    }
    HostCsr::Trips h_t;
    for (size_t nid = 0; nid < NP; nid++) {
      h_t.insert(h_t.end(), h_n[nid].begin(), h_n[nid].end());
      HostCsr::Trips().swap(h_n[nid]);
    }
    H_ = HostCsr::build(NE, NE, h_t, nth);
  } else if (method_ == 3) {
    // fem: Whitney edge mass (Discretization.hpp:7902-8060).  Per tet, the
    // barycentric coordinates l_1..l_3 = J^-1 (p - x_0), l_0 = 1 - l_1 - l_2 - l_3
    // (J the edge matrix [x_1-x_0, x_2-x_0, x_3-x_0]), the edge functions
    // w_ab = l_a grad l_b - l_b grad l_a on the local edges ab, bc, ac, ad,
    // bd, cd, and the quadrature |V| (sum over the 4 nodes + 9 x sum over
    // the 4 face barycentres) / 40 of w_k . eps w_j.  Entries j <= k, then
    // their mirror, zero values skipped, listed in tet order.
    static const int kWe[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    std::vector<double> blk(36 * (size_t)L), sblk(lossy_ ? 36 * (size_t)L : 0, 0.0);
    parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
      for (uint32_t v = (uint32_t)v0; v < (uint32_t)v1; v++) {
        const V3& x0 = pts_[vols_[v][0]];
        V3 c1 = sub(pts_[vols_[v][1]], x0), c2 = sub(pts_[vols_[v][2]], x0), c3 = sub(pts_[vols_[v][3]], x0);
        // rows of J^-1 = (c2 x c3, c3 x c1, c1 x c2) / det J: grad l_1..l_3
        const double det = dot(c1, cross(c2, c3));
        V3 g[4];
        g[1] = scale(cross(c2, c3), 1.0 / det);
        g[2] = scale(cross(c3, c1), 1.0 / det);
        g[3] = scale(cross(c1, c2), 1.0 / det);
        for (int a = 0; a < 3; a++) g[0][a] = -(g[1][a] + g[2][a] + g[3][a]);
        const Mat3& eps = sc_.materials.at(vol_mat_[v]).eps;
        const Mat3& sig = sc_.materials.at(vol_mat_[v]).sigma;
        const bool cond = sig_tet[v] != 0;
        double acc[2][6][6] = {}, accs[2][6][6] = {};
        auto add_point = [&](const V3& p, int which) {
          const V3 d = sub(p, x0);
          double l[4];
          l[1] = dot(g[1], d);
          l[2] = dot(g[2], d);
          l[3] = dot(g[3], d);
          l[0] = 1.0 - l[1] - l[2] - l[3];
          V3 w[6], ew[6];
          for (int k = 0; k < 6; k++) {
            const int a = kWe[k][0], b = kWe[k][1];
            w[k] = sub(scale(g[b], l[a]), scale(g[a], l[b]));
            ew[k] = mv(eps, w[k]);
          }
          for (int j = 0; j < 6; j++)
            for (int k = j; k < 6; k++) acc[which][j][k] += dot(w[k], ew[j]);
          if (cond) {  // SigMat by the same quadrature (:8020-8021)
            for (int k = 0; k < 6; k++) ew[k] = mv(sig, w[k]);
            for (int j = 0; j < 6; j++)
              for (int k = j; k < 6; k++) accs[which][j][k] += dot(w[k], ew[j]);
          }
        };
        for (int h = 0; h < 4; h++) {
          add_point(pts_[vols_[v][h]], 0);
          add_point(fbar(vtf_[v][h]), 1);
        }
        const double V = std::fabs(cell_vol_[v]);
        for (int j = 0; j < 6; j++)
          for (int k = 0; k < 6; k++)
            blk[36 * (size_t)v + 6 * j + k] =
                k >= j ? V * (acc[0][j][k] + acc[1][j][k] * 9.0) / 40.0 : 0.0;
        if (cond)
          for (int j = 0; j < 6; j++)
            for (int k = 0; k < 6; k++)
              sblk[36 * (size_t)v + 6 * j + k] = k >= j ? V * (accs[0][j][k] + accs[1][j][k] * 9.0) / 40.0 : 0.0;
      }
    });
    std::vector<int64_t> off(L + 1, 0);
    parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
      for (int64_t v = v0; v < v1; v++)
        for (int j = 0; j < 6; j++)
          for (int k = j; k < 6; k++)
            if (blk[36 * v + 6 * j + k] != 0) off[v + 1] += k == j ? 1 : 2;
    });
    for (uint32_t v = 0; v < L; v++) off[v + 1] += off[v];
    HostCsr::Trips t(off[L]);
    parallel_for(L, nth, [&](int64_t v0, int64_t v1) {
      for (int64_t v = v0; v < v1; v++) {
        auto el = vol_edges((uint32_t)v);
        int64_t w = off[v];
        for (int j = 0; j < 6; j++)
          for (int k = j; k < 6; k++) {
            const double x = blk[36 * v + 6 * j + k];
            if (x == 0) continue;
            t[w++] = {(uint32_t)el[j], (uint32_t)el[k], x};
            if (k != j) t[w++] = {(uint32_t)el[k], (uint32_t)el[j], x};
          }
      }
    });
    E_ = HostCsr::build(NE, NE, t, nth);
    if (lossy_) {  // SigMat entries, zero values skipped, tet order (:8041-8051)
      HostCsr::Trips ts;
      for (uint32_t v = 0; v < L; v++) {
        if (!sig_tet[v]) continue;
        auto el = vol_edges(v);
        for (int j = 0; j < 6; j++)
          for (int k = j; k < 6; k++) {
            const double x = sblk[36 * (size_t)v + 6 * j + k];
            if (x == 0) continue;
            ts.push_back({(uint32_t)el[j], (uint32_t)el[k], x});
            if (k != j) ts.push_back({(uint32_t)el[k], (uint32_t)el[j], x});
          }
      }
      Sig_ = HostCsr::build(NE, NE, ts, nth);
    }
    dt_est_ = sim_.courant * estimate_dt(E_, true);
    dt_ = dt_est_;
    if (sim_.step != 0) {  // Discretization.hpp:8029-8036
      if (sim_.step > dt_) unstable_ = true;
      else dt_ = sim_.step;
    }
    // SysMat = E * (1 / (dt dt)) + (0.5 / dt) SigMat (:8086-8093)
    split_system(1.0 / (dt_ * dt_), 0.5 / dt_);
  } else {
    // gfdtd eps-mass from the node dual bases (Discretization.hpp:8357-8621):
    // nine entries per (node, tet) pair at fixed positions, formed in parallel
    HostCsr::Trips t(9 * nvol_.size()), ts(lossy_ ? 9 * nvol_.size() : 0);
    parallel_for((int64_t)pts_.size(), nth, [&](int64_t n0, int64_t n1) {
      for (uint32_t nid = (uint32_t)n0; nid < (uint32_t)n1; nid++)
        for (int64_t q = nvol_ptr_[nid]; q < nvol_ptr_[nid + 1]; q++) {
          const int32_t vv = nvol_[q];
          auto el = vol_edges(vv);
          const double om = std::fabs(cell_vol_[vv]) / 4.0;
          const Mat3& eps = sc_.materials.at(vol_mat_[vv]).eps;
          int k = 0;
          while (vols_[vv][k] != (int32_t)nid) k++;
          int32_t e[3] = {el[kEd[k][0]], el[kEd[k][1]], el[kEd[k][2]]};
          V3 a1 = sub(ebar(e[0]), pts_[nid]), a2 = sub(ebar(e[1]), pts_[nid]), a3 = sub(ebar(e[2]), pts_[nid]);
          const double nc = std::pow(dot(a1, cross(a2, a3)), -1);
          const V3 f[3] = {scale(cross(a2, a3), nc), scale(cross(a3, a1), nc), scale(cross(a1, a2), nc)};
          Mat3 oe;
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) oe.m[i][j] = om * eps.m[i][j];
          // reference form: half-edge duals, no 1/4, no orientation signs;
          // consistent form: both applied
          double sg[3] = {1, 1, 1}, quarter = 1;
          if (opt_.consistent_mass) {
            for (int a = 0; a < 3; a++) sg[a] = edges_[e[a]][1] == (int32_t)nid ? -1.0 : 1.0;
            quarter = 0.25;
          }
          static const int kPair[9][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 0}, {0, 2}, {2, 0}, {1, 2}, {2, 1}};
          for (int k2 = 0; k2 < 9; k2++) {
            const int* pq = kPair[k2];
            t[9 * q + k2] = {(uint32_t)e[pq[0]], (uint32_t)e[pq[1]],
                             quarter * sg[pq[0]] * sg[pq[1]] * dot(f[pq[0]], mv(oe, f[pq[1]]))};
          }
          if (lossy_) {  // SigMat: the same basis with sigma on conducting tets (:8604-8616)
            const Mat3& sig = sc_.materials.at(vol_mat_[vv]).sigma;
            Mat3 os;
            for (int i = 0; i < 3; i++)
              for (int j = 0; j < 3; j++) os.m[i][j] = om * sig.m[i][j];
            for (int k2 = 0; k2 < 9; k2++) {
              const int* pq = kPair[k2];
              ts[9 * q + k2] = {(uint32_t)e[pq[0]], (uint32_t)e[pq[1]],
                                sig_tet[vv] ? quarter * sg[pq[0]] * sg[pq[1]] * dot(f[pq[0]], mv(os, f[pq[1]]))
                                            : 0.0};
            }
          }
        }
    });
    E_ = HostCsr::build(NE, NE, t, nth);
    if (lossy_) Sig_ = HostCsr::build(NE, NE, ts, nth);
    auto te = std::chrono::steady_clock::now();
    dt_est_ = sim_.courant * estimate_dt(E_, true);
    if (opt_.verbose)
      std::printf("  set-up %-14s %8.3f s\n", "(dt estimate)",
                  std::chrono::duration<double>(std::chrono::steady_clock::now() - te).count());
    dt_ = dt_est_;
    if (sim_.step != 0) {  // Discretization.hpp:8634-8641
      if (sim_.step > dt_) unstable_ = true;
      else dt_ = sim_.step;
    }
    // SysMat = E + (0.5 dt) SigMat (:8644)
    split_system(1.0, 0.5 * dt_);
  }
  if (method_ != 3) dt_ = dt_est_;
  if (method_ != 3 && sim_.step != 0) {  // Discretization.hpp:9146-9153, 8634-8641
    if (sim_.step > dt_) unstable_ = true;
    else dt_ = sim_.step;
  }
}

// A (free x free) and R (free x Dirichlet) split the rows of SysMat =
// scale * E + sig_coef * SigMat: the system of gfdtd (scale 1, sig_coef dt/2)
// and of fem (scale 1 / dt^2, sig_coef 0.5 / dt); SigMat only with conducting
// tets.  The free numbering fidx is increasing in the edge index, so each
// split row keeps the sorted, merged column order: the rows are merged, not
// re-sorted.
void TetSim::split_system(double scale, double sig_coef) {
  const uint32_t NE = (uint32_t)edges_.size();
  const int nth = opt_.setup_threads;
  {
    std::vector<int32_t> fidx(NE, -1);
    for (uint32_t e = 0; e < NE; e++) {
      if (cls_[e] != 4) {
        fidx[e] = (int32_t)free_edges_.size();
        free_edges_.push_back((int32_t)e);
      } else {
        dir_edges_.push_back((int32_t)e);
      }
    }
    const uint32_t nf = (uint32_t)free_edges_.size();
    A_.nrows = A_.ncols = nf;
    R_.nrows = nf;
    R_.ncols = NE;
    A_.ptr.assign(nf + 1, 0);
    R_.ptr.assign(nf + 1, 0);
    // row r of SysMat: E's and SigMat's entries merged by column,
    // E_rc scale + coef S_rc where both hold one (the sum the reference forms)
    const bool sg = lossy_;
    auto row = [&](int32_t r, auto&& f) {
      int64_t k = E_.ptr[r], ks = sg ? Sig_.ptr[r] : 0;
      const int64_t ke = E_.ptr[r + 1], kse = sg ? Sig_.ptr[r + 1] : 0;
      while (k < ke || ks < kse) {
        if (ks >= kse || (k < ke && E_.col[k] < Sig_.col[ks])) {
          f(E_.col[k], scale == 1.0 ? E_.val[k] : E_.val[k] * scale);
          k++;
        } else if (k >= ke || Sig_.col[ks] < E_.col[k]) {
          f(Sig_.col[ks], sig_coef * Sig_.val[ks]);
          ks++;
        } else {
          f(E_.col[k], (scale == 1.0 ? E_.val[k] : E_.val[k] * scale) + sig_coef * Sig_.val[ks]);
          k++;
          ks++;
        }
      }
    };
    parallel_for(nf, nth, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; i++)
        row(free_edges_[i], [&](int32_t c, double) { (fidx[c] < 0 ? R_.ptr[i + 1] : A_.ptr[i + 1])++; });
    });
    for (uint32_t i = 0; i < nf; i++) {
      A_.ptr[i + 1] += A_.ptr[i];
      R_.ptr[i + 1] += R_.ptr[i];
    }
    A_.col.resize(A_.ptr[nf]);
    A_.val.resize(A_.ptr[nf]);
    R_.col.resize(R_.ptr[nf]);
    R_.val.resize(R_.ptr[nf]);
    parallel_for(nf, nth, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; i++) {
        int64_t wa = A_.ptr[i], wr = R_.ptr[i];
        row(free_edges_[i], [&](int32_t c, double v) {
          if (fidx[c] < 0) {
            R_.col[wr] = c;
            R_.val[wr++] = v;
          } else {
            A_.col[wa] = fidx[c];
            A_.val[wa++] = v;
          }
        });
      }
    });
    jacobi_.resize(nf);
    for (uint32_t i = 0; i < nf; i++) {
      double dg = 0;
      for (int64_t k = A_.ptr[i]; k < A_.ptr[i + 1]; k++)
        if (A_.col[k] == (int32_t)i) dg = A_.val[k];
      jacobi_[i] = dg != 0 ? 1.0 / dg : 1.0;  // ConjugateGradientSolver.hpp:119-127
    }
  }
}

// Largest eigenvalue of Minv K (dga, Minv = node-star inverses) or of the
// pencil K x = lambda E x (gfdtd), K = C^T N C, by Lanczos in the K inner
// product; dt = 2 / sqrt(lambda).  Meshes above 3 M edges with a pinned step,
// and batch members with a pinned step, skip the estimate and take the step
// as given.
// A pinned step skips the estimate on large meshes (and in batches); dt is
// then the pinned step.
bool TetSim::dt_estimate_needed() const {
  return !(sim_.step != 0 && (edges_.size() > 3000000 || !opt_.estimate_pinned));
}

double TetSim::estimate_dt(const HostCsr& M, bool generalized) {
  const size_t n = edges_.size(), nf = faces_.size();
  if (!dt_estimate_needed()) return sim_.step / sim_.courant;
  // Lanczos on the GPU (dt_gpu.cu) from a fixed pseudo-random start vector
  std::vector<double> x(n);
  uint64_t s = 0x2545F4914F6CDD1Dull;
  for (size_t i = 0; i < n; i++) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    x[i] = (double)(s >> 11) / 9007199254740992.0 - 0.5;
  }
  std::vector<int32_t> fte(3 * nf), ct(Ct_.col.size());
  for (size_t f = 0; f < nf; f++)
    for (int a = 0; a < 3; a++) fte[3 * f + a] = fte_[f][a];
  for (size_t k = 0; k < ct.size(); k++)
    ct[k] = Ct_.val[k] < 0 ? (int32_t)((uint32_t)Ct_.col[k] | 0x80000000u) : Ct_.col[k];
  DtProblem p;
  p.device = opt_.device;
  p.n = (int64_t)n;
  p.nf = (int64_t)nf;
  p.fte = fte.data();
  p.N = {(int64_t)N_.nrows, N_.ptr.data(), N_.col.data(), N_.val.data()};
  p.Ct = {(int64_t)Ct_.nrows, Ct_.ptr.data(), ct.data(), nullptr};
  p.M = {(int64_t)M.nrows, M.ptr.data(), M.col.data(), M.val.data()};
  p.generalized = generalized;
  p.x0 = x.data();
  p.tridiag_max = tridiag_max;
  const double lam = gpu_lanczos_lambda(p);
  return 2.0 / std::sqrt(lam);
}

void TetSim::locate_probes() {
  // FindProbe (Discretization.hpp:3645-3747)
  auto det4 = [](const double m[4][4]) {
    double a = m[2][2] * m[3][3] - m[2][3] * m[3][2], b = m[2][1] * m[3][3] - m[2][3] * m[3][1];
    double c = m[2][1] * m[3][2] - m[2][2] * m[3][1], d = m[2][0] * m[3][3] - m[2][3] * m[3][0];
    double e = m[2][0] * m[3][2] - m[2][2] * m[3][0], f = m[2][0] * m[3][1] - m[2][1] * m[3][0];
    return m[0][0] * (m[1][1] * a - m[1][2] * b + m[1][3] * c) - m[0][1] * (m[1][0] * a - m[1][2] * d + m[1][3] * e) +
           m[0][2] * (m[1][0] * b - m[1][1] * d + m[1][3] * f) - m[0][3] * (m[1][0] * c - m[1][1] * e + m[1][2] * f);
  };
  const uint32_t L = (uint32_t)vols_.size();
  std::vector<uint8_t> colour(L, 0);
  std::vector<uint32_t> touched;
  uint32_t root = 0;
  const double tol = 1e-12;
  // Exact pre-test.  The walk below accepts tet v when every barycentric
  // coordinate d1_r / d0 of the point is >= -tol / |d0|.  A point beyond the
  // tet's bounding box by delta along an axis of extent `ext` has negative
  // coordinates summing to at most -delta / ext, so one of them (at most three
  // are negative) is <= -delta / (3 ext): it cannot pass once delta exceeds
  // 3 ext tol / |d0|.  Each tet's box is widened by 4 ext (2 tol) / |d0|
  // (twice the tolerance covers the rounding of the determinants) and stored
  // rounded outwards; a point outside it skips the determinants, with the same
  // outcome, and a point outside every box skips the walk.  Near-degenerate
  // tets (|d0| <= tol) get an unbounded box.
  std::vector<float> box(6 * (size_t)L);
  parallel_for(L, opt_.setup_threads, [&](int64_t v0, int64_t v1) {
    for (int64_t v = v0; v < v1; v++) {
      double rows[4][4], lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int r = 0; r < 4; r++) {
        for (int a = 0; a < 3; a++) {
          rows[r][a] = pts_[vols_[v][r]][a];
          lo[a] = std::min(lo[a], rows[r][a]);
          hi[a] = std::max(hi[a], rows[r][a]);
        }
        rows[r][3] = 1;
      }
      const double d0 = std::fabs(det4(rows));
      const double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
      const bool open = !(d0 > tol) || !std::isfinite(d0);
      const double m = open ? 0.0 : 4.0 * ext * (2.0 * tol) / d0;
      for (int a = 0; a < 3; a++) {
        float l = open ? -INFINITY : (float)(lo[a] - m), h = open ? INFINITY : (float)(hi[a] + m);
        if (!open && (double)l > lo[a] - m) l = std::nextafter(l, -INFINITY);
        if (!open && (double)h < hi[a] + m) h = std::nextafter(h, INFINITY);
        box[6 * v + a] = l;
        box[6 * v + 3 + a] = h;
      }
    }
  });
  float glo[3] = {INFINITY, INFINITY, INFINITY}, ghi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t v = 0; v < L; v++)
    for (int a = 0; a < 3; a++) {
      glo[a] = std::min(glo[a], box[6 * v + a]);
      ghi[a] = std::max(ghi[a], box[6 * v + 3 + a]);
    }
  auto in_box = [](const float* bx, const std::array<double, 3>& pv) {
    for (int a = 0; a < 3; a++)
      if (pv[a] < (double)bx[a] || pv[a] > (double)bx[3 + a]) return false;
    return true;
  };
  const float gbox[6] = {glo[0], glo[1], glo[2], ghi[0], ghi[1], ghi[2]};
  // the walk's containment test, behind the exact box pre-test
  auto passes = [&](uint32_t v, const std::array<double, 3>& pv) {
    if (!in_box(&box[6 * (size_t)v], pv)) return false;
    double rows[4][4];
    for (int r = 0; r < 4; r++) {
      for (int a = 0; a < 3; a++) rows[r][a] = pts_[vols_[v][r]][a];
      rows[r][3] = 1;
    }
    const double d0 = det4(rows);
    bool ok = true;
    for (int r = 0; r < 4 && ok; r++) {
      double m[4][4];
      std::memcpy(m, rows, sizeof(m));
      for (int a = 0; a < 3; a++) m[r][a] = pv[a];
      const double d1 = det4(m);
      ok = (d0 >= -tol && d1 >= -tol) || (d0 <= tol && d1 <= tol);
    }
    return ok;
  };
  auto neighbour = [&](uint32_t v, int32_t f) {
    int32_t n = ftv_[f][0];
    if (n == (int32_t)v) n = ftv_[f][1] >= 0 ? ftv_[f][1] : n;
    return n;
  };
  // FindProbe's walk: breadth first from the last hit, tet 0 marked visited
  // from the start, the first tet that passes wins
  auto walk = [&](const std::array<double, 3>& pv) -> int64_t {
    for (uint32_t t : touched) colour[t] = 0;
    touched.clear();
    std::vector<uint32_t> q{root};
    colour[0] = 1;
    touched.push_back(0);
    for (size_t h = 0; h < q.size(); h++) {
      const uint32_t v = q[h];
      if (passes(v, pv)) {
        root = v;
        return v;
      }
      for (int32_t f : vtf_[v]) {
        const int32_t n = neighbour(v, f);
        if (!colour[n]) {
          colour[n] = 1;
          touched.push_back(n);
          q.push_back(n);
        }
      }
      if (!colour[v]) { colour[v] = 1; touched.push_back(v); }
    }
    return -1;
  };
  // The walk's answer without the walk.  Its first passing tet is its only
  // passing tet when exactly one tet it can reach passes, and it finds none
  // when none does; only real ties (two or more) need the walk's order.
  // Candidates come from a uniform grid over the widened tet boxes (every tet
  // whose box holds the point is listed in the point's cell; unbounded boxes
  // are kept aside and tried for every point).  What the walk reaches: the
  // components of the face graph without tet 0 (it starts with tet 0
  // marked), the root's own component, or from root 0 tet 0 and the
  // components next to it.
  std::vector<int32_t> comp(L, -1);
  {
    int32_t nc = 0;
    std::vector<uint32_t> stack;
    for (uint32_t s0 = 1; s0 < L; s0++) {
      if (comp[s0] >= 0) continue;
      comp[s0] = nc;
      stack.assign(1, s0);
      while (!stack.empty()) {
        const uint32_t v = stack.back();
        stack.pop_back();
        for (int32_t f : vtf_[v]) {
          const int32_t n = neighbour(v, f);
          if (n != 0 && comp[n] < 0) {
            comp[n] = nc;
            stack.push_back((uint32_t)n);
          }
        }
      }
      nc++;
    }
  }
  std::vector<int32_t> next_to_0;
  if (L > 0)
    for (int32_t f : vtf_[0]) {
      const int32_t n = neighbour(0, f);
      if (n != 0) next_to_0.push_back(comp[n]);
    }
  auto reached = [&](uint32_t t) {
    if (root != 0) return t != 0 && comp[t] == comp[root];
    return t == 0 || std::find(next_to_0.begin(), next_to_0.end(), comp[t]) != next_to_0.end();
  };
  std::vector<uint32_t> unbounded;
  double flo[3] = {1e300, 1e300, 1e300}, fhi[3] = {-1e300, -1e300, -1e300};
  for (size_t v = 0; v < L; v++) {
    if (!std::isfinite(box[6 * v]) || !std::isfinite(box[6 * v + 3]) || !std::isfinite(box[6 * v + 1]) ||
        !std::isfinite(box[6 * v + 4]) || !std::isfinite(box[6 * v + 2]) || !std::isfinite(box[6 * v + 5])) {
      unbounded.push_back((uint32_t)v);
      continue;
    }
    for (int a = 0; a < 3; a++) {
      flo[a] = std::min(flo[a], (double)box[6 * v + a]);
      fhi[a] = std::max(fhi[a], (double)box[6 * v + 3 + a]);
    }
  }
  const int64_t G = std::max<int64_t>(1, std::min<int64_t>(256, (int64_t)std::cbrt((double)L / 8.0)));
  double cw[3];
  for (int a = 0; a < 3; a++) cw[a] = fhi[a] > flo[a] ? (fhi[a] - flo[a]) / (double)G : 1.0;
  auto cell_of = [&](int a, double x) {
    const double c = std::floor((x - flo[a]) / cw[a]);
    return c < 0 ? (int64_t)0 : (c > (double)(G - 1) ? G - 1 : (int64_t)c);
  };
  std::vector<int64_t> cstart(G * G * G + 1, 0);
  std::vector<uint32_t> cidx;
  {
    auto each_cell = [&](size_t v, auto&& f) {
      int64_t c0[3], c1[3];
      for (int a = 0; a < 3; a++) {
        c0[a] = cell_of(a, (double)box[6 * v + a]);
        c1[a] = cell_of(a, (double)box[6 * v + 3 + a]);
      }
      for (int64_t k = c0[2]; k <= c1[2]; k++)
        for (int64_t j = c0[1]; j <= c1[1]; j++)
          for (int64_t i = c0[0]; i <= c1[0]; i++) f((k * G + j) * G + i);
    };
    std::vector<uint8_t> is_unb(L, 0);
    for (uint32_t v : unbounded) is_unb[v] = 1;
    for (size_t v = 0; v < L; v++)
      if (!is_unb[v]) each_cell(v, [&](int64_t c) { cstart[c + 1]++; });
    for (int64_t c = 0; c < G * G * G; c++) cstart[c + 1] += cstart[c];
    cidx.resize(cstart[G * G * G]);
    std::vector<int64_t> pos(cstart.begin(), cstart.end() - 1);
    for (size_t v = 0; v < L; v++)
      if (!is_unb[v]) each_cell(v, [&](int64_t c) { cidx[pos[c]++] = (uint32_t)v; });
  }
  auto find = [&](const std::array<double, 3>& pv) -> int64_t {
    if (L == 0 || !in_box(gbox, pv)) return -1;
    std::vector<uint32_t> hits;
    bool inside = true;
    for (int a = 0; a < 3; a++) inside = inside && pv[a] >= flo[a] && pv[a] <= fhi[a];
    if (inside) {
      const int64_t c = (cell_of(2, pv[2]) * G + cell_of(1, pv[1])) * G + cell_of(0, pv[0]);
      for (int64_t k = cstart[c]; k < cstart[c + 1]; k++)
        if (passes(cidx[k], pv) && reached(cidx[k])) hits.push_back(cidx[k]);
    }
    for (uint32_t v : unbounded)
      if (passes(v, pv) && reached(v)) hits.push_back(v);
    if (hits.empty()) return -1;
    if (hits.size() == 1) {
      root = hits[0];
      return hits[0];
    }
    return walk(pv);
  };
  // silo mode: the reference writes E (Whitney, at the barycentre) and H of
  // every tet at each print time (ExportFields, Discretization.hpp:2601-2677);
  // here every tet is a sample point at its barycentre, (p0+p1+p2+p3)/4
  // (vol_barycenter, :10479-10484), through the same weights as a probe
  const bool silo = out_.mode == "silo";
  std::vector<std::pair<int64_t, V3>> where;
  if (out_.mode == "probepoint")
    for (auto& pv : out_.probes) where.push_back({find(pv), pv});
  if (silo) {
    where.reserve(L);
    for (uint32_t v = 0; v < L; v++) {
      const auto& n = vols_[v];
      V3 b;
      for (int a = 0; a < 3; a++) b[a] = (pts_[n[0]][a] + pts_[n[1]][a] + pts_[n[2]][a] + pts_[n[3]][a]) / 4.0;
      where.push_back({(int64_t)v, b});
    }
  }
  for (auto& [v, pv] : where) {
    {
      if (v < 0) continue;
      probe_tet_.push_back((int32_t)v);
      probe_pts_.push_back(pv);
      // Whitney weights: lambda = [x 1] G with G the inverse of the node matrix
      double W[4][8];
      for (int i = 0; i < 4; i++) {
        for (int a = 0; a < 3; a++) W[i][a] = pts_[vols_[v][i]][a];
        W[i][3] = 1;
        for (int j = 0; j < 4; j++) W[i][4 + j] = i == j ? 1.0 : 0.0;
      }
      for (int c = 0; c < 4; c++) {
        int piv = c;
        for (int r = c + 1; r < 4; r++)
          if (std::fabs(W[r][c]) > std::fabs(W[piv][c])) piv = r;
        for (int j = 0; j < 8; j++) std::swap(W[c][j], W[piv][j]);
        const double dd = W[c][c];
        for (int j = 0; j < 8; j++) W[c][j] /= dd;
        for (int r = 0; r < 4; r++)
          if (r != c) {
            const double fct = W[r][c];
            for (int j = 0; j < 8; j++) W[r][j] -= fct * W[c][j];
          }
      }
      double lam[4], grad[4][3];
      for (int i = 0; i < 4; i++) {
        lam[i] = pv[0] * W[0][4 + i] + pv[1] * W[1][4 + i] + pv[2] * W[2][4 + i] + W[3][4 + i];
        for (int a = 0; a < 3; a++) grad[i][a] = W[a][4 + i];
      }
      static const int kE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
      for (int q = 0; q < 6; q++)
        for (int a = 0; a < 3; a++)
          probe_we_.push_back(lam[kE[q][0]] * grad[kE[q][1]][a] - lam[kE[q][1]] * grad[kE[q][0]][a]);
      // H = 1/4 mu^-1 (sum of face-flux weighted primal edge combinations)/(3 V)
      // (GetMagneticField, Discretization.hpp:3877-3897)
      const auto& n = vols_[v];
      V3 pev[6] = {sub(pts_[n[1]], pts_[n[0]]), sub(pts_[n[2]], pts_[n[1]]), sub(pts_[n[2]], pts_[n[0]]),
                   sub(pts_[n[3]], pts_[n[0]]), sub(pts_[n[3]], pts_[n[1]]), sub(pts_[n[3]], pts_[n[2]])};
      const double vv = 3 * cell_vol_[v];
      const Mat3& mu = sc_.materials.at(vol_mat_[v]).mu;
      V3 hq[4];
      for (int a = 0; a < 3; a++) {
        hq[0][a] = pev[0][a] + pev[2][a] + pev[3][a];
        hq[1][a] = pev[0][a] - pev[1][a] - pev[4][a];
        hq[2][a] = -pev[2][a] - pev[1][a] + pev[5][a];
        hq[3][a] = pev[3][a] + pev[4][a] + pev[5][a];
      }
      for (int q = 0; q < 4; q++)
        for (int a = 0; a < 3; a++) probe_hf_.push_back(0.25 * (1.0 / mu.m[a][a]) * hq[q][a] / vv);
    }
  }
  // current dipoles: nearest edge of the star of the tet's first node
  // (Discretization.hpp:431-464); the reference locates them only in the
  // probepoint and maxerror output modes (:378), and so does this
  if (out_.mode == "probepoint" || out_.mode == "maxerror") {
    for (uint32_t sl : src_labels_) {
      Source& s = sc_.sources[sl];
      if (s.st != "j") continue;
      int64_t v = find(s.location);
      if (v < 0) continue;
      const int32_t node = vols_[v][0];
      int32_t best = -1;
      double bd = 0;
      for (int64_t q = star_ptr_[node]; q < star_ptr_[node + 1]; q++) {
        const int32_t e = star_edge_[q];
        const auto &a = pts_[edges_[e][0]], &b = pts_[edges_[e][1]];
        V3 d{0.5 * (a[0] + b[0]) - s.location[0], 0.5 * (a[1] + b[1]) - s.location[1],
             0.5 * (a[2] + b[2]) - s.location[2]};
        const double dd = std::sqrt(dot(d, d));
        if (best < 0 || dd < bd) { bd = dd; best = e; }
      }
      edge_src_[best].push_back(sl);
    }
  }
}

bool TetSim::mesh_arrays(std::vector<double>* xyz, std::vector<int32_t>* tets) const {
  if (xyz) {
    xyz->resize(3 * pts_.size());
    for (size_t n = 0; n < pts_.size(); n++)
      for (int a = 0; a < 3; a++) (*xyz)[3 * n + a] = pts_[n][a];
  }
  if (tets) {
    // positive volume: nodes 0 1 2 3, else 0 2 1 3 (ExportMesh, :2358-2373)
    tets->resize(4 * vols_.size());
    for (size_t v = 0; v < vols_.size(); v++) {
      const auto& n = vols_[v];
      const bool pos = cell_vol_[v] > 0;
      int32_t* o = &(*tets)[4 * v];
      o[0] = n[0];
      o[1] = pos ? n[1] : n[2];
      o[2] = pos ? n[2] : n[1];
      o[3] = n[3];
    }
  }
  return true;
}

// ------------------------------------------------------------------ device
template <typename T>
static std::vector<T> as(const std::vector<double>& v) {
  return std::vector<T>(v.begin(), v.end());
}

// Source-driven edges, their (source, profile factor) pairs, the carrier
// table per step and the t = 0 state (Discretization.hpp:3899-4202,
// Source.hpp:313-567).
void TetSim::build_sources() {
  const size_t NE = edges_.size();
  // source edges and pairs
  const size_t nsrc = src_labels_.size();
  auto src_index = [&](uint32_t l) {
    for (size_t q = 0; q < nsrc; q++)
      if (src_labels_[q] == l) return (int)q;
    return -1;
  };
  init_U_.assign(NE, 0.0);
  init_I_.assign(NE, 0.0);
  init_src_.assign(NE, 0.0);
  for (size_t e = 0; e < NE; e++) {
    if (edge_src_[e].empty() || pec_[e]) continue;
    const std::string ty = sc_.sources[edge_src_[e][0]].st;
    int kind = ty == "e" ? 1 : (ty == "h" ? 2 : (ty == "j" ? 3 : 0));
    if (kind == 0 || (kind == 2 && bnd_edge_[e] < 0)) continue;
    const auto &a = pts_[edges_[e][0]], &b = pts_[edges_[e][1]];
    const V3 eb{0.5 * (a[0] + b[0]), 0.5 * (a[1] + b[1]), 0.5 * (a[2] + b[2])};
    const V3 ev = sub(b, a);
    V3 vec = kind == 2 ? bnd_dual_[bnd_edge_[e]] : ev;
    double post = kind == 3 ? 1.0 / std::sqrt(dot(ev, ev)) : 1.0;
    src_begin_.push_back((int)pair_src_.size());
    src_edge_.push_back((int32_t)e);
    src_kind_e_.push_back((int8_t)kind);
    for (int q = 0; q < 3; q++) src_vec_.push_back(vec[q]);
    src_post_.push_back(post);
    double v0[3] = {0, 0, 0};
    for (uint32_t sl : edge_src_[e]) {
      const Source& s = sc_.sources[sl];
      if (s.st != ty) continue;  // each evaluator sums only its own type
      const int si = src_index(sl);
      double f[4] = {1, 1, 1, 1};
      if (s.decay != 0)
        f[0] = std::pow(std::pow(eb[0] - s.center[0], 2) + std::pow(eb[1] - s.center[1], 2) +
                            std::pow(eb[2] - s.center[2], 2), -0.5 * s.decay);
      if (s.prof == "gaussian")
        f[1] = std::exp(-((std::pow(eb[0] - s.center[0], 2) + std::pow(eb[1] - s.center[1], 2) +
                           std::pow(eb[2] - s.center[2], 2)) / std::pow(s.radius, 2)));
      else if (s.prof == "wave")
        for (int x = 0; x < 3; x++) {
          if (s.bfuncs[x] == "sin") f[1 + x] = std::sin((double)(2 * PI_L * s.kvec[x] * (eb[x] - s.center[x])));
          else if (s.bfuncs[x] == "cos") f[1 + x] = std::cos((double)(2 * PI_L * s.kvec[x] * (eb[x] - s.center[x])));
        }
      pair_src_.push_back(si);
      for (int q = 0; q < 4; q++) pair_fac_.push_back(f[q]);
      const int dir = s.dir == "x" ? 0 : (s.dir == "y" ? 1 : 2);
      pair_dir_.push_back((int8_t)dir);
      // value at t = 0 for the initial state
      auto r0 = s.compute(eb[0], eb[1], eb[2], 0.0);
      for (int x = 0; x < 3; x++) v0[x] += r0[x];
    }
    const double val0 = post * ((v0[0] * vec[0] + v0[1] * vec[1]) + v0[2] * vec[2]);
    if (kind == 1) { init_U_[e] = val0; init_src_[e] = val0; }
    else if (kind == 3 && method_ >= 2) init_I_[e] = val0;
  }
  src_begin_.push_back((int)pair_src_.size());
  src_amp_.resize(nsrc);
  carrier_.assign(nsteps_ * nsrc + 1, 0.0);
  for (size_t q = 0; q < nsrc; q++) {
    const Source& s = sc_.sources[src_labels_[q]];
    src_amp_[q] = s.st == "j" ? s.amp * s.impedance : s.amp;
    for (uint64_t i = 0; i < nsteps_; i++) {
      double t = (double)(i + 1) * dt_;
      if (s.st == "h") t = t - 0.5 * dt_;
      double c = 0.0;
      if (t >= 0) {
        if (s.carrier == "sin") c = std::sin((double)(2 * PI_L * s.freq * (t - s.delay)));
        else if (s.carrier == "cos") c = s.amp * std::cos((double)(2 * PI_L * s.freq * (t - s.delay)));
        else if (s.carrier == "gaussian") c = std::exp(-std::pow(t - s.delay, 2) / std::pow(s.width, 2));
        else if (s.carrier == "ricker") {
          double a = (double)(PI_L * s.freq * (t - s.delay));
          c = (1 - 2 * std::pow(a, 2)) * std::exp(-std::pow(a, 2));
        } else c = 1.0;
      }
      carrier_[i * nsrc + q] = c;
    }
  }
}

void TetSim::alloc_and_upload() {
  CU(cudaSetDevice(opt_.device));
  int major = 0;
  CU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, opt_.device));
  if (major != 10) throw CudaError("device " + std::to_string(opt_.device) + " is not an sm_100 (B200) GPU");
  CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  CU(cudaEventCreate(&ev0_));
  CU(cudaEventCreate(&ev1_));
  const bool f32 = opt_.precision == 1;
  const size_t es = f32 ? 4 : 8;
  auto dalloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    CU(cudaMalloc(&p, bytes ? bytes : 16));
    allocs_.push_back(p);
    dev_bytes_ += bytes;
    return p;
  };
  auto up = [&](const void* h, size_t bytes) -> void* {
    void* p = dalloc(bytes);
    if (bytes) CU(cudaMemcpyAsync(p, h, bytes, cudaMemcpyHostToDevice, stream_));
    return p;
  };
  auto upT = [&](const std::vector<double>& v) -> void* {
    if (!f32) return up(v.data(), v.size() * 8);
    auto f = as<float>(v);
    void* p = up(f.data(), f.size() * 4);
    CU(cudaStreamSynchronize(stream_));
    return p;
  };
  auto zeros = [&](size_t n) -> void* {
    void* p = dalloc(n * es);
    CU(cudaMemsetAsync(p, 0, n * es, stream_));
    return p;
  };
  DevPtrs& d = dp_;
  const size_t NE = edges_.size(), NF = faces_.size();
  d.nE = (int)NE;
  d.nF = (int)NF;
  d.dt = dt_;
  d.U = zeros(NE); d.F = zeros(NF); d.B = zeros(NF); d.cu = zeros(NF); d.cf = zeros(NE);
  d.I = zeros(NE); d.cb = zeros(NE);
  d.fte = (const int32_t*)up(fte_.data(), NF * 3 * 4);
  {
    std::vector<int32_t> cc(Ct_.col.size());
    for (size_t k = 0; k < cc.size(); k++) cc[k] = Ct_.val[k] < 0 ? (int32_t)((uint32_t)Ct_.col[k] | 0x80000000u) : Ct_.col[k];
    d.ct_ptr = (const int64_t*)up(Ct_.ptr.data(), Ct_.ptr.size() * 8);
    d.ct_col = (const int32_t*)up(cc.data(), cc.size() * 4);
  }
  auto upcsr = [&](const HostCsr& m, const int64_t*& ptr, const int32_t*& col, const void*& val) {
    ptr = (const int64_t*)up(m.ptr.data(), m.ptr.size() * 8);
    col = (const int32_t*)up(m.col.data(), m.col.size() * 4);
    val = upT(m.val);
  };
  upcsr(N_, d.n_ptr, d.n_col, d.n_val);
  upcsr(H_, d.h_ptr, d.h_col, d.h_val);
  if (!nr_.empty()) d.n_r = upT(nr_);
  if (dga_frac_) {
    d.h_p = upT(hp_);
    d.nq = (int)q_size_;
    d.nfe = (int)fe_edge_.size();
    if (d.nq > 0) {
      upcsr(Q_, d.q_ptr, d.q_col, d.q_val);
      upcsr(Mq_, d.mq_ptr, d.mq_col, d.mq_val);
      d.Uc = zeros(q_size_);
      d.Uc_old = zeros(q_size_);
    }
    if (d.nfe > 0) {
      d.fe_edge = (const int32_t*)up(fe_edge_.data(), fe_edge_.size() * 4);
      d.fe_a = (const int32_t*)up(fe_a_.data(), fe_a_.size() * 4);
      d.fe_b = (const int32_t*)up(fe_b_.data(), fe_b_.size() * 4);
    }
  }
  const size_t nsrc = src_labels_.size();
  d.nse = (int)src_edge_.size();
  d.nsrc = (int)nsrc;
  d.se_edge = (const int32_t*)up(src_edge_.data(), src_edge_.size() * 4);
  d.se_kind = (const int8_t*)up(src_kind_e_.data(), src_kind_e_.size());
  d.se_begin = (const int*)up(src_begin_.data(), src_begin_.size() * 4);
  d.pair_src = (const int*)up(pair_src_.data(), pair_src_.size() * 4);
  d.pair_fac = (const double*)up(pair_fac_.data(), pair_fac_.size() * 8);
  d.pair_dir = (const int8_t*)up(pair_dir_.data(), pair_dir_.size());
  d.se_vec = (const double*)up(src_vec_.data(), src_vec_.size() * 8);
  d.se_post = (const double*)up(src_post_.data(), src_post_.size() * 8);
  d.src_amp = (const double*)up(src_amp_.data(), src_amp_.size() * 8);
  d.carrier = (const double*)up(carrier_.data(), carrier_.size() * 8);
  d.flux = (double*)dalloc((nsteps_ + 1) * 8);
  CU(cudaMemsetAsync(d.flux, 0, (nsteps_ + 1) * 8, stream_));
  // tet_h_update's block partials, then tet_frac_gather's
  d.nflux_part = (int)((NE + 255) / 256);
  if (d.nflux_part < 1) d.nflux_part = 1;
  if (d.nfe > 0) d.nflux_part += (d.nfe + 255) / 256;
  d.flux_part = (double*)dalloc((size_t)d.nflux_part * 8);
  CU(cudaMemsetAsync(d.flux_part, 0, (size_t)d.nflux_part * 8, stream_));
  // probes
  const size_t np = probe_tet_.size();
  std::vector<int32_t> pe(6 * np), pf(4 * np);
  for (size_t p = 0; p < np; p++) {
    auto el = vol_edges(probe_tet_[p]);
    for (int q = 0; q < 6; q++) pe[6 * p + q] = el[q];
    for (int q = 0; q < 4; q++) pf[4 * p + q] = vtf_[probe_tet_[p]][q];
  }
  d.np = (int)np;
  d.p_edges = (const int32_t*)up(pe.data(), pe.size() * 4);
  d.p_faces = (const int32_t*)up(pf.data(), pf.size() * 4);
  d.p_we = (const double*)up(probe_we_.data(), probe_we_.size() * 8);
  d.p_hf = (const double*)up(probe_hf_.data(), probe_hf_.size() * 8);
  d.samples = (double*)dalloc((size_t)nslots_ * np * 6 * 8);
  d.slot_of_step = (const int*)up(slot_of_step_.data(), slot_of_step_.size() * 4);
  d.step = (int*)dalloc(sizeof(int));
  CU(cudaMemsetAsync(d.step, 0, sizeof(int), stream_));
  CU(cudaHostAlloc((void**)&pinned_, (nsrc + 6 * np + 1) * sizeof(double), cudaHostAllocDefault));
  // initial state (t = 0 sources, Discretization.hpp:671-791)
  auto put_state = [&](void* dst, const std::vector<double>& v) {
    if (!f32) CU(cudaMemcpyAsync(dst, v.data(), v.size() * 8, cudaMemcpyHostToDevice, stream_));
    else {
      auto f = as<float>(v);
      CU(cudaMemcpyAsync(dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice, stream_));
      CU(cudaStreamSynchronize(stream_));
    }
  };
  put_state(d.U, init_U_);
  put_state(d.I, init_I_);
  if (f32) tet_launch_initial_probes<float>(d, stream_);
  else tet_launch_initial_probes<double>(d, stream_);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(stream_));
}

void TetSim::launch_steps(int n, cudaEvent_t* ev) {
  for (int q = 0; q < n; q++) {
    cudaError_t e = opt_.precision == 1 ? tet_launch_step<float>(dp_, stream_, ev)
                                        : tet_launch_step<double>(dp_, stream_, ev);
    CU(e);
  }
}

uint64_t TetSim::step(uint64_t n) {
  if (group_) {
    const uint64_t k = group_->step(n);
    step_ = group_->step_index(0);
    return k;
  }
  if (step_ + n > nsteps_) n = nsteps_ - step_;
  if (n == 0) { last_ms_ = 0; return 0; }
  CU(cudaEventRecord(ev0_, stream_));
  launch_steps((int)n, nullptr);
  CU(cudaEventRecord(ev1_, stream_));
  CU(cudaEventSynchronize(ev1_));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, ev0_, ev1_));
  last_ms_ = ms;
  step_ += n;
  return n;
}

uint64_t TetSim::phase_times(uint64_t n, double* ms5) {
  if (group_) {
    const uint64_t k = group_->phase_times(n, ms5);
    step_ = group_->step_index(0);
    return k;
  }
  if (step_ + n > nsteps_) n = nsteps_ - step_;
  for (int q = 0; q < 5; q++) ms5[q] = 0;
  cudaEvent_t ev[6];
  for (auto& e : ev) CU(cudaEventCreate(&e));
  for (uint64_t i = 0; i < n; i++) {
    launch_steps(1, ev);
    CU(cudaEventSynchronize(ev[5]));
    for (int q = 0; q < 5; q++) {
      float ms = 0;
      CU(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
      ms5[q] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  step_ += n;
  return n;
}

uint64_t TetSim::step_io(const double* carrier_in, double* probe_out) {
  if (group_) {
    const uint64_t k = group_->step_io(carrier_in, probe_out);
    step_ = group_->step_index(0);
    return k;
  }
  if (step_ >= nsteps_) return 0;
  const size_t nsrc = src_labels_.size(), np = probe_tet_.size();
  if (!pinned_) CU(cudaHostAlloc((void**)&pinned_, (nsrc + 6 * np + 1) * sizeof(double), cudaHostAllocDefault));
  if (carrier_in && nsrc) {
    std::memcpy(pinned_, carrier_in, nsrc * sizeof(double));
    CU(cudaMemcpyAsync((double*)dp_.carrier + step_ * nsrc, pinned_, nsrc * sizeof(double), cudaMemcpyHostToDevice,
                       stream_));
  }
  launch_steps(1, nullptr);
  const uint64_t sched = method_ == 1 ? step_ + 1 : step_;
  const int slot = slot_of_step_[sched];
  if (probe_out && slot >= 0 && np)
    CU(cudaMemcpyAsync(pinned_ + nsrc, dp_.samples + (size_t)slot * np * 6, np * 6 * sizeof(double),
                       cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  if (probe_out && slot >= 0 && np) std::memcpy(probe_out, pinned_ + nsrc, np * 6 * sizeof(double));
  step_++;
  return 1;
}

size_t TetSim::n_samples() const {
  if (group_) return group_->n_samples(0);
  size_t c = 0;
  const uint64_t upto = method_ == 1 ? step_ + 1 : step_;
  for (uint64_t i = 0; i < upto && i < slot_of_step_.size(); i++)
    if (slot_of_step_[i] >= 0) c++;
  return c;
}

void TetSim::get_probes(double* times, double* values, size_t cap) const {
  if (group_) return group_->get_probes(0, times, values, cap);
  size_t ns = n_samples();
  if (ns > cap) ns = cap;
  const size_t np = probe_tet_.size();
  if (times) std::memcpy(times, sample_times_.data(), ns * 8);
  if (values && ns && np) CU(cudaMemcpy(values, dp_.samples, ns * np * 6 * 8, cudaMemcpyDeviceToHost));
}

void TetSim::probe_points(double* xyz, uint64_t* cells, size_t cap) const {
  for (size_t p = 0; p < probe_tet_.size() && p < cap; p++) {
    if (xyz) for (int a = 0; a < 3; a++) xyz[3 * p + a] = probe_pts_[p][a];
    if (cells) cells[p] = (uint64_t)probe_tet_[p];
  }
}

static void fetch(const void* d, size_t n, bool f32, double* out) {
  if (!out) return;
  if (!f32) {
    CU(cudaMemcpy(out, d, n * 8, cudaMemcpyDeviceToHost));
    return;
  }
  std::vector<float> tmp(n);
  CU(cudaMemcpy(tmp.data(), d, n * 4, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; i++) out[i] = tmp[i];
}

void TetSim::get_state(double* U, double* B, double* F) {
  if (group_) return group_->get_state(0, U, B, F);
  const bool f32 = opt_.precision == 1;
  CU(cudaStreamSynchronize(stream_));
  fetch(dp_.U, edges_.size(), f32, U);
  fetch(dp_.B, faces_.size(), f32, B);
  fetch(dp_.F, faces_.size(), f32, F);
}

void TetSim::set_state(const double* U, const double* F) {
  if (group_) return group_->set_state(0, U, F);
  if (U && q_size_ > 0)
    throw UnsupportedError("tf_set_state: a dga run with fractured edges keeps node-star fractions that U does not fix");
  const bool f32 = opt_.precision == 1;
  auto put = [&](void* dst, const double* src, size_t n) {
    if (!src) return;
    if (!f32) CU(cudaMemcpy(dst, src, n * 8, cudaMemcpyHostToDevice));
    else {
      std::vector<float> t(src, src + n);
      CU(cudaMemcpy(dst, t.data(), n * 4, cudaMemcpyHostToDevice));
    }
  };
  put(dp_.U, U, edges_.size());
  put(dp_.F, F, faces_.size());
}

void TetSim::get_flux(double* flux, size_t cap, size_t* n) const {
  if (group_) return group_->get_flux(0, flux, cap, n);
  size_t m = step_ < cap ? step_ : cap;
  if (flux && m) CU(cudaMemcpy(flux, dp_.flux, m * 8, cudaMemcpyDeviceToHost));
  if (n) *n = step_;
}

void TetSim::get_losses(double* loss, size_t cap, size_t* n) const {
  if (group_) return group_->get_losses(0, loss, cap, n);
  Sim::get_losses(loss, cap, n);  // dga: lossless here
}

size_t TetSim::solver_stats(int32_t* iters, double* resid, size_t cap) const {
  if (group_) return group_->solver_stats(0, iters, resid, cap);
  if (method_ < 2) return 0;
  size_t m = step_ < cap ? step_ : cap;
  if (iters && m) CU(cudaMemcpy(iters, dp_.cg_iters, m * 4, cudaMemcpyDeviceToHost));
  if (resid && m) CU(cudaMemcpy(resid, dp_.cg_resid, m * 8, cudaMemcpyDeviceToHost));
  return step_;
}

int TetSim::kernel_variant() const { return group_ ? group_->cg_variant() : 0; }

size_t TetSim::guess_stats(int8_t* kept, size_t cap) const {
  return group_ ? group_->guess_stats(0, kept, cap) : 0;
}

size_t TetSim::training_loss(float* loss, size_t cap) const {
  return group_ ? group_->training_loss(loss, cap) : 0;
}

double TetSim::energy() {
  // gfdtd: the group engine's GPU reduction; dga: H^-1 through a PCG solve
  if (method_ == 1) return dga_energy();
  if (method_ != 2 || !group_) throw UnsupportedError("tf_energy: fem's energy is not provided");
  return group_->energy(0);
}

// dga: W^n = 1/2 U^n.H^-1.U^{n+1} + 1/2 B.N.B over the class-1 edges
// (tet_launch_energy), H^-1 u by the standalone PCG kernel on H's class-1
// block in FP64 to 1e-15 relative.  Lossless runs only: the conducting
// classes do not conserve it.
double TetSim::dga_energy() {
  if (dga_frac_ || !nr_.empty())
    throw UnsupportedError("tf_energy: a dga run with conducting or magnetically lossy materials has no invariant");
  const bool f32 = opt_.precision == 1;
  if (!en_edges_) {
    if (H_.ptr.empty()) throw UnsupportedError("tf_energy: the dga operators were released");
    const uint32_t NE = (uint32_t)edges_.size();
    std::vector<int32_t> ie, pos(NE, -1);
    for (uint32_t e = 0; e < NE; e++)
      if (cls_[e] == 1) {
        pos[e] = (int32_t)ie.size();
        ie.push_back((int32_t)e);
      }
    const int ni = (int)ie.size();
    std::vector<int64_t> ptr(ni + 1, 0);
    std::vector<int32_t> col;
    std::vector<double> val;
    for (int i = 0; i < ni; i++) {
      for (int64_t k = H_.ptr[ie[i]]; k < H_.ptr[ie[i] + 1]; k++) {
        const int32_t c = pos[H_.col[k]];
        if (c < 0) throw CudaError("tf_energy: H has a column outside the class-1 edges");
        col.push_back(c);
        val.push_back(H_.val[k]);
      }
      ptr[i + 1] = (int64_t)col.size();
    }
    auto dalloc = [&](size_t bytes) -> void* {
      void* p = nullptr;
      CU(cudaMalloc(&p, bytes ? bytes : 16));
      allocs_.push_back(p);
      return p;
    };
    auto up = [&](const void* src, size_t bytes) -> void* {
      void* p = dalloc(bytes);
      if (bytes) CU(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice));
      return p;
    };
    en_blocks_ = tet_cg_blocks<double>(opt_.device);
    if (en_blocks_ < 1) throw CudaError("tf_energy: no co-resident blocks for the CG kernel");
    DevPtrs& c = en_cg_;
    c.nfree = ni;
    c.a_ptr = (const int64_t*)up(ptr.data(), ptr.size() * 8);
    c.a_col = (const int32_t*)up(col.data(), col.size() * 4);
    c.a_val = up(val.data(), val.size() * 8);
    double* work = (double*)dalloc(((size_t)6 * ni + 4 * (size_t)en_blocks_ + 6) * 8);
    c.jac = work;
    c.r = work + ni;
    c.p = work + 2 * (size_t)ni;
    c.q = work + 3 * (size_t)ni;
    c.rhs = work + 4 * (size_t)ni;
    c.x = work + 5 * (size_t)ni;
    c.part_a = work + 6 * (size_t)ni;
    c.part_b = c.part_a + en_blocks_;
    double* tail = c.part_a + 4 * (size_t)en_blocks_;
    c.cg_resid = tail;
    c.cg_iters = (int32_t*)(tail + 1);
    c.step = (int*)(tail + 2);
    c.cg_limit = (int32_t*)(tail + 3);
    c.err = (int*)(tail + 4);
    c.gbar = (unsigned int*)(tail + 5);
    c.tol = 1e-15;
    c.cg_maxiter = 5000;
    c.cg_criterion = 1;
    en_n_ = ni;
    en_edges_ = (int32_t*)up(ie.data(), ie.size() * 4);
    const size_t nparts = 2 * (((size_t)ni + 255) / 256 + 1) + ((faces_.size() + 255) / 256 + 1);
    en_part_ = (double*)dalloc(nparts * 8);
    en_out_ = (double*)dalloc(8);
  }
  cudaError_t e = f32 ? tet_launch_energy<float>(dp_, en_cg_, en_blocks_, en_edges_, en_n_, en_part_, en_out_, stream_)
                      : tet_launch_energy<double>(dp_, en_cg_, en_blocks_, en_edges_, en_n_, en_part_, en_out_, stream_);
  CU(e);
  double w = 0;
  int berr = 0;
  CU(cudaMemcpyAsync(&w, en_out_, 8, cudaMemcpyDeviceToHost, stream_));
  CU(cudaMemcpyAsync(&berr, en_cg_.err, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  if (berr) throw CudaError("tf_energy: a grid barrier wait of the CG kernel ran out of time");
  return w;
}

}  // namespace tf
