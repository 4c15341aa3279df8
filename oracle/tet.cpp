// ORACLE — test infrastructure only.
// FP64 CPU restatement of TetFIT's tetrahedral paths:
//   netgen reader + numbering   src/DGA/Discretization.hpp:5868-6926, unique :10173-10299
//   gmsh conversion             Discretization.hpp:5692-5866, Utilities.hpp:159-223
//   geometry helpers            Discretization.hpp:10301-10545
//   dga operators               ConstructCodecasaMaterialMatrices :8694-9513
//   gfdtd operators             ConstructGFDTDMaterialMatrices   :8132-8692
//   dga loop                    Discretization.hpp:538-953
//   gfdtd loop                  Discretization.hpp:1360-1579
//   Jacobi-PCG                  src/DGA/ConjugateGradientSolver.hpp:52-129
//   probes                      FindProbe :3645-3747, GetWhitneyElectricField :3768-3875,
//                               GetMagneticField :3877-3897, ExportFields :2403-2470
//   sources                     Discretization.hpp:3907-4202, Source.hpp:313-567
// Faces and edges are numbered as the reference numbers them (lexicographic
// order of their sorted node triples / pairs), so state vectors come out in
// the reference's order.
//
// Scope and documented divergences:
//  * conductivity (sigma) enters gfdtd and fem through SigMat and dga through
//    its edge classes (:6776-6905, :9262-9475); magnetic losses (chi) enter
//    dga through its face classes (:6357-6542, :9128-9205) where a face's
//    tets share chi (and mu); fractured faces, whose old values the
//    reference reads from the electric state (:586), and chi on gfdtd and fem
//    are rejected;
//  * tets with material label 7 are dropped (:6091); the reference also keeps 4
//    zero-initialised face slots per dropped tet (:6130-6152) that create a
//    spurious face (0,0,0); here they are not created;
//  * the first dga export uses t = 0 (the reference reads an uninitialised time,
//    :805-806);
//  * a dga edge driven by a current dipole keeps its value (the reference writes
//    an uninitialised value into it, :829-860);
//  * gfdtd eps-mass: the reference's node dual basis (:8586-8604) is dual to
//    half edges pointing away from the node and carries neither the factor 1/4
//    nor the edge orientation signs, which quadruples the mass (halves the wave
//    speed) and flips some off-diagonal terms on non-orthogonal meshes; this is
//    reproduced by default, `consistent_mass` corrects it;
//  * the time-step estimate is a Lanczos solve in the stiffness inner product
//    instead of Spectra's Arnoldi at tolerance 2e-2 (:7020-7174); `SET step`
//    pins dt.
#include "tet.hpp"

#include "lanczos.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <numeric>
#include <sstream>
#include <stdexcept>

namespace orc {

using V3 = std::array<double, 3>;
static V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static V3 cross(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static V3 scale(const V3& a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
static V3 matvec(const Mat3& m, const V3& v) {
  V3 r;
  for (int i = 0; i < 3; i++) r[i] = m.m[i][0] * v[0] + m.m[i][1] * v[1] + m.m[i][2] * v[2];
  return r;
}
// 3x3 determinant by cofactor expansion along the first row (the zero test
// the reference applies to sigma, Discretization.hpp:8604, 8041)
static double mat_det(const Mat3& a) {
  const auto& m = a.m;
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

static bool mat_zero(const Mat3& m) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      if (m.m[i][j] != 0) return false;
  return true;
}

// ------------------------------------------------------------------ CSR
Csr Csr::build(uint32_t nr, uint32_t nc, const std::vector<Trip>& t) {
  Csr m;
  m.nrows = nr;
  m.ncols = nc;
  std::vector<uint64_t> cnt(nr + 1, 0);
  for (auto& x : t) cnt[x.r + 1]++;
  for (uint32_t r = 0; r < nr; r++) cnt[r + 1] += cnt[r];
  std::vector<uint32_t> cc(t.size());
  std::vector<double> vv(t.size());
  std::vector<uint64_t> pos(cnt.begin(), cnt.end() - 1);
  for (auto& x : t) {
    cc[pos[x.r]] = x.c;
    vv[pos[x.r]] = x.v;
    pos[x.r]++;
  }
  m.ptr.assign(nr + 1, 0);
  std::vector<uint32_t> idx;
  for (uint32_t r = 0; r < nr; r++) {
    idx.resize(cnt[r + 1] - cnt[r]);
    std::iota(idx.begin(), idx.end(), 0u);
    const uint64_t b = cnt[r];
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return cc[b + x] < cc[b + y]; });
    for (size_t q = 0; q < idx.size(); q++) {
      uint32_t c = cc[b + idx[q]];
      double v = vv[b + idx[q]];
      if (!m.col.empty() && m.col.size() > m.ptr[r] && m.col.back() == c) m.val.back() += v;
      else {
        m.col.push_back(c);
        m.val.push_back(v);
      }
    }
    m.ptr[r + 1] = m.col.size();
  }
  return m;
}

void Csr::mul(const double* x, double* y) const {
  for (uint32_t r = 0; r < nrows; r++) {
    double s = 0;
    for (uint64_t k = ptr[r]; k < ptr[r + 1]; k++) s += val[k] * x[col[k]];
    y[r] = s;
  }
}

void Csr::mul_t(const double* x, double* y) const {
  std::fill(y, y + ncols, 0.0);
  for (uint32_t r = 0; r < nrows; r++)
    for (uint64_t k = ptr[r]; k < ptr[r + 1]; k++) y[col[k]] += val[k] * x[r];
}

double Csr::diag(uint32_t i) const {
  for (uint64_t k = ptr[i]; k < ptr[i + 1]; k++)
    if (col[k] == i) return val[k];
  return 0;
}

// Cholesky inverse of a small SPD matrix (Eigen llt().solve(Identity)).
static void spd_inverse(std::vector<double>& a, int n) {
  std::vector<double> L(n * n, 0.0);
  for (int k = 0; k < n; k++) {
    double x = a[k * n + k];
    for (int j = 0; j < k; j++) x -= L[k * n + j] * L[k * n + j];
    if (!(x > 0)) throw std::runtime_error("local mass matrix is not positive definite");
    L[k * n + k] = std::sqrt(x);
    for (int i = k + 1; i < n; i++) {
      double y = a[i * n + k];
      for (int j = 0; j < k; j++) y -= L[i * n + j] * L[k * n + j];
      L[i * n + k] = y / L[k * n + k];
    }
  }
  std::vector<double> inv(n * n);
  std::vector<double> y(n);
  for (int c = 0; c < n; c++) {
    for (int i = 0; i < n; i++) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int j = 0; j < i; j++) s -= L[i * n + j] * y[j];
      y[i] = s / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
      double s = y[i];
      for (int j = i + 1; j < n; j++) s -= L[j * n + i] * inv[j * n + c];
      inv[i * n + c] = s / L[i * n + i];
    }
  }
  a = inv;
}

// ------------------------------------------------------------------ mesh
std::array<double, 3> TetOracle::edge_bar(uint32_t e) const {
  const auto &a = pts[edges[e][0]], &b = pts[edges[e][1]];
  return {0.5 * (a[0] + b[0]), 0.5 * (a[1] + b[1]), 0.5 * (a[2] + b[2])};
}
std::array<double, 3> TetOracle::face_bar(uint32_t f) const {
  const auto &a = pts[faces[f][0]], &b = pts[faces[f][1]], &c = pts[faces[f][2]];
  return {(a[0] + b[0] + c[0]) / 3.0, (a[1] + b[1] + c[1]) / 3.0, (a[2] + b[2] + c[2]) / 3.0};
}
std::array<double, 3> TetOracle::vol_bar(uint32_t v) const {
  V3 r{0, 0, 0};
  for (int q = 0; q < 4; q++)
    for (int a = 0; a < 3; a++) r[a] += pts[vols[v][q]][a];
  return {r[0] / 4.0, r[1] / 4.0, r[2] / 4.0};
}

// ConvertFromGMSH (Discretization.hpp:5692-5866) with the element parser of
// Utilities.hpp:159-223, restated: skip 4 lines, node count, "id x y z" per
// node, skip 2 lines, element count, then per element "id type ntags t1 t2
// nodes" (two tags taken as given).  Tetrahedra (type 4) keep the first tag as
// material and their sorted nodes, triangles (type 2) the first tag as
// boundary id.  The result is the netgen text the reference writes to a
// temporary file: coordinates through a default ostream (6 significant
// digits), tetrahedra sorted, triangles in file order.
static std::string gmsh_as_netgen(std::istream& in) {
  std::string ln;
  for (int k = 0; k < 4; k++) std::getline(in, ln);
  std::getline(in, ln);
  const uint32_t np = (uint32_t)std::stoul(ln);
  std::ostringstream os;
  os << np << "\n";
  for (uint32_t i = 0; i < np; i++) {
    std::getline(in, ln);
    std::istringstream ls(ln);
    double id, x, y, z;
    ls >> id >> x >> y >> z;
    os << x << " " << y << " " << z << "\n";
  }
  std::getline(in, ln);
  std::getline(in, ln);
  std::getline(in, ln);
  const uint32_t ne = (uint32_t)std::stoul(ln);
  std::vector<std::pair<std::array<uint32_t, 4>, uint32_t>> tet;
  std::vector<std::array<uint32_t, 4>> tri;
  for (uint32_t i = 0; i < ne; i++) {
    std::getline(in, ln);
    std::istringstream ls(ln);
    uint32_t id, type, ntag, t1, t2;
    ls >> id >> type;
    if (type != 4 && type != 2) continue;
    ls >> ntag >> t1 >> t2;
    std::array<uint32_t, 4> n{0, 0, 0, 0};
    for (uint32_t j = 0; j < (type == 4 ? 4u : 3u); j++) ls >> n[j];
    if (type == 4) {
      std::sort(n.begin(), n.end());
      tet.push_back({n, t1});
    } else {
      tri.push_back({t1, n[0], n[1], n[2]});
    }
  }
  std::stable_sort(tet.begin(), tet.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  os << tet.size() << "\n";
  for (auto& t : tet) os << t.second << " " << t.first[0] << " " << t.first[1] << " " << t.first[2] << " " << t.first[3] << "\n";
  os << tri.size() << "\n";
  for (auto& t : tri) os << t[0] << " " << t[1] << " " << t[2] << " " << t[3] << "\n";
  return os.str();
}

void TetOracle::read_mesh() {
  const Mesh& msh = sc.meshes[sim.mesh];
  std::ifstream f(msh.file.c_str(), std::ios::binary);
  if (!f.is_open()) throw ScriptError("Invalid mesh file name");
  std::string buf;
  if (msh.mesher == "gmsh") {
    buf = gmsh_as_netgen(f);
  } else {
    std::stringstream ss;
    ss << f.rdbuf();
    buf = ss.str();
  }
  const char* p = buf.c_str();
  if (*p < '0' || *p > '9') my_throw(0, "Undefined mesh type! Available: tetrahedral, cartesian");
  char* end;
  uint32_t np = (uint32_t)std::strtoul(p, &end, 10);
  pts.reserve(np);
  for (uint32_t i = 0; i < np; i++) {
    double x = std::strtod(end, &end), y = std::strtod(end, &end), z = std::strtod(end, &end);
    pts.push_back({msh.scale * x, msh.scale * y, msh.scale * z});
  }
  uint32_t nt = (uint32_t)std::strtoul(end, &end, 10);
  std::vector<std::pair<std::array<uint32_t, 4>, uint32_t>> tt;
  tt.reserve(nt);
  for (uint32_t i = 0; i < nt; i++) {
    uint32_t m = (uint32_t)std::strtoul(end, &end, 10);
    std::array<uint32_t, 4> q;
    for (int k = 0; k < 4; k++) q[k] = (uint32_t)std::strtoul(end, &end, 10) - 1;
    std::sort(q.begin(), q.end());
    if (m != 7) tt.push_back({q, m});
  }
  std::stable_sort(tt.begin(), tt.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  const uint32_t L = (uint32_t)tt.size();
  node_vols.assign(np, {});
  std::vector<std::pair<std::array<uint32_t, 3>, uint32_t>> tri(4 * (size_t)L);
  for (uint32_t k = 0; k < L; k++) {
    auto t = tt[k].first;
    vols.push_back(t);
    vol_mat.push_back(tt[k].second);
    for (int q = 0; q < 4; q++) node_vols[t[q]].push_back(k);
    tri[k] = {{t[0], t[1], t[2]}, k};
    tri[k + L] = {{t[0], t[1], t[3]}, k + L};
    tri[k + 2 * L] = {{t[0], t[2], t[3]}, k + 2 * L};
    tri[k + 3 * L] = {{t[1], t[2], t[3]}, k + 3 * L};
    V3 v1 = sub(pts[t[1]], pts[t[0]]), v2 = sub(pts[t[2]], pts[t[0]]), v3 = sub(pts[t[3]], pts[t[0]]);
    cell_vol.push_back(dot(v1, cross(v2, v3)) / 6.0);
    const Material& mt = sc.materials[tt[k].second];
    // conductivity enters gfdtd and fem through SigMat and dga through its
    // edge classes; magnetic losses (chi) enter dga through its face classes
    if (!mat_zero(mt.chi) && method != 1)
      throw std::runtime_error("magnetic losses (chi) on tetrahedra are supported with method dga only");
  }
  // unique faces (Discretization.hpp:10173-10219)
  std::sort(tri.begin(), tri.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<uint32_t> flab(4 * (size_t)L);
  for (size_t q = 0; q < tri.size(); q++) {
    if (q == 0 || tri[q].first != tri[q - 1].first) faces.push_back(tri[q].first);
    flab[tri[q].second] = (uint32_t)faces.size() - 1;
  }
  const uint32_t NF = (uint32_t)faces.size();
  ftv.assign(NF, {});
  vtf.resize(L);
  for (uint32_t k = 0; k < L; k++) {
    ftv[flab[k]].push_back({k, -1});
    ftv[flab[k + L]].push_back({k, 1});
    ftv[flab[k + 2 * L]].push_back({k, -1});
    ftv[flab[k + 3 * L]].push_back({k, 1});
    vtf[k] = {{{flab[k + 3 * L], 1}, {flab[k + 2 * L], -1}, {flab[k + L], 1}, {flab[k], -1}}};
  }
  // unique edges (Discretization.hpp:10221-10299)
  std::vector<std::pair<std::array<uint32_t, 2>, uint32_t>> ed(3 * (size_t)NF);
  for (uint32_t f = 0; f < NF; f++) {
    auto s = faces[f];
    ed[f] = {{s[0], s[1]}, f};
    ed[f + NF] = {{s[0], s[2]}, f + NF};
    ed[f + 2 * NF] = {{s[1], s[2]}, f + 2 * NF};
  }
  std::sort(ed.begin(), ed.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<uint32_t> elab(3 * (size_t)NF);
  nte.assign(np, {});
  for (size_t q = 0; q < ed.size(); q++) {
    if (q == 0 || ed[q].first != ed[q - 1].first) {
      uint32_t e = (uint32_t)edges.size();
      edges.push_back(ed[q].first);
      nte[ed[q].first[0]].push_back({e, -1});
      nte[ed[q].first[1]].push_back({e, 1});
    }
    elab[ed[q].second] = (uint32_t)edges.size() - 1;
  }
  const uint32_t NE = (uint32_t)edges.size();
  fte.resize(NF);
  std::vector<Csr::Trip> ct;
  ct.reserve(3 * (size_t)NF);
  boundary_face.assign(NF, 0);
  bnd_edges.assign(NE, -1);
  bnd_dual.clear();
  for (uint32_t f = 0; f < NF; f++) {
    uint32_t e1 = elab[f], e2 = elab[f + NF], e3 = elab[f + 2 * NF];
    fte[f] = {{{e1, 1}, {e2, -1}, {e3, 1}}};
    ct.push_back({f, e1, 1.0});
    ct.push_back({f, e2, -1.0});
    ct.push_back({f, e3, 1.0});
    if (ftv[f].size() == 1) {
      // boundary face: boundary dual edges (Discretization.hpp:6380-6489)
      boundary_face[f] = 1;
      for (uint32_t e : {e1, e2, e3}) {
        if (bnd_edges[e] < 0) {
          bnd_edges[e] = (int32_t)bnd_dual.size();
          bnd_dual.push_back(face_bar(f));
        } else {
          V3& bd = bnd_dual[bnd_edges[e]];
          bd = sub(face_bar(f), bd);
          V3 edgvec = sub(pts[edges[e][1]], pts[edges[e][0]]);
          V3 facvec = cross(sub(pts[faces[f][1]], pts[faces[f][0]]), sub(pts[faces[f][2]], pts[faces[f][0]]));
          V3 volvec = sub(vol_bar(ftv[f][0].first), face_bar(f));
          if (dot(facvec, volvec) >= 0) facvec = scale(facvec, -1);
          if (dot(cross(edgvec, facvec), bd) > 0) bd = scale(bd, -1);
          bd = scale(bd, -1);
        }
      }
    } else if (ftv[f].empty()) {
      throw std::invalid_argument("Conductor boundary cannot be on mesh boundary!");
    }
  }
  C = Csr::build(NF, NE, ct);
  // boundary triangles (Discretization.hpp:6612-6754)
  uint32_t ntri = (uint32_t)std::strtoul(end, &end, 10);
  edge_bcs.assign(NE, 0);
  edge_src.assign(NE, {});
  is_pec.assign(NE, 0);
  for (uint32_t i = 0; i < ntri; i++) {
    uint32_t bid = (uint32_t)std::strtoul(end, &end, 10);
    std::array<uint32_t, 3> s;
    for (int k = 0; k < 3; k++) s[k] = (uint32_t)std::strtoul(end, &end, 10) - 1;
    std::sort(s.begin(), s.end());
    auto it = std::lower_bound(faces.begin(), faces.end(), s);
    if (it == faces.end() || *it != s) continue;
    uint32_t f = (uint32_t)(it - faces.begin());
    boundary_face[f] = bid;
    uint32_t which = bid < 100 ? sc.bnd_to_bc[bid] : 0;
    if (which != 0) {
      if (sc.bcs[which].type == "pec") {
        for (auto& se : fte[f]) {
          uint32_t e = se.first;
          edge_bcs[e] = which;
          edge_src[e].clear();
          is_pec[e] = 1;
          if (bnd_edges[e] >= 0) {
            bnd_dual[bnd_edges[e]] = {0, 0, 0};
            bnd_edges[e] = -1;
          }
        }
      }
    } else {
      std::vector<uint32_t> es;
      for (auto& se : fte[f])
        if (!is_pec[se.first]) es.push_back(se.first);
      for (uint32_t sl : sim.sources) {
        Source& src = sc.sources[sl];
        if (std::find(src.surfaces.begin(), src.surfaces.end(), bid) == src.surfaces.end()) continue;
        if (src.st == "b") continue;
        for (uint32_t e : es)
          if (std::find(edge_src[e].begin(), edge_src[e].end(), sl) == edge_src[e].end()) edge_src[e].push_back(sl);
      }
    }
  }
  // source consistency filter and edge classes (Discretization.hpp:6758-6859)
  cls.assign(NE, 1);
  for (uint32_t e = 0; e < NE; e++) {
    if (!edge_src[e].empty()) {
      const Source& first = sc.sources[edge_src[e][0]];
      uint32_t fs = first.surfaces.empty() ? 0 : first.surfaces[0];
      std::vector<uint32_t> keep;
      for (uint32_t s : edge_src[e]) {
        const Source& x = sc.sources[s];
        if (x.st == first.st && (x.surfaces.empty() ? 0 : x.surfaces[0]) == fs) keep.push_back(s);
      }
      edge_src[e] = keep;
    }
    bool dir = edge_bcs[e] != 0 && sc.bcs[edge_bcs[e]].type == "pec";
    for (uint32_t s : edge_src[e])
      if (sc.sources[s].st == "e") dir = true;
    if (dir) cls[e] = 4;
  }
  if (method == 1) classify_dga();
}

std::array<uint32_t, 6> TetOracle::vol_edges(uint32_t v) const {
  // local edge order ab, bc, ac, ad, bd, cd (sorted unique, then two swaps)
  std::vector<uint32_t> es;
  for (auto& sf : vtf[v])
    for (auto& se : fte[sf.first]) es.push_back(se.first);
  std::sort(es.begin(), es.end());
  es.erase(std::unique(es.begin(), es.end()), es.end());
  std::swap(es[1], es[2]);
  std::swap(es[1], es[3]);
  return {es[0], es[1], es[2], es[3], es[4], es[5]};
}

std::array<std::array<double, 3>, 6> TetOracle::dual_area_vectors(uint32_t v) const {
  // Discretization.hpp:10301-10346
  auto es = vol_edges(v);
  V3 eb[6], fb[4];
  for (int i = 0; i < 6; i++) eb[i] = edge_bar(es[i]);
  for (int i = 0; i < 4; i++) fb[i] = face_bar(vtf[v][i].first);
  V3 vb = vol_bar(v);
  double s = cell_vol[v] < 0 ? -0.5 : 0.5;
  std::array<V3, 6> r;
  r[0] = scale(cross(sub(vb, eb[0]), sub(fb[2], fb[3])), s);
  r[1] = scale(cross(sub(vb, eb[1]), sub(fb[0], fb[3])), s);
  r[2] = scale(cross(sub(vb, eb[2]), sub(fb[3], fb[1])), s);
  r[3] = scale(cross(sub(vb, eb[3]), sub(fb[1], fb[2])), s);
  r[4] = scale(cross(sub(vb, eb[4]), sub(fb[2], fb[0])), s);
  r[5] = scale(cross(sub(vb, eb[5]), sub(fb[0], fb[1])), s);
  return r;
}

std::array<std::array<double, 3>, 4> TetOracle::primal_area_vectors(uint32_t v) const {
  // Discretization.hpp:10400-10418
  const auto& n = vols[v];
  V3 e[6] = {sub(pts[n[1]], pts[n[0]]), sub(pts[n[2]], pts[n[1]]), sub(pts[n[2]], pts[n[0]]),
             sub(pts[n[3]], pts[n[0]]), sub(pts[n[3]], pts[n[1]]), sub(pts[n[3]], pts[n[2]])};
  std::array<V3, 4> r;
  r[0] = scale(cross(e[1], e[4]), 0.5);
  r[1] = scale(cross(e[2], e[3]), 0.5);
  r[2] = scale(cross(e[0], e[3]), 0.5);
  r[3] = scale(cross(e[0], e[2]), 0.5);
  return r;
}

void TetOracle::local_M(uint32_t v, double M[4][4], const Mat3* mat) const {
  // per-tet magnetic mass from dual area vectors (Discretization.hpp:8754-8776);
  // with chi in place of mu it is the magnetic-loss matrix Z (:8778-8802)
  auto fv = dual_area_vectors(v);
  const Mat3& mu = mat ? *mat : sc.materials.at(vol_mat[v]).mu;
  auto d = [&](int a, int b) { return dot(fv[a], matvec(mu, fv[b])); };
  const double c = 36.0 / std::fabs(cell_vol[v]);
  M[0][0] = (d(0, 0) + d(2, 2) + d(3, 3)) * c;
  M[1][1] = (d(0, 0) + d(1, 1) + d(4, 4)) * c;
  M[2][2] = (d(1, 1) + d(2, 2) + d(5, 5)) * c;
  M[3][3] = (d(3, 3) + d(4, 4) + d(5, 5)) * c;
  M[0][1] = (-d(1, 2) - d(3, 4)) * c;
  M[0][2] = (-d(0, 1) + d(3, 5)) * c;
  M[0][3] = (d(0, 4) + d(2, 5)) * c;
  M[1][2] = (-d(0, 2) - d(4, 5)) * c;
  M[1][3] = (d(0, 3) - d(1, 5)) * c;
  M[2][3] = (-d(2, 3) - d(1, 4)) * c;
  M[1][0] = M[0][1]; M[2][0] = M[0][2]; M[3][0] = M[0][3];
  M[2][1] = M[1][2]; M[3][1] = M[1][3]; M[3][2] = M[2][3];
}

Csr TetOracle::assemble_N() const {
  // N = sum over tets of the inverse 4x4 blocks (Discretization.hpp:9158-9255)
  std::vector<Csr::Trip> t;
  t.reserve(16 * vols.size());
  for (uint32_t v = 0; v < vols.size(); v++) {
    double M[4][4];
    local_M(v, M);
    std::vector<double> a(16);
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) a[4 * i + j] = M[i][j];
    spd_inverse(a, 4);
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++)
        if (a[4 * j + k] != 0) t.push_back({vtf[v][j].first, vtf[v][k].first, a[4 * j + k]});
  }
  return Csr::build((uint32_t)faces.size(), (uint32_t)faces.size(), t);
}

void TetOracle::apply_K(const double* x, double* y, std::vector<double>& tf) const {
  // K = C^T N C
  std::vector<double> cu(faces.size());
  C.mul(x, cu.data());
  tf.resize(faces.size());
  N.mul(cu.data(), tf.data());
  C.mul_t(tf.data(), y);
}

// Largest eigenvalue of Minv K, with K = C^T N C symmetric positive
// semi-definite and Minv symmetric positive definite, by Lanczos in the
// K inner product (the operator is self-adjoint there).
static double lanczos_K(size_t n, const std::function<void(const double*, double*)>& K,
                        const std::function<void(const double*, double*)>& Minv, int max_iter, double tol) {
  std::vector<double> x(n), v(n), Kv(n), w(n), Kw(n), vp(n, 0.0), Kvp(n, 0.0);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < n; i++) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    x[i] = (double)(s >> 11) / 9007199254740992.0 - 0.5;
  }
  // start in the range of Minv K
  K(x.data(), Kv.data());
  Minv(Kv.data(), v.data());
  K(v.data(), Kv.data());
  double nrm = 0;
  for (size_t i = 0; i < n; i++) nrm += v[i] * Kv[i];
  nrm = std::sqrt(nrm);
  for (size_t i = 0; i < n; i++) { v[i] /= nrm; Kv[i] /= nrm; }
  std::vector<double> al, be;
  double beta = 0, last = 0, lam = 0;
  for (int it = 0; it < max_iter; it++) {
    Minv(Kv.data(), w.data());  // w = Minv K v
    double alpha = 0;
    for (size_t i = 0; i < n; i++) alpha += w[i] * Kv[i];
    for (size_t i = 0; i < n; i++) w[i] -= alpha * v[i] + beta * vp[i];
    al.push_back(alpha);
    K(w.data(), Kw.data());
    double nb = 0;
    for (size_t i = 0; i < n; i++) nb += w[i] * Kw[i];
    nb = nb > 0 ? std::sqrt(nb) : 0;
    if (it % 10 == 9 || nb == 0 || it == max_iter - 1) {
      std::vector<double> bb(be.begin(), be.end());
      lam = tridiag_max_eig(al, bb);
      if (nb == 0 || std::fabs(lam - last) <= tol * std::fabs(lam)) break;
      last = lam;
    }
    be.push_back(nb);
    beta = nb;
    vp.swap(v);
    Kvp.swap(Kv);
    for (size_t i = 0; i < n; i++) { v[i] = w[i] / nb; Kv[i] = Kw[i] / nb; }
  }
  return lam;
}

void TetOracle::build_dga() {
  // ConstructCodecasaMaterialMatrices (Discretization.hpp:8694-9513)
  N = assemble_N();
  const uint32_t NE = (uint32_t)edges.size();
  // node-star matrix of eps (or of sigma, from the tets whose sigma has a
  // non-zero determinant, :8897): the dual basis of the star's edges
  // (:8900-9080), entries j <= k accumulated, then mirrored
  auto star_mass = [&](uint32_t nid, const std::vector<uint32_t>& gi, bool sigma) {
    const int n = (int)gi.size();
    std::vector<double> E(n * n, 0.0);
    for (uint32_t vv : node_vols[nid]) {
      const Mat3& mat = sigma ? sc.materials.at(vol_mat[vv]).sigma : sc.materials.at(vol_mat[vv]).eps;
      if (sigma && mat_det(mat) == 0) continue;
      auto el = vol_edges(vv);
      auto fv = primal_area_vectors(vv);
      const double V = std::fabs(cell_vol[vv]);
      int k = 0;
      while (vols[vv][k] != nid) k++;
      // (local edges, face vector index, sign of the 2/3V factor) per node position
      static const int kEd[4][3] = {{0, 2, 3}, {0, 1, 4}, {1, 2, 5}, {3, 4, 5}};
      static const int kFv[4][3] = {{1, 2, 3}, {0, 2, 3}, {1, 0, 3}, {0, 1, 2}};
      static const double kSg[4][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {1, 1, 1}};
      int ei[3];
      V3 w[3];
      for (int q = 0; q < 3; q++) {
        ei[q] = (int)(std::lower_bound(gi.begin(), gi.end(), el[kEd[k][q]]) - gi.begin());
        const double s = kSg[k][q] * 2.0 / 3.0 / V * vtf[vv][kFv[k][q]].second;
        w[q] = scale(fv[kFv[k][q]], s);
      }
      for (int a = 0; a < 3; a++)
        for (int b = a; b < 3; b++) {
          double val = dot(w[a], matvec(mat, w[b])) * V / 4;
          E[ei[a] * n + ei[b]] += val;
          if (a != b) E[ei[b] * n + ei[a]] = E[ei[a] * n + ei[b]];
        }
    }
    return E;
  };
  auto star_edges = [&](uint32_t nid) {
    std::vector<uint32_t> gi;
    for (auto& se : nte[nid]) gi.push_back(se.first);
    return gi;
  };
  std::vector<Csr::Trip> einv_t;
  for (uint32_t nid = 0; nid < pts.size(); nid++) {
    auto gi = star_edges(nid);
    const int n = (int)gi.size();
    std::vector<double> Hl = star_mass(nid, gi, false);
    spd_inverse(Hl, n);
    for (int j = 0; j < n; j++)
      for (int k = j; k < n; k++)
        if (Hl[j * n + k] != 0) {
          einv_t.push_back({gi[j], gi[k], Hl[j * n + k]});
          if (j != k) einv_t.push_back({gi[k], gi[j], Hl[j * n + k]});
        }
  }
  Csr Einv = Csr::build(NE, NE, einv_t);
  // dt (ComputeDGATimeStep, :7121-7174), from the unmasked eps inverses
  const char* skip = std::getenv("TF_ORACLE_SKIP_DT");
  if (skip && skip[0] == '1' && sim.step != 0) {
    dt_estimate = sim.step;
  } else {
    std::vector<double> tf;
    auto K = [&](const double* x, double* y) { apply_K(x, y, tf); };
    auto Mi = [&](const double* x, double* y) { Einv.mul(x, y); };
    double lam = lanczos_K(NE, K, Mi, 400, 1e-9);
    dt_estimate = sim.courant * 2.0 / std::sqrt(lam);
  }
  dt = dt_estimate;
  if (sim.step != 0) {
    if (sim.step > dt) possibly_unstable = true;
    else dt = sim.step;
  }
  // face classes (:6357-6542): a face is class 1 when its first tet has
  // chi = 0, else 2, unless its tets differ in chi (or, with chi, in mu): the
  // reference then makes it fractured (3), whose old values it maps onto the
  // electric state vector (Old_F_c, :586), which is refused here.  Per tet
  // (:9128-9205): N = (M + dt/2 Z)^-1 and RS = N (M - dt/2 Z) when chi has a
  // non-zero determinant, else N = M^-1 and RS = I; class-1 rows of N go to
  // Na, class-2 rows to Tr with R_r the diagonal of RS (the face's last tet
  // writes it).
  {
    const uint32_t NF = (uint32_t)faces.size();
    auto same = [](const Mat3& a, const Mat3& b) {
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          if (a.m[i][j] != b.m[i][j]) return false;
      return true;
    };
    fcls.assign(NF, 1);
    n_index.assign(NF, 0);
    r_index.assign(NF, 0);
    N_size = R_size = 0;
    for (uint32_t f = 0; f < NF; f++) {
      const Material& m0 = sc.materials.at(vol_mat[ftv[f][0].first]);
      if (ftv[f].size() == 2) {
        const Material& m1 = sc.materials.at(vol_mat[ftv[f][1].first]);
        if ((!mat_zero(m0.chi) || !mat_zero(m1.chi)) && (!same(m0.chi, m1.chi) || !same(m0.mu, m1.mu)))
          throw std::runtime_error("fractured magnetic-loss faces (chi or mu changing across a face with chi) are "
                                   "outside the supported path: the reference reads their old values from the "
                                   "electric state");
      }
      if (mat_zero(m0.chi)) {
        fcls[f] = 1;
        n_index[f] = N_size++;
      } else {
        fcls[f] = 2;
        r_index[f] = R_size++;
      }
    }
    std::vector<Csr::Trip> na_t, tr_t;
    R_r.assign(R_size, 0.0);
    for (uint32_t v = 0; v < vols.size(); v++) {
      const Mat3& chi = sc.materials.at(vol_mat[v]).chi;
      double M[4][4], Z[4][4];
      local_M(v, M);
      std::vector<double> Nl(16), RS(16, 0.0);
      if (mat_det(chi) != 0) {
        local_M(v, Z, &chi);
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) Nl[4 * i + j] = M[i][j] + 0.5 * dt * Z[i][j];
        spd_inverse(Nl, 4);
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) {
            double acc = 0;
            for (int m = 0; m < 4; m++) acc += Nl[4 * i + m] * (M[m][j] - 0.5 * dt * Z[m][j]);
            RS[4 * i + j] = acc;
          }
      } else {
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) Nl[4 * i + j] = M[i][j];
        spd_inverse(Nl, 4);
        for (int i = 0; i < 4; i++) RS[5 * i] = 1;
      }
      for (int j = 0; j < 4; j++) {
        const uint32_t f = vtf[v][j].first;
        if (fcls[f] == 2) R_r[r_index[f]] = RS[5 * j];
        for (int k = 0; k < 4; k++)
          if (Nl[4 * j + k] != 0) {
            if (fcls[f] == 1) na_t.push_back({n_index[f], vtf[v][k].first, Nl[4 * j + k]});
            else tr_t.push_back({r_index[f], vtf[v][k].first, Nl[4 * j + k]});
          }
      }
    }
    Na = Csr::build(N_size, NF, na_t);
    Tr = Csr::build(R_size, NF, tr_t);
    std::vector<Csr::Trip> nv;
    for (uint32_t f = 0; f < NF; f++) {
      const Csr& m = fcls[f] == 1 ? Na : Tr;
      const uint32_t r = fcls[f] == 1 ? n_index[f] : r_index[f];
      for (uint64_t q = m.ptr[r]; q < m.ptr[r + 1]; q++) nv.push_back({f, m.col[q], m.val[q]});
    }
    Nv = Csr::build(NF, NF, nv);
  }
  // masked node-star inverses (:9262-9475).  A star with a conducting tet
  // (sigma_node, :8897) gets H = (E + dt/2 S)^-1 and PQ = H (E - dt/2 S),
  // else H = E^-1 and PQ = I; Dirichlet rows and columns are masked.
  // Class-1 rows go to Ha, class-2 rows to Mp with the diagonal of PQ in
  // P_p (the star of the higher node writes it last), and a fractured
  // star's rows to Q and Mq.  Ha and Mp are filled from the upper triangle
  // and its mirror, whose row is h_index / p_index of the column's edge: 0
  // for an edge of another class, as the reference's zero-filled index
  // vectors give (:6546-6547).
  std::vector<Csr::Trip> h_t, mp_t, q_t, mq_t;
  P_p.assign(P_size, 0.0);
  for (uint32_t nid = 0; nid < pts.size(); nid++) {
    auto gi = star_edges(nid);
    const int n = (int)gi.size();
    bool sig_node = false;
    for (uint32_t vv : node_vols[nid])
      if (mat_det(sc.materials.at(vol_mat[vv]).sigma) != 0) sig_node = true;
    std::vector<double> E = star_mass(nid, gi, false);
    std::vector<double> S = sig_node ? star_mass(nid, gi, true) : std::vector<double>(n * n, 0.0);
    for (int j = 0; j < n; j++)
      if (cls[gi[j]] == 4) {
        for (int k = 0; k < n; k++) E[j * n + k] = E[k * n + j] = 0;
        E[j * n + j] = 1;
        if (sig_node)
          for (int k = 0; k < n; k++) S[j * n + k] = S[k * n + j] = 0;
      }
    std::vector<double> Hl(n * n), PQ(n * n, 0.0);
    if (sig_node) {
      for (int q = 0; q < n * n; q++) Hl[q] = E[q] + 0.5 * dt * S[q];
      spd_inverse(Hl, n);
      for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) {
          double acc = 0;
          for (int m = 0; m < n; m++) acc += Hl[j * n + m] * (E[m * n + k] - 0.5 * dt * S[m * n + k]);
          PQ[j * n + k] = acc;
        }
    } else {
      Hl = E;
      spd_inverse(Hl, n);
      for (int j = 0; j < n; j++) PQ[j * n + j] = 1;
    }
    for (int j = 0; j < n; j++)
      if (cls[gi[j]] == 4) {
        for (int k = 0; k < n; k++) Hl[j * n + k] = Hl[k * n + j] = PQ[j * n + k] = PQ[k * n + j] = 0;
        PQ[j * n + j] = 1;
      }
    const bool frac = dual_frac[nid] > 0;
    const uint32_t off = frac ? dual_frac[nid] - 1 : 0;
    for (int j = 0; j < n; j++) {
      const uint32_t ej = gi[j];
      if (cls[ej] == 1 || cls[ej] == 2) {
        const bool c1 = cls[ej] == 1;
        const std::vector<uint32_t>& idx = c1 ? h_index : p_index;
        std::vector<Csr::Trip>& t = c1 ? h_t : mp_t;
        if (!c1) P_p[p_index[ej]] = PQ[j * n + j];
        for (int k = j; k < n; k++)
          if (cls[gi[k]] != 4 && Hl[j * n + k] != 0) {
            t.push_back({idx[ej], gi[k], Hl[j * n + k]});
            if (j != k) t.push_back({idx[gi[k]], ej, Hl[j * n + k]});
          }
      }
      if (frac && cls[ej] != 4)
        for (int k = 0; k < n; k++) {
          if (cls[gi[k]] == 4) continue;
          if (PQ[j * n + k] != 0) q_t.push_back({off + (uint32_t)j, off + (uint32_t)k, PQ[j * n + k]});
          if (Hl[j * n + k] != 0) mq_t.push_back({off + (uint32_t)j, gi[k], Hl[j * n + k]});
        }
    }
  }
  Ha = Csr::build(H_size, NE, h_t);
  Mp = Csr::build(P_size, NE, mp_t);
  Q = Csr::build(Q_size, Q_size, q_t);
  Mq = Csr::build(Q_size, NE, mq_t);
  // edge-indexed view for the operator export: the Ha row of each class-1
  // edge and the Mp row of each class-2 edge
  std::vector<Csr::Trip> hv;
  for (uint32_t e = 0; e < NE; e++) {
    const Csr* m = cls[e] == 1 ? &Ha : cls[e] == 2 ? &Mp : nullptr;
    if (!m) continue;
    const uint32_t r = cls[e] == 1 ? h_index[e] : p_index[e];
    for (uint64_t q = m->ptr[r]; q < m->ptr[r + 1]; q++) hv.push_back({e, m->col[q], m->val[q]});
  }
  H = Csr::build(NE, NE, hv);
}

// dga edge classes (Discretization.hpp:6186-6215, 6776-6903).  Each node
// keeps the eps and sigma of the first tet that lists it; bit 0 of its class
// says that sigma is non-zero, bit 1 that a later tet has another eps, bit 2
// another sigma.  A free edge is fractured (3) when an end has class > 2,
// the ends' classes sum to 1 or 3, or their first sigmas differ; else
// lossless (1) when an end has class 0 or 2; else uniformly conducting (2).
// A fractured edge's ends get a block of U_c as long as their star, in the
// order the edges first reach them.
void TetOracle::classify_dga() {
  const uint32_t NE = (uint32_t)edges.size(), NP = (uint32_t)pts.size();
  std::vector<uint8_t> ncls(NP, 0);
  std::vector<Mat3> first_eps(NP), first_sig(NP);
  auto same = [](const Mat3& a, const Mat3& b) {
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        if (a.m[i][j] != b.m[i][j]) return false;
    return true;
  };
  for (uint32_t v = 0; v < vols.size(); v++) {
    const Material& mt = sc.materials.at(vol_mat[v]);
    for (int q = 0; q < 4; q++) {
      const uint32_t p = vols[v][q];
      if (!mat_zero(first_eps[p])) {
        if (!same(mt.sigma, first_sig[p])) ncls[p] |= 4;
        if (!same(mt.eps, first_eps[p])) ncls[p] |= 2;
        if (!mat_zero(first_sig[p])) ncls[p] |= 1;
      } else {
        first_eps[p] = mt.eps;
        first_sig[p] = mt.sigma;
        if (!mat_zero(mt.sigma)) ncls[p] |= 1;
      }
    }
  }
  h_index.assign(NE, 0);
  p_index.assign(NE, 0);
  dual_frac.assign(NP, 0);
  H_size = P_size = Q_size = 0;
  for (uint32_t e = 0; e < NE; e++) {
    if (cls[e] == 4) continue;
    const uint32_t p0 = edges[e][0], p1 = edges[e][1];
    const int r0 = ncls[p0], r1 = ncls[p1];
    if (r0 > 2 || r1 > 2 || r0 + r1 == 1 || r0 + r1 == 3 || !same(first_sig[p0], first_sig[p1])) {
      cls[e] = 3;
      for (uint32_t p : {p0, p1})
        if (dual_frac[p] == 0) {
          dual_frac[p] = Q_size + 1;
          Q_size += (uint32_t)nte[p].size();
        }
    } else if (r0 == 2 || r1 == 2 || r0 == 0 || r1 == 0) {
      cls[e] = 1;
      h_index[e] = H_size++;
    } else {
      cls[e] = 2;
      p_index[e] = P_size++;
    }
  }
  // U of a fractured edge is the sum of its entries in its two ends' blocks
  frac_cols.assign(NE, {0, 0});
  for (uint32_t e = 0; e < NE; e++) {
    if (cls[e] != 3) continue;
    for (int a = 0; a < 2; a++) {
      const uint32_t p = edges[e][a];
      uint32_t pos = 0;
      while (nte[p][pos].first != e) pos++;
      frac_cols[e][a] = dual_frac[p] - 1 + pos;
    }
  }
}

void TetOracle::build_gfdtd() {
  // ConstructGFDTDMaterialMatrices (Discretization.hpp:8132-8692), lossless
  const uint32_t NE = (uint32_t)edges.size();
  free_index.assign(NE, -1);
  free_edges.clear();
  for (uint32_t e = 0; e < NE; e++)
    if (cls[e] != 4) {
      free_index[e] = (int64_t)free_edges.size();
      free_edges.push_back(e);
    }
  N = assemble_N();
  std::vector<Csr::Trip> et, st;
  for (uint32_t nid = 0; nid < pts.size(); nid++) {
    for (uint32_t vv : node_vols[nid]) {
      auto el = vol_edges(vv);
      const double om = std::fabs(cell_vol[vv]) / 4.0;
      const Mat3& eps = sc.materials.at(vol_mat[vv]).eps;
      int k = 0;
      while (vols[vv][k] != nid) k++;
      static const int kEd[4][3] = {{0, 2, 3}, {0, 1, 4}, {1, 2, 5}, {3, 4, 5}};
      uint32_t e[3] = {el[kEd[k][0]], el[kEd[k][1]], el[kEd[k][2]]};
      V3 a1 = sub(edge_bar(e[0]), pts[nid]), a2 = sub(edge_bar(e[1]), pts[nid]), a3 = sub(edge_bar(e[2]), pts[nid]);
      double nc = std::pow(dot(a1, cross(a2, a3)), -1);
      V3 f[3] = {scale(cross(a2, a3), nc), scale(cross(a3, a1), nc), scale(cross(a1, a2), nc)};
      Mat3 oe;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) oe.m[i][j] = om * eps.m[i][j];
      static const int kPair[9][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 0}, {0, 2}, {2, 0}, {1, 2}, {2, 1}};
      // The reference's dual basis is built on half edges oriented away from
      // the node, without the factor 1/4 and without the edge orientation
      // signs.  consistent_mass applies both (a corrected eps-mass that
      // matches the dga and FIT discretisations); off by default for parity.
      double sg[3] = {1.0, 1.0, 1.0}, quarter = 1.0;
      if (consistent_mass) {
        for (int q = 0; q < 3; q++) sg[q] = edges[e[q]][1] == nid ? -1.0 : 1.0;
        quarter = 0.25;
      }
      for (auto& pq : kPair)
        et.push_back({e[pq[0]], e[pq[1]], quarter * sg[pq[0]] * sg[pq[1]] * dot(f[pq[0]], matvec(oe, f[pq[1]]))});
      // SigMat: the same dual basis with sigma, for tets whose sigma has a
      // non-zero determinant (:8604-8616)
      const Mat3& sig = sc.materials.at(vol_mat[vv]).sigma;
      if (mat_det(sig) != 0) {
        Mat3 os;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) os.m[i][j] = om * sig.m[i][j];
        for (auto& pq : kPair)
          st.push_back({e[pq[0]], e[pq[1]], quarter * sg[pq[0]] * sg[pq[1]] * dot(f[pq[0]], matvec(os, f[pq[1]]))});
      }
    }
  }
  E = Csr::build(NE, NE, et);
  Sig = Csr::build(NE, NE, st);
  lossy = !st.empty();
  estimate_dt_pencil();
  // SysMat = E + (0.5 dt) SigMat (:8644)
  split_system(1.0, 0.5 * dt);
}

void TetOracle::estimate_dt_pencil() {
  // dt (ComputeFEMTimeStep, :6928-7034): generalized problem K x = lambda E x
  const uint32_t NE = (uint32_t)edges.size();
  const char* skip = std::getenv("TF_ORACLE_SKIP_DT");
  if (skip && skip[0] == '1' && sim.step != 0) {
    dt_estimate = sim.step;
  } else {
    std::vector<double> tf, pre(NE);
    for (uint32_t e = 0; e < NE; e++) {
      double d = E.diag(e);
      pre[e] = d != 0 ? 1.0 / d : 1.0;
    }
    auto K = [&](const double* x, double* y) { apply_K(x, y, tf); };
    auto Mi = [&](const double* x, double* y) {
      std::fill(y, y + NE, 0.0);
      cg_solve(E, pre, x, y, 1e-12, 1000, nullptr);
    };
    double lam = lanczos_K(NE, K, Mi, 400, 1e-9);
    dt_estimate = sim.courant * 2.0 / std::sqrt(lam);
  }
  dt = dt_estimate;
  if (sim.step != 0) {
    if (sim.step > dt) possibly_unstable = true;
    else dt = sim.step;
  }
}

void TetOracle::split_system(double scale, double sig_coef) {
  // SysMat = scale * E + sig_coef * SigMat; A = SysMat on free rows/cols,
  // RHSmat1 = SysMat on free rows x Dirichlet cols (gfdtd :8644-8670 with
  // scale 1 and sig_coef dt / 2; fem :8086-8120 with scale 1 / dt^2, applied
  // as E * (1 / (dt dt)), and sig_coef 0.5 / dt).  The rows of E and SigMat
  // are merged by column: E_rc scale + coef S_rc where both hold an entry,
  // the one present otherwise.
  const uint32_t NE = (uint32_t)edges.size();
  std::vector<Csr::Trip> at, rt;
  for (uint32_t r = 0; r < NE; r++) {
    if (free_index[r] < 0) continue;
    uint64_t k = E.ptr[r], ks = lossy ? Sig.ptr[r] : 0;
    const uint64_t ke = E.ptr[r + 1], kse = lossy ? Sig.ptr[r + 1] : 0;
    while (k < ke || ks < kse) {
      uint32_t c;
      double v;
      if (ks >= kse || (k < ke && E.col[k] < Sig.col[ks])) {
        c = E.col[k];
        v = scale == 1.0 ? E.val[k] : E.val[k] * scale;
        k++;
      } else if (k >= ke || Sig.col[ks] < E.col[k]) {
        c = Sig.col[ks];
        v = sig_coef * Sig.val[ks];
        ks++;
      } else {
        c = E.col[k];
        v = (scale == 1.0 ? E.val[k] : E.val[k] * scale) + sig_coef * Sig.val[ks];
        k++;
        ks++;
      }
      if (free_index[c] < 0) rt.push_back({r, c, v});
      else at.push_back({(uint32_t)free_index[r], (uint32_t)free_index[c], v});
    }
  }
  A = Csr::build((uint32_t)free_edges.size(), (uint32_t)free_edges.size(), at);
  RHS1 = Csr::build(NE, NE, rt);
  jacobi.resize(free_edges.size());
  for (uint32_t i = 0; i < free_edges.size(); i++) {
    double d = A.diag(i);
    jacobi[i] = d != 0 ? 1.0 / d : 1.0;
  }
}

void TetOracle::build_fem() {
  // ConstructFEMaterialMatrices (Discretization.hpp:7687-8130), lossless:
  // N as for dga/gfdtd; E the Whitney edge mass by the quadrature with weight
  // 1/40 at the tet's nodes and 9/40 at its face barycentres (:7985-8060)
  const uint32_t NE = (uint32_t)edges.size();
  free_index.assign(NE, -1);
  free_edges.clear();
  for (uint32_t e = 0; e < NE; e++)
    if (cls[e] != 4) {
      free_index[e] = (int64_t)free_edges.size();
      free_edges.push_back(e);
    }
  N = assemble_N();
  std::vector<Csr::Trip> et, st;
  static const int kEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  for (uint32_t vv = 0; vv < vols.size(); vv++) {
    const Mat3& eps = sc.materials.at(vol_mat[vv]).eps;
    auto el = vol_edges(vv);
    // barycentric coordinates: [x y z 1] wn = (l0 l1 l2 l3), wn the inverse
    // of the matrix whose rows are [x_i y_i z_i 1] (:7960-7977), by cofactors
    double P[4][4], wn[4][4];
    for (int i = 0; i < 4; i++) {
      for (int a = 0; a < 3; a++) P[i][a] = pts[vols[vv][i]][a];
      P[i][3] = 1.0;
    }
    auto minor3 = [&](int r, int c) {
      double m[3][3];
      for (int i = 0, ii = 0; i < 4; i++) {
        if (i == r) continue;
        for (int j = 0, jj = 0; j < 4; j++) {
          if (j == c) continue;
          m[ii][jj++] = P[i][j];
        }
        ii++;
      }
      return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
             m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    };
    double det = 0.0;
    for (int c = 0; c < 4; c++) det += ((c & 1) ? -1.0 : 1.0) * P[0][c] * minor3(0, c);
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) wn[c][r] = (((r + c) & 1) ? -1.0 : 1.0) * minor3(r, c) / det;
    // Whitney edge functions at a point: w_ab = l_a grad l_b - l_b grad l_a
    auto whitney = [&](const V3& p, V3 w[6]) {
      double l[4];
      for (int i = 0; i < 4; i++) l[i] = p[0] * wn[0][i] + p[1] * wn[1][i] + p[2] * wn[2][i] + wn[3][i];
      for (int k = 0; k < 6; k++) {
        const int a = kEdge[k][0], b = kEdge[k][1];
        for (int x = 0; x < 3; x++) w[k][x] = l[a] * wn[x][b] - l[b] * wn[x][a];
      }
    };
    const Mat3& sig = sc.materials.at(vol_mat[vv]).sigma;
    const bool lossy_vol = mat_det(sig) != 0;
    double sumn[6][6] = {}, sumf[6][6] = {}, sumn_s[6][6] = {}, sumf_s[6][6] = {};
    for (int h = 0; h < 4; h++) {
      V3 w1[6], w2[6];
      whitney(pts[vols[vv][h]], w1);
      whitney(face_bar(vtf[vv][h].first), w2);
      for (int j = 0; j < 6; j++)
        for (int k = j; k < 6; k++) {
          sumn[j][k] += dot(w1[k], matvec(eps, w1[j]));
          sumf[j][k] += dot(w2[k], matvec(eps, w2[j]));
          if (lossy_vol) {  // (:8020-8021)
            sumn_s[j][k] += dot(w1[k], matvec(sig, w1[j]));
            sumf_s[j][k] += dot(w2[k], matvec(sig, w2[j]));
          }
        }
    }
    const double vol = std::fabs(cell_vol[vv]);
    for (int j = 0; j < 6; j++)
      for (int k = j; k < 6; k++) {
        const double val = vol * (sumn[j][k] + sumf[j][k] * 9.0) / 40.0;
        if (val != 0) {
          et.push_back({el[j], el[k], val});
          if (k != j) et.push_back({el[k], el[j], val});
        }
        if (lossy_vol) {  // SigMat (:8041-8051)
          const double sv = vol * (sumn_s[j][k] + sumf_s[j][k] * 9.0) / 40.0;
          if (sv != 0) {
            st.push_back({el[j], el[k], sv});
            if (k != j) st.push_back({el[k], el[j], sv});
          }
        }
      }
  }
  E = Csr::build(NE, NE, et);
  Sig = Csr::build(NE, NE, st);
  lossy = !st.empty();
  estimate_dt_pencil();
  // SysMat = E (1 / dt^2) + (0.5 / dt) SigMat (:8092-8093)
  split_system(1.0 / (dt * dt), 0.5 / dt);
}

int TetOracle::cg_solve(const Csr& M, const std::vector<double>& pre, const double* b, double* x, double tol,
                        int maxit, double* err) const {
  // ConjugateGradientSolver::solveWithGuess (ConjugateGradientSolver.hpp:52-103)
  const size_t n = pre.size();
  std::vector<double> r(n), z(n), p(n), q(n);
  M.mul(x, q.data());
  double r0 = 0;
  for (size_t i = 0; i < n; i++) {
    r[i] = b[i] - q[i];
    r0 += r[i] * r[i];
  }
  r0 = std::sqrt(r0);
  double res = r0, rho = 0, rho_p;
  int it = 0;
  while (res / r0 > tol && it < maxit) {
    for (size_t i = 0; i < n; i++) z[i] = pre[i] * r[i];
    rho_p = rho;
    rho = 0;
    for (size_t i = 0; i < n; i++) rho += r[i] * z[i];
    if (it == 0) p = z;
    else {
      double beta = rho / rho_p;
      for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    M.mul(p.data(), q.data());
    double pq = 0;
    for (size_t i = 0; i < n; i++) pq += p[i] * q[i];
    double a = rho / pq;
    res = 0;
    for (size_t i = 0; i < n; i++) {
      x[i] += a * p[i];
      r[i] -= a * q[i];
      res += r[i] * r[i];
    }
    res = std::sqrt(res);
    it++;
  }
  if (err) *err = res / r0;
  return it;
}

uint32_t TetOracle::find_probe(const std::array<double, 3>& pv) {
  // FindProbe (Discretization.hpp:3645-3747): breadth-first from the last hit,
  // orientation tests by 4x4 determinants with tolerance 1e-12.
  const double tol = 1e-12;
  auto det4 = [](const double m[4][4]) {
    double a = m[2][2] * m[3][3] - m[2][3] * m[3][2], b = m[2][1] * m[3][3] - m[2][3] * m[3][1];
    double c = m[2][1] * m[3][2] - m[2][2] * m[3][1], d = m[2][0] * m[3][3] - m[2][3] * m[3][0];
    double e = m[2][0] * m[3][2] - m[2][2] * m[3][0], f = m[2][0] * m[3][1] - m[2][1] * m[3][0];
    return m[0][0] * (m[1][1] * a - m[1][2] * b + m[1][3] * c) - m[0][1] * (m[1][0] * a - m[1][2] * d + m[1][3] * e) +
           m[0][2] * (m[1][0] * b - m[1][1] * d + m[1][3] * f) - m[0][3] * (m[1][0] * c - m[1][1] * e + m[1][2] * f);
  };
  std::vector<uint8_t> colour(vols.size(), 0);
  std::vector<uint32_t> q{root};
  colour[0]++;
  for (size_t h = 0; h < q.size(); h++) {
    uint32_t v = q[h];
    double rows[4][4];
    for (int r = 0; r < 4; r++) {
      for (int a = 0; a < 3; a++) rows[r][a] = pts[vols[v][r]][a];
      rows[r][3] = 1;
    }
    double det0 = det4(rows);
    bool ok = true;
    for (int r = 0; r < 4 && ok; r++) {
      double m[4][4];
      std::memcpy(m, rows, sizeof(m));
      for (int a = 0; a < 3; a++) m[r][a] = pv[a];
      double d1 = det4(m);
      ok = (det0 >= -tol && d1 >= -tol) || (det0 <= tol && d1 <= tol);
    }
    if (ok) {
      root = v;
      return v;
    }
    for (auto& sf : vtf[v]) {
      uint32_t n = ftv[sf.first].front().first;
      if (n == v) n = ftv[sf.first].back().first;
      if (!colour[n]) {
        q.push_back(n);
        colour[n]++;
      }
    }
    if (colour[v] < 255) colour[v]++;
  }
  return (uint32_t)vols.size();
}

double TetOracle::efield_source(uint32_t e, double t) {
  if (t < 0) return 0;
  V3 eb = edge_bar(e), v{0, 0, 0};
  for (auto s : edge_src[e])
    if (sc.sources[s].st == "e") {
      auto r = sc.sources[s].compute(eb[0], eb[1], eb[2], t);
      for (int a = 0; a < 3; a++) v[a] += r[a];
    }
  return dot(v, sub(pts[edges[e][1]], pts[edges[e][0]]));
}

double TetOracle::current_source(uint32_t e, double t) {
  if (t < 0) return 0;
  V3 eb = edge_bar(e), v{0, 0, 0};
  for (auto s : edge_src[e])
    if (sc.sources[s].st == "j") {
      auto r = sc.sources[s].compute(eb[0], eb[1], eb[2], t);
      for (int a = 0; a < 3; a++) v[a] += r[a];
    }
  V3 ev = sub(pts[edges[e][1]], pts[edges[e][0]]);
  return (1.0 / std::sqrt(dot(ev, ev))) * dot(v, ev);
}

double TetOracle::hfield_source(uint32_t e, double t) {
  // ComputeHfieldSource, tetrahedral branch (:4088-4148)
  if (t < 0) return 0;
  V3 eb = edge_bar(e), v{0, 0, 0};
  for (auto s : edge_src[e])
    if (sc.sources[s].st == "h") {
      auto r = sc.sources[s].compute(eb[0], eb[1], eb[2], t);
      for (int a = 0; a < 3; a++) v[a] += r[a];
    }
  return dot(v, bnd_dual[bnd_edges[e]]);
}

void TetOracle::export_probes(double t) {
  // ExportFields "probepoint": Whitney E at the point, H from the 4 face fluxes
  for (size_t p = 0; p < probe_elem.size(); p++) {
    uint32_t v = probe_elem[p];
    const auto& n = vols[v];
    // barycentric coordinates lambda(x) = [x y z 1] W and their gradients
    // (the rows of W): inverse of the node matrix [p_i 1]
    double Mt[4][4];
    for (int i = 0; i < 4; i++) {
      for (int a = 0; a < 3; a++) Mt[i][a] = pts[n[i]][a];
      Mt[i][3] = 1;
    }
    // W = inverse(Mt) by Gauss-Jordan with partial pivoting
    double W[4][8];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 8; j++) W[i][j] = j < 4 ? Mt[i][j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
      int piv = c;
      for (int r = c + 1; r < 4; r++)
        if (std::fabs(W[r][c]) > std::fabs(W[piv][c])) piv = r;
      for (int j = 0; j < 8; j++) std::swap(W[c][j], W[piv][j]);
      double d = W[c][c];
      for (int j = 0; j < 8; j++) W[c][j] /= d;
      for (int r = 0; r < 4; r++)
        if (r != c) {
          double f = W[r][c];
          for (int j = 0; j < 8; j++) W[r][j] -= f * W[c][j];
        }
    }
    // lambda_i = sum_a x_a W^-1... : Mt * G = I with G = W[:,4:]; lambda = [x 1] G
    double lam[4], grad[4][3];
    for (int i = 0; i < 4; i++) {
      lam[i] = probe_pts[p][0] * W[0][4 + i] + probe_pts[p][1] * W[1][4 + i] + probe_pts[p][2] * W[2][4 + i] +
               W[3][4 + i];
      for (int a = 0; a < 3; a++) grad[i][a] = W[a][4 + i];
    }
    static const int kE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    auto el = vol_edges(v);
    double E[3] = {0, 0, 0};
    for (int q = 0; q < 6; q++) {
      int a = kE[q][0], b = kE[q][1];
      for (int x = 0; x < 3; x++) E[x] += (lam[a] * grad[b][x] - lam[b] * grad[a][x]) * U[el[q]];
    }
    // H (GetMagneticField, :3877-3897)
    double fq[4];
    for (int i = 0; i < 4; i++) fq[i] = B[vtf[v][i].first];
    V3 pev[6] = {sub(pts[n[1]], pts[n[0]]), sub(pts[n[2]], pts[n[1]]), sub(pts[n[2]], pts[n[0]]),
                 sub(pts[n[3]], pts[n[0]]), sub(pts[n[3]], pts[n[1]]), sub(pts[n[3]], pts[n[2]])};
    const double vv = 3 * cell_vol[v];
    V3 r{0, 0, 0};
    for (int a = 0; a < 3; a++) {
      r[a] += (pev[0][a] * fq[1] - pev[2][a] * fq[2] + pev[3][a] * fq[3]) / vv;
      r[a] += (pev[0][a] * fq[0] - pev[1][a] * fq[2] + pev[4][a] * fq[3]) / vv;
      r[a] += (-pev[1][a] * fq[1] + pev[2][a] * fq[0] + pev[5][a] * fq[3]) / vv;
      r[a] += (pev[3][a] * fq[0] - pev[4][a] * fq[1] + pev[5][a] * fq[2]) / vv;
    }
    const Mat3& mu = sc.materials.at(vol_mat[v]).mu;
    for (int x = 0; x < 3; x++) samples.push_back(E[x]);
    for (int x = 0; x < 3; x++) samples.push_back(0.25 * (1.0 / mu.m[x][x]) * r[x]);
  }
  times.push_back(t);
}

void TetOracle::prepare(uint32_t label) {
  sim_label = label;
  sim = sc.simulations.at(label);
  const Mesh& msh = sc.meshes[sim.mesh];
  if (msh.type != "tetrahedral") throw std::runtime_error("tet oracle needs a tetrahedral mesh");
  if (sim.method == "dga") method = 1;
  else if (sim.method == "gfdtd") method = 2;
  else if (sim.method == "fem") method = 3;
  else throw std::runtime_error("tet oracle supports methods dga, gfdtd and fem");
  out = sc.outputs[sim.output];
  out.initialize();
  root = 0;
  read_mesh();
  if (method == 1) build_dga();
  else if (method == 2) build_gfdtd();
  else build_fem();
  const size_t NE = edges.size(), NF = faces.size();
  U.assign(NE, 0); I.assign(NE, 0); F.assign(NF, 0); B.assign(NF, 0);
  U_a.assign(H_size, 0); U_b.assign(P_size, 0); U_c.assign(Q_size, 0); U_c_old = U_c;
  F_a.assign(N_size, 0); F_b.assign(R_size, 0);
  Fb.assign(bnd_dual.size(), 0); Fb_old = Fb; SrcFld.assign(NE, 0);
  solution.assign(free_edges.size(), 0);
  if (out.mode == "silo") {
    // ExportFields "silo" (:2601-2677): E (Whitney) at the barycentre
    // (p0+p1+p2+p3)/4 (:10479-10484) and H of every tet at each print time,
    // sampled here like probes
    for (uint32_t v = 0; v < vols.size(); v++) {
      std::array<double, 3> b;
      for (int a = 0; a < 3; a++)
        b[a] = (pts[vols[v][0]][a] + pts[vols[v][1]][a] + pts[vols[v][2]][a] + pts[vols[v][3]][a]) / 4.0;
      probe_elem.push_back(v);
      probe_pts.push_back(b);
    }
  }
  // probes and point dipoles are located in the probepoint and maxerror
  // output modes only (:378-464)
  if (out.mode == "probepoint" || out.mode == "maxerror") {
    if (out.mode == "probepoint")
      for (auto& pv : out.probes) {
        uint32_t v = find_probe(pv);
        if (v < vols.size()) {
          probe_elem.push_back(v);
          probe_pts.push_back(pv);
        }
      }
    // point dipoles: nearest edge of the star of the tet's first node (:436-464)
    for (uint32_t sl : sim.sources) {
      Source& s = sc.sources[sl];
      if (s.st != "j") continue;
      uint32_t v = find_probe(s.location);
      if (v >= vols.size()) continue;
      uint32_t node = vols[v][0];
      uint32_t best = nte[node][0].first;
      auto d2 = [&](uint32_t e) {
        V3 b = edge_bar(e);
        V3 d = sub(b, {s.location[0], s.location[1], s.location[2]});
        return std::sqrt(dot(d, d));
      };
      double bd = d2(best);
      for (size_t q = 1; q < nte[node].size(); q++) {
        double d = d2(nte[node][q].first);
        if (d < bd) { bd = d; best = nte[node][q].first; }
      }
      edge_src[best].push_back(sl);
    }
  }
  nsteps_total = 0;
  while ((double)(nsteps_total + 1) * dt <= sim.duration) nsteps_total++;
  step_index = 0;
  // initial sources at t = 0 (dga :671-791, gfdtd :1425-1445)
  for (uint32_t e = 0; e < NE; e++) {
    if (edge_bcs[e] != 0 && sc.bcs[edge_bcs[e]].type != "none") {
      U[e] = 0;
      SrcFld[e] = 0;
    } else if (!edge_src[e].empty()) {
      const std::string& ty = sc.sources[edge_src[e][0]].st;
      if (method == 1) {
        if (cls[e] == 4) U[e] = efield_source(e, 0);
      } else if (ty != "h") {
        if (ty == "j") I[e] = current_source(e, 0);
        else U[e] = efield_source(e, 0);
        SrcFld[e] = U[e];
      }
    }
  }
  U_old = U;
  U_older = U;
  if (method == 1 && (out.mode == "probepoint" || out.mode == "silo") && out.allow_print(0.0)) export_probes(0.0);
}

void TetOracle::dga_step(double t) {
  // Discretization.hpp:810-931
  const size_t NE = edges.size();
  Fb_old = Fb;
  std::fill(Fb.begin(), Fb.end(), 0.0);
  U_old = U;
  U_c_old = U_c;
  for (uint32_t e = 0; e < NE; e++) {
    if (edge_bcs[e] != 0 && sc.bcs[edge_bcs[e]].type != "none") {
      U[e] = 0;
    } else if (!edge_src[e].empty()) {
      const std::string& ty = sc.sources[edge_src[e][0]].st;
      if (ty == "h") Fb[bnd_edges[e]] = hfield_source(e, t - 0.5 * dt);
      else if (ty == "j") I[e] = current_source(e, t);
      else U[e] = efield_source(e, t);
    }
  }
  std::vector<double> curl_b(NE, 0.0), curl_f(NE);
  for (uint32_t e = 0; e < NE; e++)
    if (bnd_edges[e] >= 0) curl_b[e] = Fb[bnd_edges[e]];
  C.mul_t(F.data(), curl_f.data());
  for (uint32_t e = 0; e < NE; e++) curl_f[e] = curl_f[e] + curl_b[e] - I[e];
  // U_a += dt Ha cf, U_b = P_p .* U_b + dt Mp cf, U_c = Q U_c_old + dt Mq cf,
  // U = M U_frac (:887-891)
  std::vector<double> ha(H_size), mp(P_size), qo(Q_size), mq(Q_size);
  Ha.mul(curl_f.data(), ha.data());
  Mp.mul(curl_f.data(), mp.data());
  Q.mul(U_c_old.data(), qo.data());
  Mq.mul(curl_f.data(), mq.data());
  for (uint32_t r = 0; r < H_size; r++) U_a[r] = U_a[r] + dt * ha[r];
  for (uint32_t r = 0; r < P_size; r++) U_b[r] = P_p[r] * U_b[r] + dt * mp[r];
  for (uint32_t r = 0; r < Q_size; r++) U_c[r] = qo[r] + dt * mq[r];
  for (uint32_t e = 0; e < NE; e++) {
    if (cls[e] == 1) U[e] = U_a[h_index[e]];
    else if (cls[e] == 2) U[e] = U_b[p_index[e]];
    else if (cls[e] == 3) U[e] = U_c[frac_cols[e][0]] + U_c[frac_cols[e][1]];
  }
  double fl = 0;
  for (uint32_t e = 0; e < NE; e++) fl += (U_old[e] + U[e]) * curl_b[e];
  flux.push_back(0.5 * fl);
  // B -= dt cu, F_a -= dt Na cu, F_b = R_r .* F_b - dt Tr cu, F = T F_frac
  // (:912-918)
  std::vector<double> cu(faces.size()), na(N_size), tr(R_size);
  C.mul(U.data(), cu.data());
  Na.mul(cu.data(), na.data());
  Tr.mul(cu.data(), tr.data());
  for (size_t f = 0; f < faces.size(); f++) B[f] = B[f] - dt * cu[f];
  for (uint32_t r = 0; r < N_size; r++) F_a[r] = F_a[r] - dt * na[r];
  for (uint32_t r = 0; r < R_size; r++) F_b[r] = R_r[r] * F_b[r] - dt * tr[r];
  for (size_t f = 0; f < faces.size(); f++) F[f] = fcls[f] == 1 ? F_a[n_index[f]] : F_b[r_index[f]];
  if ((out.mode == "probepoint" || out.mode == "silo") && out.allow_print(t)) export_probes(t);
}

void TetOracle::gfdtd_step(double t, double t_prev) {
  // Discretization.hpp:1459-1565
  const size_t NE = edges.size(), NF = faces.size();
  std::vector<double> cu(NF);
  C.mul(U.data(), cu.data());
  for (size_t f = 0; f < NF; f++) B[f] -= dt * cu[f];
  N.mul(B.data(), F.data());
  if ((out.mode == "probepoint" || out.mode == "silo") && out.allow_print(t_prev)) export_probes(t_prev);
  Fb_old = Fb;
  for (uint32_t e = 0; e < NE; e++) {
    if (edge_bcs[e] != 0 && sc.bcs[edge_bcs[e]].type != "none") {
      U[e] = 0;
      SrcFld[e] = U[e];
    } else if (!edge_src[e].empty()) {
      const std::string& ty = sc.sources[edge_src[e][0]].st;
      if (ty == "h" && bnd_edges[e] >= 0) Fb[bnd_edges[e]] = hfield_source(e, t - 0.5 * dt);
      else if (ty != "h") {
        if (ty == "j") I[e] = current_source(e, t);
        else U[e] = efield_source(e, t);
        SrcFld[e] = U[e];
      }
    }
  }
  // Psi = E U_old - (dt/2) SigMat U_old - RHSmat1 SrcFld - dt I + dt C^T F
  //       + dt Ctb Fb   (:1516-1519)
  std::vector<double> eu(NE), rs(NE), ctf(NE), psi(NE), su(NE, 0.0);
  E.mul(U_old.data(), eu.data());
  if (lossy) Sig.mul(U_old.data(), su.data());
  RHS1.mul(SrcFld.data(), rs.data());
  C.mul_t(F.data(), ctf.data());
  push_loss_pre(su);
  double fl = 0;
  for (uint32_t e = 0; e < NE; e++) {
    double cb = bnd_edges[e] >= 0 ? Fb[bnd_edges[e]] : 0.0;
    psi[e] = eu[e] - (0.5 * dt) * su[e] - rs[e] - dt * I[e] + dt * ctf[e] + dt * cb;
    double cbh = bnd_edges[e] >= 0 ? 0.5 * (Fb[bnd_edges[e]] + Fb_old[bnd_edges[e]]) : 0.0;
    fl += U_old[e] * cbh;
  }
  flux.push_back(fl);
  std::vector<double> rhs(free_edges.size());
  for (size_t k = 0; k < free_edges.size(); k++) rhs[k] = psi[free_edges[k]];
  double err = 0;
  int it = cg_solve(A, jacobi, rhs.data(), solution.data(), sim.tol, cg_maxiter, &err);
  cg_iters.push_back(it);
  cg_err.push_back(err);
  for (size_t k = 0; k < free_edges.size(); k++) U[free_edges[k]] = solution[k];
  push_loss_post();
  U_old = U;
}

// poynting.dat's third column for gfdtd and fem: each step pushes
// 0.5 U_old^T SigMat U_old before the solve and, from the second step on,
// U^T SigMat U after it (:1518-1546, :1733-1757), and the file prints the
// first n entries of that list (one row per step)
void TetOracle::push_loss_pre(const std::vector<double>& su) {
  double a = 0;
  if (lossy)
    for (size_t e = 0; e < su.size(); e++) a += U_old[e] * su[e];
  losses.push_back(0.5 * a);
}
void TetOracle::push_loss_post() {
  if (step_index + 1 <= 1) return;  // `if (i > 1)`
  double a = 0;
  if (lossy) {
    std::vector<double> su(U.size());
    Sig.mul(U.data(), su.data());
    for (size_t e = 0; e < su.size(); e++) a += U[e] * su[e];
  }
  losses.push_back(a);
}

void TetOracle::fem_step(double t, double t_prev) {
  // Discretization.hpp:1676-1776: central differences of the second-order
  // wave equation, E (U^{n+1} - 2 U^n + U^{n-1}) / dt^2 + C^T N C U^n = ...
  const size_t NE = edges.size(), NF = faces.size();
  std::vector<double> cu(NF);
  C.mul(U.data(), cu.data());
  for (size_t f = 0; f < NF; f++) B[f] -= dt * cu[f];
  if ((out.mode == "probepoint" || out.mode == "silo") && out.allow_print(t_prev)) export_probes(t_prev);
  Fb_old = Fb;
  for (uint32_t e = 0; e < NE; e++) {
    if (edge_bcs[e] != 0 && sc.bcs[edge_bcs[e]].type != "none") {
      U[e] = 0;
      SrcFld[e] = U[e];
    } else if (!edge_src[e].empty()) {
      const std::string& ty = sc.sources[edge_src[e][0]].st;
      if (ty == "h" && bnd_edges[e] >= 0) Fb[bnd_edges[e]] = hfield_source(e, t - 0.5 * dt);
      else if (ty != "h") {
        if (ty == "j") I[e] = current_source(e, t);
        else U[e] = efield_source(e, t);
        SrcFld[e] = U[e];
      }
    }
  }
  // Psi = 2 (E U_old) / dt^2 - C^T N C U_old + (1/dt) Ctb (Fb - Fb_old)
  //       - (E U_older) / dt^2 - RHSmat1 SrcFld - (1/dt) I   (:1713-1716)
  //       + (0.5/dt) SigMat U_older (lossy materials)
  std::vector<double> cuo(NF), ncu(NF), cc(NE), eu(NE), euo(NE), rs(NE), psi(NE), suo(NE, 0.0), su(NE, 0.0);
  C.mul(U_old.data(), cuo.data());
  N.mul(cuo.data(), ncu.data());
  C.mul_t(ncu.data(), cc.data());
  E.mul(U_old.data(), eu.data());
  E.mul(U_older.data(), euo.data());
  if (lossy) {
    Sig.mul(U_older.data(), suo.data());
    Sig.mul(U_old.data(), su.data());
  }
  RHS1.mul(SrcFld.data(), rs.data());
  push_loss_pre(su);
  const double idt2 = 1.0 / (dt * dt), idt = 1.0 / dt;
  double fl = 0;
  for (uint32_t e = 0; e < NE; e++) {
    const double fb = bnd_edges[e] >= 0 ? Fb[bnd_edges[e]] : 0.0;
    const double fbo = bnd_edges[e] >= 0 ? Fb_old[bnd_edges[e]] : 0.0;
    psi[e] = 2.0 * eu[e] * idt2 - cc[e] + idt * (fb - fbo) - euo[e] * idt2 + (0.5 / dt) * suo[e] - rs[e] -
             idt * I[e];
    fl += U_old[e] * (0.5 * (fb + fbo));
  }
  flux.push_back(fl);
  std::vector<double> rhs(free_edges.size());
  for (size_t k = 0; k < free_edges.size(); k++) rhs[k] = psi[free_edges[k]];
  double err = 0;
  int it = cg_solve(A, jacobi, rhs.data(), solution.data(), sim.tol, cg_maxiter, &err);
  cg_iters.push_back(it);
  cg_err.push_back(err);
  for (size_t k = 0; k < free_edges.size(); k++) U[free_edges[k]] = solution[k];
  push_loss_post();
  U_older = U_old;
  U_old = U;
}

uint64_t TetOracle::step(uint64_t n) {
  uint64_t done = 0;
  for (; done < n && step_index < nsteps_total; done++, step_index++) {
    const uint64_t i = step_index + 1;
    const double t = (double)i * dt;
    if (method == 1) dga_step(t);
    else if (method == 2) gfdtd_step(t, t - dt);
    else fem_step(t, t - dt);
  }
  return done;
}

}  // namespace orc
