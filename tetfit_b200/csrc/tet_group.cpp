// Host side of a gfdtd simulation group: lays S host-built simulations out in
// one device image (tet_group_kernels.cuh), partitions the CG rows among the
// persistent kernel's blocks and drives the step loop.
#include "tet_group.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <queue>
#include <numeric>
#include <string>

#include "cuda_util.hpp"
#include "host_parallel.hpp"

namespace tf {

namespace {

constexpr int kTuneSteps = 10;  // 2 warm-up steps, then 4 timed steps per CG variant
int64_t up32(int64_t n) { return (n + 31) & ~int64_t(31); }

// SELL-32 under construction (global slice offsets across simulations)
template <typename T>
struct SellHost {
  std::vector<int64_t> ptr{0};
  std::vector<int32_t, default_init_allocator<int32_t>> col;  // every slot is written
  std::vector<T, default_init_allocator<T>> val;
  // rows [0, nrows) of one simulation, nrows % 32 == 0; rows p >= nreal are
  // padding.  len(p): entries of row p; ent(p, j, c, v): entry j; pad(p):
  // column of a padding entry.
  template <typename L, typename E, typename P>
  void append(int64_t nrows, int64_t nreal, L len, E ent, P pad, bool values, int threads = 1) {
    // slice widths and offsets, then every slice filled at its own place
    const int64_t ns = nrows / 32, s_base = (int64_t)ptr.size() - 1;
    ptr.resize(ptr.size() + ns);
    parallel_for(ns, threads, [&](int64_t q0, int64_t q1) {
      for (int64_t q = q0; q < q1; q++) {
        int ml = 0;
        for (int l = 0; l < 32; l++)
          if (32 * q + l < nreal) ml = std::max(ml, (int)len(32 * q + l));
        ptr[s_base + q + 1] = 32 * (int64_t)ml;
      }
    }, 64);
    for (int64_t q = 0; q < ns; q++) ptr[s_base + q + 1] += ptr[s_base + q];
    col.resize(ptr.back());
    if (values) val.resize(ptr.back());
    parallel_for(ns, threads, [&](int64_t q0, int64_t q1) {
      for (int64_t q = q0; q < q1; q++) {
        const size_t base = (size_t)ptr[s_base + q];
        const int ml = (int)((ptr[s_base + q + 1] - ptr[s_base + q]) / 32);
        for (int l = 0; l < 32; l++) {
          const int64_t p = 32 * q + l;
          const int n = p < nreal ? (int)len(p) : 0;
          for (int j = 0; j < ml; j++) {
            int32_t c = 0;
            double v = 0.0;
            if (j < n) ent(p, j, c, v);
            else c = pad(p);
            col[base + 32 * (size_t)j + l] = c;
            if (values) val[base + 32 * (size_t)j + l] = (T)v;
          }
        }
      }
    }, 64);
  }
};

}  // namespace

void* TetGroup::dalloc(size_t bytes) {
  void* p = nullptr;
  CU(cudaMalloc(&p, bytes ? bytes : 16));
  allocs_.push_back(p);
  dev_bytes_ += bytes;
  return p;
}

template <typename V, typename A>
void* TetGroup::upload(const std::vector<V, A>& v) {
  void* p = dalloc(v.size() * sizeof(V));
  if (!v.empty()) CU(cudaMemcpy(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice));
  return p;
}

TetGroup::TetGroup(std::vector<TetSim*> sims, const RunOptions& opt, bool release_host) : opt_(opt) {
  if (sims.empty()) throw std::invalid_argument("empty simulation group");
  if (sims.size() > (size_t)kMaxGroup)
    throw std::invalid_argument("a group holds at most " + std::to_string(kMaxGroup) + " simulations");
  for (TetSim* t : sims)
    if (t->method() < 2) throw std::invalid_argument("simulation groups run methods gfdtd and fem only");
  CU(cudaSetDevice(opt_.device));
  int major = 0;
  CU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, opt_.device));
  if (major != 10) throw CudaError("device " + std::to_string(opt_.device) + " is not an sm_100 (B200) GPU");
  CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  CU(cudaEventCreate(&ev0_));
  CU(cudaEventCreate(&ev1_));
  if (opt_.precision == 1) build<float>(sims, release_host);
  else build<double>(sims, release_host);
}

TetGroup::~TetGroup() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (pinned_) cudaFreeHost(pinned_);
  for (void* p : allocs_) cudaFree(p);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

template <typename T>
void TetGroup::build(std::vector<TetSim*>& sims, bool release_host) {
  const int S = (int)sims.size();
  SellHost<T> A, Ef, N, Ct, Sg, Sa;
  std::vector<int32_t> sa_edge;
  std::vector<uint16_t> sa_slice_sim;
  std::vector<uint8_t> lossy(S, 0);
  std::vector<int32_t, default_init_allocator<int32_t>> fte, free_edge;  // filled completely
  std::vector<int32_t> dir_edge;
  std::vector<T, default_init_allocator<T>> pre, U0, I0, Src0;
  {
    // capacity for the stored entries (plus slice padding, which the class
    // grouping keeps small), so the members' appends rarely reallocate
    size_t na = 0, ne = 0, nc = 0, nn = 0;
    for (TetSim* t : sims) {
      na += t->A_.val.size();
      ne += t->E_.val.size();
      nc += t->Ct_.col.size();
      nn += t->N_.val.size();
    }
    auto room = [](size_t x) { return x + x / 8 + 4096; };
    A.col.reserve(room(na));
    A.val.reserve(room(na));
    Ef.col.reserve(room(ne));
    Ef.val.reserve(room(ne));
    Ct.col.reserve(room(nc));
    N.col.reserve(room(nn));
    N.val.reserve(room(nn));
  }
  std::vector<uint16_t> slice_sim, fslice_sim;
  std::vector<double> dt(S), tol(S);
  std::vector<uint8_t> fem(S, 0);
  std::vector<int> nsteps(S);
  std::vector<int64_t> stat_off(S), samp_off(S), sched_off(S), car_off(S);
  std::vector<int> nsrc(S), src_off(S), sim_se(S + 1), sim_probe(S + 1);
  std::vector<int32_t> se_edge;
  std::vector<int8_t> se_kind, pair_dir;
  std::vector<int> se_begin, pair_src, probe_sim, sched;
  std::vector<double> pair_fac, se_vec, se_post, src_amp, carrier, p_we, p_hf;
  std::vector<int32_t> p_edges, p_faces;
  int64_t eoff = 0, foff = 0, roff = 0, stat = 0, samp = 0;
  meta_.resize(S);
  for (int s = 0; s < S; s++) {
    TetSim& t = *sims[s];
    Meta& m = meta_[s];
    const int64_t NE = (int64_t)t.edges_.size(), NF = (int64_t)t.faces_.size();
    const int64_t nf = (int64_t)t.free_edges_.size();
    const int64_t NFp = up32(NF), nfp = up32(nf);
    m.nE = NE;
    m.nF = NF;
    m.nsteps = t.nsteps_;
    m.eoff = eoff;
    m.foff = foff;
    m.roff = roff;
    m.nrow_pad = nfp;
    m.nface_pad = NFp;
    dofs_ += (uint64_t)(NE + NF);
    nnz_a_real_ += t.A_.val.size();
    m.nnz_a = t.A_.val.size();
    // Free rows grouped by stencil: rows whose column offsets (col - row) are
    // the same form a class, classes in order of first appearance, rows of a
    // class in their own order.  On meshes with repeated local structure the
    // 32 rows of a slice then gather their j-th entries from consecutive
    // positions; each class has one row length, so slices carry little
    // padding.
    std::vector<int32_t> old_of_new(nf), pos(nf), cls(nf);
    auto alen_old = [&](int32_t k) { return t.A_.ptr[k + 1] - t.A_.ptr[k]; };
    {
      std::map<std::vector<int32_t>, int32_t> classes;
      std::vector<int32_t> key;
      for (int64_t k = 0; k < nf; k++) {
        key.clear();
        for (int64_t q = t.A_.ptr[k]; q < t.A_.ptr[k + 1]; q++) key.push_back((int32_t)(t.A_.col[q] - k));
        cls[k] = classes.try_emplace(key, (int32_t)classes.size()).first->second;  // no node for known keys
      }
    }
    std::iota(old_of_new.begin(), old_of_new.end(), 0);
    parallel_stable_sort(old_of_new.begin(), old_of_new.end(), opt_.setup_threads,
                         [&](int32_t a, int32_t b) { return cls[a] < cls[b]; });
    for (int64_t p = 0; p < nf; p++) pos[old_of_new[p]] = (int32_t)p;
    A.append(
        nfp, nf, [&](int64_t p) { return alen_old(old_of_new[p]); },
        [&](int64_t p, int j, int32_t& c, double& v) {
          const int64_t q = t.A_.ptr[old_of_new[p]] + j;
          c = (int32_t)(roff + pos[t.A_.col[q]]);
          v = t.A_.val[q];
        },
        [&](int64_t p) { return (int32_t)(roff + p); }, true, opt_.setup_threads);
    auto erow = [&](int64_t p) { return (int64_t)t.free_edges_[old_of_new[p]]; };
    Ef.append(
        nfp, nf, [&](int64_t p) { return t.E_.ptr[erow(p) + 1] - t.E_.ptr[erow(p)]; },
        [&](int64_t p, int j, int32_t& c, double& v) {
          const int64_t q = t.E_.ptr[erow(p)] + j;
          c = (int32_t)(eoff + t.E_.col[q]);
          v = t.E_.val[q];
        },
        [&](int64_t) { return (int32_t)eoff; }, true, opt_.setup_threads);
    // SigMat rows of the free edges (empty for a member without conducting
    // tets), in the rows' order, for the right-hand side
    const bool sig = t.lossy_;
    lossy[s] = sig ? 1 : 0;
    Sg.append(
        nfp, nf, [&](int64_t p) { return sig ? t.Sig_.ptr[erow(p) + 1] - t.Sig_.ptr[erow(p)] : (int64_t)0; },
        [&](int64_t p, int j, int32_t& c, double& v) {
          const int64_t q = t.Sig_.ptr[erow(p)] + j;
          c = (int32_t)(eoff + t.Sig_.col[q]);
          v = t.Sig_.val[q];
        },
        [&](int64_t) { return (int32_t)eoff; }, true, opt_.setup_threads);
    if (sig) {
      // every edge's SigMat row, in edge order, for the Joule losses
      const int64_t NEp = up32(NE);
      Sa.append(
          NEp, NE, [&](int64_t e) { return t.Sig_.ptr[e + 1] - t.Sig_.ptr[e]; },
          [&](int64_t e, int j, int32_t& c, double& v) {
            const int64_t q = t.Sig_.ptr[e] + j;
            c = (int32_t)(eoff + t.Sig_.col[q]);
            v = t.Sig_.val[q];
          },
          [&](int64_t) { return (int32_t)eoff; }, true, opt_.setup_threads);
      for (int64_t e = 0; e < NEp; e++) sa_edge.push_back(e < NE ? (int32_t)(eoff + e) : -1);
      sa_slice_sim.insert(sa_slice_sim.end(), NEp / 32, (uint16_t)s);
    }
    Ct.append(
        nfp, nf, [&](int64_t p) { return t.Ct_.ptr[erow(p) + 1] - t.Ct_.ptr[erow(p)]; },
        [&](int64_t p, int j, int32_t& c, double& v) {
          const int64_t q = t.Ct_.ptr[erow(p)] + j;
          c = (int32_t)(foff + t.Ct_.col[q]);
          if (t.Ct_.val[q] < 0) c = (int32_t)((uint32_t)c | 0x80000000u);
          v = 0.0;
        },
        [&](int64_t) { return kPadCol; }, false, opt_.setup_threads);
    N.append(
        NFp, NF, [&](int64_t f) { return t.N_.ptr[f + 1] - t.N_.ptr[f]; },
        [&](int64_t f, int j, int32_t& c, double& v) {
          const int64_t q = t.N_.ptr[f] + j;
          c = (int32_t)(foff + t.N_.col[q]);
          v = t.N_.val[q];
        },
        [&](int64_t f) { return (int32_t)(foff + f); }, true, opt_.setup_threads);
    const int nth = opt_.setup_threads;
    const size_t f0 = fte.size(), r0 = pre.size(), e0 = U0.size();
    fte.resize(f0 + 3 * (size_t)NFp);
    pre.resize(r0 + nfp);
    free_edge.resize(r0 + nfp);
    U0.resize(e0 + NE);
    I0.resize(e0 + NE);
    Src0.resize(e0 + NE);
    parallel_for(NFp, nth, [&](int64_t a0, int64_t a1) {
      for (int64_t f = a0; f < a1; f++)
        for (int k = 0; k < 3; k++) fte[f0 + 3 * f + k] = f < NF ? (int32_t)(eoff + t.fte_[f][k]) : -1;
    });
    parallel_for(nfp, nth, [&](int64_t a0, int64_t a1) {
      for (int64_t p = a0; p < a1; p++) {
        pre[r0 + p] = p < nf ? (T)t.jacobi_[old_of_new[p]] : (T)0;
        free_edge[r0 + p] = p < nf ? (int32_t)(eoff + t.free_edges_[old_of_new[p]]) : -1;
      }
    });
    parallel_for(NE, nth, [&](int64_t a0, int64_t a1) {
      for (int64_t e = a0; e < a1; e++) {
        U0[e0 + e] = (T)t.init_U_[e];
        I0[e0 + e] = (T)t.init_I_[e];
        Src0[e0 + e] = (T)t.init_src_[e];
      }
    });
    for (int32_t e : t.dir_edges_) dir_edge.push_back((int32_t)(eoff + e));
    slice_sim.insert(slice_sim.end(), nfp / 32, (uint16_t)s);
    fslice_sim.insert(fslice_sim.end(), NFp / 32, (uint16_t)s);
    dt[s] = t.dt_;
    fem[s] = t.method_ == 3 ? 1 : 0;
    tol[s] = t.sim_.tol;
    nsteps[s] = (int)t.nsteps_;
    // sources
    m.nsrc = t.src_labels_.size();
    nsrc[s] = (int)m.nsrc;
    src_off[s] = (int)src_amp.size();
    car_off[s] = (int64_t)carrier.size();
    m.car_off = car_off[s];
    sim_se[s] = (int)se_edge.size();
    const int pair_base = (int)pair_src.size();
    for (size_t k = 0; k < t.src_edge_.size(); k++) {
      se_edge.push_back((int32_t)(eoff + t.src_edge_[k]));
      se_kind.push_back(t.src_kind_e_[k]);
      se_begin.push_back(pair_base + t.src_begin_[k]);
      for (int a = 0; a < 3; a++) se_vec.push_back(t.src_vec_[3 * k + a]);
      se_post.push_back(t.src_post_[k]);
    }
    for (size_t p = 0; p < t.pair_src_.size(); p++) {
      pair_src.push_back(src_off[s] + t.pair_src_[p]);
      pair_dir.push_back(t.pair_dir_[p]);
      for (int a = 0; a < 4; a++) pair_fac.push_back(t.pair_fac_[4 * p + a]);
    }
    src_amp.insert(src_amp.end(), t.src_amp_.begin(), t.src_amp_.end());
    carrier.insert(carrier.end(), t.carrier_.begin(), t.carrier_.end());
    // probes
    m.np = t.probe_tet_.size();
    sim_probe[s] = (int)probe_sim.size();
    for (size_t p = 0; p < m.np; p++) {
      const int32_t v = t.probe_tet_[p];
      auto el = t.vol_edges(v);
      probe_sim.push_back(s);
      for (int q = 0; q < 6; q++) p_edges.push_back((int32_t)(eoff + el[q]));
      for (int q = 0; q < 4; q++) p_faces.push_back((int32_t)(foff + t.vtf_[v][q]));
      for (int q = 0; q < 18; q++) p_we.push_back(t.probe_we_[18 * p + q]);
      for (int q = 0; q < 12; q++) p_hf.push_back(t.probe_hf_[12 * p + q]);
    }
    m.nslots = t.nslots_;
    m.slot_of_step = t.slot_of_step_;
    m.sample_times = t.sample_times_;
    samp_off[s] = samp;
    m.samp_off = samp;
    samp += (int64_t)m.nslots * (int64_t)m.np * 6;
    sched_off[s] = (int64_t)sched.size();
    sched.insert(sched.end(), t.slot_of_step_.begin(), t.slot_of_step_.end());
    stat_off[s] = stat;
    m.stat_off = stat;
    stat += (int64_t)t.nsteps_ + 1;
    eoff += NE;
    foff += NFp;
    roff += nfp;
    if (eoff >= INT32_MAX || foff >= INT32_MAX || roff >= INT32_MAX)
      throw std::invalid_argument("simulation group exceeds 2^31 edges, faces or rows");
    if (release_host) t.release_host();
  }
  sim_se[S] = (int)se_edge.size();
  se_begin.push_back((int)pair_src.size());
  sim_probe[S] = (int)probe_sim.size();
  carrier_host_ = carrier;
  nnz_a_ = A.col.size();

  GroupDev& d = dev_;
  d.S = S;
  d.nE = eoff;
  d.nF = foff;
  d.nrow = roff;
  d.ndir = (int64_t)dir_edge.size();
  d.nse = (int64_t)se_edge.size();
  d.np = (int64_t)probe_sim.size();
  d.dt = (const double*)upload(dt);
  d.tol = (const double*)upload(tol);
  d.nsteps = (const int*)upload(nsteps);
  d.step = (int*)dalloc(sizeof(int) * S);
  CU(cudaMemset(d.step, 0, sizeof(int) * S));
  d.fslice_sim = (const uint16_t*)upload(fslice_sim);
  d.slice_sim = (const uint16_t*)upload(slice_sim);
  const size_t es = sizeof(T);
  auto zeros = [&](int64_t n) {
    void* p = dalloc((size_t)n * es);
    CU(cudaMemset(p, 0, (size_t)n * es));
    return p;
  };
  d.U = upload(U0);
  d.I = upload(I0);
  d.src = upload(Src0);
  d.F = zeros(d.nF);
  d.B = zeros(d.nF);
  d.cb = zeros(d.nE);
  if (std::find(fem.begin(), fem.end(), 1) != fem.end()) {
    d.fem = (const uint8_t*)upload(fem);
    d.cu = zeros(d.nF);
    d.Uo = upload(U0);  // U_older = U_old = U at t = 0 (Discretization.hpp:1664-1665)
  }
  d.fte = (const int32_t*)upload(fte);
  auto put = [&](SellHost<T>& m, SellDev& o, bool values) {
    o.ptr = (const int64_t*)upload(m.ptr);
    o.col = (const int32_t*)upload(m.col);
    o.val = values ? upload(m.val) : nullptr;
    decltype(m.ptr)().swap(m.ptr);
    decltype(m.col)().swap(m.col);
    decltype(m.val)().swap(m.val);
  };
  put(N, d.N, true);
  put(Ef, d.Ef, true);
  lossy_host_.assign(lossy.begin(), lossy.end());
  if (std::find(lossy.begin(), lossy.end(), 1) != lossy.end()) {
    // conducting members: SigMat terms of the right-hand side, and the
    // Joule-loss reduction over every edge's row
    put(Sg, d.Sg, true);
    put(Sa, d.Sa, true);
    d.lossy = (const uint8_t*)upload(lossy);
    d.nsa = (int64_t)sa_edge.size();
    d.sa_edge = (const int32_t*)upload(sa_edge);
    d.sa_slice_sim = (const uint16_t*)upload(sa_slice_sim);
    d.loss_part = (double*)dalloc(sizeof(double) * (size_t)(d.nsa / 32));
    std::vector<int> sim_sa(S + 1, 0);
    for (uint16_t q : sa_slice_sim) sim_sa[q + 1]++;
    for (int q = 0; q < S; q++) sim_sa[q + 1] += sim_sa[q];
    d.sim_sa = (const int*)upload(sim_sa);
  }
  put(Ct, d.Ct, false);
  put(A, d.A, true);
  d.pre = upload(pre);
  d.free_edge = (const int32_t*)upload(free_edge);
  d.dir_edge = (const int32_t*)upload(dir_edge);
  d.x = zeros(d.nrow);
  d.r = zeros(d.nrow);
  d.z = zeros(d.nrow);
  d.p0 = zeros(d.nrow);
  d.p1 = zeros(d.nrow);
  d.q = zeros(d.nrow);
  d.rhs = zeros(d.nrow);
  if (opt_.warm_start == 2 || opt_.warm_start == 3) {
    d.xh1 = zeros(d.nrow);
    d.xh2 = zeros(d.nrow);
    d.xh3 = zeros(d.nrow);
  }
  if (opt_.warm_start == 3) {
    d.xe = zeros(d.nrow);
    d.r_alt = zeros(d.nrow);
    d.z_alt = zeros(d.nrow);
    d.kept = (int8_t*)dalloc((size_t)stat);
    CU(cudaMemset(d.kept, 0, (size_t)stat));
    // sampled rows: every samp_stride-th free row, the first one rotating
    // through the stride from step to step
    samp_stride_ = std::max<int64_t>(1, d.nrow / std::max(1, opt_.learn_samples));
    samp_n_ = (d.nrow + samp_stride_ - 1) / samp_stride_;
    auto fz = [&](int64_t n) {
      float* p = (float*)dalloc(sizeof(float) * (size_t)std::max<int64_t>(n, 1));
      CU(cudaMemset(p, 0, sizeof(float) * (size_t)std::max<int64_t>(n, 1)));
      return p;
    };
    d.samp_in = fz(6 * samp_n_);
    d.samp_e = fz(samp_n_);
    d.samp_s = fz(samp_n_);
    d.samp_t = fz(samp_n_);
    d.samp_w = fz(samp_n_);
    d.samp_row = (int32_t*)dalloc(sizeof(int32_t) * (size_t)samp_n_);
    CU(cudaMemset(d.samp_row, 0xff, sizeof(int32_t) * (size_t)samp_n_));
    mlp_.max_blocks = (int)((samp_n_ + mlp_train_rows_per_block() - 1) / mlp_train_rows_per_block());
    std::vector<float> p0(kNParam);
    mlp_init_params(p0.data(), 0x5EEDF00Dull);
    mlp_.params = (float*)upload(p0);
    mlp_.adam_m = fz(kNParam);
    mlp_.adam_v = fz(kNParam);
    mlp_.image = (unsigned char*)dalloc(kImgBytes);
    mlp_.grad_part = fz((int64_t)mlp_.max_blocks * kNParam);
    mlp_.loss_part = fz(mlp_.max_blocks);
    mlp_.grad = fz(kNParam);
    mlp_.loss = fz(1);
    CU(mlp_launch_pack(mlp_.params, mlp_.image, stream_));
    d.mlp_img = mlp_.image;
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    d.guess_blocks = 3 * sms;
    d.tc_blocks = opt_.precision == 1 ? group_guess_tc_blocks<float>(opt_.device)
                                      : group_guess_tc_blocks<double>(opt_.device);
    loss_cap_ = (int64_t)std::max(1, opt_.learn_steps) * std::max(1, opt_.learn_inner);
    loss_hist_ = fz(loss_cap_);
  }
  d.cg_maxiter = opt_.cg_maxiter > 0 ? opt_.cg_maxiter : 100;
  d.cg_criterion = opt_.cg_criterion;
  d.warm_start = opt_.warm_start;
  d.cg_iters = (int32_t*)dalloc(sizeof(int32_t) * stat);
  d.cg_resid = (double*)dalloc(sizeof(double) * stat);
  d.cg_limit = (int32_t*)dalloc(sizeof(int32_t) * stat);
  d.flux = (double*)dalloc(sizeof(double) * stat);
  CU(cudaMemset(d.cg_iters, 0, sizeof(int32_t) * stat));
  CU(cudaMemset(d.cg_resid, 0, sizeof(double) * stat));
  CU(cudaMemset(d.cg_limit, 0, sizeof(int32_t) * stat));
  CU(cudaMemset(d.flux, 0, sizeof(double) * stat));
  if (d.lossy) {
    d.loss_a = (double*)dalloc(sizeof(double) * stat);
    CU(cudaMemset(d.loss_a, 0, sizeof(double) * stat));
  }
  d.stat_off = (const int64_t*)upload(stat_off);
  d.sim_se = (const int*)upload(sim_se);
  d.se_edge = (const int32_t*)upload(se_edge);
  d.se_kind = (const int8_t*)upload(se_kind);
  d.se_begin = (const int*)upload(se_begin);
  d.pair_src = (const int*)upload(pair_src);
  d.pair_fac = (const double*)upload(pair_fac);
  d.pair_dir = (const int8_t*)upload(pair_dir);
  d.se_vec = (const double*)upload(se_vec);
  d.se_post = (const double*)upload(se_post);
  d.src_amp = (const double*)upload(src_amp);
  d.carrier = (const double*)upload(carrier);
  d.car_off = (const int64_t*)upload(car_off);
  d.nsrc = (const int*)upload(nsrc);
  d.src_off = (const int*)upload(src_off);
  d.probe_sim = (const int*)upload(probe_sim);
  d.sim_probe = (const int*)upload(sim_probe);
  d.p_edges = (const int32_t*)upload(p_edges);
  d.p_faces = (const int32_t*)upload(p_faces);
  d.p_we = (const double*)upload(p_we);
  d.p_hf = (const double*)upload(p_hf);
  d.samples = (double*)dalloc(sizeof(double) * (size_t)std::max<int64_t>(samp, 1));
  d.samp_off = (const int64_t*)upload(samp_off);
  d.sched = (const int*)upload(sched);
  d.sched_off = (const int64_t*)upload(sched_off);
  cg_blocks_ = opt_.precision == 1 ? group_cg_blocks<float>(opt_.device, S, &cg_smem_)
                                   : group_cg_blocks<double>(opt_.device, S, &cg_smem_);
  if (cg_blocks_ < 1) throw CudaError("no co-resident blocks for the cooperative CG kernel");
  partition();
  // step_io staging: every member's carrier values of a step in one
  // contiguous H2D buffer, every member's exported sample in one D2H buffer
  std::vector<int> io_src_sim, io_in_off(S + 1, 0);
  std::vector<int64_t> io_out_off(S + 1, 0);
  for (int q = 0; q < S; q++) {
    const Meta& m = meta_[q];
    io_in_off[q + 1] = io_in_off[q] + (int)m.nsrc;
    io_out_off[q + 1] = io_out_off[q] + 6 * (int64_t)m.np;
    io_src_sim.insert(io_src_sim.end(), m.nsrc, q);
  }
  io_src_ = (size_t)io_in_off[S];
  io_probe_ = (size_t)io_out_off[S];
  d.n_io_in = (int64_t)io_src_;
  d.io_src_sim = (const int*)upload(io_src_sim);
  d.io_in_off = (const int*)upload(io_in_off);
  d.io_out_off = (const int64_t*)upload(io_out_off);
  dio_in_ = (double*)dalloc(sizeof(double) * std::max<size_t>(io_src_, 1));
  dio_out_ = (double*)dalloc(sizeof(double) * std::max<size_t>(io_probe_, 1));
  const size_t mp = io_src_ + io_probe_ + 1;
  pinned_len_ = mp;
  CU(cudaHostAlloc((void**)&pinned_, mp * sizeof(double), cudaHostAllocDefault));
  CU(cudaDeviceSynchronize());
}

#ifndef TF_CG_MIX
#define TF_CG_MIX 1
#endif
#ifndef TF_CG_CHUNKS
#define TF_CG_CHUNKS 12
#endif

// The CG blocks' rows.  A group of several members: chunks of each member's
// slices dealt to the blocks by work (below).  A single simulation:
// contiguous slice ranges of about equal work (stored entries of A plus the
// vector passes).  Either way a block's rows form segments of one member
// each, the unit of the partial sums.  The block count follows the problem
// size (at most one slice per warp and pass) so that small systems keep
// their grid barriers cheap.
void TetGroup::partition() {
  GroupDev& d = dev_;
  const int64_t nslice = d.nrow / 32;
  std::vector<int64_t> aptr(nslice + 1);
  CU(cudaMemcpy(aptr.data(), d.A.ptr, sizeof(int64_t) * (nslice + 1), cudaMemcpyDeviceToHost));
  std::vector<uint16_t> ssim(nslice);
  if (nslice) CU(cudaMemcpy(ssim.data(), d.slice_sim, sizeof(uint16_t) * nslice, cudaMemcpyDeviceToHost));
  const int warps = opt_.precision == 1 ? cg_warps<float>() : cg_warps<double>();
  int64_t want = (nslice + warps - 1) / warps;
  int G = (int)std::max<int64_t>(1, std::min<int64_t>(cg_blocks_, want));
  std::vector<double> cum(nslice + 1, 0.0);
  for (int64_t s = 0; s < nslice; s++) cum[s + 1] = cum[s] + (double)((aptr[s + 1] - aptr[s]) >> 5) + 8.0;
  std::vector<int64_t> cut(G + 1, 0);
  cut[G] = nslice;
  for (int b = 1; b < G; b++) {
    const double target = cum[nslice] * b / G;
    cut[b] = std::lower_bound(cum.begin(), cum.end(), target) - cum.begin();
    cut[b] = std::max(cut[b], cut[b - 1]);
  }
  std::vector<int> blk_seg(G + 1, 0), seg_sim, sim_seg(d.S + 1, 0), seg_of;
  std::vector<int64_t> seg_s0, seg_s1;
  bool mixed = false;
#if TF_CG_MIX
  if (d.S > 1 && G > 1) {
    // Members converge after different numbers of iterations, and a block
    // whose rows all belong to converged members waits at the barriers.  So
    // every member's slices are cut into chunks of about K slices (segments,
    // numbered member by member) and the chunks are dealt to the blocks
    // largest first, each to the least loaded block: a block then holds
    // chunks of about a dozen members, and as members converge every block
    // loses a similar share of its work.
    const int64_t per = TF_CG_CHUNKS;  // chunks per block aimed at
    for (int64_t K = std::max<int64_t>(16, (nslice + per * G - 1) / (per * G));; K *= 2) {
      seg_sim.clear(); seg_s0.clear(); seg_s1.clear();
      for (int64_t a = 0; a < nslice;) {
        int64_t e = a;
        while (e < nslice && ssim[e] == ssim[a]) e++;
        const int64_t pieces = (e - a + K - 1) / K;
        for (int64_t q = 0; q < pieces; q++) {
          seg_sim.push_back(ssim[a]);
          seg_s0.push_back(a + (e - a) * q / pieces);
          seg_s1.push_back(a + (e - a) * (q + 1) / pieces);
        }
        a = e;
      }
      const int C = (int)seg_sim.size();
      std::vector<int> order(C);
      std::iota(order.begin(), order.end(), 0);
      auto work = [&](int c) { return cum[seg_s1[c]] - cum[seg_s0[c]]; };
      std::stable_sort(order.begin(), order.end(), [&](int a2, int b2) { return work(a2) > work(b2); });
      using Load = std::pair<double, int>;
      std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
      for (int b = 0; b < G; b++) heap.push({0.0, b});
      std::vector<std::vector<int>> mine(G);
      for (int c : order) {
        Load l = heap.top();
        heap.pop();
        mine[l.second].push_back(c);
        heap.push({l.first + work(c), l.second});
      }
      size_t most = 0;
      for (auto& v : mine) most = std::max(most, v.size());
      if ((int)most > kMaxSeg) continue;  // too many chunks for a block's partial slots: coarser chunks
      seg_of.clear();
      for (int b = 0; b < G; b++) {
        std::sort(mine[b].begin(), mine[b].end());
        blk_seg[b] = (int)seg_of.size();
        seg_of.insert(seg_of.end(), mine[b].begin(), mine[b].end());
      }
      mixed = true;
      break;
    }
  }
#endif
  if (!mixed) {
    seg_sim.clear(); seg_s0.clear(); seg_s1.clear();
    for (int b = 0; b < G; b++) {
      blk_seg[b] = (int)seg_sim.size();
      int64_t s = cut[b];
      while (s < cut[b + 1]) {
        int64_t e = s;
        while (e < cut[b + 1] && ssim[e] == ssim[s]) e++;
        seg_sim.push_back(ssim[s]);
        seg_s0.push_back(s);
        seg_s1.push_back(e);
        s = e;
      }
      if ((int)seg_sim.size() - blk_seg[b] > kMaxSeg)
        throw std::invalid_argument("CG block spans more than " + std::to_string(kMaxSeg) + " simulations");
    }
    seg_of.resize(seg_sim.size());
    std::iota(seg_of.begin(), seg_of.end(), 0);
  }
  blk_seg[G] = (int)seg_of.size();
  // segments of a simulation are consecutive
  for (size_t g = 0; g < seg_sim.size(); g++) sim_seg[seg_sim[g] + 1]++;
  for (int s = 0; s < d.S; s++) sim_seg[s + 1] += sim_seg[s];
  for (size_t g = 1; g < seg_sim.size(); g++)
    if (seg_sim[g] < seg_sim[g - 1]) throw std::logic_error("CG segments out of simulation order");
  cg_blocks_ = G;
  blk_seg_.assign(blk_seg.begin(), blk_seg.end());
  d.blk_seg = (const int*)upload(blk_seg);
  d.seg_of = (const int*)upload(seg_of);
  d.seg_sim = (const int*)upload(seg_sim);
  d.seg_s0 = (const int64_t*)upload(seg_s0);
  d.seg_s1 = (const int64_t*)upload(seg_s1);
  d.sim_seg = (const int*)upload(sim_seg);
  d.part = (double*)dalloc(sizeof(double) * kCgPart * std::max<size_t>(seg_sim.size(), 1));
  d.gbar = (unsigned int*)dalloc(2 * sizeof(unsigned int));
  d.err = (int*)dalloc(sizeof(int));
  CU(cudaMemset(d.gbar, 0, 2 * sizeof(unsigned int)));
  CU(cudaMemset(d.err, 0, sizeof(int)));
}

// A grid-barrier timeout in the CG kernel leaves the step's results invalid:
// report it (and reset the barrier so the group can be closed cleanly).
void TetGroup::check_err() {
  int e = 0;
  CU(cudaMemcpy(&e, dev_.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (!e) return;
  CU(cudaMemset(dev_.err, 0, sizeof(int)));
  CU(cudaMemset(dev_.gbar, 0, 2 * sizeof(unsigned int)));
  throw CudaError("CG kernel: a grid barrier wait ran out of time; the step's results are not valid");
}

void TetGroup::launch(int n, cudaEvent_t* ev) {
  const bool f32 = opt_.precision == 1;
  for (int k = 0; k < n; k++) {
    const bool learned = opt_.warm_start == 3;
    const bool training = learned && launched_ < opt_.learn_steps;
    if (learned) {
      dev_.mlp_on = training ? 0 : 1;
      dev_.dual = training ? 0 : 1;
      dev_.nsamp = training ? samp_n_ : 0;
      dev_.samp_stride = samp_stride_;
      dev_.samp_first = launched_ % samp_stride_;
    }
    cudaError_t e = f32 ? group_launch_step<float>(dev_, cg_blocks_, cg_variant_, cg_smem_, stream_, ev)
                        : group_launch_step<double>(dev_, cg_blocks_, cg_variant_, cg_smem_, stream_, ev);
    CU(e);
    if (training) {
      // the step's solutions are the training targets of its sampled rows
      CU(f32 ? group_launch_targets<float>(dev_, stream_) : group_launch_targets<double>(dev_, stream_));
      for (int q = 0; q < std::max(1, opt_.learn_inner); q++) {
        CU(mlp_launch_train(mlp_, dev_.samp_in, dev_.samp_t, dev_.samp_w, (int)samp_n_, ++adam_step_,
                            opt_.learn_rate, stream_));
        if (adam_step_ - 1 < loss_cap_)
          CU(cudaMemcpyAsync(loss_hist_ + adam_step_ - 1, mlp_.loss, sizeof(float), cudaMemcpyDeviceToDevice,
                             stream_));
      }
    }
    launched_++;
  }
}

uint64_t TetGroup::step(uint64_t n) {
  uint64_t left = 0;
  for (const Meta& m : meta_) left = std::max(left, m.nsteps - m.step);
  n = std::min(n, left);
  if (n == 0) {
    last_ms_ = 0;
    return 0;
  }
  float total = 0;
  uint64_t done = 0;
  // the first steps alternate the two CG variants (bitwise identical
  // iterates) and keep the one with the smaller total CG time
  while (done < n && tune_pos_ < kTuneSteps) {
    cudaEvent_t ev[6];
    for (auto& e : ev) CU(cudaEventCreate(&e));
    cg_variant_ = tune_pos_ & 1;
    launch(1, ev);
    CU(cudaEventSynchronize(ev[5]));
    float a = 0, c = 0;
    CU(cudaEventElapsedTime(&a, ev[2], ev[3]));
    CU(cudaEventElapsedTime(&c, ev[0], ev[5]));
    if (tune_pos_ >= 2) tune_ms_[cg_variant_] += a;  // first pair is warm-up
    total += c;
    for (auto& e : ev) cudaEventDestroy(e);
    tune_pos_++;
    done++;
    if (tune_pos_ == kTuneSteps) cg_variant_ = tune_ms_[0] <= tune_ms_[1] ? 0 : 1;
  }
  if (done < n) {
    uint64_t rest = n - done;
    // Once the CG variant is chosen and the network (if any) has finished
    // training, every step launches the same kernels with the same
    // arguments (per-step state lives in device memory), so runs of
    // graph_len_ steps replay one captured CUDA graph.  A capture this call
    // will replay is made before the timed region opens (the device idles
    // while the host captures and instantiates).
    const int glen = opt_.graph_steps > 0 ? opt_.graph_steps : 16;
    if (glen > 1 && rest >= (uint64_t)glen && !graph_exec_ && !graph_failed_ &&
        !(opt_.warm_start == 3 && launched_ < opt_.learn_steps))
      capture_graph(glen);
    CU(cudaEventRecord(ev0_, stream_));
    while (rest > 0) {
      const bool training = opt_.warm_start == 3 && launched_ < opt_.learn_steps;
      if (glen > 1 && rest >= (uint64_t)glen && !training && !graph_failed_) {
        if (!graph_exec_) capture_graph(glen);
        if (graph_exec_) {
          CU(cudaGraphLaunch(graph_exec_, stream_));
          launched_ += glen;
          rest -= glen;
          continue;
        }
      }
      launch(1, nullptr);
      rest--;
    }
    CU(cudaEventRecord(ev1_, stream_));
    CU(cudaEventSynchronize(ev1_));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, ev0_, ev1_));
    total += ms;
  }
  last_ms_ = total;
  for (Meta& m : meta_) m.step = std::min(m.nsteps, m.step + n);
  check_err();
  return n;
}

// Captures `len` steps of kernel launches into graph_exec_.  A capture that
// the runtime refuses leaves graph_exec_ null and graph_failed_ set; the
// steps are then launched one by one (same kernels, same results).
void TetGroup::capture_graph(int len) {
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    graph_failed_ = true;
    return;
  }
  const int64_t before = launched_;
  bool ok = true;
  try {
    launch(len, nullptr);
  } catch (const CudaError&) {
    ok = false;  // a launch the capture refused; end the capture below
  }
  launched_ = before;  // captured, not run
  cudaError_t e = cudaStreamEndCapture(stream_, &g);
  if (!ok && e == cudaSuccess) e = cudaErrorStreamCaptureInvalidated;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&graph_exec_, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    graph_exec_ = nullptr;
    graph_failed_ = true;
    return;
  }
  graph_len_ = len;
}

uint64_t TetGroup::phase_times(uint64_t n, double* ms5) {
  uint64_t left = 0;
  for (const Meta& m : meta_) left = std::max(left, m.nsteps - m.step);
  n = std::min(n, left);
  for (int q = 0; q < 5; q++) ms5[q] = 0;
  cudaEvent_t ev[6];
  for (auto& e : ev) CU(cudaEventCreate(&e));
  for (uint64_t i = 0; i < n; i++) {
    launch(1, ev);
    CU(cudaEventSynchronize(ev[5]));
    for (int q = 0; q < 5; q++) {
      float ms = 0;
      CU(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
      ms5[q] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (Meta& m : meta_) m.step = std::min(m.nsteps, m.step + n);
  check_err();
  return n;
}

uint64_t TetGroup::step_io(const double* car_in, double* probe_out) {
  uint64_t left = 0;
  for (const Meta& m : meta_) left = std::max(left, m.nsteps - m.step);
  if (left == 0) return 0;
  double* hin = pinned_;
  double* hout = pinned_ + io_src_;
  // one copy each way: the carriers land in a staging buffer that a kernel
  // writes into each running member's carrier row of this step, and the
  // probe kernel writes this step's samples to a contiguous staging buffer
  if (car_in && io_src_) {
    std::memcpy(hin, car_in, io_src_ * sizeof(double));
    CU(cudaMemcpyAsync(dio_in_, hin, io_src_ * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CU(group_launch_io_carriers(dev_, dio_in_, stream_));
  }
  std::vector<char> got(meta_.size(), 0);
  bool any = false;
  for (size_t s = 0; s < meta_.size(); s++) {
    const Meta& m = meta_[s];
    const int slot = m.step < m.nsteps ? m.slot_of_step[m.step] : -1;
    got[s] = probe_out && slot >= 0 && m.np ? 1 : 0;
    any = any || got[s];
  }
  dev_.io_out = any ? dio_out_ : nullptr;
  launch(1, nullptr);
  dev_.io_out = nullptr;
  if (any) CU(cudaMemcpyAsync(hout, dio_out_, io_probe_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  size_t o = 0;
  for (size_t s = 0; s < meta_.size(); s++) {
    if (got[s]) std::memcpy(probe_out + o, hout + o, meta_[s].np * 6 * sizeof(double));
    o += meta_[s].np * 6;
  }
  for (Meta& m : meta_) m.step = std::min(m.nsteps, m.step + 1);
  check_err();
  return 1;
}

size_t TetGroup::n_samples(int s) const {
  const Meta& m = meta_[s];
  size_t c = 0;
  for (uint64_t i = 0; i < m.step && i < m.slot_of_step.size(); i++)
    if (m.slot_of_step[i] >= 0) c++;
  return c;
}

void TetGroup::get_probes(int s, double* times, double* values, size_t cap) const {
  const Meta& m = meta_[s];
  size_t ns = std::min(n_samples(s), cap);
  if (times) std::memcpy(times, m.sample_times.data(), ns * 8);
  if (values && ns && m.np)
    CU(cudaMemcpy(values, dev_.samples + m.samp_off, ns * m.np * 6 * 8, cudaMemcpyDeviceToHost));
}

static void fetch_range(const void* base, int64_t off, size_t n, bool f32, double* out) {
  if (!out || !n) return;
  if (!f32) {
    CU(cudaMemcpy(out, (const double*)base + off, n * 8, cudaMemcpyDeviceToHost));
    return;
  }
  std::vector<float> tmp(n);
  CU(cudaMemcpy(tmp.data(), (const float*)base + off, n * 4, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; i++) out[i] = tmp[i];
}

void TetGroup::get_state(int s, double* U, double* B, double* F) {
  const Meta& m = meta_[s];
  const bool f32 = opt_.precision == 1;
  CU(cudaStreamSynchronize(stream_));
  fetch_range(dev_.U, m.eoff, m.nE, f32, U);
  fetch_range(dev_.B, m.foff, m.nF, f32, B);
  fetch_range(dev_.F, m.foff, m.nF, f32, F);
}

void TetGroup::set_state(int s, const double* U, const double* F) {
  const Meta& m = meta_[s];
  const bool f32 = opt_.precision == 1;
  auto put = [&](void* base, int64_t off, const double* src, size_t n) {
    if (!src) return;
    if (!f32) CU(cudaMemcpy((double*)base + off, src, n * 8, cudaMemcpyHostToDevice));
    else {
      std::vector<float> t(src, src + n);
      CU(cudaMemcpy((float*)base + off, t.data(), n * 4, cudaMemcpyHostToDevice));
    }
  };
  CU(cudaStreamSynchronize(stream_));
  put(dev_.U, m.eoff, U, m.nE);
  put(dev_.F, m.foff, F, m.nF);
}

size_t TetGroup::solver_stats(int s, int32_t* iters, double* resid, size_t cap) const {
  const Meta& m = meta_[s];
  const size_t n = std::min<size_t>(m.step, cap);
  if (iters && n) CU(cudaMemcpy(iters, dev_.cg_iters + m.stat_off, n * 4, cudaMemcpyDeviceToHost));
  if (resid && n) CU(cudaMemcpy(resid, dev_.cg_resid + m.stat_off, n * 8, cudaMemcpyDeviceToHost));
  return m.step;
}

size_t TetGroup::guess_stats(int s, int8_t* kept, size_t cap) const {
  const Meta& m = meta_[s];
  if (!dev_.kept) return 0;
  const size_t n = std::min<size_t>(m.step, cap);
  if (kept && n) CU(cudaMemcpy(kept, dev_.kept + m.stat_off, n, cudaMemcpyDeviceToHost));
  return m.step;
}

double TetGroup::energy(int s) {
  constexpr int kBlocks = 592;  // 4 x 148 SMs
  if (!energy_part_) energy_part_ = (double*)dalloc(kBlocks * sizeof(double));
  const Meta& m = meta_[s];
  cudaError_t e = opt_.precision == 1
                      ? group_launch_energy<float>(dev_, s, m.roff, m.nrow_pad, m.foff, m.nface_pad, energy_part_,
                                                   kBlocks, stream_)
                      : group_launch_energy<double>(dev_, s, m.roff, m.nrow_pad, m.foff, m.nface_pad, energy_part_,
                                                    kBlocks, stream_);
  CU(e);
  std::vector<double> h(kBlocks);
  CU(cudaMemcpyAsync(h.data(), energy_part_, kBlocks * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  double w = 0.0;
  for (double x : h) w += x;
  return w;
}

size_t TetGroup::training_loss(float* loss, size_t cap) const {
  if (!loss_hist_) return 0;
  const size_t have = (size_t)std::min<int64_t>(adam_step_, loss_cap_);
  const size_t n = std::min(have, cap);
  if (loss && n) CU(cudaMemcpy(loss, loss_hist_, n * sizeof(float), cudaMemcpyDeviceToHost));
  return have;
}

bool TetGroup::mlp_params(float* out) const {
  if (!mlp_.params) return false;
  if (out) CU(cudaMemcpy(out, mlp_.params, sizeof(float) * kNParam, cudaMemcpyDeviceToHost));
  return true;
}

// poynting.dat's third column for gfdtd and fem (Discretization.hpp
// :1518-1546, :1733-1757): the reference pushes 0.5 a_{i-1} before the solve
// of step i and, from step 2 on, a_i after it, with a_j = U_j^T SigMat U_j,
// and prints the first n entries: 0.5 a_0, then 0.5 a_{(k+1)/2} for odd k and
// a_{k/2+1} for even k.  a_{j} is formed at the start of step j + 1.
void TetGroup::get_losses(int s, double* loss, size_t cap, size_t* n) const {
  const Meta& m = meta_[s];
  const size_t k = (size_t)m.step;
  if (n) *n = k;
  if (!loss) return;
  const size_t w = std::min(k, cap);
  if (!dev_.loss_a || !dev_.lossy || !lossy_host_[s]) {
    std::fill(loss, loss + w, 0.0);
    return;
  }
  std::vector<double> a(k);
  if (k) CU(cudaMemcpy(a.data(), dev_.loss_a + m.stat_off, k * 8, cudaMemcpyDeviceToHost));
  for (size_t q = 0; q < w; q++) {
    const size_t j = q == 0 ? 0 : (q % 2 ? (q + 1) / 2 : q / 2 + 1);
    loss[q] = (q == 0 || q % 2) ? 0.5 * a[j] : a[j];
  }
}

void TetGroup::get_flux(int s, double* flux, size_t cap, size_t* n) const {
  const Meta& m = meta_[s];
  const size_t k = std::min<size_t>(m.step, cap);
  if (flux && k) CU(cudaMemcpy(flux, dev_.flux + m.stat_off, k * 8, cudaMemcpyDeviceToHost));
  if (n) *n = m.step;
}

template void TetGroup::build<float>(std::vector<TetSim*>&, bool);
template void TetGroup::build<double>(std::vector<TetSim*>&, bool);

}  // namespace tf
