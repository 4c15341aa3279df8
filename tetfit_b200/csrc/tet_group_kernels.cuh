// Device layout of a group of gfdtd simulations advanced together.
//
// A group holds S >= 1 independent tetrahedral simulations (their own mesh,
// materials, sources, time step and probes) concatenated in one device image:
//
//   edges      per-simulation ranges, unpadded (eoff[s])
//   faces      per-simulation ranges padded to 32 faces; fslice_sim[f >> 5]
//              names the simulation of a face; padding faces have fte = -1
//   free rows  the CG unknowns (free edges) of every simulation, each range
//              padded to 32 rows and grouped by stencil class (rows with the
//              same column offsets side by side); slice_sim[i >> 5] names the
//              simulation, free_edge[i] the edge (-1 on padding rows)
//
// Matrices are SELL-32: a slice of 32 rows stores len = (ptr[s+1]-ptr[s])/32
// entries per row column-major (entry j of row lane l at ptr[s] + 32 j + l),
// so a warp's loads of one entry slot are one 128-byte transaction.  Entries
// keep the row order of the CSR they come from; padding entries point at the
// row itself with value 0 (Ct, which has no values, uses kPadCol).
//
// Per-simulation scalars (time step, step counter, tolerance) are indexed by
// the simulation id.  The CG kernel partitions the slices among its blocks in
// contiguous ranges; a block's range cut at simulation boundaries gives its
// segments, and every inner product is summed per segment, then per
// simulation in segment order, so results do not depend on timing.
#pragma once
#include <cstdint>

namespace tf {

constexpr int32_t kPadCol = 0x7fffffff;
// Threads of a CG block, per precision (FP32 blocks of 1024 threads, two
// per SM, ran the batch CG 2 % faster than four of 512; 256 and 128 were
// slower: the grid barrier's cost grows with the block count).
#ifndef TF_CG_THREADS32
#define TF_CG_THREADS32 1024
#endif
#ifndef TF_CG_THREADS64
#define TF_CG_THREADS64 512
#endif
#if defined(__CUDACC__)
#define TF_CG_HD __host__ __device__
#else
#define TF_CG_HD
#endif
template <typename T>
TF_CG_HD constexpr int cg_threads() { return sizeof(T) == 4 ? TF_CG_THREADS32 : TF_CG_THREADS64; }
template <typename T>
TF_CG_HD constexpr int cg_warps() { return cg_threads<T>() / 32; }
constexpr int kMaxSeg = 32;       // segments per CG block
constexpr int kMaxGroup = 1024;   // simulations per group
constexpr int kCgPart = 8;        // CG partial-sum slots per segment (three disjoint groups)

struct SellDev {
  const int64_t* ptr = nullptr;  // [nslice + 1]
  const int32_t* col = nullptr;
  const void* val = nullptr;     // T; nullptr for the sign-only C^T (sign in bit 31)
};

struct GroupDev {
  int S = 0;
  int64_t nE = 0, nF = 0, nrow = 0, ndir = 0, nse = 0, np = 0;
  // per simulation
  const double* dt = nullptr;
  const double* tol = nullptr;
  const int* nsteps = nullptr;
  int* step = nullptr;
  const uint16_t* fslice_sim = nullptr;
  const uint16_t* slice_sim = nullptr;
  // state (T)
  void *U = nullptr, *F = nullptr, *B = nullptr, *I = nullptr, *cb = nullptr, *src = nullptr;
  // method fem (central differences of the second-order equation): per
  // simulation flag, C U_old on the faces and U one step further back
  const uint8_t* fem = nullptr;
  void *cu = nullptr, *Uo = nullptr;
  // complex and operators
  const int32_t* fte = nullptr;  // [nF][3] global edges (signs +, -, +), -1 on padding faces
  SellDev N;                     // faces x faces
  SellDev Ef;                    // free rows x edges: eps-mass rows of the free edges
  SellDev Ct;                    // free rows x faces, +-1
  SellDev A;                     // free rows x free rows
  // conducting members (SigMat, gfdtd and fem): Sg the SigMat rows of the
  // free edges (empty rows for the other members) for the right-hand side;
  // Sa every edge's SigMat row of the conducting members, member by member
  // (32-row slices of one member, sa_edge the row's edge or -1), for the
  // per-step Joule-loss term a = U^T SigMat U into loss_a[stat_off + step]
  SellDev Sg, Sa;
  const uint8_t* lossy = nullptr;
  int64_t nsa = 0;
  const int32_t* sa_edge = nullptr;
  const uint16_t* sa_slice_sim = nullptr;
  const int* sim_sa = nullptr;   // [S + 1] first Sa slice of each member
  double* loss_part = nullptr;   // [nsa / 32] slice partials
  double* loss_a = nullptr;      // [stat]
  // step_io staging: io_out (when set) receives each member's sample of this
  // step at io_out_off[s]; the carriers of a step arrive contiguous, member
  // s's at io_in_off[s], io_src_sim[k] the member of entry k
  double* io_out = nullptr;
  const int64_t* io_out_off = nullptr;
  const int* io_in_off = nullptr;
  const int* io_src_sim = nullptr;
  int64_t n_io_in = 0;
  const void* pre = nullptr;     // Jacobi 1/diag (0 on padding rows)
  const int32_t* free_edge = nullptr;
  const int32_t* dir_edge = nullptr;
  // CG
  void *x = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr, *rhs = nullptr;
  void *xh1 = nullptr, *xh2 = nullptr, *xh3 = nullptr;
  const int* blk_seg = nullptr;  // [G + 1] block b's positions blk_seg[b] .. blk_seg[b+1] in seg_of
  const int* seg_of = nullptr;   // position -> segment (segments numbered member by member)
  const int* seg_sim = nullptr;
  const int64_t *seg_s0 = nullptr, *seg_s1 = nullptr;  // slice range of a segment
  const int* sim_seg = nullptr;  // [S + 1]
  double* part = nullptr;        // [nseg][kCgPart]
  unsigned int* gbar = nullptr;  // grid barrier: arrivals, generation
  int* err = nullptr;            // set when a grid barrier wait ran out of time
  int cg_maxiter = 100, cg_criterion = 0, warm_start = 0;
  // learned warm start (warm_start 3): the network's guess goes to x, the
  // quadratic extrapolation to xe; with dual set, the CG starts from the one
  // whose residual is smaller, per simulation (sel: extrapolation won), and
  // kept[stat_off + step] records 1 when the network's guess was kept
  void *xe = nullptr, *r_alt = nullptr, *z_alt = nullptr;
  int mlp_on = 0, dual = 0;
  int guess_blocks = 1;           // grid of the learned-guess kernel (a few blocks per SM)
  int tc_blocks = 1;              // grid of the tensor-core guess kernel (resident CTAs x SMs)
  int8_t* kept = nullptr;
  const unsigned char* mlp_img = nullptr;
  // training samples: rows i = samp_first + k * samp_stride, k < nsamp
  float *samp_in = nullptr, *samp_e = nullptr, *samp_s = nullptr, *samp_t = nullptr, *samp_w = nullptr;
  int32_t* samp_row = nullptr;
  int64_t nsamp = 0, samp_stride = 1, samp_first = 0;
  int32_t* cg_iters = nullptr;
  double* cg_resid = nullptr;
  int32_t* cg_limit = nullptr;
  const int64_t* stat_off = nullptr;  // per simulation: first entry of its per-step arrays
  // sources (simulation s owns source edges [sim_se[s], sim_se[s+1]))
  const int* sim_se = nullptr;
  const int32_t* se_edge = nullptr;
  const int8_t* se_kind = nullptr;
  const int* se_begin = nullptr;
  const int* pair_src = nullptr;     // global source index
  const double* pair_fac = nullptr;
  const int8_t* pair_dir = nullptr;
  const double *se_vec = nullptr, *se_post = nullptr;
  const double* src_amp = nullptr;
  const double* carrier = nullptr;   // simulation s: carrier[car_off[s] + step * nsrc[s] + local source]
  const int64_t* car_off = nullptr;
  const int* nsrc = nullptr;
  const int* src_off = nullptr;      // global index of the simulation's first source
  double* flux = nullptr;            // per simulation, per step (stat_off)
  // probes (simulation s owns probes [sim_probe[s], sim_probe[s+1]))
  const int* probe_sim = nullptr;
  const int* sim_probe = nullptr;
  const int32_t *p_edges = nullptr, *p_faces = nullptr;
  const double *p_we = nullptr, *p_hf = nullptr;
  double* samples = nullptr;
  const int64_t* samp_off = nullptr;
  const int* sched = nullptr;        // slot of each step, per simulation at sched_off[s]
  const int64_t* sched_off = nullptr;
};

template <typename T>
cudaError_t group_launch_step(const GroupDev& d, int cg_blocks, int cg_variant, size_t cg_smem, cudaStream_t st,
                              cudaEvent_t* ev);
template <typename T>
int group_cg_blocks(int device, int S, size_t* smem);
// step_io: this step's carrier values (staging, contiguous) into each
// running member's carrier row
cudaError_t group_launch_io_carriers(const GroupDev& d, const double* in, cudaStream_t st);
template <typename T>
int group_guess_tc_blocks(int device);
template <typename T>
cudaError_t group_launch_targets(const GroupDev& d, cudaStream_t st);
// Energy partials of member s (free rows [r0, r0 + nr), faces [f0, f0 + nf))
// into part[0 .. blocks).
template <typename T>
cudaError_t group_launch_energy(const GroupDev& d, int s, int64_t r0, int64_t nr, int64_t f0, int64_t nf,
                                double* part, int blocks, cudaStream_t st);

}  // namespace tf
