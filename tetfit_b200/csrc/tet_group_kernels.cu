// Kernels of a group of gfdtd simulations (Discretization.hpp:1459-1565 per
// simulation), all simulations advanced by the same launches:
//
//   grp_curl_u     B -= dt C U on the faces (3 signed edges per face)
//   grp_nmul       F = N B (SELL-32)
//   grp_probes     Whitney E and face-flux H at the probe points (:3768-3897)
//   grp_sources    one block per simulation: source-edge values from the
//                  carrier table, boundary flux of the step (:1478-1504)
//   grp_rhs        Psi = E (U_old - Src) - dt I + dt C^T F + dt Ctb Fb on the
//                  free rows (:1516-1523) and the CG initial guess
//   grp_cg         persistent cooperative Jacobi-PCG over every simulation's
//                  system at once (ConjugateGradientSolver.hpp:52-103), each
//                  simulation with its own scalars and stopping test
//   grp_scatter    U[free] = x, U[Dirichlet] = source values (:1540-1541)
//   grp_bump       step counters of the running simulations
//
// CG arithmetic.  Iteration j of the reference computes q = A p_j, alpha_j =
// rz / p_j.q, x += alpha_j p_j, r -= alpha_j q, z = pre r, beta = rz'/rz,
// p_{j+1} = z + beta p_j.  Here p alternates between two buffers, and the x
// update of iteration j is applied while p_{j+1} is formed (p_j is read there
// anyway), with one final update after the loop.  The residual phase stores
// z = pre r.  In the fused variant the SpMV forms p_{j+1} at every gathered
// column from (z, p_j) with the same explicitly rounded operation the row's
// owner uses, so p_{j+1} needs no barrier before the SpMV: two grid barriers
// per iteration instead of three.
// Both variants give bitwise identical iterates.
#include <cuda_runtime.h>

#include "grid_barrier.cuh"
#include "mlp.cuh"
#include "mlp_tc.cuh"
#include "tet_group_kernels.cuh"


namespace tf {

constexpr int kGB = 256;

__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mulT(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulT(double a, double b) { return __dmul_rn(a, b); }

__device__ __forceinline__ bool running(const GroupDev& d, int s) { return d.step[s] < d.nsteps[s]; }

// Loads of a matrix's index and value streams: each entry is read once per
// sweep, so they bypass L1 (read-only path, no L1 allocation) and leave it to
// the gathered vector entries, which neighbouring rows reuse.  Measured on a
// 64-member batch (11.3 M rows): 7 % (FP32) and 10 % (FP64) less time per CG
// iteration than plain read-only loads.
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) {
  int32_t v;
  asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// sum over the row's entries, in stored order, of val * g(col).  Entries
// are taken 4 at a time: the index and value loads of a chunk are all issued
// before its gathers, so a row costs about two memory latencies instead of
// one per entry group.
// The same sweep with the sum in A (values of type T read from the matrix):
// sell_dot<double>(m, row, g, (const float*)nullptr) sums FP32 entries in FP64.
#ifndef TF_SPMV_CH
#define TF_SPMV_CH 4
#endif
template <typename A, typename G, typename T, int CH = TF_SPMV_CH>
__device__ __forceinline__ A sell_dot(const SellDev& m, int64_t row, G g, const T*) {
  const int64_t sl = row >> 5;
  const int64_t b = m.ptr[sl];
  const int len = (int)((m.ptr[sl + 1] - b) >> 5);
  const int32_t* col = m.col + b + (row & 31);
  const T* val = (const T*)m.val + b + (row & 31);
  A s = 0;
  for (int j0 = 0; j0 < len; j0 += CH) {
    int32_t c[CH];
    T v[CH];
#pragma unroll
    for (int k = 0; k < CH; k++)
      if (j0 + k < len) {
        c[k] = ld_stream(col + 32 * (j0 + k));
        v[k] = ld_stream(val + 32 * (j0 + k));
      }
#pragma unroll
    for (int k = 0; k < CH; k++)
      if (j0 + k < len) s += (A)v[k] * g(c[k]);
  }
  return s;
}

template <typename T, typename G, int CH = TF_SPMV_CH>
__device__ __forceinline__ T sell_dot(const SellDev& m, int64_t row, G g) {
  const int64_t sl = row >> 5;
  const int64_t b = m.ptr[sl];
  const int len = (int)((m.ptr[sl + 1] - b) >> 5);
  const int32_t* col = m.col + b + (row & 31);
  const T* val = (const T*)m.val + b + (row & 31);
  T s = 0;
  for (int j0 = 0; j0 < len; j0 += CH) {
    int32_t c[CH];
    T v[CH];
#pragma unroll
    for (int k = 0; k < CH; k++)
      if (j0 + k < len) {
        c[k] = ld_stream(col + 32 * (j0 + k));
        v[k] = ld_stream(val + 32 * (j0 + k));
      }
#pragma unroll
    for (int k = 0; k < CH; k++)
      if (j0 + k < len) s += v[k] * g(c[k]);
  }
  return s;
}

#ifndef TF_CG_PIPE
#define TF_CG_PIPE 0
#endif
// The CG kernel's sweep over A.  TF_CG_PIPE 0: sell_dot.  1: software
// pipelined -- the index and value loads of chunk k + 1 are issued before the
// gathers of chunk k, so the matrix stream stays in flight while the gathers
// wait.  2: the whole row's index and value loads first (rows of up to 16
// entries), then its gathers.  Same entry order and arithmetic in all forms.
template <typename T, typename G>
__device__ __forceinline__ T sell_dot_cg(const SellDev& m, int64_t row, G g) {
#if TF_CG_PIPE == 0
  return sell_dot<T, G, 4>(m, row, g);  // 4-entry chunks: the CG's register budget
#elif TF_CG_PIPE == 1
  constexpr int CH = 4;
  const int64_t sl = row >> 5;
  const int64_t b = m.ptr[sl];
  const int len = (int)((m.ptr[sl + 1] - b) >> 5);
  const int32_t* col = m.col + b + (row & 31);
  const T* val = (const T*)m.val + b + (row & 31);
  T s = 0;
  int32_t c[CH];
  T v[CH];
#pragma unroll
  for (int k = 0; k < CH; k++)
    if (k < len) {
      c[k] = ld_stream(col + 32 * k);
      v[k] = ld_stream(val + 32 * k);
    }
  for (int j0 = 0; j0 < len; j0 += CH) {
    int32_t cn[CH];
    T vn[CH];
#pragma unroll
    for (int k = 0; k < CH; k++)
      if (j0 + CH + k < len) {
        cn[k] = ld_stream(col + 32 * (j0 + CH + k));
        vn[k] = ld_stream(val + 32 * (j0 + CH + k));
      }
#pragma unroll
    for (int k = 0; k < CH; k++)
      if (j0 + k < len) s += v[k] * g(c[k]);
#pragma unroll
    for (int k = 0; k < CH; k++) {
      c[k] = cn[k];
      v[k] = vn[k];
    }
  }
  return s;
#else
  constexpr int LM = 16;
  const int64_t sl = row >> 5;
  const int64_t b = m.ptr[sl];
  const int len = (int)((m.ptr[sl + 1] - b) >> 5);
  if (len > LM) return sell_dot<T>(m, row, g);
  const int32_t* col = m.col + b + (row & 31);
  const T* val = (const T*)m.val + b + (row & 31);
  int32_t c[LM];
  T v[LM];
#pragma unroll
  for (int k = 0; k < LM; k++)
    if (k < len) {
      c[k] = ld_stream(col + 32 * k);
      v[k] = ld_stream(val + 32 * k);
    }
  T s = 0;
#pragma unroll
  for (int k = 0; k < LM; k++)
    if (k < len) s += v[k] * g(c[k]);
  return s;
#endif
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// deterministic block sum of one double (all threads get the result)
__device__ double grp_block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) sh[32] = s;
  }
  __syncthreads();
  return sh[32];
}

template <typename T>
__global__ void __launch_bounds__(kGB) grp_curl_u(GroupDev d) {
  const int64_t f = (int64_t)blockIdx.x * kGB + threadIdx.x;
  if (f >= d.nF) return;
  const int s = d.fslice_sim[f >> 5];
  if (!running(d, s)) return;
  const int32_t* e = d.fte + 3 * f;
  const int32_t e0 = e[0];
  if (e0 < 0) return;
  const T* U = (const T*)d.U;
  const T c = U[e0] - U[e[1]] + U[e[2]];
  T* B = (T*)d.B;
  B[f] = B[f] - (T)d.dt[s] * c;
  if (d.fem && d.fem[s]) ((T*)d.cu)[f] = c;  // fem: C U_old for C^T N C U_old
}

template <typename T>
__global__ void __launch_bounds__(kGB) grp_nmul(GroupDev d) {
  const int64_t f = (int64_t)blockIdx.x * kGB + threadIdx.x;
  if (f >= d.nF) return;
  const int s = d.fslice_sim[f >> 5];
  if (!running(d, s)) return;
  // gfdtd: F = N B; fem: F = N C U_old (Discretization.hpp:1709-1711)
  const T* B = (const T*)(d.fem && d.fem[s] ? d.cu : d.B);
  ((T*)d.F)[f] = sell_dot<T>(d.N, f, [&](int32_t c) { return B[c]; });
}

// gfdtd exports U^{i-1} and B^{i-1/2} inside step i (Discretization.hpp:1469-1475)
template <typename T>
__global__ void grp_probes(GroupDev d) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.np) return;
  const int s = d.probe_sim[p];
  if (!running(d, s)) return;
  const int slot = d.sched[d.sched_off[s] + d.step[s]];
  if (slot < 0) return;
  const T* U = (const T*)d.U;
  const T* B = (const T*)d.B;
  double E[3] = {0, 0, 0}, H[3] = {0, 0, 0};
  for (int q = 0; q < 6; q++) {
    const double u = (double)U[d.p_edges[6 * p + q]];
    for (int a = 0; a < 3; a++) E[a] += d.p_we[18 * p + 3 * q + a] * u;
  }
  for (int q = 0; q < 4; q++) {
    const double b = (double)B[d.p_faces[4 * p + q]];
    for (int a = 0; a < 3; a++) H[a] += d.p_hf[12 * p + 3 * q + a] * b;
  }
  const int64_t nps = d.sim_probe[s + 1] - d.sim_probe[s];
  double* out = d.samples + d.samp_off[s] + ((int64_t)slot * nps + (p - d.sim_probe[s])) * 6;
  for (int a = 0; a < 3; a++) {
    out[a] = E[a];
    out[3 + a] = H[a];
  }
  if (d.io_out) {  // step_io: the same sample, contiguous per member
    double* o2 = d.io_out + d.io_out_off[s] + (p - d.sim_probe[s]) * 6;
    for (int a = 0; a < 3; a++) {
      o2[a] = E[a];
      o2[3 + a] = H[a];
    }
  }
}

__global__ void grp_io_carriers(GroupDev d, const double* in) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_io_in) return;
  const int s = d.io_src_sim[k];
  if (d.step[s] >= d.nsteps[s]) return;
  const_cast<double*>(d.carrier)[d.car_off[s] + (int64_t)d.step[s] * d.nsrc[s] + (k - d.io_in_off[s])] = in[k];
}

cudaError_t group_launch_io_carriers(const GroupDev& d, const double* in, cudaStream_t st) {
  if (d.n_io_in == 0) return cudaSuccess;
  grp_io_carriers<<<(unsigned)((d.n_io_in + 255) / 256), 256, 0, st>>>(d, in);
  return cudaGetLastError();
}

// One block per simulation.  E sources write the Dirichlet values, H sources
// the boundary dual-edge term, currents I; the step's flux sum is
// U_prev . 0.5 (Fb(t) + Fb(t - dt)) over the H-source edges.
template <typename T>
__global__ void __launch_bounds__(kGB) grp_sources(GroupDev d) {
  __shared__ double sh[33];
  const int s = blockIdx.x;
  if (!running(d, s)) return;
  const int step = d.step[s];
  const int ns = d.nsrc[s];
  const double* car = d.carrier + d.car_off[s];
  const int s0 = d.src_off[s];
  double fl = 0.0;
  for (int k = d.sim_se[s] + threadIdx.x; k < d.sim_se[s + 1]; k += kGB) {
    auto value = [&](int row) {
      double v[3] = {0.0, 0.0, 0.0};
      for (int p = d.se_begin[k]; p < d.se_begin[k + 1]; p++) {
        const int si = d.pair_src[p];
        double ret = d.src_amp[si] * car[(int64_t)row * ns + (si - s0)];
        ret *= d.pair_fac[4 * p + 0];
        ret *= d.pair_fac[4 * p + 1];
        ret *= d.pair_fac[4 * p + 2];
        ret *= d.pair_fac[4 * p + 3];
        v[d.pair_dir[p]] += ret;
      }
      const double* w = d.se_vec + 3 * (int64_t)k;
      return d.se_post[k] * ((v[0] * w[0] + v[1] * w[1]) + v[2] * w[2]);
    };
    const int e = d.se_edge[k];
    const int kind = d.se_kind[k];
    const double val = value(step);
    if (kind == 1) {
      ((T*)d.src)[e] = (T)val;
    } else if (kind == 2) {
      const double prev = step > 0 ? value(step - 1) : 0.0;
      // gfdtd: Ctb Fb; fem: Ctb (Fb - Fb_old) (Discretization.hpp:1713)
      ((T*)d.cb)[e] = (T)(d.fem && d.fem[s] ? val - prev : val);
      fl += (double)((const T*)d.U)[e] * (0.5 * (val + prev));
    } else if (kind == 3) {
      ((T*)d.I)[e] = (T)val;
    }
  }
  fl = grp_block_sum(fl, sh);
  if (threadIdx.x == 0) d.flux[d.stat_off[s] + step] = fl;
}

// Right-hand side on the free rows and the initial guess: 0 previous
// solution (x kept), 1 zero, 2 quadratic extrapolation from the last three
// solutions (history shifted here).
template <typename T>
__global__ void __launch_bounds__(kGB) grp_rhs(GroupDev d) {
  const int64_t i = (int64_t)blockIdx.x * kGB + threadIdx.x;
  if (i >= d.nrow) return;
  const int s = d.slice_sim[i >> 5];
  if (!running(d, s)) return;
  const int32_t e = d.free_edge[i];
  if (e < 0) return;
  const T* U = (const T*)d.U;
  const T* S = (const T*)d.src;
  const T* F = (const T*)d.F;
  const bool fem = d.fem && d.fem[s];
  const T* Uo = (const T*)d.Uo;
  // gfdtd: E U_old - RHSmat1 SrcFld; fem: E (2 U_old - U_older) - E_dir SrcFld
  // (the source values live on the Dirichlet columns only).  fem sums in
  // FP64: its right-hand side is dominated by E U / dt^2 terms whose
  // difference carries the update, so FP32 sums would lose it.
  double eu_fem = 0.0, su_fem = 0.0;
  if (fem)
    eu_fem = sell_dot<double>(d.Ef, i, [&](int32_t c) {
      return 2.0 * (double)U[c] - (double)Uo[c] - (double)S[c];
    }, (const T*)nullptr);
  T eu = fem ? (T)0 : sell_dot<T>(d.Ef, i, [&](int32_t c) { return U[c] - S[c]; });
  // conducting members: SysMat = scale E + coef SigMat, so the SigMat rows add
  // gfdtd  - (dt/2) SigMat U_old - (dt/2) SigMat_dir SrcFld   (:1516-1519)
  // fem    + (0.5/dt) SigMat U_older - (0.5/dt) SigMat_dir SrcFld   (:1729-1731)
  if (d.lossy && d.lossy[s]) {
    if (fem)
      su_fem = sell_dot<double>(d.Sg, i, [&](int32_t c) { return (double)Uo[c] - (double)S[c]; }, (const T*)nullptr);
    else
      eu -= (T)(0.5 * d.dt[s]) * sell_dot<T>(d.Sg, i, [&](int32_t c) { return U[c] + S[c]; });
  }
  // C^T F over the edge's faces in stored order; the face indices of 4
  // entries are loaded before their gathers (padding entries hold kPadCol
  // and add nothing)
  T cf = 0;
  {
    constexpr int CH = TF_SPMV_CH;
    const int64_t sl = i >> 5;
    const int64_t b = d.Ct.ptr[sl];
    const int len = (int)((d.Ct.ptr[sl + 1] - b) >> 5);
    const int32_t* col = d.Ct.col + b + (i & 31);
    for (int j0 = 0; j0 < len; j0 += CH) {
      int32_t c[CH];
#pragma unroll
      for (int k = 0; k < CH; k++) c[k] = j0 + k < len ? ld_stream(col + 32 * (j0 + k)) : kPadCol;
#pragma unroll
      for (int k = 0; k < CH; k++)
        if (c[k] != kPadCol) {
          const T v = F[c[k] & 0x7fffffff];
          cf = c[k] < 0 ? cf - v : cf + v;
        }
    }
  }
  const T dt = (T)d.dt[s];
  if (fem) {
    // Psi = (2 E U_old - E U_older - E_dir SrcFld) / dt^2 - C^T N C U_old
    //       + (Fb - Fb_old) / dt - I / dt   (Discretization.hpp:1713-1716)
    const double idt = 1.0 / d.dt[s];
    ((T*)d.rhs)[i] = (T)(eu_fem * (idt * idt) + (0.5 * idt) * su_fem - (double)cf +
                         idt * (double)((const T*)d.cb)[e] - idt * (double)((const T*)d.I)[e]);
  } else {
    ((T*)d.rhs)[i] = eu - dt * ((const T*)d.I)[e] + dt * cf + dt * ((const T*)d.cb)[e];
  }
  T* x = (T*)d.x;
  if (d.warm_start == 1) {
    x[i] = 0;
  } else if (d.warm_start == 2) {
    T* h1 = (T*)d.xh1;
    T* h2 = (T*)d.xh2;
    T* h3 = (T*)d.xh3;
    const int step = d.step[s];
    const T a = x[i], b = h1[i], c = h2[i];
    h3[i] = c;
    h2[i] = b;
    h1[i] = a;
    if (step >= 3) x[i] = (T)3 * a - (T)3 * b + c;
    else if (step >= 2) x[i] = (T)2 * a - b;
  } else if (d.warm_start == 3) {
    // the learned warm start's base guess, the same extrapolation, to xe
    const T a = x[i], b = ((const T*)d.xh1)[i], c = ((const T*)d.xh2)[i];
    const int step = d.step[s];
    ((T*)d.xe)[i] = step >= 3 ? (T)3 * a - (T)3 * b + c : (step >= 2 ? (T)2 * a - b : a);
  }
}

// Learned warm start (warm_start 3): grp_rhs puts the quadratic
// extrapolation e of the last three solutions in xe, then
//   grp_resid_e  r_e = b - A e -> r_alt, the right-hand side of the
//                correction system A (x_n - e) = r_e
//   grp_guess_mlp  per free row the network reads the last four solutions as
//                the third difference D3 = x - 3 xh1 + 3 xh2 - xh3 and the
//                compressed D2, D1 and level (sign log2(1 + |.|)), the Jacobi-scaled
//                correction right-hand side pre r_e with its mean over the
//                row's neighbours (A's pattern), all divided by the row scale
//                sigma = rms(D3, pre r_e); its output y gives the guess
//                e + sigma y in x.  Until the network is trained (mlp_on 0)
//                x = e.  Sampled rows store their inputs, e and sigma for
//                training.  A warp takes the 32 rows of one slice.
template <typename T>
__global__ void __launch_bounds__(kGB) grp_resid_e(GroupDev d) {
  const int64_t i = (int64_t)blockIdx.x * kGB + threadIdx.x;
  if (i >= d.nrow) return;
  const int s = d.slice_sim[i >> 5];
  if (!running(d, s)) return;
  const T* xe = (const T*)d.xe;
  ((T*)d.r_alt)[i] = ((const T*)d.rhs)[i] - sell_dot<T>(d.A, i, [&](int32_t c) { return xe[c]; });
}

// Inputs of one row of the learned guess (see above), with the history
// shift, the extrapolated guess in x and the training sample written here:
// f[6] the network's inputs, sg the row scale, ok whether the guess applies.
template <typename T>
__device__ __forceinline__ void guess_row(const GroupDev& d, int64_t sl, int64_t i, int s, float f[6], float& sg,
                                          bool& ok) {
  T* x = (T*)d.x;
  T* h1 = (T*)d.xh1;
  T* h2 = (T*)d.xh2;
  T* h3 = (T*)d.xh3;
  const T* re = (const T*)d.r_alt;
  const T* pre = (const T*)d.pre;
  const bool real = d.free_edge[i] >= 0;
  const double a = x[i], b1 = h1[i], c = h2[i], dd = h3[i];
  const double e = (double)((const T*)d.xe)[i];
  float sum = 0.0f;
  int cnt = 0;
  {
    // the row's columns are fetched CH at a time and their r_e gathered
    // together (independent loads in flight); the sum keeps column order
    constexpr int CH = 8;
    const int64_t b0 = d.A.ptr[sl];
    const int len = (int)((d.A.ptr[sl + 1] - b0) >> 5);
    const int32_t* col = d.A.col + b0 + (i & 31);
    for (int j0 = 0; j0 < len; j0 += CH) {
      int32_t cc[CH];
      float rv[CH];
#pragma unroll
      for (int k = 0; k < CH; k++) cc[k] = j0 + k < len ? ld_stream(col + 32 * (j0 + k)) : (int32_t)i;
#pragma unroll
      for (int k = 0; k < CH; k++) rv[k] = cc[k] != (int32_t)i ? (float)re[cc[k]] : 0.0f;
#pragma unroll
      for (int k = 0; k < CH; k++)
        if (cc[k] != (int32_t)i) {
          sum += rv[k];
          cnt++;
        }
    }
  }
  const float pr = (float)pre[i];
  const float jr = pr * (float)re[i];
  const float jm = cnt ? pr * sum / (float)cnt : jr;
  const float d3 = (float)(a - 3.0 * b1 + 3.0 * c - dd), d2 = (float)(a - 2.0 * b1 + c), d1 = (float)(a - b1);
  sg = sqrtf(0.5f * (d3 * d3 + jr * jr));
  ok = real && sg > 0.0f && isfinite(sg) && d.step[s] >= 4;
  const float inv = ok ? 1.0f / sg : 0.0f;
  f[0] = d3 * inv;
  f[1] = mlp_compress(d2 * inv);
  f[2] = mlp_compress(d1 * inv);
  f[3] = mlp_compress((float)a * inv);
  f[4] = jr * inv;
  f[5] = jm * inv;
  if (real) {
    h3[i] = (T)c;
    h2[i] = (T)b1;
    h1[i] = (T)a;
    x[i] = (T)e;
    if (d.nsamp && i >= d.samp_first && (i - d.samp_first) % d.samp_stride == 0) {
      const int64_t k = (i - d.samp_first) / d.samp_stride;
      if (k < d.nsamp) {
        for (int q = 0; q < 6; q++) d.samp_in[6 * k + q] = f[q];
        d.samp_e[k] = (float)e;
        d.samp_s[k] = sg;
        d.samp_row[k] = ok ? (int32_t)i : -1;
      }
    }
  }
}

// The trained network's guess on the 5th-generation tensor cores
// (mlp_tc.cuh): a CTA of four warps takes four slices (128 rows) per tile,
// warp w the slice whose rows are TMEM lanes 32w..32w+31.  Same inputs and
// outputs as grp_guess_mlp with mlp_on set.
template <typename T>
__global__ void __launch_bounds__(kTcRows) grp_guess_tc(GroupDev d) {
  extern __shared__ __align__(128) unsigned char tc_raw[];
  MlpTcSmem& sm = *reinterpret_cast<MlpTcSmem*>(tc_raw);
  mlp_tc_setup(sm, d.mlp_img);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nsl = d.nrow >> 5, tiles = (nsl + 3) / 4;
  T* x = (T*)d.x;
  uint32_t phase = 0;
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t sl = 4 * t + warp;
    const int64_t i = sl * 32 + lane;
    const int s = sl < nsl ? d.slice_sim[sl] : 0;
    const bool act = sl < nsl && running(d, s);
    float f[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, sg = 0.0f, y = 0.0f;
    bool ok = false;
    if (act) guess_row<T>(d, sl, i, s, f, sg, ok);
    if (!mlp_tc_forward(sm, phase, f, y, d.err)) break;
    if (act && ok) x[i] = (T)((double)x[i] + (double)sg * (double)y);
  }
  mlp_tc_teardown(sm);
}

template <typename T>
__global__ void __launch_bounds__(kGB, 3) grp_guess_mlp(GroupDev d) {
  __shared__ __align__(16) unsigned char img[kImgBytes];
  if (d.mlp_on) mlp_load_image(img, d.mlp_img);
  __syncthreads();
  const MlpSmem w = mlp_view(img);
  const int lane = threadIdx.x & 31;
  const int64_t nsl = d.nrow >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kGB) >> 5;
  T* x = (T*)d.x;
  // a warp takes whole slices (one simulation each), the grid strides over them
  for (int64_t sl = ((int64_t)blockIdx.x * kGB + threadIdx.x) >> 5; sl < nsl; sl += nw) {
    const int s = d.slice_sim[sl];
    if (!running(d, s)) continue;
    const int64_t i = sl * 32 + lane;
    float f[6], sg;
    bool ok;
    guess_row<T>(d, sl, i, s, f, sg, ok);
    if (d.mlp_on) {
      uint32_t a1[2][4];
      float y[2][4];
      mlp_input_fragment(a1[0], f, 0, lane);
      mlp_input_fragment(a1[1], f, 16, lane);
      mlp_infer2(w, a1, y, lane);
      const float v0 = mlp_output_to_rows(y[0], lane), v1 = mlp_output_to_rows(y[1], lane);
      const float yv = lane < 16 ? v0 : v1;
      if (ok) x[i] = (T)((double)x[i] + (double)sg * (double)yv);
    }
  }
}

// Training targets of the sampled rows after the solve: (x_n - e) / sigma
template <typename T>
__global__ void grp_mlp_targets(GroupDev d) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.nsamp) return;
  const int32_t i = d.samp_row[k];
  if (i < 0) {
    d.samp_t[k] = 0.0f;
    d.samp_w[k] = 0.0f;
    return;
  }
  // during training the CG starts from xe = e and leaves it untouched
  const double t = ((double)((const T*)d.x)[i] - (double)((const T*)d.xe)[i]) / (double)d.samp_s[k];
  d.samp_t[k] = (float)t;
  d.samp_w[k] = isfinite(t) ? 1.0f : 0.0f;
  if (!isfinite(t)) d.samp_t[k] = 0.0f;
}

struct SimCg {
  double rz, res0, bnorm, res, alpha, beta;
  int it, active, sel, pad;
};
constexpr int kPart = 6;  // per-warp partials a segment flushes (shared memory)
// Global partial slots of a segment: the initial residual's sums at 0..4, the
// p.q sums at 5 and the residual update's at 6..7.  Disjoint groups matter:
// no grid barrier separates a block's reads of one reduction's partials from
// another block's writes of the next reduction, so consecutive reductions may
// not share slots (the barrier after a reduction's writes does separate
// reads of a group from its next writes).
constexpr int kSlotStart = 0, kSlotPq = 5, kSlotRes = 6;
static_assert(kCgPart >= 8, "global CG partial slots");

// p_{j+1} at one row from z = pre r (stored by the residual phase), rounded
// the same way wherever it is formed
template <typename T>
__device__ __forceinline__ T p_next(T z, T pold, T beta, bool first) {
  return first ? z : fmaT(beta, pold, z);
}

// Co-resident CG blocks per SM the register budget is set for: more warps
// in flight hide the SELL sweep's load latency better than longer load
// chunks (measured: FP32 two blocks of 1024 threads, 2048 per SM; FP64 three
// of 512, where four spill).
#ifndef TF_CG_MINB32
#define TF_CG_MINB32 2
#endif
#ifndef TF_CG_MINB64
#define TF_CG_MINB64 3
#endif
template <typename T>
constexpr int cg_min_blocks() { return sizeof(T) == 4 ? TF_CG_MINB32 : TF_CG_MINB64; }

template <typename T, bool kFused>
__global__ void __launch_bounds__(cg_threads<T>(), cg_min_blocks<T>()) grp_cg(GroupDev d) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SimCg* st = reinterpret_cast<SimCg*>(smem_raw);
  auto grid_sync = [&]() { grid_barrier(d.gbar, d.err, gridDim.x); };
  double* wp = reinterpret_cast<double*>(smem_raw + sizeof(SimCg) * d.S);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g0 = d.blk_seg[blockIdx.x], g1 = d.blk_seg[blockIdx.x + 1];
  T* x = (T*)d.x;
  T* r = (T*)d.r;
  T* q = (T*)d.q;
  const T* b = (const T*)d.rhs;
  const T* pre = (const T*)d.pre;
  T* z = (T*)d.z;
  auto pbuf = [&](int k) { return (k & 1) ? (T*)d.p1 : (T*)d.p0; };
  // the buffers of a simulation's start (dual start: the extrapolation's)
  auto xs_of = [&](const SimCg& c) { return c.sel ? (T*)d.xe : x; };
  auto rs_of = [&](const SimCg& c) { return c.sel ? (T*)d.r_alt : r; };
  auto zs_of = [&](const SimCg& c) { return c.sel ? (T*)d.z_alt : z; };

  auto flush5 = [&](int g, double a0, double a1, double a2, double a3, double a4) {
    a3 = warp_sum(a3);
    a4 = warp_sum(a4);
    if (lane == 0) {
      double* w = wp + ((g - g0) * cg_warps<T>() + warp) * kPart;
      w[3] = a3;
      w[4] = a4;
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    if (lane == 0) {
      double* w = wp + ((g - g0) * cg_warps<T>() + warp) * kPart;
      w[0] = a0;
      w[1] = a1;
      w[2] = a2;
    }
  };
  auto flush = [&](int g, double a0, double a1, double a2) {
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    if (lane == 0) {
      double* w = wp + ((g - g0) * cg_warps<T>() + warp) * kPart;
      w[0] = a0;
      w[1] = a1;
      w[2] = a2;
    }
  };
  auto publish = [&](int nq, int slot) {
    __syncthreads();
    for (int gl = threadIdx.x; gl < g1 - g0; gl += cg_threads<T>())
      for (int k = 0; k < nq; k++) {
        double a = 0.0;
        for (int w = 0; w < cg_warps<T>(); w++) a += wp[(gl * cg_warps<T>() + w) * kPart + k];
        d.part[kCgPart * (int64_t)d.seg_of[g0 + gl] + slot + k] = a;
      }
  };
  // per-simulation totals of the published partials: one warp per
  // simulation, lanes over its segments, then a fixed shuffle tree; f(s, t)
  // runs on lane 0 with the nq totals t[]
  auto totals = [&](int nq, int slot, auto&& f) {
    for (int s = warp; s < d.S; s += cg_warps<T>()) {
      double t[kPart] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      for (int g = d.sim_seg[s] + lane; g < d.sim_seg[s + 1]; g += 32)
        for (int k = 0; k < nq; k++) t[k] += d.part[kCgPart * (int64_t)g + slot + k];
      for (int k = 0; k < nq; k++) t[k] = warp_sum(t[k]);
      if (lane == 0) f(s, t);
    }
  };
  auto go_on = [&](const SimCg& c, int s) {
    if (c.it >= d.cg_maxiter) return false;
    if (d.cg_criterion == 0) return c.res / c.res0 > d.tol[s];  // NaN (res0 = 0) stops, as the reference
    return c.res > d.tol[s] * c.bnorm;
  };

  // r = b - A x; rr = r.r, rz = r.(pre r), bb = b.b; in the dual start the
  // same for the second guess xe (its residual r_alt is already formed)
  T* ra = (T*)d.r_alt;
  T* za = (T*)d.z_alt;
  const bool dual = d.dual != 0;
  for (int g = g0; g < g1; g++) {
    const int s = d.seg_sim[d.seg_of[g]];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
    if (running(d, s))
      for (int64_t sl = d.seg_s0[d.seg_of[g]] + warp; sl < d.seg_s1[d.seg_of[g]]; sl += cg_warps<T>()) {
        const int64_t i = sl * 32 + lane;
        const T ri = b[i] - sell_dot_cg<T>(d.A, i, [&](int32_t c) { return x[c]; });
        r[i] = ri;
        const T zi = mulT(pre[i], ri);
        z[i] = zi;
        const double rd = (double)ri;
        a0 += rd * rd;
        a1 += rd * (double)zi;
        a2 += (double)b[i] * (double)b[i];
        if (dual) {
          // r_alt = b - A xe was formed by grp_resid_e from the same b and xe
          const T r2 = ra[i];
          const T z2 = mulT(pre[i], r2);
          za[i] = z2;
          a3 += (double)r2 * (double)r2;
          a4 += (double)r2 * (double)z2;
        }
      }
    flush5(g, a0, a1, a2, a3, a4);
  }
  publish(dual ? 5 : 3, kSlotStart);
  grid_sync();
  totals(dual ? 5 : 3, kSlotStart, [&](int s, const double* t) {
    SimCg c;
    c.sel = dual && t[3] < t[0] ? 1 : 0;
    c.pad = 0;
    c.res0 = sqrt(c.sel ? t[3] : t[0]);
    c.rz = c.sel ? t[4] : t[1];
    c.bnorm = sqrt(t[2]);
    c.res = c.res0;
    c.alpha = c.beta = 0.0;
    c.it = 0;
    c.active = running(d, s) && go_on(c, s);
    st[s] = c;
  });
  __syncthreads();

  for (;;) {
    int any = 0;
    for (int s = threadIdx.x; s < d.S; s += cg_threads<T>()) any |= st[s].active;
    if (!__syncthreads_or(any)) break;
    // p_{j+1} = z + beta p_j, x += alpha_j p_j (lazy), and in the fused
    // variant q = A p_{j+1} with p.q partials
    for (int g = g0; g < g1; g++) {
      const int s = d.seg_sim[d.seg_of[g]];
      const SimCg c = st[s];
      double a0 = 0.0;
      if (c.active) {
        const bool first = c.it == 0;
        const T beta = (T)c.beta, alpha = (T)c.alpha;
        const T* pold = pbuf(c.it + 1);
        T* pn = pbuf(c.it);
        T* xs = xs_of(c);
        const T* zs = zs_of(c);
        for (int64_t sl = d.seg_s0[d.seg_of[g]] + warp; sl < d.seg_s1[d.seg_of[g]]; sl += cg_warps<T>()) {
          const int64_t i = sl * 32 + lane;
          const T po = first ? (T)0 : pold[i];
          const T pi = p_next<T>(zs[i], po, beta, first);
          if (!first) xs[i] = fmaT(alpha, po, xs[i]);
          pn[i] = pi;
          if (kFused) {
            const T qi = sell_dot_cg<T>(d.A, i, [&](int32_t cc) {
              return p_next<T>(zs[cc], first ? (T)0 : pold[cc], beta, first);
            });
            q[i] = qi;
            a0 += (double)pi * (double)qi;
          }
        }
      }
      if (kFused) flush(g, a0, 0.0, 0.0);
    }
    if (!kFused) {
      grid_sync();
      for (int g = g0; g < g1; g++) {
        const int s = d.seg_sim[d.seg_of[g]];
        const SimCg c = st[s];
        double a0 = 0.0;
        if (c.active) {
          const T* pn = pbuf(c.it);
          for (int64_t sl = d.seg_s0[d.seg_of[g]] + warp; sl < d.seg_s1[d.seg_of[g]]; sl += cg_warps<T>()) {
            const int64_t i = sl * 32 + lane;
            const T qi = sell_dot_cg<T>(d.A, i, [&](int32_t cc) { return pn[cc]; });
            q[i] = qi;
            a0 += (double)pn[i] * (double)qi;
          }
        }
        flush(g, a0, 0.0, 0.0);
      }
    }
    publish(1, kSlotPq);
    grid_sync();
    totals(1, kSlotPq, [&](int s, const double* t) {
      if (st[s].active) st[s].alpha = st[s].rz / t[0];
    });
    __syncthreads();
    // r -= alpha q; rr, rz partials
    for (int g = g0; g < g1; g++) {
      const int s = d.seg_sim[d.seg_of[g]];
      double a0 = 0.0, a1 = 0.0;
      if (st[s].active) {
        const T alpha = (T)st[s].alpha;
        T* rs = rs_of(st[s]);
        T* zs = zs_of(st[s]);
        for (int64_t sl = d.seg_s0[d.seg_of[g]] + warp; sl < d.seg_s1[d.seg_of[g]]; sl += cg_warps<T>()) {
          const int64_t i = sl * 32 + lane;
          const T ri = rs[i] - alpha * q[i];
          rs[i] = ri;
          const T zi = mulT(pre[i], ri);
          zs[i] = zi;
          const double rd = (double)ri;
          a0 += rd * rd;
          a1 += rd * (double)zi;
        }
      }
      flush(g, a0, a1, 0.0);
    }
    publish(2, kSlotRes);
    grid_sync();
    totals(2, kSlotRes, [&](int s, const double* t) {
      SimCg c = st[s];
      if (!c.active) return;
      const double rz_prev = c.rz;
      c.res = sqrt(t[0]);
      c.rz = t[1];
      c.it++;
      c.beta = c.rz / rz_prev;
      c.active = go_on(c, s);
      st[s] = c;
    });
    __syncthreads();
  }
  // the last x update, x += alpha_{J-1} p_{J-1}
  for (int g = g0; g < g1; g++) {
    const int s = d.seg_sim[d.seg_of[g]];
    const SimCg c = st[s];
    if (!running(d, s)) continue;
    const T alpha = (T)c.alpha;
    const T* pl = pbuf(c.it - 1);
    T* xs = xs_of(c);
    for (int64_t sl = d.seg_s0[d.seg_of[g]] + warp; sl < d.seg_s1[d.seg_of[g]]; sl += cg_warps<T>()) {
      const int64_t i = sl * 32 + lane;
      T v = xs[i];
      if (c.it > 0) v = fmaT(alpha, pl[i], v);
      if (c.it > 0 || c.sel) x[i] = v;  // the solution always ends in x
    }
  }
  if (blockIdx.x == 0)
    for (int s = threadIdx.x; s < d.S; s += cg_threads<T>()) {
      if (!running(d, s)) continue;
      const SimCg c = st[s];
      const int64_t k = d.stat_off[s] + d.step[s];
      d.cg_iters[k] = c.it;
      d.cg_resid[k] = c.res / c.res0;
      const bool unmet = d.cg_criterion == 0 ? c.res / c.res0 > d.tol[s] : c.res > d.tol[s] * c.bnorm;
      d.cg_limit[k] = unmet ? 1 : 0;
      if (d.kept) d.kept[k] = dual && !c.sel ? 1 : 0;
    }
}

// Leapfrog energy of member s in the state after a step, (U^n, B^{n-1/2}):
// W^n = 0.5 U^n.E.U^n + 0.5 B^{n-1/2}.N.B^{n+1/2}, with B^{n+1/2} =
// B^{n-1/2} - dt C U^n recomputed per gathered face (what the next step's
// grp_curl_u forms).  The electric sum runs over the member's free rows (E's
// rows of the free edges; the Dirichlet edges hold 0 once the sources are
// off).  FP64 products and sums; one partial per block, in a fixed order.
template <typename T>
__global__ void __launch_bounds__(kGB) grp_energy(GroupDev d, int s, int64_t r0, int64_t nr, int64_t f0,
                                                  int64_t nf, double* part) {
  __shared__ double sh[33];
  const T* U = (const T*)d.U;
  const T* B = (const T*)d.B;
  const double dt = d.dt[s];
  auto row_dot = [&](const SellDev& m, int64_t row, auto&& g) {
    const int64_t sl = row >> 5;
    const int64_t b = m.ptr[sl];
    const int len = (int)((m.ptr[sl + 1] - b) >> 5);
    double acc = 0.0;
    for (int j = 0; j < len; j++) {
      const int64_t q = b + 32 * j + (row & 31);
      acc += (double)((const T*)m.val)[q] * g(m.col[q]);
    }
    return acc;
  };
  double acc = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * kGB + threadIdx.x; k < nr + nf; k += (int64_t)gridDim.x * kGB) {
    if (k < nr) {
      const int64_t i = r0 + k;
      const int32_t e = d.free_edge[i];
      if (e < 0) continue;
      const double eu = row_dot(d.Ef, i, [&](int32_t c) { return (double)U[c]; });
      acc += 0.5 * (double)U[e] * eu;
    } else {
      const int64_t f = f0 + (k - nr);
      if (d.fte[3 * f] < 0) continue;
      const double nb = row_dot(d.N, f, [&](int32_t c) {
        const int32_t* e = d.fte + 3 * (int64_t)c;
        if (e[0] < 0) return 0.0;
        const double cu = ((double)U[e[0]] - (double)U[e[1]]) + (double)U[e[2]];
        return (double)B[c] - dt * cu;
      });
      acc += 0.5 * (double)B[f] * nb;
    }
  }
  acc = grp_block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

template <typename T>
cudaError_t group_launch_energy(const GroupDev& d, int s, int64_t r0, int64_t nr, int64_t f0, int64_t nf,
                                double* part, int blocks, cudaStream_t st) {
  grp_energy<T><<<blocks, kGB, 0, st>>>(d, s, r0, nr, f0, nf, part);
  return cudaGetLastError();
}
template cudaError_t group_launch_energy<float>(const GroupDev&, int, int64_t, int64_t, int64_t, int64_t, double*,
                                                int, cudaStream_t);
template cudaError_t group_launch_energy<double>(const GroupDev&, int, int64_t, int64_t, int64_t, int64_t, double*,
                                                 int, cudaStream_t);

template <typename T>
__global__ void __launch_bounds__(kGB) grp_scatter(GroupDev d) {
  const int64_t k = (int64_t)blockIdx.x * kGB + threadIdx.x;
  T* U = (T*)d.U;
  T* Uo = (T*)d.Uo;  // fem groups: U_older = U_old before U takes the new values
  if (k < d.nrow) {
    const int32_t e = d.free_edge[k];
    if (e >= 0) {
      if (Uo) Uo[e] = U[e];
      U[e] = ((const T*)d.x)[k];
    }
  }
  if (k < d.ndir) {
    const int32_t e = d.dir_edge[k];
    if (Uo) Uo[e] = U[e];
    U[e] = ((const T*)d.src)[e];
  }
}

// Joule-loss term of conducting members at the start of a step, with U the
// previous step's state: one warp per 32-row slice of Sa writes the slice's
// sum of U_e (SigMat U)_e in FP64 (fixed shuffle tree)...
template <typename T>
__global__ void __launch_bounds__(kGB) grp_loss_rows(GroupDev d) {
  const int64_t i = (int64_t)blockIdx.x * kGB + threadIdx.x;
  if (i >= d.nsa) return;
  const int s = d.sa_slice_sim[i >> 5];
  const T* U = (const T*)d.U;
  double a = 0.0;
  const int32_t e = d.sa_edge[i];
  if (running(d, s) && e >= 0)
    a = (double)U[e] * sell_dot<double>(d.Sa, i, [&](int32_t c) { return (double)U[c]; }, (const T*)nullptr);
  a = warp_sum(a);
  if ((threadIdx.x & 31) == 0) d.loss_part[i >> 5] = a;
}

// ... and one warp per member adds its slices' sums in slice order into
// loss_a[stat_off + step]
__global__ void grp_loss_sum(GroupDev d) {
  const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= d.S || !d.lossy[s] || !running(d, s)) return;
  double a = 0.0;
  for (int g = d.sim_sa[s] + lane; g < d.sim_sa[s + 1]; g += 32) a += d.loss_part[g];
  a = warp_sum(a);
  if (lane == 0) d.loss_a[d.stat_off[s] + d.step[s]] = a;
}

__global__ void grp_bump(GroupDev d) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < d.S && d.step[s] < d.nsteps[s]) d.step[s] += 1;
}

// ------------------------------------------------------------------ launch
static inline unsigned gblk(int64_t n) { return (unsigned)(n > 0 ? (n + kGB - 1) / kGB : 1); }

template <typename T>
static size_t cg_smem(int S) { return sizeof(SimCg) * (size_t)S + sizeof(double) * kMaxSeg * cg_warps<T>() * kPart; }

template <typename T>
int group_cg_blocks(int device, int S, size_t* smem) {
  const size_t sm = cg_smem<T>(S);
  if (smem) *smem = sm;
  int sms = 0, a = 0, b = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaFuncSetAttribute(grp_cg<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess ||
      cudaFuncSetAttribute(grp_cg<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, grp_cg<T, true>, cg_threads<T>(), sm);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, grp_cg<T, false>, cg_threads<T>(), sm);
  return (a < b ? a : b) * sms;
}

// Resident CTAs of the tensor-core guess kernel over the whole GPU, from its
// registers and shared memory against the SM's limits, capped at the 8 CTAs
// whose 64 TMEM columns each fill the SM's 512 (the runtime's occupancy
// query reported 1 for this kernel, a fraction of what ncu measured).
template <typename T>
int group_guess_tc_blocks(int device) {
  int sms = 0, regs_sm = 0, smem_sm = 0, thr_sm = 0, blk_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
  cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device);
  cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, device);
  cudaFuncSetAttribute(grp_guess_tc<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
  cudaFuncAttributes fa{};
  int a = 6;  // what the shared operands allow at any carveout of 192 KB or more
  if (cudaFuncGetAttributes(&fa, grp_guess_tc<T>) == cudaSuccess && fa.numRegs > 0) {
    const int warps = kTcRows / 32;
    const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;  // 256-register allocation unit
    const int by_regs = regs_sm / (regs_warp * warps);
    const int by_smem = smem_sm / (int)(sizeof(MlpTcSmem) + fa.sharedSizeBytes + 1024);  // 1 KB reserved per CTA
    const int by_thr = thr_sm / kTcRows;
    a = by_regs < by_smem ? by_regs : by_smem;
    if (by_thr < a) a = by_thr;
    if (blk_sm > 0 && blk_sm < a) a = blk_sm;
    if (a < 1) a = 1;
  } else {
    cudaGetLastError();
  }
  const int tmem_cap = 512 / kTcCols;
  return (a < tmem_cap ? a : tmem_cap) * sms;
}

// One step of every running simulation.  ev (optional, 6 events) brackets:
// H update + probes, sources + rhs, CG, scatter, step end.
template <typename T>
cudaError_t group_launch_step(const GroupDev& d, int cg_blocks, int cg_variant, size_t smem, cudaStream_t st,
                              cudaEvent_t* ev) {
  if (ev) cudaEventRecord(ev[0], st);
  if (d.nsa > 0) {  // Joule losses of the conducting members, before U changes
    grp_loss_rows<T><<<gblk(d.nsa), kGB, 0, st>>>(d);
    grp_loss_sum<<<(unsigned)((d.S * 32 + 255) / 256), 256, 0, st>>>(d);
  }
  grp_curl_u<T><<<gblk(d.nF), kGB, 0, st>>>(d);
  grp_nmul<T><<<gblk(d.nF), kGB, 0, st>>>(d);
  if (d.np) grp_probes<T><<<(unsigned)((d.np + 127) / 128), 128, 0, st>>>(d);
  if (ev) cudaEventRecord(ev[1], st);
  grp_sources<T><<<d.S, kGB, 0, st>>>(d);
  grp_rhs<T><<<gblk(d.nrow), kGB, 0, st>>>(d);
  if (d.warm_start == 3) {
    grp_resid_e<T><<<gblk(d.nrow), kGB, 0, st>>>(d);
    const int64_t slices = d.nrow >> 5, per_block = kGB / 32;
    const int64_t want = (slices + per_block - 1) / per_block;
    if (d.mlp_on) {
      // trained network: the tensor-core form, 128 rows per tile
      const int64_t tiles = (slices + 3) / 4;
      const int64_t g = tiles < (int64_t)d.tc_blocks ? tiles : (int64_t)d.tc_blocks;
      grp_guess_tc<T><<<(unsigned)(g > 0 ? g : 1), kTcRows, sizeof(MlpTcSmem), st>>>(d);
    } else {
      grp_guess_mlp<T><<<(unsigned)(want < d.guess_blocks ? (want > 0 ? want : 1) : d.guess_blocks), kGB, 0, st>>>(d);
    }
  }
  if (ev) cudaEventRecord(ev[2], st);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cg_blocks);
  cfg.blockDim = dim3(cg_threads<T>());
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t err = cg_variant == 0 ? cudaLaunchKernelEx(&cfg, grp_cg<T, true>, d)
                                    : cudaLaunchKernelEx(&cfg, grp_cg<T, false>, d);
  if (err != cudaSuccess) return err;
  if (ev) cudaEventRecord(ev[3], st);
  grp_scatter<T><<<gblk(d.nrow > d.ndir ? d.nrow : d.ndir), kGB, 0, st>>>(d);
  if (ev) cudaEventRecord(ev[4], st);
  grp_bump<<<(d.S + 127) / 128, 128, 0, st>>>(d);
  if (ev) cudaEventRecord(ev[5], st);
  return cudaGetLastError();
}

template <typename T>
cudaError_t group_launch_targets(const GroupDev& d, cudaStream_t st) {
  if (d.nsamp) grp_mlp_targets<T><<<(unsigned)((d.nsamp + 255) / 256), 256, 0, st>>>(d);
  return cudaGetLastError();
}
template cudaError_t group_launch_targets<double>(const GroupDev&, cudaStream_t);
template cudaError_t group_launch_targets<float>(const GroupDev&, cudaStream_t);

template cudaError_t group_launch_step<double>(const GroupDev&, int, int, size_t, cudaStream_t, cudaEvent_t*);
template cudaError_t group_launch_step<float>(const GroupDev&, int, int, size_t, cudaStream_t, cudaEvent_t*);
template int group_cg_blocks<double>(int, int, size_t*);
template int group_cg_blocks<float>(int, int, size_t*);
template int group_guess_tc_blocks<double>(int);
template int group_guess_tc_blocks<float>(int);

}  // namespace tf
