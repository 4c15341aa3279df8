// Tetrahedral DGA kernels for sm_100a.
//
//   tet_curl_u        cu = C U (3 signed edges per face), B -= dt cu
//                     (Discretization.hpp:902-916, 1466-1467)
//   tet_nmul          F -= dt N cu (dga, :917) or F = N B (gfdtd, :1468)
//   tet_curl_f        cf = C^T F + Ctb Fb - I (dga, :878-879)
//   tet_h_update      U += dt H cf on interior edges, boundary flux (dga, :889-894)
//   tet_sources       source edges from the carrier table: E values, boundary
//                     dual-edge H sources, currents (:821-868, :1478-1504)
//   tet_rhs           Psi = E U_old - R Src - dt I + dt C^T F + dt Ctb Fb on
//                     the free edges (gfdtd, :1516-1523)
//   tet_cg            persistent cooperative Jacobi-PCG on the free edges
//                     (ConjugateGradientSolver.hpp:52-103): SpMV, dots and
//                     axpys fused, FP64 reductions in a fixed order, a hard
//                     iteration limit and three grid barriers per iteration
//   tet_scatter       U[free] = x, U[Dirichlet] = source values (:1540-1541)
//   tet_probes        Whitney E and face-flux H at probe points (:3768-3897)
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "tet_kernels.cuh"

namespace cg = cooperative_groups;

namespace tf {

constexpr int kBlock = 256;

template <typename T>
__device__ __forceinline__ T ld(const void* p, int64_t i) {
  return ((const T*)p)[i];
}

// deterministic block sum of one double (all threads get the result)
__device__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) sh[32] = s;
  }
  __syncthreads();
  return sh[32];
}

template <typename T>
__global__ void __launch_bounds__(kBlock) tet_curl_u(DevPtrs d, int update_B) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nF) return;
  const T* U = (const T*)d.U;
  const int32_t* e = d.fte + 3 * (int64_t)f;
  T c = U[e[0]] - U[e[1]] + U[e[2]];
  ((T*)d.cu)[f] = c;
  if (update_B) {
    T* B = (T*)d.B;
    B[f] = B[f] - (T)d.dt * c;
  }
}

// mode 0: F -= dt N cu (dga); mode 1: F = N B (gfdtd)
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_nmul(DevPtrs d, int mode) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nF) return;
  const T* x = (const T*)(mode == 0 ? d.cu : d.B);
  T s = 0;
  for (int64_t k = d.n_ptr[f]; k < d.n_ptr[f + 1]; k++) s += ld<T>(d.n_val, k) * x[d.n_col[k]];
  T* F = (T*)d.F;
  if (mode == 0) F[f] = F[f] - (T)d.dt * s;
  else F[f] = s;
}

template <typename T>
__device__ __forceinline__ T ctf(const DevPtrs& d, int e) {
  const T* F = (const T*)d.F;
  T s = 0;
  for (int64_t k = d.ct_ptr[e]; k < d.ct_ptr[e + 1]; k++) {
    const int32_t c = d.ct_col[k];
    const T v = F[c & 0x7fffffff];
    s = c < 0 ? s - v : s + v;
  }
  return s;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) tet_curl_f(DevPtrs d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.nE) return;
  ((T*)d.cf)[e] = ctf<T>(d, e) + ((const T*)d.cb)[e] - ((const T*)d.I)[e];
}

template <typename T>
__global__ void __launch_bounds__(kBlock) tet_h_update(DevPtrs d) {
  __shared__ double sh[33];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double fl = 0.0;
  if (e < d.nE && d.h_ptr[e + 1] > d.h_ptr[e]) {
    const T* cf = (const T*)d.cf;
    T s = 0;
    for (int64_t k = d.h_ptr[e]; k < d.h_ptr[e + 1]; k++) s += ld<T>(d.h_val, k) * cf[d.h_col[k]];
    T* U = (T*)d.U;
    const T uo = U[e];
    const T un = uo + (T)d.dt * s;
    U[e] = un;
    const T cb = ((const T*)d.cb)[e];
    if (cb != (T)0) fl = ((double)uo + (double)un) * (double)cb;
  }
  fl = block_sum(fl, sh);
  if (threadIdx.x == 0) d.flux_part[blockIdx.x] = fl;
}

// Source edges.  method 1 (dga): E sources write U, H sources write cb (reset
// each step), currents write I.  method 2 (gfdtd): E sources write the
// Dirichlet value array, flux partials use U (the previous solution).
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_sources(DevPtrs d, int method) {
  __shared__ double sh[33];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int step = *d.step;
  double fl = 0.0;
  if (s < d.nse) {
    auto value = [&](int row) {
      double v[3] = {0.0, 0.0, 0.0};
      for (int p = d.se_begin[s]; p < d.se_begin[s + 1]; p++) {
        const int si = d.pair_src[p];
        double ret = d.src_amp[si] * d.carrier[(int64_t)row * d.nsrc + si];
        ret *= d.pair_fac[4 * p + 0];
        ret *= d.pair_fac[4 * p + 1];
        ret *= d.pair_fac[4 * p + 2];
        ret *= d.pair_fac[4 * p + 3];
        v[d.pair_dir[p]] += ret;
      }
      const double* w = d.se_vec + 3 * (int64_t)s;
      return d.se_post[s] * ((v[0] * w[0] + v[1] * w[1]) + v[2] * w[2]);
    };
    const int e = d.se_edge[s];
    const int kind = d.se_kind[s];
    const double val = value(step);
    if (kind == 1) {
      if (method == 1) ((T*)d.U)[e] = (T)val;
      else ((T*)d.src)[e] = (T)val;
    } else if (kind == 2) {
      ((T*)d.cb)[e] = (T)val;
      if (method == 2) {
        const double prev = step > 0 ? value(step - 1) : 0.0;
        fl = (double)((const T*)d.U)[e] * (0.5 * (val + prev));
      }
    } else if (kind == 3) {
      ((T*)d.I)[e] = (T)val;
    }
  }
  if (method == 2) {
    fl = block_sum(fl, sh);
    if (threadIdx.x == 0) d.flux_part[blockIdx.x] = fl;
  }
}

__global__ void flux_reduce(DevPtrs d, double scale) {
  __shared__ double sh[33];
  double a = 0.0;
  for (int b = threadIdx.x; b < d.nflux_part; b += blockDim.x) a += d.flux_part[b];
  a = block_sum(a, sh);
  if (threadIdx.x == 0) d.flux[*d.step] = scale * a;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) tet_rhs(DevPtrs d) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.nfree) return;
  const int e = d.free_edges[k];
  const T* U = (const T*)d.U;
  const T* S = (const T*)d.src;
  T eu = 0, rs = 0;
  for (int64_t q = d.e_ptr[e]; q < d.e_ptr[e + 1]; q++) eu += ld<T>(d.e_val, q) * U[d.e_col[q]];
  for (int64_t q = d.r_ptr[k]; q < d.r_ptr[k + 1]; q++) rs += ld<T>(d.r_val, q) * S[d.r_col[q]];
  const T dt = (T)d.dt;
  ((T*)d.rhs)[k] = eu - rs - dt * ((const T*)d.I)[e] + dt * ctf<T>(d, e) + dt * ((const T*)d.cb)[e];
}

// Initial guess: 0 previous solution (x kept), 1 zero, 2 quadratic
// extrapolation from the last three solutions; history shifts here.
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_guess(DevPtrs d) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.nfree) return;
  T* x = (T*)d.x;
  T* h1 = (T*)d.xh1;
  T* h2 = (T*)d.xh2;
  T* h3 = (T*)d.xh3;
  const int step = *d.step;
  if (d.warm_start == 1) {
    x[k] = 0;
  } else if (d.warm_start == 2) {
    // x_{n-1} = x (last solution); keep three levels
    const T a = x[k], b = h1[k], c = h2[k];
    h3[k] = c;
    h2[k] = b;
    h1[k] = a;
    if (step >= 3) x[k] = (T)3 * a - (T)3 * b + c;
    else if (step >= 2) x[k] = (T)2 * a - b;
  }
}

template <typename T>
__device__ __forceinline__ T spmv_row(const int64_t* ptr, const int32_t* col, const void* val, const T* x, int i) {
  T s = 0;
  for (int64_t k = ptr[i]; k < ptr[i + 1]; k++) s += ld<T>(val, k) * x[col[k]];
  return s;
}

// deterministic grid sum of per-block partials (every block computes it)
__device__ double sum_parts(const double* part, int nb, int stride, int off, double* sh) {
  double a = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) a += part[(int64_t)b * stride + off];
  return block_sum(a, sh);
}

// Persistent Jacobi-PCG (ConjugateGradientSolver.hpp:52-103).  Stops when
// ||r||/||r0|| <= tol (criterion 0, the reference) or ||r|| <= tol ||b||
// (criterion 1), or after cg_maxiter iterations.  State in T, every inner
// product and norm accumulated in FP64.
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_cg(DevPtrs d) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[33];
  const int n = d.nfree;
  const int nb = gridDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)nb * blockDim.x;
  T* x = (T*)d.x;
  T* r = (T*)d.r;
  T* p = (T*)d.p;
  T* q = (T*)d.q;
  const T* b = (const T*)d.rhs;
  const T* pre = (const T*)d.jac;
  // r = b - A x, rz = r.(pre r), rr = r.r, bb = b.b
  double rr = 0, rz = 0, bb = 0;
  for (int64_t i = tid; i < n; i += nth) {
    const T ri = b[i] - spmv_row<T>(d.a_ptr, d.a_col, d.a_val, x, (int)i);
    r[i] = ri;
    const double rd = (double)ri;
    rr += rd * rd;
    rz += rd * (double)(pre[i] * ri);
    bb += (double)b[i] * (double)b[i];
  }
  rr = block_sum(rr, sh);
  rz = block_sum(rz, sh);
  bb = block_sum(bb, sh);
  if (threadIdx.x == 0) {
    d.part_b[3 * blockIdx.x + 0] = rr;
    d.part_b[3 * blockIdx.x + 1] = rz;
    d.part_b[3 * blockIdx.x + 2] = bb;
  }
  grid.sync();
  rr = sum_parts(d.part_b, nb, 3, 0, sh);
  rz = sum_parts(d.part_b, nb, 3, 1, sh);
  bb = sum_parts(d.part_b, nb, 3, 2, sh);
  const double res0 = sqrt(rr);
  const double bnorm = sqrt(bb);
  double res = res0;
  int it = 0;
  double rz_prev = 1.0;
  auto go_on = [&](double rs) {
    if (it >= d.cg_maxiter) return false;
    if (d.cg_criterion == 0) return rs / res0 > d.tol;  // NaN (res0 = 0) stops, as the reference
    return rs > d.tol * bnorm;
  };
  while (go_on(res)) {
    const T beta = it == 0 ? (T)0 : (T)(rz / rz_prev);
    for (int64_t i = tid; i < n; i += nth) {
      const T z = pre[i] * r[i];
      p[i] = it == 0 ? z : z + beta * p[i];
    }
    grid.sync();
    double pq = 0;
    for (int64_t i = tid; i < n; i += nth) {
      const T qi = spmv_row<T>(d.a_ptr, d.a_col, d.a_val, p, (int)i);
      q[i] = qi;
      pq += (double)p[i] * (double)qi;
    }
    pq = block_sum(pq, sh);
    if (threadIdx.x == 0) d.part_a[blockIdx.x] = pq;
    grid.sync();
    pq = sum_parts(d.part_a, nb, 1, 0, sh);
    const T alpha = (T)(rz / pq);
    double rr2 = 0, rz2 = 0;
    for (int64_t i = tid; i < n; i += nth) {
      x[i] = x[i] + alpha * p[i];
      const T ri = r[i] - alpha * q[i];
      r[i] = ri;
      const double rd = (double)ri;
      rr2 += rd * rd;
      rz2 += rd * (double)(pre[i] * ri);
    }
    rr2 = block_sum(rr2, sh);
    rz2 = block_sum(rz2, sh);
    if (threadIdx.x == 0) {
      d.part_b[3 * blockIdx.x + 0] = rr2;
      d.part_b[3 * blockIdx.x + 1] = rz2;
    }
    grid.sync();
    rr = sum_parts(d.part_b, nb, 3, 0, sh);
    rz_prev = rz;
    rz = sum_parts(d.part_b, nb, 3, 1, sh);
    res = sqrt(rr);
    it++;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int step = *d.step;
    d.cg_iters[step] = it;
    d.cg_resid[step] = res / res0;
    if (d.cg_limit) {
      const bool unmet = d.cg_criterion == 0 ? res / res0 > d.tol : res > d.tol * bnorm;
      d.cg_limit[step] = unmet ? 1 : 0;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) tet_scatter(DevPtrs d) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  T* U = (T*)d.U;
  if (k < d.nfree) U[d.free_edges[k]] = ((const T*)d.x)[k];
  if (k < d.ndir) {
    const int e = d.dir_edges[k];
    U[e] = ((const T*)d.src)[e];
  }
}

// Probe export.  The print schedule is indexed by step counter + offset
// (dga exports after the step, time (s+1) dt: offset 1; gfdtd exports U^{s}
// before the solve, time s dt: offset 0).
template <typename T>
__global__ void tet_probes(DevPtrs d, int offset) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int step = *d.step;
  const int slot = d.slot_of_step[step + offset];
  if (p < d.np && slot >= 0) {
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
    double* out = d.samples + ((int64_t)slot * d.np + p) * 6;
    for (int a = 0; a < 3; a++) {
      out[a] = E[a];
      out[3 + a] = H[a];
    }
  }
}

__global__ void bump_step(int* step) { *step += 1; }

// ------------------------------------------------------------------ launch
static inline unsigned nblk(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock > 0 ? (n + kBlock - 1) / kBlock : 1); }

template <typename T>
int tet_cg_blocks(int device) {
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tet_cg<T>, kBlock, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (per_sm > 2) per_sm = 2;
  return per_sm * sms;
}

// One leapfrog step.  ev (optional, 6 events) brackets: sources, E half,
// scatter/flux, probes, H half.
template <typename T>
cudaError_t tet_launch_step(const DevPtrs& d, int method, int cg_blocks, cudaStream_t st, cudaEvent_t* ev) {
  if (method == 1) {  // dga (Discretization.hpp:810-931)
    if (ev) cudaEventRecord(ev[0], st);
    cudaMemsetAsync(d.cb, 0, sizeof(T) * (size_t)d.nE, st);
    if (d.nse) tet_sources<T><<<nblk(d.nse), kBlock, 0, st>>>(d, 1);
    if (ev) cudaEventRecord(ev[1], st);
    tet_curl_f<T><<<nblk(d.nE), kBlock, 0, st>>>(d);
    tet_h_update<T><<<nblk(d.nE), kBlock, 0, st>>>(d);
    if (ev) cudaEventRecord(ev[2], st);
    flux_reduce<<<1, kBlock, 0, st>>>(d, 0.5);
    if (ev) cudaEventRecord(ev[3], st);
    tet_curl_u<T><<<nblk(d.nF), kBlock, 0, st>>>(d, 1);
    tet_nmul<T><<<nblk(d.nF), kBlock, 0, st>>>(d, 0);
    if (ev) cudaEventRecord(ev[4], st);
    if (d.np) tet_probes<T><<<nblk(d.np), kBlock, 0, st>>>(d, 1);
    bump_step<<<1, 1, 0, st>>>(d.step);
    if (ev) cudaEventRecord(ev[5], st);
  } else {  // gfdtd (Discretization.hpp:1459-1565)
    if (ev) cudaEventRecord(ev[0], st);
    tet_curl_u<T><<<nblk(d.nF), kBlock, 0, st>>>(d, 1);
    tet_nmul<T><<<nblk(d.nF), kBlock, 0, st>>>(d, 1);
    if (d.np) tet_probes<T><<<nblk(d.np), kBlock, 0, st>>>(d, 0);
    if (ev) cudaEventRecord(ev[1], st);
    tet_sources<T><<<nblk(d.nse), kBlock, 0, st>>>(d, 2);
    flux_reduce<<<1, kBlock, 0, st>>>(d, 1.0);
    tet_rhs<T><<<nblk(d.nfree), kBlock, 0, st>>>(d);
    tet_guess<T><<<nblk(d.nfree), kBlock, 0, st>>>(d);
    if (ev) cudaEventRecord(ev[2], st);
    DevPtrs dd = d;
    void* args[] = {(void*)&dd};
    cudaError_t err = cudaLaunchCooperativeKernel((void*)tet_cg<T>, dim3(cg_blocks), dim3(kBlock), args, 0, st);
    if (err != cudaSuccess) return err;
    if (ev) cudaEventRecord(ev[3], st);
    tet_scatter<T><<<nblk(d.nfree > d.ndir ? d.nfree : d.ndir), kBlock, 0, st>>>(d);
    if (ev) cudaEventRecord(ev[4], st);
    bump_step<<<1, 1, 0, st>>>(d.step);
    if (ev) cudaEventRecord(ev[5], st);
  }
  return cudaGetLastError();
}

// Jacobi preconditioner from the CSR diagonal (1 where the diagonal is
// missing or zero, ConjugateGradientSolver.hpp:119-127)
__global__ void jacobi_from_csr(const int64_t* ptr, const int32_t* col, const double* val, double* pre, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dg = 0.0;
  for (int64_t k = ptr[i]; k < ptr[i + 1]; k++)
    if (col[k] == i) dg = val[k];
  pre[i] = dg != 0.0 ? 1.0 / dg : 1.0;
}

// Standalone FP64 solve: preconditioner, then the persistent PCG kernel.
cudaError_t pcg_launch_solve(DevPtrs d, int blocks, cudaStream_t st) {
  jacobi_from_csr<<<nblk(d.nfree), kBlock, 0, st>>>(d.a_ptr, d.a_col, (const double*)d.a_val, (double*)d.jac,
                                                    d.nfree);
  cudaMemsetAsync(d.step, 0, sizeof(int), st);
  void* args[] = {(void*)&d};
  cudaError_t err = cudaLaunchCooperativeKernel((void*)tet_cg<double>, dim3(blocks), dim3(kBlock), args, 0, st);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

// export before the first step (dga: t = 0)
template <typename T>
void tet_launch_initial_probes(const DevPtrs& d, cudaStream_t st) {
  if (d.np) tet_probes<T><<<nblk(d.np), kBlock, 0, st>>>(d, 0);
}

template cudaError_t tet_launch_step<double>(const DevPtrs&, int, int, cudaStream_t, cudaEvent_t*);
template cudaError_t tet_launch_step<float>(const DevPtrs&, int, int, cudaStream_t, cudaEvent_t*);
template int tet_cg_blocks<double>(int);
template int tet_cg_blocks<float>(int);
template void tet_launch_initial_probes<double>(const DevPtrs&, cudaStream_t);
template void tet_launch_initial_probes<float>(const DevPtrs&, cudaStream_t);

}  // namespace tf
