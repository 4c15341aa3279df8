// Kernels of the explicit tetrahedral DGA method (dga) for sm_100a, and the
// standalone CG solve of the C ABI.  (gfdtd simulations run on the group
// engine, tet_group_kernels.cu, also when a simulation is alone.)
//
//   tet_curl_u        cu = C U (3 signed edges per face), B -= dt cu
//                     (Discretization.hpp:902-916)
//   tet_nmul          F = R F - dt N cu (:917-918; R = 1 without magnetic
//                     losses)
//   tet_curl_f        cf = C^T F + Ctb Fb - I (:878-879)
//   tet_h_update      U = P U + dt H cf on interior edges (P = 1 when
//                     lossless), boundary flux (:887-894)
//   tet_frac_update   U_c = Q U_c_old + dt Mq cf: node-star fractions of the
//                     fractured edges (:891)
//   tet_frac_gather   U = sum of a fractured edge's two fractions (:892), flux
//   tet_sources       source edges from the carrier table: E values, boundary
//                     dual-edge H sources, currents (:821-868)
//   tet_probes        Whitney E and face-flux H at probe points (:3768-3897)
//   tet_cg            persistent cooperative Jacobi-PCG on a CSR system
//                     (ConjugateGradientSolver.hpp:52-103): SpMV, dots and
//                     axpys fused, FP64 reductions in a fixed order, a hard
//                     iteration limit and three bounded grid barriers per
//                     iteration
#include <cuda_runtime.h>

#include "grid_barrier.cuh"
#include "tet_kernels.cuh"

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
__global__ void __launch_bounds__(kBlock) tet_curl_u(DevPtrs d) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nF) return;
  const T* U = (const T*)d.U;
  const int32_t* e = d.fte + 3 * (int64_t)f;
  T c = U[e[0]] - U[e[1]] + U[e[2]];
  ((T*)d.cu)[f] = c;
  T* B = (T*)d.B;
  B[f] = B[f] - (T)d.dt * c;
}

// F -= dt N cu
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_nmul(DevPtrs d) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nF) return;
  const T* x = (const T*)d.cu;
  T s = 0;
  for (int64_t k = d.n_ptr[f]; k < d.n_ptr[f + 1]; k++) s += ld<T>(d.n_val, k) * x[d.n_col[k]];
  T* F = (T*)d.F;
  F[f] = d.n_r ? ((const T*)d.n_r)[f] * F[f] - (T)d.dt * s : F[f] - (T)d.dt * s;
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
    const T un = d.h_p ? ((const T*)d.h_p)[e] * uo + (T)d.dt * s : uo + (T)d.dt * s;
    U[e] = un;
    const T cb = ((const T*)d.cb)[e];
    if (cb != (T)0) fl = ((double)uo + (double)un) * (double)cb;
  }
  fl = block_sum(fl, sh);
  if (threadIdx.x == 0) d.flux_part[blockIdx.x] = fl;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) tet_frac_update(DevPtrs d) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.nq) return;
  const T* uo = (const T*)d.Uc_old;
  const T* cf = (const T*)d.cf;
  T a = 0, b = 0;
  for (int64_t k = d.q_ptr[r]; k < d.q_ptr[r + 1]; k++) a += ld<T>(d.q_val, k) * uo[d.q_col[k]];
  for (int64_t k = d.mq_ptr[r]; k < d.mq_ptr[r + 1]; k++) b += ld<T>(d.mq_val, k) * cf[d.mq_col[k]];
  ((T*)d.Uc)[r] = a + (T)d.dt * b;
}

// flux partials after tet_h_update's, at flux_part[nblk(nE) + block]
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_frac_gather(DevPtrs d, int part0) {
  __shared__ double sh[33];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double fl = 0.0;
  if (i < d.nfe) {
    const T* uc = (const T*)d.Uc;
    const int e = d.fe_edge[i];
    T* U = (T*)d.U;
    const T uo = U[e];
    const T un = uc[d.fe_a[i]] + uc[d.fe_b[i]];
    U[e] = un;
    const T cb = ((const T*)d.cb)[e];
    if (cb != (T)0) fl = ((double)uo + (double)un) * (double)cb;
  }
  fl = block_sum(fl, sh);
  if (threadIdx.x == 0) d.flux_part[part0 + blockIdx.x] = fl;
}

// dga energy (tf_energy).  W^n = 1/2 U^n.H^-1.U^{n+1} + 1/2 B.N.B over the
// class-1 edges, the leapfrog invariant of the lossless scheme; with
// U^{n+1} = U^n + dt H cf it is 1/2 u.x + 1/2 dt u.cf + 1/2 B.N.B, u the
// class-1 values of U^n, x = H^-1 u (a PCG solve), cf from the current F.
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_energy_gather(DevPtrs d, const int32_t* ie, double* u, int ni) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ni) u[i] = (double)((const T*)d.U)[ie[i]];
}

// part[2 b] = sum of u.x, part[2 b + 1] = sum of u.cf over block b's rows
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_energy_e(DevPtrs d, const int32_t* ie, const double* x, int ni,
                                                      double* part) {
  __shared__ double sh[33];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0.0, b = 0.0;
  if (i < ni) {
    const double u = (double)((const T*)d.U)[ie[i]];
    a = u * x[i];
    b = u * (double)((const T*)d.cf)[ie[i]];
  }
  a = block_sum(a, sh);
  b = block_sum(b, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

// part[b] = sum over block b's faces of B_f (N B)_f
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_energy_m(DevPtrs d, double* part) {
  __shared__ double sh[33];
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  double c = 0.0;
  if (f < d.nF) {
    const T* B = (const T*)d.B;
    double s = 0.0;
    for (int64_t k = d.n_ptr[f]; k < d.n_ptr[f + 1]; k++) s += (double)ld<T>(d.n_val, k) * (double)B[d.n_col[k]];
    c = (double)B[f] * s;
  }
  c = block_sum(c, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = c;
}

// out = 1/2 (sum u.x) + 1/2 dt (sum u.cf) + 1/2 (sum B.N.B), partials in order
__global__ void tet_energy_sum(const double* pe, int nbe, const double* pm, int nbm, double dt, double* out) {
  double a = 0.0, b = 0.0, c = 0.0;
  for (int q = 0; q < nbe; q++) {
    a += pe[2 * q];
    b += pe[2 * q + 1];
  }
  for (int q = 0; q < nbm; q++) c += pm[q];
  *out = 0.5 * a + 0.5 * dt * b + 0.5 * c;
}

// Source edges: E sources write U, H sources write cb (reset each step),
// currents write I.
template <typename T>
__global__ void __launch_bounds__(kBlock) tet_sources(DevPtrs d) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int step = *d.step;
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
    if (kind == 1) ((T*)d.U)[e] = (T)val;
    else if (kind == 2) ((T*)d.cb)[e] = (T)val;
    else if (kind == 3) ((T*)d.I)[e] = (T)val;
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
  grid_barrier(d.gbar, d.err, nb);
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
    grid_barrier(d.gbar, d.err, nb);
    double pq = 0;
    for (int64_t i = tid; i < n; i += nth) {
      const T qi = spmv_row<T>(d.a_ptr, d.a_col, d.a_val, p, (int)i);
      q[i] = qi;
      pq += (double)p[i] * (double)qi;
    }
    pq = block_sum(pq, sh);
    if (threadIdx.x == 0) d.part_a[blockIdx.x] = pq;
    grid_barrier(d.gbar, d.err, nb);
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
    grid_barrier(d.gbar, d.err, nb);
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

// Probe export.  The print schedule is indexed by step counter + offset:
// after a step, time (s+1) dt, offset 1; before the first step, offset 0.
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

// One leapfrog step of the dga method (Discretization.hpp:810-931).  ev
// (optional, 6 events) brackets: sources, H half, flux, E half, probes.
template <typename T>
cudaError_t tet_launch_step(const DevPtrs& d, cudaStream_t st, cudaEvent_t* ev) {
  if (ev) cudaEventRecord(ev[0], st);
  cudaMemsetAsync(d.cb, 0, sizeof(T) * (size_t)d.nE, st);
  if (d.nse) tet_sources<T><<<nblk(d.nse), kBlock, 0, st>>>(d);
  if (ev) cudaEventRecord(ev[1], st);
  tet_curl_f<T><<<nblk(d.nE), kBlock, 0, st>>>(d);
  tet_h_update<T><<<nblk(d.nE), kBlock, 0, st>>>(d);
  if (d.nq > 0) {
    cudaMemcpyAsync(d.Uc_old, d.Uc, sizeof(T) * (size_t)d.nq, cudaMemcpyDeviceToDevice, st);
    tet_frac_update<T><<<nblk(d.nq), kBlock, 0, st>>>(d);
  }
  if (d.nfe > 0) tet_frac_gather<T><<<nblk(d.nfe), kBlock, 0, st>>>(d, (int)nblk(d.nE));
  if (ev) cudaEventRecord(ev[2], st);
  flux_reduce<<<1, kBlock, 0, st>>>(d, 0.5);
  if (ev) cudaEventRecord(ev[3], st);
  tet_curl_u<T><<<nblk(d.nF), kBlock, 0, st>>>(d);
  tet_nmul<T><<<nblk(d.nF), kBlock, 0, st>>>(d);
  if (ev) cudaEventRecord(ev[4], st);
  if (d.np) tet_probes<T><<<nblk(d.np), kBlock, 0, st>>>(d, 1);
  bump_step<<<1, 1, 0, st>>>(d.step);
  if (ev) cudaEventRecord(ev[5], st);
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
  cudaMemsetAsync(d.gbar, 0, 2 * sizeof(unsigned int), st);
  cudaMemsetAsync(d.err, 0, sizeof(int), st);
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

// dga energy: gather u, solve H x = u (d_cg: the class-1 block of H and the
// PCG work), then the three sums; *out receives W (device)
template <typename T>
cudaError_t tet_launch_energy(const DevPtrs& d, DevPtrs d_cg, int cg_blocks, const int32_t* ie, int ni,
                              double* part, double* out, cudaStream_t st) {
  tet_curl_f<T><<<nblk(d.nE), kBlock, 0, st>>>(d);
  tet_energy_gather<T><<<nblk(ni), kBlock, 0, st>>>(d, ie, (double*)d_cg.rhs, ni);
  cudaMemsetAsync(d_cg.x, 0, sizeof(double) * (size_t)ni, st);
  cudaError_t e = pcg_launch_solve(d_cg, cg_blocks, st);
  if (e != cudaSuccess) return e;
  const int nbe = (int)nblk(ni), nbm = (int)nblk(d.nF);
  tet_energy_e<T><<<nbe, kBlock, 0, st>>>(d, ie, (const double*)d_cg.x, ni, part);
  tet_energy_m<T><<<nbm, kBlock, 0, st>>>(d, part + 2 * nbe);
  tet_energy_sum<<<1, 1, 0, st>>>(part, nbe, part + 2 * nbe, nbm, d.dt, out);
  return cudaGetLastError();
}

template cudaError_t tet_launch_energy<double>(const DevPtrs&, DevPtrs, int, const int32_t*, int, double*, double*,
                                               cudaStream_t);
template cudaError_t tet_launch_energy<float>(const DevPtrs&, DevPtrs, int, const int32_t*, int, double*, double*,
                                              cudaStream_t);
template cudaError_t tet_launch_step<double>(const DevPtrs&, cudaStream_t, cudaEvent_t*);
template cudaError_t tet_launch_step<float>(const DevPtrs&, cudaStream_t, cudaEvent_t*);
template int tet_cg_blocks<double>(int);
template void tet_launch_initial_probes<double>(const DevPtrs&, cudaStream_t);
template void tet_launch_initial_probes<float>(const DevPtrs&, cudaStream_t);

}  // namespace tf
