// Stability estimate of the tetrahedral methods on the GPU (FP64).  The
// reference bounds dt by the largest eigenvalue of M^-1 K, K = C^T N C, with
// M^-1 the unmasked node-star inverses for dga (ComputeDGATimeStep,
// Discretization.hpp:7121-7174) or the eps-mass E for gfdtd and fem
// (:6928-7120), found with Spectra's Arnoldi solver.  Here a Lanczos
// recurrence in the K inner product runs on the device: every product,
// update and inner product is a kernel, and for gfdtd and fem each E^-1 x is
// the persistent Jacobi-PCG kernel of the standalone solve (tet_cg) from
// zero to 1e-12 relative.  Inner products sum fixed 4096-row chunks, each in
// one block with a fixed tree, and then the chunks in order, so the estimate
// is the same on every run.  The host keeps only the tridiagonal matrix and
// its largest eigenvalue (bisection, every 10 steps).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "cuda_util.hpp"
#include "dt_gpu.hpp"
#include "tet_kernels.cuh"

namespace tf {
cudaError_t pcg_launch_solve(DevPtrs d, int blocks, cudaStream_t st);
template <typename T>
int tet_cg_blocks(int device);

namespace {

constexpr int kB = 256;
constexpr int kChunk = 4096;  // rows per inner-product partial

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kB - 1) / kB > 0 ? (n + kB - 1) / kB : 1); }

// cu = C x: a face's three edges with signs +, -, + (fte order)
__global__ void __launch_bounds__(kB) dt_curl(const double* x, const int32_t* fte, double* cu, int64_t nf) {
  const int64_t f = (int64_t)blockIdx.x * kB + threadIdx.x;
  if (f >= nf) return;
  const int32_t* e = fte + 3 * f;
  cu[f] = x[e[0]] - x[e[1]] + x[e[2]];
}

// y = A x, one row per thread, entries in column order
__global__ void __launch_bounds__(kB) dt_spmv(const int64_t* ptr, const int32_t* col, const double* val,
                                             const double* x, double* y, int64_t n) {
  const int64_t r = (int64_t)blockIdx.x * kB + threadIdx.x;
  if (r >= n) return;
  double t = 0;
  for (int64_t k = ptr[r]; k < ptr[r + 1]; k++) t += val[k] * x[col[k]];
  y[r] = t;
}

// y = C^T x with the face index's sign in bit 31
__global__ void __launch_bounds__(kB) dt_ct(const int64_t* ptr, const int32_t* col, const double* x, double* y,
                                           int64_t n) {
  const int64_t e = (int64_t)blockIdx.x * kB + threadIdx.x;
  if (e >= n) return;
  double t = 0;
  for (int64_t k = ptr[e]; k < ptr[e + 1]; k++) {
    const int32_t c = col[k];
    const double v = x[c & 0x7fffffff];
    t = c < 0 ? t - v : t + v;
  }
  y[e] = t;
}

// part[c] = sum of a_i b_i over chunk c: each thread a fixed stride of the
// chunk, then a fixed shuffle and shared-memory tree
__global__ void __launch_bounds__(kB) dt_dot(const double* a, const double* b, double* part, int64_t n) {
  __shared__ double sh[kB / 32];
  const int64_t base = (int64_t)blockIdx.x * kChunk;
  double t = 0;
  for (int q = threadIdx.x; q < kChunk; q += kB) {
    const int64_t i = base + q;
    if (i < n) t += a[i] * b[i];
  }
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < kB / 32; w++) s += sh[w];
    part[blockIdx.x] = s;
  }
}

// out = sum of the partials in order (one thread: a few thousand at most)
__global__ void dt_sum(const double* part, int np, double* out) {
  double s = 0;
  for (int c = 0; c < np; c++) s += part[c];
  *out = s;
}

// w -= alpha v + beta vp
__global__ void __launch_bounds__(kB) dt_three_term(double* w, const double* v, const double* vp, double alpha,
                                                   double beta, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * kB + threadIdx.x;
  if (i < n) w[i] -= alpha * v[i] + beta * vp[i];
}

// a = b / s, c = d / s
__global__ void __launch_bounds__(kB) dt_div2(double* a, const double* b, double* c, const double* d, double s,
                                             int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * kB + threadIdx.x;
  if (i >= n) return;
  a[i] = b[i] / s;
  c[i] = d[i] / s;
}

}  // namespace

double gpu_lanczos_lambda(const DtProblem& p) {
  const int64_t n = p.n, nf = p.nf;
  CU(cudaSetDevice(p.device));
  cudaStream_t st = nullptr;
  CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  std::vector<void*> owned;
  auto dalloc = [&](size_t bytes) -> void* {
    void* q = nullptr;
    CU(cudaMalloc(&q, bytes > 0 ? bytes : 8));
    owned.push_back(q);
    return q;
  };
  auto up = [&](const void* src, size_t bytes) -> void* {
    void* q = dalloc(bytes);
    if (bytes) CU(cudaMemcpyAsync(q, src, bytes, cudaMemcpyHostToDevice, st));
    return q;
  };
  struct Dev {
    const int64_t* ptr;
    const int32_t* col;
    const double* val;
  };
  auto up_csr = [&](const DtCsr& m, bool with_val) {
    Dev d;
    d.ptr = (const int64_t*)up(m.ptr, (size_t)(m.nrows + 1) * 8);
    const size_t nnz = (size_t)m.ptr[m.nrows];
    d.col = (const int32_t*)up(m.col, nnz * 4);
    d.val = with_val ? (const double*)up(m.val, nnz * 8) : nullptr;
    return d;
  };
  double lam = 0;
  try {
    const int32_t* fte = (const int32_t*)up(p.fte, (size_t)nf * 12);
    const Dev N = up_csr(p.N, true), Ct = up_csr(p.Ct, false), M = up_csr(p.M, true);
    auto vec = [&](int64_t m) { return (double*)dalloc((size_t)m * 8); };
    double *x = vec(n), *v = vec(n), *Kv = vec(n), *w = vec(n), *Kw = vec(n), *vp = vec(n);
    double *cu = vec(nf), *ncu = vec(nf);
    const int nparts = (int)((n + kChunk - 1) / kChunk);
    double *part = vec(nparts > 0 ? nparts : 1), *scal = vec(1);
    CU(cudaMemcpyAsync(x, p.x0, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(vp, 0, (size_t)n * 8, st));
    auto dot = [&](const double* a, const double* b) {
      dt_dot<<<nparts > 0 ? nparts : 1, kB, 0, st>>>(a, b, part, n);
      dt_sum<<<1, 1, 0, st>>>(part, nparts, scal);
      double h = 0;
      CU(cudaMemcpyAsync(&h, scal, 8, cudaMemcpyDeviceToHost, st));
      CU(cudaStreamSynchronize(st));
      return h;
    };
    auto K = [&](const double* in, double* out) {
      dt_curl<<<blocks_for(nf), kB, 0, st>>>(in, fte, cu, nf);
      dt_spmv<<<blocks_for(nf), kB, 0, st>>>(N.ptr, N.col, N.val, cu, ncu, nf);
      dt_ct<<<blocks_for(n), kB, 0, st>>>(Ct.ptr, Ct.col, ncu, out, n);
    };
    // E^-1 x by the standalone Jacobi-PCG kernel: x0 = 0, ||r|| <= 1e-12 ||b||
    DevPtrs cg;
    int cg_blocks = 0;
    if (p.generalized) {
      cg_blocks = tet_cg_blocks<double>(p.device);
      if (cg_blocks < 1) throw CudaError("dt estimate: no co-resident blocks for the CG kernel");
      double* work = vec(4 * n + 4 * (int64_t)cg_blocks + 6);
      cg.nfree = (int)n;
      cg.a_ptr = M.ptr;
      cg.a_col = M.col;
      cg.a_val = M.val;
      cg.jac = work;
      cg.r = work + n;
      cg.p = work + 2 * n;
      cg.q = work + 3 * n;
      cg.part_a = work + 4 * n;
      cg.part_b = work + 4 * n + cg_blocks;
      double* tail = work + 4 * n + 4 * (int64_t)cg_blocks;
      cg.cg_resid = tail;
      cg.cg_iters = (int32_t*)(tail + 1);
      cg.step = (int*)(tail + 2);
      cg.cg_limit = (int32_t*)(tail + 3);
      cg.err = (int*)(tail + 4);
      cg.gbar = (unsigned int*)(tail + 5);
      cg.tol = 1e-12;
      cg.cg_maxiter = 1000;
      cg.cg_criterion = 1;
    }
    auto Minv = [&](const double* in, double* out) {
      if (!p.generalized) {
        dt_spmv<<<blocks_for(n), kB, 0, st>>>(M.ptr, M.col, M.val, in, out, n);
        return;
      }
      CU(cudaMemsetAsync(out, 0, (size_t)n * 8, st));
      DevPtrs d = cg;
      d.rhs = (void*)in;
      d.x = out;
      CU(pcg_launch_solve(d, cg_blocks, st));
      int berr = 0;
      CU(cudaMemcpyAsync(&berr, d.err, sizeof(int), cudaMemcpyDeviceToHost, st));
      CU(cudaStreamSynchronize(st));
      if (berr) throw CudaError("dt estimate: a grid barrier wait of the CG kernel ran out of time");
    };
    // start: v = M^-1 K x normalised in the K inner product
    K(x, Kv);
    Minv(Kv, v);
    K(v, Kv);
    const double nrm = std::sqrt(dot(v, Kv));
    dt_div2<<<blocks_for(n), kB, 0, st>>>(v, v, Kv, Kv, nrm, n);
    std::vector<double> al, be;
    double beta = 0, last = 0;
    for (int it = 0; it < 400; it++) {
      Minv(Kv, w);
      const double alpha = dot(w, Kv);
      dt_three_term<<<blocks_for(n), kB, 0, st>>>(w, v, vp, alpha, beta, n);
      al.push_back(alpha);
      K(w, Kw);
      double nb = dot(w, Kw);
      nb = nb > 0 ? std::sqrt(nb) : 0;
      if (it % 10 == 9 || nb == 0 || it == 399) {
        lam = p.tridiag_max(al, be);
        if (nb == 0 || std::fabs(lam - last) <= 1e-9 * std::fabs(lam)) break;
        last = lam;
      }
      be.push_back(nb);
      beta = nb;
      std::swap(vp, v);
      dt_div2<<<blocks_for(n), kB, 0, st>>>(v, w, Kv, Kw, nb, n);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st));
  } catch (...) {
    for (void* q : owned) cudaFree(q);
    cudaStreamDestroy(st);
    throw;
  }
  for (void* q : owned) cudaFree(q);
  cudaStreamDestroy(st);
  return lam;
}

}  // namespace tf
