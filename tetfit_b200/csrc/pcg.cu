// Standalone Jacobi-PCG solve through the C ABI: the persistent cooperative
// kernel of the gfdtd path (tet_cg, tet_kernels.cu) applied to a caller's CSR
// system in device memory (ConjugateGradientSolver.hpp:52-129 semantics:
// Jacobi preconditioner, ||r||/||r0|| <= tol or ||r|| <= tol ||b||, hard
// iteration limit).
#include <cuda_runtime.h>

#include <string>

#include "../../include/tetfit.h"
#include "tet_kernels.cuh"

namespace tf {
cudaError_t pcg_launch_solve(DevPtrs d, int blocks, cudaStream_t st);
template <typename T>
int tet_cg_blocks(int device);
void set_thread_error(const std::string& m);
}  // namespace tf

using tf::DevPtrs;

namespace {

int check_args(const tf_pcg_args* a) {
  if (!a || a->n <= 0 || !a->row_ptr || !a->col || !a->val || !a->b || !a->x || a->maxiter < 0 ||
      !(a->tol >= 0)) {
    tf::set_thread_error("tf_pcg_solve: missing pointer or invalid size / tolerance / iteration limit");
    return TF_E_ARG;
  }
  return TF_OK;
}

DevPtrs make_ptrs(const tf_pcg_args* a, double* work, int blocks) {
  // work layout: pre, r, p, q [n each], part_a [blocks], part_b [3 blocks],
  // resid [1], then int32 iters, step counter and limit flag
  const int64_t n = a->n;
  DevPtrs d;
  d.nfree = a->n;
  d.a_ptr = a->row_ptr;
  d.a_col = a->col;
  d.a_val = a->val;
  d.rhs = (void*)a->b;
  d.x = a->x;
  d.jac = work;
  d.r = work + n;
  d.p = work + 2 * n;
  d.q = work + 3 * n;
  d.part_a = work + 4 * n;
  d.part_b = work + 4 * n + blocks;
  d.cg_resid = work + 4 * n + 4 * blocks;
  d.cg_iters = (int32_t*)(work + 4 * n + 4 * blocks + 1);
  d.step = (int*)(work + 4 * n + 4 * blocks + 2);
  d.cg_limit = (int32_t*)(work + 4 * n + 4 * blocks + 3);
  d.tol = a->tol;
  d.cg_maxiter = a->maxiter > 0 ? a->maxiter : 100;
  d.cg_criterion = a->criterion;
  return d;
}

size_t work_doubles(int64_t n, int blocks) { return (size_t)(4 * n + 4 * blocks + 4); }

int finish(cudaStream_t st, const DevPtrs& d, int32_t* iters, double* resid) {
  int32_t it = 0, lim = 0;
  double rs = 0;
  cudaError_t e = cudaMemcpyAsync(&it, d.cg_iters, sizeof(it), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&rs, d.cg_resid, sizeof(rs), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&lim, d.cg_limit, sizeof(lim), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    tf::set_thread_error(std::string("tf_pcg_solve: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  if (iters) *iters = it;
  if (resid) *resid = rs;
  if (lim) {
    tf::set_thread_error("tf_pcg_solve: iteration limit reached before the tolerance");
    return TF_E_SOLVER;
  }
  return TF_OK;
}

}  // namespace

extern "C" int tf_pcg_solve(const tf_pcg_args* a, int32_t* iters, double* rel_resid) {
  int rc = check_args(a);
  if (rc) return rc;
  cudaError_t e = cudaSetDevice(a->device);
  if (e != cudaSuccess) {
    tf::set_thread_error(std::string("tf_pcg_solve: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  cudaStream_t st = (cudaStream_t)a->stream;
  const int blocks = tf::tet_cg_blocks<double>(a->device);
  double* work = nullptr;
  e = cudaMalloc(&work, work_doubles(a->n, blocks) * sizeof(double));
  if (e != cudaSuccess) {
    tf::set_thread_error(std::string("tf_pcg_solve: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  DevPtrs d = make_ptrs(a, work, blocks);
  e = tf::pcg_launch_solve(d, blocks, st);
  if (e != cudaSuccess) {
    cudaFree(work);
    tf::set_thread_error(std::string("tf_pcg_solve: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  rc = finish(st, d, iters, rel_resid);
  cudaFree(work);
  return rc;
}
