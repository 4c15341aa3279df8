// Standalone Jacobi-PCG solve through the C ABI: the persistent cooperative
// kernel of the gfdtd path (tet_cg, tet_kernels.cu) applied to a caller's CSR
// system in device memory (ConjugateGradientSolver.hpp:52-129 semantics:
// Jacobi preconditioner, ||r||/||r0|| <= tol or ||r|| <= tol ||b||, hard
// iteration limit).
#include <cuda_runtime.h>

#include <mutex>
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
  // resid [1], then one 8-byte slot each for the int32 iters, step counter,
  // limit flag, barrier error flag, and the grid barrier's two uint32 words
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
  d.err = (int*)(work + 4 * n + 4 * blocks + 4);
  d.gbar = (unsigned int*)(work + 4 * n + 4 * blocks + 5);
  d.tol = a->tol;
  d.cg_maxiter = a->maxiter > 0 ? a->maxiter : 100;
  d.cg_criterion = a->criterion;
  return d;
}

size_t work_doubles(int64_t n, int blocks) { return (size_t)(4 * n + 4 * blocks + 6); }

int finish(cudaStream_t st, const DevPtrs& d, int32_t* iters, double* resid) {
  int32_t it = 0, lim = 0, berr = 0;
  double rs = 0;
  cudaError_t e = cudaMemcpyAsync(&it, d.cg_iters, sizeof(it), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&rs, d.cg_resid, sizeof(rs), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&lim, d.cg_limit, sizeof(lim), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&berr, d.err, sizeof(berr), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    tf::set_thread_error(std::string("tf_pcg_solve: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  if (berr) {
    tf::set_thread_error("tf_pcg_solve: a grid barrier wait of the CG kernel ran out of time; no valid result");
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

// ---------------------------------------------------------------------------
// tf_pcg_solve_noalloc: the same solve with its work space in a file-scope
// device array instead of cudaMalloc.  For callers that cannot allocate device
// memory while they solve: a host whose own pool allocator already holds the
// GPU's memory (a cudaMalloc there fails or fragments the pool), or a loop
// that must not stall other streams (cudaMalloc and cudaFree can synchronize
// the device).  The array holds kNoAllocMaxN unknowns (4 vectors of 8 B each,
// 8 MiB plus reduction slots) and stays resident on every GPU that loads the
// library until the process exits.
namespace {

constexpr int kNoAllocMaxN = 1 << 18;   // 262,144 unknowns
constexpr int kNoAllocMaxBlocks = 1024; // reduction slots for the cooperative grid

__device__ __align__(256) double g_pcg_scratch[4 * (size_t)kNoAllocMaxN + 4 * kNoAllocMaxBlocks + 6];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};
int g_scratch_blocks[kMaxDevices] = {0};

// Device address of the array on `device` (which must be current), looked
// up once per device: in host code the symbol name is only a host-side handle.
// The address is kept for the life of the process; cudaDeviceReset reloads
// the module and may move the array, so it is not supported while this
// library is loaded.
int scratch_for(int device, double** addr, int* blocks) {
  if (device < 0 || device >= kMaxDevices) {
    tf::set_thread_error("tf_pcg_solve_noalloc: device ordinal out of range");
    return TF_E_ARG;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
    if (e != cudaSuccess) {
      tf::set_thread_error(std::string("tf_pcg_solve_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return TF_E_CUDA;
    }
    int b = tf::tet_cg_blocks<double>(device);
    if (b < 1) {
      tf::set_thread_error("tf_pcg_solve_noalloc: no co-resident blocks for the cooperative kernel");
      return TF_E_CUDA;
    }
    g_scratch_blocks[device] = b < kNoAllocMaxBlocks ? b : kNoAllocMaxBlocks;
    g_scratch_addr[device] = (double*)p;
  }
  *addr = g_scratch_addr[device];
  *blocks = g_scratch_blocks[device];
  return TF_OK;
}

}  // namespace

extern "C" int tf_pcg_solve_noalloc(const tf_pcg_args* a, int32_t* iters, double* rel_resid) {
  int rc = check_args(a);
  if (rc) return rc;
  if (a->n > kNoAllocMaxN) {
    tf::set_thread_error("tf_pcg_solve_noalloc: n = " + std::to_string(a->n) +
                         " exceeds the static work space of " + std::to_string(kNoAllocMaxN) + " unknowns");
    return TF_E_ARG;
  }
  cudaError_t e = cudaSetDevice(a->device);
  if (e != cudaSuccess) {
    tf::set_thread_error(std::string("tf_pcg_solve_noalloc: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  double* work = nullptr;
  int blocks = 0;
  rc = scratch_for(a->device, &work, &blocks);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)a->stream;
  // the layout places the n-sized vectors first; the reduction slots and
  // counters sit after 4 * n, inside the array for any n <= kNoAllocMaxN.
  // Every value the kernel reads is written earlier in the same call (the
  // step counter, barrier words and error flag are cleared by
  // pcg_launch_solve).
  DevPtrs d = make_ptrs(a, work, blocks);
  e = tf::pcg_launch_solve(d, blocks, st);
  if (e != cudaSuccess) {
    tf::set_thread_error(std::string("tf_pcg_solve_noalloc: ") + cudaGetErrorString(e));
    return TF_E_CUDA;
  }
  return finish(st, d, iters, rel_resid);
}
