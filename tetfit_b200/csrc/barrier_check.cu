// tf_barrier_check: self-check of the bounded grid barrier (grid_barrier.cuh)
// that the persistent CG kernels use.  No reference counterpart: it shows, on
// the GPU, that a barrier wait which can never complete ends with the error
// status instead of a hung launch, and it measures the barrier's latency.
#include <cuda_runtime.h>

#include <string>

#include "../../include/tetfit.h"
#include "grid_barrier.cuh"

namespace tf {
void set_thread_error(const std::string& m);
}

namespace {

// Every block passes `rounds` barriers that wait for `expected` arrivals.
__global__ void barrier_check_kernel(unsigned int* bar, int* err, unsigned int expected, int rounds,
                                     uint64_t limit_ns) {
  for (int k = 0; k < rounds; k++) tf::grid_barrier(bar, err, expected, limit_ns);
}

int fail(int code, const std::string& m) {
  tf::set_thread_error("tf_barrier_check: " + m);
  return code;
}

}  // namespace

extern "C" int tf_barrier_check(int32_t device, uint32_t blocks, uint32_t expected, uint32_t rounds,
                                uint32_t timeout_us, int32_t* status, double* ms) {
  if (!status) return fail(TF_E_ARG, "status is NULL");
  if (blocks < 1 || expected < 1 || expected > 2 * blocks || rounds < 1 || rounds > 100000 || timeout_us < 1 ||
      timeout_us > 1000000)
    return fail(TF_E_ARG, "blocks >= 1, 1 <= expected <= 2 blocks, 1 <= rounds <= 100000, "
                          "1 <= timeout_us <= 1000000");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(TF_E_CUDA, cudaGetErrorString(e));
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if ((int)blocks > sms) return fail(TF_E_ARG, "blocks exceeds the SM count (" + std::to_string(sms) + ")");
  unsigned int* words = nullptr;  // bar[0], bar[1], err
  e = cudaMalloc(&words, 3 * sizeof(unsigned int));
  if (e != cudaSuccess) return fail(TF_E_CUDA, cudaGetErrorString(e));
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int32_t flag = 0;
  float t = 0.f;
  e = cudaMemset(words, 0, 3 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaEventCreate(&ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
  if (e == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(128);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaEventRecord(ev[0]);
    e = cudaLaunchKernelEx(&cfg, barrier_check_kernel, words, (int*)(words + 2), expected, (int)rounds,
                           (uint64_t)timeout_us * 1000ull);
    cudaEventRecord(ev[1]);
  }
  if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev[0], ev[1]);
  if (e == cudaSuccess) e = cudaMemcpy(&flag, words + 2, sizeof(flag), cudaMemcpyDeviceToHost);
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  cudaFree(words);
  if (e != cudaSuccess) return fail(TF_E_CUDA, cudaGetErrorString(e));
  *status = flag;
  if (ms) *ms = t;
  return TF_OK;
}
