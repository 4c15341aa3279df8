// Error types and the CUDA-call check used across the host runtime.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace tf {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct UnsupportedError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct SolverError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess)
    throw CudaError(std::string(what) + " failed at " + file + ":" + std::to_string(line) + ": " +
                    cudaGetErrorString(e));
}

}  // namespace tf

#define CU(call) ::tf::cuda_check((call), #call, __FILE__, __LINE__)
