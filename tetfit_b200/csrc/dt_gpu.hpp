// Stability estimate of the tetrahedral methods on the GPU (dt_gpu.cu).
#pragma once
#include <cstdint>
#include <vector>

namespace tf {

struct DtCsr {  // host CSR: nrows + 1 row offsets, int32 columns, FP64 values
  int64_t nrows = 0;
  const int64_t* ptr = nullptr;
  const int32_t* col = nullptr;
  const double* val = nullptr;
};

struct DtProblem {
  int device = 0;
  int64_t n = 0, nf = 0;          // edges, faces
  const int32_t* fte = nullptr;   // 3 edges per face (signs +, -, +)
  DtCsr N, Ct, M;                 // Ct: face index with the sign in bit 31
  bool generalized = false;       // M is E (solve) rather than E^-1 (product)
  const double* x0 = nullptr;     // start vector (n)
  double (*tridiag_max)(const std::vector<double>&, const std::vector<double>&) = nullptr;
};

// Largest eigenvalue of M^-1 K (K = C^T N C) by Lanczos on the device.
double gpu_lanczos_lambda(const DtProblem& p);

}  // namespace tf
