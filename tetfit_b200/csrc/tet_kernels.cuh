// Device layout of the tetrahedral DGA paths.
//
// Complex: faces carry their three edges (p0p1, p0p2, p1p2 with signs +, -, +,
// the reference's fte order, Discretization.hpp:6327-6352); C^T is a CSR over
// edges whose int32 entries hold the face index with the sign in bit 31.  The
// material operators are CSR with int32 columns: N (faces x faces, per-tet
// inverse blocks summed), H (dga: masked node-star inverses), E / A / R
// (gfdtd eps-mass, its free-free block and its free-Dirichlet block).
#pragma once
#include <cstdint>

namespace tf {

// Type-erased device pointers (T = float or double arrays are void*).
struct DevPtrs {
  int nE = 0, nF = 0, nfree = 0, ndir = 0;
  double dt = 0;
  // state (T)
  void *U = nullptr, *F = nullptr, *B = nullptr, *cu = nullptr, *cf = nullptr, *I = nullptr, *cb = nullptr,
       *src = nullptr;
  // complex
  const int32_t* fte = nullptr;
  const int64_t* ct_ptr = nullptr;
  const int32_t* ct_col = nullptr;
  // operators (values T)
  const int64_t *n_ptr = nullptr, *h_ptr = nullptr, *e_ptr = nullptr, *a_ptr = nullptr, *r_ptr = nullptr;
  const int32_t *n_col = nullptr, *h_col = nullptr, *e_col = nullptr, *a_col = nullptr, *r_col = nullptr;
  const void *n_val = nullptr, *h_val = nullptr, *e_val = nullptr, *a_val = nullptr, *r_val = nullptr;
  const void* jac = nullptr;
  const int32_t *free_edges = nullptr, *dir_edges = nullptr;
  // CG work (T) and statistics
  void *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *rhs = nullptr, *xh1 = nullptr, *xh2 = nullptr,
       *xh3 = nullptr;
  double *part_a = nullptr, *part_b = nullptr;
  int32_t* cg_iters = nullptr;
  double* cg_resid = nullptr;
  int32_t* cg_limit = nullptr;  // optional: 1 when the iteration limit stopped the solve
  int cg_maxiter = 100, cg_criterion = 0, warm_start = 0;
  double tol = 1e-8;
  // sources
  int nse = 0, nsrc = 0;
  const int32_t* se_edge = nullptr;
  const int8_t* se_kind = nullptr;  // 1 e, 2 h, 3 j
  const int* se_begin = nullptr;
  const int* pair_src = nullptr;
  const double* pair_fac = nullptr;
  const int8_t* pair_dir = nullptr;
  const double *se_vec = nullptr, *se_post = nullptr;
  const double *src_amp = nullptr, *carrier = nullptr;
  double *flux = nullptr, *flux_part = nullptr;
  int nflux_part = 0;
  // probes
  int np = 0;
  const int32_t *p_edges = nullptr, *p_faces = nullptr;
  const double *p_we = nullptr, *p_hf = nullptr;
  double* samples = nullptr;
  const int* slot_of_step = nullptr;
  int* step = nullptr;
};

template <typename T>
struct TetDev {
  DevPtrs d;
  __host__ __device__ T* U() const { return (T*)d.U; }
};

}  // namespace tf
