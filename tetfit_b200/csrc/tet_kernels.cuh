// Device layout of the explicit tetrahedral DGA method (dga) and of the
// standalone CG solve.
//
// Complex: faces carry their three edges (p0p1, p0p2, p1p2 with signs +, -, +,
// the reference's fte order, Discretization.hpp:6327-6352); C^T is a CSR over
// edges whose int32 entries hold the face index with the sign in bit 31.  The
// material operators are CSR with int32 columns: N (faces x faces, per-tet
// inverse blocks summed) and H (masked node-star inverses); the CG solve takes
// the caller's CSR system A.
#pragma once
#include <cstdint>

namespace tf {

// Type-erased device pointers (T = float or double arrays are void*).  The
// dga step uses the complex, N, H, the state and the sources; the standalone
// CG solve (tf_pcg_solve) uses the system A, jac and the CG work.
struct DevPtrs {
  int nE = 0, nF = 0, nfree = 0;
  double dt = 0;
  // state (T)
  void *U = nullptr, *F = nullptr, *B = nullptr, *cu = nullptr, *cf = nullptr, *I = nullptr, *cb = nullptr;
  // complex
  const int32_t* fte = nullptr;
  const int64_t* ct_ptr = nullptr;
  const int32_t* ct_col = nullptr;
  // operators (values T)
  const int64_t *n_ptr = nullptr, *h_ptr = nullptr, *a_ptr = nullptr;
  const int32_t *n_col = nullptr, *h_col = nullptr, *a_col = nullptr;
  const void *n_val = nullptr, *h_val = nullptr, *a_val = nullptr;
  const void* jac = nullptr;
  // dga with conducting tets: P per edge (null when lossless), the node-star
  // fractions U_c (and their copy from the step before) with their operators
  // Q (U_c x U_c) and Mq (U_c x edges), and the fractured edges with their
  // two U_c entries
  const void* h_p = nullptr;
  const void* n_r = nullptr;  // dga with chi: R per face (F = R F - dt N cu), null without
  int nq = 0, nfe = 0;
  const int64_t *q_ptr = nullptr, *mq_ptr = nullptr;
  const int32_t *q_col = nullptr, *mq_col = nullptr;
  const void *q_val = nullptr, *mq_val = nullptr;
  void *Uc = nullptr, *Uc_old = nullptr;
  const int32_t *fe_edge = nullptr, *fe_a = nullptr, *fe_b = nullptr;
  // CG work (T), reductions, grid barrier and statistics
  void *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *rhs = nullptr;
  double *part_a = nullptr, *part_b = nullptr;
  unsigned int* gbar = nullptr;  // grid barrier: arrivals, generation
  int* err = nullptr;            // raised when a grid barrier wait ran out of time
  int32_t* cg_iters = nullptr;
  double* cg_resid = nullptr;
  int32_t* cg_limit = nullptr;  // optional: 1 when the iteration limit stopped the solve
  int cg_maxiter = 100, cg_criterion = 0;
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

}  // namespace tf
