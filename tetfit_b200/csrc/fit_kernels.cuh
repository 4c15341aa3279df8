// Device-side layout of the Cartesian FIT (Yee) path.
//
// Field state lives in six padded arrays, one per component, all with the same
// shape [Nz+1][Ny+1][sx] (x fastest, sx = Nx+1 rounded up to 8):
//   Ux[i,j,k]  x-edge (i,j,k)->(i+1,j,k)      Fx[i,j,k]  x-normal face at x=i
//   Uy[i,j,k]  y-edge (i,j,k)->(i,j+1,k)      Fy[i,j,k]  y-normal face at y=j
//   Uz[i,j,k]  z-edge (i,j,k)->(i,j,k+1)      Fz[i,j,k]  z-normal face at z=k
// Slots outside an array's valid range stay zero.  U is the edge voltage and
// F the face magnetomotive force of TetFIT's FIT scheme (Discretization.hpp
// :1869-1915); B (face flux) is not stored: it is recomputed where sampled.
//
// Material coefficients are not stored per dof.  Each cell carries a compact
// material index (uint8), and the edge/face coefficients are rebuilt in the
// kernels from per-material tables with the same additions, in the same order,
// as the reference's averaging (Discretization.hpp:5234-5330, 5485-5609), so
// they are bit-identical to precomputed per-dof values.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace tf {

template <typename T>
struct FitGrid {
  T *Ux, *Uy, *Uz, *Fx, *Fy, *Fz;
  const uint8_t* mat;  // [Nz][Ny][Nx] compact material index per cell
  int Nx, Ny, Nz;
  int64_t sx, sxy;     // strides of the state arrays
  double dt;
  // per-material tables, 3 entries per material (axis x,y,z)
  const double* P;     // da_a * eps_aa           (edge permittivity share)
  const double* S;     // da_a * sigma_aa         (edge conductivity share)
  const double* R;     // (L_a/2) / mu_aa         (face reluctance share, 0 if mu = 0)
  const double* X;     // (L_a/2) / chi_aa        (face magnetic loss share, 0 if chi = 0)
  const T* mh_pure;    // M_h of an edge whose 4 cells share the material
  const T* mq_pure;    // M_q  "
  const T* mnu_pure;   // M_nu of a face whose 2 cells share the material
  const T* mmu_pure;   // M_mu "
  const uint8_t* live; // material label != 0 (the cell takes part in the H update)
  double len[3], area[3];
  // optional per-dof coefficients (state-array shape, one array per axis),
  // computed once from the tables above by fit_coef_kernel: M_h, M_q per
  // edge, M_nu, M_mu per face (M_nu = -0.0 marks a face the H update skips)
  T *Ch[3], *Cq[3], *Cn[3], *Cm[3];
  // optional coefficient classes: a uint16 class per updated edge and face
  // (state-array shape, one array per axis) into tables of coefficient
  // pairs, lut_e[2c] = M_h, lut_e[2c+1] = M_q and lut_f[2c] = M_nu,
  // lut_f[2c+1] = M_mu (M_nu = -0.0 marks a face the H update skips).  A
  // class is a distinct tuple (axis, materials of the dof's cells), and its
  // pair is computed from the tuple by the same functions as above.
  uint16_t *Ke[3], *Kf[3];
  T *lut_e, *lut_f;
};

// Hash tables of the class build (device memory, kClassTable slots each).
constexpr int kClassTable = 1 << 20;
constexpr int kMaxClasses = 65535;
struct FitClassWork {
  unsigned long long* keys[2];  // edge and face tuples, ~0 empty
  int* ids[2];                  // dense class of an occupied slot
  int* count;                   // [2] classes found; [2] overflow flag
};

// Edges whose update is not the 4-face interior stencil: boundary edges on
// source or natural surfaces, interface PEC edges, E-source and dipole edges.
// Structure of arrays, n entries.
template <typename T>
struct SpecialEdges {
  int n;
  const int64_t* slot;     // index into U array `comp`
  const int8_t* comp;      // 0 x, 1 y, 2 z
  const int8_t* op;        // 0 hold value, 1 explicit-face update, 2 stencil with current
  const int8_t* nface;     // faces used by op 1/2 (<= 4)
  const int8_t* fcomp;     // [n][4] face component
  const int64_t* fslot;    // [n][4] face slot
  const int8_t* fsign;     // [n][4] sign
  const double* mh;        // coefficients (double, converted to T at use)
  const double* mq;
  const int* src_begin;    // [n+1] range into the (edge, source) pair table
  const int* pair_src;     // source index of the pair
  const double* pair_fac;  // [npairs][4]: decay, s0, s1, s2 spatial factors
  const double* pair_vec;  // [n][3]: projection vector per edge (dual edge / edge vector)
  const double* post;      // [n] factor applied after the projection (1/|edge| for currents)
  const int8_t* pair_dir;  // source direction 0/1/2
  const double* src_amp;   // [nsrc] amplitude (times impedance for j)
  const double* carrier;   // [nsteps][nsrc] carrier factor at the sampling time
  const int8_t* src_kind;  // [nsrc] 0 e, 1 h, 2 j
  int nsrc;
  T* out;                  // [n] new value
  double* flux_part;       // [blocks] flux partial sums of this step
};

// Joule loss of each E half step, 0.25 (U_old + U)^T Si (U_old + U)
// (Discretization.hpp:1902), with Si = sigma-bar / length per edge.  The
// reference fills Si only for l2norm outputs (:5368, :5594-5597); the loss
// kernels run only then, and only when some material conducts.
template <typename T>
struct FitLoss {
  T *Ox, *Oy, *Oz;   // U before the E half step (state-array shape)
  double* part;      // [nparts] per-block partial sums
  double* loss;      // [nsteps] loss per step
  int nparts;
};

// Tensor maps of the TMA z-march (kernel variant 4): Ux, Uy, Uz and Fx, Fy,
// Fz over their [Nz+1][Ny+1][sx] arrays, box (32 + 16 bytes) x 9 x 1; err
// receives 1 when an mbarrier wait gave up.
struct FitTmaMaps {
  CUtensorMap U[3], F[3];
  int* err;
};

template <typename T>
cudaError_t fit_build_coefficients(const FitGrid<T>& g, cudaStream_t st);
// Fills g.Ke, g.Kf and the class tables; ncls[0..1] receive the edge and
// face class counts, -1 when there are more than kMaxClasses.
template <typename T>
cudaError_t fit_build_classes(const FitGrid<T>& g, const FitClassWork& w, int ncls[2], cudaStream_t st);

struct ProbeSet {
  int n;
  const int* ci; const int* cj; const int* ck;  // probe cell
  const double* inv_mu;                          // [n][3] 1/mu_aa of the cell material
  double* samples;                               // [slots][n][6]
  const int* slot_of_step;                       // print slot per step, -1 none
};

}  // namespace tf
