// Cartesian FIT (Yee) leapfrog kernels for sm_100a.
//
//   fit_e_kernel        interior E update  (Discretization.hpp:1869-1876)
//   fit_special_pre     boundary / source / interface edges, into a side buffer
//                       (Discretization.hpp:1850-1863, 1880-1895, 3899-4202)
//   fit_special_post    scatter of the side buffer + per-step boundary flux
//                       (Discretization.hpp:1901)
//   fit_probe_kernel    E and H at probe cells (Discretization.hpp:3555-3588)
//   fit_h_kernel        H update (Discretization.hpp:1908-1915)
//
// The update arithmetic uses explicitly rounded operations (no contraction to
// FMA) in the reference's operation order, so the FP64 path reproduces the
// CPU reference arithmetic exactly; the FP32 path runs the same code on
// float state with coefficients rounded from their double values.
#include <cuda.h>
#include <cuda_runtime.h>

#include "fit_kernels.cuh"

// z-march loop unrolling: with two planes per iteration the compiler issues
// the next plane's loads before the current plane's stores (measured at 512^3
// FP32: E 2.46 -> 2.07 ms, H 2.71 -> 2.26 ms, results bitwise unchanged; four
// planes spill registers and lose)
#ifndef TF_FIT_UNROLL
#define TF_FIT_UNROLL 2
#endif
#define TF_PRAGMA(x) _Pragma(#x)
#define TF_UNROLL(n) TF_PRAGMA(unroll n)

namespace tf {

template <typename T>
struct Ar;
template <>
struct Ar<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
template <>
struct Ar<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};

__device__ __forceinline__ int64_t cell_index(int i, int j, int k, int Nx, int Ny) {
  return (int64_t)i + (int64_t)Nx * ((int64_t)j + (int64_t)Ny * k);
}

// Edge coefficients from the materials of its cells, listed in sweep order
// (Discretization.hpp:5294-5330 accumulation, :5591-5609 M_h/M_q).
template <typename T>
__device__ void edge_coef(const FitGrid<T>& g, int a, const uint8_t* m, int nm, double& mh, double& mq) {
  double eps = 0.0, sig = 0.0;
  bool lossy = false;
  for (int q = 0; q < nm; q++) {
    eps = __dadd_rn(eps, g.P[3 * m[q] + a]);
    double s = g.S[3 * m[q] + a];
    if (s != 0.0) {
      sig = __dadd_rn(sig, s);
      lossy = true;
    }
  }
  const double len = g.len[a];
  if (eps != 0.0) {
    if (lossy) {
      double hs = __dmul_rn(__dmul_rn(0.5, g.dt), sig);
      mh = len / __dadd_rn(eps, hs);
      mq = __dsub_rn(eps, hs) / len;
    } else {
      mh = len / eps;
      mq = eps / len;
    }
  } else {
    mh = 0.0;
    mq = 0.0;
  }
}

// Face coefficients (Discretization.hpp:5270-5292 accumulation, :5488-5514).
template <typename T>
__device__ void face_coef(const FitGrid<T>& g, int a, const uint8_t* m, int nm, double& mnu, double& mmu) {
  double ni = 0.0, ms = 0.0;
  bool lossy = false;
  for (int q = 0; q < nm; q++) {
    ni = __dadd_rn(ni, g.R[3 * m[q] + a]);
    double x = g.X[3 * m[q] + a];
    if (x != 0.0) {
      ms = __dadd_rn(ms, x);
      lossy = true;
    }
  }
  const double area = g.area[a];
  if (ni != 0.0) {
    if (lossy) {
      double hd = __dmul_rn(0.5, g.dt) / ms;
      mnu = 1.0 / __dmul_rn(area, __dadd_rn(1.0 / ni, hd));
      mmu = __dmul_rn(area, __dsub_rn(1.0 / ni, hd));
    } else {
      mnu = ni / area;
      mmu = area / ni;
    }
  } else {
    mnu = 0.0;
    mmu = 0.0;
  }
}

template <typename T>
__device__ __forceinline__ void edge_coef_t(const FitGrid<T>& g, int a, const uint8_t* m, T& mh, T& mq) {
  if (m[0] == m[1] && m[0] == m[2] && m[0] == m[3]) {
    mh = g.mh_pure[3 * m[0] + a];
    mq = g.mq_pure[3 * m[0] + a];
  } else {
    double h, q;
    edge_coef(g, a, m, 4, h, q);
    mh = (T)h;
    mq = (T)q;
  }
}

// Face (axis a) at slot s whose lower cell is (il,jl,kl) and upper cell (i,j,k).
template <typename T>
__device__ __forceinline__ bool face_coef_t(const FitGrid<T>& g, int a, bool has_lo, bool has_hi, uint8_t mlo,
                                            uint8_t mhi, T& mnu, T& mmu) {
  if (!((has_lo && g.live[mlo]) || (has_hi && g.live[mhi]))) return false;
  if (has_lo && has_hi && mlo == mhi) {
    mnu = g.mnu_pure[3 * mlo + a];
    mmu = g.mmu_pure[3 * mlo + a];
  } else {
    uint8_t m[2];
    int nm = 0;
    if (has_lo) m[nm++] = mlo;
    if (has_hi) m[nm++] = mhi;
    double nu, mu;
    face_coef(g, a, m, nm, nu, mu);
    mnu = (T)nu;
    mmu = (T)mu;
  }
  return true;
}

// Interior E update: one thread per node slot (i,j,k) updates the x, y and z
// edges leaving that node, when they have all four faces.
template <typename T>
__global__ void __launch_bounds__(256) fit_e_kernel(FitGrid<T> g) {
  using A = Ar<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.Nx || j > g.Ny) return;
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const T dt = (T)g.dt;
  const bool xin = i > 0 && i < g.Nx, yin = j > 0 && j < g.Ny, zin = k > 0 && k < g.Nz;
  // materials of the 8 cells around the node: c[dz][dy][dx], d=0 is the lower cell
  uint8_t c[2][2][2];
#pragma unroll
  for (int dz = 0; dz < 2; dz++)
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
      for (int dx = 0; dx < 2; dx++) {
        int ci = i - 1 + dx, cj = j - 1 + dy, ck = k - 1 + dz;
        bool ok = ci >= 0 && ci < g.Nx && cj >= 0 && cj < g.Ny && ck >= 0 && ck < g.Nz;
        c[dz][dy][dx] = ok ? g.mat[cell_index(ci, cj, ck, g.Nx, g.Ny)] : 0;
      }
  if (i < g.Nx && yin && zin) {  // x-edge: faces Fy(k-1), Fz(j-1), Fz, Fy (Ct order)
    uint8_t m[4] = {c[0][0][1], c[0][1][1], c[1][0][1], c[1][1][1]};
    T mh, mq;
    edge_coef_t(g, 0, m, mh, mq);
    T cf = A::sub(A::add(A::sub(g.Fy[s - g.sxy], g.Fz[s - g.sx]), g.Fz[s]), g.Fy[s]);
    g.Ux[s] = A::mul(mh, A::add(A::mul(mq, g.Ux[s]), A::mul(dt, cf)));
  }
  if (j < g.Ny && xin && zin) {  // y-edge: faces Fx(k-1), Fz(i-1), Fz, Fx; dual curl -1
    uint8_t m[4] = {c[0][1][0], c[0][1][1], c[1][1][0], c[1][1][1]};
    T mh, mq;
    edge_coef_t(g, 1, m, mh, mq);
    T cf = -A::sub(A::add(A::sub(g.Fx[s - g.sxy], g.Fz[s - 1]), g.Fz[s]), g.Fx[s]);
    g.Uy[s] = A::mul(mh, A::add(A::mul(mq, g.Uy[s]), A::mul(dt, cf)));
  }
  if (k < g.Nz && xin && yin) {  // z-edge: faces Fx(j-1), Fy(i-1), Fy, Fx
    uint8_t m[4] = {c[1][0][0], c[1][0][1], c[1][1][0], c[1][1][1]};
    T mh, mq;
    edge_coef_t(g, 2, m, mh, mq);
    T cf = A::sub(A::add(A::sub(g.Fx[s - g.sx], g.Fy[s - 1]), g.Fy[s]), g.Fx[s]);
    g.Uz[s] = A::mul(mh, A::add(A::mul(mq, g.Uz[s]), A::mul(dt, cf)));
  }
}

// Interior E update, z-marching form: a thread owns the node column (i,j)
// over planes [k0, k1) and carries the z-1 faces and cell materials of the
// previous plane in registers, so each plane costs 7 face loads, 3 edge
// loads/stores and 4 material bytes.  Same arithmetic as fit_e_kernel.
template <typename T>
__global__ void __launch_bounds__(256) fit_e_march(FitGrid<T> g, int kchunk) {
  using A = Ar<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = blockIdx.z * kchunk;
  if (i > g.Nx || j > g.Ny || k0 > g.Nz) return;
  const int k1 = min(k0 + kchunk, g.Nz + 1);
  const T dt = (T)g.dt;
  // the E half only reads F and the materials: read-only, non-aliasing loads
  const T* __restrict__ Fx = g.Fx;
  const T* __restrict__ Fy = g.Fy;
  const T* __restrict__ Fz = g.Fz;
  T* __restrict__ Ux = g.Ux;
  T* __restrict__ Uy = g.Uy;
  T* __restrict__ Uz = g.Uz;
  const uint8_t* __restrict__ mat = g.mat;
  const bool xin = i > 0 && i < g.Nx, yin = j > 0 && j < g.Ny;
  const bool xe = i < g.Nx && yin, ye = j < g.Ny && xin, ze = xin && yin;  // column has x/y/z edges
  const bool ci0 = i > 0, ci1 = i < g.Nx, cj0 = j > 0, cj1 = j < g.Ny;
  int64_t s = (int64_t)i + g.sx * j + g.sxy * k0;
  const int64_t cb = (int64_t)(i - 1) + (int64_t)g.Nx * (j - 1);  // cell (i-1,j-1) in a plane
  const int64_t cplane = (int64_t)g.Nx * g.Ny;
  // materials of the plane below, c[dy][dx]
  uint8_t lo[2][2] = {{0, 0}, {0, 0}};
  if (k0 > 0) {
    const uint8_t* m = mat + cb + cplane * (k0 - 1);
    lo[0][0] = (ci0 && cj0) ? __ldg(m) : 0;
    lo[0][1] = (ci1 && cj0) ? __ldg(m + 1) : 0;
    lo[1][0] = (ci0 && cj1) ? __ldg(m + g.Nx) : 0;
    lo[1][1] = (ci1 && cj1) ? __ldg(m + g.Nx + 1) : 0;
  }
  T fy_lo = (k0 > 0 && xe) ? __ldg(Fy + s - g.sxy) : (T)0;
  T fx_lo = (k0 > 0 && ye) ? __ldg(Fx + s - g.sxy) : (T)0;
TF_UNROLL(TF_FIT_UNROLL)
  for (int k = k0; k < k1; k++, s += g.sxy) {
    const bool zin = k > 0 && k < g.Nz;
    uint8_t hi[2][2] = {{0, 0}, {0, 0}};
    if (k < g.Nz) {
      const uint8_t* m = mat + cb + cplane * k;
      hi[0][0] = (ci0 && cj0) ? __ldg(m) : 0;
      hi[0][1] = (ci1 && cj0) ? __ldg(m + 1) : 0;
      hi[1][0] = (ci0 && cj1) ? __ldg(m + g.Nx) : 0;
      hi[1][1] = (ci1 && cj1) ? __ldg(m + g.Nx + 1) : 0;
    }
    const T fx = (j < g.Ny && k < g.Nz) ? __ldg(Fx + s) : (T)0;
    const T fy = (i < g.Nx && k < g.Nz) ? __ldg(Fy + s) : (T)0;
    if (zin) {
      const T fz = __ldg(Fz + s);
      const bool same = lo[0][0] == lo[0][1] && lo[0][0] == lo[1][0] && lo[0][0] == lo[1][1] &&
                        lo[0][0] == hi[0][0] && lo[0][0] == hi[0][1] && lo[0][0] == hi[1][0] &&
                        lo[0][0] == hi[1][1];
      if (xe) {  // x-edge: faces Fy(k-1), Fz(j-1), Fz, Fy
        T mh, mq;
        if (same) { mh = g.mh_pure[3 * lo[0][0]]; mq = g.mq_pure[3 * lo[0][0]]; }
        else { uint8_t m[4] = {lo[0][1], lo[1][1], hi[0][1], hi[1][1]}; edge_coef_t(g, 0, m, mh, mq); }
        const T cf = A::sub(A::add(A::sub(fy_lo, __ldg(Fz + s - g.sx)), fz), fy);
        Ux[s] = A::mul(mh, A::add(A::mul(mq, Ux[s]), A::mul(dt, cf)));
      }
      if (ye) {  // y-edge: faces Fx(k-1), Fz(i-1), Fz, Fx; dual curl -1
        T mh, mq;
        if (same) { mh = g.mh_pure[3 * lo[0][0] + 1]; mq = g.mq_pure[3 * lo[0][0] + 1]; }
        else { uint8_t m[4] = {lo[1][0], lo[1][1], hi[1][0], hi[1][1]}; edge_coef_t(g, 1, m, mh, mq); }
        const T cf = -A::sub(A::add(A::sub(fx_lo, __ldg(Fz + s - 1)), fz), fx);
        Uy[s] = A::mul(mh, A::add(A::mul(mq, Uy[s]), A::mul(dt, cf)));
      }
    }
    if (ze && k < g.Nz) {  // z-edge: faces Fx(j-1), Fy(i-1), Fy, Fx
      T mh, mq;
      if (hi[0][0] == hi[0][1] && hi[0][0] == hi[1][0] && hi[0][0] == hi[1][1]) {
        mh = g.mh_pure[3 * hi[0][0] + 2];
        mq = g.mq_pure[3 * hi[0][0] + 2];
      } else {
        uint8_t m[4] = {hi[0][0], hi[0][1], hi[1][0], hi[1][1]};
        edge_coef_t(g, 2, m, mh, mq);
      }
      const T cf = A::sub(A::add(A::sub(__ldg(Fx + s - g.sx), __ldg(Fy + s - 1)), fy), fx);
      Uz[s] = A::mul(mh, A::add(A::mul(mq, Uz[s]), A::mul(dt, cf)));
    }
    fy_lo = fy;
    fx_lo = fx;
    lo[0][0] = hi[0][0]; lo[0][1] = hi[0][1]; lo[1][0] = hi[1][0]; lo[1][1] = hi[1][1];
  }
}

// New flux B of a face from F (old) and U (new); F_new = M_nu B.
template <typename T>
__device__ __forceinline__ T face_flux(T mmu, T Fold, T dtc, T cs) {
  using A = Ar<T>;
  return A::sub(A::mul(mmu, Fold), A::mul(dtc, cs));
}

template <typename T>
__device__ __forceinline__ T curl_x(const FitGrid<T>& g, int64_t s) {  // Fx at slot s
  using A = Ar<T>;
  return A::sub(A::add(A::sub(g.Uy[s], g.Uz[s]), g.Uz[s + g.sx]), g.Uy[s + g.sxy]);
}
template <typename T>
__device__ __forceinline__ T curl_y(const FitGrid<T>& g, int64_t s) {
  using A = Ar<T>;
  return A::sub(A::add(A::sub(g.Ux[s], g.Uz[s]), g.Uz[s + 1]), g.Ux[s + g.sxy]);
}
template <typename T>
__device__ __forceinline__ T curl_z(const FitGrid<T>& g, int64_t s) {
  using A = Ar<T>;
  return A::sub(A::add(A::sub(g.Ux[s], g.Uy[s]), g.Uy[s + 1]), g.Ux[s + g.sx]);
}

template <typename T>
__device__ __forceinline__ uint8_t cell_mat(const FitGrid<T>& g, int i, int j, int k) {
  return g.mat[cell_index(i, j, k, g.Nx, g.Ny)];
}

// B of face (axis a) at (i,j,k) recomputed from the current F and U; returns
// false (B = 0) for faces the H update leaves alone.
template <typename T>
__device__ bool face_B(const FitGrid<T>& g, int a, int i, int j, int k, T& B, T& mnu, T* mmu_out = nullptr) {
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const T dt = (T)g.dt;
  int li = i, lj = j, lk = k;
  bool has_lo, has_hi;
  if (a == 0) { li = i - 1; has_lo = i > 0; has_hi = i < g.Nx; }
  else if (a == 1) { lj = j - 1; has_lo = j > 0; has_hi = j < g.Ny; }
  else { lk = k - 1; has_lo = k > 0; has_hi = k < g.Nz; }
  uint8_t mlo = has_lo ? cell_mat(g, li, lj, lk) : 0, mhi = has_hi ? cell_mat(g, i, j, k) : 0;
  T mmu;
  if (!face_coef_t(g, a, has_lo, has_hi, mlo, mhi, mnu, mmu)) {
    B = (T)0;
    return false;
  }
  if (mmu_out) *mmu_out = mmu;
  if (a == 0) B = face_flux(mmu, g.Fx[s], dt, curl_x(g, s));
  else if (a == 1) B = face_flux(mmu, g.Fy[s], -dt, curl_y(g, s));
  else B = face_flux(mmu, g.Fz[s], dt, curl_z(g, s));
  return true;
}

template <typename T>
__global__ void __launch_bounds__(256) fit_h_kernel(FitGrid<T> g, int* step_counter) {
  using A = Ar<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (step_counter && i == 0 && j == 0 && k == 0) atomicAdd(step_counter, 1);
  if (i > g.Nx || j > g.Ny) return;
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const T dt = (T)g.dt;
  const bool ci = i < g.Nx, cj = j < g.Ny, ck = k < g.Nz;
  const uint8_t m0 = (ci && cj && ck) ? cell_mat(g, i, j, k) : 0;
  T mnu, mmu;
  if (cj && ck) {  // Fx(i,j,k): cells (i-1,j,k), (i,j,k)
    uint8_t ml = i > 0 ? cell_mat(g, i - 1, j, k) : 0;
    if (face_coef_t(g, 0, i > 0, ci, ml, m0, mnu, mmu)) {
      T B = face_flux(mmu, g.Fx[s], dt, curl_x(g, s));
      g.Fx[s] = A::mul(mnu, B);
    }
  }
  if (ci && ck) {  // Fy(i,j,k): cells (i,j-1,k), (i,j,k); curl -1
    uint8_t ml = j > 0 ? cell_mat(g, i, j - 1, k) : 0;
    if (face_coef_t(g, 1, j > 0, cj, ml, m0, mnu, mmu)) {
      T B = face_flux(mmu, g.Fy[s], -dt, curl_y(g, s));
      g.Fy[s] = A::mul(mnu, B);
    }
  }
  if (ci && cj) {  // Fz(i,j,k): cells (i,j,k-1), (i,j,k)
    uint8_t ml = k > 0 ? cell_mat(g, i, j, k - 1) : 0;
    if (face_coef_t(g, 2, k > 0, ck, ml, m0, mnu, mmu)) {
      T B = face_flux(mmu, g.Fz[s], dt, curl_z(g, s));
      g.Fz[s] = A::mul(mnu, B);
    }
  }
}

// H update, z-marching form: the thread owns face column (i,j) over planes
// [k0, k1), carrying Ux, Uy at plane k+1 (needed again as plane k of the next
// iteration) and the cell material below.  Same arithmetic as fit_h_kernel.
template <typename T>
__global__ void __launch_bounds__(256) fit_h_march(FitGrid<T> g, int kchunk, int* step_counter) {
  using A = Ar<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = blockIdx.z * kchunk;
  if (step_counter && i == 0 && j == 0 && k0 == 0) atomicAdd(step_counter, 1);
  if (i > g.Nx || j > g.Ny || k0 > g.Nz) return;
  const int k1 = min(k0 + kchunk, g.Nz + 1);
  const T dt = (T)g.dt;
  const bool ci = i < g.Nx, cj = j < g.Ny;
  // the H half only reads U and the materials
  const T* __restrict__ Ux = g.Ux;
  const T* __restrict__ Uy = g.Uy;
  const T* __restrict__ Uz = g.Uz;
  T* __restrict__ Fx = g.Fx;
  T* __restrict__ Fy = g.Fy;
  T* __restrict__ Fz = g.Fz;
  const uint8_t* __restrict__ mat = g.mat;
  int64_t s = (int64_t)i + g.sx * j + g.sxy * k0;
  const int64_t cplane = (int64_t)g.Nx * g.Ny;
  const int64_t cc = (int64_t)i + (int64_t)g.Nx * j;
  T ux = (ci) ? __ldg(Ux + s) : (T)0, uy = (cj) ? __ldg(Uy + s) : (T)0;
  uint8_t m_lo = (ci && cj && k0 > 0) ? __ldg(mat + cc + cplane * (k0 - 1)) : 0;
TF_UNROLL(TF_FIT_UNROLL)
  for (int k = k0; k < k1; k++, s += g.sxy) {
    const bool ck = k < g.Nz;
    const uint8_t m0 = (ci && cj && ck) ? __ldg(mat + cc + cplane * k) : 0;
    const T ux1 = (ci && ck) ? __ldg(Ux + s + g.sxy) : (T)0;
    const T uy1 = (cj && ck) ? __ldg(Uy + s + g.sxy) : (T)0;
    T mnu, mmu;
    if (cj && ck) {  // Fx(i,j,k): cells (i-1,j,k), (i,j,k)
      const uint8_t ml = i > 0 ? __ldg(mat + cc - 1 + cplane * k) : 0;
      if (face_coef_t(g, 0, i > 0, ci, ml, m0, mnu, mmu)) {
        const T cs = A::sub(A::add(A::sub(uy, __ldg(Uz + s)), __ldg(Uz + s + g.sx)), uy1);
        Fx[s] = A::mul(mnu, face_flux(mmu, Fx[s], dt, cs));
      }
    }
    if (ci && ck) {  // Fy(i,j,k): cells (i,j-1,k), (i,j,k); curl -1
      const uint8_t ml = j > 0 ? __ldg(mat + cc - g.Nx + cplane * k) : 0;
      if (face_coef_t(g, 1, j > 0, cj, ml, m0, mnu, mmu)) {
        const T cs = A::sub(A::add(A::sub(ux, __ldg(Uz + s)), __ldg(Uz + s + 1)), ux1);
        Fy[s] = A::mul(mnu, face_flux(mmu, Fy[s], -dt, cs));
      }
    }
    if (ci && cj) {  // Fz(i,j,k): cells (i,j,k-1), (i,j,k)
      if (face_coef_t(g, 2, k > 0, ck, m_lo, m0, mnu, mmu)) {
        const T cs = A::sub(A::add(A::sub(ux, uy), __ldg(Uy + s + 1)), __ldg(Ux + s + g.sx));
        Fz[s] = A::mul(mnu, face_flux(mmu, Fz[s], dt, cs));
      }
    }
    ux = ux1;
    uy = uy1;
    m_lo = m0;
  }
}

// ---------------------------------------------------------------- TMA z-march
// The same E and H updates with the face (E) or edge (H) planes a tile of
// 32 x 8 node columns needs staged in shared memory by the tensor memory
// accelerator: the elected thread of a ninth (producer) warp keeps
// kTmaStages planes in flight (cp.async.bulk.tensor into a ring of buffers,
// a "full" mbarrier per buffer with the expected byte count, an "empty"
// mbarrier the eight consumer warps release it on), the consumer warps
// compute from shared memory.
// A box covers the tile plus its one-node halo (E: the x-1 / y-1 side, H:
// the x+1 / y+1 side), its x extent rounded to 16 bytes; the E box starts
// 16 bytes left of the tile so that every x coordinate stays 16-byte aligned.
// Coordinates beyond the arrays (the halo at the domain's faces, plane -1 or
// Nz+1) read as zero and are never used unguarded.  One-GPU code: the tensor
// maps cover this GPU's arrays only, no multicast.
constexpr int kTmaTX = 32, kTmaTY = 8;
// resident blocks per SM the TMA kernels are compiled for (4: no register cap)
#ifndef TF_TMA_MINB
#define TF_TMA_MINB 4
#endif
// planes in flight: four (FP32) or three (FP64), within 48 KB of static shared memory
template <typename T>
__host__ __device__ constexpr int tma_stages() { return sizeof(T) == 4 ? 4 : 3; }
constexpr long kTmaWaitLimit = 1L << 22;  // mbarrier polls before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Shared state of one TMA march: ring buffers for three arrays per plane.
template <typename T, int BX, int BY, int kTmaStages = tma_stages<T>()>
struct TmaRing {
  static constexpr int kPlane = BX * BY;                    // elements per array and plane
  static constexpr uint32_t kBytes = 6u * kPlane * sizeof(T);  // bytes a plane's six boxes bring
  alignas(128) T buf[kTmaStages][6][kPlane + (128 / sizeof(T) - kPlane % (128 / sizeof(T))) % (128 / sizeof(T))];
  alignas(8) uint64_t full[kTmaStages];   // plane arrived: the producer's expect_tx and the copies' bytes
  alignas(8) uint64_t empty[kTmaStages];  // plane consumed: one arrival per consumer warp
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// bounded wait for the completion of the phase with this parity
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long it = 0; !mbar_try_wait(bar, parity); it++)
    if (it > kTmaWaitLimit) return false;
  return true;
}

// Ring control with a producer warp and kTmaTY consumer warps, no block-wide
// barrier per plane.  The producer's elected thread runs produce(): plane q
// of the march (global plane zbase + q) goes into buffer q % kTmaStages as
// soon as every consumer warp has released the plane that buffer held.  A
// consumer warp wait()s for a plane and release()s it when it no longer
// reads it, so consumer warps drift apart by up to kTmaStages planes.  Every
// wait is bounded: one that runs out raises *err; the consumers then return,
// the producer stops issuing and waits (bounded) for the copies it still has
// in flight, so no copy lands in the shared memory of an exited block.
template <typename T, int BX, int BY, int kTmaStages = tma_stages<T>()>
struct TmaMarch {
  TmaRing<T, BX, BY>& r;
  const CUtensorMap* m[6];  // the three staged-neighbour arrays, then the three updated ones
  int x, y, zbase, nplanes;
  int* err;
  // one thread, followed by a __syncthreads of the block
  __device__ void init(int consumers) const {
    for (int q = 0; q < kTmaStages; q++) {
      mbar_init(&r.full[q], 1);
      mbar_init(&r.empty[q], consumers);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __device__ void produce() const {
    int issued = 0;
    for (int q = 0; q < nplanes; q++) {
      const int st = q % kTmaStages;
      if (q >= kTmaStages && !mbar_wait(&r.empty[st], (uint32_t)((q / kTmaStages - 1) & 1))) {
        atomicExch(err, 1);
        break;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&r.full[st], TmaRing<T, BX, BY>::kBytes);
#pragma unroll
      for (int a = 0; a < 6; a++) tma_load_3d(r.buf[st][a], m[a], &r.full[st], x, y, zbase + q);
      issued = q + 1;
    }
    // the last kTmaStages planes issued are the only ones that can still be
    // in flight (each earlier one was released, so it had arrived)
    for (int q = issued > kTmaStages ? issued - kTmaStages : 0; q < issued; q++)
      mbar_wait(&r.full[q % kTmaStages], (uint32_t)((q / kTmaStages) & 1));
  }
  __device__ bool wait(int q) const {
    if (mbar_wait(&r.full[q % kTmaStages], (uint32_t)((q / kTmaStages) & 1))) return true;
    atomicExch(err, 1);
    return false;
  }
  __device__ void release(int q) const {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&r.empty[q % kTmaStages]);
  }
};

// H update, TMA form of fit_h_march: the boxes of plane q hold (i0 .. i0+BX-1)
// x (j0 .. j0+kTmaTY) of Ux, Uy, Uz and of the updated Fx, Fy, Fz; plane k
// uses the U of planes k and k+1 and the F of plane k.
template <typename T>
__global__ void __launch_bounds__(kTmaTX * (kTmaTY + 1), TF_TMA_MINB) fit_h_tma(FitGrid<T> g, int kchunk, int* step_counter,
                                                            const __grid_constant__ CUtensorMap mUx,
                                                            const __grid_constant__ CUtensorMap mUy,
                                                            const __grid_constant__ CUtensorMap mUz,
                                                            const __grid_constant__ CUtensorMap mFx,
                                                            const __grid_constant__ CUtensorMap mFy,
                                                            const __grid_constant__ CUtensorMap mFz, int* err) {
  using A = Ar<T>;
  constexpr int BX = kTmaTX + 16 / (int)sizeof(T), BY = kTmaTY + 1;
  constexpr int kTmaStages = tma_stages<T>();
  __shared__ TmaRing<T, BX, BY> ring;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * kTmaTX, j0 = blockIdx.y * kTmaTY, k0 = blockIdx.z * kchunk;
  const int i = i0 + tx, j = j0 + ty;
  if (step_counter && i == 0 && j == 0 && k0 == 0) atomicAdd(step_counter, 1);
  const int k1 = min(k0 + kchunk, g.Nz + 1);
  const int nplanes = k1 - k0 + 1;  // planes k0 .. k1
  const TmaMarch<T, BX, BY> mr{ring, {&mUx, &mUy, &mUz, &mFx, &mFy, &mFz}, i0, j0, k0, nplanes, err};
  if (tx == 0 && ty == 0) mr.init(kTmaTY);
  __syncthreads();
  if (ty == kTmaTY) {  // the producer warp
    if (tx == 0) mr.produce();
    return;
  }
  const bool valid = i <= g.Nx && j <= g.Ny;
  const T dt = (T)g.dt;
  const bool ci = i < g.Nx, cj = j < g.Ny;
  T* __restrict__ Fx = g.Fx;
  T* __restrict__ Fy = g.Fy;
  T* __restrict__ Fz = g.Fz;
  const uint8_t* __restrict__ mat = g.mat;
  int64_t s = (int64_t)i + g.sx * j + g.sxy * k0;
  const int64_t cplane = (int64_t)g.Nx * g.Ny;
  const int64_t cc = (int64_t)i + (int64_t)g.Nx * j;
  uint8_t m_lo = (valid && ci && cj && k0 > 0) ? __ldg(mat + cc + cplane * (k0 - 1)) : 0;
  const int o = ty * BX + tx;  // this node in a box
  if (!mr.wait(0)) return;
  for (int k = k0; k < k1; k++, s += g.sxy) {
    const int q = k - k0;
    if (!mr.wait(q + 1)) return;
    const T* Ux = ring.buf[q % kTmaStages][0];
    const T* Uy = ring.buf[q % kTmaStages][1];
    const T* Uz = ring.buf[q % kTmaStages][2];
    const T* Ux1 = ring.buf[(q + 1) % kTmaStages][0];
    const T* Uy1 = ring.buf[(q + 1) % kTmaStages][1];
    const T* Fxs = ring.buf[q % kTmaStages][3];
    const T* Fys = ring.buf[q % kTmaStages][4];
    const T* Fzs = ring.buf[q % kTmaStages][5];
    if (valid) {
      const bool ck = k < g.Nz;
      const uint8_t m0 = (ci && cj && ck) ? __ldg(mat + cc + cplane * k) : 0;
      const T ux = ci ? Ux[o] : (T)0, uy = cj ? Uy[o] : (T)0;
      const T ux1 = (ci && ck) ? Ux1[o] : (T)0, uy1 = (cj && ck) ? Uy1[o] : (T)0;
      T mnu, mmu;
      if (cj && ck) {  // Fx(i,j,k): cells (i-1,j,k), (i,j,k)
        const uint8_t ml = i > 0 ? __ldg(mat + cc - 1 + cplane * k) : 0;
        if (face_coef_t(g, 0, i > 0, ci, ml, m0, mnu, mmu)) {
          const T cs = A::sub(A::add(A::sub(uy, Uz[o]), Uz[o + BX]), uy1);
          Fx[s] = A::mul(mnu, face_flux(mmu, Fxs[o], dt, cs));
        }
      }
      if (ci && ck) {  // Fy(i,j,k): cells (i,j-1,k), (i,j,k); curl -1
        const uint8_t ml = j > 0 ? __ldg(mat + cc - g.Nx + cplane * k) : 0;
        if (face_coef_t(g, 1, j > 0, cj, ml, m0, mnu, mmu)) {
          const T cs = A::sub(A::add(A::sub(ux, Uz[o]), Uz[o + 1]), ux1);
          Fy[s] = A::mul(mnu, face_flux(mmu, Fys[o], -dt, cs));
        }
      }
      if (ci && cj) {  // Fz(i,j,k): cells (i,j,k-1), (i,j,k)
        if (face_coef_t(g, 2, k > 0, ck, m_lo, m0, mnu, mmu)) {
          const T cs = A::sub(A::add(A::sub(ux, uy), Uy[o + 1]), Ux[o + BX]);
          Fz[s] = A::mul(mnu, face_flux(mmu, Fzs[o], dt, cs));
        }
      }
      m_lo = m0;
    }
    mr.release(q);  // plane q is not read again
  }
}

// E update, TMA form of fit_e_march: the boxes of plane q hold
// (i0-H .. i0+kTmaTX-1) x (j0-1 .. j0+kTmaTY-1) of Fx, Fy, Fz and of the
// updated Ux, Uy, Uz, H = 16 bytes of elements; plane k uses the F of planes
// k-1 and k and the U of plane k.
template <typename T>
__global__ void __launch_bounds__(kTmaTX * (kTmaTY + 1), TF_TMA_MINB) fit_e_tma(FitGrid<T> g, int kchunk,
                                                            const __grid_constant__ CUtensorMap mFx,
                                                            const __grid_constant__ CUtensorMap mFy,
                                                            const __grid_constant__ CUtensorMap mFz,
                                                            const __grid_constant__ CUtensorMap mUx,
                                                            const __grid_constant__ CUtensorMap mUy,
                                                            const __grid_constant__ CUtensorMap mUz, int* err) {
  using A = Ar<T>;
  constexpr int H = 16 / (int)sizeof(T);
  constexpr int BX = kTmaTX + H, BY = kTmaTY + 1;
  constexpr int kTmaStages = tma_stages<T>();
  __shared__ TmaRing<T, BX, BY> ring;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * kTmaTX, j0 = blockIdx.y * kTmaTY, k0 = blockIdx.z * kchunk;
  const int i = i0 + tx, j = j0 + ty;
  const int k1 = min(k0 + kchunk, g.Nz + 1);
  const int nplanes = k1 - k0 + 1;  // planes k0-1 .. k1-1
  const TmaMarch<T, BX, BY> mr{ring, {&mFx, &mFy, &mFz, &mUx, &mUy, &mUz}, i0 - H, j0 - 1, k0 - 1, nplanes, err};
  if (tx == 0 && ty == 0) mr.init(kTmaTY);
  __syncthreads();
  if (ty == kTmaTY) {  // the producer warp
    if (tx == 0) mr.produce();
    return;
  }
  const bool valid = i <= g.Nx && j <= g.Ny;
  const T dt = (T)g.dt;
  T* __restrict__ Ux = g.Ux;
  T* __restrict__ Uy = g.Uy;
  T* __restrict__ Uz = g.Uz;
  const uint8_t* __restrict__ mat = g.mat;
  const bool xin = i > 0 && i < g.Nx, yin = j > 0 && j < g.Ny;
  const bool xe = i < g.Nx && yin, ye = j < g.Ny && xin, ze = xin && yin;
  const bool ci0 = i > 0, ci1 = i < g.Nx, cj0 = j > 0, cj1 = j < g.Ny;
  int64_t s = (int64_t)i + g.sx * j + g.sxy * k0;
  const int64_t cb = (int64_t)(i - 1) + (int64_t)g.Nx * (j - 1);
  const int64_t cplane = (int64_t)g.Nx * g.Ny;
  uint8_t lo[2][2] = {{0, 0}, {0, 0}};
  if (valid && k0 > 0) {
    const uint8_t* m = mat + cb + cplane * (k0 - 1);
    lo[0][0] = (ci0 && cj0) ? __ldg(m) : 0;
    lo[0][1] = (ci1 && cj0) ? __ldg(m + 1) : 0;
    lo[1][0] = (ci0 && cj1) ? __ldg(m + g.Nx) : 0;
    lo[1][1] = (ci1 && cj1) ? __ldg(m + g.Nx + 1) : 0;
  }
  const int o = (ty + 1) * BX + tx + H;  // this node in a box
  if (!mr.wait(0)) return;
  for (int k = k0; k < k1; k++, s += g.sxy) {
    const int q = k - k0;  // plane k-1 is ring plane q, plane k is q + 1
    if (!mr.wait(q + 1)) return;
    const T* Fxl = ring.buf[q % kTmaStages][0];
    const T* Fyl = ring.buf[q % kTmaStages][1];
    const T* Fx = ring.buf[(q + 1) % kTmaStages][0];
    const T* Fy = ring.buf[(q + 1) % kTmaStages][1];
    const T* Fz = ring.buf[(q + 1) % kTmaStages][2];
    const T* Uxs = ring.buf[(q + 1) % kTmaStages][3];
    const T* Uys = ring.buf[(q + 1) % kTmaStages][4];
    const T* Uzs = ring.buf[(q + 1) % kTmaStages][5];
    if (valid) {
      const bool zin = k > 0 && k < g.Nz;
      uint8_t hi[2][2] = {{0, 0}, {0, 0}};
      if (k < g.Nz) {
        const uint8_t* m = mat + cb + cplane * k;
        hi[0][0] = (ci0 && cj0) ? __ldg(m) : 0;
        hi[0][1] = (ci1 && cj0) ? __ldg(m + 1) : 0;
        hi[1][0] = (ci0 && cj1) ? __ldg(m + g.Nx) : 0;
        hi[1][1] = (ci1 && cj1) ? __ldg(m + g.Nx + 1) : 0;
      }
      const T fx = (j < g.Ny && k < g.Nz) ? Fx[o] : (T)0;
      const T fy = (i < g.Nx && k < g.Nz) ? Fy[o] : (T)0;
      if (zin) {
        const T fz = Fz[o];
        const bool same = lo[0][0] == lo[0][1] && lo[0][0] == lo[1][0] && lo[0][0] == lo[1][1] &&
                          lo[0][0] == hi[0][0] && lo[0][0] == hi[0][1] && lo[0][0] == hi[1][0] &&
                          lo[0][0] == hi[1][1];
        if (xe) {  // x-edge: faces Fy(k-1), Fz(j-1), Fz, Fy
          T mh, mq;
          if (same) { mh = g.mh_pure[3 * lo[0][0]]; mq = g.mq_pure[3 * lo[0][0]]; }
          else { uint8_t m[4] = {lo[0][1], lo[1][1], hi[0][1], hi[1][1]}; edge_coef_t(g, 0, m, mh, mq); }
          const T cf = A::sub(A::add(A::sub(Fyl[o], Fz[o - BX]), fz), fy);
          Ux[s] = A::mul(mh, A::add(A::mul(mq, Uxs[o]), A::mul(dt, cf)));
        }
        if (ye) {  // y-edge: faces Fx(k-1), Fz(i-1), Fz, Fx; dual curl -1
          T mh, mq;
          if (same) { mh = g.mh_pure[3 * lo[0][0] + 1]; mq = g.mq_pure[3 * lo[0][0] + 1]; }
          else { uint8_t m[4] = {lo[1][0], lo[1][1], hi[1][0], hi[1][1]}; edge_coef_t(g, 1, m, mh, mq); }
          const T cf = -A::sub(A::add(A::sub(Fxl[o], Fz[o - 1]), fz), fx);
          Uy[s] = A::mul(mh, A::add(A::mul(mq, Uys[o]), A::mul(dt, cf)));
        }
      }
      if (ze && k < g.Nz) {  // z-edge: faces Fx(j-1), Fy(i-1), Fy, Fx
        T mh, mq;
        if (hi[0][0] == hi[0][1] && hi[0][0] == hi[1][0] && hi[0][0] == hi[1][1]) {
          mh = g.mh_pure[3 * hi[0][0] + 2];
          mq = g.mq_pure[3 * hi[0][0] + 2];
        } else {
          uint8_t m[4] = {hi[0][0], hi[0][1], hi[1][0], hi[1][1]};
          edge_coef_t(g, 2, m, mh, mq);
        }
        const T cf = A::sub(A::add(A::sub(Fx[o - BX], Fy[o - 1]), fy), fx);
        Uz[s] = A::mul(mh, A::add(A::mul(mq, Uzs[o]), A::mul(dt, cf)));
      }
      lo[0][0] = hi[0][0]; lo[0][1] = hi[0][1]; lo[1][0] = hi[1][0]; lo[1][1] = hi[1][1];
    }
    mr.release(q);
  }
}

template <typename T>
__device__ __forceinline__ T* comp_ptr(T* x, T* y, T* z, int c) {
  return c == 0 ? x : (c == 1 ? y : z);
}

// Special edges: new values into sp.out, flux partial sums per block.
template <typename T>
__global__ void __launch_bounds__(256) fit_special_pre(FitGrid<T> g, SpecialEdges<T> sp, const int* step_counter) {
  using A = Ar<T>;
  __shared__ double red[256];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int step = *step_counter;
  double contrib = 0.0;
  if (e < sp.n) {
    T* U = comp_ptr(g.Ux, g.Uy, g.Uz, sp.comp[e]);
    const int64_t slot = sp.slot[e];
    const T Uo = U[slot];
    // source value: sum of source vectors, dotted with the projection vector
    double v[3] = {0.0, 0.0, 0.0};
    int kind = 0;
    for (int p = sp.src_begin[e]; p < sp.src_begin[e + 1]; p++) {
      const int si = sp.pair_src[p];
      kind = sp.src_kind[si] + 1;
      double ret = __dmul_rn(sp.src_amp[si], sp.carrier[(int64_t)step * sp.nsrc + si]);
      ret = __dmul_rn(ret, sp.pair_fac[4 * p + 0]);
      ret = __dmul_rn(ret, sp.pair_fac[4 * p + 1]);
      ret = __dmul_rn(ret, sp.pair_fac[4 * p + 2]);
      ret = __dmul_rn(ret, sp.pair_fac[4 * p + 3]);
      const int d = sp.pair_dir[p];
      v[d] = __dadd_rn(v[d], ret);
    }
    double val = 0.0;
    if (kind) {
      const double* w = sp.pair_vec + 3 * (int64_t)e;
      val = __dadd_rn(__dadd_rn(__dmul_rn(v[0], w[0]), __dmul_rn(v[1], w[1])), __dmul_rn(v[2], w[2]));
      val = __dmul_rn(sp.post[e], val);
    }
    const int op = sp.op[e];
    T Un;
    if (op == 0) {
      Un = kind == 1 ? (T)val : (T)0;
    } else {
      const T dt = (T)g.dt;
      T f[4];
      const int nf = sp.nface[e];
      for (int q = 0; q < 4; q++) {
        f[q] = (T)0;
        if (q < nf) {
          const T* F = comp_ptr(g.Fx, g.Fy, g.Fz, sp.fcomp[4 * e + q]);
          f[q] = F[sp.fslot[4 * e + q]];
        }
      }
      const T I = kind == 3 ? (T)val : (T)0;
      const T mh = (T)sp.mh[e], mq = (T)sp.mq[e];
      T cf;
      if (op == 1) {  // explicit signed faces, Eigen 3-vector dot order
        T acc = A::add(A::mul(f[0], (T)sp.fsign[4 * e]), A::mul(f[1], (T)sp.fsign[4 * e + 1]));
        acc = A::add(acc, A::mul(f[2], (T)sp.fsign[4 * e + 2]));
        if (nf > 3) acc = A::add(acc, A::mul(f[3], (T)sp.fsign[4 * e + 3]));
        const T cfb = kind == 2 ? (T)val : (T)0;
        cf = A::sub(A::add(acc, cfb), I);
        Un = A::mul(mh, A::add(A::mul(mq, Uo), A::mul(dt, cf)));
        contrib = __dmul_rn(__dadd_rn((double)Uo, (double)Un), (double)cfb);
      } else {  // interior stencil with a dipole current
        T st = A::sub(A::add(A::sub(f[0], f[1]), f[2]), f[3]);
        cf = A::sub(A::mul((T)sp.fsign[4 * e], st), I);
        Un = A::mul(mh, A::add(A::mul(mq, Uo), A::mul(dt, cf)));
      }
    }
    sp.out[e] = Un;
  }
  red[threadIdx.x] = contrib;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) sp.flux_part[blockIdx.x] = red[0];
}

template <typename T>
__global__ void __launch_bounds__(256) fit_special_post(FitGrid<T> g, SpecialEdges<T> sp, const int* step_counter,
                                                         double* flux, int nparts) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < sp.n) {
    T* U = comp_ptr(g.Ux, g.Uy, g.Uz, sp.comp[e]);
    U[sp.slot[e]] = sp.out[e];
  }
  if (blockIdx.x == 0) {
    // fixed-order reduction of the per-block flux partials
    __shared__ double red[256];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) acc = __dadd_rn(acc, sp.flux_part[b]);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
      __syncthreads();
    }
    if (threadIdx.x == 0) flux[*step_counter] = __dmul_rn(0.5, red[0]);
  }
}

template <typename T>
__global__ void fit_probe_kernel(FitGrid<T> g, ProbeSet pr, const int* step_counter) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pr.n) return;
  const int slotn = pr.slot_of_step[*step_counter];
  if (slotn < 0) return;
  const int i = pr.ci[p], j = pr.cj[p], k = pr.ck[p];
  const double Lx = g.len[0], Ly = g.len[1], Lz = g.len[2];
  const double vol = __dmul_rn(__dmul_rn(Lx, Ly), Lz);
  const double dax = __dmul_rn(Ly, Lz) / 4, day = __dmul_rn(Lx, Lz) / 4, daz = __dmul_rn(Lx, Ly) / 4;
  auto U = [&](const T* a, int ii, int jj, int kk) { return (double)a[(int64_t)ii + g.sx * jj + g.sxy * kk]; };
  auto sum4 = [&](double a, double b, double c, double d, double w) {
    return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, w), __dmul_rn(b, w)), __dmul_rn(c, w)), __dmul_rn(d, w));
  };
  double* out = pr.samples + ((int64_t)slotn * pr.n + p) * 6;
  out[0] = sum4(U(g.Ux, i, j, k), U(g.Ux, i, j + 1, k), U(g.Ux, i, j, k + 1), U(g.Ux, i, j + 1, k + 1), dax) / vol;
  out[1] = sum4(U(g.Uy, i, j, k), U(g.Uy, i + 1, j, k), U(g.Uy, i, j, k + 1), U(g.Uy, i + 1, j, k + 1), day) / vol;
  out[2] = sum4(U(g.Uz, i, j, k), U(g.Uz, i + 1, j, k), U(g.Uz, i, j + 1, k), U(g.Uz, i + 1, j + 1, k), daz) / vol;
  const double half[3] = {__dmul_rn(0.5, Lx), __dmul_rn(0.5, Ly), __dmul_rn(0.5, Lz)};
  for (int a = 0; a < 3; a++) {
    T B0, B1, nu;
    face_B(g, a, i, j, k, B0, nu);
    face_B(g, a, i + (a == 0), j + (a == 1), k + (a == 2), B1, nu);
    double h = __dadd_rn(__dmul_rn((double)B0, half[a]), __dmul_rn((double)B1, half[a]));
    out[3 + a] = __dmul_rn(pr.inv_mu[3 * p + a], h) / vol;
  }
}

// ---------------------------------------------------- per-dof coefficients
// M_h, M_q of the interior stencil edges leaving node slot (i,j,k) and M_nu,
// M_mu of the faces at that slot, with the same functions (and so the same
// rounded values) the table-driven kernels use.
template <typename T>
__global__ void __launch_bounds__(256) fit_coef_kernel(FitGrid<T> g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.Nx || j > g.Ny) return;
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const bool xin = i > 0 && i < g.Nx, yin = j > 0 && j < g.Ny, zin = k > 0 && k < g.Nz;
  uint8_t c[2][2][2];
#pragma unroll
  for (int dz = 0; dz < 2; dz++)
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
      for (int dx = 0; dx < 2; dx++) {
        int ci = i - 1 + dx, cj = j - 1 + dy, ck = k - 1 + dz;
        bool ok = ci >= 0 && ci < g.Nx && cj >= 0 && cj < g.Ny && ck >= 0 && ck < g.Nz;
        c[dz][dy][dx] = ok ? g.mat[cell_index(ci, cj, ck, g.Nx, g.Ny)] : 0;
      }
  T mh = 0, mq = 0;
  if (i < g.Nx && yin && zin) {
    uint8_t m[4] = {c[0][0][1], c[0][1][1], c[1][0][1], c[1][1][1]};
    edge_coef_t(g, 0, m, mh, mq);
    g.Ch[0][s] = mh;
    g.Cq[0][s] = mq;
  }
  if (j < g.Ny && xin && zin) {
    uint8_t m[4] = {c[0][1][0], c[0][1][1], c[1][1][0], c[1][1][1]};
    edge_coef_t(g, 1, m, mh, mq);
    g.Ch[1][s] = mh;
    g.Cq[1][s] = mq;
  }
  if (k < g.Nz && xin && yin) {
    uint8_t m[4] = {c[1][0][0], c[1][0][1], c[1][1][0], c[1][1][1]};
    edge_coef_t(g, 2, m, mh, mq);
    g.Ch[2][s] = mh;
    g.Cq[2][s] = mq;
  }
  const bool ci = i < g.Nx, cj = j < g.Ny, ck = k < g.Nz;
  const uint8_t m0 = (ci && cj && ck) ? c[1][1][1] : 0;
  T mnu, mmu;
  if (cj && ck) {
    const uint8_t ml = i > 0 ? c[1][1][0] : 0;
    const bool live = face_coef_t(g, 0, i > 0, ci, ml, m0, mnu, mmu);
    g.Cn[0][s] = live ? mnu : (T)-0.0;
    g.Cm[0][s] = live ? mmu : (T)0;
  }
  if (ci && ck) {
    const uint8_t ml = j > 0 ? c[1][0][1] : 0;
    const bool live = face_coef_t(g, 1, j > 0, cj, ml, m0, mnu, mmu);
    g.Cn[1][s] = live ? mnu : (T)-0.0;
    g.Cm[1][s] = live ? mmu : (T)0;
  }
  if (ci && cj) {
    const uint8_t ml = k > 0 ? c[0][1][1] : 0;
    const bool live = face_coef_t(g, 2, k > 0, ck, ml, m0, mnu, mmu);
    g.Cn[2][s] = live ? mnu : (T)-0.0;
    g.Cm[2][s] = live ? mmu : (T)0;
  }
}

template <typename T>
cudaError_t fit_build_coefficients(const FitGrid<T>& g, cudaStream_t st) {
  dim3 blk(32, 8, 1);
  dim3 grd((unsigned)((g.Nx + 1 + 31) / 32), (unsigned)((g.Ny + 1 + 7) / 8), (unsigned)(g.Nz + 1));
  fit_coef_kernel<T><<<grd, blk, 0, st>>>(g);
  return cudaGetLastError();
}
template cudaError_t fit_build_coefficients<double>(const FitGrid<double>&, cudaStream_t);
template cudaError_t fit_build_coefficients<float>(const FitGrid<float>&, cudaStream_t);

// ------------------------------------------------------------ coefficient classes
// An edge's coefficients are a function of its axis and the materials of its
// four cells (cells outside the grid read as material 0, as above), a face's
// of its axis, which of its two cells exist, and their materials.  The build
// packs each updated dof's tuple into a 64-bit key, inserts the keys into an
// open-addressing hash table (linear probing; MurmurHash3's 64-bit finalizer
// as the hash), numbers the occupied slots, computes one coefficient pair per
// class with edge_coef_t / face_coef_t, and writes each dof's class.  Class
// numbers depend on insertion order; the coefficients a dof reads do not.
constexpr unsigned long long kNoKey = ~0ull;

__device__ __forceinline__ uint32_t class_hash(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return (uint32_t)k & (kClassTable - 1);
}

__device__ __forceinline__ int class_insert(unsigned long long* keys, unsigned long long k) {
  uint32_t h = class_hash(k);
  for (int p = 0; p < kClassTable; p++, h = (h + 1) & (kClassTable - 1)) {
    const unsigned long long cur = *(volatile unsigned long long*)&keys[h];
    if (cur == k) return (int)h;
    if (cur == kNoKey) {
      const unsigned long long prev = atomicCAS(&keys[h], kNoKey, k);
      if (prev == kNoKey || prev == k) return (int)h;
    }
  }
  return -1;
}

__device__ __forceinline__ int class_find(const unsigned long long* keys, unsigned long long k) {
  uint32_t h = class_hash(k);
  for (int p = 0; p < kClassTable; p++, h = (h + 1) & (kClassTable - 1)) {
    const unsigned long long cur = keys[h];
    if (cur == k) return (int)h;
    if (cur == kNoKey) return -1;
  }
  return -1;
}

__device__ __forceinline__ unsigned long long edge_key(int a, const uint8_t m[4]) {
  return ((unsigned long long)a << 32) | (uint32_t)m[0] | ((uint32_t)m[1] << 8) | ((uint32_t)m[2] << 16) |
         ((uint32_t)m[3] << 24);
}
__device__ __forceinline__ unsigned long long face_key(int a, bool has_lo, bool has_hi, uint8_t mlo, uint8_t mhi) {
  return ((unsigned long long)a << 32) | (uint32_t)has_lo | ((uint32_t)has_hi << 1) | ((uint32_t)mlo << 8) |
         ((uint32_t)mhi << 16);
}

// The tuples of the dofs at node slot (i, j, k), in the order and under the
// conditions fit_coef_kernel uses; f(kind, axis, key, slot) per updated dof,
// kind 0 edge, 1 face.
template <typename T, typename F>
__device__ __forceinline__ void for_each_dof_key(const FitGrid<T>& g, int i, int j, int k, F f) {
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const bool xin = i > 0 && i < g.Nx, yin = j > 0 && j < g.Ny, zin = k > 0 && k < g.Nz;
  uint8_t c[2][2][2];
#pragma unroll
  for (int dz = 0; dz < 2; dz++)
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
      for (int dx = 0; dx < 2; dx++) {
        const int ci = i - 1 + dx, cj = j - 1 + dy, ck = k - 1 + dz;
        const bool ok = ci >= 0 && ci < g.Nx && cj >= 0 && cj < g.Ny && ck >= 0 && ck < g.Nz;
        c[dz][dy][dx] = ok ? g.mat[cell_index(ci, cj, ck, g.Nx, g.Ny)] : 0;
      }
  if (i < g.Nx && yin && zin) {
    const uint8_t m[4] = {c[0][0][1], c[0][1][1], c[1][0][1], c[1][1][1]};
    f(0, 0, edge_key(0, m), s);
  }
  if (j < g.Ny && xin && zin) {
    const uint8_t m[4] = {c[0][1][0], c[0][1][1], c[1][1][0], c[1][1][1]};
    f(0, 1, edge_key(1, m), s);
  }
  if (k < g.Nz && xin && yin) {
    const uint8_t m[4] = {c[1][0][0], c[1][0][1], c[1][1][0], c[1][1][1]};
    f(0, 2, edge_key(2, m), s);
  }
  const bool ci = i < g.Nx, cj = j < g.Ny, ck = k < g.Nz;
  const uint8_t m0 = (ci && cj && ck) ? c[1][1][1] : 0;
  if (cj && ck) f(1, 0, face_key(0, i > 0, ci, i > 0 ? c[1][1][0] : 0, m0), s);
  if (ci && ck) f(1, 1, face_key(1, j > 0, cj, j > 0 ? c[1][0][1] : 0, m0), s);
  if (ci && cj) f(1, 2, face_key(2, k > 0, ck, k > 0 ? c[0][1][1] : 0, m0), s);
}

template <typename T>
__global__ void __launch_bounds__(256) fit_class_insert(FitGrid<T> g, FitClassWork w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.Nx || j > g.Ny) return;
  for_each_dof_key(g, i, j, k, [&](int kind, int, unsigned long long key, int64_t) {
    if (class_insert(w.keys[kind], key) < 0) atomicExch(&w.count[2], 1);
  });
}

// One thread per table slot: number the occupied slots and fill the tables.
template <typename T>
__global__ void __launch_bounds__(256) fit_class_number(FitGrid<T> g, FitClassWork w, int kind) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= kClassTable) return;
  const unsigned long long key = w.keys[kind][h];
  if (key == kNoKey) return;
  const int id = atomicAdd(&w.count[kind], 1);
  w.ids[kind][h] = id;
  if (id >= kMaxClasses) return;
  const int a = (int)(key >> 32);
  if (kind == 0) {
    const uint8_t m[4] = {(uint8_t)key, (uint8_t)(key >> 8), (uint8_t)(key >> 16), (uint8_t)(key >> 24)};
    T mh, mq;
    edge_coef_t(g, a, m, mh, mq);
    g.lut_e[2 * id] = mh;
    g.lut_e[2 * id + 1] = mq;
  } else {
    T mnu, mmu;
    const bool live = face_coef_t(g, a, (key & 1) != 0, (key & 2) != 0, (uint8_t)(key >> 8), (uint8_t)(key >> 16),
                                  mnu, mmu);
    g.lut_f[2 * id] = live ? mnu : (T)-0.0;
    g.lut_f[2 * id + 1] = live ? mmu : (T)0;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) fit_class_assign(FitGrid<T> g, FitClassWork w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.Nx || j > g.Ny) return;
  for_each_dof_key(g, i, j, k, [&](int kind, int a, unsigned long long key, int64_t s) {
    const int h = class_find(w.keys[kind], key);
    const uint16_t c = (uint16_t)(h >= 0 ? w.ids[kind][h] : 0);
    if (kind == 0) g.Ke[a][s] = c;
    else g.Kf[a][s] = c;
  });
}

template <typename T>
cudaError_t fit_build_classes(const FitGrid<T>& g, const FitClassWork& w, int ncls[2], cudaStream_t st) {
  for (int q = 0; q < 2; q++)
    if (cudaMemsetAsync(w.keys[q], 0xff, sizeof(unsigned long long) * kClassTable, st) != cudaSuccess)
      return cudaGetLastError();
  if (cudaMemsetAsync(w.count, 0, 3 * sizeof(int), st) != cudaSuccess) return cudaGetLastError();
  dim3 blk(32, 8, 1);
  dim3 grd((unsigned)((g.Nx + 1 + 31) / 32), (unsigned)((g.Ny + 1 + 7) / 8), (unsigned)(g.Nz + 1));
  fit_class_insert<T><<<grd, blk, 0, st>>>(g, w);
  for (int q = 0; q < 2; q++) fit_class_number<T><<<kClassTable / 256, 256, 0, st>>>(g, w, q);
  int c[3] = {0, 0, 0};
  cudaMemcpyAsync(c, w.count, sizeof(c), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  for (int q = 0; q < 2; q++) ncls[q] = (c[2] || c[q] > kMaxClasses) ? -1 : c[q];
  if (ncls[0] < 0 || ncls[1] < 0) return cudaSuccess;
  fit_class_assign<T><<<grd, blk, 0, st>>>(g, w);
  return cudaGetLastError();
}
template cudaError_t fit_build_classes<double>(const FitGrid<double>&, const FitClassWork&, int*, cudaStream_t);
template cudaError_t fit_build_classes<float>(const FitGrid<float>&, const FitClassWork&, int*, cudaStream_t);

// Plane-per-block E and H updates with the coefficients streamed per dof
// (CLS false: M_h, M_q / M_nu, M_mu arrays) or looked up by class (CLS true:
// a 2-byte class per dof into the class tables); same arithmetic as
// fit_e_kernel / fit_h_kernel.  Every load of a node comes first and the
// stores last: the six arrays do not alias, which the compiler cannot know,
// and with stores in between it would wait for each dof's loads in turn.
template <typename T, bool CLS>
__device__ __forceinline__ void coef_pair(const T* const* C0, const T* const* C1, const uint16_t* const* K,
                                          const T* lut, int a, int64_t s, T& c0, T& c1) {
  if (CLS) {
    const int c = __ldg(K[a] + s);
    c0 = __ldg(lut + 2 * c);
    c1 = __ldg(lut + 2 * c + 1);
  } else {
    c0 = __ldg(C0[a] + s);
    c1 = __ldg(C1[a] + s);
  }
}

template <typename T, bool CLS>
__device__ __forceinline__ void e_update_streamed(const FitGrid<T>& g) {
  using A = Ar<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.Nx || j > g.Ny) return;
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const T dt = (T)g.dt;
  const bool xin = i > 0 && i < g.Nx, yin = j > 0 && j < g.Ny, zin = k > 0 && k < g.Nz;
  const bool ex = i < g.Nx && yin && zin, ey = j < g.Ny && xin && zin, ez = k < g.Nz && xin && yin;
  T fx = 0, fy = 0, fz = 0, fy_b = 0, fz_y = 0, fx_b = 0, fz_x = 0, fx_y = 0, fy_x = 0, ux = 0, uy = 0, uz = 0;
  T h0 = 0, q0 = 0, h1 = 0, q1 = 0, h2 = 0, q2 = 0;
  if (ex || ey) fz = g.Fz[s];
  if (ex || ez) fy = g.Fy[s];
  if (ey || ez) fx = g.Fx[s];
  if (ex) {
    fy_b = g.Fy[s - g.sxy];
    fz_y = g.Fz[s - g.sx];
    ux = g.Ux[s];
    coef_pair<T, CLS>(g.Ch, g.Cq, g.Ke, g.lut_e, 0, s, h0, q0);
  }
  if (ey) {
    fx_b = g.Fx[s - g.sxy];
    fz_x = g.Fz[s - 1];
    uy = g.Uy[s];
    coef_pair<T, CLS>(g.Ch, g.Cq, g.Ke, g.lut_e, 1, s, h1, q1);
  }
  if (ez) {
    fx_y = g.Fx[s - g.sx];
    fy_x = g.Fy[s - 1];
    uz = g.Uz[s];
    coef_pair<T, CLS>(g.Ch, g.Cq, g.Ke, g.lut_e, 2, s, h2, q2);
  }
  if (ex) {
    const T cf = A::sub(A::add(A::sub(fy_b, fz_y), fz), fy);
    g.Ux[s] = A::mul(h0, A::add(A::mul(q0, ux), A::mul(dt, cf)));
  }
  if (ey) {
    const T cf = -A::sub(A::add(A::sub(fx_b, fz_x), fz), fx);
    g.Uy[s] = A::mul(h1, A::add(A::mul(q1, uy), A::mul(dt, cf)));
  }
  if (ez) {
    const T cf = A::sub(A::add(A::sub(fx_y, fy_x), fy), fx);
    g.Uz[s] = A::mul(h2, A::add(A::mul(q2, uz), A::mul(dt, cf)));
  }
}

// A skipped face (M_nu = -0.0) gets its own value back.
template <typename T, bool CLS>
__device__ __forceinline__ void h_update_streamed(const FitGrid<T>& g, int* step_counter) {
  using A = Ar<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (step_counter && i == 0 && j == 0 && k == 0) atomicAdd(step_counter, 1);
  if (i > g.Nx || j > g.Ny) return;
  const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
  const T dt = (T)g.dt;
  const bool ci = i < g.Nx, cj = j < g.Ny, ck = k < g.Nz;
  const bool hx = cj && ck, hy = ci && ck, hz = ci && cj;
  T ux = 0, uy = 0, uz = 0, uz_y = 0, uy_z = 0, uz_x = 0, ux_z = 0, uy_x = 0, ux_y = 0, fx = 0, fy = 0, fz = 0;
  T n0 = 0, m0 = 0, n1 = 0, m1 = 0, n2 = 0, m2 = 0;
  if (hy || hz) ux = g.Ux[s];
  if (hx || hz) uy = g.Uy[s];
  if (hx || hy) uz = g.Uz[s];
  if (hx) {
    uz_y = g.Uz[s + g.sx];
    uy_z = g.Uy[s + g.sxy];
    fx = g.Fx[s];
    coef_pair<T, CLS>(g.Cn, g.Cm, g.Kf, g.lut_f, 0, s, n0, m0);
  }
  if (hy) {
    uz_x = g.Uz[s + 1];
    ux_z = g.Ux[s + g.sxy];
    fy = g.Fy[s];
    coef_pair<T, CLS>(g.Cn, g.Cm, g.Kf, g.lut_f, 1, s, n1, m1);
  }
  if (hz) {
    uy_x = g.Uy[s + 1];
    ux_y = g.Ux[s + g.sx];
    fz = g.Fz[s];
    coef_pair<T, CLS>(g.Cn, g.Cm, g.Kf, g.lut_f, 2, s, n2, m2);
  }
  auto skip = [](T v) { return v == (T)0 && signbit(v); };
  if (hx) {
    const T cs = A::sub(A::add(A::sub(uy, uz), uz_y), uy_z);
    g.Fx[s] = skip(n0) ? fx : A::mul(n0, face_flux(m0, fx, dt, cs));
  }
  if (hy) {
    const T cs = A::sub(A::add(A::sub(ux, uz), uz_x), ux_z);
    g.Fy[s] = skip(n1) ? fy : A::mul(n1, face_flux(m1, fy, -dt, cs));
  }
  if (hz) {
    const T cs = A::sub(A::add(A::sub(ux, uy), uy_x), ux_y);
    g.Fz[s] = skip(n2) ? fz : A::mul(n2, face_flux(m2, fz, dt, cs));
  }
}

template <typename T>
__global__ void __launch_bounds__(256) fit_e_coef(FitGrid<T> g) { e_update_streamed<T, false>(g); }
template <typename T>
__global__ void __launch_bounds__(256) fit_h_coef(FitGrid<T> g, int* step_counter) {
  h_update_streamed<T, false>(g, step_counter);
}
template <typename T>
__global__ void __launch_bounds__(256) fit_e_class(FitGrid<T> g) { e_update_streamed<T, true>(g); }
template <typename T>
__global__ void __launch_bounds__(256) fit_h_class(FitGrid<T> g, int* step_counter) {
  h_update_streamed<T, true>(g, step_counter);
}

// Joule loss partials: one thread per node slot sums Si_e (U_old + U)_e^2 over
// the x, y and z edges leaving the node, Si_e = (sum of da_a sigma over the
// edge's cells) / L_a (Discretization.hpp:5294-5330, :5597); FP64 throughout.
template <typename T>
__global__ void __launch_bounds__(256) fit_loss_kernel(FitGrid<T> g, FitLoss<T> lb) {
  __shared__ double red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  double acc = 0.0;
  if (i <= g.Nx && j <= g.Ny) {
    const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
    const T* Us[3] = {g.Ux, g.Uy, g.Uz};
    const T* Os[3] = {lb.Ox, lb.Oy, lb.Oz};
    const bool valid[3] = {i < g.Nx, j < g.Ny, k < g.Nz};
    for (int a = 0; a < 3; a++) {
      if (!valid[a]) continue;
      // the edge's cells: offsets -1/0 on the two axes other than a
      double sig = 0.0, eps = 0.0;
      for (int q = 0; q < 4; q++) {
        int ci = i, cj = j, ck = k;
        const int d0 = (q & 1) - 1, d1 = ((q >> 1) & 1) - 1;
        if (a == 0) { cj += d0; ck += d1; }
        else if (a == 1) { ci += d0; ck += d1; }
        else { ci += d0; cj += d1; }
        if (ci >= 0 && ci < g.Nx && cj >= 0 && cj < g.Ny && ck >= 0 && ck < g.Nz) {
          const int m = g.mat[cell_index(ci, cj, ck, g.Nx, g.Ny)];
          sig += g.S[3 * m + a];
          eps += g.P[3 * m + a];
        }
      }
      if (sig != 0.0 && eps != 0.0) {  // Si is set only where avg_eps != 0 (:5579)
        const double w = (double)Os[a][s] + (double)Us[a][s];
        acc += w * ((sig / g.len[a]) * w);
      }
    }
  }
  red[tid] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) lb.part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (uint64_t)blockIdx.z)] = red[0];
}

// Fixed-order sum of the partials into loss[step] (before the H half step
// advances the step counter).
__global__ void __launch_bounds__(256) fit_loss_finish(const double* part, int nparts, double* loss,
                                                      const int* step_counter) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) acc += part[b];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[*step_counter] = 0.25 * red[0];
}

// ---------------------------------------------------------------- launchers
// Block shape of the streamed variants (x by y node slots of one plane; at
// most 256 threads, the kernels' launch bound).  32 x 4 and 64 x 2 measured
// fastest at 256^3 and 512^3 (FP32, B200): 4 % below 32 x 8; 32 x 1 took twice
// as long, 256 x 1 and 16 x 16 were slower than 32 x 8.
#ifndef TF_FIT_SBX
#define TF_FIT_SBX 32
#endif
#ifndef TF_FIT_SBY
#define TF_FIT_SBY 4
#endif
// Kernel variants for the E and H halves (all compute bit-identical results):
// 0 one thread per node slot, 1 z-march over 4 planes, 2 z-march over 16,
// 3 one thread per node slot with per-dof coefficient arrays.
template <typename T>
void fit_launch_step(const FitGrid<T>& g, const SpecialEdges<T>& sp, const ProbeSet& pr, int* step_counter,
                     double* flux, cudaStream_t st, cudaEvent_t* ev, int e_variant, int h_variant,
                     const FitLoss<T>* loss, const FitTmaMaps* tma) {
  // ev (optional): 6 events recorded around the 5 phases, for per-phase timing;
  // loss (optional): Joule loss of the E half step
  dim3 blk(32, 8, 1);
  dim3 grd((unsigned)((g.Nx + 1 + 31) / 32), (unsigned)((g.Ny + 1 + 7) / 8), (unsigned)(g.Nz + 1));
  // the streamed variants (3, 5): one node slot per thread, one plane per block
  const dim3 sblk(TF_FIT_SBX, TF_FIT_SBY, 1);
  const dim3 sgrd((unsigned)((g.Nx + TF_FIT_SBX) / TF_FIT_SBX), (unsigned)((g.Ny + TF_FIT_SBY) / TF_FIT_SBY),
                  (unsigned)(g.Nz + 1));
  auto mgrid = [&](int kc) {
    return dim3((unsigned)((g.Nx + 1 + 31) / 32), (unsigned)((g.Ny + 1 + 7) / 8), (unsigned)((g.Nz + 1 + kc - 1) / kc));
  };
  const int nsb = (sp.n + 255) / 256;
  if (ev) cudaEventRecord(ev[0], st);
  if (loss) {
    const size_t bytes = (size_t)(g.sxy * (g.Nz + 1)) * sizeof(T);
    cudaMemcpyAsync(loss->Ox, g.Ux, bytes, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(loss->Oy, g.Uy, bytes, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(loss->Oz, g.Uz, bytes, cudaMemcpyDeviceToDevice, st);
  }
  if (sp.n > 0) fit_special_pre<T><<<nsb, 256, 0, st>>>(g, sp, step_counter);
  if (ev) cudaEventRecord(ev[1], st);
  if (e_variant == 0) fit_e_kernel<T><<<grd, blk, 0, st>>>(g);
  else if (e_variant == 3) fit_e_coef<T><<<sgrd, sblk, 0, st>>>(g);
  else if (e_variant == 5 && g.lut_e) fit_e_class<T><<<sgrd, sblk, 0, st>>>(g);
  else if (e_variant == 4 && tma)
    fit_e_tma<T><<<mgrid(16), dim3(kTmaTX, kTmaTY + 1), 0, st>>>(g, 16, tma->F[0], tma->F[1], tma->F[2], tma->U[0], tma->U[1], tma->U[2],
                                             tma->err);
  else {
    const int kc = e_variant == 1 ? 4 : 16;  // variants 1, 2 (and 4, 5 without their tensor maps or tables)
    fit_e_march<T><<<mgrid(kc), blk, 0, st>>>(g, kc);
  }
  if (ev) cudaEventRecord(ev[2], st);
  fit_special_post<T><<<nsb > 0 ? nsb : 1, 256, 0, st>>>(g, sp, step_counter, flux, nsb);
  if (loss) {
    fit_loss_kernel<T><<<grd, blk, 0, st>>>(g, *loss);
    fit_loss_finish<<<1, 256, 0, st>>>(loss->part, loss->nparts, loss->loss, step_counter);
  }
  if (ev) cudaEventRecord(ev[3], st);
  if (pr.n > 0) fit_probe_kernel<T><<<(pr.n + 127) / 128, 128, 0, st>>>(g, pr, step_counter);
  if (ev) cudaEventRecord(ev[4], st);
  if (h_variant == 0) fit_h_kernel<T><<<grd, blk, 0, st>>>(g, step_counter);
  else if (h_variant == 3) fit_h_coef<T><<<sgrd, sblk, 0, st>>>(g, step_counter);
  else if (h_variant == 5 && g.lut_f) fit_h_class<T><<<sgrd, sblk, 0, st>>>(g, step_counter);
  else if (h_variant == 4 && tma)
    fit_h_tma<T><<<mgrid(16), dim3(kTmaTX, kTmaTY + 1), 0, st>>>(g, 16, step_counter, tma->U[0], tma->U[1], tma->U[2], tma->F[0],
                                             tma->F[1], tma->F[2], tma->err);
  else {
    const int kc = h_variant == 1 ? 4 : 16;
    fit_h_march<T><<<mgrid(kc), blk, 0, st>>>(g, kc, step_counter);
  }
  if (ev) cudaEventRecord(ev[5], st);
}

int fit_kernels_per_step(int n_special, int n_probes, bool losses) {
  return 3 + (n_special > 0) + (n_probes > 0) + (losses ? 2 : 0);
}

// Number of partial sums fit_loss_kernel writes.
size_t fit_loss_parts(int Nx, int Ny, int Nz) {
  return (size_t)((Nx + 1 + 31) / 32) * ((Ny + 1 + 7) / 8) * (Nz + 1);
}

template void fit_launch_step<double>(const FitGrid<double>&, const SpecialEdges<double>&, const ProbeSet&, int*,
                                      double*, cudaStream_t, cudaEvent_t*, int, int, const FitLoss<double>*,
                                      const FitTmaMaps*);
template void fit_launch_step<float>(const FitGrid<float>&, const SpecialEdges<float>&, const ProbeSet&, int*,
                                     double*, cudaStream_t, cudaEvent_t*, int, int, const FitLoss<float>*,
                                     const FitTmaMaps*);

// Tensor maps for the TMA z-march; false when the driver offers no encoder
// or refuses the layout (the variant is then not offered).
bool fit_make_tma_maps(void* const U[3], void* const F[3], int es, int Nx, int Ny, int Nz, int64_t sx,
                       FitTmaMaps* out) {
  typedef CUresult (*Encode)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
      q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    return false;
  }
  Encode enc = (Encode)fn;
  const cuuint64_t dims[3] = {(cuuint64_t)sx, (cuuint64_t)Ny + 1, (cuuint64_t)Nz + 1};
  const cuuint64_t strides[2] = {(cuuint64_t)(sx * es), (cuuint64_t)(sx * es * (Ny + 1))};
  const cuuint32_t box[3] = {(cuuint32_t)(kTmaTX + 16 / es), (cuuint32_t)(kTmaTY + 1), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dtype = es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  if ((sx * es) % 16 != 0) return false;
  for (int a = 0; a < 3; a++) {
    if (enc(&out->U[a], dtype, 3, U[a], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    if (enc(&out->F[a], dtype, 3, F[a], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  (void)Nx;
  return true;
}

// Discrete leapfrog energy of the state after a step, (U^n, F^{n+1/2}):
// W^n = 0.5 sum M_e (U^n)^2 + 0.5 sum M_mu F^{n+1/2} F^{n-1/2}, an invariant of
// the lossless leapfrog.  F^{n-1/2} is recomputed (not stored): the H update
// gave M_mu F^{n+1/2} = M_mu F^{n-1/2} - dt curl U^n, so its B is
// 2 M_mu F^{n+1/2} - B(F^{n+1/2}, U^n).  FP64 accumulation, one partial per
// block.
template <typename T>
__global__ void __launch_bounds__(256) fit_energy_kernel(FitGrid<T> g, double* part) {
  __shared__ double red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  double acc = 0.0;
  if (i <= g.Nx && j <= g.Ny) {
    const int64_t s = (int64_t)i + g.sx * j + g.sxy * k;
    uint8_t c[2][2][2];
    for (int dz = 0; dz < 2; dz++)
      for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) {
          int ci = i - 1 + dx, cj = j - 1 + dy, ck = k - 1 + dz;
          bool ok = ci >= 0 && ci < g.Nx && cj >= 0 && cj < g.Ny && ck >= 0 && ck < g.Nz;
          c[dz][dy][dx] = ok ? g.mat[cell_index(ci, cj, ck, g.Nx, g.Ny)] : 255;
        }
    // electric part: M_e = avg_eps / len over the edge's existing cells
    const T* Us[3] = {g.Ux, g.Uy, g.Uz};
    const bool valid[3] = {i < g.Nx, j < g.Ny, k < g.Nz};
    for (int a = 0; a < 3; a++) {
      if (!valid[a]) continue;
      uint8_t m[4];
      int nm = 0;
      for (int q = 0; q < 4; q++) {
        int b0 = q & 1, b1 = (q >> 1) & 1;
        uint8_t cm;
        if (a == 0) cm = c[b1][b0][1];
        else if (a == 1) cm = c[b1][1][b0];
        else cm = c[1][b1][b0];
        if (cm != 255) m[nm++] = cm;
      }
      double eps = 0.0;
      for (int q = 0; q < nm; q++) eps += g.P[3 * m[q] + a];
      double u = (double)Us[a][s];
      acc += 0.5 * (eps / g.len[a]) * u * u;
    }
    for (int a = 0; a < 3; a++) {
      T B, nu;
      if ((a == 0 && j < g.Ny && k < g.Nz) || (a == 1 && i < g.Nx && k < g.Nz) || (a == 2 && i < g.Nx && j < g.Ny)) {
        const T* Fs = a == 0 ? g.Fx : (a == 1 ? g.Fy : g.Fz);
        double Fold = (double)Fs[s];
        T mmu;
        if (face_B(g, a, i, j, k, B, nu, &mmu)) {
          const double Bprev = 2.0 * (double)mmu * Fold - (double)B;
          const double Fprev = (double)nu * Bprev;
          acc += 0.5 * ((double)mmu * Fold) * Fprev;
        }
      }
    }
  }
  red[tid] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (uint64_t)blockIdx.z)] = red[0];
}

template <typename T>
size_t fit_launch_energy(const FitGrid<T>& g, double* part, cudaStream_t st) {
  dim3 blk(32, 8, 1);
  dim3 grd((unsigned)((g.Nx + 1 + 31) / 32), (unsigned)((g.Ny + 1 + 7) / 8), (unsigned)(g.Nz + 1));
  if (part) fit_energy_kernel<T><<<grd, blk, 0, st>>>(g, part);
  return (size_t)grd.x * grd.y * grd.z;
}
template size_t fit_launch_energy<double>(const FitGrid<double>&, double*, cudaStream_t);
template size_t fit_launch_energy<float>(const FitGrid<float>&, double*, cudaStream_t);

}  // namespace tf
