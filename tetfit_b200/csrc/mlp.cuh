// Per-edge MLP of the learned CG warm start: 6 inputs -> 64 -> 64 -> 1, SiLU
// between layers, BF16 weights and activations on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation), FP32 master parameters.
//
// Parameter vector (FP32, kNParam values):
//   W1[64][16] (inputs 6..15 are padding and stay 0) | b1[64] | W2[64][64] |
//   b2[64] | W3[64] | b3
// W[n][k] is the weight from input k to output n.
//
// BF16 weight image (what the kernels load into shared memory), row strides
// padded by 8 elements against bank conflicts:
//   W1T[64][24]  W1 (n-major, k contiguous)
//   W2T[64][72]  W2 (n-major, k contiguous): forward B fragments
//   W2K[64][72]  W2 transposed (k-major, n contiguous): backward B fragments
//   W3T[8][72]   row 0 = W3, rows 1..7 zero (output padded to 8 columns)
//   then FP32 b1[64], b2[64], b3 (as floats after the BF16 part)
//
// Fragment layouts (PTX ISA, mma.m16n8k16 .bf16): with g = lane / 4 and
// t = lane % 4, A registers hold (row g | g+8, cols 2t..2t+1 | 2t+8..2t+9),
// B registers (k = 2t..2t+1 | 2t+8..2t+9, n = g), C floats (row g | g+8,
// cols 2t, 2t+1).  A layer's C tiles n = 2kt and 2kt+1 are exactly the A
// registers of k-tile kt of the next layer, so activations stay in registers.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "mlp.hpp"

namespace tf {

__device__ __forceinline__ uint32_t mlp_pack(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mlp_mma(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// B fragment of k-tile kt, n-tile nt from a matrix stored n-major with k
// contiguous (B[k][n] = W[n * ld + k])
__device__ __forceinline__ void mlp_ldb(uint32_t b[2], const __nv_bfloat16* W, int ld, int kt, int nt, int lane) {
  const __nv_bfloat16* p = W + (nt * 8 + (lane >> 2)) * ld + kt * 16 + 2 * (lane & 3);
  b[0] = *reinterpret_cast<const uint32_t*>(p);
  b[1] = *reinterpret_cast<const uint32_t*>(p + 8);
}

// A fragment of m-tile mt, k-tile kt from a matrix stored m-major with k
// contiguous (A[m][k] = M[m * ld + k])
__device__ __forceinline__ void mlp_lda(uint32_t a[4], const __nv_bfloat16* M, int ld, int mt, int kt, int lane) {
  const __nv_bfloat16* p = M + (mt * 16 + (lane >> 2)) * ld + kt * 16 + 2 * (lane & 3);
  a[0] = *reinterpret_cast<const uint32_t*>(p);
  a[1] = *reinterpret_cast<const uint32_t*>(p + 8 * ld);
  a[2] = *reinterpret_cast<const uint32_t*>(p + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(p + 8 * ld + 8);
}

// sigmoid(z) = (1 + tanh(z / 2)) / 2 with the hardware tanh approximation
// (one special-function op); training and inference share it.
__device__ __forceinline__ float mlp_sigmoid(float z) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
  return 0.5f + 0.5f * t;
}
__device__ __forceinline__ float mlp_silu(float z) { return z * mlp_sigmoid(z); }
__device__ __forceinline__ float mlp_dsilu(float z) {
  const float s = mlp_sigmoid(z);
  return s * (1.0f + z * (1.0f - s));
}
// silu of two values packed as the next layer's BF16 pair, in BF16x2
// arithmetic: z is converted once, tanh(z / 2) is one bf16x2 special-function
// op, silu = z (1 + tanh(z / 2)) / 2 two bf16x2 FMA-pipe ops (the result is
// BF16 anyway)
__device__ __forceinline__ uint32_t mlp_silu_pack(float z0, float z1) {
  const uint32_t zz = mlp_pack(z0, z1);
  const uint32_t half = 0x3f003f00u;  // (0.5, 0.5) in BF16
  uint32_t hz, th, u, h;
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(hz) : "r"(zz), "r"(half));
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(th) : "r"(hz));
  asm("fma.rn.bf16x2 %0, %1, %2, %2;" : "=r"(u) : "r"(th), "r"(half));
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(h) : "r"(zz), "r"(u));
  return h;
}
__device__ __forceinline__ float mlp_silu_bf16(float z) {
  const uint32_t p = mlp_silu_pack(z, 0.0f);
  return __uint_as_float(p << 16);
}

// sign(x) log2(1 + |x|): compresses large inputs, linear near 0
__device__ __forceinline__ float mlp_compress(float x) { return copysignf(__log2f(1.0f + fabsf(x)), x); }

// Shared-memory view of the weight image
struct MlpSmem {
  const __nv_bfloat16* w1;
  const __nv_bfloat16* w2t;
  const __nv_bfloat16* w2k;
  const __nv_bfloat16* w3;
  const float* b1;
  const float* b2;
  const float* b3;
};
__device__ __forceinline__ MlpSmem mlp_view(const unsigned char* img) {
  MlpSmem v;
  const __nv_bfloat16* w = reinterpret_cast<const __nv_bfloat16*>(img);
  v.w1 = w + kImgW1;
  v.w2t = w + kImgW2T;
  v.w2k = w + kImgW2K;
  v.w3 = w + kImgW3;
  const float* f = reinterpret_cast<const float*>(img + kImgBf16 * 2);
  v.b1 = f;
  v.b2 = f + 64;
  v.b3 = f + 128;
  return v;
}

// cooperative copy of the weight image (global -> shared), 16 bytes a thread
__device__ __forceinline__ void mlp_load_image(unsigned char* dst, const unsigned char* src) {
  for (int k = threadIdx.x; k < kImgBytes / 16; k += blockDim.x)
    reinterpret_cast<uint4*>(dst)[k] = reinterpret_cast<const uint4*>(src)[k];
}

// Forward pass of one 16-row tile.  a1: layer-1 A fragment (inputs);
// z1, z2: pre-activations (C layout, kept for the backward pass); y[0] and
// y[2] hold the outputs of rows g and g + 8 in the lanes with t = 0.
__device__ __forceinline__ void mlp_forward(const MlpSmem& w, const uint32_t a1[4], float z1[8][4], float z2[8][4],
                                            uint32_t a2[4][4], uint32_t a3[4][4], float y[4], int lane) {
  const int t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    const float b0 = w.b1[nt * 8 + 2 * t], b1v = w.b1[nt * 8 + 2 * t + 1];
    z1[nt][0] = b0;
    z1[nt][1] = b1v;
    z1[nt][2] = b0;
    z1[nt][3] = b1v;
    uint32_t b[2];
    mlp_ldb(b, w.w1, kLd1, 0, nt, lane);
    mlp_mma(z1[nt], a1, b);
  }
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    a2[kt][0] = mlp_silu_pack(z1[2 * kt][0], z1[2 * kt][1]);
    a2[kt][1] = mlp_silu_pack(z1[2 * kt][2], z1[2 * kt][3]);
    a2[kt][2] = mlp_silu_pack(z1[2 * kt + 1][0], z1[2 * kt + 1][1]);
    a2[kt][3] = mlp_silu_pack(z1[2 * kt + 1][2], z1[2 * kt + 1][3]);
  }
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    const float b0 = w.b2[nt * 8 + 2 * t], b1v = w.b2[nt * 8 + 2 * t + 1];
    z2[nt][0] = b0;
    z2[nt][1] = b1v;
    z2[nt][2] = b0;
    z2[nt][3] = b1v;
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
      uint32_t b[2];
      mlp_ldb(b, w.w2t, kLd2, kt, nt, lane);
      mlp_mma(z2[nt], a2[kt], b);
    }
  }
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    a3[kt][0] = mlp_silu_pack(z2[2 * kt][0], z2[2 * kt][1]);
    a3[kt][1] = mlp_silu_pack(z2[2 * kt][2], z2[2 * kt][3]);
    a3[kt][2] = mlp_silu_pack(z2[2 * kt + 1][0], z2[2 * kt + 1][1]);
    a3[kt][3] = mlp_silu_pack(z2[2 * kt + 1][2], z2[2 * kt + 1][3]);
  }
  const float bo = t == 0 ? w.b3[0] : 0.0f;
  y[0] = bo;
  y[1] = 0.0f;
  y[2] = bo;
  y[3] = 0.0f;
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    uint32_t b[2];
    mlp_ldb(b, w.w3, kLd2, kt, 0, lane);
    mlp_mma(y, a3[kt], b);
  }
}

// Inference-only forward pass of one 16-row tile: layer by layer, nothing
// kept for a backward pass (same arithmetic as mlp_forward).
__device__ __forceinline__ void mlp_infer(const MlpSmem& w, const uint32_t a1[4], float y[4], int lane) {
  const int t = lane & 3;
  uint32_t a2[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    float c[2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int nt = 2 * kt + h;
      const float b0 = w.b1[nt * 8 + 2 * t], b1v = w.b1[nt * 8 + 2 * t + 1];
      c[h][0] = b0;
      c[h][1] = b1v;
      c[h][2] = b0;
      c[h][3] = b1v;
      uint32_t b[2];
      mlp_ldb(b, w.w1, kLd1, 0, nt, lane);
      mlp_mma(c[h], a1, b);
    }
    a2[kt][0] = mlp_silu_pack(c[0][0], c[0][1]);
    a2[kt][1] = mlp_silu_pack(c[0][2], c[0][3]);
    a2[kt][2] = mlp_silu_pack(c[1][0], c[1][1]);
    a2[kt][3] = mlp_silu_pack(c[1][2], c[1][3]);
  }
  const float bo = t == 0 ? w.b3[0] : 0.0f;
  y[0] = bo;
  y[1] = 0.0f;
  y[2] = bo;
  y[3] = 0.0f;
#pragma unroll
  for (int k3 = 0; k3 < 4; k3++) {
    float o[2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int nt = 2 * k3 + h;
      const float b0 = w.b2[nt * 8 + 2 * t], b1v = w.b2[nt * 8 + 2 * t + 1];
      o[h][0] = b0;
      o[h][1] = b1v;
      o[h][2] = b0;
      o[h][3] = b1v;
#pragma unroll
      for (int kt = 0; kt < 4; kt++) {
        uint32_t b[2];
        mlp_ldb(b, w.w2t, kLd2, kt, nt, lane);
        mlp_mma(o[h], a2[kt], b);
      }
    }
    uint32_t a3[4];
    a3[0] = mlp_silu_pack(o[0][0], o[0][1]);
    a3[1] = mlp_silu_pack(o[0][2], o[0][3]);
    a3[2] = mlp_silu_pack(o[1][0], o[1][1]);
    a3[3] = mlp_silu_pack(o[1][2], o[1][3]);
    uint32_t b[2];
    mlp_ldb(b, w.w3, kLd2, k3, 0, lane);
    mlp_mma(y, a3, b);
  }
}

// mlp_infer for the two 16-row tiles of a warp at once: every weight
// fragment read from shared memory feeds both tiles' MMAs.
__device__ __forceinline__ void mlp_infer2(const MlpSmem& w, const uint32_t a1[2][4], float y[2][4], int lane) {
  const int t = lane & 3;
  uint32_t a2[2][4][4];
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    float c[2][2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int nt = 2 * kt + h;
      const float b0 = w.b1[nt * 8 + 2 * t], b1v = w.b1[nt * 8 + 2 * t + 1];
      uint32_t b[2];
      mlp_ldb(b, w.w1, kLd1, 0, nt, lane);
#pragma unroll
      for (int q = 0; q < 2; q++) {
        c[q][h][0] = b0;
        c[q][h][1] = b1v;
        c[q][h][2] = b0;
        c[q][h][3] = b1v;
        mlp_mma(c[q][h], a1[q], b);
      }
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
      a2[q][kt][0] = mlp_silu_pack(c[q][0][0], c[q][0][1]);
      a2[q][kt][1] = mlp_silu_pack(c[q][0][2], c[q][0][3]);
      a2[q][kt][2] = mlp_silu_pack(c[q][1][0], c[q][1][1]);
      a2[q][kt][3] = mlp_silu_pack(c[q][1][2], c[q][1][3]);
    }
  }
  const float bo = t == 0 ? w.b3[0] : 0.0f;
#pragma unroll
  for (int q = 0; q < 2; q++) {
    y[q][0] = bo;
    y[q][1] = 0.0f;
    y[q][2] = bo;
    y[q][3] = 0.0f;
  }
#pragma unroll
  for (int k3 = 0; k3 < 4; k3++) {
    float o[2][2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int nt = 2 * k3 + h;
      const float b0 = w.b2[nt * 8 + 2 * t], b1v = w.b2[nt * 8 + 2 * t + 1];
#pragma unroll
      for (int q = 0; q < 2; q++) {
        o[q][h][0] = b0;
        o[q][h][1] = b1v;
        o[q][h][2] = b0;
        o[q][h][3] = b1v;
      }
#pragma unroll
      for (int kt = 0; kt < 4; kt++) {
        uint32_t b[2];
        mlp_ldb(b, w.w2t, kLd2, kt, nt, lane);
        mlp_mma(o[0][h], a2[0][kt], b);
        mlp_mma(o[1][h], a2[1][kt], b);
      }
    }
    uint32_t b[2];
    mlp_ldb(b, w.w3, kLd2, k3, 0, lane);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      uint32_t a3[4];
      a3[0] = mlp_silu_pack(o[q][0][0], o[q][0][1]);
      a3[1] = mlp_silu_pack(o[q][0][2], o[q][0][3]);
      a3[2] = mlp_silu_pack(o[q][1][0], o[q][1][1]);
      a3[3] = mlp_silu_pack(o[q][1][2], o[q][1][3]);
      mlp_mma(y[q], a3, b);
    }
  }
}

// Layer-1 A fragment of a 16-row tile whose row r inputs are held by lane
// src0 + r (6 floats f[0..5] in every lane; all lanes take part)
__device__ __forceinline__ void mlp_input_fragment(uint32_t a[4], const float f[6], int src0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  float v0[6], v1[6];
#pragma unroll
  for (int k = 0; k < 6; k++) {
    v0[k] = __shfl_sync(0xffffffffu, f[k], src0 + g);
    v1[k] = __shfl_sync(0xffffffffu, f[k], src0 + g + 8);
  }
  float lo0 = 0.f, hi0 = 0.f, lo1 = 0.f, hi1 = 0.f;
  if (t == 0) { lo0 = v0[0]; hi0 = v0[1]; lo1 = v1[0]; hi1 = v1[1]; }
  if (t == 1) { lo0 = v0[2]; hi0 = v0[3]; lo1 = v1[2]; hi1 = v1[3]; }
  if (t == 2) { lo0 = v0[4]; hi0 = v0[5]; lo1 = v1[4]; hi1 = v1[5]; }
  a[0] = mlp_pack(lo0, hi0);
  a[1] = mlp_pack(lo1, hi1);
  a[2] = 0u;
  a[3] = 0u;
}

// Output of row src0 + r of a 16-row tile back to the lane that owns it
// (returns the lane's own row value when its row is in this tile)
__device__ __forceinline__ float mlp_output_to_rows(const float y[4], int lane) {
  const int r = lane & 15;
  const int src = (r & 7) * 4;
  const float a = __shfl_sync(0xffffffffu, y[0], src);
  const float b = __shfl_sync(0xffffffffu, y[2], src);
  return r < 8 ? a : b;
}

}  // namespace tf
