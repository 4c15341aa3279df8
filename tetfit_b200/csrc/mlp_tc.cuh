// Forward pass of the learned warm start's network on the 5th-generation
// tensor cores (sm_100a tcgen05): one CTA of 128 threads evaluates 128 rows
// at a time, thread t owning row t.
//
//   layer 1  D = A1 (128 x 16, the 6 inputs padded) x W1^T   (one MMA, K = 16)
//   layer 2  D = A2 (128 x 64, SiLU of layer 1)     x W2^T   (four MMAs, K = 16 each)
//   output   y = W3 . SiLU(D + b2) + b3                    (FP32 on the CUDA cores)
//
// Operands are BF16 in shared memory in the canonical K-major layout without
// swizzle: the matrix is cut into core matrices of 8 rows x 8 elements
// (16 bytes per row, 128 bytes contiguous), the core matrices of one 8-row
// group are consecutive along K (leading-dimension byte offset 128) and the
// row groups follow each other (stride-dimension byte offset = 128 x K / 8).
// The FP32 accumulator (128 lanes x 64 columns) lives in tensor memory,
// allocated once per CTA; one thread issues tcgen05.mma and tcgen05.commit,
// whose completion arrives on an mbarrier that thread polls (bounded) while
// the others wait in a barrier, and each warp reads its 32 lanes back with
// tcgen05.ld after tcgen05.fence::after_thread_sync.
// Numerics: BF16 products and FP32 accumulation as on the mma.sync path; the
// activation works on z' = z / 2 = fma(acc, 1/2, b / 2) in FP32, packed to a
// BF16 pair by integer adds on the bit patterns (magnitude rounded half up,
// no conversion-unit op), and forms silu(z) = z' (1 + tanh z') with one
// bf16x2 tanh and one bf16x2 FMA: the special-function unit sees one op per
// pair of activations instead of three, and the result is rounded once
// where the mma.sync path's BF16x2 SiLU rounds twice.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "mlp.cuh"

namespace tf {

constexpr int kTcRows = 128;
constexpr int kTcCols = 64;                // TMEM columns a CTA allocates
constexpr long kTcWaitLimit = 1L << 22;    // mbarrier polls before a wait gives up

struct MlpTcSmem {
  alignas(128) __nv_bfloat16 w1[64 * 16];   // layer-1 B: 8 n-groups x 2 k-groups of core matrices
  alignas(128) __nv_bfloat16 w2[64 * 64];   // layer-2 B: 8 x 8
  // layer-2 A (16 row groups x 8 k-groups); its first 4 KB also hold layer-1
  // A (16 x 2), which the first MMA has finished reading before A2 is written
  alignas(128) __nv_bfloat16 a2[128 * 64];
  float b1h[64], b2h[64], w3[64], b3;  // b1h, b2h: the biases halved
  alignas(8) uint64_t bar;
  uint32_t tmem;
  __device__ __nv_bfloat16* a1() { return a2; }
};

// element (r, k) of a K-major operand with `kg` 8-element k-groups
__device__ __forceinline__ int tc_off(int r, int k, int kg) { return ((r >> 3) * kg + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7); }

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading and stride
// dimension byte offsets (all in 16-byte units), descriptor version 1, no
// swizzle, base offset 0.
__device__ __forceinline__ uint64_t tc_desc(const void* start, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = tc_smem(start);
  return (uint64_t)((a & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N / 8 and M / 16.
__host__ __device__ constexpr uint32_t tc_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float v[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int c = 0; c < 32; c++) v[c] = __uint_as_float(r[c]);
}

__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity) {
  for (long it = 0;; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(tc_smem(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it > kTcWaitLimit) return false;
  }
}

// Set-up by all 128 threads: weights into the canonical layout from the
// packed BF16 image (mlp.hpp), biases and W3 in FP32, the mbarrier, and the
// TMEM columns (allocated by warp 0).
__device__ __forceinline__ void mlp_tc_setup(MlpTcSmem& sm, const unsigned char* image) {
  const int tid = threadIdx.x;
  const __nv_bfloat16* img = reinterpret_cast<const __nv_bfloat16*>(image);
  for (int q = tid; q < 64 * 16; q += blockDim.x) sm.w1[tc_off(q >> 4, q & 15, 2)] = img[kImgW1 + (q >> 4) * kLd1 + (q & 15)];
  for (int q = tid; q < 64 * 64; q += blockDim.x) sm.w2[tc_off(q >> 6, q & 63, 8)] = img[kImgW2T + (q >> 6) * kLd2 + (q & 63)];
  const float* fb = reinterpret_cast<const float*>(image + kImgBf16 * 2);
  if (tid < 64) {
    sm.b1h[tid] = 0.5f * fb[tid];
    sm.b2h[tid] = 0.5f * fb[64 + tid];
    sm.w3[tid] = __bfloat162float(img[kImgW3 + tid]);
  }
  if (tid == 0) {
    sm.b3 = fb[128];
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&sm.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((tid >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&sm.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_proxy_fence();  // the weights are read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ __forceinline__ void mlp_tc_teardown(MlpTcSmem& sm) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem), "r"(kTcCols) : "memory");
}

// BF16 pair of two FP32 values, magnitudes rounded half up (integer adds on
// the bit patterns, then the upper halves; first value in the low half)
__device__ __forceinline__ uint32_t tc_pack_half_up(float x0, float x1) {
  return __byte_perm(__float_as_uint(x0) + 0x8000u, __float_as_uint(x1) + 0x8000u, 0x7632);
}
// silu(z) for a BF16 pair zz = z / 2: z' (1 + tanh z') = fma(z', tanh z', z')
__device__ __forceinline__ uint32_t tc_silu_of_half(uint32_t zz) {
  uint32_t th, h;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(th) : "r"(zz));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(h) : "r"(zz), "r"(th));
  return h;
}

// One 128-row tile: f[6] are this thread's inputs; returns false (on every
// thread) when an MMA completion wait ran out, after raising *err.  `phase`
// counts the completions seen so far.
__device__ __forceinline__ bool mlp_tc_forward(MlpTcSmem& sm, uint32_t& phase, const float f[6], float& y,
                                               int* err) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t tmem = sm.tmem;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 TMEM lanes
  constexpr uint32_t kId = tc_idesc(kTcRows, 64);
  // layer-1 A row
#pragma unroll
  for (int k = 0; k < 16; k += 2) {
    const float lo = k < 6 ? f[k] : 0.0f, hi = k + 1 < 6 ? f[k + 1] : 0.0f;
    *reinterpret_cast<uint32_t*>(&sm.a1()[tc_off(tid, k, 2)]) = mlp_pack(lo, hi);
  }
  tc_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid == 0) {
    tc_mma(tmem, tc_desc(sm.a1(), 128, 256), tc_desc(sm.w1, 128, 256), kId, 0);
    tc_commit(&sm.bar);
  }
  // thread 0 polls the completion; the others wait in the barrier (no
  // issue slots spent polling) and order their TMEM reads after it
  bool ok = tid == 0 ? tc_wait(&sm.bar, phase & 1) : true;
  phase++;
  if (!__syncthreads_and(ok)) {
    // give the MMA one more bounded wait before the caller frees its TMEM
    if (tid == 0) {
      atomicExch(err, 4);
      tc_wait(&sm.bar, (phase - 1) & 1);
    }
    __syncthreads();
    return false;
  }
  tc_fence_after();
  // SiLU(D + b1) -> layer-2 A row, in BF16 pairs
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float v[32];
    tc_ld32(lane_addr + 32 * h, v);
#pragma unroll
    for (int c = 0; c < 32; c += 2) {
      const int n = 32 * h + c;
      const uint32_t zz = tc_pack_half_up(__fmaf_rn(v[c], 0.5f, sm.b1h[n]), __fmaf_rn(v[c + 1], 0.5f, sm.b1h[n + 1]));
      *reinterpret_cast<uint32_t*>(&sm.a2[tc_off(tid, n, 8)]) = tc_silu_of_half(zz);
    }
  }
  tc_proxy_fence();
  tc_fence_before();
  __syncthreads();  // every lane read, every A2 row written
  tc_fence_after();
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < 4; s++)
      // k-step s: k-groups 2s and 2s + 1, 128 elements further along
      tc_mma(tmem, tc_desc(sm.a2 + 128 * s, 128, 1024), tc_desc(sm.w2 + 128 * s, 128, 1024), kId, s > 0 ? 1u : 0u);
    tc_commit(&sm.bar);
  }
  ok = tid == 0 ? tc_wait(&sm.bar, phase & 1) : true;
  phase++;
  if (!__syncthreads_and(ok)) {
    if (tid == 0) {
      atomicExch(err, 4);
      tc_wait(&sm.bar, (phase - 1) & 1);
    }
    __syncthreads();
    return false;
  }
  tc_fence_after();
  float acc = sm.b3;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float v[32];
    tc_ld32(lane_addr + 32 * h, v);
#pragma unroll
    for (int c = 0; c < 32; c += 2) {
      const int n = 32 * h + c;
      const uint32_t p = tc_silu_of_half(
          tc_pack_half_up(__fmaf_rn(v[c], 0.5f, sm.b2h[n]), __fmaf_rn(v[c + 1], 0.5f, sm.b2h[n + 1])));
      acc += sm.w3[n] * __uint_as_float(p << 16) + sm.w3[n + 1] * __uint_as_float(p & 0xffff0000u);
    }
  }
  y = acc;
  tc_fence_before();
  __syncthreads();  // the accumulator and A tiles are free for the next tile
  tc_fence_after();
  return true;
}

}  // namespace tf
