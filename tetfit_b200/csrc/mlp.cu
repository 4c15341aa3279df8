// Training and evaluation kernels of the learned CG warm-start network
// (mlp.cuh): BF16 tensor-core forward and backward passes with FP32
// accumulation, weight gradients as tensor-core GEMMs over the rows of a
// block, a fixed-order reduction of the block partials and an Adam step on
// the FP32 master parameters.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include <string>

#include "../../include/tetfit.h"
#include "mlp.cuh"
#include "mlp_tc.cuh"

namespace tf {
void set_thread_error(const std::string& m);

namespace {
constexpr int kTrainWarps = 8;
constexpr int kTrainRows = 16 * kTrainWarps;  // rows per block
constexpr int kLdR = kTrainRows + 8;
constexpr int kTrainSmem = kImgBytes + (16 + 4 * 64 + 2 * 8) * kLdR * 2 + 16 * 4;
}  // namespace

int mlp_train_rows_per_block() { return kTrainRows; }

// image = BF16 weights (+ FP32 biases) from the FP32 parameters
__global__ void mlp_pack_kernel(const float* __restrict__ p, unsigned char* img) {
  __nv_bfloat16* w = reinterpret_cast<__nv_bfloat16*>(img);
  float* fb = reinterpret_cast<float*>(img + kImgBf16 * 2);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kImgBf16 + 132; i += gridDim.x * blockDim.x) {
    if (i >= kImgBf16) {
      const int k = i - kImgBf16;
      fb[k] = k < 64 ? p[kOffB1 + k] : (k < 128 ? p[kOffB2 + k - 64] : (k == 128 ? p[kOffB3] : 0.0f));
      continue;
    }
    float v = 0.0f;
    if (i < kImgW2T) {
      const int n = i / kLd1, k = i % kLd1;
      v = k < kMlpInP ? p[kOffW1 + n * kMlpInP + k] : 0.0f;
    } else if (i < kImgW2K) {
      const int n = (i - kImgW2T) / kLd2, k = (i - kImgW2T) % kLd2;
      v = k < kMlpH ? p[kOffW2 + n * kMlpH + k] : 0.0f;
    } else if (i < kImgW3) {
      const int k = (i - kImgW2K) / kLd2, n = (i - kImgW2K) % kLd2;
      v = n < kMlpH ? p[kOffW2 + n * kMlpH + k] : 0.0f;
    } else {
      const int r = (i - kImgW3) / kLd2, k = (i - kImgW3) % kLd2;
      v = (r == 0 && k < kMlpH) ? p[kOffW3 + k] : 0.0f;
    }
    w[i] = __float2bfloat16_rn(v);
  }
}

cudaError_t mlp_launch_pack(const float* params, unsigned char* image, cudaStream_t st) {
  mlp_pack_kernel<<<(kImgBf16 + 132 + 255) / 256, 256, 0, st>>>(params, image);
  return cudaGetLastError();
}

// Evaluation of n rows (inputs [n][6] -> outputs [n]); a warp takes 32 rows
// as two 16-row tiles.
__global__ void __launch_bounds__(256) mlp_eval_kernel(const unsigned char* image, const float* in, int64_t n,
                                                       float* out) {
  __shared__ __align__(16) unsigned char img[kImgBytes];
  mlp_load_image(img, image);
  __syncthreads();
  const MlpSmem w = mlp_view(img);
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t row = wid * 32 + lane;
  float f[6];
  for (int k = 0; k < 6; k++) f[k] = row < n ? in[row * 6 + k] : 0.0f;
  float res = 0.0f;
#pragma unroll
  for (int q = 0; q < 2; q++) {
    uint32_t a1[4];
    float y[4];
    mlp_input_fragment(a1, f, 16 * q, lane);
    mlp_infer(w, a1, y, lane);
    const float v = mlp_output_to_rows(y, lane);
    if ((lane >> 4) == q) res = v;
  }
  if (row < n) out[row] = res;
}

// Forward and backward pass of kTrainRows rows; the block's gradient of
// sum_i w_i (y_i - t_i)^2 / n goes to grad_part[block][kNParam].
__global__ void __launch_bounds__(32 * kTrainWarps) mlp_train_kernel(const unsigned char* image, const float* in,
                                                                    const float* tg, const float* wt, int n,
                                                                    float* grad_part, float* loss_part) {
  extern __shared__ __align__(16) unsigned char sm[];
  unsigned char* img = sm;
  __nv_bfloat16* fT = reinterpret_cast<__nv_bfloat16*>(sm + kImgBytes);  // [16][kLdR] inputs
  __nv_bfloat16* dz1T = fT + 16 * kLdR;                                   // [64][kLdR]
  __nv_bfloat16* h1T = dz1T + 64 * kLdR;
  __nv_bfloat16* dz2T = h1T + 64 * kLdR;
  __nv_bfloat16* h2T = dz2T + 64 * kLdR;
  __nv_bfloat16* dyT = h2T + 64 * kLdR;   // [8][kLdR], row 0 = dL/dy
  __nv_bfloat16* oneT = dyT + 8 * kLdR;   // [8][kLdR], row 0 = 1
  float* red = reinterpret_cast<float*>(oneT + 8 * kLdR);  // [8] loss, [8] sum of dL/dy
  mlp_load_image(img, image);
  for (int i = threadIdx.x; i < 8 * kLdR; i += blockDim.x) {
    dyT[i] = __float2bfloat16_rn(0.0f);
    oneT[i] = __float2bfloat16_rn(i < kLdR ? 1.0f : 0.0f);
  }
  __syncthreads();
  const MlpSmem w = mlp_view(img);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int row0 = blockIdx.x * kTrainRows + warp * 16;
  const int myrow = row0 + (lane & 15);
  float f[6];
  for (int k = 0; k < 6; k++) f[k] = myrow < n ? in[(int64_t)myrow * 6 + k] : 0.0f;
  uint32_t a1[4], a2[4][4], a3[4][4];
  float z1[8][4], z2[8][4], y[4];
  mlp_input_fragment(a1, f, 0, lane);
  mlp_forward(w, a1, z1, z2, a2, a3, y, lane);
  if (lane < 16)
    for (int k = 0; k < 16; k++)
      fT[k * kLdR + warp * 16 + lane] = __float2bfloat16_rn(k < kMlpIn ? f[k] : 0.0f);
  // dL/dy of rows g and g + 8
  float dy0 = 0.0f, dy1 = 0.0f, l = 0.0f;
  if (t == 0) {
    const int r0 = row0 + g, r1 = row0 + g + 8;
    if (r0 < n) {
      const float e = y[0] - tg[r0];
      dy0 = 2.0f * wt[r0] * e / (float)n;
      l += wt[r0] * e * e;
    }
    if (r1 < n) {
      const float e = y[2] - tg[r1];
      dy1 = 2.0f * wt[r1] * e / (float)n;
      l += wt[r1] * e * e;
    }
    dyT[warp * 16 + g] = __float2bfloat16_rn(dy0);
    dyT[warp * 16 + g + 8] = __float2bfloat16_rn(dy1);
  }
  float ls = l, ds = dy0 + dy1;
  for (int o = 16; o > 0; o >>= 1) {
    ls += __shfl_down_sync(0xffffffffu, ls, o);
    ds += __shfl_down_sync(0xffffffffu, ds, o);
  }
  if (lane == 0) {
    red[warp] = ls;
    red[8 + warp] = ds;
  }
  dy0 = __shfl_sync(0xffffffffu, dy0, lane & ~3);
  dy1 = __shfl_sync(0xffffffffu, dy1, lane & ~3);
  // activations of the tile, transposed (feature-major, rows contiguous)
#pragma unroll
  for (int nt = 0; nt < 8; nt++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int nn = nt * 8 + 2 * t + (c & 1), rr = warp * 16 + g + (c >= 2 ? 8 : 0);
      h1T[nn * kLdR + rr] = __float2bfloat16_rn(mlp_silu_bf16(z1[nt][c]));
      h2T[nn * kLdR + rr] = __float2bfloat16_rn(mlp_silu_bf16(z2[nt][c]));
    }
  // dL/dz2 = dL/dy W3 silu'(z2)
  float d2[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; nt++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int nn = nt * 8 + 2 * t + (c & 1);
      d2[nt][c] = (c < 2 ? dy0 : dy1) * __bfloat162float(w.w3[nn]) * mlp_dsilu(z2[nt][c]);
      dz2T[nn * kLdR + warp * 16 + g + (c >= 2 ? 8 : 0)] = __float2bfloat16_rn(d2[nt][c]);
    }
  // dL/dh1 = dL/dz2 W2 (tensor cores, B = W2 transposed), dL/dz1 = dL/dh1 silu'(z1)
  uint32_t ad[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    ad[kt][0] = mlp_pack(d2[2 * kt][0], d2[2 * kt][1]);
    ad[kt][1] = mlp_pack(d2[2 * kt][2], d2[2 * kt][3]);
    ad[kt][2] = mlp_pack(d2[2 * kt + 1][0], d2[2 * kt + 1][1]);
    ad[kt][3] = mlp_pack(d2[2 * kt + 1][2], d2[2 * kt + 1][3]);
  }
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    float d1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
      uint32_t b[2];
      mlp_ldb(b, w.w2k, kLd2, kt, nt, lane);
      mlp_mma(d1, ad[kt], b);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int nn = nt * 8 + 2 * t + (c & 1);
      dz1T[nn * kLdR + warp * 16 + g + (c >= 2 ? 8 : 0)] = __float2bfloat16_rn(d1[c] * mlp_dsilu(z1[nt][c]));
    }
  }
  __syncthreads();
  // weight gradients over the block's rows (K = kTrainRows): 52 C tiles
  float* gp = grad_part + (int64_t)blockIdx.x * kNParam;
  for (int tile = warp; tile < 52; tile += kTrainWarps) {
    const __nv_bfloat16 *A, *B;
    int mt, nt, kind;
    if (tile < 32) { kind = 0; mt = tile / 8; nt = tile % 8; A = dz2T; B = h1T; }         // W2
    else if (tile < 40) { kind = 1; mt = (tile - 32) / 2; nt = (tile - 32) % 2; A = dz1T; B = fT; }  // W1
    else if (tile < 44) { kind = 2; mt = tile - 40; nt = 0; A = h2T; B = dyT; }           // W3
    else if (tile < 48) { kind = 3; mt = tile - 44; nt = 0; A = dz2T; B = oneT; }         // b2
    else { kind = 4; mt = tile - 48; nt = 0; A = dz1T; B = oneT; }                       // b1
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < kTrainRows / 16; kt++) {
      uint32_t a[4], b[2];
      mlp_lda(a, A, kLdR, mt, kt, lane);
      mlp_ldb(b, B, kLdR, kt, nt, lane);
      mlp_mma(c, a, b);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int m = mt * 16 + g + (q >= 2 ? 8 : 0), nn = nt * 8 + 2 * t + (q & 1);
      if (kind == 0) gp[kOffW2 + m * kMlpH + nn] = c[q];
      else if (kind == 1) gp[kOffW1 + m * kMlpInP + nn] = c[q];
      else if (nn == 0) gp[(kind == 2 ? kOffW3 : kind == 3 ? kOffB2 : kOffB1) + m] = c[q];
    }
  }
  if (threadIdx.x == 0) {
    float a = 0.f, b = 0.f;
    for (int k = 0; k < kTrainWarps; k++) {
      a += red[k];
      b += red[8 + k];
    }
    loss_part[blockIdx.x] = a / (float)n;
    gp[kOffB3] = b;
  }
}

// grad = sum of the block partials (block order); optional Adam step
__global__ void mlp_reduce_adam_kernel(const float* __restrict__ grad_part, const float* __restrict__ loss_part,
                                       int nb, float* grad, float* loss, float* p, float* am, float* av, int step,
                                       float lr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    float l = 0.f;
    for (int b = 0; b < nb; b++) l += loss_part[b];
    *loss = l;
  }
  if (i >= kNParam) return;
  float gs = 0.f;
  for (int b = 0; b < nb; b++) gs += grad_part[(int64_t)b * kNParam + i];
  grad[i] = gs;
  if (step <= 0) return;
  const float b1 = 0.9f, b2 = 0.999f;
  const float m = b1 * am[i] + (1.f - b1) * gs;
  const float v = b2 * av[i] + (1.f - b2) * gs * gs;
  am[i] = m;
  av[i] = v;
  const float mh = m / (1.f - powf(b1, (float)step)), vh = v / (1.f - powf(b2, (float)step));
  p[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

cudaError_t mlp_launch_train(const MlpTrain& m, const float* inputs, const float* targets, const float* weights, int n,
                             int adam_step, float lr, cudaStream_t st) {
  const int nb = (n + kTrainRows - 1) / kTrainRows;
  if (nb < 1 || nb > m.max_blocks) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
  if (e != cudaSuccess) return e;
  mlp_train_kernel<<<nb, 32 * kTrainWarps, kTrainSmem, st>>>(m.image, inputs, targets, weights, n, m.grad_part,
                                                             m.loss_part);
  mlp_reduce_adam_kernel<<<(kNParam + 255) / 256, 256, 0, st>>>(m.grad_part, m.loss_part, nb, m.grad, m.loss,
                                                                 m.params, m.adam_m, m.adam_v, adam_step, lr);
  if (adam_step > 0) return mlp_launch_pack(m.params, m.image, st);
  return cudaGetLastError();
}

// Inference on the 5th-generation tensor cores (mlp_tc.cuh): 128 rows per
// tile, a grid-stride loop of tiles per CTA.  err receives 4 when an MMA
// completion wait gave up.
__global__ void __launch_bounds__(kTcRows) mlp_eval_tc_kernel(const unsigned char* image, const float* in, int64_t n,
                                                              float* out, int* err) {
  extern __shared__ __align__(128) unsigned char tc_raw[];
  MlpTcSmem& sm = *reinterpret_cast<MlpTcSmem*>(tc_raw);
  mlp_tc_setup(sm, image);
  uint32_t phase = 0;
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t row = t * kTcRows + threadIdx.x;
    float f[6];
    for (int k = 0; k < 6; k++) f[k] = row < n ? in[row * 6 + k] : 0.0f;
    float y = 0.0f;
    if (!mlp_tc_forward(sm, phase, f, y, err)) break;
    if (row < n) out[row] = y;
  }
  mlp_tc_teardown(sm);
}

cudaError_t mlp_launch_eval(const unsigned char* image, const float* in, int64_t n, float* out, cudaStream_t st) {
  const int64_t warps = (n + 31) / 32;
  mlp_eval_kernel<<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(image, in, n, out);
  return cudaGetLastError();
}

cudaError_t mlp_launch_eval_tc(const unsigned char* image, const float* in, int64_t n, float* out, int* err,
                               cudaStream_t st) {
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t grid = tiles < 4 * (int64_t)sms ? tiles : 4 * (int64_t)sms;
  mlp_eval_tc_kernel<<<(unsigned)(grid > 0 ? grid : 1), kTcRows, sizeof(MlpTcSmem), st>>>(image, in, n, out, err);
  return cudaGetLastError();
}

// Uniform(-a, a) with a = sqrt(6 / fan_in) (He uniform) from a 64-bit xorshift;
// the output layer starts 10x smaller so the first guesses stay near the
// extrapolation they correct.
void mlp_init_params(float* p, uint64_t seed) {
  uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ull;
  auto uni = [&]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return (double)(s >> 11) / 9007199254740992.0 * 2.0 - 1.0;
  };
  std::memset(p, 0, sizeof(float) * kNParam);
  const double a1 = std::sqrt(6.0 / kMlpIn), a2 = std::sqrt(6.0 / kMlpH), a3 = 0.1 * std::sqrt(6.0 / kMlpH);
  for (int n = 0; n < kMlpH; n++)
    for (int k = 0; k < kMlpIn; k++) p[kOffW1 + n * kMlpInP + k] = (float)(a1 * uni());
  for (int i = 0; i < kMlpH * kMlpH; i++) p[kOffW2 + i] = (float)(a2 * uni());
  for (int i = 0; i < kMlpH; i++) p[kOffW3 + i] = (float)(a3 * uni());
}

}  // namespace tf

// ------------------------------------------------------------------ C ABI
namespace {
struct DevBuf {
  std::vector<void*> ptrs;
  ~DevBuf() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n ? n * sizeof(T) : 16) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (T*)p;
  }
};
int mlp_fail(int code, const std::string& m) {
  tf::set_thread_error(m);
  return code;
}
int mlp_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TF_OK;
  return mlp_fail(TF_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

extern "C" {

TF_API int tf_mlp_param_count(void) { return tf::kNParam; }

TF_API int tf_mlp_init(uint64_t seed, float* params) {
  if (!params) return mlp_fail(TF_E_ARG, "params is NULL");
  tf::mlp_init_params(params, seed);
  return TF_OK;
}

TF_API int tf_mlp_forward(const float* params, int64_t n, const float* inputs, float* outputs) {
  if (!params || !inputs || !outputs || n <= 0) return mlp_fail(TF_E_ARG, "tf_mlp_forward: bad arguments");
  DevBuf b;
  float* p = b.get<float>(tf::kNParam);
  unsigned char* img = b.get<unsigned char>(tf::kImgBytes);
  float* in = b.get<float>((size_t)n * 6);
  float* out = b.get<float>((size_t)n);
  if (!p || !img || !in || !out) return mlp_fail(TF_E_CUDA, "tf_mlp_forward: device allocation failed");
  int rc;
  if ((rc = mlp_cuda(cudaMemcpy(p, params, sizeof(float) * tf::kNParam, cudaMemcpyHostToDevice), "copy"))) return rc;
  if ((rc = mlp_cuda(cudaMemcpy(in, inputs, sizeof(float) * 6 * n, cudaMemcpyHostToDevice), "copy"))) return rc;
  int* err = b.get<int>(1);
  if (!err) return mlp_fail(TF_E_CUDA, "tf_mlp_forward: device allocation failed");
  if ((rc = mlp_cuda(cudaMemset(err, 0, sizeof(int)), "memset"))) return rc;
  if ((rc = mlp_cuda(tf::mlp_launch_pack(p, img, 0), "pack"))) return rc;
  if ((rc = mlp_cuda(tf::mlp_launch_eval_tc(img, in, n, out, err, 0), "eval"))) return rc;
  int e = 0;
  if ((rc = mlp_cuda(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost), "copy"))) return rc;
  if (e) return mlp_fail(TF_E_CUDA, "tf_mlp_forward: a tensor-core completion wait ran out of time");
  return mlp_cuda(cudaMemcpy(outputs, out, sizeof(float) * n, cudaMemcpyDeviceToHost), "copy");
}

TF_API int tf_mlp_gradient(const float* params, int64_t n, const float* inputs, const float* targets,
                           const float* weights, float* grad, float* loss) {
  if (!params || !inputs || !targets || !grad || n <= 0 || n > (1 << 24))
    return mlp_fail(TF_E_ARG, "tf_mlp_gradient: bad arguments");
  DevBuf b;
  tf::MlpTrain m;
  m.max_blocks = (int)((n + tf::mlp_train_rows_per_block() - 1) / tf::mlp_train_rows_per_block());
  m.params = b.get<float>(tf::kNParam);
  m.adam_m = b.get<float>(tf::kNParam);
  m.adam_v = b.get<float>(tf::kNParam);
  m.image = b.get<unsigned char>(tf::kImgBytes);
  m.grad_part = b.get<float>((size_t)m.max_blocks * tf::kNParam);
  m.loss_part = b.get<float>(m.max_blocks);
  m.grad = b.get<float>(tf::kNParam);
  m.loss = b.get<float>(1);
  float* in = b.get<float>((size_t)n * 6);
  float* tg = b.get<float>((size_t)n);
  float* wt = b.get<float>((size_t)n);
  if (!m.params || !m.grad_part || !in || !tg || !wt || !m.grad || !m.loss)
    return mlp_fail(TF_E_CUDA, "tf_mlp_gradient: device allocation failed");
  std::vector<float> ones;
  if (!weights) {
    ones.assign((size_t)n, 1.0f);
    weights = ones.data();
  }
  int rc;
  if ((rc = mlp_cuda(cudaMemcpy(m.params, params, sizeof(float) * tf::kNParam, cudaMemcpyHostToDevice), "copy")))
    return rc;
  if ((rc = mlp_cuda(cudaMemcpy(in, inputs, sizeof(float) * 6 * n, cudaMemcpyHostToDevice), "copy"))) return rc;
  if ((rc = mlp_cuda(cudaMemcpy(tg, targets, sizeof(float) * n, cudaMemcpyHostToDevice), "copy"))) return rc;
  if ((rc = mlp_cuda(cudaMemcpy(wt, weights, sizeof(float) * n, cudaMemcpyHostToDevice), "copy"))) return rc;
  if ((rc = mlp_cuda(tf::mlp_launch_pack(m.params, m.image, 0), "pack"))) return rc;
  if ((rc = mlp_cuda(tf::mlp_launch_train(m, in, tg, wt, (int)n, 0, 0.0f, 0), "train"))) return rc;
  if ((rc = mlp_cuda(cudaMemcpy(grad, m.grad, sizeof(float) * tf::kNParam, cudaMemcpyDeviceToHost), "copy")))
    return rc;
  if (loss) return mlp_cuda(cudaMemcpy(loss, m.loss, sizeof(float), cudaMemcpyDeviceToHost), "copy");
  return TF_OK;
}

}  // extern "C"
