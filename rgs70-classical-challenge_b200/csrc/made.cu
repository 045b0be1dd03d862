// Masked autoregressive proposal network (MADE, Germain et al. 2015): BF16 GEMMs with
// FP32 accumulation on the tensor cores (mma.sync m16n8k16), fused epilogues, and the
// loss / gradient / Adam kernels of its training.
//
// Network: x in {0,1}^n (scan order) -> h1 = relu((W1*M1) x + b1) -> h2 = relu((W2*M2) h1
// + b2) -> z = (W3*M3) h2 + b3, q(x_d = 1 | x_<d) = sigmoid(z_d).  Masks M1..M3 enforce
// the autoregressive order; the masked weights are kept as BF16 copies for the GEMMs and
// as FP32 masters for the optimiser.
//
// The network is a few percent of a sample's cost next to the scan, so its GEMMs use the
// warp-level MMA; everything stays on the device (no host round trips per step).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "common.hpp"
#include "made.hpp"

namespace rgs {

namespace {

constexpr int BM = 64, BN = 64, BK = 32, PADK = 8;

__device__ __forceinline__ unsigned pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M x N] = op(A)[M x K] * op(B)[K x N]; A row-major [M][lda] (transA: [K][lda]), B
// row-major [K][ldb] (transB: [N][ldb]).  128 threads: 4 warps in a 2x2 grid of 32x32.
__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmArgs g) {
  __shared__ __nv_bfloat16 As[BM][BK + PADK];
  __shared__ __nv_bfloat16 Bs[BN][BK + PADK];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int grp = lane >> 2, tig = lane & 3;
  float acc[2][4][4];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 4; ++j)
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < g.K; k0 += BK) {
    for (int idx = threadIdx.x; idx < BM * BK; idx += blockDim.x) {
      const int r = idx / BK, c = idx % BK;  // (m, k) of the tile
      const int m = m0 + r, k = k0 + c;
      __nv_bfloat16 v = zero;
      if (m < g.M && k < g.K) v = g.transA ? g.A[(size_t)k * g.lda + m] : g.A[(size_t)m * g.lda + k];
      As[r][c] = v;
    }
    for (int idx = threadIdx.x; idx < BN * BK; idx += blockDim.x) {
      const int r = idx / BK, c = idx % BK;  // (n, k) of the tile
      const int n = n0 + r, k = k0 + c;
      __nv_bfloat16 v = zero;
      if (n < g.N && k < g.K) v = g.transB ? g.B[(size_t)n * g.ldb + k] : g.B[(size_t)k * g.ldb + n];
      Bs[r][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + grp;
        a[i][0] = pack_bf16(As[r][kk + tig * 2], As[r][kk + tig * 2 + 1]);
        a[i][1] = pack_bf16(As[r + 8][kk + tig * 2], As[r + 8][kk + tig * 2 + 1]);
        a[i][2] = pack_bf16(As[r][kk + tig * 2 + 8], As[r][kk + tig * 2 + 9]);
        a[i][3] = pack_bf16(As[r + 8][kk + tig * 2 + 8], As[r + 8][kk + tig * 2 + 9]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + grp;
        b[j][0] = pack_bf16(Bs[c][kk + tig * 2], Bs[c][kk + tig * 2 + 1]);
        b[j][1] = pack_bf16(Bs[c][kk + tig * 2 + 8], Bs[c][kk + tig * 2 + 9]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  // Epilogue: + bias[n], relu, * mask[m][n], * (gate[m][n] > 0); fp32 and/or bf16 out.
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + i * 16 + grp + (e >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + tig * 2 + (e & 1);
        if (m >= g.M || n >= g.N) continue;
        float v = acc[i][j][e] * g.alpha;
        if (g.bias) v += g.bias[n];
        if (g.relu) v = fmaxf(v, 0.f);
        if (g.mask) v *= (float)g.mask[(size_t)m * g.N + n];
        if (g.gate && !(__bfloat162float(g.gate[(size_t)m * g.ldc + n]) > 0.f)) v = 0.f;
        if (g.C) g.C[(size_t)m * g.ldc + n] = v;
        if (g.Cb) g.Cb[(size_t)m * g.ldc + n] = __float2bfloat16(v);
      }
}

// dz = sigmoid(z) - target; loss partials: softplus(z) - target * z (per block, float64).
__global__ void bce_grad_kernel(const float* __restrict__ z, const float* __restrict__ target, int count,
                                float scale, __nv_bfloat16* __restrict__ dz, double* __restrict__ partial) {
  __shared__ double red[256];
  double loss = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float x = z[i], t = target[i];
    const float s = 1.f / (1.f + __expf(-x));
    dz[i] = __float2bfloat16((s - t) * scale);
    const float sp = x > 0.f ? x + log1pf(__expf(-x)) : log1pf(__expf(x));
    loss += (double)(sp - t * x);
  }
  red[threadIdx.x] = loss;
  __syncthreads();
  for (int off = blockDim.x / 2; off; off >>= 1) {
    if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Column sums of a [rows x cols] bf16 matrix (bias gradients).
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ x, int rows, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += __bfloat162float(x[(size_t)r * cols + c]);
  out[c] = s;
}

// Adam step on FP32 masters, then the masked BF16 copy used by the GEMMs.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m1,
                            float* __restrict__ m2, const unsigned char* __restrict__ mask,
                            __nv_bfloat16* __restrict__ wb, int count, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gr = grad[i];
  const float a = b1 * m1[i] + (1.f - b1) * gr;
  const float v = b2 * m2[i] + (1.f - b2) * gr * gr;
  m1[i] = a;
  m2[i] = v;
  const float nw = w[i] - lr * (a / c1) / (sqrtf(v / c2) + eps);
  w[i] = nw;
  if (wb) wb[i] = __float2bfloat16(mask ? nw * (float)mask[i] : nw);
}

// One autoregressive position for a batch: x[:, d] ~ Bernoulli(sigmoid(z[:, d])) with a
// Philox-free counter hash uniform, and log q accumulation.  Rows of x are bf16 {0, 1}.
__device__ __forceinline__ double hash_uniform(unsigned long long seed, unsigned long long a, unsigned b) {
  unsigned long long h = seed ^ (a * 0x9E3779B97F4A7C15ull) ^ ((unsigned long long)b * 0xC2B2AE3D27D4EB4Full);
  h ^= h >> 31;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 27;
  h *= 0x94D049BB133111EBull;
  h ^= h >> 31;
  return (double)(h >> 11) * 0x1.0p-53;
}

__global__ void sample_position_kernel(const float* __restrict__ z, int n, int d, int count, unsigned long long seed,
                                       unsigned long long first, __nv_bfloat16* __restrict__ x,
                                       double* __restrict__ logq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float zd = z[(size_t)i * n + d];
  const double q1 = 1.0 / (1.0 + exp(-(double)zd));
  const double u = hash_uniform(seed, first + i, (unsigned)d);
  const int bit = u < q1 ? 1 : 0;
  x[(size_t)i * n + d] = __float2bfloat16((float)bit);
  logq[i] += log(bit ? q1 : 1.0 - q1);
}

// log q(x) = sum_d log sigmoid(+-z_d) for given x.
__global__ void logq_kernel(const float* __restrict__ z, const __nv_bfloat16* __restrict__ x, int n, int count,
                            double* __restrict__ logq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  double s = 0.0;
  for (int d = 0; d < n; ++d) {
    const double zd = z[(size_t)i * n + d];
    const double sign = __bfloat162float(x[(size_t)i * n + d]) > 0.5f ? 1.0 : -1.0;
    const double t = sign * zd;  // log sigmoid(t) = -softplus(-t)
    s += t > 0 ? -log1p(exp(-t)) : t - log1p(exp(t));
  }
  logq[i] = s;
}

}  // namespace

int gemm_bf16(const GemmArgs& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0 || !g.A || !g.B || (!g.C && !g.Cb)) return fail(RGS_ERR_ARG, "bad GEMM");
  dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM);
  gemm_bf16_kernel<<<grid, 128, 0, s>>>(g);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int bce_grad(const float* z, const float* target, int count, float scale, __nv_bfloat16* dz, double* partial,
             int blocks, cudaStream_t s) {
  bce_grad_kernel<<<blocks, 256, 0, s>>>(z, target, count, scale, dz, partial);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int colsum_bf16(const __nv_bfloat16* x, int rows, int cols, float* out, cudaStream_t s) {
  colsum_kernel<<<(cols + 127) / 128, 128, 0, s>>>(x, rows, cols, out);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int adam_step(float* w, const float* grad, float* m1, float* m2, const unsigned char* mask, __nv_bfloat16* wb,
              int count, float lr, float b1, float b2, float eps, int t, cudaStream_t s) {
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  adam_kernel<<<(count + 255) / 256, 256, 0, s>>>(w, grad, m1, m2, mask, wb, count, lr, b1, b2, eps, c1, c2);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int sample_position(const float* z, int n, int d, int count, unsigned long long seed, unsigned long long first,
                    __nv_bfloat16* x, double* logq, cudaStream_t s) {
  sample_position_kernel<<<(count + 255) / 256, 256, 0, s>>>(z, n, d, count, seed, first, x, logq);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int log_q(const float* z, const __nv_bfloat16* x, int n, int count, double* logq, cudaStream_t s) {
  logq_kernel<<<(count + 255) / 256, 256, 0, s>>>(z, x, n, count, logq);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

}  // namespace rgs
