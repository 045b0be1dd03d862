// Masked autoregressive proposal network (MADE, Germain et al. 2015): BF16 GEMMs with
// FP32 accumulation on the Blackwell tensor cores (tcgen05.mma, accumulators in TMEM),
// fused epilogues, and the loss / gradient / Adam kernels of its training.
//
// Network: x in {0,1}^n (scan order) -> h1 = relu((W1*M1) x + b1) -> h2 = relu((W2*M2) h1
// + b2) -> z = (W3*M3) h2 + b3, q(x_d = 1 | x_<d) = sigmoid(z_d).  Masks M1..M3 enforce
// the autoregressive order; the masked weights are kept as BF16 copies for the GEMMs and
// as FP32 masters for the optimiser.  Everything stays on the device (no host round
// trips per step).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "common.hpp"
#include "made.hpp"
#include "tcgen05.cuh"
#include "tma_map.hpp"

namespace rgs {

// Set when a bounded wait of this file's GEMM gave up (read by tensor_core_status).
__device__ int g_tc_timeout = 0;

int wht_tensor_core_timeout(int* timed_out);
int fourier_tma_timeout(int* timed_out);

namespace {

// CTA tile of the tensor-core GEMM: 128 x 128 outputs (one TMEM accumulator of 128 lanes
// x 128 fp32 columns), K in slices of 64.  Operands staged by the threads use two
// shared-memory stages; TMA-loaded operands a three-stage pipeline (the loads of slices
// k + 1 and k + 2 in flight while slice k is multiplied), two CTAs per SM.
constexpr int TBM = 128, TBN = 128, TBK = 64, kStages = 2, kTmaStages = 3;
constexpr int kTileBytes = TBM * TBK * 2;  // one 128 x 64 bf16 operand tile (16 KiB)
constexpr int kGemmSmem = kTmaStages * 2 * kTileBytes + 1024 + 64;

// Byte offset of the 16-byte chunk (row r, k-chunk kc) of a 128 x 64 operand tile in the
// K-major no-swizzle layout: core matrices of 8 rows x 16 bytes, the eight k-chunks of a
// row group 128 bytes apart (LBO), row groups 1024 bytes apart (SBO).
__device__ __forceinline__ uint32_t cm_off(int r, int kc) { return (uint32_t)((r >> 3) * 1024 + kc * 128 + (r & 7) * 16); }

__device__ __forceinline__ unsigned bf_bits(const __nv_bfloat16* p) { return (unsigned)__bfloat16_as_ushort(*p); }

__device__ __forceinline__ unsigned word_of(const uint4& v, int w) {
  return w == 0 ? v.x : (w == 1 ? v.y : (w == 2 ? v.z : v.w));
}

// Eight consecutive bf16 values, those at index >= valid replaced by zero.
__device__ __forceinline__ uint4 load8_partial(const __nv_bfloat16* src, int valid) {
  unsigned w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int j = 0; j < 8; ++j)
    if (j < valid) w[j >> 1] |= bf_bits(src + j) << (16 * (j & 1));
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// Rows [r0, r0 + 128) x k [k0, k0 + 64) of a logical R x K operand into the K-major
// layout; zero outside the operand.  kmajor: element (r, k) at G[r * ld + k]; otherwise
// at G[k * ld + r] (MN-major: transposed in registers on the way).  128 threads, one
// 8 x 8 core matrix each; vec: 16-byte loads are aligned (ld % 8 == 0, G 16-byte aligned).
__device__ __forceinline__ void stage_tile(unsigned char* tile, const __nv_bfloat16* __restrict__ G, int ld, int R,
                                           int K, int r0, int k0, bool kmajor, bool vec) {
  const int t = threadIdx.x;
  if (kmajor) {
    const int kc = t & 7, rg = t >> 3;
    const int k = k0 + kc * 8;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int ii = (i + kc) & 7;  // rotated so that a quarter warp hits distinct banks
      const int r = r0 + rg * 8 + ii;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (r < R && k < K) {
        const __nv_bfloat16* src = G + (size_t)r * ld + k;
        v = (vec && k + 8 <= K) ? __ldg(reinterpret_cast<const uint4*>(src)) : load8_partial(src, K - k);
      }
      *reinterpret_cast<uint4*>(tile + cm_off(rg * 8 + ii, kc)) = v;
    }
  } else {
    const int rg = t & 15, kc = t >> 4;
    const int r = r0 + rg * 8;
    uint4 rows[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + kc * 8 + j;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (k < K && r < R) {
        const __nv_bfloat16* src = G + (size_t)k * ld + r;
        v = (vec && r + 8 <= R) ? __ldg(reinterpret_cast<const uint4*>(src)) : load8_partial(src, R - r);
      }
      rows[j] = v;
    }
    // Row e of the core matrix = element e of the eight loaded k-rows.
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int e = (i + rg) & 7;
      const unsigned sel = (e & 1) ? 0x7632u : 0x5410u;
      unsigned w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const unsigned a = word_of(rows[2 * j], e >> 1), b = word_of(rows[2 * j + 1], e >> 1);
        w[j] = __byte_perm(a, b, sel);
      }
      *reinterpret_cast<uint4*>(tile + cm_off(rg * 8 + e, kc)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// TMA descriptors of the operands that are K-major with 16-byte aligned rows (boxes of
// 64 K-elements x 128 rows, 128-byte swizzle); the others are staged by the threads.
struct GemmMaps {
  CUtensorMap a, b;
  int tma_a, tma_b;
};

// C[M x N] = op(A)[M x K] * op(B)[K x N]; A row-major [M][lda] (transA: [K][lda]), B
// row-major [K][ldb] (transB: [N][ldb]).  One CTA of 128 threads per 128 x 128 tile of C,
// K in slices of 64 over two shared-memory stages.  Per slice: thread 0 starts the TMA
// loads of the K-major aligned operands (one 64 x 128 box each, completing on the stage's
// `full` mbarrier), the threads stage the other operands (MN-major operands transposed
// in registers); thread 0 then waits for the TMA bytes, issues four tcgen05.mma (K = 16
// each) into the TMEM accumulator and commits them to the stage's `done` mbarrier,
// which gates the reuse of that stage.  After the last slice every warp reads its 32 TMEM
// lanes (rows) and applies the epilogue.
__global__ void __launch_bounds__(128) gemm_tc_kernel(GemmArgs g, const __grid_constant__ GemmMaps maps) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kTmaStages * 2 * kTileBytes);  // done[3], full[3]
  uint64_t* full = bars + kTmaStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kTmaStages);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * TBM, n0 = blockIdx.x * TBN;
  const bool tma = maps.tma_a || maps.tma_b;
  const uint32_t tx_bytes = (maps.tma_a ? kTileBytes : 0) + (maps.tma_b ? kTileBytes : 0);
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2 * kTmaStages; ++s) tc::mbar_init(&bars[s], 1);
    tc::fence_barrier_init();
  }
  if (warp == 0) tc::tmem_alloc(tmem_slot, TBN);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const bool vecA = (g.lda % 8 == 0) && (((uintptr_t)g.A & 15) == 0);
  const bool vecB = (g.ldb % 8 == 0) && (((uintptr_t)g.B & 15) == 0);
  const int KT = (g.K + TBK - 1) / TBK;
  const uint32_t idesc = tc::instr_desc(TBM, TBN, 1);
  bool ok = true;
  if (maps.tma_a && maps.tma_b) {
    // One thread issues the loads kTmaStages slices ahead and the MMAs; a stage is refilled
    // once the MMAs that read it have completed (its done barrier).  Every wait is bounded;
    // after one gives up, the loads still in flight and the last MMAs are waited for (also
    // bounded) before the block frees its TMEM.
    if (threadIdx.x == 0) {
      int issued = 0, consumed = 0, committed = -1;
      auto issue = [&](int kt) {
        const int s = kt % kTmaStages;
        unsigned char* As = base + s * 2 * kTileBytes;
        tc::mbar_expect_tx(&full[s], 2 * kTileBytes);
        tc::tma_load_2d(As, &maps.a, kt * TBK, m0, &full[s]);
        tc::tma_load_2d(As + kTileBytes, &maps.b, kt * TBK, n0, &full[s]);
        ++issued;
      };
      for (int kt = 0; kt < KT && kt < kTmaStages; ++kt) issue(kt);
      for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % kTmaStages;
        const uint32_t ph = (uint32_t)(kt / kTmaStages) & 1u;
        if (!tc::mbar_wait(&full[s], ph)) {
          ok = false;
          break;
        }
        ++consumed;
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(base + s * 2 * kTileBytes), b0 = a0 + kTileBytes;
#pragma unroll
        for (int k = 0; k < TBK / 16; ++k)
          tc::mma_f16(tmem, tc::smem_desc(a0 + k * 32, 16, 1024, 2), tc::smem_desc(b0 + k * 32, 16, 1024, 2), idesc,
                      (kt > 0 || k > 0) ? 1u : 0u);
        tc::mma_commit(&bars[s]);
        committed = kt;
        if (kt + kTmaStages < KT) {
          if (!tc::mbar_wait(&bars[s], ph)) {
            ok = false;
            break;
          }
          issue(kt + kTmaStages);
        }
      }
      if (committed >= 0 && !tc::mbar_wait(&bars[committed % kTmaStages], (uint32_t)(committed / kTmaStages) & 1u))
        ok = false;
      if (!ok)
        for (int kt = consumed; kt < issued; ++kt) tc::mbar_wait(&full[kt % kTmaStages], (uint32_t)(kt / kTmaStages) & 1u);
    }
  } else {
  for (int kt = 0; kt < KT; ++kt) {
    const int s = kt & 1;
    if (kt >= kStages && !tc::mbar_wait(&bars[s], (uint32_t)((kt >> 1) - 1) & 1u)) ok = false;
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    unsigned char* As = base + s * 2 * kTileBytes;
    unsigned char* Bs = As + kTileBytes;
    if (tma && threadIdx.x == 0) {
      tc::mbar_expect_tx(&full[s], tx_bytes);
      if (maps.tma_a) tc::tma_load_2d(As, &maps.a, kt * TBK, m0, &full[s]);
      if (maps.tma_b) tc::tma_load_2d(Bs, &maps.b, kt * TBK, n0, &full[s]);
    }
    if (!maps.tma_a) stage_tile(As, g.A, g.lda, g.M, g.K, m0, kt * TBK, !g.transA, vecA);
    if (!maps.tma_b) stage_tile(Bs, g.B, g.ldb, g.N, g.K, n0, kt * TBK, g.transB != 0, vecB);
    tc::fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      if (tma && !tc::mbar_wait(&full[s], (uint32_t)(kt >> 1) & 1u)) {
        ok = false;  // no MMA: the next wait on this stage gives up too, and every thread leaves
      } else {
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(As), b0 = tc::smem_u32(Bs);
#pragma unroll
        for (int k = 0; k < TBK / 16; ++k) {
          // TMA tiles: rows 128 bytes apart (128-byte swizzle), slice k at +32 k bytes;
          // staged tiles: core matrices (LBO 128, SBO 1024), slice k at +256 k bytes.
          const uint64_t ad = maps.tma_a ? tc::smem_desc(a0 + k * 32, 16, 1024, 2)
                                         : tc::smem_desc(a0 + k * 256, 128, 1024, 0);
          const uint64_t bd = maps.tma_b ? tc::smem_desc(b0 + k * 32, 16, 1024, 2)
                                         : tc::smem_desc(b0 + k * 256, 128, 1024, 0);
          tc::mma_f16(tmem, ad, bd, idesc, (kt > 0 || k > 0) ? 1u : 0u);
        }
        tc::mma_commit(&bars[s]);
      }
    }
  }
  if (ok && KT > 0 && !tc::mbar_wait(&bars[(KT - 1) & 1], (uint32_t)((KT - 1) >> 1) & 1u)) ok = false;
  }
  ok = __syncthreads_and(ok);
  tc::fence_after_sync();
  if (ok) {
    const int m = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < TBN && n0 + c0 < g.N; c0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      tc::tmem_ld_wait();
      if (m >= g.M) continue;
      if (g.C && !g.Cb && !g.mask && !g.gate && n0 + c0 + 16 <= g.N && (g.ldc & 3) == 0 &&
          (((uintptr_t)g.C) & 15) == 0) {
        // 16 consecutive columns of row m: four 16-byte stores.
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          v[j] = __uint_as_float(r[j]) * g.alpha;
          if (g.bias) v[j] += g.bias[n0 + c0 + j];
          if (g.relu) v[j] = fmaxf(v[j], 0.f);
        }
        float4* dst = reinterpret_cast<float4*>(g.C + (size_t)m * g.ldc + n0 + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        continue;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + c0 + j;
        if (n >= g.N) break;
        float v = __uint_as_float(r[j]) * g.alpha;
        if (g.bias) v += g.bias[n];
        if (g.relu) v = fmaxf(v, 0.f);
        if (g.mask) v *= (float)g.mask[(size_t)m * g.N + n];
        if (g.gate && !(__bfloat162float(g.gate[(size_t)m * g.ldc + n]) > 0.f)) v = 0.f;
        if (g.C) g.C[(size_t)m * g.ldc + n] = v;
        if (g.Cb) g.Cb[(size_t)m * g.ldc + n] = __float2bfloat16(v);
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(&g_tc_timeout, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TBN);
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

namespace {
// Tensor map of a K-major bf16 operand [rows][ld] (K innermost): boxes of 64 x 128 with
// 128-byte swizzle, zero fill outside the operand.  False when TMA cannot load it (row
// pitch not a multiple of 16 bytes, unaligned base, or no encoder).
bool tma_operand(CUtensorMap* map, const __nv_bfloat16* ptr, int ld, int K, int rows) {
  if (((uintptr_t)ptr & 15) != 0 || (ld % 8) != 0 || K <= 0 || rows <= 0) return false;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TBK, (cuuint32_t)TBM};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)ptr, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// TMA operand loads on (default) or off (every operand staged by the threads).
bool g_gemm_tma = true;
}  // namespace

int gemm_set_tma(int on) {
  g_gemm_tma = on != 0;
  return RGS_OK;
}

int gemm_bf16(const GemmArgs& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0 || !g.A || !g.B || (!g.C && !g.Cb)) return fail(RGS_ERR_ARG, "bad GEMM");
  static bool configured[64] = {false};
  int device = 0;
  RGS_CUDA_TRY(cudaGetDevice(&device));
  if (device >= 0 && device < 64 && !configured[device]) {
    RGS_CUDA_TRY(cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
    configured[device] = true;
  }
  GemmMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  // A is K-major unless transposed; B is K-major when transposed ([N][ldb]).
  if (g_gemm_tma && !g.transA && tma_operand(&maps.a, g.A, g.lda, g.K, g.M)) maps.tma_a = 1;
  if (g_gemm_tma && g.transB && tma_operand(&maps.b, g.B, g.ldb, g.K, g.N)) maps.tma_b = 1;
  dim3 grid((g.N + TBN - 1) / TBN, (g.M + TBM - 1) / TBM);
  gemm_tc_kernel<<<grid, 128, kGemmSmem, s>>>(g, maps);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int tensor_core_status(int* timed_out) {
  int h = 0, zero = 0;
  RGS_CUDA_TRY(cudaMemcpyFromSymbol(&h, g_tc_timeout, sizeof(int)));
  RGS_CUDA_TRY(cudaMemcpyToSymbol(g_tc_timeout, &zero, sizeof(int)));
  int w = 0, f = 0;
  int rc = wht_tensor_core_timeout(&w);
  if (rc) return rc;
  if ((rc = fourier_tma_timeout(&f))) return rc;
  *timed_out = h | w | f;
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
