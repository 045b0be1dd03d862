// Walsh-Hadamard butterflies on the tensor cores: 16 x 16 Hadamard blocks applied with
// tcgen05.mma on a split-BF16 copy of the complex64 state (the optional precision path
// of the Fourier-cut sampler's WHT; FP32 butterflies are fourier.cu).
//
// Reference ops replaced (whyihaveyou/rgs70-classical-challenge, W/ = work/rgs_attack/):
// lowfwht / localfwht (W/distributed_sampler.py:21-31) and fusedfwht
// (W/fourier_fused_sampler.py:19-32), in-place butterflies (x + y, x - y) on a bit range.
//
// A pass streams the state in tiles of 4096 elements held in shared memory as FP32:
// contiguous tiles for bits 0..11, or (strided passes) 2^c contiguous elements x 2^k
// target bits [b0, b0 + k) with c + k = 12.  Each round acts on a 4-bit window [w, w + 4)
// of the tile-local index: the 16 values of every fibre of that window are multiplied by
// B = (x) over the window's bits of (H = [[1, 1], [1, -1]] if the bit is transformed, else
// I), whose entries 0 / +-1 are exact in BF16.  As a GEMM: D[512 x 16] = A[512 x 16] B^T, rows =
// (fibre, re / im) in four blocks of M = 128, K = N = 16, A = the fibres split into T
// BF16 terms (x = hi + mid + lo) accumulated into the same TMEM columns, so the product
// carries about 8 T significant bits of each input (T = 2: ~4e-6 relative per round,
// T = 3: FP32 level).  Per round: stage A from the FP32 tile (generic stores, proxy fence),
// one thread issues 4 T MMAs and commits to an mbarrier, all threads wait (bounded), read
// their TMEM lanes (tcgen05.ld) and write the results back into the tile.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "common.hpp"
#include "fourier.cuh"
#include "tcgen05.cuh"

namespace rgs {

// Set when a bounded wait of this file's kernel gave up (read by tensor_core_status).
__device__ int g_wht_timeout = 0;

namespace {

constexpr int kTileElems = 4096;      // complex64 elements per tile (32 KiB of FP32)
constexpr int kBlockBytes = 128 * 32;  // one 128-row x 16-column bf16 A block (4 KiB)
constexpr int kThreads = 256;

struct WhtPass {
  int m;         // state bits
  int b0, k, c;  // target bits [b0, b0 + k) of the global index, c contiguous low bits
  int rounds;
  int w[3];         // tile-local window start (0, 4 or 8)
  unsigned mask[3];  // transformed bits of the window (bit i <-> tile-local bit w + i)
};

template <int T>
struct WhtSmem {
  float tile[2 * kTileElems];
  __align__(1024) unsigned char a[T][4][kBlockBytes];
  __align__(128) unsigned char b[3][512];
  uint64_t bar;
  uint32_t tmem;
};

// Byte offset of (row, k) in a K-major no-swizzle operand of 16 columns: core matrices of
// 8 rows x 16 bytes, the two k-chunks of a row group 128 bytes apart (LBO), row groups
// 256 bytes apart (SBO).
__device__ __forceinline__ int kmaj16(int row, int k) { return (row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2; }

__device__ __forceinline__ unsigned pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (unsigned)__bfloat16_as_ushort(a) | ((unsigned)__bfloat16_as_ushort(b) << 16);
}

// Global element index of tile-local element i of tile base `base`.
__device__ __forceinline__ unsigned long long global_index(const WhtPass& P, unsigned long long base, int i) {
  const int low = i & ((1 << P.c) - 1), t = i >> P.c;
  return base + ((unsigned long long)t << P.b0) + (unsigned long long)low;
}

template <int T>
__global__ void __launch_bounds__(kThreads, 2) wht_tc_kernel(float2* __restrict__ v, const __grid_constant__ WhtPass P) {
  extern __shared__ unsigned char smem_raw[];
  WhtSmem<T>& S = *reinterpret_cast<WhtSmem<T>*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // B matrices of the rounds: entry (n, k) = prod over window bits of H or I.
  for (int r = 0; r < P.rounds; ++r)
    for (int e = tid; e < 256; e += kThreads) {
      const int n = e >> 4, k = e & 15;
      int val = 1;
      for (int i = 0; i < 4; ++i) {
        const int a = (n >> i) & 1, b = (k >> i) & 1;
        if ((P.mask[r] >> i) & 1u)
          val = (a & b) ? -val : val;
        else if (a != b)
          val = 0;
      }
      *reinterpret_cast<__nv_bfloat16*>(S.b[r] + kmaj16(n, k)) = __float2bfloat16((float)val);
    }
  if (tid == 0) {
    tc::mbar_init(&S.bar, 1);
    tc::fence_barrier_init();
  }
  if (warp == 0) tc::tmem_alloc(&S.tmem, 64);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t idesc = tc::instr_desc(128, 16, 1);
  const unsigned long long ntiles = 1ull << (P.m - 12);
  const unsigned long long lowmask = (1ull << (P.b0 - P.c)) - 1ull;
  uint32_t phase = 0;
  bool ok = true;

  for (unsigned long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const unsigned long long base = ((tile & lowmask) << P.c) | ((tile >> (P.b0 - P.c)) << (P.b0 + P.k));
    // Load: pairs of consecutive tile-local elements are consecutive in memory (c >= 1).
    for (int q = tid; q < kTileElems / 2; q += kThreads) {
      const float4 x = __ldg(reinterpret_cast<const float4*>(v + global_index(P, base, 2 * q)));
      reinterpret_cast<float4*>(S.tile)[q] = x;
    }
    __syncthreads();
    for (int r = 0; r < P.rounds; ++r) {
      const int w = P.w[r];
      // Stage A: thread tid owns fibre j = tid (rows 2j: real, 2j + 1: imaginary parts).
      {
        const int j = tid;
        const int lo = j & ((1 << w) - 1), hi = j >> w;
        const int i0 = (hi << (w + 4)) | lo;
        float re[16], im[16];
        if (w == 0) {
          // The 16 values are contiguous: float4 reads.
#pragma unroll
          for (int p = 0; p < 8; ++p) {
            const float4 x = reinterpret_cast<const float4*>(S.tile)[(i0 >> 1) + p];
            re[2 * p] = x.x, im[2 * p] = x.y, re[2 * p + 1] = x.z, im[2 * p + 1] = x.w;
          }
        } else {
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const float2 x = reinterpret_cast<const float2*>(S.tile)[i0 | (k << w)];
            re[k] = x.x, im[k] = x.y;
          }
        }
        const int blk = j >> 6, row = (2 * j) & 127;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          const float* x = part ? im : re;
          float rem[16];
#pragma unroll
          for (int k = 0; k < 16; ++k) rem[k] = x[k];
#pragma unroll
          for (int t = 0; t < T; ++t) {
            unsigned wv[8];
#pragma unroll
            for (int k = 0; k < 16; k += 2) {
              const __nv_bfloat16 a = __float2bfloat16_rn(rem[k]), b = __float2bfloat16_rn(rem[k + 1]);
              rem[k] -= __bfloat162float(a);
              rem[k + 1] -= __bfloat162float(b);
              wv[k >> 1] = pack2(a, b);
            }
            unsigned char* dst = S.a[t][blk];
            *reinterpret_cast<uint4*>(dst + kmaj16(row + part, 0)) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            *reinterpret_cast<uint4*>(dst + kmaj16(row + part, 8)) = make_uint4(wv[4], wv[5], wv[6], wv[7]);
          }
        }
      }
      tc::fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t bdesc_addr = tc::smem_u32(S.b[r]);
#pragma unroll
        for (int blk = 0; blk < 4; ++blk)
#pragma unroll
          for (int t = 0; t < T; ++t)
            tc::mma_f16(tmem + 16u * blk, tc::smem_desc(tc::smem_u32(S.a[t][blk]), 128, 256, 0),
                        tc::smem_desc(bdesc_addr, 128, 256, 0), idesc, t > 0 ? 1u : 0u);
        tc::mma_commit(&S.bar);
      }
      if (!tc::mbar_wait(&S.bar, phase & 1u)) ok = false;
      ++phase;
      ok = __syncthreads_and(ok);
      if (!ok) break;
      tc::fence_after_sync();
      // Epilogue: warps 0-3 read blocks 0-1, warps 4-7 blocks 2-3 (TMEM lanes 32 (warp % 4) + lane).
      const int wq = warp & 3;
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        const int blk = (warp >> 2) * 2 + bb;
        uint32_t d[16];
        tc::tmem_ld16(tmem + ((uint32_t)(32 * wq) << 16) + 16u * blk, d);
        tc::tmem_ld_wait();
        const int mi = 128 * blk + 32 * wq + lane;
        const int j = mi >> 1, part = mi & 1;
        const int lo = j & ((1 << w) - 1), hi = j >> w;
        const int i0 = (hi << (w + 4)) | lo;
#pragma unroll
        for (int n = 0; n < 16; ++n) S.tile[2 * (i0 | (n << w)) + part] = __uint_as_float(d[n]);
      }
      tc::fence_before_sync();
      __syncthreads();
    }
    if (!ok) break;
    for (int q = tid; q < kTileElems / 2; q += kThreads)
      *reinterpret_cast<float4*>(v + global_index(P, base, 2 * q)) = reinterpret_cast<const float4*>(S.tile)[q];
    __syncthreads();
  }
  if (!ok && tid == 0) atomicExch(&g_wht_timeout, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

template <int T>
int launch_pass(float2* v, const WhtPass& P, int device, cudaStream_t s) {
  static bool configured[64] = {false};
  const int bytes = (int)sizeof(WhtSmem<T>) + 1024;
  if (device >= 0 && device < 64 && !configured[device]) {
    RGS_CUDA_TRY(cudaFuncSetAttribute(wht_tc_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    configured[device] = true;
  }
  const unsigned long long ntiles = 1ull << (P.m - 12);
  const unsigned grid = (unsigned)std::min<unsigned long long>(ntiles, (unsigned long long)sm_count(device) * 2);
  wht_tc_kernel<T><<<grid, kThreads, bytes, s>>>(v, P);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

// Rounds of a pass: the 4-bit tile-local windows holding transformed bits.
// target(i): tile-local bit i is transformed in this pass.
template <typename F>
void set_rounds(WhtPass& P, F target) {
  P.rounds = 0;
  for (int w = 0; w < 12; w += 4) {
    unsigned mask = 0;
    for (int i = 0; i < 4; ++i)
      if (target(w + i)) mask |= 1u << i;
    if (!mask) continue;
    P.w[P.rounds] = w;
    P.mask[P.rounds] = mask;
    ++P.rounds;
  }
}

}  // namespace

int wht_tensor_core_timeout(int* timed_out) {
  int h = 0, zero = 0;
  RGS_CUDA_TRY(cudaMemcpyFromSymbol(&h, g_wht_timeout, sizeof(int)));
  RGS_CUDA_TRY(cudaMemcpyToSymbol(g_wht_timeout, &zero, sizeof(int)));
  *timed_out = h;
  return RGS_OK;
}

int fwht_tensor_core(void* state, int nbits, int lo, int hi, int terms, cudaStream_t s) {
  if (!state) return fail(RGS_ERR_ARG, "state is NULL");
  if (nbits < 12 || nbits > 40) return fail(RGS_ERR_UNSUPPORTED, "the tensor-core WHT needs 12 <= nbits <= 40");
  if (lo < 0 || hi > nbits || lo > hi) return fail(RGS_ERR_ARG, "bad bit range");
  if (terms != 2 && terms != 3) return fail(RGS_ERR_ARG, "split terms must be 2 or 3");
  if (((uintptr_t)state & 15) != 0) return fail(RGS_ERR_ARG, "state must be 16-byte aligned");
  int device = 0;
  int rc = bind_device_of(state, &device);
  if (rc) return rc;
  float2* v = (float2*)state;
  auto run = [&](const WhtPass& P) { return terms == 2 ? launch_pass<2>(v, P, device, s) : launch_pass<3>(v, P, device, s); };
  // Bits 0..11: contiguous tiles.
  if (lo < 12) {
    WhtPass P{};
    P.m = nbits;
    P.b0 = 12, P.k = 0, P.c = 12;
    set_rounds(P, [&](int i) { return i >= lo && i < hi; });
    if (P.rounds && (rc = run(P))) return rc;
  }
  // Bits 12..nbits-1: strided tiles of up to 8 target bits over 16 or more contiguous elements.
  for (int b0 = 12; b0 < nbits; b0 += 8) {
    const int k = std::min(8, nbits - b0);
    if (b0 + k <= lo || b0 >= hi) continue;
    WhtPass P{};
    P.m = nbits;
    P.b0 = b0, P.k = k, P.c = 12 - k;
    set_rounds(P, [&](int i) { return i >= P.c && b0 + (i - P.c) >= lo && b0 + (i - P.c) < hi; });
    if (P.rounds && (rc = run(P))) return rc;
  }
  return RGS_OK;
}

}  // namespace rgs
