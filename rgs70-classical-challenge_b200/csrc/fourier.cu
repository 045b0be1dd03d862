// Conditional (Fourier-cut) sampler on one B200.
//
// Replaces the multi-kernel CuPy pipeline of whyihaveyou/rgs70-classical-challenge
// (W/ = work/rgs_attack/): initialisation (initv / initcov / initcov_specialized*,
// W/distributed_sampler.py:14-20, W/fourier_covariant_sampler.py:78-86,
// W/init_specialization.py:196-246), Walsh-Hadamard transform (lowfwht / localfwht /
// fusedfwht, distributed_sampler.py:21-31, fourier_fused_sampler.py:19-32), q_A phase and
// per-qubit products (lowprod / localprod / lowprodphase / fusedprod), the index map
// (permute, distributed_sampler.py:35-41) and tile masses + draw (blockmass / draw,
// distributed_sampler.py:50-54, 145-157; deferred_global_sampler.py:65-78).
//
// Pass structure.  The state is 2^m complex64 values in HBM.  A pass streams it once
// in tiles of 2^12 elements (three or four 256-thread blocks per SM): either a contiguous
// tile (the 12 low bits) or a strided tile (at least 3 contiguous low bits = 64-byte runs,
// times up to 9 "target" bits at position q).  Inside a tile each thread holds 16
// elements in registers along 4 tile axes and applies every 2x2 operation on those axes.
// fourier_sched_kernel (12-bit tiles) transforms the axes that sit in registers right
// after the load and before the store there, and the rest in at most three padded
// shared-memory rounds chosen per pass by the host (plan_sched); optionally
// (rgs_fourier_set_tma) its loading passes stage each next tile with a tensor-map (TMA)
// load while the current one is transformed.  fourier_pass_kernel (tiles of fewer bits,
// the generic chunk init, general 2x2 products) runs one round per four axes.  The whole
// transform is
//   pass 0          : init (computed, not loaded) + WHT on bits [0, 12)
//   strided passes  : WHT on the next groups of <= 9 bits (balanced)
//   middle pass     : WHT on the last group, q_A phase, products on that group
//   strided passes  : products on the earlier groups (reverse order)
//   last pass       : products on bits [0, 12) + per-tile masses (float64)
// = 2k+1 passes with k = ceil((m-12)/9): 8 + 16*2k bytes per element (the reference
// streams 2 + 2*ceil((m-10)/5) passes of 16 bytes, plus a mass pass).
//
// Lookup tables (init and phase) are evaluated per element only for the 8-bit chunks
// of z that vary inside the tile; the chunks that are constant over a tile are folded
// into per-tile constants once (parity is linear: XOR_c (x_c & z) = (XOR_c x_c) & z).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <atomic>
#include <cstring>
#include <type_traits>
#include <mutex>

#include "common.hpp"
#include "f32x2.cuh"
#include "fourier.cuh"
#include "tcgen05.cuh"
#include "tma_map.hpp"

namespace rgs {

// Set when a bounded wait of a TMA-staged pass gave up (read by tensor_core_status).
__device__ int g_fourier_timeout = 0;

typedef unsigned long long u64;

FourierPlan::~FourierPlan() {
  if (device < 0) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  for (void* p : {d_lut_z, d_lut_a, d_lut_cols, d_uA, d_uB, d_rot, d_dg, d_dh, d_rg, d_rh, d_tt_init, d_tt_phase,
                  d_tt_init_shard, d_tt_phase_shard, d_qsym_z, d_qsym_a})
    if (p) cudaFree(p);
  if (prev >= 0) cudaSetDevice(prev);
}

namespace {

// ------------------------------------------------------------------------------------- device
enum InitKind : int { INIT_LOAD = 0, INIT_COV_GENERIC = 1, INIT_COV_SPECIAL = 2, INIT_PRODUCT = 3 };

// Per-pass tables of a quadratic phase q (and, for the init, the covariant map b = N z)
// over the tile-local bits f of a pass configuration: with the tile's varying bits zero
// in `base`, b(base ^ f) = b(base) ^ mlo[f & 63] ^ mhi[f >> 6] and
// q(base ^ f) = q(base) ^ qtab[f] ^ parity(L & f), L_a = parity(qsym[global(a)] & base)
// (q is a polynomial of degree 2, so q(x ^ y) = q(x) ^ q(y) ^ x^T (Q + Q^T) y).
// Register-first schedule of a 12-bit tile (see fourier_sched_kernel): the tile axes
// applied in registers after the load (layout L0), in up to three shared-memory rounds
// (window [rw0, rw0 + 4)), and in registers before the store (layout L0 or L1).
struct PassSched {
  unsigned ld_w, ld_u;            // WHT / product axes at the load stage
  int nr;                         // shared-memory rounds
  int rw0[3];
  unsigned rw[3], ru[3];
  int fin_l1;                     // final layout L1 (else L0)
  unsigned fw, fu;
  int phase_at;                   // stage of the phase: 0 load, 1..nr rounds, nr + 1 final, -1 none
  int ld_w0;                      // load stage: -1 layout L0, else the window [ld_w0, ld_w0 + 4) (computed init)
};

struct PassParams {
  float2* v;
  int m, c, K, q;                 // tile = c low bits + K target bits at q
  unsigned wht_mask, u_mask;      // tile-local axes
  int phase;                      // q_A phase after the WHT rounds
  int init;                       // InitKind
  int chunks;
  const u64* lut_z;               // covariant map + q_B (INIT_COV_*), or q_B over b (INIT_PRODUCT)
  const u64* lut_a;               // q_A
  const double2* wgen;            // [chunks][256] complex128 chunk weights
  const double2* wspec;           // [(m+1)^2] popcount weights
  u64 outmask;
  const double2* u;               // [m][2][2] complex128 per global bit
  const float2* rot;              // [m] (k, form): scaled real rotations (Euler-factorised path)
  const float2* dg;               // chunk tables of the diagonal applied with the q_A phase, or null
  const float2* dh;               // chunk tables of the diagonal applied after the products, or null
  const float2* rg;               // [m] per-bit ratios d_j(1) / d_j(0) of the dg diagonal
  const float2* rh;               // [m] per-bit ratios of the dh diagonal
  const float2* wspecf;           // [(m+1)^2] popcount weights as complex64
  const TileTables* tt_init;      // init tables of this pass configuration (lut_z), or null
  const unsigned long long* qsym_z;  // [m] rows of Q + Q^T of the init phase
  const TileTables* tt_phase;     // q_A tables of this pass configuration, or null
  const unsigned long long* qsym_a;  // [m] rows of Q_A + Q_A^T
  int variant;                    // launch variant (see fourier_pass_kernel)
  double* masses;                 // per tile or null
  int store;
  // Sharded state (top bit of the index split over devices): v holds the global indices
  // g with g & ~amask fixed, at v[g & amask]; a launch runs tiles [tile0, tile0 + grid);
  // store_top >= 0 stores only the elements whose top bit (m - 1) equals it.
  u64 amask;
  u64 tile0;
  u64 ntiles;                     // tiles of this launch (0: every tile of the index space)
  int store_top;
  int sched;                      // 1: register-first schedule below (fourier_sched_kernel)
  int top_axis;                   // tile axis at global bit m - 1, or -1 (sharded stores)
  int tma_mid_dim, tma_high_dim;  // tensor-map dimensions of the mid and high index bits, or -1
  PassSched s;
};

// Shared memory of a pass: the padded work buffer (kWorkElems float2), and for the
// TMA-staged kernel a dense staging buffer behind it (1024-byte aligned).
constexpr int kWorkElems = (1 << kTileBits) + (1 << (kTileBits - 4));
constexpr size_t kTmaSmemBytes = kWorkElems * sizeof(float2) + 1024 + (sizeof(float2) << kTileBits);

// Padded shared-memory layout: one spare slot per 16 elements, so the 16 threads of a
// half-warp hit distinct 8-byte bank pairs in every access pattern used here, and a
// round's 16 element offsets are linear in the register index (constant strides).
__device__ __forceinline__ int pad(int f) { return f + (f >> 4); }

__device__ __forceinline__ u64 tile_global(const PassParams& P, u64 tile, int f) {
  const int mid = P.q - P.c;  // bits between the low part and the target bits
  const u64 base = ((tile & ((1ull << mid) - 1ull)) << P.c) | ((tile >> mid) << (P.q + P.K));
  return base | (u64)(f & ((1 << P.c) - 1)) | ((u64)(f >> P.c) << P.q);
}

__device__ __forceinline__ int local_to_global_bit(const PassParams& P, int a) {
  return a < P.c ? a : P.q + (a - P.c);
}

__device__ __forceinline__ u64 lut_parity_mask(const u64* lut, int chunks, u64 z) {
  const u64 marked = z | (1ull << 63);
  u64 pm = 0;
  for (int cc = 0; cc < chunks; ++cc) pm ^= __ldg(lut + ((((u64)cc << 8) + ((z >> (8 * cc)) & 255ull)) << 1) + 1) & marked;
  return pm;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Chunk lookups that are constant over a tile, folded once per tile: b and the
// phase mask of every chunk whose 8 bits of z do not vary in the tile.
struct TileLut {
  u64 b_const, pm_const;
  unsigned var;  // bit c: chunk c varies in the tile
  int chunks;
};

__device__ __forceinline__ void tile_lut(const u64* lut, int chunks, u64 base, u64 varying, TileLut& t) {
  t.b_const = 0;
  t.pm_const = 0;
  t.var = 0;
  t.chunks = chunks;
  for (int cc = 0; cc < chunks; ++cc) {
    if ((varying >> (8 * cc)) & 255ull) {
      t.var |= 1u << cc;
    } else {
      const u64* e = lut + ((((u64)cc << 8) + ((base >> (8 * cc)) & 255ull)) << 1);
      t.b_const ^= __ldg(e);
      t.pm_const ^= __ldg(e + 1);
    }
  }
}

// (b, phase-parity mask) of z from the varying chunks plus the tile constants.
__device__ __forceinline__ void tile_lut_eval(const u64* lut, const TileLut& t, u64 z, u64& b, u64& pm) {
  b = t.b_const;
  pm = t.pm_const;
  for (int cc = 0; cc < t.chunks; ++cc) {
    if (!((t.var >> cc) & 1u)) continue;
    const u64* e = lut + ((((u64)cc << 8) + ((z >> (8 * cc)) & 255ull)) << 1);
    b ^= __ldg(e);
    pm ^= __ldg(e + 1);
  }
  pm &= z | (1ull << 63);
}

// Phase-parity mask of z alone (the q_A phase needs no map part).
__device__ __forceinline__ u64 tile_lut_pm(const u64* lut, const TileLut& t, u64 z) {
  u64 pm = t.pm_const;
  for (int cc = 0; cc < t.chunks; ++cc) {
    if (!((t.var >> cc) & 1u)) continue;
    pm ^= __ldg(lut + ((((u64)cc << 8) + ((z >> (8 * cc)) & 255ull)) << 1) + 1);
  }
  return pm & (z | (1ull << 63));
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// A diagonal D(z) = prod_j d_j(z_j) over the state index, applied inside a tile: with the
// tile's varying bits zero in `base`, D(base ^ f) = D(base) prod_{a: f_a = 1} r_a for the
// tile-local bits a (r_a = d(1) / d(0) of that bit).  Three 16-entry window tables
// (tile-local bits 0-3, 4-7, 8-11; D(base) folded into the first) make the factor of
// element f two complex products.  D(base) comes from the 8-bit chunk tables T.
__device__ __forceinline__ void window_tables(float2 (*wt)[16], const PassParams& P, const float2* T,
                                              const float2* ratio, u64 base, int TB) {
  for (int t = threadIdx.x; t < 48; t += blockDim.x) {
    const int w = t >> 4, i = t & 15;
    float2 v = make_float2(1.f, 0.f);
    if (w == 0)
      for (int cc = 0; cc < P.chunks; ++cc) v = cmulf(v, __ldg(T + ((u64)cc << 8) + ((base >> (8 * cc)) & 255ull)));
    for (int a = 0; a < 4; ++a) {
      const int la = 4 * w + a;
      if (la < TB && ((i >> a) & 1)) v = cmulf(v, __ldg(ratio + local_to_global_bit(P, la)));
    }
    wt[w][i] = v;
  }
}

__device__ __forceinline__ float2 window_factor(const float2 (*wt)[16], int f) {
  return cmulf(cmulf(wt[0][f & 15], wt[1][(f >> 4) & 15]), wt[2][(f >> 8) & 15]);
}

// The elements of thread t are f = 2 t + 2 k nt + e (k < 8, e < 2).  With nt >= 128 their
// low 8 bits are those of 2 t + e for every k, so the first two windows' factor is one
// value per e for the whole loop (lo[e]) and each element needs the third window only.
struct WindowSplit {
  bool on;
  float2 lo[2];
};
__device__ __forceinline__ WindowSplit window_split(const float2 (*wt)[16], int nt) {
  WindowSplit w;
  w.on = nt >= 128;
  const int f = (2 * threadIdx.x) & 255;
#pragma unroll
  for (int e = 0; e < 2; ++e) w.lo[e] = cmulf(wt[0][(f + e) & 15], wt[1][((f + e) >> 4) & 15]);
  return w;
}
__device__ __forceinline__ float2 window_factor(const float2 (*wt)[16], const WindowSplit& w, int f, int e) {
  return w.on ? cmulf(w.lo[e], wt[2][(f >> 8) & 15]) : window_factor(wt, f + e);
}

// Loads a pass's tables into shared memory and evaluates the tile constants: b(base)
// (when `map`), q(base) and the 12-bit linear mask L of the cross term.
__device__ __forceinline__ void tile_tables_setup(const PassParams& P, const TileTables* tt, const u64* lut,
                                                  const u64* qsym, u64 base, int TB, bool map, TileTables& st,
                                                  u64& b0, int& q0, unsigned& lmask) {
  const int t = threadIdx.x;
  for (int i = t; i < 128; i += blockDim.x) {
    st.qtab[i] = __ldg(&tt->qtab[i]);
    if (map && i < 64) {
      st.mlo[i] = __ldg(&tt->mlo[i]);
      st.mhi[i] = __ldg(&tt->mhi[i]);
    }
  }
  if (t < 32) {
    // Blocks of small tiles have fewer than 32 threads: vote over the lanes that exist.
    const unsigned lanes = blockDim.x >= 32 ? 0xffffffffu : ((1u << blockDim.x) - 1u);
    unsigned bitv = 0;
    if (t < TB) bitv = __popcll(__ldg(qsym + local_to_global_bit(P, t)) & base) & 1;
    const unsigned lm = __ballot_sync(lanes, bitv);
    if (t == 0) {
      u64 b = 0, pm = 0;
      for (int cc = 0; cc < P.chunks; ++cc) {
        const u64* e = lut + ((((u64)cc << 8) + ((base >> (8 * cc)) & 255ull)) << 1);
        if (map) b ^= __ldg(e);
        pm ^= __ldg(e + 1);
      }
      b0 = b;
      q0 = __popcll(pm & (base | (1ull << 63))) & 1;
      lmask = lm;
    }
  }
}

__device__ __forceinline__ int tile_q(const TileTables& st, int q0, unsigned lmask, int f) {
  return q0 ^ (int)((st.qtab[f >> 5] >> (f & 31)) & 1u) ^ (__popc(lmask & (unsigned)f) & 1);
}

// Initial value at index z (fourier_covariant_sampler.py:78-86, init_specialization.py:196-214,
// distributed_sampler.py:14-20).  For INIT_PRODUCT the table has no map part (b = z).
__device__ float2 init_value(const PassParams& P, const TileLut& t, u64 z) {
  u64 b, pm;
  tile_lut_eval(P.lut_z, t, z, b, pm);
  if (P.init == INIT_PRODUCT) b = z;
  double2 w;
  if (P.init == INIT_COV_SPECIAL) {
    const float2 wf = __ldg(P.wspecf + __popcll(b) * (P.m + 1) + __popcll(b & P.outmask));
    const float s = (__popcll(pm) & 1) ? -1.f : 1.f;
    return make_float2(s * wf.x, s * wf.y);
  } else {
    w = __ldg(P.wgen + ((b & 255ull)));
    for (int cc = 1; cc < P.chunks; ++cc) w = cmul(w, __ldg(P.wgen + ((u64)cc << 8) + ((b >> (8 * cc)) & 255ull)));
  }
  const float s = (__popcll(pm) & 1) ? -1.f : 1.f;
  return make_float2(s * (float)w.x, s * (float)w.y);
}

__device__ __forceinline__ void apply_u(float2& x, float2& y, const float2 (&u)[4]) {
  const float2 nx = make_float2(u[0].x * x.x - u[0].y * x.y + u[1].x * y.x - u[1].y * y.y,
                                u[0].x * x.y + u[0].y * x.x + u[1].x * y.y + u[1].y * y.x);
  const float2 ny = make_float2(u[2].x * x.x - u[2].y * x.y + u[3].x * y.x - u[3].y * y.y,
                                u[2].x * x.y + u[2].y * x.x + u[3].x * y.y + u[3].y * y.x);
  x = nx;
  y = ny;
}

// Scaled real rotation on a pair of complex values, one packed FMA per output (the
// rotation's scale and sign are folded into the diagonal applied after the products):
//   form 0: [[1, -k], [k, 1]]   (k = s / c, |c| >= |s|)
//   form 1: [[-k, 1], [1, k]]   (k = c / s, |s| > |c|)
__device__ __forceinline__ void apply_rot0(float2& x, float2& y, float2 k, float2 nk) {
  const float2 nx = f2fma(nk, y, x), ny = f2fma(k, x, y);
  x = nx;
  y = ny;
}
__device__ __forceinline__ void apply_rot1(float2& x, float2& y, float2 k, float2 nk) {
  const float2 nx = f2fma(nk, x, y), ny = f2fma(k, y, x);
  x = nx;
  y = ny;
}

// One four-axis round: registers hold the 16 elements whose tile-local bits
// [w0, w0+4) vary (w0 a multiple of 4); axes in `mask` (tile-local) get the WHT or
// their unitary.  With the padded layout element i sits at pad(f0) + i * stride.
__device__ void tile_round(float2* sm, const PassParams& P, int w0, unsigned mask, bool wht) {
  const int t = threadIdx.x;
  const int f0 = ((t >> w0) << (w0 + 4)) | (t & ((1 << w0) - 1));
  const bool linear = (w0 & 3) == 0;  // windows clipped at a tile edge use general addressing
  float2* base = sm + pad(f0);
  const int stride = w0 >= 4 ? (1 << w0) + (1 << (w0 - 4)) : 1;
  float2 r[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = linear ? base[i * stride] : sm[pad(f0 | (i << w0))];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    if (!((mask >> (w0 + a)) & 1u)) continue;
    if (wht) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        if (i & (1 << a)) continue;
        const float2 x = r[i], y = r[i | (1 << a)];
        r[i] = f2add(x, y);
        r[i | (1 << a)] = f2sub(x, y);
      }
    } else if (P.rot) {
      const float2 kf = __ldg(P.rot + local_to_global_bit(P, w0 + a));
      const float2 k = make_float2(kf.x, kf.x), nk = make_float2(-kf.x, -kf.x);
      if (kf.y == 0.f) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (!(i & (1 << a))) apply_rot0(r[i], r[i | (1 << a)], k, nk);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (!(i & (1 << a))) apply_rot1(r[i], r[i | (1 << a)], k, nk);
      }
    } else {
      const double2* u4 = P.u + 4 * local_to_global_bit(P, w0 + a);
      float2 uu[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double2 d = __ldg(u4 + e);
        uu[e] = make_float2((float)d.x, (float)d.y);
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        if (i & (1 << a)) continue;
        apply_u(r[i], r[i | (1 << a)], uu);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    if (linear)
      base[i * stride] = r[i];
    else
      sm[pad(f0 | (i << w0))] = r[i];
  }
}

// Rounds over the windows [0,4), [4,8), [8,12) that hold an axis of `mask`; in a tile
// of TB < 12 bits the last window is clipped to [TB-4, TB) (its lower axes already done).
__device__ void tile_rounds(float2* sm, const PassParams& P, int TB, unsigned mask, bool wht) {
  for (int g0 = 0; g0 < TB; g0 += 4) {
    const int w0 = g0 + 4 <= TB ? g0 : TB - 4;
    const unsigned sel = mask & (15u << w0) & ~((1u << g0) - 1u);
    if (!sel) continue;
    __syncthreads();
    tile_round(sm, P, w0, sel, wht);
  }
  __syncthreads();
}

// MINB resident blocks per SM: 3 (80 registers, no spills) or 4 (64 registers, a few
// spilled); the plan's tuned variant picks one (fourier_tune).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) fourier_pass_kernel(const __grid_constant__ PassParams P) {
  extern __shared__ float2 sm[];
  __shared__ float2 wt[3][16];  // window tables of a diagonal (see window_tables)
  __shared__ TileTables s_tt;   // pass tables of the init map / a phase (see TileTables)
  __shared__ u64 s_b0;
  __shared__ int s_q0;
  __shared__ unsigned s_lm;
  const int TB = P.c + P.K;
  const int nt = 1 << (TB - 4);
  const u64 tile = blockIdx.x + P.tile0;
  const u64 base = tile_global(P, tile, 0);
  const u64 varying = ((1ull << P.c) - 1ull) | (((1ull << P.K) - 1ull) << P.q);
  // Load (or compute) the tile: each thread owns 8 element pairs (16-byte accesses,
  // pairs are adjacent in memory because tile bit 0 is a contiguous bit).
  if (P.init == INIT_COV_SPECIAL && P.tt_init) {
    // Covariant init from the pass tables: per element two shared-memory map lookups,
    // two popcounts, one phase bit and the popcount weight.
    tile_tables_setup(P, P.tt_init, P.lut_z, P.qsym_z, base, TB, true, s_tt, s_b0, s_q0, s_lm);
    __syncthreads();
    const u64 b0 = s_b0;
    const int q0 = s_q0;
    const unsigned lm = s_lm;
    // Elements f = 2 t + 2 k nt + e: with nt >= 32 the low 6 bits of f are those of 2 t + e
    // for every k, so b0 ^ mlo[f & 63] is one value per e for the whole loop.
    const bool lo_const = nt >= 32;
    const int t2 = 2 * (int)threadIdx.x;
    const u64 blo[2] = {b0 ^ s_tt.mlo[t2 & 63], b0 ^ s_tt.mlo[(t2 + 1) & 63]};
#pragma unroll 2
    for (int k = 0; k < 8; ++k) {
      const int f0 = t2 + 2 * k * nt;
      const u64 bhi = s_tt.mhi[(f0 >> 6) & 63];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int f = f0 + e;
        const u64 b = (lo_const ? blo[e] : b0 ^ s_tt.mlo[f & 63]) ^ bhi;
        const float2 w = __ldg(P.wspecf + __popcll(b) * (P.m + 1) + __popcll(b & P.outmask));
        sm[pad(f)] = tile_q(s_tt, q0, lm, f) ? make_float2(-w.x, -w.y) : w;
      }
    }
  } else if (P.init) {
    TileLut t;
    tile_lut(P.lut_z, P.chunks, base, varying, t);
#pragma unroll 2
    for (int k = 0; k < 8; ++k) {
      const int f = 2 * (threadIdx.x + k * nt);
      const u64 g = tile_global(P, tile, f);
      sm[pad(f)] = init_value(P, t, g);
      sm[pad(f + 1)] = init_value(P, t, g + 1);
    }
  } else {
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
      float4 x[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int f = 2 * (threadIdx.x + (h + k) * nt);
        x[k] = *reinterpret_cast<const float4*>(P.v + (tile_global(P, tile, f) & P.amask));
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int f = 2 * (threadIdx.x + (h + k) * nt);
        sm[pad(f)] = make_float2(x[k].x, x[k].y);
        sm[pad(f + 1)] = make_float2(x[k].z, x[k].w);
      }
    }
  }
  if (P.wht_mask) tile_rounds(sm, P, TB, P.wht_mask, true);
  if (P.phase && P.tt_phase) {
    // q_A phase from the pass tables, times the diagonal dg when given.
    __syncthreads();  // readers of s_tt (init) are done
    tile_tables_setup(P, P.tt_phase, P.lut_a, P.qsym_a, base, TB, false, s_tt, s_b0, s_q0, s_lm);
    if (P.dg) window_tables(wt, P, P.dg, P.rg, base, TB);
    __syncthreads();
    const int q0 = s_q0;
    const unsigned lm = s_lm;
    const WindowSplit ws = window_split(wt, nt);
    for (int k = 0; k < 8; ++k) {
      const int f0 = 2 * (threadIdx.x + k * nt);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int f = f0 + e;
        float2 x = sm[pad(f)];
        if (P.dg) x = cmulf(x, window_factor(wt, ws, f0, e));
        if (tile_q(s_tt, q0, lm, f)) x = make_float2(-x.x, -x.y);
        sm[pad(f)] = x;
      }
    }
  } else if (P.phase) {
    // q_A phase (-1)^{q_A(z)}, times the diagonal dg when given.
    TileLut t;
    tile_lut(P.lut_a, P.chunks, base, varying, t);
    if (P.dg) window_tables(wt, P, P.dg, P.rg, base, TB);
    __syncthreads();
    for (int k = 0; k < 8; ++k) {
      const int f = 2 * (threadIdx.x + k * nt);
      const u64 g = tile_global(P, tile, f);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        float2 x = sm[pad(f + e)];
        if (P.dg) x = cmulf(x, window_factor(wt, f + e));
        if (__popcll(tile_lut_pm(P.lut_a, t, g + e)) & 1) x = make_float2(-x.x, -x.y);
        sm[pad(f + e)] = x;
      }
    }
  }
  if (P.u_mask) tile_rounds(sm, P, TB, P.u_mask, false);
  if (P.dh) {
    __syncthreads();  // the phase loop's readers of wt are done
    window_tables(wt, P, P.dh, P.rh, base, TB);
  }
  __syncthreads();
  const WindowSplit ws = window_split(wt, nt);
  double mass = 0.0;  // per element pair: a float sum of four squares, then float64
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int f = 2 * (threadIdx.x + k * nt);
    const u64 g = tile_global(P, tile, f);
    float2 a = sm[pad(f)], b = sm[pad(f + 1)];
    if (P.dh) {
      a = cmulf(a, window_factor(wt, ws, f, 0));
      b = cmulf(b, window_factor(wt, ws, f, 1));
    }
    if (P.store && (P.store_top < 0 || (int)((g >> (P.m - 1)) & 1ull) == P.store_top))
      *reinterpret_cast<float4*>(P.v + (g & P.amask)) = make_float4(a.x, a.y, b.x, b.y);
    if (P.masses) {
      const float2 q = f2fma(b, b, make_float2(a.x * a.x, a.y * a.y));
      mass += (double)(q.x + q.y);
    }
  }
  if (P.masses) {
    __shared__ double red[32];
    double m2 = mass;
    for (int off = 16; off; off >>= 1) m2 += __shfl_xor_sync(0xffffffffu, m2, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m2;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (nt + 31) / 32; ++w) s += red[w];
      P.masses[tile - P.tile0] = s;
    }
  }
}


// ---------------------------------------------------------------------------
// Register-first passes (12-bit tiles, 256 threads).  Thread t holds 16 elements of the
// tile in registers (index i = 2 k + e) in one of three arrangements:
//   L0    : f = e + 2 t + 512 k                        axes 0, 9, 10, 11
//   L1    : f = e + 2 (t & 31) + 64 k + 512 (t >> 5)   axes 0, 6, 7, 8
//   round : f = f0(t) | (i << w0)                      axes w0 .. w0 + 3
// L0 and L1 keep the lanes of a warp on axes 1..5, so global loads and stores stay
// 16-byte accesses filling whole 32-byte sectors; every arrangement gives the 16 lanes
// of a half-warp distinct 8-byte bank pairs in the padded layout.  The host schedule
// (PassSched) applies every axis once -- at the load (L0), in a shared-memory round, or
// before the store (L0 or L1) -- with all WHT axes before the phase and all products
// after it.  Against one shared-memory round per four axes this saves up to two
// exchanges per element and pass (four in the middle pass).

__device__ __forceinline__ void reg_wht(float2 (&r)[16], const int (&ax)[4], unsigned wm) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    if (!((wm >> ax[a]) & 1u)) continue;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      if (i & (1 << a)) continue;
      const float2 x = r[i], y = r[i | (1 << a)];
      r[i] = f2add(x, y);
      r[i | (1 << a)] = f2sub(x, y);
    }
  }
}

// srot[a] = the scaled rotation of tile axis a (shared); the register-first kernel runs
// products only as scaled rotations (general 2x2 products take fourier_pass_kernel).
__device__ __forceinline__ void reg_prod(float2 (&r)[16], const PassParams& P, const float2* srot, const int (&ax)[4],
                                         unsigned um) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    if (!((um >> ax[a]) & 1u)) continue;
    const float2 kf = srot[ax[a]];
    const float2 k = make_float2(kf.x, kf.x), nk = make_float2(-kf.x, -kf.x);
    if (kf.y == 0.f) {
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (!(i & (1 << a))) apply_rot0(r[i], r[i | (1 << a)], k, nk);
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (!(i & (1 << a))) apply_rot1(r[i], r[i | (1 << a)], k, nk);
    }
  }
}

// Register axes of the schedule's phase stage.
__device__ __forceinline__ void phase_axes(const PassSched& S, int (&ax)[4]) {
  const bool round = (S.phase_at >= 1 && S.phase_at <= S.nr) || (S.phase_at == 0 && S.ld_w0 >= 0);
  const bool l1 = S.phase_at == S.nr + 1 && S.fin_l1;
  const int w0 = S.phase_at == 0 ? S.ld_w0 : (round ? S.rw0[S.phase_at - 1] : 0);
#pragma unroll
  for (int a = 0; a < 4; ++a) ax[a] = round ? w0 + a : (a == 0 ? 0 : (l1 ? 5 : 8) + a);
}

// Tile-local part of a quadratic phase at tile index f (pass table bit, no tile constants).
__device__ __forceinline__ int qt_bit(const TileTables& st, int f) { return (st.qtab[f >> 5] >> (f & 31)) & 1u; }

// Signs (-1)^{q(f)} of a stage's 16 registers as a 16-bit mask, f = fb | X(i): the
// thread's q(fb), the block's window part qw (bit i = qt(X) ^ parity(L & X), or 0 when the
// caller folds it elsewhere) and the cross terms of q between fb and each axis.
__device__ __forceinline__ unsigned sign_mask(const TileTables& st, int q0, unsigned lm, int fb,
                                              const int (&ax)[4], unsigned qw) {
  const unsigned pat[4] = {0xAAAAu, 0xCCCCu, 0xF0F0u, 0xFF00u};  // bit i set where i_a = 1
  unsigned L = (tile_q(st, q0, lm, fb) ? 0xFFFFu : 0u) ^ qw;
  const int qb = qt_bit(st, fb);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int e = 1 << ax[a];
    if (qt_bit(st, fb ^ e) ^ qb ^ qt_bit(st, e)) L ^= pat[a];
  }
  return L;
}

// q_A phase times the diagonal dg on the 16 registers of a stage, f = fb | X(i) with
// X(i) = sum of i_a 2^{ax[a]} (fb: the thread's element 0, zero on the register axes).
// dg is a product over bits and q is quadratic, so the factor of register i is
//   dg(fb) * rt[i] * (-1)^{bit i of sign_mask(fb)}
// with rt[i] = (-1)^{qt(X) ^ parity(L & X)} times the product of dg's per-bit ratios over
// X (per block, shared): one shared broadcast load and two complex products per element
// instead of a table walk and three.
__device__ __forceinline__ void reg_phase(float2 (&r)[16], const PassParams& P, const float2 (*wt)[16],
                                          const TileTables& st, int q0, unsigned lm, const float2* rt, int fb) {
  int ax[4];
  phase_axes(P.s, ax);
  const float2 F0 = P.dg ? window_factor(wt, fb) : make_float2(1.f, 0.f);
  const unsigned L = sign_mask(st, q0, lm, fb, ax, 0u);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float2 fac = cmulf(F0, rt[i]);
    if ((L >> i) & 1u) fac = make_float2(-fac.x, -fac.y);
    r[i] = cmulf(r[i], fac);
  }
}

template <int W0>
__device__ __forceinline__ int round_f0(int t) {
  return (t & ((1 << W0) - 1)) | ((t >> W0) << (W0 + 4));
}

template <int W0, bool STORE>
__device__ __forceinline__ void round_io(float2* sm, float2 (&r)[16]) {
  float2* b = sm + pad(round_f0<W0>(threadIdx.x));
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    if (STORE)
      b[pad(i << W0)] = r[i];
    else
      r[i] = b[pad(i << W0)];
  }
}

template <bool STORE>
__device__ __forceinline__ void round_io_at(float2* sm, float2 (&r)[16], int w0) {
  switch (w0) {
    case 0: round_io<0, STORE>(sm, r); break;
    case 1: round_io<1, STORE>(sm, r); break;
    case 2: round_io<2, STORE>(sm, r); break;
    case 3: round_io<3, STORE>(sm, r); break;
    case 4: round_io<4, STORE>(sm, r); break;
    case 5: round_io<5, STORE>(sm, r); break;
    case 6: round_io<6, STORE>(sm, r); break;
    case 7: round_io<7, STORE>(sm, r); break;
    default: round_io<8, STORE>(sm, r); break;
  }
}

__device__ __forceinline__ int round_f0(int t, int w0) {
  return (t & ((1 << w0) - 1)) | ((t >> w0) << (w0 + 4));
}

// Tile index of register i in layout L0 / L1 (t = thread).
__device__ __forceinline__ int lay_f(int l1, int t, int i) {
  const int e = i & 1, k = i >> 1;
  return l1 ? e + 2 * (t & 31) + 64 * k + 512 * (t >> 5) : e + 2 * t + 512 * k;
}

// Element offset of tile index f from the tile's first element (tile_global is a sum
// over the bits of f), with the shard mask applied.
__device__ __forceinline__ u64 tile_off(const PassParams& P, int f) {
  return ((u64)(f & ((1 << P.c) - 1)) | ((u64)(f >> P.c) << P.q)) & P.amask;
}

// Offsets of a layout: element (k, e) of the thread sits at o0 + at(k) + e.  With m <= 32
// (O = 32 bits) every offset fits and an access is one wide multiply-add from the tile
// pointer; larger states use 64-bit offsets.
template <typename O>
struct LayOff {
  O o0, d[3];
  __device__ __forceinline__ O at(int k) const {
    return o0 + ((k & 1) ? d[0] : (O)0) + ((k & 2) ? d[1] : (O)0) + ((k & 4) ? d[2] : (O)0);
  }
};
template <typename O>
__device__ __forceinline__ LayOff<O> lay_off(const PassParams& P, int l1) {
  LayOff<O> A;
  A.o0 = (O)tile_off(P, lay_f(l1, threadIdx.x, 0));
  const int kb = l1 ? 6 : 9;
#pragma unroll
  for (int j = 0; j < 3; ++j) A.d[j] = (O)tile_off(P, 1 << (kb + j));
  return A;
}

// Issues the tensor-map load of tile `tile` into the staging buffer (one thread).  The
// map's dimensions (innermost first) follow the index bits: the tile's low bits, the mid
// bits [c, q), the target bits, the high bits [q + K, ...) -- boxes are full on the tile's
// dimensions and 1 on the others, so the box lands in tile index order.
__device__ __forceinline__ void tma_tile(const PassParams& P, const CUtensorMap& map, u64 tile, float2* stage,
                                         uint64_t* bar) {
  const u64 bm = tile_global(P, tile, 0) & P.amask;
  int c[5] = {0, 0, 0, 0, 0};
  if (P.tma_mid_dim >= 0) c[P.tma_mid_dim] = (int)((bm >> P.c) & ((1ull << (P.q - P.c)) - 1ull));
  if (P.tma_high_dim >= 0) c[P.tma_high_dim] = (int)(bm >> (P.q + P.K));
  tc::mbar_expect_tx(bar, (uint32_t)(sizeof(float2) << kTileBits));
  tc::tma_load_5d(stage, &map, c[0], c[1], c[2], c[3], c[4], bar);
}

// TMA = true: a persistent loop over the launch's tiles (tile blockIdx.x + i gridDim.x) in
// which one thread prefetches the next tile with a tensor-map load into a dense staging
// buffer while the block transforms the current one; the load stage then reads the tile
// from shared memory (16-byte accesses, layout L0) instead of from HBM.
// Per-tile constants of the register-first kernel, computed by one full warp in one round
// trip to memory (the block waits for them at its first barrier): one lane per 8-bit
// chunk of the tile base loads that chunk's table entry and the entries are combined by
// shuffles.  tile_consts: b(base) and q(base) of a pass table (XOR over the chunks) and
// the cross-term mask L of the tile axes; diag_base: the diagonal's factor D(base)
// (product over the chunks, lane 0's value broadcast so every lane holds the same).
__device__ __forceinline__ void tile_consts(const PassParams& P, const u64* lut, const u64* qsym, u64 base, bool map,
                                            u64& b0, int& q0, unsigned& lm) {
  const int lane = threadIdx.x & 31;
  u64 b = 0, pm = 0;
  if (lane < P.chunks) {
    const u64* e = lut + ((((u64)lane << 8) + ((base >> (8 * lane)) & 255ull)) << 1);
    if (map) b = __ldg(e);
    pm = __ldg(e + 1);
  }
#pragma unroll
  for (int off = 4; off; off >>= 1) {
    b ^= __shfl_xor_sync(0xffffffffu, b, off);
    pm ^= __shfl_xor_sync(0xffffffffu, pm, off);
  }
  const unsigned bitv = lane < kTileBits ? (__popcll(__ldg(qsym + local_to_global_bit(P, lane)) & base) & 1) : 0u;
  lm = __ballot_sync(0xffffffffu, bitv);
  b0 = b;
  q0 = __popcll(pm & (base | (1ull << 63))) & 1;
}

__device__ __forceinline__ float2 diag_base(const PassParams& P, const float2* T, u64 base) {
  const int lane = threadIdx.x & 31;
  float2 d = make_float2(1.f, 0.f);
  if (lane < P.chunks) d = __ldg(T + ((u64)lane << 8) + ((base >> (8 * lane)) & 255ull));
#pragma unroll
  for (int off = 4; off; off >>= 1)
    d = cmulf(d, make_float2(__shfl_xor_sync(0xffffffffu, d.x, off), __shfl_xor_sync(0xffffffffu, d.y, off)));
  return make_float2(__shfl_sync(0xffffffffu, d.x, 0), __shfl_sync(0xffffffffu, d.y, 0));
}

// Window tables (see window_tables) by two full warps: entry e = thread - 32 < 48.
__device__ __forceinline__ void window_tables_warps(float2 (*wt)[16], const PassParams& P, const float2* T,
                                                    const float2* ratio, u64 base) {
  const float2 d = diag_base(P, T, base);
  const int e = (int)threadIdx.x - 32;
  if (e >= 48) return;
  const int w = e >> 4, i = e & 15;
  float2 v = w == 0 ? d : make_float2(1.f, 0.f);
#pragma unroll
  for (int a = 0; a < 4; ++a)
    if ((i >> a) & 1) v = cmulf(v, __ldg(ratio + local_to_global_bit(P, 4 * w + a)));
  wt[w][i] = v;
}

// INIT = true: the init pass (table init computed in registers, nothing loaded), a
// separate instantiation so the loading passes carry none of its code or registers.
template <int MINB, bool W64, bool TMA, bool INIT>
__global__ void __launch_bounds__(256, MINB)
    fourier_sched_kernel(const __grid_constant__ PassParams P, const __grid_constant__ CUtensorMap tmap) {
  using O = typename std::conditional<W64, u64, unsigned>::type;
  extern __shared__ float2 sm[];
  // TMA staging buffer (dense tile) after the padded work buffer, 1024-byte aligned.
  const uint32_t sa = tc::smem_u32(sm + kWorkElems);
  float2* stage = sm + kWorkElems + ((((sa + 1023u) & ~1023u) - sa) / sizeof(float2));
  __shared__ __align__(8) uint64_t s_full;
  __shared__ float2 wt[3][16];  // window tables of the pass's diagonal (dg or dh)
  __shared__ TileTables s_tt;   // init or q_A pass tables
  __shared__ u64 s_b0;
  __shared__ int s_q0;
  __shared__ unsigned s_lm, s_qw;
  __shared__ float2 s_rt[16];   // phase stage: per-block factors (see reg_phase)
  __shared__ float2 s_rot[kTileBits];  // scaled rotation (k, form) per tile axis
  const PassSched& S = P.s;
  const int t = threadIdx.x;
  const u64 ntl = P.ntiles ? P.ntiles : (1ull << (P.m - kTileBits));
  constexpr bool init_tab = INIT;
  uint32_t phase = 0;
  if (TMA) {
    if (t == 0) {
      tc::mbar_init(&s_full, 1);
      tc::fence_barrier_init();
    }
    __syncthreads();
    if (t == 0 && blockIdx.x < ntl) tma_tile(P, tmap, blockIdx.x + P.tile0, stage, &s_full);
  }
  for (u64 it = blockIdx.x; it < ntl; it += TMA ? gridDim.x : ntl) {
  const u64 tile = it + P.tile0;
  const u64 base = tile_global(P, tile, 0);
  if (TMA) __syncthreads();  // the previous tile's readers of the shared tables and buffers are done
  if (init_tab || P.phase) {
    const TileTables* tt = init_tab ? P.tt_init : P.tt_phase;
    for (int i = t; i < 128; i += 256) {
      s_tt.qtab[i] = __ldg(&tt->qtab[i]);
      if (init_tab && i < 64) {
        s_tt.mlo[i] = __ldg(&tt->mlo[i]);
        s_tt.mhi[i] = __ldg(&tt->mhi[i]);
      }
    }
    if (t < 32) {
      u64 b0;
      int q0;
      unsigned lm;
      if (init_tab)
        tile_consts(P, P.lut_z, P.qsym_z, base, true, b0, q0, lm);
      else
        tile_consts(P, P.lut_a, P.qsym_a, base, false, b0, q0, lm);
      if (t == 0) {
        s_b0 = b0;
        s_q0 = q0;
        s_lm = lm;
      }
    }
  }
  if (t >= 32 && t < 96) {
    if (P.dg)
      window_tables_warps(wt, P, P.dg, P.rg, base);
    else if (P.dh)
      window_tables_warps(wt, P, P.dh, P.rh, base);
  }
  if (P.rot && t >= 96 && t < 96 + kTileBits) s_rot[t - 96] = __ldg(P.rot + local_to_global_bit(P, t - 96));
  __syncthreads();
  const int q0 = s_q0;
  const unsigned lm = s_lm;
  if (init_tab || P.phase) {
    // Per-block window parts of the quadratic phase: the init's (layout L0) as a sign
    // mask, the q_A phase's folded into its factors rt.
    if (t < 32) {
      int pax[4] = {0, 9, 10, 11};
      if (!init_tab) {
        phase_axes(S, pax);
      } else if (S.ld_w0 >= 0) {
#pragma unroll
        for (int a = 0; a < 4; ++a) pax[a] = S.ld_w0 + a;
      }
      const int i = t & 15;
      int X = 0;
      float2 v = make_float2(1.f, 0.f);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (!((i >> a) & 1)) continue;
        X |= 1 << pax[a];
        if (P.dg) v = cmulf(v, __ldg(P.rg + local_to_global_bit(P, pax[a])));
      }
      const int w = qt_bit(s_tt, X) ^ (__popc(lm & (unsigned)X) & 1);
      const unsigned mask = __ballot_sync(0xffffffffu, t < 16 && w);
      if (t == 0) s_qw = mask;
      if (t < 16) s_rt[t] = w ? make_float2(-v.x, -v.y) : v;
    }
    __syncthreads();
  }
  float2 r[16];
  // Load stage: init computed in registers (layout L0 or a window), or the state loaded (L0).
  if (init_tab && S.ld_w0 >= 0) {
    const int w0 = S.ld_w0;
    const int fb = round_f0(t, w0);
    const int axw[4] = {w0, w0 + 1, w0 + 2, w0 + 3};
    const unsigned sg = sign_mask(s_tt, q0, lm, fb, axw, s_qw);
    const u64 b0 = s_b0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int f = fb | (i << w0);
      const u64 b = b0 ^ s_tt.mlo[f & 63] ^ s_tt.mhi[(f >> 6) & 63];
      const float2 w = W64 ? __ldg(P.wspecf + __popcll(b) * (P.m + 1) + __popcll(b & P.outmask))
                           : __ldg(P.wspecf + __popc((unsigned)b) * (P.m + 1) + __popc((unsigned)(b & P.outmask)));
      r[i] = ((sg >> i) & 1u) ? make_float2(-w.x, -w.y) : w;
    }
  } else if (init_tab) {
    const int ax0[4] = {0, 9, 10, 11};
    const unsigned sg = sign_mask(s_tt, q0, lm, 2 * t, ax0, s_qw);
    const u64 b0 = s_b0;
    if (W64) {
      const u64 blo[2] = {b0 ^ s_tt.mlo[(2 * t) & 63], b0 ^ s_tt.mlo[(2 * t + 1) & 63]};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const u64 bhi = s_tt.mhi[((2 * t + 512 * k) >> 6) & 63];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const u64 b = blo[e] ^ bhi;
          const float2 w = __ldg(P.wspecf + __popcll(b) * (P.m + 1) + __popcll(b & P.outmask));
          r[2 * k + e] = ((sg >> (2 * k + e)) & 1u) ? make_float2(-w.x, -w.y) : w;
        }
      }
    } else {
      // m <= 32: b and the outcome mask fit 32 bits.
      const unsigned out = (unsigned)P.outmask;
      const unsigned blo[2] = {(unsigned)(b0 ^ s_tt.mlo[(2 * t) & 63]), (unsigned)(b0 ^ s_tt.mlo[(2 * t + 1) & 63])};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const unsigned bhi = (unsigned)s_tt.mhi[((2 * t + 512 * k) >> 6) & 63];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const unsigned b = blo[e] ^ bhi;
          const float2 w = __ldg(P.wspecf + __popc(b) * (P.m + 1) + __popc(b & out));
          r[2 * k + e] = ((sg >> (2 * k + e)) & 1u) ? make_float2(-w.x, -w.y) : w;
        }
      }
    }
  } else if (TMA) {
    // The tile is in the staging buffer (dense, tile index order): wait for it, read it,
    // then refill the buffer with the next tile while this one is transformed.  A wait
    // that gives up sets the error flag and ends the block (uniformly).
    const bool ok = tc::mbar_wait(&s_full, phase);
    phase ^= 1;
    if (__syncthreads_or(!ok)) {
      if (t == 0) {
        atomicExch(&g_fourier_timeout, 1);
        tc::mbar_wait(&s_full, phase ^ 1);  // bounded: the copy in flight, if any
      }
      return;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float4 x = *reinterpret_cast<const float4*>(stage + 2 * t + 512 * k);
      r[2 * k] = make_float2(x.x, x.y);
      r[2 * k + 1] = make_float2(x.z, x.w);
    }
    __syncthreads();
    if (t == 0 && it + gridDim.x < ntl) tma_tile(P, tmap, it + gridDim.x + P.tile0, stage, &s_full);
  } else {
    const float2* vt = P.v + (base & P.amask);
    const LayOff<O> A = lay_off<O>(P, 0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float4 x = *reinterpret_cast<const float4*>(vt + A.at(k));
      r[2 * k] = make_float2(x.x, x.y);
      r[2 * k + 1] = make_float2(x.z, x.w);
    }
  }
  // Stages 0 (load, L0), 1..nr (shared-memory rounds) and nr + 1 (final, L0 or L1) share
  // one copy of the register operations (a rolled loop): the kernel's code stays small
  // enough for the instruction cache.
  const int fl = S.fin_l1;
  const bool exchange = S.nr > 0 || fl || S.ld_w0 >= 0;
#pragma unroll 1
  for (int st = 0; st <= S.nr + 1; ++st) {
    int ax[4];
    unsigned wm, um;
    int fb;
    if (st == 0 && S.ld_w0 >= 0) {
      const int w0 = S.ld_w0;
      ax[0] = w0, ax[1] = w0 + 1, ax[2] = w0 + 2, ax[3] = w0 + 3;
      wm = S.ld_w, um = S.ld_u, fb = round_f0(t, w0);
    } else if (st == 0) {
      ax[0] = 0, ax[1] = 9, ax[2] = 10, ax[3] = 11;
      wm = S.ld_w, um = S.ld_u, fb = 2 * t;
    } else if (st <= S.nr) {
      const int w0 = S.rw0[st - 1];
      ax[0] = w0, ax[1] = w0 + 1, ax[2] = w0 + 2, ax[3] = w0 + 3;
      wm = S.rw[st - 1], um = S.ru[st - 1], fb = round_f0(t, w0);
      __syncthreads();
      round_io_at<false>(sm, r, w0);
    } else {
      ax[0] = 0, ax[1] = fl ? 6 : 9, ax[2] = fl ? 7 : 10, ax[3] = fl ? 8 : 11;
      wm = S.fw, um = S.fu, fb = lay_f(fl, t, 0);
      if (exchange) {
        __syncthreads();
        const float2* bf = sm + pad(fb);
#pragma unroll
        for (int i = 0; i < 16; ++i) r[i] = bf[(i & 1) + (fl ? 68 : 544) * (i >> 1)];
      }
    }
    reg_wht(r, ax, wm);
    if (P.phase && S.phase_at == st) reg_phase(r, P, wt, s_tt, q0, lm, s_rt, fb);
    reg_prod(r, P, s_rot, ax, um);
    if (st == 0 && S.ld_w0 >= 0) {
      round_io_at<true>(sm, r, S.ld_w0);
    } else if (st == 0 && exchange) {
      float2* b0p = sm + pad(2 * t);
#pragma unroll
      for (int i = 0; i < 16; ++i) b0p[(i & 1) + 544 * (i >> 1)] = r[i];
    } else if (st >= 1 && st <= S.nr) {
      round_io_at<true>(sm, r, ax[0]);
    }
  }
  // Diagonal after the products (final layout L0 only), masses, store.
  if (P.dh) {
    const WindowSplit ws = window_split(wt, 256);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int f = lay_f(0, t, 2 * k);
      r[2 * k] = cmulf(r[2 * k], window_factor(wt, ws, f, 0));
      r[2 * k + 1] = cmulf(r[2 * k + 1], window_factor(wt, ws, f, 1));
    }
  }
  float2* vt = P.v + (base & P.amask);
  const LayOff<O> Af = lay_off<O>(P, fl);
  // Sharded pass 0 stores only the elements whose top bit (m - 1) equals store_top.
  const int base_top = (int)((base >> (P.m - 1)) & 1ull);
  double mass = 0.0;  // per element pair: a float sum of four squares, then float64
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float2 a = r[2 * k], b = r[2 * k + 1];
    bool st = P.store != 0;
    if (P.store_top >= 0) {
      const int top = P.top_axis >= 0 ? base_top ^ ((lay_f(fl, t, 2 * k) >> P.top_axis) & 1) : base_top;
      st = st && top == P.store_top;
    }
    if (st) *reinterpret_cast<float4*>(vt + Af.at(k)) = make_float4(a.x, a.y, b.x, b.y);
    if (P.masses) {
      const float2 q = f2fma(b, b, make_float2(a.x * a.x, a.y * a.y));
      mass += (double)(q.x + q.y);
    }
  }
  if (P.masses) {
    __shared__ double red[8];
    double m2 = mass;
    for (int off = 16; off; off >>= 1) m2 += __shfl_xor_sync(0xffffffffu, m2, off);
    if ((t & 31) == 0) red[t >> 5] = m2;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int w = 0; w < 8; ++w) sum += red[w];
      P.masses[tile - P.tile0] = sum;
    }
  }
  if (!TMA) break;  // one tile per block
  }  // tiles
}

// Per-sample weight tables: generic chunk products over b (with 2^{-m/2} in chunk 0)
// or the popcount table of identical B unitaries (init_specialization.py:98-115).
__global__ void fourier_weights_kernel(int m, int chunks, const double2* __restrict__ uB, u64 outmask, int special,
                                       double2* __restrict__ wgen, double2* __restrict__ wspec,
                                       float2* __restrict__ wspecf, int scale_half_m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const double scale = scale_half_m ? exp2(-0.5 * m) : 1.0;
  if (!special) {
    if (e >= chunks * 256) return;
    const int cc = e >> 8, code = e & 255;
    double2 w = make_double2(cc == 0 ? scale : 1.0, 0.0);
    for (int j = 8 * cc; j < min(m, 8 * cc + 8); ++j) {
      const int bit = (code >> (j - 8 * cc)) & 1, out = (int)((outmask >> j) & 1ull);
      w = cmul(w, uB[(j * 2 + out) * 2 + bit]);
    }
    wgen[e] = w;
  } else {
    if (e >= (m + 1) * (m + 1)) return;
    const int k = e / (m + 1), h = e % (m + 1);
    const int r = __popcll(outmask);
    double2 w = make_double2(0.0, 0.0);
    if (h >= max(0, r + k - m) && h <= min(r, k)) {
      const int n[4] = {m - r - k + h, k - h, r - h, h};  // (out,b) = 00, 01, 10, 11
      w = make_double2(scale, 0.0);
      for (int t = 0; t < 4; ++t) {
        const double2 base = uB[t];  // U_B[out][b] of site 0: flat order u00, u01, u10, u11
        for (int p = 0; p < n[t]; ++p) w = cmul(w, base);
      }
    }
    wspec[e] = w;
    wspecf[e] = make_float2((float)w.x, (float)w.y);
  }
}

// Index map with q_A phase and scale (distributed_sampler.py:35-41), single device:
// dst[z] = src[y(z)] (-1)^{q_A(z)} 2^{-m/2}, y = XOR_{k: z_k} cols[k].
__global__ void fourier_index_map_kernel(const float2* __restrict__ src, float2* __restrict__ dst, int m, int chunks,
                                         const u64* __restrict__ lut_cols, const u64* __restrict__ lut_a, float scale) {
  const u64 n = 1ull << m;
  for (u64 z = (u64)blockIdx.x * blockDim.x + threadIdx.x; z < n; z += (u64)gridDim.x * blockDim.x) {
    u64 y = 0;
    for (int cc = 0; cc < chunks; ++cc) y ^= __ldg(lut_cols + ((((u64)cc << 8) + ((z >> (8 * cc)) & 255ull)) << 1));
    const float s = (__popcll(lut_parity_mask(lut_a, chunks, z)) & 1) ? -scale : scale;
    const float2 x = src[y];
    dst[z] = make_float2(s * x.x, s * x.y);
  }
}

__global__ void block_mass_kernel(const float2* __restrict__ v, u64 n, int tile_bits, double* __restrict__ out) {
  const u64 start = (u64)blockIdx.x << tile_bits;
  const u64 end = min(n, start + (1ull << tile_bits));
  double s = 0.0;
  for (u64 i = start + threadIdx.x; i < end; i += blockDim.x) {
    const float2 x = v[i];
    s += (double)x.x * x.x + (double)x.y * x.y;
  }
  __shared__ double red[32];
  for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) t += red[w];
    out[blockIdx.x] = t;
  }
}

struct DrawResult {
  unsigned long long index;
  double pa, norm;
  int status;
};

// First position i of v[0..n) with prefix(i) <= target < prefix(i) + v[i] (searchsorted
// side='right' on the inclusive cumulative sum), found by one 1024-thread block.
// Each thread sums a contiguous chunk; chunk sums are scanned in shared memory.
template <class Get>
__device__ long long block_search(long long n, double target, Get get, double* total_out) {
  __shared__ double part[1024];
  __shared__ long long found;
  const int t = threadIdx.x, nt = blockDim.x;
  const long long chunk = (n + nt - 1) / nt;
  const long long lo = min(n, (long long)t * chunk), hi = min(n, lo + chunk);
  double s = 0.0;
  for (long long i = lo; i < hi; ++i) s += get(i);
  part[t] = s;
  if (t == 0) found = -1;
  __syncthreads();
  if (t == 0) {
    double acc = 0.0;
    for (int k = 0; k < nt; ++k) {
      const double x = part[k];
      part[k] = acc;
      acc += x;
    }
    *total_out = acc;
  }
  __syncthreads();
  const double pre = part[t];
  if (pre <= target && target < pre + s) {
    double acc = pre;
    for (long long i = lo; i < hi; ++i) {
      const double x = get(i);
      if (target < acc + x) {
        found = i;
        break;
      }
      acc += x;
    }
  }
  __syncthreads();
  long long r = found;
  __syncthreads();
  if (r < 0) {  // target at/after the total (rounding): last non-zero entry
    if (t == 0) {
      for (long long i = n - 1; i >= 0; --i)
        if (get(i) > 0.0) {
          found = i;
          break;
        }
    }
    __syncthreads();
    r = found;
  }
  return r;
}

__global__ void __launch_bounds__(1024) fourier_draw_kernel(const double* __restrict__ masses, long long ntiles,
                                                            const float2* __restrict__ v, int m, int tile_bits,
                                                            int deferred, const double2* __restrict__ uT,
                                                            double u1, double u2, double u3,
                                                            DrawResult* __restrict__ out) {
  __shared__ double norm, tile_total;
  double tot;
  // First search (target 0) only establishes the total, then the draw itself.
  block_search(ntiles, 0.0, [&](long long i) { return masses[i]; }, &tot);
  if (threadIdx.x == 0) norm = tot;
  __syncthreads();
  const long long chosen = block_search(ntiles, u1 * norm, [&](long long i) { return masses[i]; }, &tot);
  if (chosen < 0) {  // no tile with positive mass: report, read nothing
    if (threadIdx.x == 0) {
      DrawResult r{0ull, 0.0, norm, 2};
      *out = r;
    }
    return;
  }
  const u64 base = (u64)chosen << tile_bits;
  auto p_at = [&](long long i) {
    const float2 x = v[base + (u64)i];
    return (double)x.x * x.x + (double)x.y * x.y;
  };
  double tt;
  block_search(1ll << tile_bits, 0.0, p_at, &tt);
  if (threadIdx.x == 0) tile_total = tt;
  __syncthreads();
  const long long within = block_search(1ll << tile_bits, u2 * tile_total, p_at, &tt);
  if (within < 0) {
    if (threadIdx.x == 0) {
      DrawResult r{0ull, 0.0, norm, 2};
      *out = r;
    }
    return;
  }
  if (threadIdx.x == 0) {
    const u64 idx = base + (u64)within;
    DrawResult r;
    r.norm = norm;
    r.status = 0;
    if (deferred) {
      const u64 half = 1ull << (m - 1);
      const u64 local = idx & (half - 1ull);
      const float2 a = v[local], b = v[local + half];
      const double2 A = make_double2(a.x, a.y), B = make_double2(b.x, b.y);
      const double2 p0 = make_double2(cmul(uT[0], A).x + cmul(uT[1], B).x, cmul(uT[0], A).y + cmul(uT[1], B).y);
      const double2 p1 = make_double2(cmul(uT[2], A).x + cmul(uT[3], B).x, cmul(uT[2], A).y + cmul(uT[3], B).y);
      const double q0 = p0.x * p0.x + p0.y * p0.y, q1 = p1.x * p1.x + p1.y * p1.y;
      const double total = q0 + q1;
      if (!(total > 0.0) || !isfinite(total)) r.status = 1;
      const int bit = (u3 * total >= q0) ? 1 : 0;
      r.index = bit ? local + half : local;
      r.pa = bit ? q1 : q0;
    } else {
      r.index = idx;
      const float2 x = v[idx];
      r.pa = (double)x.x * x.x + (double)x.y * x.y;
    }
    *out = r;
  }
}

// Total of the tile masses of a shard (the same fixed-order reduction as the draw).
__global__ void __launch_bounds__(1024) shard_mass_kernel(const double* __restrict__ masses, long long ntiles,
                                                          double* __restrict__ out) {
  double tot;
  block_search(ntiles, 0.0, [&](long long i) { return masses[i]; }, &tot);
  if (threadIdx.x == 0) *out = tot;
}

// ------------------------------------------------------------------------------------- host
std::mutex g_fourier_mutex;
std::atomic<bool> g_fourier_legacy{false};  // true: every pass on fourier_pass_kernel
std::atomic<bool> g_fourier_tma{false};     // TMA-staged loads of the register-first passes (opt-in)

// Tensor map of a loading pass's tiles over the state buffer (8-byte elements): the index
// bits in runs -- the tile's low bits [0, c), the mid bits [c, q), the target bits
// [q, q + K), the high bits -- runs of tile bits split at 8 bits (box dimensions <= 256),
// boxes full on tile runs and 1 elsewhere.  False when the geometry does not fit five
// dimensions or the TMA limits (then the pass loads with plain 16-byte accesses).
bool tma_pass_map(PassParams& P, CUtensorMap* map) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc || ((uintptr_t)P.v & 15) != 0) return false;
  const int mm = P.amask == ~0ull ? P.m : P.m - 1;  // index bits of the buffer
  if (P.q + P.K > mm) return false;
  struct Run {
    int lo, bits;
    bool tile;
  };
  std::vector<Run> runs;
  auto tile_run = [&](int lo, int bits) {
    for (int b = 0; b < bits; b += 8) runs.push_back({lo + b, std::min(8, bits - b), true});
  };
  tile_run(0, P.c);
  P.tma_mid_dim = P.tma_high_dim = -1;
  if (P.q > P.c) {
    P.tma_mid_dim = (int)runs.size();
    runs.push_back({P.c, P.q - P.c, false});
  }
  tile_run(P.q, P.K);
  if (mm > P.q + P.K) {
    P.tma_high_dim = (int)runs.size();
    runs.push_back({P.q + P.K, mm - P.q - P.K, false});
  }
  if (runs.size() > 5) return false;
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
  for (int d = 0; d < 5; ++d) {
    const bool real = d < (int)runs.size();
    dims[d] = real ? (1ull << runs[d].bits) : 1ull;
    box[d] = real && runs[d].tile ? (1u << runs[d].bits) : 1u;
    if (d > 0) {
      strides[d - 1] = real ? (8ull << runs[d].lo) : 16ull;
      if (strides[d - 1] >= (1ull << 40) || dims[d] > (1ull << 32)) return false;
    }
  }
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, (void*)P.v, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MINB>
int set_smem_attr() {
  static bool done[64] = {false};
  int device = 0;
  RGS_CUDA_TRY(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(g_fourier_mutex);
  if (device >= 0 && device < 64 && done[device]) return RGS_OK;
  const int bytes = ((1 << kTileBits) + (1 << (kTileBits - 4))) * (int)sizeof(float2);
  RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_pass_kernel<MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_sched_kernel<MINB, false, false, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_sched_kernel<MINB, true, false, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_sched_kernel<MINB, false, false, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_sched_kernel<MINB, true, false, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if (MINB == 3) {
    RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_sched_kernel<3, false, true, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmemBytes));
    RGS_CUDA_TRY(cudaFuncSetAttribute(fourier_sched_kernel<3, true, true, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmemBytes));
  }
  if (device >= 0 && device < 64) done[device] = true;
  return RGS_OK;
}

// One stage sequence of the register-first kernel for a given round count and final
// layout: every axis goes to the earliest stage that holds it, the phase (or the
// WHT -> products boundary) to the stage where the last WHT axis is done.
bool simulate_sched(unsigned W, unsigned U, bool phase, int n, const int* w0, int fl, int ldw, PassSched& T) {
  const unsigned R0 = 1u | (7u << 9), R1 = 1u | (7u << 6);
  const unsigned Rl = ldw < 0 ? R0 : (15u << ldw);  // registers of the load stage
  T = PassSched{};
  T.ld_w0 = ldw;
  bool pending = W != 0 || phase;
  unsigned Wr = W, Ur = U;
  T.phase_at = -1;
  T.ld_w = Wr & Rl;
  Wr &= ~Rl;
  if (pending && !Wr) {
    T.phase_at = 0;
    pending = false;
  }
  T.ld_u = pending ? 0u : (Ur & Rl);
  Ur &= ~T.ld_u;
  T.nr = n;
  for (int j = 0; j < n; ++j) {
    const unsigned win = 15u << w0[j];
    T.rw0[j] = w0[j];
    T.rw[j] = Wr & win;
    Wr &= ~T.rw[j];
    if (pending && !Wr) {
      T.phase_at = j + 1;
      pending = false;
    }
    T.ru[j] = pending ? 0u : (Ur & win);
    Ur &= ~T.ru[j];
  }
  const unsigned Rf = fl ? R1 : R0;
  if (Wr & ~Rf) return false;
  T.fw = Wr;
  if (pending) T.phase_at = n + 1;
  if (Ur & ~Rf) return false;
  T.fu = Ur;
  T.fin_l1 = fl;
  return true;
}

// Fewest shared-memory rounds (windows w0 in 0..8, all conflict-free in the padded
// layout), final layout L0 preferred; false when three rounds do not suffice.  A pass
// that computes its tile (the init) may also hold any window in registers at the load
// stage (its elements need no coalesced load), which saves the init pass a round.
bool plan_sched(const PassParams& P, PassSched& S) {
  const bool phase = P.phase != 0;
#ifdef RGS_NO_INIT_WINDOW
  const int ldmax = -1;
#else
  const int ldmax = P.init ? 8 : -1;
#endif
  for (int n = 0; n <= 3; ++n) {
    int count = 1;
    for (int j = 0; j < n; ++j) count *= 9;
    for (int ldw = -1; ldw <= ldmax; ++ldw)
      for (int fl = 0; fl < 2; ++fl) {
        if (fl && P.dh) continue;  // the diagonal after the products uses layout L0
        for (int code = 0; code < count; ++code) {
          int w0[3] = {0, 0, 0};
          for (int j = 0, c = code; j < n; ++j, c /= 9) w0[j] = c % 9;
          if (simulate_sched(P.wht_mask, P.u_mask, phase, n, w0, fl, ldw, S)) return true;
        }
      }
  }
  return false;
}

int launch_pass(const PassParams& Pin, cudaStream_t s) {
  const int TB = Pin.c + Pin.K;
  if (TB < 4 || TB > kTileBits) return fail(RGS_ERR_UNSUPPORTED, "tile must span 4..13 bits");
  const u64 tiles = Pin.ntiles ? Pin.ntiles : (1ull << (Pin.m - TB));
  const size_t smem = ((1 << TB) + (1 << (TB - 4))) * sizeof(float2);
  int rc = Pin.variant ? set_smem_attr<4>() : set_smem_attr<3>();
  if (rc) return rc;
  PassParams P = Pin;
  // The register-first kernel: 12-bit tiles, the phase from pass tables, at most one
  // diagonal, not both the init and the phase, the table init only, products as scaled
  // rotations (the rest takes fourier_pass_kernel).
  P.sched = TB == kTileBits && !(P.init && P.phase) && !(P.phase && !P.tt_phase) && !(P.dg && P.dh) &&
            !(P.u_mask && !P.rot) && !(P.init && !(P.init == INIT_COV_SPECIAL && P.tt_init)) && !g_fourier_legacy &&
            plan_sched(P, P.s);
  P.top_axis = -1;
  for (int a = 0; a < TB; ++a)
    if ((a < P.c ? a : P.q + (a - P.c)) == P.m - 1) P.top_axis = a;
  if (P.sched) {
    // 32-bit element offsets inside a tile while the state has at most 2^32 elements.
    const bool w64 = P.m > 32;
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (!P.init && g_fourier_tma && tma_pass_map(P, &map)) {
      // TMA-staged persistent blocks: three per SM (work + staging buffers).
      if (P.variant) {
        const int rc3 = set_smem_attr<3>();
        if (rc3) return rc3;
      }
      int dev = 0;
      RGS_CUDA_TRY(cudaGetDevice(&dev));
      const unsigned grid = (unsigned)std::min<u64>(tiles, (u64)3 * sm_count(dev));
      if (w64)
        fourier_sched_kernel<3, true, true, false><<<grid, 256, kTmaSmemBytes, s>>>(P, map);
      else
        fourier_sched_kernel<3, false, true, false><<<grid, 256, kTmaSmemBytes, s>>>(P, map);
    } else if (P.init) {
      // The table init (the only init this kernel takes, see P.sched above).
      const unsigned g = (unsigned)tiles;
      if (P.variant && w64)
        fourier_sched_kernel<4, true, false, true><<<g, 256, smem, s>>>(P, map);
      else if (P.variant)
        fourier_sched_kernel<4, false, false, true><<<g, 256, smem, s>>>(P, map);
      else if (w64)
        fourier_sched_kernel<3, true, false, true><<<g, 256, smem, s>>>(P, map);
      else
        fourier_sched_kernel<3, false, false, true><<<g, 256, smem, s>>>(P, map);
    } else if (P.variant && w64) {
      fourier_sched_kernel<4, true, false, false><<<(unsigned)tiles, 256, smem, s>>>(P, map);
    } else if (P.variant) {
      fourier_sched_kernel<4, false, false, false><<<(unsigned)tiles, 256, smem, s>>>(P, map);
    } else if (w64) {
      fourier_sched_kernel<3, true, false, false><<<(unsigned)tiles, 256, smem, s>>>(P, map);
    } else {
      fourier_sched_kernel<3, false, false, false><<<(unsigned)tiles, 256, smem, s>>>(P, map);
    }
  } else if (P.variant) {
    fourier_pass_kernel<4><<<(unsigned)tiles, 1 << (TB - 4), smem, s>>>(P);
  } else {
    fourier_pass_kernel<3><<<(unsigned)tiles, 1 << (TB - 4), smem, s>>>(P);
  }
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

// Bit groups above the low tile, as equal as possible and at most 10 bits each
// (a strided tile keeps at least 3 contiguous low bits = 64-byte runs).
std::vector<std::pair<int, int>> strided_groups(int m) {
  std::vector<std::pair<int, int>> g;
  const int rest = m - kTileBits;
  if (rest <= 0) return g;
  const int maxk = kTileBits - kLowBits;
  const int k = (rest + maxk - 1) / maxk;
  int lo = kTileBits;
  for (int i = 0; i < k; ++i) {
    const int size = rest / k + (i < rest % k ? 1 : 0);
    g.push_back({lo, lo + size});
    lo += size;
  }
  return g;
}

PassParams base_params(const FourierPlan& p, float2* v) {
  PassParams P{};
  P.v = v;
  P.amask = ~0ull;
  P.store_top = -1;
  P.m = p.m;
  P.chunks = p.chunks;
  P.lut_a = (const u64*)p.d_lut_a;
  P.u = (const double2*)p.d_uA;
  P.store = 1;
  return P;
}

void contiguous(PassParams& P, int m) {
  P.c = std::min(m, kTileBits);
  P.K = 0;
  P.q = P.c;
}

// A strided tile spans 13 bits: the target bits [lo, hi) plus as many contiguous low
// bits as fit (longer runs when the group is small).
void strided(PassParams& P, int lo, int hi) {
  P.K = hi - lo;
  P.c = kTileBits - P.K;
  P.q = lo;
}

// Two-shard schedule: the bits [11, m - 1) in balanced groups of at most 9 bits (bit
// 11 is not in the shard's init tile, which holds bits 0..10 and the top bit m - 1).
std::vector<std::pair<int, int>> shard_groups(int m) {
  std::vector<std::pair<int, int>> g;
  const int lo0 = kTileBits - 1, rest = (m - 1) - lo0;
  if (rest <= 0) return g;
  const int maxk = kTileBits - kLowBits;
  const int k = (rest + maxk - 1) / maxk;
  int lo = lo0;
  for (int i = 0; i < k; ++i) {
    const int size = rest / k + (i < rest % k ? 1 : 0);
    g.push_back({lo, lo + size});
    lo += size;
  }
  return g;
}

unsigned target_mask(const PassParams& P) { return ((1u << P.K) - 1u) << P.c; }

int local_to_global_host(const PassParams& P, int a) { return a < P.c ? a : P.q + (a - P.c); }

// Product axes of a contiguous/strided tile, without the deferred terminal bit.
unsigned product_mask(const FourierPlan& p, const PassParams& P, unsigned axes) {
  if (!p.deferred) return axes;
  for (int a = 0; a < P.c + P.K; ++a)
    if (((axes >> a) & 1u) && local_to_global_host(P, a) == p.m - 1) axes &= ~(1u << a);
  return axes;
}

// Passes applying `op` (WHT or products) to the bits [lo, hi) of an nbits state.
int transform_range(PassParams P, int nbits, int lo, int hi, bool wht, cudaStream_t s) {
  if (nbits < 4) return fail(RGS_ERR_UNSUPPORTED, "states of fewer than 4 qubits are not supported");
  if (lo < 0 || hi > nbits || lo >= hi) return fail(RGS_ERR_ARG, "bad bit range");
  P.m = nbits;
  contiguous(P, nbits);
  unsigned low = 0;
  for (int b = lo; b < std::min(hi, P.c); ++b) low |= 1u << b;
  if (low) {
    P.wht_mask = wht ? low : 0;
    P.u_mask = wht ? 0 : low;
    int rc = launch_pass(P, s);
    if (rc) return rc;
  }
  for (auto g : strided_groups(nbits)) {
    const int a = std::max(lo, g.first), b = std::min(hi, g.second);
    if (a >= b) continue;
    strided(P, g.first, g.second);
    unsigned mask = 0;
    for (int bit = a; bit < b; ++bit) mask |= 1u << (P.c + bit - g.first);
    P.wht_mask = wht ? mask : 0;
    P.u_mask = wht ? 0 : mask;
    int rc = launch_pass(P, s);
    if (rc) return rc;
  }
  return RGS_OK;
}

int build_weights(FourierPlan& p, uint64_t outB, char* ws, const FourierLayout& L, bool special, bool scale,
                  cudaStream_t s) {
  double2* w = (double2*)(ws + L.off_weights);
  const int entries = special ? (p.m + 1) * (p.m + 1) : p.chunks * 256;
  fourier_weights_kernel<<<(entries + 255) / 256, 256, 0, s>>>(p.m, p.chunks, (const double2*)p.d_uB, outB,
                                                               special ? 1 : 0, w, w, (float2*)(ws + L.off_wspecf),
                                                               scale ? 1 : 0);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int check_state(FourierPlan& p, const void* state, void* ws, size_t ws_bytes, FourierLayout& L) {
  if (!state || !ws) return fail(RGS_ERR_ARG, "null state or workspace");
  if (((uintptr_t)state & 15) || ((uintptr_t)ws & 255)) return fail(RGS_ERR_ARG, "misaligned state or workspace");
  fourier_layout(p, L);
  if (ws_bytes < L.total) return fail(RGS_ERR_OOM, "workspace smaller than rgs_fourier_workspace_bytes()");
  int device = 0;
  int rc = bind_device_of(state, &device);
  if (rc) return rc;
  return fourier_upload(p, device);
}

// Euler factorisation of a 2x2 unitary: U = diag(h) R diag(g) with R = [[c, -s], [s, c]]
// (c = cos(beta/2), s = sin(beta/2) >= 0) and unit-modulus h, g -- the ZYZ decomposition
// with the global phase folded into h.  All products on the A sites then split into one
// diagonal before (folded into the q_A phase), real rotations (4 FFMA per element and
// axis instead of 8 for a complex 2x2), and one diagonal after them.  Returns false if
// the reconstruction misses U by more than 1e-9 (a non-unitary input).
bool euler_factors(const double* u, std::complex<double> g[2], std::complex<double> h[2], double& c, double& s) {
  typedef std::complex<double> C;
  const C a(u[0], u[1]), b(u[2], u[3]), cc(u[4], u[5]), d(u[6], u[7]);
  c = std::sqrt(0.5 * (std::norm(a) + std::norm(d)));
  s = std::sqrt(0.5 * (std::norm(b) + std::norm(cc)));
  const double nrm = std::hypot(c, s);
  if (!(nrm > 0.0)) return false;
  c /= nrm;
  s /= nrm;
  g[0] = g[1] = C(1.0, 0.0);
  if (s < 1e-12) {
    c = 1.0;
    s = 0.0;
    h[0] = a / std::abs(a);
    h[1] = d / std::abs(d);
  } else if (c < 1e-12) {
    c = 0.0;
    s = 1.0;
    h[0] = -b / std::abs(b);
    h[1] = cc / std::abs(cc);
  } else {
    h[0] = a / std::abs(a);
    h[1] = cc / std::abs(cc);
    g[1] = (-b / std::abs(b)) / h[0];
  }
  const C r[4] = {h[0] * c * g[0], -h[0] * s * g[1], h[1] * s * g[0], h[1] * c * g[1]};
  const C v[4] = {a, b, cc, d};
  double err = 0.0;
  for (int k = 0; k < 4; ++k) err = std::max(err, std::abs(r[k] - v[k]));
  return err < 1e-9;
}

// Host evaluation of the chunk tables (as the device does): the map part b(z) and the
// quadratic phase q(z).
u64 host_lut_map(const std::vector<u64h>& lut, int chunks, u64 z) {
  u64 b = 0;
  for (int cc = 0; cc < chunks; ++cc) b ^= lut[(((size_t)cc << 8) + ((z >> (8 * cc)) & 255ull)) * 2];
  return b;
}
int host_lut_q(const std::vector<u64h>& lut, int chunks, u64 z) {
  u64 pm = 0;
  for (int cc = 0; cc < chunks; ++cc) pm ^= lut[(((size_t)cc << 8) + ((z >> (8 * cc)) & 255ull)) * 2 + 1];
  return __builtin_popcountll(pm & (z | (1ull << 63))) & 1;
}

// Pass tables (TileTables) of a tile whose local bit a sits at global bit
// a < c ? a : q + (a - c), and the rows of Q + Q^T of the phase (see the kernel).
void pass_tables(const std::vector<u64h>& lut, int chunks, int m, int c, int K, int q, bool map, TileTables& tt,
                 std::vector<u64h>& qsym) {
  const int TB = c + K;
  auto global = [&](int f) {
    u64 z = 0;
    for (int a = 0; a < TB; ++a)
      if ((f >> a) & 1) z |= 1ull << (a < c ? a : q + (a - c));
    return z;
  };
  for (int i = 0; i < 64; ++i) {
    tt.mlo[i] = (map && i < (1 << TB)) ? host_lut_map(lut, chunks, global(i)) : 0ull;
    tt.mhi[i] = (map && (i << 6) < (1 << TB)) ? host_lut_map(lut, chunks, global(i << 6)) : 0ull;
  }
  for (int w = 0; w < 128; ++w) tt.qtab[w] = 0u;
  for (int f = 0; f < (1 << TB); ++f)
    if (host_lut_q(lut, chunks, global(f))) tt.qtab[f >> 5] |= 1u << (f & 31);
  qsym.assign(m, 0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j)
      if (i != j && (host_lut_q(lut, chunks, (1ull << i) ^ (1ull << j)) ^ host_lut_q(lut, chunks, 1ull << i) ^
                     host_lut_q(lut, chunks, 1ull << j)))
        qsym[i] |= 1ull << j;
}

// Chunk tables of a diagonal over m bits: T[c][code] = prod over bits t of chunk c of
// f_j[bit t of code], j = 8c + t.
void diag_tables(int m, int chunks, const std::vector<std::complex<double>>& f, std::vector<float>& out) {
  out.assign((size_t)chunks * 256 * 2, 0.f);
  for (int cc = 0; cc < chunks; ++cc)
    for (int code = 0; code < 256; ++code) {
      std::complex<double> v(1.0, 0.0);
      for (int t = 0; t < 8; ++t) {
        const int j = 8 * cc + t;
        if (j < m) v *= f[2 * j + ((code >> t) & 1)];
      }
      out[((size_t)cc * 256 + code) * 2] = (float)v.real();
      out[((size_t)cc * 256 + code) * 2 + 1] = (float)v.imag();
    }
}

}  // namespace

int fourier_set_register_schedule(int on) {
  g_fourier_legacy = !on;
  return RGS_OK;
}

int fourier_set_tma(int on) {
  g_fourier_tma = on != 0;
  return RGS_OK;
}

int fourier_tma_timeout(int* timed_out) {
  int h = 0, zero = 0;
  RGS_CUDA_TRY(cudaMemcpyFromSymbol(&h, g_fourier_timeout, sizeof(int)));
  RGS_CUDA_TRY(cudaMemcpyToSymbol(g_fourier_timeout, &zero, sizeof(int)));
  *timed_out = h;
  return RGS_OK;
}

std::string fourier_build(int n, const uint8_t* graph, const double* unitaries, int m, const int* A, const int* B,
                          bool deferred, FourierPlan& p, int& status) {
  status = RGS_ERR_ARG;
  if (n < 2 || n > 128 || !graph || !unitaries || !A || !B) return "bad arguments";
  if (m < 4 || m > 40) return "conditional size m must be in [4, 40]";
  std::vector<char> seen(n, 0);
  for (int j = 0; j < m; ++j) {
    if (A[j] < 0 || A[j] >= n || B[j] < 0 || B[j] >= n) return "A/B vertex out of range";
    if (seen[A[j]] || seen[B[j]] || A[j] == B[j]) return "A and B must be disjoint sets of distinct vertices";
    seen[A[j]] = seen[B[j]] = 1;
  }
  auto g = [&](int a, int b) { return graph[(size_t)a * n + b] != 0; };
  p.n = n;
  p.m = m;
  p.A.assign(A, A + m);
  p.B.assign(B, B + m);
  p.deferred = deferred;
  std::vector<u64h> M(m, 0), gB(m, 0), gA(m, 0);
  p.cols.assign(m, 0);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      if (g(B[j], A[i])) M[j] |= 1ull << i;
      if (g(B[j], B[i])) gB[j] |= 1ull << i;
      if (g(A[j], A[i])) gA[j] |= 1ull << i;
      if (g(A[j], B[i])) p.cols[j] |= 1ull << i;
    }
  if (gf2_rank(M, m) != m) {
    status = RGS_ERR_SINGULAR;
    return "B marginal is not uniform: rank(G[B,A]) < |B|";
  }
  std::vector<u64h> inv;
  if (!gf2_inverse(M, m, inv)) {
    status = RGS_ERR_SINGULAR;
    return "singular GF(2) matrix";
  }
  // N = inv^T: b_j = parity(row_j(N) & z); column j of N = row j of inv.
  p.inv_rows = gf2_transpose(inv, m);
  std::vector<u64h> Q;
  u64h lin = 0;
  transformed_quadratic(gB, p.inv_rows, m, Q, lin);
  chunk_tables(m, kChunkBits, inv, Q, lin, p.lut_z, p.chunks);
  p.qA = upper_masks(gA, m);
  p.qB = upper_masks(gB, m);
  int ch = 0;
  chunk_tables(m, kChunkBits, {}, p.qA, 0, p.lut_a, ch);
  chunk_tables(m, kChunkBits, p.cols, std::vector<u64h>(m, 0), 0, p.lut_cols, ch);
  p.uA.resize((size_t)m * 8);
  p.uB.resize((size_t)m * 8);
  for (int j = 0; j < m; ++j)
    for (int e = 0; e < 8; ++e) {
      p.uA[(size_t)j * 8 + e] = unitaries[(size_t)A[j] * 8 + e];
      p.uB[(size_t)j * 8 + e] = unitaries[(size_t)B[j] * 8 + e];
    }
  p.specialized = true;
  for (int j = 1; j < m && p.specialized; ++j)
    for (int e = 0; e < 8; ++e)
      if (p.uB[(size_t)j * 8 + e] != p.uB[e]) p.specialized = false;
  // Euler factors of the A-site unitaries (trivial for the deferred terminal bit).
  std::vector<std::complex<double>> fg(2 * m, 1.0), fh(2 * m, 1.0);
  p.rot.assign((size_t)2 * m, 0.f);
  p.rot_ok = true;
  for (int j = 0; j < m && p.rot_ok; ++j) {
    if (deferred && j == m - 1) continue;  // form 0 with k = 0: never applied
    std::complex<double> g2[2], h2[2];
    double c = 0.0, sn = 0.0;
    if (!euler_factors(&p.uA[(size_t)j * 8], g2, h2, c, sn)) p.rot_ok = false;
    // R(c, s) = c [[1, -s/c], [s/c, 1]] (form 0) or s diag(-1, 1) [[-c/s, 1], [1, c/s]]
    // (form 1); the scalar and diag(-1, 1) join the diagonal h applied after the products.
    fg[2 * j] = g2[0];
    fg[2 * j + 1] = g2[1];
    if (c >= sn) {
      fh[2 * j] = h2[0] * c;
      fh[2 * j + 1] = h2[1] * c;
      p.rot[2 * j] = (float)(sn / c);
      p.rot[2 * j + 1] = 0.f;
    } else {
      fh[2 * j] = -h2[0] * sn;
      fh[2 * j + 1] = h2[1] * sn;
      p.rot[2 * j] = (float)(c / sn);
      p.rot[2 * j + 1] = 1.f;
    }
  }
  if (p.rot_ok) {
    diag_tables(m, p.chunks, fg, p.dg);
    diag_tables(m, p.chunks, fh, p.dh);
    p.rg.resize((size_t)2 * m);
    p.rh.resize((size_t)2 * m);
    for (int j = 0; j < m; ++j) {
      const std::complex<double> a = fg[2 * j + 1] / fg[2 * j], b = fh[2 * j + 1] / fh[2 * j];
      p.rg[2 * j] = (float)a.real();
      p.rg[2 * j + 1] = (float)a.imag();
      p.rh[2 * j] = (float)b.real();
      p.rh[2 * j + 1] = (float)b.imag();
    }
  }
  // Pass tables of the init (pass 0, contiguous) and of the q_A phase (its pass).
  {
    const int c0 = std::min(m, kTileBits);
    pass_tables(p.lut_z, p.chunks, m, c0, 0, c0, true, p.tt_init, p.qsym_z);
    const auto groups = strided_groups(m);
    if (groups.empty()) {
      pass_tables(p.lut_a, p.chunks, m, c0, 0, c0, false, p.tt_phase, p.qsym_a);
    } else {
      const auto g = groups.back();
      const int K = g.second - g.first;
      pass_tables(p.lut_a, p.chunks, m, kTileBits - K, K, g.first, false, p.tt_phase, p.qsym_a);
    }
  }
  p.ngroups = (int)strided_groups(m).size();
  // Two-shard schedule tables (see fourier_compute_shard).
  p.shardable = deferred && m >= kTileBits + 1;
  if (p.shardable) {
    std::vector<u64h> qs;
    pass_tables(p.lut_z, p.chunks, m, kTileBits - 1, 1, m - 1, true, p.tt_init_shard, qs);
    const auto g = shard_groups(m).back();
    const int K = g.second - g.first;
    pass_tables(p.lut_a, p.chunks, m, kTileBits - K, K, g.first, false, p.tt_phase_shard, qs);
  }
  status = RGS_OK;
  return "";
}

void fourier_layout(const FourierPlan& p, FourierLayout& L) {
  const int TB = std::min(p.m, kTileBits);
  L.ntiles = 1ll << (p.m - TB);
  L.off_masses = 0;
  L.off_weights = align_up((size_t)L.ntiles * sizeof(double), 256);
  const size_t wentries = std::max<size_t>((size_t)p.chunks * 256, (size_t)(p.m + 1) * (p.m + 1));
  L.off_wspecf = L.off_weights + align_up(wentries * 16, 256);
  L.off_result = L.off_wspecf + align_up((size_t)(p.m + 1) * (p.m + 1) * 8, 256);
  L.total = L.off_result + 256;
}

int fourier_upload(FourierPlan& p, int device) {
  std::lock_guard<std::mutex> lock(g_fourier_mutex);
  if (p.device == device) return RGS_OK;
  if (p.device >= 0) return fail(RGS_ERR_ARG, "a conditional-sampler plan is bound to one device");
  std::vector<u64h> bq;
  int ch = 0;
  chunk_tables(p.m, kChunkBits, {}, p.qB, 0, bq, ch);
  // lut_z holds [covariant | q_B-over-b] back to back.
  std::vector<u64h> z(p.lut_z);
  z.insert(z.end(), bq.begin(), bq.end());
  auto up = [&](void** dst, const void* src, size_t bytes) -> int {
    RGS_CUDA_TRY(cudaMalloc(dst, bytes));
    RGS_CUDA_TRY(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return RGS_OK;
  };
  int rc;
  if ((rc = up(&p.d_lut_z, z.data(), z.size() * 8))) return rc;
  if ((rc = up(&p.d_lut_a, p.lut_a.data(), p.lut_a.size() * 8))) return rc;
  if ((rc = up(&p.d_lut_cols, p.lut_cols.data(), p.lut_cols.size() * 8))) return rc;
  if ((rc = up(&p.d_uA, p.uA.data(), p.uA.size() * 8))) return rc;
  if ((rc = up(&p.d_uB, p.uB.data(), p.uB.size() * 8))) return rc;
  if ((rc = up(&p.d_tt_init, &p.tt_init, sizeof(TileTables)))) return rc;
  if ((rc = up(&p.d_tt_phase, &p.tt_phase, sizeof(TileTables)))) return rc;
  if (p.shardable) {
    if ((rc = up(&p.d_tt_init_shard, &p.tt_init_shard, sizeof(TileTables)))) return rc;
    if ((rc = up(&p.d_tt_phase_shard, &p.tt_phase_shard, sizeof(TileTables)))) return rc;
  }
  if ((rc = up(&p.d_qsym_z, p.qsym_z.data(), p.qsym_z.size() * 8))) return rc;
  if ((rc = up(&p.d_qsym_a, p.qsym_a.data(), p.qsym_a.size() * 8))) return rc;
  if (p.rot_ok) {
    if ((rc = up(&p.d_rot, p.rot.data(), p.rot.size() * 4))) return rc;
    if ((rc = up(&p.d_dg, p.dg.data(), p.dg.size() * 4))) return rc;
    if ((rc = up(&p.d_dh, p.dh.data(), p.dh.size() * 4))) return rc;
    if ((rc = up(&p.d_rg, p.rg.data(), p.rg.size() * 4))) return rc;
    if ((rc = up(&p.d_rh, p.rh.data(), p.rh.size() * 4))) return rc;
  }
  p.device = device;
  return RGS_OK;
}

int fourier_compute(FourierPlan& p, uint64_t outB, void* state, void* ws, size_t ws_bytes, cudaStream_t s,
                    FourierStages* stages) {
  FourierLayout L;
  int rc = check_state(p, state, ws, ws_bytes, L);
  if (rc) return rc;
  char* w = (char*)ws;
  rc = build_weights(p, outB, w, L, p.specialized, true, s);
  if (rc) return rc;
  cudaEvent_t ev[4];
  if (stages)
    for (auto& e : ev) RGS_CUDA_TRY(cudaEventCreate(&e));
  if (stages) RGS_CUDA_TRY(cudaEventRecord(ev[0], s));
  PassParams P = base_params(p, (float2*)state);
  P.init = p.specialized ? INIT_COV_SPECIAL : INIT_COV_GENERIC;
  P.lut_z = (const u64*)p.d_lut_z;
  P.wgen = (const double2*)(w + L.off_weights);
  P.wspec = (const double2*)(w + L.off_weights);
  P.wspecf = (const float2*)(w + L.off_wspecf);
  P.outmask = outB;
  P.rg = (const float2*)p.d_rg;
  P.rh = (const float2*)p.d_rh;
  if (p.specialized) {
    P.tt_init = (const TileTables*)p.d_tt_init;
    P.qsym_z = (const u64*)p.d_qsym_z;
  }
  P.tt_phase = (const TileTables*)p.d_tt_phase;
  P.qsym_a = (const u64*)p.d_qsym_a;
  P.variant = p.variant;
  // Products as real rotations between the two Euler diagonals: dg with the q_A phase,
  // dh after the last products.
  const float2* dg = p.rot_ok ? (const float2*)p.d_dg : nullptr;
  const float2* dh = p.rot_ok ? (const float2*)p.d_dh : nullptr;
  P.rot = p.rot_ok ? (const float2*)p.d_rot : nullptr;
  double* masses = (double*)(w + L.off_masses);
  const int m = p.m;
  if (m <= kTileBits) {
    contiguous(P, m);
    P.wht_mask = (1u << m) - 1u;
    P.phase = 1;
    P.dg = dg;
    P.dh = dh;
    P.u_mask = product_mask(p, P, (1u << m) - 1u);
    P.masses = masses;
    if ((rc = launch_pass(P, s))) return rc;
    if (stages) {
      RGS_CUDA_TRY(cudaEventRecord(ev[1], s));
      RGS_CUDA_TRY(cudaEventRecord(ev[2], s));
    }
  } else {
    const auto groups = strided_groups(m);
    const int k = (int)groups.size();
    contiguous(P, m);
    P.wht_mask = (1u << kTileBits) - 1u;
    if ((rc = launch_pass(P, s))) return rc;
    if (stages) RGS_CUDA_TRY(cudaEventRecord(ev[1], s));
    P.init = INIT_LOAD;
    for (int i = 0; i + 1 < k; ++i) {
      strided(P, groups[i].first, groups[i].second);
      P.wht_mask = target_mask(P);
      if ((rc = launch_pass(P, s))) return rc;
    }
    strided(P, groups[k - 1].first, groups[k - 1].second);
    P.wht_mask = target_mask(P);
    P.phase = 1;
    P.dg = dg;
    P.u_mask = product_mask(p, P, target_mask(P));
    if ((rc = launch_pass(P, s))) return rc;
    if (stages) RGS_CUDA_TRY(cudaEventRecord(ev[2], s));
    P.phase = 0;
    P.dg = nullptr;
    P.wht_mask = 0;
    for (int i = k - 2; i >= 0; --i) {
      strided(P, groups[i].first, groups[i].second);
      P.u_mask = product_mask(p, P, target_mask(P));
      if ((rc = launch_pass(P, s))) return rc;
    }
    contiguous(P, m);
    P.u_mask = product_mask(p, P, (1u << kTileBits) - 1u);
    P.dh = dh;
    P.masses = masses;
    if ((rc = launch_pass(P, s))) return rc;
  }
  if (stages) {
    RGS_CUDA_TRY(cudaEventRecord(ev[3], s));
    RGS_CUDA_TRY(cudaEventSynchronize(ev[3]));
    cudaEventElapsedTime(&stages->init_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&stages->walsh_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&stages->product_ms, ev[2], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return RGS_OK;
}

// Shard `shard` of two: the top bit m - 1 is the device index.  Pass schedule:
//   pass 0        : tile = bits 0..10 and bit m - 1 (c = 11, K = 1, q = m - 1); the init is
//                   computed for both values of the top bit and the WHT runs on all 12
//                   tile bits, so the top bit's Walsh factor needs no exchange; only the
//                   elements of this shard are stored
//   strided passes: WHT on the groups of bits [11, m - 1) (this shard's tiles only)
//   middle pass   : WHT on the last group, q_A phase (global index), products on it
//   strided passes: products on the earlier groups, reverse order
//   last pass     : products on bits 0..10 (contiguous tile of 12 bits) + tile masses
// The products skip the top bit (its unitary is the deferred terminal one, applied at
// draw time to the pair of values at one local index on the two shards).
int fourier_compute_shard(FourierPlan& p, uint64_t outB, int shard, void* state, void* ws, size_t ws_bytes,
                          cudaStream_t s) {
  if (shard != 0 && shard != 1) return fail(RGS_ERR_ARG, "shard must be 0 or 1");
  if (!p.shardable) return fail(RGS_ERR_UNSUPPORTED, "two-shard schedule needs the deferred sampler and m >= 13");
  FourierLayout L;
  int rc = check_state(p, state, ws, ws_bytes, L);
  if (rc) return rc;
  char* w = (char*)ws;
  if ((rc = build_weights(p, outB, w, L, p.specialized, true, s))) return rc;
  const int m = p.m;
  PassParams P = base_params(p, (float2*)state);
  P.amask = (1ull << (m - 1)) - 1ull;
  P.init = p.specialized ? INIT_COV_SPECIAL : INIT_COV_GENERIC;
  P.lut_z = (const u64*)p.d_lut_z;
  P.wgen = (const double2*)(w + L.off_weights);
  P.wspec = (const double2*)(w + L.off_weights);
  P.wspecf = (const float2*)(w + L.off_wspecf);
  P.outmask = outB;
  P.rg = (const float2*)p.d_rg;
  P.rh = (const float2*)p.d_rh;
  if (p.specialized) {
    P.tt_init = (const TileTables*)p.d_tt_init_shard;
    P.qsym_z = (const u64*)p.d_qsym_z;
  }
  P.tt_phase = (const TileTables*)p.d_tt_phase_shard;
  P.qsym_a = (const u64*)p.d_qsym_a;
  P.variant = p.variant;
  const float2* dg = p.rot_ok ? (const float2*)p.d_dg : nullptr;
  const float2* dh = p.rot_ok ? (const float2*)p.d_dh : nullptr;
  P.rot = p.rot_ok ? (const float2*)p.d_rot : nullptr;
  // Pass 0: every tile of the index space, this shard's half of each stored.
  P.c = kTileBits - 1;
  P.K = 1;
  P.q = m - 1;
  P.wht_mask = (1u << kTileBits) - 1u;
  P.store_top = shard;
  if ((rc = launch_pass(P, s))) return rc;
  P.store_top = -1;
  P.init = INIT_LOAD;
  // Later passes: tiles of 12 bits that never hold bit m - 1; this shard's half of them.
  const u64 half_tiles = 1ull << (m - kTileBits - 1);
  P.tile0 = (u64)shard * half_tiles;
  P.ntiles = half_tiles;
  const auto groups = shard_groups(m);
  const int k = (int)groups.size();
  for (int i = 0; i + 1 < k; ++i) {
    strided(P, groups[i].first, groups[i].second);
    P.wht_mask = target_mask(P);
    if ((rc = launch_pass(P, s))) return rc;
  }
  strided(P, groups[k - 1].first, groups[k - 1].second);
  P.wht_mask = target_mask(P);
  P.phase = 1;
  P.dg = dg;
  P.u_mask = product_mask(p, P, target_mask(P));
  if ((rc = launch_pass(P, s))) return rc;
  P.phase = 0;
  P.dg = nullptr;
  P.wht_mask = 0;
  for (int i = k - 2; i >= 0; --i) {
    strided(P, groups[i].first, groups[i].second);
    P.u_mask = product_mask(p, P, target_mask(P));
    if ((rc = launch_pass(P, s))) return rc;
  }
  contiguous(P, m);
  P.u_mask = product_mask(p, P, (1u << (kTileBits - 1)) - 1u);
  P.dh = dh;
  P.masses = (double*)(w + L.off_masses);
  return launch_pass(P, s);
}

int fourier_shard_mass(FourierPlan& p, void* ws, double* mass, cudaStream_t s) {
  if (!ws || !mass) return fail(RGS_ERR_ARG, "null workspace or output");
  FourierLayout L;
  fourier_layout(p, L);
  char* w = (char*)ws;
  double* d = (double*)(w + L.off_result);
  shard_mass_kernel<<<1, 1024, 0, s>>>((const double*)(w + L.off_masses), L.ntiles / 2, d);
  RGS_CUDA_TRY(cudaGetLastError());
  RGS_CUDA_TRY(cudaMemcpyAsync(mass, d, sizeof(double), cudaMemcpyDeviceToHost, s));
  RGS_CUDA_TRY(cudaStreamSynchronize(s));
  return RGS_OK;
}

int fourier_shard_draw(FourierPlan& p, const void* state, void* ws, double u1, double u2, uint64_t* local_index,
                       cudaStream_t s) {
  FourierLayout L;
  int rc = check_state(p, state, ws, (size_t)-1, L);
  if (rc) return rc;
  if (!local_index) return fail(RGS_ERR_ARG, "null output");
  if (!(u1 >= 0.0 && u1 < 1.0 && u2 >= 0.0 && u2 < 1.0)) return fail(RGS_ERR_ARG, "uniforms must lie in [0, 1)");
  char* w = (char*)ws;
  DrawResult* d = (DrawResult*)(w + L.off_result);
  fourier_draw_kernel<<<1, 1024, 0, s>>>((const double*)(w + L.off_masses), L.ntiles / 2, (const float2*)state,
                                         p.m - 1, kTileBits, 0, nullptr, u1, u2, 0.0, d);
  RGS_CUDA_TRY(cudaGetLastError());
  DrawResult h;
  RGS_CUDA_TRY(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  RGS_CUDA_TRY(cudaStreamSynchronize(s));
  if (h.status || !(h.norm > 0.0) || !std::isfinite(h.norm)) return fail(RGS_ERR_ZERO_NORM, "shard has no mass");
  *local_index = h.index;
  return RGS_OK;
}

int fourier_tune(FourierPlan& p, void* state, void* ws, size_t ws_bytes, cudaStream_t s, float* ms) {
  cudaEvent_t e0, e1;
  RGS_CUDA_TRY(cudaEventCreate(&e0));
  RGS_CUDA_TRY(cudaEventCreate(&e1));
  float best = 0.f;
  int chosen = 0;
  for (int v = 0; v < 2; ++v) {
    p.variant = v;
    int rc = fourier_compute(p, 0, state, ws, ws_bytes, s, nullptr);
    if (rc) return rc;
    RGS_CUDA_TRY(cudaEventRecord(e0, s));
    for (int r = 0; r < 2; ++r)
      if ((rc = fourier_compute(p, 0, state, ws, ws_bytes, s, nullptr))) return rc;
    RGS_CUDA_TRY(cudaEventRecord(e1, s));
    RGS_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    RGS_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    t *= 0.5f;
    if (ms) ms[v] = t;
    if (v == 0 || t < best) {
      best = t;
      chosen = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  p.variant = chosen;
  return RGS_OK;
}

int fourier_compute_permute(FourierPlan& p, uint64_t outB, void* state, void* scratch, void* ws, size_t ws_bytes,
                            cudaStream_t s) {
  FourierLayout L;
  int rc = check_state(p, state, ws, ws_bytes, L);
  if (rc) return rc;
  if (!scratch || ((uintptr_t)scratch & 15)) return fail(RGS_ERR_ARG, "bad scratch state");
  char* w = (char*)ws;
  rc = build_weights(p, outB, w, L, false, false, s);
  if (rc) return rc;
  const int m = p.m;
  PassParams P = base_params(p, (float2*)state);
  P.init = INIT_PRODUCT;
  P.lut_z = (const u64*)p.d_lut_z + (size_t)p.chunks * 256 * 2;  // q_B over b
  P.wgen = (const double2*)(w + L.off_weights);
  contiguous(P, m);
  P.wht_mask = (1u << P.c) - 1u;
  if ((rc = launch_pass(P, s))) return rc;
  P.init = INIT_LOAD;
  if (m > kTileBits && (rc = transform_range(P, m, kTileBits, m, true, s))) return rc;
  const u64 n = 1ull << m;
  const unsigned blocks = (unsigned)std::min<u64>((n + 255) / 256, (u64)sm_count(p.device) * 32);
  fourier_index_map_kernel<<<blocks, 256, 0, s>>>((const float2*)state, (float2*)scratch, m, p.chunks,
                                                  (const u64*)p.d_lut_cols, (const u64*)p.d_lut_a,
                                                  (float)std::exp2(-0.5 * m));
  RGS_CUDA_TRY(cudaGetLastError());
  PassParams Q = base_params(p, (float2*)scratch);
  // Products on all bits but the deferred terminal one, then the masses.
  const int top = p.deferred ? m - 1 : m;
  if (top > std::min(m, kTileBits) && (rc = transform_range(Q, m, std::min(m, kTileBits), top, false, s))) return rc;
  contiguous(Q, m);
  Q.u_mask = product_mask(p, Q, (1u << Q.c) - 1u);
  Q.masses = (double*)(w + L.off_masses);
  return launch_pass(Q, s);
}

int fourier_masses(FourierPlan& p, const void* state, void* ws, cudaStream_t s) {
  FourierLayout L;
  int rc = check_state(p, state, ws, (size_t)-1, L);
  if (rc) return rc;
  return block_mass(state, p.m, std::min(p.m, kTileBits), (double*)((char*)ws + L.off_masses), s);
}

int fourier_draw(FourierPlan& p, const void* state, void* ws, double u1, double u2, double u3, uint64_t* index,
                 double* pa, double* norm, cudaStream_t s) {
  FourierLayout L;
  int rc = check_state(p, state, ws, (size_t)-1, L);
  if (rc) return rc;
  if (!(u1 >= 0.0 && u1 < 1.0 && u2 >= 0.0 && u2 < 1.0 && u3 >= 0.0 && u3 < 1.0))
    return fail(RGS_ERR_ARG, "uniforms must lie in [0, 1)");
  char* w = (char*)ws;
  DrawResult* d = (DrawResult*)(w + L.off_result);
  fourier_draw_kernel<<<1, 1024, 0, s>>>((const double*)(w + L.off_masses), L.ntiles, (const float2*)state, p.m,
                                         std::min(p.m, kTileBits), p.deferred ? 1 : 0,
                                         (const double2*)p.d_uA + 4 * (p.m - 1), u1, u2, u3, d);
  RGS_CUDA_TRY(cudaGetLastError());
  DrawResult h;
  RGS_CUDA_TRY(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  RGS_CUDA_TRY(cudaStreamSynchronize(s));
  if (!std::isfinite(h.norm) || std::fabs(h.norm - 1.0) > 1e-3)
    return fail(RGS_ERR_ZERO_NORM, "conditional norm check failed: " + std::to_string(h.norm));
  if (h.status || !(h.pa > 0.0) || !std::isfinite(h.pa)) return fail(RGS_ERR_NONFINITE, "invalid drawn probability");
  *index = h.index;
  *pa = h.pa;
  *norm = h.norm;
  return RGS_OK;
}

int fourier_index_map(FourierPlan& p, const void* src, void* dst, cudaStream_t s) {
  if (!src || !dst || src == dst) return fail(RGS_ERR_ARG, "index map needs distinct source and destination");
  int device = 0;
  int rc = bind_device_of(dst, &device);
  if (rc) return rc;
  if ((rc = fourier_upload(p, device))) return rc;
  const u64 n = 1ull << p.m;
  const unsigned blocks = (unsigned)std::min<u64>((n + 255) / 256, (u64)sm_count(device) * 32);
  fourier_index_map_kernel<<<blocks, 256, 0, s>>>((const float2*)src, (float2*)dst, p.m, p.chunks,
                                                  (const u64*)p.d_lut_cols, (const u64*)p.d_lut_a,
                                                  (float)std::exp2(-0.5 * p.m));
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

int fourier_quadphase(FourierPlan& p, void* state, cudaStream_t s) {
  int device = 0;
  int rc = bind_device_of(state, &device);
  if (rc) return rc;
  if ((rc = fourier_upload(p, device))) return rc;
  PassParams P = base_params(p, (float2*)state);
  contiguous(P, p.m);
  P.phase = 1;
  return launch_pass(P, s);
}

int fwht_bits(void* state, int nbits, int lo, int hi, cudaStream_t s) {
  int device = 0;
  int rc = bind_device_of(state, &device);
  if (rc) return rc;
  PassParams P{};
  P.v = (float2*)state;
  P.amask = ~0ull;
  P.store_top = -1;
  P.store = 1;
  return transform_range(P, nbits, lo, hi, true, s);
}

int product_bits(void* state, int nbits, const double* u_dev, int lo, int hi, cudaStream_t s) {
  int device = 0;
  int rc = bind_device_of(state, &device);
  if (rc) return rc;
  if (!u_dev) return fail(RGS_ERR_ARG, "unitaries are required");
  PassParams P{};
  P.v = (float2*)state;
  P.amask = ~0ull;
  P.store_top = -1;
  P.store = 1;
  P.u = (const double2*)u_dev;
  return transform_range(P, nbits, lo, hi, false, s);
}

int block_mass(const void* state, int nbits, int tile_bits, double* masses, cudaStream_t s) {
  if (!state || !masses || nbits < 0 || nbits > 40 || tile_bits < 0 || tile_bits > nbits)
    return fail(RGS_ERR_ARG, "bad block-mass arguments");
  const u64 n = 1ull << nbits;
  const unsigned blocks = (unsigned)(n >> tile_bits);
  block_mass_kernel<<<blocks, 256, 0, s>>>((const float2*)state, n, tile_bits, masses);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

}  // namespace rgs
