// Fused pair kernel: scan positions A = j and B = j + 1 in one pass over HBM.
//
// The unfused sweep writes A's output table and reads it back for B.  Here a warp (or a
// sub-warp, for rows shorter than 32 chunks) takes one group of rows at a time (DevPair,
// plan.hpp): the group's input rows of A are gathered once, A's outputs for the group
// (the |W| intermediate rows, at most 8) are formed in registers and rounded to the
// storage type exactly as the unfused step stores them, and B's outputs of the group are
// formed from those registers and stored.  Every intermediate row belongs to exactly
// one group, so each input entry is read once and each output entry written once; the
// intermediate table never reaches memory.
//
// Renormalisation.  A is scaled by 2^-e from the previous maximum as usual; B runs
// unscaled (the scale of an intermediate table is not known until the whole table
// exists) and the pass records max |E|^2 = 1/4 for A, whose exponent is 0, so the
// finalisation's sum of exponents stays exact; B's maximum is recorded as usual and
// scales the position after B.  A value therefore differs from the unfused sweep's by an
// exact power of two in (value, logscale), not in the amplitude value * 2^logscale.
//
// Lanes: a lane owns one 16-byte chunk column of every row it touches (VE items);
// rows of more than 32 chunks are split into 32-chunk column slices, one slice per
// warp (the grid's warp count is a multiple of the slice count).
#pragma once
#include "scan_device.cuh"

namespace rgs {

template <int C>
struct PairMode {
  static constexpr bool pair = C != PC_M2;
  static constexpr int nc = C == PC_P1 ? 1 : (C == PC_P4H ? 4 : 2);
  static constexpr int ng0 = C == PC_P1 ? 1 : (C == PC_P2H ? 1 : (C == PC_P2F ? 2 : (C == PC_P4H ? 2 : 2)));
};

// Group index and chunk offset arithmetic in the index type I: 32-bit where every rank
// of the pair plus log2(chunks per row) is at most 31 (fewer instructions per group),
// 64-bit otherwise.
template <typename I>
__device__ __forceinline__ int parity_of(I x);
template <>
__device__ __forceinline__ int parity_of<unsigned>(unsigned x) {
  return __popc(x) & 1;
}
template <>
__device__ __forceinline__ int parity_of<u64>(u64 x) {
  return __popcll(x) & 1;
}

// Both maps of a group from the interleaved byte tables (the XOR of one entry per byte
// of c): p = L_A c, q = M_B (c | 0).
template <typename I>
__device__ __forceinline__ void lookup2_as(const u64* __restrict__ T2, int nbytes, I c, I& p, I& q) {
  p = 0;
  q = 0;
  for (int b = 0; b < nbytes; ++b) {
    const ulonglong2 t = __ldg(reinterpret_cast<const ulonglong2*>(T2) + (b << 8) + (int)((c >> (8 * b)) & (I)255));
    p ^= (I)t.x;
    q ^= (I)t.y;
  }
}

// Group representative q0: the group index with zeros inserted at W's pivots.
template <typename I>
__device__ __forceinline__ I deposit_pivots(I it, const DevPair& P) {
  I q = it;
  for (int k = 0; k < P.dw; ++k) {
    const I low = ((I)1 << P.piv[k]) - (I)1;
    q = ((q & ~low) << 1) | (q & low);
  }
  return q;
}

// Resident 256-thread blocks per SM: RGS_PAIR_MINB (scan_device.cuh) where the registers
// suffice; one for float64 arithmetic on complex64 tables, whose conversions need more.
template <typename S, typename M>
struct PairBlocks {
  static constexpr int value = sizeof(M) > sizeof(S) ? 1 : RGS_PAIR_MINB;
};

// GRAM = true (chain-rule sampling, the first of two passes over a pair): instead of B's
// outputs, the 2x2 Gram matrix of B's branch masses per item (see chain.cu) from the
// group's intermediate rows, nothing stored; per-block partials (G00, G11, Re G01,
// Im G01) of every item go to partial[block][item][4] (dynamic shared memory: 8 warps x
// Bt x 4 doubles).  B's weights are not read.
template <typename S, typename M, int VE, int CA, int CB, typename I, bool GRAM = false>
__global__ void __launch_bounds__(256, PairBlocks<S, M>::value)
    scan_pair_kernel(const S* __restrict__ Ein, S* __restrict__ Eout, const __grid_constant__ DevPair P,
                     const u64* __restrict__ tables, const double4* __restrict__ WA, const double4* __restrict__ WB,
                     const u64* __restrict__ maxprev, u64* __restrict__ maxA, u64* __restrict__ maxcur, int lbt,
                     u64 e_stride, double* __restrict__ partial) {
  using MA = PairMode<CA>;
  using MB = PairMode<CB>;
  constexpr int NCA = MA::nc, NCB = MB::nc;
  constexpr int NW = MA::pair ? 2 * NCB : NCB;  // intermediate rows per group
  constexpr int NUA = NCB;                      // A units: register pairs (PAIR A) or registers
  constexpr int NUB = MA::pair ? 2 : 1;         // B units
  constexpr int LOADS = NUA * NCA;
  constexpr int U = LOADS >= RGS_PAIR_LOADS ? 1 : RGS_PAIR_LOADS / LOADS;  // groups per lane per iteration
  __shared__ u64 smax[256];
  // Group maps of the low bits of a group index (see the loop below), per block.
  __shared__ I s_low[256][2];
  __shared__ unsigned char s_lowpar[256];
  const int Bt = 1 << lbt;
  const int lC = lbt - (VE == 2 ? 1 : 0);  // log2 chunks per row
  const int lL = lC < 5 ? lC : 5;          // log2 lanes per row
  const int lR = 5 - lL;                   // log2 groups side by side in a warp
  const int lS = lC - lL;                  // log2 column slices per row
  const int lane = threadIdx.x & 31;
  const int sub = lane >> lL;
  const int l = lane & ((1 << lL) - 1);

  if (blockIdx.y) {  // tile k of a chunk of tiles
    const u64 k = blockIdx.y;
    Ein += 2 * k * e_stride;
    Eout += 2 * k * e_stride;
    WA += k << lbt;
    WB += k << lbt;
    maxprev += k << lbt;
    maxA += k << lbt;
    maxcur += k << lbt;
  }
  if (!GRAM) {
    for (int i = threadIdx.x; i < Bt; i += blockDim.x) smax[i] = 0;
    if (blockIdx.x == 0)
      for (int i = threadIdx.x; i < Bt; i += blockDim.x) maxA[i] = max_bits<S>((S)0.25);
  }

  const u64 gwarp = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u64 slice = gwarp & ((1ull << lS) - 1ull);
  const u64 col = (slice << 5) + (u64)l;  // this lane's chunk column

  Cx<M> wAa[VE], wAb[VE], wBa[VE], wBb[VE];
#pragma unroll
  for (int v = 0; v < VE; ++v) {
    const int b = (int)(col * VE) + v;
    const double s = ldexp(1.0, -scale_exponent(max_value<S>(maxprev[b])));
    const double4 fa = WA[b], fb = GRAM ? WA[b] : WB[b];
    double ar = fa.x * s, ai = fa.y * s, br = fa.z * s, bi = fa.w * s;
    if (!MA::pair) {
      const double pr = ar + br, pi = ai + bi, mr = ar - br, mi = ai - bi;
      ar = pr, ai = pi, br = mr, bi = mi;
    }
    wAa[v] = Cx<M>{(M)ar, (M)ai};
    wAb[v] = Cx<M>{(M)br, (M)bi};
    double cr = fb.x, ci = fb.y, dr = fb.z, di = fb.w;
    if (!MB::pair) {
      const double pr = cr + dr, pi = ci + di, mr = cr - dr, mi = ci - di;
      cr = pr, ci = pi, dr = mr, di = mi;
    }
    wBa[v] = Cx<M>{(M)cr, (M)ci};
    wBb[v] = Cx<M>{(M)dr, (M)di};
  }
  __syncthreads();

  const u64* T2 = tables + P.tab2_off;
  const I maskA = (I)P.maskA, betaA = (I)P.betaA, betaB = (I)P.betaB;
  const u64 groups = 1ull << (P.m - P.dw);
  const u64 per_iter = (u64)U << lR;
  const u64 wslice = nwarps >> lS;  // warps per column slice
  S mx[VE];
  double gacc[VE][4];  // GRAM: Gram partials per item
#pragma unroll
  for (int v = 0; v < VE; ++v) {
    mx[v] = (S)0;
    gacc[v][0] = gacc[v][1] = gacc[v][2] = gacc[v][3] = 0.0;
  }
  // A warp iteration takes the groups base | idx, idx < per_iter (base a multiple of
  // per_iter).  q0 (zeros deposited at W's pivots), both table maps and the parity of
  // q0 & beta_B are GF(2)-linear in the group index, so the part of idx comes from this
  // block table and only base needs the byte-table lookups, once per iteration.
  for (int i = threadIdx.x; i < (int)per_iter; i += blockDim.x) {
    const I q = deposit_pivots<I>((I)i, P);
    I pl = 0, cl = 0;
    lookup2_as<I>(T2, P.nbMB, q, pl, cl);
    s_low[i][0] = pl;
    s_low[i][1] = cl;
    s_lowpar[i] = (unsigned char)parity_of<I>(q & betaB);
  }
  __syncthreads();

  for (u64 base = (gwarp >> lS) * per_iter; base < groups; base += wslice * per_iter) {
    bool ok[U];
    I c0[U];
    int pq[U], ya[U][NUA], pa[U][NUA][NCA];
    Chunk<S, VE> e[U][NUA][NCA];
    const I qb = deposit_pivots<I>((I)base, P);
    I pb = 0, cb = 0;
    lookup2_as<I>(T2, P.nbMB, qb, pb, cb);
    const int pqb = parity_of<I>(qb & betaB);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = (u << lR) + sub;
      ok[u] = base + (u64)idx < groups;
      const I p0 = pb ^ s_low[idx][0];
      c0[u] = cb ^ s_low[idx][1];
      pq[u] = pqb ^ (int)s_lowpar[idx];
#pragma unroll
      for (int a = 0; a < NUA; ++a) {
        const I pu = p0 ^ (I)P.LAw[a];
        ya[u][a] = (int)((pu >> P.a) & (I)1);
#pragma unroll
        for (int k = 0; k < NCA; ++k) {
          const I row = (pu ^ (I)P.combA[k]) & maskA;
          pa[u][a][k] = parity_of<I>(row & betaA);
          if (ok[u]) e[u][a][k].load(Ein, (u64)(((I)row << lC) | (I)col));
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!ok[u]) continue;
      Chunk<S, VE> outX[NUB], outY[NUB];
#pragma unroll
      for (int v = 0; v < VE; ++v) {
        S ir[NW], ii[NW];
        // A: the group's intermediate rows, rounded to the storage type.
#pragma unroll
        for (int a = 0; a < NUA; ++a) {
          if (MA::pair) {
            Cx<M> x{(M)0, (M)0}, y{(M)0, (M)0};
#pragma unroll
            for (int k = 0; k < NCA; ++k) {
              const M er = (M)e[u][a][k].re(v), ei = (M)e[u][a][k].im(v);
              const M nr = flip_sign(er, pa[u][a][k]), ni = flip_sign(ei, pa[u][a][k]);
              if (k < MA::ng0) {
                cmad(x, er, ei, wAa[v]);
                cmad(y, nr, ni, wAb[v]);
              } else {
                cmad(x, nr, ni, wAb[v]);
                cmad(y, er, ei, wAa[v]);
              }
            }
            const S xr = (S)x.re, xi = (S)x.im, yr = (S)y.re, yi = (S)y.im;
            const bool sw = ya[u][a];
            ir[2 * a] = sw ? yr : xr;
            ii[2 * a] = sw ? yi : xi;
            ir[2 * a + 1] = sw ? xr : yr;
            ii[2 * a + 1] = sw ? xi : yi;
          } else {
            Cx<M> x{(M)0, (M)0};
#pragma unroll
            for (int k = 0; k < NCA; ++k)
              cmad(x, (M)e[u][a][k].re(v), (M)e[u][a][k].im(v), pa[u][a][k] ? wAb[v] : wAa[v]);
            ir[a] = (S)x.re;
            ii[a] = (S)x.im;
          }
        }
        if constexpr (GRAM) {
          // Every output of B is alpha f(0) + beta f(1): PAIR B, output X: alpha = the
          // kappa-0 rows, beta = the others with their signs, output Y the mirror image;
          // MERGE B: alpha = all rows, beta = all rows with their signs.
#pragma unroll
          for (int b = 0; b < NUB; ++b) {
            double axr = 0.0, axi = 0.0, bxr = 0.0, bxi = 0.0, ayr = 0.0, ayi = 0.0, byr = 0.0, byi = 0.0;
#pragma unroll
            for (int a = 0; a < NCB; ++a) {
              const int i = MA::pair ? (a << 1) | b : a;
              const int par = pq[u] ^ (int)((P.pwB >> i) & 1u);
              const double er = (double)ir[i], ei = (double)ii[i];
              const double nr = par ? -er : er, ni = par ? -ei : ei;
              if (MB::pair) {
                if (a < MB::ng0) {
                  axr += er, axi += ei, byr += nr, byi += ni;
                } else {
                  bxr += nr, bxi += ni, ayr += er, ayi += ei;
                }
              } else {
                axr += er, axi += ei, bxr += nr, bxi += ni;
              }
            }
            gacc[v][0] = fma(axr, axr, fma(axi, axi, gacc[v][0]));
            gacc[v][1] = fma(bxr, bxr, fma(bxi, bxi, gacc[v][1]));
            gacc[v][2] = fma(axr, bxr, fma(axi, bxi, gacc[v][2]));
            gacc[v][3] = fma(axi, bxr, fma(-axr, bxi, gacc[v][3]));
            if (MB::pair) {
              gacc[v][0] = fma(ayr, ayr, fma(ayi, ayi, gacc[v][0]));
              gacc[v][1] = fma(byr, byr, fma(byi, byi, gacc[v][1]));
              gacc[v][2] = fma(ayr, byr, fma(ayi, byi, gacc[v][2]));
              gacc[v][3] = fma(ayi, byr, fma(-ayr, byi, gacc[v][3]));
            }
          }
          continue;
        }
        // B: the group's output rows from the registers.
#pragma unroll
        for (int b = 0; b < NUB; ++b) {
          Cx<M> x{(M)0, (M)0}, y{(M)0, (M)0};
#pragma unroll
          for (int a = 0; a < NCB; ++a) {
            const int i = MA::pair ? (a << 1) | b : a;
            const int par = pq[u] ^ (int)((P.pwB >> i) & 1u);
            const M er = (M)ir[i], ei = (M)ii[i];
            if (MB::pair) {
              const M nr = flip_sign(er, par), ni = flip_sign(ei, par);
              if (a < MB::ng0) {
                cmad(x, er, ei, wBa[v]);
                cmad(y, nr, ni, wBb[v]);
              } else {
                cmad(x, nr, ni, wBb[v]);
                cmad(y, er, ei, wBa[v]);
              }
            } else {
              cmad(x, er, ei, par ? wBb[v] : wBa[v]);
            }
          }
          const S xr = (S)x.re, xi = (S)x.im;
          outX[b].set(v, xr, xi);
          mx[v] = fmax(mx[v], norm2(xr, xi));
          if (MB::pair) {
            const S yr = (S)y.re, yi = (S)y.im;
            outY[b].set(v, yr, yi);
            mx[v] = fmax(mx[v], norm2(yr, yi));
          }
        }
      }
      if (!GRAM) {
#pragma unroll
        for (int b = 0; b < NUB; ++b) {
          const I cx = c0[u] ^ (I)P.MB0[b];
          outX[b].store(Eout, (u64)(((I)cx << lC) | (I)col));
          if (MB::pair) outY[b].store(Eout, (u64)(((I)(cx ^ (I)P.tB) << lC) | (I)col));
        }
      }
    }
  }

  if constexpr (GRAM) {
    // Deterministic reduction: lanes of other groups that own the same column
    // (shuffles), warps (shared memory, fixed order), one partial per block and item.
    extern __shared__ double red[];  // [8 warps][Bt][4]
    const int wib = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < VE; ++v)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double a = gacc[v][q];
        for (int off = 16; off >= (1 << lL); off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
        gacc[v][q] = a;
      }
    for (int i = threadIdx.x; i < 8 * Bt * 4; i += blockDim.x) red[i] = 0.0;
    __syncthreads();
    if (sub == 0)
#pragma unroll
      for (int v = 0; v < VE; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) red[((size_t)wib * Bt + (int)(col * VE) + v) * 4 + q] = gacc[v][q];
    __syncthreads();
    for (int b = threadIdx.x; b < Bt; b += blockDim.x)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double t = 0.0;
        for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) t += red[((size_t)wv * Bt + b) * 4 + q];
        partial[((size_t)blockIdx.x * Bt + b) * 4 + q] = t;
      }
    return;
  }

  // Maximum |E|^2 of B's outputs per item: lanes of other groups in the warp that own
  // the same column, then shared memory, then one global atomicMax per item per block.
#pragma unroll
  for (int v = 0; v < VE; ++v) {
    u64 bits = max_bits<S>(mx[v]);
    for (int off = 16; off >= (1 << lL); off >>= 1) {
      const u64 o = __shfl_xor_sync(0xffffffffu, bits, off);
      bits = bits > o ? bits : o;
    }
    if (sub == 0 && bits) atomicMax(&smax[(int)(col * VE) + v], bits);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Bt; i += blockDim.x)
    if (smax[i]) atomicMax(&maxcur[i], smax[i]);
}

}  // namespace rgs
