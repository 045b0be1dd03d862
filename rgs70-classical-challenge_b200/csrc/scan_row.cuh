// Streaming scan-step kernel: one scan position over a batch tile (or, along grid.y,
// several tiles whose tables lie e_stride entries apart), rows of the interleaved table
// handled by (sub-)warps.
//
// A row of Bt items is 2^lC chunks of 16 bytes.  L = min(32, 2^lC) lanes share a row
// and each lane owns CPL chunks (CPL = 2^lC / L), so the row's gather index (byte-table
// lookups, parities) is computed once per lane for CPL chunks instead of once per
// chunk; a warp holds 32/L rows at a time, U of them per lane per iteration, so each
// lane keeps U * NC * CPL (= 8 where possible) independent 16-byte loads in flight.
//
// Modes (see plan.hpp): PAIR writes rows c' and c'^t from the same NC gathered rows;
// MERGE and FIXED write one row.  The per-item weight pair (wA, wB) is prepared per
// mode so that the inner loop is a complex FMA:
//   PAIR : wA = f(0) s, wB = f(1) s       row c'  : y ? wB : wA, negated iff y & par
//                                          row c'^t: y ? wA : wB, negated iff !y & par
//   MERGE: wA = (f0 + f1) s, wB = (f0 - f1) s        par ? wB : wA
//   FIXED: wA = f(y) s                              negated iff y & par
// with par = popc(c & beta) ^ ov and s = 2^-e the renormalisation of gpu_kernel.py:146-148.
//
// PAIR without per-item selects.  The y bit of gather k is y_k = y(p0) ^ kappa_k, where
// kappa_k is bit r_in of combo k, a constant of the step; the compiler orders the combos
// with kappa = 0 first (NG0 of them).  With X = sum_{k<NG0} e wA + sum_{k>=NG0} (-1)^par e wB
// and Y = sum_{k<NG0} (-1)^par e wB + sum_{k>=NG0} e wA, row c' receives X and row c'^t
// receives Y when y(p0) = 0, and the other way round when y(p0) = 1: the choice is one
// swap of the two store addresses per row, and the sign is applied to the gathered value
// (exactly the negated product), so no weight is selected per item.
#pragma once
#include "scan_device.cuh"

namespace rgs {

// Rows per lane per iteration: LOADS 16-byte gathers in flight per lane (eight; four
// when float64 arithmetic on complex64 tables needs the registers).
template <int NC, int CPL, int LOADS>
struct RowsPerIter {
  static constexpr int value = (NC * CPL >= LOADS) ? 1 : LOADS / (NC * CPL);
};
template <typename S, typename M>
struct LoadsInFlight {
  static constexpr int value = sizeof(M) > sizeof(S) ? 4 : 8;
};
// Chunks of a row a lane gathers at once: all CPL of them up to two (complex128 or
// float64 arithmetic) or four (float32 arithmetic) -- longer rows are walked in groups,
// with the row's index work still done once per lane.
template <typename S, typename M, int CPL>
struct ChunkGroup {
  static constexpr int cap = (sizeof(S) == 8 || sizeof(M) == 8) ? 2 : 4;
  static constexpr int value = CPL < cap ? CPL : cap;
};

template <typename S, typename M, int VE, int MODE, int NC, int CPL, int NG0>
__global__ void __launch_bounds__(256, 2) scan_row_kernel(const S* __restrict__ Ein, S* __restrict__ Eout,
                                                       const __grid_constant__ DevStep st,
                                                       const u64* __restrict__ T, const double4* __restrict__ W,
                                                       const unsigned char* __restrict__ F,
                                                       const u64* __restrict__ maxprev, u64* __restrict__ maxcur,
                                                       int lbt, int unit_input, u64 e_stride) {
  constexpr int CPLG = ChunkGroup<S, M, CPL>::value;
  constexpr int U = RowsPerIter<NC, CPLG, LoadsInFlight<S, M>::value>::value;
  constexpr int NI = CPL * VE;             // items owned by a lane
  __shared__ u64 smax[256];
  const int Bt = 1 << lbt;
  const int lC = lbt - (VE == 2 ? 1 : 0);  // log2 chunks per row
  const int lL = lC < 5 ? lC : 5;          // log2 lanes per row
  const int lR = 5 - lL;                   // log2 rows per warp
  const int lane = threadIdx.x & 31;
  const int sub = lane >> lL;
  const int l = lane & ((1 << lL) - 1);

  // Several tiles in one launch (grid.y): tile k's table starts k * e_stride entries in,
  // its weights, flags and maxima k * Bt items in.
  if (blockIdx.y) {
    const u64 k = blockIdx.y;
    Ein += 2 * k * e_stride;
    Eout += 2 * k * e_stride;
    W += k << lbt;
    if (F) F += k << lbt;
    if (maxprev) maxprev += k << lbt;
    maxcur += k << lbt;
  }
  for (int i = threadIdx.x; i < Bt; i += blockDim.x) smax[i] = 0;

  Cx<M> wA[NI], wB[NI];
  int ov[NI], yf[NI];
#pragma unroll
  for (int k = 0; k < CPL; ++k) {
#pragma unroll
    for (int v = 0; v < VE; ++v) {
      const int i = k * VE + v;
      const int b = ((l + (k << lL)) * VE) + v;
      const double m2 = maxprev ? max_value<S>(maxprev[b]) : 1.0;
      const double s = ldexp(1.0, -scale_exponent(m2));
      const double4 f = W[b];
      const int fl = F ? F[b] : 0;
      yf[i] = fl & 1;
      ov[i] = (fl >> 1) & 1;
      double ar = f.x * s, ai = f.y * s, br = f.z * s, bi = f.w * s;
      if (MODE == MODE_MERGE) {
        const double pr = ar + br, pi = ai + bi, mr = ar - br, mi = ai - bi;
        ar = pr;
        ai = pi;
        br = mr;
        bi = mi;
      } else if (MODE == MODE_FIXED) {
        if (yf[i]) {
          ar = br;
          ai = bi;
        }
      }
      wA[i].re = (M)ar;
      wA[i].im = (M)ai;
      wB[i].re = (M)br;
      wB[i].im = (M)bi;
    }
  }
  __syncthreads();

  const u64 items = (MODE == MODE_PAIR) ? (1ull << (st.r_out - 1)) : (1ull << st.r_out);
  const u64 warp = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u64 per_iter = (u64)U << lR;  // rows per warp per iteration
  const u64 mask = (1ull << st.r_in) - 1ull;
  S mx[NI];
#pragma unroll
  for (int i = 0; i < NI; ++i) mx[i] = (S)0;

  for (u64 base = warp * per_iter; base < items; base += nwarps * per_iter) {
    u64 ca[U], cb[U];
    u64 cc[U][NC];
    int pc[U][NC];
    bool ok[U];
    Chunk<S, VE> e[U][NC][CPLG];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 it = base + ((u64)u << lR) + sub;
      ok[u] = it < items;
      if (MODE == MODE_PAIR) {
        ca[u] = deposit_zero(it, st.pi);
        cb[u] = ca[u] ^ st.t;
      } else {
        ca[u] = it;
        cb[u] = it;
      }
      const u64 p0 = ok[u] ? table_lookup(T, st.nbytes, ca[u]) : 0ull;
      if (MODE == MODE_PAIR && ((p0 >> st.r_in) & 1ull)) {  // y(p0) = 1: swap the two output rows
        const u64 tmp = ca[u];
        ca[u] = cb[u];
        cb[u] = tmp;
      }
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const u64 p = p0 ^ st.combos[k];
        cc[u][k] = p & mask;
        pc[u][k] = __popcll(cc[u][k] & st.beta) & 1;
      }
    }
#pragma unroll
    for (int g = 0; g < CPL; g += CPLG) {
      // All gathers of this chunk group before any arithmetic.
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int k = 0; k < NC; ++k) {
#pragma unroll
          for (int jj = 0; jj < CPLG; ++jj) {
            if (unit_input || !ok[u])
              e[u][k][jj].unit();
            else
              e[u][k][jj].load(Ein, (cc[u][k] << lC) + (u64)(l + ((g + jj) << lL)));
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
#pragma unroll
        for (int jj = 0; jj < CPLG; ++jj) {
          const int j = g + jj;
          Chunk<S, VE> outA, outB;
#pragma unroll
          for (int v = 0; v < VE; ++v) {
            const int i = j * VE + v;
            Cx<M> oa{(M)0, (M)0}, ob{(M)0, (M)0};
#pragma unroll
            for (int k = 0; k < NC; ++k) {
              const int par = pc[u][k] ^ ov[i];
              if (MODE == MODE_PAIR) {
                const M pr = (M)e[u][k][jj].re(v), pi = (M)e[u][k][jj].im(v);
                const M nr = flip_sign(pr, par), ni = flip_sign(pi, par);
                if (k < NG0) {
                  cmad(oa, pr, pi, wA[i]);
                  cmad(ob, nr, ni, wB[i]);
                } else {
                  cmad(oa, nr, ni, wB[i]);
                  cmad(ob, pr, pi, wA[i]);
                }
              } else if (MODE == MODE_MERGE) {
                const M er = (M)e[u][k][jj].re(v), ei = (M)e[u][k][jj].im(v);
                cmad(oa, er, ei, par ? wB[i] : wA[i]);
              } else {
                const M er = (M)e[u][k][jj].re(v), ei = (M)e[u][k][jj].im(v);
                Cx<M> w = wA[i];
                if (yf[i] & par) {
                  w.re = -w.re;
                  w.im = -w.im;
                }
                cmad(oa, er, ei, w);
              }
            }
            const S ar = (S)oa.re, ai = (S)oa.im;
            outA.set(v, ar, ai);
            mx[i] = fmax(mx[i], norm2(ar, ai));
            if (MODE == MODE_PAIR) {
              const S br = (S)ob.re, bi = (S)ob.im;
              outB.set(v, br, bi);
              mx[i] = fmax(mx[i], norm2(br, bi));
            }
          }
          const u64 col = (u64)(l + (j << lL));
          outA.store(Eout, (ca[u] << lC) + col);
          if (MODE == MODE_PAIR) outB.store(Eout, (cb[u] << lC) + col);
        }
      }
    }
  }

  // Maximum |E|^2 per item: lanes owning the same items (same l, other rows of the
  // warp), then shared memory, then one global atomicMax per item per block
  // (gpu_kernel.py:98-101).
#pragma unroll
  for (int k = 0; k < CPL; ++k) {
#pragma unroll
    for (int v = 0; v < VE; ++v) {
      const int i = k * VE + v;
      u64 bits = max_bits<S>(mx[i]);
      for (int off = 16; off >= (1 << lL); off >>= 1) {
        const u64 o = __shfl_xor_sync(0xffffffffu, bits, off);
        bits = bits > o ? bits : o;
      }
      if (sub == 0 && bits) atomicMax(&smax[((l + (k << lL)) * VE) + v], bits);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Bt; i += blockDim.x)
    if (smax[i]) atomicMax(&maxcur[i], smax[i]);
}

}  // namespace rgs
