// Device building blocks of the scan executor, shared by the streaming step
// kernel (one launch per scan position, tables in HBM), the shared-memory
// resident sweep and the chain-rule sampler.
//
// Table layout: complex entries interleaved over a batch tile of Bt = 2^lbt
// items, E[c][b] (b fastest).  A thread owns V consecutive items of one row, so a
// gather of row c is one 8- or 16-byte load per thread and lpr = Bt/V threads
// cover the row: 128-bit coalesced for complex64 with Bt >= 2.
#pragma once
#include <cuda_runtime.h>

#include "plan.hpp"

namespace rgs {

typedef unsigned long long u64;

template <typename M>
struct Cx {
  M re, im;
};

template <typename M>
__device__ __forceinline__ void cmad(Cx<M>& acc, M er, M ei, const Cx<M>& w) {
  acc.re += er * w.re - ei * w.im;
  acc.im += er * w.im + ei * w.re;
}

// Loads V complex values of row `row` at item offset b0.  S = storage real type.
template <typename S, int V>
struct RowIO;

template <>
struct RowIO<float, 1> {
  static __device__ __forceinline__ void load(const float* E, u64 idx, float (&re)[1], float (&im)[1]) {
    float2 x = __ldg(reinterpret_cast<const float2*>(E) + idx);
    re[0] = x.x;
    im[0] = x.y;
  }
  static __device__ __forceinline__ void store(float* E, u64 idx, const float (&re)[1], const float (&im)[1]) {
    reinterpret_cast<float2*>(E)[idx] = make_float2(re[0], im[0]);
  }
};
template <>
struct RowIO<float, 2> {
  static __device__ __forceinline__ void load(const float* E, u64 idx, float (&re)[2], float (&im)[2]) {
    float4 x = __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(E) + idx));
    re[0] = x.x;
    im[0] = x.y;
    re[1] = x.z;
    im[1] = x.w;
  }
  static __device__ __forceinline__ void store(float* E, u64 idx, const float (&re)[2], const float (&im)[2]) {
    *reinterpret_cast<float4*>(reinterpret_cast<float2*>(E) + idx) = make_float4(re[0], im[0], re[1], im[1]);
  }
};
template <>
struct RowIO<double, 1> {
  static __device__ __forceinline__ void load(const double* E, u64 idx, double (&re)[1], double (&im)[1]) {
    double2 x = __ldg(reinterpret_cast<const double2*>(E) + idx);
    re[0] = x.x;
    im[0] = x.y;
  }
  static __device__ __forceinline__ void store(double* E, u64 idx, const double (&re)[1], const double (&im)[1]) {
    reinterpret_cast<double2*>(E)[idx] = make_double2(re[0], im[0]);
  }
};

// Generic-address variants (shared or global) without the read-only cache hint.
template <typename S, int V>
struct RowIOGeneric;
template <>
struct RowIOGeneric<float, 1> {
  static __device__ __forceinline__ void load(const float* E, u64 idx, float (&re)[1], float (&im)[1]) {
    float2 x = reinterpret_cast<const float2*>(E)[idx];
    re[0] = x.x;
    im[0] = x.y;
  }
  static __device__ __forceinline__ void store(float* E, u64 idx, const float (&re)[1], const float (&im)[1]) {
    reinterpret_cast<float2*>(E)[idx] = make_float2(re[0], im[0]);
  }
};
template <>
struct RowIOGeneric<float, 2> {
  static __device__ __forceinline__ void load(const float* E, u64 idx, float (&re)[2], float (&im)[2]) {
    float4 x = *reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(E) + idx);
    re[0] = x.x;
    im[0] = x.y;
    re[1] = x.z;
    im[1] = x.w;
  }
  static __device__ __forceinline__ void store(float* E, u64 idx, const float (&re)[2], const float (&im)[2]) {
    *reinterpret_cast<float4*>(reinterpret_cast<float2*>(E) + idx) = make_float4(re[0], im[0], re[1], im[1]);
  }
};
template <>
struct RowIOGeneric<double, 1> {
  static __device__ __forceinline__ void load(const double* E, u64 idx, double (&re)[1], double (&im)[1]) {
    double2 x = reinterpret_cast<const double2*>(E)[idx];
    re[0] = x.x;
    im[0] = x.y;
  }
  static __device__ __forceinline__ void store(double* E, u64 idx, const double (&re)[1], const double (&im)[1]) {
    reinterpret_cast<double2*>(E)[idx] = make_double2(re[0], im[0]);
  }
};

// p0 = L c' by XOR of byte tables (scan_plan.py:133-145, gpu_kernel.py:73-75).
__device__ __forceinline__ u64 table_lookup(const u64* __restrict__ T, int nbytes, u64 c) {
  u64 p = 0;
  for (int b = 0; b < nbytes; ++b) p ^= __ldg(T + (b << 8) + ((c >> (8 * b)) & 255ull));
  return p;
}

// Inserts a zero bit at position pi of i.
__device__ __forceinline__ u64 deposit_zero(u64 i, int pi) {
  const u64 low = (1ull << pi) - 1ull;
  return ((i & ~low) << 1) | (i & low);
}

// Power-of-two scale for the next step from the previous maximum |E|^2, exactly as
// GPUMixin._sweep (gpu_kernel.py:146-148): m = sqrt(max|E|^2), m = f 2^e with
// f in [0.5, 1), scale = 2^-e.  Returns e; m2 = 1 for the first step.
__device__ __forceinline__ int scale_exponent(double m2) {
  int e = 0;
  frexp(sqrt(m2), &e);
  return e;
}

// Maximum-slot encoding: non-negative floats (complex64 tables) or doubles
// (complex128 tables) as their IEEE bits, so unsigned max is float max.
template <typename S>
__device__ __forceinline__ u64 max_bits(S x);
template <>
__device__ __forceinline__ u64 max_bits<float>(float x) {
  return (u64)__float_as_uint(x);
}
template <>
__device__ __forceinline__ u64 max_bits<double>(double x) {
  return (u64)__double_as_longlong(x);
}
template <typename S>
__device__ __forceinline__ double max_value(u64 bits);
template <>
__device__ __forceinline__ double max_value<float>(u64 bits) {
  return (double)__uint_as_float((unsigned)bits);
}
template <>
__device__ __forceinline__ double max_value<double>(u64 bits) {
  return __longlong_as_double((long long)bits);
}

// Per-thread weights of one scan position for its V items: f(0), f(1) scaled by
// 2^-e, plus the fixed-vertex value y and the syndrome-offset bit ov.
template <typename M, int V>
struct StepWeights {
  Cx<M> w0[V], w1[V];
  int y[V], ov[V];
};

// One output pair / output of a step (see StepMode).  Returns the values; the
// caller stores them.  E is addressed through IO (global or shared).
template <typename S, typename M, int V, int MODE, class IO>
__device__ __forceinline__ void step_item(const S* __restrict__ E, const DevStep& st, const u64* __restrict__ T,
                                          const StepWeights<M, V>& w, u64 item, int lbt, int b0, bool unit_input,
                                          u64& ca, u64& cb, Cx<M> (&oa)[V], Cx<M> (&ob)[V]) {
  const u64 mask = (1ull << st.r_in) - 1ull;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    oa[v].re = oa[v].im = ob[v].re = ob[v].im = (M)0;
  }
  if (MODE == MODE_PAIR) {
    ca = deposit_zero(item, st.pi);
    cb = ca ^ st.t;
  } else {
    ca = item;
    cb = item;
  }
  const u64 p0 = table_lookup(T, st.nbytes, ca);
  // Issue every gather first (at most four rows), then the arithmetic.
  S er[4][V], ei[4][V];
  u64 pk[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    pk[k] = p0 ^ st.combos[k];
    if (k < st.ncombos) {
      const u64 c = pk[k] & mask;
      if (unit_input) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
          er[k][v] = (S)1;
          ei[k][v] = (S)0;
        }
      } else {
        IO::load(E, (c << lbt) + (u64)b0, er[k], ei[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= st.ncombos) break;
    const u64 c = pk[k] & mask;
    const int pc = __popcll(c & st.beta) & 1;
    if (MODE == MODE_PAIR) {
      const int y = (int)((pk[k] >> st.r_in) & 1ull);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int par = pc ^ w.ov[v];
        Cx<M> wa = y ? w.w1[v] : w.w0[v];
        Cx<M> wb = y ? w.w0[v] : w.w1[v];
        if (y & par) {
          wa.re = -wa.re;
          wa.im = -wa.im;
        }
        if ((y ^ 1) & par) {
          wb.re = -wb.re;
          wb.im = -wb.im;
        }
        cmad(oa[v], (M)er[k][v], (M)ei[k][v], wa);
        cmad(ob[v], (M)er[k][v], (M)ei[k][v], wb);
      }
    } else if (MODE == MODE_MERGE) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int par = pc ^ w.ov[v];
        Cx<M> ww;
        ww.re = par ? w.w0[v].re - w.w1[v].re : w.w0[v].re + w.w1[v].re;
        ww.im = par ? w.w0[v].im - w.w1[v].im : w.w0[v].im + w.w1[v].im;
        cmad(oa[v], (M)er[k][v], (M)ei[k][v], ww);
      }
    } else {  // MODE_FIXED
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int par = pc ^ w.ov[v];
        Cx<M> ww = w.y[v] ? w.w1[v] : w.w0[v];
        if (w.y[v] & par) {
          ww.re = -ww.re;
          ww.im = -ww.im;
        }
        cmad(oa[v], (M)er[k][v], (M)ei[k][v], ww);
      }
    }
  }
}

}  // namespace rgs
