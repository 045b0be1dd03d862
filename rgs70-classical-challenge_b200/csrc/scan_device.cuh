// Device building blocks of the scan executor, shared by the streaming step
// kernel (one launch per scan position, tables in HBM), the shared-memory
// resident sweep and the chain-rule sampler.
//
// Table layout: complex entries interleaved over a batch tile of Bt = 2^lbt
// items, E[c][b] (b fastest).  A row is cut into 16-byte chunks (two complex64 or
// one complex128 values); lanes of a warp own consecutive chunks, so a gather of
// row c is a fully coalesced run of 128-bit loads.
#pragma once
#include <cuda_runtime.h>

#include "plan.hpp"

// Launch shape of the fused pair kernel (scan_pair.cuh): resident 256-thread blocks per
// SM (two: 128 registers per thread) and gathers in flight per lane and loop iteration.
#ifndef RGS_PAIR_MINB
#define RGS_PAIR_MINB 2
#endif
#ifndef RGS_PAIR_LOADS
#define RGS_PAIR_LOADS 8
#endif
// RGS_STREAM_HINTS: table rows are read once and written once per pass, so loads and
// stores may carry the evict-first (streaming) cache hint.
#ifdef RGS_STREAM_HINTS
#define RGS_LD(p) __ldcs(p)
#define RGS_ST(p, v) __stcs(p, v)
#else
#define RGS_LD(p) __ldg(p)
#define RGS_ST(p, v) (*(p) = (v))
#endif

namespace rgs {

typedef unsigned long long u64;

template <typename M>
struct Cx {
  M re, im;
};

// acc += e * w with an explicit fused-multiply-add order, so the result of an item
// does not depend on how the compiler schedules a particular kernel instantiation
// (batch tiles of every size give bitwise-identical amplitudes).
template <typename M>
__device__ __forceinline__ void cmad(Cx<M>& acc, M er, M ei, const Cx<M>& w) {
  acc.re = fma(er, w.re, acc.re);
  acc.re = fma(-ei, w.im, acc.re);
  acc.im = fma(er, w.im, acc.im);
  acc.im = fma(ei, w.re, acc.im);
}

// x with its sign flipped iff neg (exact).
__device__ __forceinline__ float flip_sign(float x, int neg) {
  return __int_as_float(__float_as_int(x) ^ (neg << 31));
}
__device__ __forceinline__ double flip_sign(double x, int neg) {
  return __hiloint2double(__double2hiint(x) ^ (neg << 31), __double2loint(x));
}

// |x|^2 with a fixed rounding sequence.
template <typename S>
__device__ __forceinline__ S norm2(S re, S im) {
  return fma(re, re, im * im);
}

// One 16-byte (or, for single-item complex64 rows, 8-byte) chunk of a table row:
// VE consecutive complex values of storage type S.
template <typename S, int VE>
struct Chunk;
template <>
struct Chunk<float, 2> {
  float4 v;
  __device__ __forceinline__ void load(const float* E, u64 chunk) {
    v = RGS_LD(reinterpret_cast<const float4*>(E) + chunk);
  }
  __device__ __forceinline__ void store(float* E, u64 chunk) const { RGS_ST(reinterpret_cast<float4*>(E) + chunk, v); }
  __device__ __forceinline__ float re(int i) const { return i ? v.z : v.x; }
  __device__ __forceinline__ float im(int i) const { return i ? v.w : v.y; }
  __device__ __forceinline__ void set(int i, float r, float m) {
    if (i) {
      v.z = r;
      v.w = m;
    } else {
      v.x = r;
      v.y = m;
    }
  }
  __device__ __forceinline__ void unit() { v = make_float4(1.f, 0.f, 1.f, 0.f); }
};
template <>
struct Chunk<float, 1> {
  float2 v;
  __device__ __forceinline__ void load(const float* E, u64 chunk) {
    v = RGS_LD(reinterpret_cast<const float2*>(E) + chunk);
  }
  __device__ __forceinline__ void store(float* E, u64 chunk) const { RGS_ST(reinterpret_cast<float2*>(E) + chunk, v); }
  __device__ __forceinline__ float re(int) const { return v.x; }
  __device__ __forceinline__ float im(int) const { return v.y; }
  __device__ __forceinline__ void set(int, float r, float m) { v = make_float2(r, m); }
  __device__ __forceinline__ void unit() { v = make_float2(1.f, 0.f); }
};
template <>
struct Chunk<double, 1> {
  double2 v;
  __device__ __forceinline__ void load(const double* E, u64 chunk) {
    v = RGS_LD(reinterpret_cast<const double2*>(E) + chunk);
  }
  __device__ __forceinline__ void store(double* E, u64 chunk) const { RGS_ST(reinterpret_cast<double2*>(E) + chunk, v); }
  __device__ __forceinline__ double re(int) const { return v.x; }
  __device__ __forceinline__ double im(int) const { return v.y; }
  __device__ __forceinline__ void set(int, double r, double m) { v = make_double2(r, m); }
  __device__ __forceinline__ void unit() { v = make_double2(1.0, 0.0); }
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

// Mass of one branch of a position from the position's Gram matrix G (chain rule):
// u = U_v[x, :] (two complex128), M = G00 |u0|^2 + G11 |u1|^2 + 2 Re(G01 u0 conj(u1)),
// clamped at zero against rounding.
__device__ __forceinline__ double branch_mass(const double2* u, double g00, double g11, double g01r, double g01i) {
  const double2 a = u[0], c = u[1];
  const double zr = a.x * c.x + a.y * c.y, zi = a.y * c.x - a.x * c.y;
  const double m = g00 * (a.x * a.x + a.y * a.y) + g11 * (c.x * c.x + c.y * c.y) + 2.0 * (g01r * zr - g01i * zi);
  return m > 0.0 ? m : 0.0;
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

}  // namespace rgs
