// Packed two-lane FP32 arithmetic of sm_100 (PTX add/sub/fma .f32x2): one instruction
// on a (re, im) pair, round-to-nearest like the scalar forms.  Each lane is the IEEE
// single-precision operation, so results equal two scalar add.rn / sub.rn / fma.rn.
#pragma once

#include <cuda_runtime.h>

#ifndef RGS_NO_F32X2
__device__ __forceinline__ float2 f2add(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}

__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}

// a * b + c per lane.
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
#else
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
}
#endif

// The same operations on a (re, im) pair held as one 64-bit register (v2): a pass keeps
// its registers in this form, so the packed instructions need no pairing moves.
typedef unsigned long long v2;

__device__ __forceinline__ v2 v2pack(float2 a) {
  v2 d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(a.x), "f"(a.y));
  return d;
}
__device__ __forceinline__ float2 v2unpack(v2 a) {
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(a));
  return d;
}
#ifndef RGS_NO_F32X2
__device__ __forceinline__ v2 v2add(v2 a, v2 b) {
  v2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ v2 v2sub(v2 a, v2 b) {
  v2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// a * b + c per lane.
__device__ __forceinline__ v2 v2fma(v2 a, v2 b, v2 c) {
  v2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
#else
__device__ __forceinline__ v2 v2add(v2 a, v2 b) { return v2pack(f2add(v2unpack(a), v2unpack(b))); }
__device__ __forceinline__ v2 v2sub(v2 a, v2 b) { return v2pack(f2sub(v2unpack(a), v2unpack(b))); }
__device__ __forceinline__ v2 v2fma(v2 a, v2 b, v2 c) { return v2pack(f2fma(v2unpack(a), v2unpack(b), v2unpack(c))); }
#endif
