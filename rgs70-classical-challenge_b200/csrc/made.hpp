// Host interface of the proposal-network kernels (made.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace rgs {

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16* A;
  int lda, transA;
  const __nv_bfloat16* B;
  int ldb, transB;
  float alpha;
  const float* bias;             // [N] or null
  int relu;
  const unsigned char* mask;     // [M][N] or null
  const __nv_bfloat16* gate;     // [M][ldc]: keep only where gate > 0, or null
  float* C;                      // [M][ldc] fp32 out or null
  __nv_bfloat16* Cb;             // [M][ldc] bf16 out or null
  int ldc;
};

int gemm_bf16(const GemmArgs& g, cudaStream_t s);
// TMA loads of the K-major aligned GEMM operands on (1, default) or off (0).
int gemm_set_tma(int on);
// Reads and clears the flag that a bounded tensor-core wait gave up (synchronous).
int tensor_core_status(int* timed_out);
int bce_grad(const float* z, const float* target, int count, float scale, __nv_bfloat16* dz, double* partial,
             int blocks, cudaStream_t s);
int colsum_bf16(const __nv_bfloat16* x, int rows, int cols, float* out, cudaStream_t s);
int adam_step(float* w, const float* grad, float* m1, float* m2, const unsigned char* mask, __nv_bfloat16* wb,
              int count, float lr, float b1, float b2, float eps, int t, cudaStream_t s);
int sample_position(const float* z, int n, int d, int count, unsigned long long seed, unsigned long long first,
                    __nv_bfloat16* x, double* logq, cudaStream_t s);
int log_q(const float* z, const __nv_bfloat16* x, int n, int count, double* logq, cudaStream_t s);

}  // namespace rgs
