// C ABI of the proposal network: GEMM, forward, backward, Adam, sampling, log q.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.hpp"
#include "made.hpp"

using namespace rgs;

namespace {
typedef const __nv_bfloat16* cbf;
typedef __nv_bfloat16* bf;

int bind(const void* p) {
  int device = 0;
  return bind_device_of(p, &device);
}

GemmArgs make(int M, int N, int K, const void* A, int lda, int tA, const void* B, int ldb, int tB) {
  GemmArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = (cbf)A;
  g.lda = lda;
  g.transA = tA;
  g.B = (cbf)B;
  g.ldb = ldb;
  g.transB = tB;
  g.alpha = 1.f;
  return g;
}

// Forward of the three layers; h1b, h2b bf16 [batch][hidden], z fp32 [batch][n].
int forward(int batch, int n, int hidden, const void* x, const void* w1b, const float* b1, const void* w2b,
            const float* b2, const void* w3b, const float* b3, void* h1b, void* h2b, float* z, cudaStream_t s) {
  GemmArgs g = make(batch, hidden, n, x, n, 0, w1b, n, 1);
  g.bias = b1;
  g.relu = 1;
  g.Cb = (bf)h1b;
  g.ldc = hidden;
  int rc = gemm_bf16(g, s);
  if (rc) return rc;
  g = make(batch, hidden, hidden, h1b, hidden, 0, w2b, hidden, 1);
  g.bias = b2;
  g.relu = 1;
  g.Cb = (bf)h2b;
  g.ldc = hidden;
  if ((rc = gemm_bf16(g, s))) return rc;
  g = make(batch, n, hidden, h2b, hidden, 0, w3b, hidden, 1);
  g.bias = b3;
  g.C = z;
  g.ldc = n;
  return gemm_bf16(g, s);
}
}  // namespace

extern "C" {

int rgs_gemm_bf16(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, int32_t transA, const void* B,
                  int32_t ldb, int32_t transB, float alpha, const float* bias, int32_t relu, const uint8_t* mask,
                  const void* gate, float* C, void* Cb, int32_t ldc, void* stream) {
  int rc = bind(A);
  if (rc) return rc;
  GemmArgs g = make(M, N, K, A, lda, transA, B, ldb, transB);
  g.alpha = alpha;
  g.bias = bias;
  g.relu = relu;
  g.mask = mask;
  g.gate = (cbf)gate;
  g.C = C;
  g.Cb = (bf)Cb;
  g.ldc = ldc;
  return gemm_bf16(g, (cudaStream_t)stream);
}

int rgs_tensor_core_status(int32_t* timed_out) {
  if (!timed_out) return fail(RGS_ERR_ARG, "timed_out is NULL");
  int v = 0;
  int rc = tensor_core_status(&v);
  *timed_out = v;
  return rc;
}

int rgs_gemm_set_tma(int32_t on) { return gemm_set_tma(on); }

int rgs_mlp_fwd(int32_t batch, int32_t n, int32_t hidden, const void* x, const void* w1b, const float* b1,
                const void* w2b, const float* b2, const void* w3b, const float* b3, void* h1b, void* h2b, float* z,
                void* stream) {
  int rc = bind(x);
  if (rc) return rc;
  return forward(batch, n, hidden, x, w1b, b1, w2b, b2, w3b, b3, h1b, h2b, z, (cudaStream_t)stream);
}

int rgs_mlp_bwd(int32_t batch, int32_t n, int32_t hidden, const void* x, const void* w2b, const void* w3b,
                const void* h1b, const void* h2b, const float* z, const float* target, const uint8_t* m1,
                const uint8_t* m2, const uint8_t* m3, void* dzb, void* dh2b, void* dh1b, float* gw1, float* gb1,
                float* gw2, float* gb2, float* gw3, float* gb3, double* loss_partials, int32_t loss_blocks,
                void* stream) {
  int rc = bind(x);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = bce_grad(z, target, batch * n, 1.f / batch, (bf)dzb, loss_partials, loss_blocks, s))) return rc;
  GemmArgs g = make(n, hidden, batch, dzb, n, 1, h2b, hidden, 0);  // gw3 = dz^T h2
  g.mask = m3;
  g.C = gw3;
  g.ldc = hidden;
  if ((rc = gemm_bf16(g, s))) return rc;
  if ((rc = colsum_bf16((cbf)dzb, batch, n, gb3, s))) return rc;
  g = make(batch, hidden, n, dzb, n, 0, w3b, hidden, 0);  // dh2 = dz W3 * [h2 > 0]
  g.gate = (cbf)h2b;
  g.Cb = (bf)dh2b;
  g.ldc = hidden;
  if ((rc = gemm_bf16(g, s))) return rc;
  g = make(hidden, hidden, batch, dh2b, hidden, 1, h1b, hidden, 0);  // gw2 = dh2^T h1
  g.mask = m2;
  g.C = gw2;
  g.ldc = hidden;
  if ((rc = gemm_bf16(g, s))) return rc;
  if ((rc = colsum_bf16((cbf)dh2b, batch, hidden, gb2, s))) return rc;
  g = make(batch, hidden, hidden, dh2b, hidden, 0, w2b, hidden, 0);  // dh1 = dh2 W2 * [h1 > 0]
  g.gate = (cbf)h1b;
  g.Cb = (bf)dh1b;
  g.ldc = hidden;
  if ((rc = gemm_bf16(g, s))) return rc;
  g = make(hidden, n, batch, dh1b, hidden, 1, x, n, 0);  // gw1 = dh1^T x
  g.mask = m1;
  g.C = gw1;
  g.ldc = n;
  if ((rc = gemm_bf16(g, s))) return rc;
  return colsum_bf16((cbf)dh1b, batch, hidden, gb1, s);
}

int rgs_mlp_adam(float* w, const float* grad, float* m1, float* m2, const uint8_t* mask, void* wb, int32_t count,
                 float lr, float beta1, float beta2, float eps, int32_t t, void* stream) {
  int rc = bind(w);
  if (rc) return rc;
  return adam_step(w, grad, m1, m2, mask, (bf)wb, count, lr, beta1, beta2, eps, t, (cudaStream_t)stream);
}

int rgs_mlp_sample(int32_t batch, int32_t n, int32_t hidden, const void* w1b, const float* b1, const void* w2b,
                   const float* b2, const void* w3b, const float* b3, uint64_t seed, uint64_t first, void* x,
                   double* logq, void* h1b, void* h2b, float* z, void* stream) {
  int rc = bind(x);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  RGS_CUDA_TRY(cudaMemsetAsync(x, 0, (size_t)batch * n * sizeof(__nv_bfloat16), s));
  RGS_CUDA_TRY(cudaMemsetAsync(logq, 0, (size_t)batch * sizeof(double), s));
  for (int d = 0; d < n; ++d) {
    if ((rc = forward(batch, n, hidden, x, w1b, b1, w2b, b2, w3b, b3, h1b, h2b, z, s))) return rc;
    if ((rc = sample_position(z, n, d, batch, seed, first, (bf)x, logq, s))) return rc;
  }
  return RGS_OK;
}

int rgs_mlp_logq(int32_t batch, int32_t n, int32_t hidden, const void* x, const void* w1b, const float* b1,
                 const void* w2b, const float* b2, const void* w3b, const float* b3, double* logq, void* h1b,
                 void* h2b, float* z, void* stream) {
  int rc = bind(x);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = forward(batch, n, hidden, x, w1b, b1, w2b, b2, w3b, b3, h1b, h2b, z, s))) return rc;
  return log_q(z, (cbf)x, n, batch, logq, s);
}

}  // extern "C"
