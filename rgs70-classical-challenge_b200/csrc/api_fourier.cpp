// C ABI of the conditional (Fourier-cut) sampler and its building blocks.
#include <cuda_runtime.h>

#include <cstring>
#include <new>

#include "common.hpp"
#include "fourier.cuh"

struct rgs_fourier {
  rgs::FourierPlan plan;
};

using namespace rgs;

namespace {
void copy_table(const std::vector<u64h>& src, uint64_t* dst) {
  if (dst) std::memcpy(dst, src.data(), src.size() * sizeof(uint64_t));
}
}  // namespace

extern "C" {

int rgs_fourier_create(int32_t n, const uint8_t* graph, const double* unitaries, int32_t m, const int32_t* A,
                       const int32_t* B, int32_t deferred, rgs_fourier** out) {
  if (!out) return fail(RGS_ERR_ARG, "out is NULL");
  *out = nullptr;
  rgs_fourier* f = new (std::nothrow) rgs_fourier;
  if (!f) return fail(RGS_ERR_OOM, "host allocation failed");
  int status = RGS_OK;
  std::string err = fourier_build(n, graph, unitaries, m, (const int*)A, (const int*)B, deferred != 0, f->plan, status);
  if (!err.empty()) {
    delete f;
    return fail(status, err);
  }
  *out = f;
  return RGS_OK;
}

void rgs_fourier_destroy(rgs_fourier* f) { delete f; }

int rgs_fourier_info(const rgs_fourier* f, int32_t* m, int32_t* specialized, int32_t* tile_bits, int64_t* ntiles,
                     int32_t* passes) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  const FourierPlan& p = f->plan;
  FourierLayout L;
  fourier_layout(p, L);
  if (m) *m = p.m;
  if (specialized) *specialized = p.specialized ? 1 : 0;
  if (tile_bits) *tile_bits = p.m < kTileBits ? p.m : kTileBits;
  if (ntiles) *ntiles = L.ntiles;
  if (passes) *passes = p.m <= kTileBits ? 1 : 2 * p.ngroups + 1;
  return RGS_OK;
}

int rgs_fourier_tables(const rgs_fourier* f, uint64_t* lut_z, uint64_t* lut_a, uint64_t* lut_cols,
                       uint64_t* inv_rows, int32_t* chunks) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  const FourierPlan& p = f->plan;
  if (chunks) *chunks = p.chunks;
  copy_table(p.lut_z, lut_z);
  copy_table(p.lut_a, lut_a);
  copy_table(p.lut_cols, lut_cols);
  copy_table(p.inv_rows, inv_rows);
  return RGS_OK;
}

int rgs_fourier_workspace_bytes(const rgs_fourier* f, size_t* bytes) {
  if (!f || !bytes) return fail(RGS_ERR_ARG, "null argument");
  FourierLayout L;
  fourier_layout(f->plan, L);
  *bytes = L.total;
  return RGS_OK;
}

int rgs_fourier_compute_shard(rgs_fourier* f, uint64_t outB, int32_t shard, void* state, void* workspace,
                              size_t workspace_bytes, void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  if (f->plan.m < 64 && (outB >> f->plan.m) != 0) return fail(RGS_ERR_ARG, "outB has bits above m");
  return fourier_compute_shard(f->plan, outB, shard, state, workspace, workspace_bytes, (cudaStream_t)stream);
}

int rgs_fourier_shard_mass(rgs_fourier* f, void* workspace, double* mass, void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  return fourier_shard_mass(f->plan, workspace, mass, (cudaStream_t)stream);
}

int rgs_fourier_shard_draw(rgs_fourier* f, const void* state, void* workspace, double u1, double u2,
                           uint64_t* local_index, void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  return fourier_shard_draw(f->plan, state, workspace, u1, u2, local_index, (cudaStream_t)stream);
}

int rgs_fourier_tune(rgs_fourier* f, void* state, void* workspace, size_t workspace_bytes, void* stream,
                     int32_t* variant, float* ms) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  int rc = fourier_tune(f->plan, state, workspace, workspace_bytes, (cudaStream_t)stream, ms);
  if (!rc && variant) *variant = f->plan.variant;
  return rc;
}

int rgs_fourier_set_register_schedule(int32_t on) { return fourier_set_register_schedule(on); }

int rgs_fourier_set_tma(int32_t on) { return fourier_set_tma(on); }

int rgs_fourier_compute(rgs_fourier* f, uint64_t outB, void* state, void* workspace, size_t workspace_bytes,
                        void* stream, float* stage_ms) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  FourierStages st;
  int rc = fourier_compute(f->plan, outB, state, workspace, workspace_bytes, (cudaStream_t)stream,
                           stage_ms ? &st : nullptr);
  if (!rc && stage_ms) {
    stage_ms[0] = st.init_ms;
    stage_ms[1] = st.walsh_ms;
    stage_ms[2] = st.product_ms;
  }
  return rc;
}

int rgs_fourier_compute_permute(rgs_fourier* f, uint64_t outB, void* state, void* scratch, void* workspace,
                                size_t workspace_bytes, void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  return fourier_compute_permute(f->plan, outB, state, scratch, workspace, workspace_bytes, (cudaStream_t)stream);
}

int rgs_fourier_masses(rgs_fourier* f, const void* state, void* workspace, double* host_masses, double* norm,
                       void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = fourier_masses(f->plan, state, workspace, s);
  if (rc) return rc;
  FourierLayout L;
  fourier_layout(f->plan, L);
  std::vector<double> h(L.ntiles);
  RGS_CUDA_TRY(cudaMemcpyAsync(h.data(), (char*)workspace + L.off_masses, h.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
  RGS_CUDA_TRY(cudaStreamSynchronize(s));
  double t = 0.0;
  for (double x : h) t += x;
  if (host_masses) std::memcpy(host_masses, h.data(), h.size() * sizeof(double));
  if (norm) *norm = t;
  return RGS_OK;
}

int rgs_fourier_draw(rgs_fourier* f, const void* state, void* workspace, double u1, double u2, double u3,
                     uint64_t* index, double* pa, double* norm, void* stream) {
  if (!f || !index || !pa || !norm) return fail(RGS_ERR_ARG, "null argument");
  return fourier_draw(f->plan, state, workspace, u1, u2, u3, index, pa, norm, (cudaStream_t)stream);
}

int rgs_fourier_index_map(rgs_fourier* f, const void* src, void* dst, void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  return fourier_index_map(f->plan, src, dst, (cudaStream_t)stream);
}

int rgs_fourier_quadphase(rgs_fourier* f, void* state, void* stream) {
  if (!f) return fail(RGS_ERR_ARG, "plan is NULL");
  return fourier_quadphase(f->plan, state, (cudaStream_t)stream);
}

int rgs_fwht(void* state, int32_t nbits, int32_t lo, int32_t hi, void* stream) {
  return fwht_bits(state, nbits, lo, hi, (cudaStream_t)stream);
}

int rgs_fwht_precision(void* state, int32_t nbits, int32_t lo, int32_t hi, int32_t precision, void* stream) {
  if (precision == RGS_WHT_FP32) return fwht_bits(state, nbits, lo, hi, (cudaStream_t)stream);
  if (precision == RGS_WHT_SPLIT_BF16X2 || precision == RGS_WHT_SPLIT_BF16X3)
    return fwht_tensor_core(state, nbits, lo, hi, precision, (cudaStream_t)stream);
  return fail(RGS_ERR_ARG, "unknown WHT precision");
}

int rgs_product(void* state, int32_t nbits, const double* unitaries, int32_t lo, int32_t hi, void* stream) {
  return product_bits(state, nbits, unitaries, lo, hi, (cudaStream_t)stream);
}

int rgs_block_mass(const void* state, int32_t nbits, int32_t tile_bits, double* masses, void* stream) {
  int device = 0;
  int rc = bind_device_of(state, &device);
  if (rc) return rc;
  return block_mass(state, nbits, tile_bits, masses, (cudaStream_t)stream);
}

}  // extern "C"
