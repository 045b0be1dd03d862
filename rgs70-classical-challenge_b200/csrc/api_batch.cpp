// C ABI of the shared-memory-resident batch executor (include/rgs_b200.h, rgs_batch_*).
#include <cuda_runtime.h>

#include <new>
#include <vector>

#include "common.hpp"
#include "plan.hpp"
#include "resident.hpp"
#include "scan.hpp"

struct rgs_batch {
  int precision = RGS_PREC_C64;
  int variant = 0;  // launch variant (rgs_batch_tune)
  std::vector<rgs::ResInstance> insts;
  rgs::ResDevice dev;
  bool dirty = true;
  long long units = 0;
};

using namespace rgs;

namespace {

int same_device(rgs_batch* b, const void* p) {
  int device = -1;
  int rc = bind_device_of(p, &device);
  if (rc) return rc;
  if (b->dev.device < 0) b->dev.device = device;
  if (device != b->dev.device) return fail(RGS_ERR_ARG, "all buffers of a batch must be on one device");
  return RGS_OK;
}

}  // namespace

extern "C" {

int rgs_batch_max_rank(int32_t precision, int32_t* rmax) {
  if (!rmax) return fail(RGS_ERR_ARG, "null argument");
  if (precision < RGS_PREC_C64 || precision > RGS_PREC_C128) return fail(RGS_ERR_ARG, "unknown precision");
  *rmax = resident_max_rank(precision);
  return RGS_OK;
}

int rgs_batch_create(int32_t precision, rgs_batch** out) {
  if (!out) return fail(RGS_ERR_ARG, "null argument");
  if (precision < RGS_PREC_C64 || precision > RGS_PREC_C128) return fail(RGS_ERR_ARG, "unknown precision");
  rgs_batch* b = new (std::nothrow) rgs_batch();
  if (!b) return fail(RGS_ERR_OOM, "out of host memory");
  b->precision = precision;
  *out = b;
  return RGS_OK;
}

void rgs_batch_destroy(rgs_batch* batch) { delete batch; }

int rgs_batch_add(rgs_batch* batch, rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t count,
                  void* out_value, double* out_logscale, int64_t nsamples, uint64_t seed, uint64_t* sample_bits,
                  void* sample_value, double* sample_logscale, double* sample_logp, int32_t* index) {
  if (!batch || !plan) return fail(RGS_ERR_ARG, "null batch or plan");
  if (count < 0 || nsamples < 0) return fail(RGS_ERR_ARG, "counts must be >= 0");
  if (!unitaries) return fail(RGS_ERR_ARG, "unitaries are required");
  if (count > 0 && (!bits || !out_value || !out_logscale))
    return fail(RGS_ERR_ARG, "amplitudes need bits, out_value and out_logscale");
  if (nsamples > 0 && (!sample_bits || !sample_value || !sample_logscale))
    return fail(RGS_ERR_ARG, "samples need sample_bits, sample_value and sample_logscale");
  Plan& p = plan->plan;
  if (!p.exec_ok) return fail(RGS_ERR_UNSUPPORTED, p.exec_reason);
  const int nb = resident_items(p.rmax, batch->precision);
  if (nb < 1)
    return fail(RGS_ERR_UNSUPPORTED, "plan rank " + std::to_string(p.rmax) + " is above the resident maximum " +
                                         std::to_string(resident_max_rank(batch->precision)));
  bool fixed = false;
  for (auto& st : p.steps)
    if (!st.free) fixed = true;
  if (fixed && nsamples > 0) return fail(RGS_ERR_UNSUPPORTED, "samples of plans with fixed vertices");
  int rc = same_device(batch, unitaries);
  if (rc) return rc;
  const void* outs[] = {bits, out_value, out_logscale, sample_bits, sample_value, sample_logscale, sample_logp};
  for (const void* o : outs)
    if (o && (rc = same_device(batch, o))) return rc;
  const Plan::DeviceCopy* dc = nullptr;
  if ((rc = plan_device_copy(p, batch->dev.device, &dc))) return rc;
  ResInstance in;
  in.steps = (const DevStep*)dc->steps;
  in.tables = (const unsigned long long*)dc->tables;
  in.verts = (const DevVert*)dc->verts;
  in.U = unitaries;
  in.bits = (const unsigned long long*)bits;
  in.out_value = out_value;
  in.out_logscale = out_logscale;
  in.sample_bits = (unsigned long long*)sample_bits;
  in.sample_value = sample_value;
  in.sample_logscale = sample_logscale;
  in.sample_logp = sample_logp;
  in.count = count;
  in.nsamples = nsamples;
  in.seed = seed;
  in.n = p.n;
  in.nb = nb;
  in.rmax = p.rmax;
  in.has_fixed = fixed ? 1 : 0;
  if (resident_items(p.rmax, batch->precision, batch->variant) < 1) batch->variant = 0;  // the tuned variant is too small
  if (index) *index = (int32_t)batch->insts.size();
  batch->insts.push_back(in);
  batch->units += (count + nb - 1) / nb + (nsamples + nb - 1) / nb;
  batch->dirty = true;
  return RGS_OK;
}

int rgs_batch_info(const rgs_batch* batch, int32_t* instances, int64_t* units) {
  if (!batch) return fail(RGS_ERR_ARG, "null batch");
  if (instances) *instances = (int32_t)batch->insts.size();
  if (units) *units = batch->units;
  return RGS_OK;
}

int rgs_batch_tune(rgs_batch* batch, void* stream, int32_t* variant, float* ms) {
  if (!batch) return fail(RGS_ERR_ARG, "null batch");
  if (batch->insts.empty()) return RGS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int best = -1;
  float best_ms = 0.f;
  for (int v = 0; v < kResVariants; ++v) {
    if (ms) ms[v] = -1.f;
    bool fits = true;
    for (auto& in : batch->insts)
      if (resident_items(in.rmax, batch->precision, v) < 1) fits = false;
    if (!fits) continue;
    int rc = resident_prepare(batch->insts, batch->precision, v, batch->dev);
    if (rc) return rc;
    if ((rc = resident_launch(batch->dev, batch->precision, s, nullptr))) return rc;
    cudaEvent_t e0, e1;
    RGS_CUDA_TRY(cudaEventCreate(&e0));
    RGS_CUDA_TRY(cudaEventCreate(&e1));
    RGS_CUDA_TRY(cudaEventRecord(e0, s));
    for (int r = 0; r < 2; ++r)
      if ((rc = resident_launch(batch->dev, batch->precision, s, nullptr))) return rc;
    RGS_CUDA_TRY(cudaEventRecord(e1, s));
    RGS_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    RGS_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    t *= 0.5f;
    if (ms) ms[v] = t;
    if (best < 0 || t < best_ms) {
      best = v;
      best_ms = t;
    }
  }
  if (best < 0) return fail(RGS_ERR_UNSUPPORTED, "no launch variant holds every instance");
  batch->variant = best;
  int rc = resident_prepare(batch->insts, batch->precision, best, batch->dev);
  if (rc) return rc;
  batch->units = batch->dev.nwork;
  batch->dirty = false;
  if (variant) *variant = best;
  return RGS_OK;
}

int rgs_batch_run(rgs_batch* batch, int32_t check, void* stream) {
  if (!batch) return fail(RGS_ERR_ARG, "null batch");
  if (batch->insts.empty()) return RGS_OK;
  int rc;
  if (batch->dirty) {
    if ((rc = resident_prepare(batch->insts, batch->precision, batch->variant, batch->dev))) return rc;
    batch->units = batch->dev.nwork;
    batch->dirty = false;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = resident_launch(batch->dev, batch->precision, s, nullptr))) return rc;
  if (check) {
    int h[2] = {0, 0};
    RGS_CUDA_TRY(cudaMemcpyAsync(h, batch->dev.counter, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    RGS_CUDA_TRY(cudaStreamSynchronize(s));
    if (h[1]) return fail(RGS_ERR_ZERO_NORM, "a branch pair had zero or non-finite total mass");
  }
  return RGS_OK;
}

}  // extern "C"
