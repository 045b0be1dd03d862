// Allocation-free variant of the batched scan executor.
//
// Some callers cannot let this library allocate device memory: hosts that hand it a
// fixed device-memory budget and forbid it from growing, and integrations whose own
// allocator owns every byte of the GPU and would not see a cudaMalloc made behind its
// back.  rgs_scan_amplitudes_noalloc serves them: the caller passes only inputs and
// outputs, and all scratch (the step byte tables, the two ping-pong environment
// tables, per-item weights and per-step maxima) lives in one file-scope device array
// of fixed size, RGS_NOALLOC_SCRATCH_BYTES, which every GPU that loads this library
// holds until the process exits.  "Allocation-free" means no device allocation only:
// the call still takes a host mutex, builds small host vectors, makes CUDA runtime
// calls and launches kernels, so it must not be called from a CUDA host callback
// (cudaLaunchHostFunc / stream callbacks forbid CUDA calls) or from a signal handler.
//
// Set-up: the first call on a device, with that device current, looks up the
// device address of the array with cudaGetSymbolAddress and caches it for the life
// of the process; a cudaDeviceReset on that device invalidates the cached address,
// so the library must not be used on a device after it was reset.  Every call
// uploads the plan's step tables and vertex records from host memory with pageable
// copies, so it is rejected (RGS_ERR_UNSUPPORTED) on a stream that is being captured.
// The array is shared by every call and keeps the last call's contents; everything
// that must start at zero is cleared by the call itself.  Calls whose work overlaps
// on the GPU (different streams, or threads without ordering) race on the array:
// serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "common.hpp"
#include "plan.hpp"
#include "scan.hpp"

namespace rgs {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[RGS_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[64] = {nullptr};

// Device address of the scratch array on `device` (already current), looked up once.
int noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= 64) return fail(RGS_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_addr[device] = p;
  }
  *out = g_noalloc_addr[device];
  return RGS_OK;
}

struct NoallocLayout {
  size_t off_tables = 0, off_verts = 0, off_ws = 0, total = 0;
  ScanLayout ws;
};

// u64 entries of the per-step byte tables: they come first in plan.tables, before the
// tables of fused pairs, which the position-by-position sweep here never reads.
size_t step_table_entries(const Plan& plan) {
  size_t n = 0;
  for (const auto& d : plan.dev) n = std::max(n, (size_t)d.table_off + ((size_t)d.nbytes << 8));
  return n;
}

int noalloc_layout(const Plan& plan, int Bt, int precision, NoallocLayout& L) {
  int rc = scan_layout(plan, Bt, precision, L.ws);
  if (rc) return rc;
  L.off_tables = 0;
  L.off_verts = align_up(std::max<size_t>(1, step_table_entries(plan)) * sizeof(unsigned long long), 256);
  L.off_ws = L.off_verts + align_up(sizeof(DevVert) * plan.n, 256);
  L.total = L.off_ws + L.ws.total();
  return RGS_OK;
}

}  // namespace
}  // namespace rgs

using namespace rgs;

extern "C" int rgs_scan_amplitudes_noalloc(rgs_plan* handle, const double* unitaries, const uint64_t* bits,
                                           int64_t batch, int32_t precision, void* out_value, double* out_logscale,
                                           void* stream_ptr) {
  if (!handle) return fail(RGS_ERR_ARG, "plan is NULL");
  if (batch < 0) return fail(RGS_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return RGS_OK;
  if (!unitaries || !bits || !out_value || !out_logscale) return fail(RGS_ERR_ARG, "null input or output pointer");
  Plan& plan = handle->plan;
  if (!plan.exec_ok) return fail(RGS_ERR_UNSUPPORTED, plan.exec_reason);
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  RGS_CUDA_TRY(cudaStreamIsCapturing(stream, &capture));
  if (capture != cudaStreamCaptureStatusNone)
    return fail(RGS_ERR_UNSUPPORTED, "rgs_scan_amplitudes_noalloc uploads plan data from pageable host memory on "
                                     "every call: call it on a stream that is not being captured");

  // Largest batch tile (<= 64 items) whose layout fits the fixed scratch array.
  NoallocLayout L;
  int Bt = 1;
  int rc = noalloc_layout(plan, 1, precision, L);
  if (rc) return rc;
  if (L.total > (size_t)RGS_NOALLOC_SCRATCH_BYTES)
    return fail(RGS_ERR_OOM, "plan needs " + std::to_string(L.total) + " bytes of scratch; the allocation-free entry " +
                                 "point has " + std::to_string((size_t)RGS_NOALLOC_SCRATCH_BYTES) +
                                 " (rank too large: use rgs_scan_amplitudes with a caller workspace)");
  while (Bt < 64 && Bt < batch) {
    NoallocLayout next;
    if (noalloc_layout(plan, Bt * 2, precision, next) != RGS_OK || next.total > (size_t)RGS_NOALLOC_SCRATCH_BYTES) break;
    Bt *= 2;
    L = next;
  }

  int device = 0;
  rc = bind_device_of(out_value, &device);
  if (rc) return rc;
  void* base = nullptr;
  rc = noalloc_scratch(device, &base);
  if (rc) return rc;
  char* scratch = (char*)base;

  // Step tables and vertex records into the scratch (copies, not allocations).
  std::vector<DevVert> verts(plan.n);
  for (int j = 0; j < plan.n; ++j) {
    verts[j].fut_lo = (unsigned long long)plan.future[j];
    verts[j].fut_hi = (unsigned long long)(plan.future[j] >> 64);
    verts[j].v = plan.steps[j].v;
    verts[j].fixed = plan.steps[j].free ? 0 : 1;
  }
  unsigned long long* tables = (unsigned long long*)(scratch + L.off_tables);
  DevVert* d_verts = (DevVert*)(scratch + L.off_verts);
  const size_t ntab = step_table_entries(plan);
  if (ntab)
    RGS_CUDA_TRY(cudaMemcpyAsync(tables, plan.tables.data(), ntab * sizeof(unsigned long long),
                                 cudaMemcpyHostToDevice, stream));
  RGS_CUDA_TRY(cudaMemcpyAsync(d_verts, verts.data(), sizeof(DevVert) * plan.n, cudaMemcpyHostToDevice, stream));

  char* ws = scratch + L.off_ws;
  void* buf[2] = {ws + L.ws.off_buf0, ws + L.ws.off_buf1};
  void* W = ws + L.ws.off_w;
  bool has_fixed = false;
  for (auto& st : plan.steps) has_fixed |= !st.free;
  unsigned char* F = has_fixed ? (unsigned char*)(ws + L.ws.off_f) : nullptr;
  unsigned long long* maxbuf = (unsigned long long*)(ws + L.ws.off_max);
  const size_t vsize = precision == RGS_PREC_C128 ? 16 : 8;

  for (long long first = 0; first < batch; first += Bt) {
    const int count = (int)std::min<long long>(Bt, batch - first);
    RGS_CUDA_TRY(scan_launch_weights(d_verts, plan.n, unitaries, (const unsigned long long*)bits, nullptr, first,
                                     count, Bt, W, F, stream));
    // The maxima are accumulated with atomics: they must start at zero on every tile.
    RGS_CUDA_TRY(cudaMemsetAsync(maxbuf, 0, (size_t)plan.n * Bt * sizeof(unsigned long long), stream));
    for (int j = 0; j < plan.n; ++j) {
      const DevStep& st = plan.dev[j];
      RGS_CUDA_TRY(scan_launch_step(precision, Bt, device, st, buf[j & 1], buf[(j + 1) & 1], tables + st.table_off,
                                    (const char*)W + (size_t)j * Bt * 32, F ? F + (size_t)j * Bt : nullptr,
                                    j ? maxbuf + (size_t)(j - 1) * Bt : nullptr, maxbuf + (size_t)j * Bt, j == 0,
                                    stream));
    }
    RGS_CUDA_TRY(scan_launch_finalize(precision, buf[plan.n & 1], maxbuf, plan.n, Bt, count,
                                      (char*)out_value + (size_t)first * vsize, out_logscale + first, stream));
  }
  return RGS_OK;
}
