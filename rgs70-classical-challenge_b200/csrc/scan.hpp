// Host interface of the scan executor (scan.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "plan.hpp"

namespace rgs {

// Workspace partition for one batch tile: two ping-pong tables, weights, flags and
// per-step maxima (all offsets 256-byte aligned).
struct ScanLayout {
  int Bt = 1;
  size_t esize = 8;
  size_t bytes_buf = 0, bytes_w = 0, bytes_f = 0, bytes_max = 0;
  size_t off_buf0 = 0, off_buf1 = 0, off_w = 0, off_f = 0, off_max = 0;
  size_t total() const;
};

struct ScanStats {
  long long launches = 0;
};

int scan_layout(const Plan& plan, int Bt, int precision, ScanLayout& L);

// Largest batch tile the step kernel supports for a precision.
int scan_max_tile(int precision);


// Uploads (once per device) the plan's step records, byte tables and vertex records.
int plan_device_copy(Plan& plan, int device, const Plan::DeviceCopy** out);

// Runs the sweep for `batch` items: either bits (+ unitaries) or explicit contraction
// vectors fvec.  All work is queued on `stream`.
int scan_run(Plan& plan, const double* U, const unsigned long long* bits, const double* fvec, long long batch,
             int precision, void* out_value, double* out_logscale, void* workspace, size_t ws_bytes, int Bt,
             cudaStream_t stream, ScanStats* stats);

// Single-kernel launch wrappers (same kernels as scan_run), for drivers that manage
// their own device memory layout.
cudaError_t scan_launch_weights(const DevVert* verts, int n, const double* U, const unsigned long long* bits,
                                const double* fvec, long long first, int count, int Bt, void* W, unsigned char* F,
                                cudaStream_t stream);
cudaError_t scan_launch_step(int precision, int Bt, int device, const DevStep& st, const void* Ein, void* Eout,
                             const unsigned long long* T, const void* W, const unsigned char* F,
                             const unsigned long long* maxprev, unsigned long long* maxcur, bool unit_input,
                             cudaStream_t stream);
cudaError_t scan_launch_finalize(int precision, const void* E, const unsigned long long* maxbuf, int n, int Bt,
                                 int count, void* out_value, double* out_logscale, cudaStream_t stream);

}  // namespace rgs
