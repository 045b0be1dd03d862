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

// Chunked sweep (scan_run): S tiles share one launch per small position (input and output
// rank at most kSmallRank); the positions between the leading and trailing small ones
// (h <= j < t) run tile by tile.  Workspace: two small-table buffers of S tiles, two
// full-size tables for the middle positions, weights / flags / maxima of S tiles.
constexpr int kChunkItems = 8192;  // default items per chunk (S = kChunkItems / Bt tiles)
struct ChunkLayout {
  int Bt = 1, S = 1, h = 0, t = 0;
  size_t esize = 8;
  unsigned long long e_stride = 0;  // entries per tile in the small buffers
  size_t bytes_small = 0, bytes_big = 0;
  size_t off_small0 = 0, off_small1 = 0, off_big0 = 0, off_big1 = 0, off_w = 0, off_f = 0, off_max = 0, total = 0;
};
int scan_chunk_layout(const Plan& plan, int Bt, int precision, int S, ChunkLayout& L);
int scan_chunk_tiles(int Bt);
// Tiles per chunk that scan_run uses with a workspace of ws_bytes (the largest S <=
// scan_chunk_tiles(Bt), S >= 2, whose layout fits, with C filled in); 0: tile by tile.
int scan_pick_chunk(const Plan& plan, int Bt, int precision, size_t ws_bytes, ChunkLayout& C, int* S);
// Kernel launches scan_run queues for `batch` items with that workspace.
int scan_launch_count(const Plan& plan, long long batch, int Bt, int precision, size_t ws_bytes, long long* out);

// Fused pair launches (scan_pair_{c128,c64,f32}.cu): one instantiation set per precision.
cudaError_t launch_pair_c128(int VE, dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                             const unsigned long long* tables, const double4* WA, const double4* WB,
                             const unsigned long long* mp, unsigned long long* mA, unsigned long long* mc, int lbt,
                             unsigned long long es);
cudaError_t launch_pair_c64(int VE, dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                            const unsigned long long* tables, const double4* WA, const double4* WB,
                            const unsigned long long* mp, unsigned long long* mA, unsigned long long* mc, int lbt,
                            unsigned long long es);
cudaError_t launch_pair_f32(int VE, dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                            const unsigned long long* tables, const double4* WA, const double4* WB,
                            const unsigned long long* mp, unsigned long long* mA, unsigned long long* mc, int lbt,
                            unsigned long long es);

// Gram partials of B of a fused pair (chain-rule sampling, scan_pair_kernel GRAM mode),
// complex64 tables with float64 arithmetic and complex128 tables.
cudaError_t launch_pair_gram_c64(int VE, dim3 grid, cudaStream_t s, const void* Ein, const DevPair& P,
                                 const unsigned long long* tables, const double4* WA, const unsigned long long* mp,
                                 int lbt, double* partial);
cudaError_t launch_pair_gram_c128(int VE, dim3 grid, cudaStream_t s, const void* Ein, const DevPair& P,
                                  const unsigned long long* tables, const double4* WA, const unsigned long long* mp,
                                  int lbt, double* partial);
cudaError_t launch_pair_gram_f32(int VE, dim3 grid, cudaStream_t s, const void* Ein, const DevPair& P,
                                 const unsigned long long* tables, const double4* WA, const unsigned long long* mp,
                                 int lbt, double* partial);
// One fused pair (positions P.j, P.j + 1) over one batch tile.
cudaError_t scan_launch_pair(int precision, int Bt, int device, const DevPair& P, const void* Ein, void* Eout,
                             const unsigned long long* tables, const double4* WA, const double4* WB,
                             const unsigned long long* mp, unsigned long long* mA, unsigned long long* mc,
                             cudaStream_t s);
// B's Gram partials of a fused pair over one batch tile: `blocks` blocks write
// partial[blocks][Bt][4] (G00, G11, Re G01, Im G01 of B's branch masses, float64 sums).
cudaError_t scan_launch_pair_gram(int precision, int Bt, int blocks, const DevPair& P, const void* Ein,
                                  const unsigned long long* tables, const double4* WA, const unsigned long long* mp,
                                  double* partial, cudaStream_t s);

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
