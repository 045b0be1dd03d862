// Scan executor: batched graph-state amplitudes on sm_100a.
//
// Replaces the per-step CuPy kernel and host loop of whyihaveyou/rgs70-classical-challenge
// (W/upstream_scan/gpu_kernel.py:59-170 and gpu_kernel_fp64.py:24-135):
//  * a batch tile of Bt bitstrings runs as one interleaved table E[c][b], so every
//    gather is a contiguous Bt-item row (128-bit loads);
//  * outputs c' and c'^t (t = image of the y unit vector) read the same inputs, so a
//    thread produces both and each input entry is read once per step (the reference
//    reads every input twice and relies on caches for the second read);
//  * the power-of-two renormalisation is derived on the device from the previous
//    step's maximum, so a sweep is a fixed launch sequence with no host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.hpp"
#include "plan.hpp"
#include "scan.hpp"
#include "scan_device.cuh"
#include "scan_row.cuh"

namespace rgs {

Plan::~Plan() {
  int prev = -1;
  cudaGetDevice(&prev);
  for (auto& d : device_copies) {
    if (d.device < 0) continue;
    cudaSetDevice(d.device);
    if (d.steps) cudaFree(d.steps);
    if (d.tables) cudaFree(d.tables);
    if (d.verts) cudaFree(d.verts);
  }
  if (prev >= 0) cudaSetDevice(prev);
}

int sm_count(int device) {
  static int cache[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (!cache[device]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
    cache[device] = v;
  }
  return cache[device];
}

// The library carries its own CUDA runtime, whose current device is independent of
// the caller's runtime; the device is taken from a caller-owned device pointer.
int bind_device_of(const void* p, int* device) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RGS_ERR_ARG, std::string("pointer is not CUDA memory: ") + cudaGetErrorString(e));
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return fail(RGS_ERR_ARG, "workspace/output must be device memory");
  RGS_CUDA_TRY(cudaSetDevice(a.device));
  *device = a.device;
  return RGS_OK;
}

static std::mutex g_upload_mutex;

int plan_device_copy(Plan& plan, int device, const Plan::DeviceCopy** out) {
  std::lock_guard<std::mutex> lock(g_upload_mutex);
  for (auto& d : plan.device_copies)
    if (d.device == device) {
      *out = &d;
      return RGS_OK;
    }
  if (!plan.exec_ok) return fail(RGS_ERR_UNSUPPORTED, plan.exec_reason);
  Plan::DeviceCopy d;
  d.device = device;
  std::vector<DevVert> verts(plan.n);
  for (int j = 0; j < plan.n; ++j) {
    verts[j].fut_lo = (unsigned long long)plan.future[j];
    verts[j].fut_hi = (unsigned long long)(plan.future[j] >> 64);
    verts[j].v = plan.steps[j].v;
    verts[j].fixed = plan.steps[j].free ? 0 : 1;
  }
  const size_t tb = std::max<size_t>(1, plan.tables.size()) * sizeof(unsigned long long);
  RGS_CUDA_TRY(cudaMalloc(&d.steps, sizeof(DevStep) * plan.n));
  RGS_CUDA_TRY(cudaMalloc(&d.tables, tb));
  RGS_CUDA_TRY(cudaMalloc(&d.verts, sizeof(DevVert) * plan.n));
  RGS_CUDA_TRY(cudaMemcpy(d.steps, plan.dev.data(), sizeof(DevStep) * plan.n, cudaMemcpyHostToDevice));
  if (!plan.tables.empty())
    RGS_CUDA_TRY(cudaMemcpy(d.tables, plan.tables.data(), plan.tables.size() * sizeof(unsigned long long),
                            cudaMemcpyHostToDevice));
  RGS_CUDA_TRY(cudaMemcpy(d.verts, verts.data(), sizeof(DevVert) * plan.n, cudaMemcpyHostToDevice));
  plan.device_copies.push_back(d);
  *out = &plan.device_copies.back();
  return RGS_OK;
}

// ------------------------------------------------------------------------------------------------
// Weights: W[j][b] = (f_v(0), f_v(1)) of item b at position j, and for plans with fixed
// vertices the flags y | ov << 1 (the affine syndrome offset of scan_plan.py:167-172).
__global__ void scan_weights_kernel(const DevVert* __restrict__ verts, int n, const double2* __restrict__ U,
                                    const u64* __restrict__ bits, const double2* __restrict__ fvec,
                                    long long first, int count, int Bt, double4* __restrict__ W,
                                    unsigned char* __restrict__ F) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= Bt) return;
  if (b >= count) {
    for (int j = 0; j < n; ++j) {
      W[(size_t)j * Bt + b] = make_double4(0.0, 0.0, 0.0, 0.0);
      if (F) F[(size_t)j * Bt + b] = 0;
    }
    return;
  }
  const long long item = first + b;
  u64 lo = 0, hi = 0;
  if (bits) {
    lo = bits[2 * item];
    hi = bits[2 * item + 1];
  }
  u64 olo = 0, ohi = 0;
  for (int j = 0; j < n; ++j) {
    const DevVert vt = verts[j];
    double2 f0, f1;
    if (fvec) {
      f0 = fvec[((size_t)item * n + vt.v) * 2 + 0];
      f1 = fvec[((size_t)item * n + vt.v) * 2 + 1];
    } else {
      const int x = (int)((vt.v < 64 ? (lo >> vt.v) : (hi >> (vt.v - 64))) & 1ull);
      f0 = U[(vt.v * 2 + x) * 2 + 0];
      f1 = U[(vt.v * 2 + x) * 2 + 1];
    }
    const int ov = (int)((j < 64 ? (olo >> j) : (ohi >> (j - 64))) & 1ull);
    if (j < 64)
      olo &= ~(1ull << j);
    else
      ohi &= ~(1ull << (j - 64));
    int y = 0;
    if (vt.fixed) {
      y = hypot(f0.x, f0.y) > 1e-12 ? 0 : 1;
      if (y) {
        olo ^= vt.fut_lo;
        ohi ^= vt.fut_hi;
      }
    }
    W[(size_t)j * Bt + b] = make_double4(f0.x, f0.y, f1.x, f1.y);
    if (F) F[(size_t)j * Bt + b] = (unsigned char)(y | (ov << 1));
  }
}

// ------------------------------------------------------------------------------------------------
// Final value and log-scale per item (gpu_kernel.py:126-170): value = E[0], logscale =
// ln2 * sum_j e_j, with e_0 = 1 and e_j from the maximum after step j-1.  An all-zero
// table ends the sum as in the reference (value 0); a non-finite maximum yields NaN.
template <typename S>
__global__ void scan_finalize_kernel(const S* __restrict__ E, const u64* __restrict__ maxbuf, int n, int Bt,
                                     int count, S* __restrict__ out_value, double* __restrict__ out_logscale) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= count) return;
  long long esum = 0;
  bool zero = false, bad = false;
  double m2prev = 1.0;
  for (int j = 0; j < n; ++j) {
    esum += scale_exponent(m2prev);
    const double m2 = max_value<S>(maxbuf[(size_t)j * Bt + b]);
    if (!isfinite(m2)) {
      bad = true;
      break;
    }
    if (!(m2 > 0.0)) {
      zero = true;
      break;
    }
    m2prev = m2;
  }
  S re = E[2 * (size_t)b], im = E[2 * (size_t)b + 1];
  if (zero) re = im = (S)0;
  if (bad) re = im = (S)NAN;
  out_value[2 * (size_t)b] = re;
  out_value[2 * (size_t)b + 1] = im;
  out_logscale[b] = (double)esum * 0.69314718055994530942;
}

// The same over a chunk of tiles: item i is item i % Bt of tile i / Bt, whose final
// table starts (i / Bt) * e_stride entries into E; maxima rows are `stride` items long.
template <typename S>
__global__ void scan_finalize_chunk_kernel(const S* __restrict__ E, u64 e_stride, int lbt,
                                           const u64* __restrict__ maxbuf, int n, int stride, int count,
                                           S* __restrict__ out_value, double* __restrict__ out_logscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  long long esum = 0;
  bool zero = false, bad = false;
  double m2prev = 1.0;
  for (int j = 0; j < n; ++j) {
    esum += scale_exponent(m2prev);
    const double m2 = max_value<S>(maxbuf[(size_t)j * stride + i]);
    if (!isfinite(m2)) {
      bad = true;
      break;
    }
    if (!(m2 > 0.0)) {
      zero = true;
      break;
    }
    m2prev = m2;
  }
  const u64 e = ((u64)(i >> lbt) * e_stride + (u64)(i & ((1 << lbt) - 1))) * 2;
  S re = E[e], im = E[e + 1];
  if (zero) re = im = (S)0;
  if (bad) re = im = (S)NAN;
  out_value[2 * (size_t)i] = re;
  out_value[2 * (size_t)i + 1] = im;
  out_logscale[i] = (double)esum * 0.69314718055994530942;
}

// ------------------------------------------------------------------------------------------------
// Largest batch tile per precision: a lane owns at most 4 chunks (complex128: gathered
// two at a time) or, with float32 arithmetic, 4 chunks of two items.
int scan_max_tile(int precision) {
  if (precision == RGS_PREC_C128) return 128;
  if (precision == RGS_PREC_C64_F32) return 256;
  return 128;
}

size_t ScanLayout::total() const { return off_max + bytes_max; }

int scan_layout(const Plan& plan, int Bt, int precision, ScanLayout& L) {
  if (Bt < 1 || Bt > 512 || (Bt & (Bt - 1))) return fail(RGS_ERR_ARG, "batch_tile must be a power of two in [1, 512]");
  if (precision < RGS_PREC_C64 || precision > RGS_PREC_C128) return fail(RGS_ERR_ARG, "unknown precision");
  if (!plan.exec_ok) return fail(RGS_ERR_UNSUPPORTED, plan.exec_reason);
  const size_t esize = precision == RGS_PREC_C128 ? 16 : 8;
  if (Bt > scan_max_tile(precision))
    return fail(RGS_ERR_ARG, "batch_tile above the maximum for this precision (rgs_scan_max_batch_tile)");
  L.Bt = Bt;
  L.esize = esize;
  L.bytes_buf = align_up(((size_t)1 << plan.rmax) * (size_t)Bt * esize, 256);
  L.bytes_w = align_up((size_t)plan.n * Bt * sizeof(double4), 256);
  L.bytes_f = align_up((size_t)plan.n * Bt, 256);
  L.bytes_max = align_up((size_t)plan.n * Bt * sizeof(u64), 256);
  L.off_buf0 = 0;
  L.off_buf1 = L.bytes_buf;
  L.off_w = 2 * L.bytes_buf;
  L.off_f = L.off_w + L.bytes_w;
  L.off_max = L.off_f + L.bytes_f;
  return RGS_OK;
}

// A chunk of S tiles whose small positions -- the leading and trailing positions whose
// input and output ranks are at most kSmallRank -- run as one launch over all S tiles:
// those tables are tiny, and one launch per tile and position would be launch-bound.  The
// positions in between run tile by tile through two full-size tables as before.
int scan_chunk_layout(const Plan& plan, int Bt, int precision, int S, ChunkLayout& L) {
  ScanLayout base;
  int rc = scan_layout(plan, Bt, precision, base);
  if (rc) return rc;
  if (S < 1) return fail(RGS_ERR_ARG, "chunk must hold at least one tile");
  const int n = plan.n;
  int h = 0, t = 0;
  small_runs(plan, h, t);
  int rs = 0, rmid = 0;
  for (int j = 0; j < n; ++j) {
    const int r = std::max(plan.steps[j].r_in, plan.steps[j].r_out);
    if (j < h || j >= t)
      rs = std::max(rs, r);
    else
      rmid = std::max(rmid, r);
  }
  L.Bt = Bt;
  L.S = S;
  L.h = h;
  L.t = t;
  L.esize = base.esize;
  L.e_stride = (unsigned long long)Bt << rs;
  L.bytes_small = align_up((size_t)S * L.e_stride * L.esize, 256);
  L.bytes_big = h < t ? align_up(((size_t)Bt << rmid) * L.esize, 256) : 0;
  const size_t items = (size_t)S * Bt;
  L.off_small0 = 0;
  L.off_small1 = L.bytes_small;
  L.off_big0 = 2 * L.bytes_small;
  L.off_big1 = L.off_big0 + L.bytes_big;
  L.off_w = L.off_big1 + L.bytes_big;
  L.off_f = L.off_w + align_up((size_t)n * items * sizeof(double4), 256);
  L.off_max = L.off_f + align_up((size_t)n * items, 256);
  L.total = L.off_max + align_up((size_t)n * items * sizeof(u64), 256);
  return RGS_OK;
}

int scan_chunk_tiles(int Bt) { return std::max(2, kChunkItems / Bt); }

namespace {

template <typename S, typename M, int VE, int CPL, int MODE, int NC, int NG0>
cudaError_t launch_row(dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevStep& st, const u64* T,
                       const double4* W, const unsigned char* F, const u64* mp, u64* mc, int lbt, int unit,
                       u64 es) {
  scan_row_kernel<S, M, VE, MODE, NC, CPL, NG0><<<grid, 256, 0, s>>>((const S*)Ein, (S*)Eout, st, T, W, F, mp, mc,
                                                                     lbt, unit, es);
  return cudaGetLastError();
}

template <typename S, typename M, int VE, int CPL>
cudaError_t launch_modes(dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevStep& st, const u64* T,
                         const double4* W, const unsigned char* F, const u64* mp, u64* mc, int lbt, int unit,
                         u64 es) {
#define RGS_ROW(MODE, NC, NG0) \
  launch_row<S, M, VE, CPL, MODE, NC, NG0>(grid, s, Ein, Eout, st, T, W, F, mp, mc, lbt, unit, es)
  if (st.mode == MODE_PAIR) {
    // The combos with kappa = 0 come first: all of them, or half (kappa is linear in the combo).
    if (st.ncombos == 1) return RGS_ROW(MODE_PAIR, 1, 1);
    if (st.ncombos == 2) return st.ng0 == 2 ? RGS_ROW(MODE_PAIR, 2, 2) : RGS_ROW(MODE_PAIR, 2, 1);
    return st.ng0 == 4 ? RGS_ROW(MODE_PAIR, 4, 4) : RGS_ROW(MODE_PAIR, 4, 2);
  }
  if (st.mode == MODE_MERGE) {
    if (st.ncombos == 1) return RGS_ROW(MODE_MERGE, 1, 1);
    return RGS_ROW(MODE_MERGE, 2, 2);
  }
  if (st.ncombos == 1) return RGS_ROW(MODE_FIXED, 1, 1);
  return RGS_ROW(MODE_FIXED, 2, 2);
#undef RGS_ROW
}

// Launch geometry of one step: chunk size, chunks per lane, and a grid of 256-thread
// blocks with enough warps for every row (capped; the kernel strides over the rest).
struct StepGeometry {
  int VE, CPL;
  long long blocks;
};

StepGeometry step_geometry(int precision, int Bt, const DevStep& st, int device) {
  StepGeometry g;
  const int lbt = __builtin_ctz((unsigned)Bt);
  g.VE = (precision != RGS_PREC_C128 && Bt >= 2) ? 2 : 1;
  const int lC = lbt - (g.VE == 2 ? 1 : 0);
  const int lL = lC < 5 ? lC : 5;
  g.CPL = 1 << (lC - lL);
  const int loads = precision == RGS_PREC_C64 ? 4 : 8;  // LoadsInFlight of the kernel
  const int group = std::min(g.CPL, (precision == RGS_PREC_C64_F32) ? 4 : 2);  // ChunkGroup of the kernel
  const int U = (st.ncombos * group >= loads) ? 1 : loads / (st.ncombos * group);
  const unsigned long long items = st.mode == MODE_PAIR ? (1ull << (st.r_out - 1)) : (1ull << st.r_out);
  const unsigned long long per_warp = (unsigned long long)U << (5 - lL);
  const unsigned long long warps = (items + per_warp - 1) / per_warp;
  const long long cap = (long long)sm_count(device) * 16;
  g.blocks = std::max<long long>(1, std::min<long long>((long long)((warps + 7) / 8), cap));
  return g;
}

// One position over `tiles` tiles (grid.y) whose tables lie `es` entries apart.
cudaError_t launch_step(int precision, int Bt, int device, cudaStream_t s, const void* Ein, void* Eout,
                        const DevStep& st, const u64* T, const double4* W, const unsigned char* F, const u64* mp,
                        u64* mc, int unit, int tiles = 1, u64 es = 0) {
  const StepGeometry g = step_geometry(precision, Bt, st, device);
  const int lbt = __builtin_ctz((unsigned)Bt);
  const dim3 grid((unsigned)g.blocks, (unsigned)tiles);
#define RGS_MODES(S_, M_, VE_, CPL_) \
  launch_modes<S_, M_, VE_, CPL_>(grid, s, Ein, Eout, st, T, W, F, mp, mc, lbt, unit, es)
  if (precision == RGS_PREC_C128) {
    if (g.CPL == 1) return RGS_MODES(double, double, 1, 1);
    if (g.CPL == 2) return RGS_MODES(double, double, 1, 2);
    return RGS_MODES(double, double, 1, 4);
  }
  if (precision == RGS_PREC_C64) {
    if (g.VE == 1) return RGS_MODES(float, double, 1, 1);
    if (g.CPL == 1) return RGS_MODES(float, double, 2, 1);
    return RGS_MODES(float, double, 2, 2);
  }
  if (g.VE == 1) return RGS_MODES(float, float, 1, 1);
  if (g.CPL == 1) return RGS_MODES(float, float, 2, 1);
  if (g.CPL == 2) return RGS_MODES(float, float, 2, 2);
  return RGS_MODES(float, float, 2, 4);
#undef RGS_MODES
}

int pair_nc(int code) { return code == PC_P1 ? 1 : (code == PC_P4H ? 4 : 2); }

// Fused pair (j, j + 1) over `tiles` tiles: grid of 256-thread blocks whose warp count is
// a multiple of the row's column slices (a warp keeps one slice).
cudaError_t launch_pair(int precision, int Bt, int device, cudaStream_t s, const void* Ein, void* Eout,
                        const DevPair& P, const u64* tables, const double4* WA, const double4* WB, const u64* mp,
                        u64* mA, u64* mc, int tiles = 1, u64 es = 0) {
  const int lbt = __builtin_ctz((unsigned)Bt);
  const int VE = (precision != RGS_PREC_C128 && Bt >= 2) ? 2 : 1;
  const int lC = lbt - (VE == 2 ? 1 : 0);
  const int lL = lC < 5 ? lC : 5;
  const int lS = lC - lL;
  if (lS > 3) return cudaErrorInvalidValue;  // more column slices than warps in a block
  const int loads = pair_nc(P.codeA) * pair_nc(P.codeB);
  const int U = loads >= RGS_PAIR_LOADS ? 1 : RGS_PAIR_LOADS / loads;
  const unsigned long long groups = 1ull << (P.m - P.dw);
  const unsigned long long per_warp = (unsigned long long)U << (5 - lL);
  const unsigned long long warps = ((groups + per_warp - 1) / per_warp) << lS;
  const long long cap = (long long)sm_count(device) * 16;
  const long long blocks = std::max<long long>(1, std::min<long long>((long long)((warps + 7) / 8), cap));
  const dim3 grid((unsigned)blocks, (unsigned)tiles);
  if (precision == RGS_PREC_C128) return launch_pair_c128(VE, grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
  if (precision == RGS_PREC_C64) return launch_pair_c64(VE, grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
  return launch_pair_f32(VE, grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
}

}  // namespace

cudaError_t scan_launch_pair(int precision, int Bt, int device, const DevPair& P, const void* Ein, void* Eout,
                             const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA, u64* mc,
                             cudaStream_t s) {
  return launch_pair(precision, Bt, device, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc);
}

cudaError_t scan_launch_pair_gram(int precision, int Bt, int blocks, const DevPair& P, const void* Ein,
                                  const u64* tables, const double4* WA, const u64* mp, double* partial,
                                  cudaStream_t s) {
  const int lbt = __builtin_ctz((unsigned)Bt);
  const int VE = (precision != RGS_PREC_C128 && Bt >= 2) ? 2 : 1;
  const int lC = lbt - (VE == 2 ? 1 : 0);
  const int lL = lC < 5 ? lC : 5;
  if (lC - lL > 3) return cudaErrorInvalidValue;  // more column slices than warps in a block
  const dim3 grid((unsigned)blocks);
  if (precision == RGS_PREC_C128) return launch_pair_gram_c128(VE, grid, s, Ein, P, tables, WA, mp, lbt, partial);
  if (precision == RGS_PREC_C64) return launch_pair_gram_c64(VE, grid, s, Ein, P, tables, WA, mp, lbt, partial);
  return launch_pair_gram_f32(VE, grid, s, Ein, P, tables, WA, mp, lbt, partial);
}

namespace {

// The sweep as segments: one position, or a fused pair (plan.pair_at).
struct Segment {
  int j, len, pair;
};
std::vector<Segment> segments_of(const Plan& plan, int from, int to) {
  std::vector<Segment> out;
  for (int j = from; j < to;) {
    const int pa = plan.pair_at.empty() ? -1 : plan.pair_at[j];
    if (pa >= 0 && j + 1 < to) {
      out.push_back({j, 2, pa});
      j += 2;
    } else {
      out.push_back({j, 1, -1});
      j += 1;
    }
  }
  return out;
}

// One segment over `tiles` tiles: rows of weights / maxima start at W / mx (item stride
// `stride` between positions).
cudaError_t launch_segment(const Plan& plan, const Segment& g, int precision, int Bt, int device, cudaStream_t s,
                           const void* Ein, void* Eout, const u64* tables, const double4* W,
                           const unsigned char* F, u64* mx, size_t stride, int tiles, u64 es) {
  const int j = g.j;
  if (g.len == 2)
    return launch_pair(precision, Bt, device, s, Ein, Eout, plan.pairs[g.pair], tables, W + (size_t)j * stride,
                       W + (size_t)(j + 1) * stride, mx + (size_t)(j - 1) * stride, mx + (size_t)j * stride,
                       mx + (size_t)(j + 1) * stride, tiles, es);
  const DevStep& st = plan.dev[j];
  return launch_step(precision, Bt, device, s, Ein, Eout, st, tables + st.table_off, W + (size_t)j * stride,
                     F ? F + (size_t)j * stride : nullptr, j ? mx + (size_t)(j - 1) * stride : nullptr,
                     mx + (size_t)j * stride, j == 0, tiles, es);
}

bool plan_has_fixed(const Plan& p) {
  for (auto& st : p.steps)
    if (!st.free) return true;
  return false;
}

}  // namespace

int scan_pick_chunk(const Plan& plan, int Bt, int precision, size_t ws_bytes, ChunkLayout& C, int* S_out) {
  *S_out = 0;
  for (int S = scan_chunk_tiles(Bt); S >= 2; S >>= 1) {
    int rc = scan_chunk_layout(plan, Bt, precision, S, C);
    if (rc) return rc;
    if (C.total <= ws_bytes) {
      *S_out = S;
      return RGS_OK;
    }
  }
  return RGS_OK;
}

int scan_launch_count(const Plan& plan, long long batch, int Bt, int precision, size_t ws_bytes, long long* out) {
  if (batch < 0) return fail(RGS_ERR_ARG, "batch must be >= 0");
  ScanLayout L;
  int rc = scan_layout(plan, Bt, precision, L);
  if (rc) return rc;
  ChunkLayout C;
  int S = 0;
  if ((rc = scan_pick_chunk(plan, Bt, precision, ws_bytes, C, &S))) return rc;
  const long long n = plan.n;
  long long total = 0;
  if (S < 2) {
    total = (batch + Bt - 1) / Bt * ((long long)segments_of(plan, 0, (int)n).size() + 2);
  } else {
    const long long stride = (long long)S * Bt;
    const long long nh = (long long)segments_of(plan, 0, C.h).size();
    const long long nm = (long long)segments_of(plan, C.h, C.t).size();
    const long long nt = (long long)segments_of(plan, std::max(C.t, C.h), (int)n).size();
    for (long long first = 0; first < batch; first += stride) {
      const long long tiles = (std::min(stride, batch - first) + Bt - 1) / Bt;
      total += 1 + nh;
      if (C.h < C.t) total += tiles * nm + (C.t == n ? tiles : 0);
      if (C.t < n || C.h == n) total += nt + 1;
    }
  }
  *out = total;
  return RGS_OK;
}

namespace {

// Tile-by-tile sweep (every position, one launch per tile): the path for workspaces sized
// by scan_layout alone.
int scan_run_tiles(Plan& plan, const double* U, const u64* bits, const double* fvec, long long batch, int precision,
                   void* out_value, double* out_logscale, void* workspace, size_t ws_bytes, int Bt,
                   cudaStream_t stream, ScanStats* stats) {
  if (batch < 0) return fail(RGS_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return RGS_OK;
  if (!out_value || !out_logscale || !workspace) return fail(RGS_ERR_ARG, "null output or workspace pointer");
  if (!fvec && (!U || !bits)) return fail(RGS_ERR_ARG, "need unitaries and bits, or contraction vectors");
  ScanLayout L;
  int rc = scan_layout(plan, Bt, precision, L);
  if (rc) return rc;
  if (ws_bytes < L.total()) return fail(RGS_ERR_OOM, "workspace smaller than one tile's layout (rgs_scan_workspace_bytes)");
  if (((uintptr_t)workspace & 255) != 0) return fail(RGS_ERR_ARG, "workspace must be 256-byte aligned");
  int device = 0;
  rc = bind_device_of(workspace, &device);
  if (rc) return rc;
  const Plan::DeviceCopy* dc = nullptr;
  rc = plan_device_copy(plan, device, &dc);
  if (rc) return rc;

  char* ws = (char*)workspace;
  void* buf[2] = {ws + L.off_buf0, ws + L.off_buf1};
  double4* W = (double4*)(ws + L.off_w);
  unsigned char* F = plan_has_fixed(plan) ? (unsigned char*)(ws + L.off_f) : nullptr;
  u64* maxbuf = (u64*)(ws + L.off_max);
  const u64* tables = (const u64*)dc->tables;
  long long launches = 0;
  const std::vector<Segment> segs = segments_of(plan, 0, plan.n);

  for (long long first = 0; first < batch; first += Bt) {
    const int count = (int)std::min<long long>(Bt, batch - first);
    scan_weights_kernel<<<(Bt + 127) / 128, 128, 0, stream>>>((const DevVert*)dc->verts, plan.n, (const double2*)U,
                                                              bits, (const double2*)fvec, first, count, Bt, W, F);
    RGS_CUDA_TRY(cudaGetLastError());
    RGS_CUDA_TRY(cudaMemsetAsync(maxbuf, 0, (size_t)plan.n * Bt * sizeof(u64), stream));
    launches += 1;
    int cur = 0;
    for (const Segment& g : segs) {
      RGS_CUDA_TRY(launch_segment(plan, g, precision, Bt, device, stream, buf[cur], buf[cur ^ 1], tables, W, F,
                                  maxbuf, (size_t)Bt, 1, 0));
      cur ^= 1;
      launches += 1;
    }
    const void* fin = buf[cur];
    if (precision == RGS_PREC_C128)
      scan_finalize_kernel<double><<<(count + 127) / 128, 128, 0, stream>>>(
          (const double*)fin, maxbuf, plan.n, Bt, count, (double*)out_value + 2 * first, out_logscale + first);
    else
      scan_finalize_kernel<float><<<(count + 127) / 128, 128, 0, stream>>>(
          (const float*)fin, maxbuf, plan.n, Bt, count, (float*)out_value + 2 * first, out_logscale + first);
    RGS_CUDA_TRY(cudaGetLastError());
    launches += 1;
  }
  if (stats) stats->launches = launches;
  return RGS_OK;
}

}  // namespace

int scan_run(Plan& plan, const double* U, const u64* bits, const double* fvec, long long batch, int precision,
             void* out_value, double* out_logscale, void* workspace, size_t ws_bytes, int Bt, cudaStream_t stream,
             ScanStats* stats) {
  if (batch < 0) return fail(RGS_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return RGS_OK;
  if (!out_value || !out_logscale || !workspace) return fail(RGS_ERR_ARG, "null output or workspace pointer");
  if (!fvec && (!U || !bits)) return fail(RGS_ERR_ARG, "need unitaries and bits, or contraction vectors");
  ChunkLayout C;
  int S = 0;
  int rc = scan_pick_chunk(plan, Bt, precision, ws_bytes, C, &S);
  if (rc) return rc;
  if (S < 2)
    return scan_run_tiles(plan, U, bits, fvec, batch, precision, out_value, out_logscale, workspace, ws_bytes, Bt,
                          stream, stats);
  if (((uintptr_t)workspace & 255) != 0) return fail(RGS_ERR_ARG, "workspace must be 256-byte aligned");
  int device = 0;
  rc = bind_device_of(workspace, &device);
  if (rc) return rc;
  const Plan::DeviceCopy* dc = nullptr;
  rc = plan_device_copy(plan, device, &dc);
  if (rc) return rc;

  const int n = plan.n, h = C.h, t = C.t;
  const int stride = S * Bt;  // items per row of the weights, flags and maxima
  const size_t esize = C.esize;
  char* ws = (char*)workspace;
  char* small[2] = {ws + C.off_small0, ws + C.off_small1};
  char* big[2] = {ws + C.off_big0, ws + C.off_big1};
  double4* W = (double4*)(ws + C.off_w);
  unsigned char* F = plan_has_fixed(plan) ? (unsigned char*)(ws + C.off_f) : nullptr;
  u64* maxbuf = (u64*)(ws + C.off_max);
  const u64* tables = (const u64*)dc->tables;
  const int lbt = __builtin_ctz((unsigned)Bt);
  long long launches = 0;
  const std::vector<Segment> head = segments_of(plan, 0, h), mid = segments_of(plan, h, t),
                             tail = segments_of(plan, std::max(t, h), n);

  for (long long first = 0; first < batch; first += stride) {
    const int count = (int)std::min<long long>(stride, batch - first);
    const int tiles = (count + Bt - 1) / Bt;
    scan_weights_kernel<<<(stride + 127) / 128, 128, 0, stream>>>((const DevVert*)dc->verts, n, (const double2*)U,
                                                                  bits, (const double2*)fvec, first, count, stride, W,
                                                                  F);
    RGS_CUDA_TRY(cudaGetLastError());
    RGS_CUDA_TRY(cudaMemsetAsync(maxbuf, 0, (size_t)n * stride * sizeof(u64), stream));
    launches += 1;
    int cur = 0;
    // Leading small positions: all tiles of the chunk per launch.
    for (const Segment& g : head) {
      RGS_CUDA_TRY(launch_segment(plan, g, precision, Bt, device, stream, small[cur], small[cur ^ 1], tables, W, F,
                                  maxbuf, (size_t)stride, tiles, C.e_stride));
      cur ^= 1;
      launches += 1;
    }
    // Middle positions, tile by tile: from the tile's slice of the small buffer through the
    // full-size tables to its slice of the other small buffer (or to the final value).
    if (!mid.empty()) {
      for (int k = 0; k < tiles; ++k) {
        const size_t koff = (size_t)k * C.e_stride * esize;
        const size_t ik = (size_t)k * Bt;
        int bb = 0;
        for (size_t gi = 0; gi < mid.size(); ++gi) {
          const bool first_seg = gi == 0, last_seg = gi + 1 == mid.size();
          const void* in = first_seg ? (const void*)(small[cur] + koff) : (const void*)big[bb];
          void* out = (last_seg && t < n) ? (void*)(small[cur ^ 1] + koff) : (void*)big[first_seg ? 0 : bb ^ 1];
          RGS_CUDA_TRY(launch_segment(plan, mid[gi], precision, Bt, device, stream, in, out, tables, W + ik,
                                      F ? F + ik : nullptr, maxbuf + ik, (size_t)stride, 1, 0));
          if (!first_seg) bb ^= 1;
          launches += 1;
        }
        if (t == n) {  // the sweep ends in the full-size tables: finalise this tile now
          const int kc = std::min(Bt, count - k * Bt);
          const void* fin = big[mid.size() == 1 ? 0 : bb];
          if (precision == RGS_PREC_C128)
            scan_finalize_chunk_kernel<double><<<(kc + 127) / 128, 128, 0, stream>>>(
                (const double*)fin, 0ull, lbt, maxbuf + ik, n, stride, kc,
                (double*)out_value + 2 * (first + (long long)ik), out_logscale + first + (long long)ik);
          else
            scan_finalize_chunk_kernel<float><<<(kc + 127) / 128, 128, 0, stream>>>(
                (const float*)fin, 0ull, lbt, maxbuf + ik, n, stride, kc,
                (float*)out_value + 2 * (first + (long long)ik), out_logscale + first + (long long)ik);
          RGS_CUDA_TRY(cudaGetLastError());
          launches += 1;
        }
      }
      if (t < n) cur ^= 1;
    }
    // Trailing small positions: all tiles per launch again.
    if (t < n || h == n) {
      for (const Segment& g : tail) {
        RGS_CUDA_TRY(launch_segment(plan, g, precision, Bt, device, stream, small[cur], small[cur ^ 1], tables, W,
                                    F, maxbuf, (size_t)stride, tiles, C.e_stride));
        cur ^= 1;
        launches += 1;
      }
      if (precision == RGS_PREC_C128)
        scan_finalize_chunk_kernel<double><<<(count + 127) / 128, 128, 0, stream>>>(
            (const double*)small[cur], C.e_stride, lbt, maxbuf, n, stride, count, (double*)out_value + 2 * first,
            out_logscale + first);
      else
        scan_finalize_chunk_kernel<float><<<(count + 127) / 128, 128, 0, stream>>>(
            (const float*)small[cur], C.e_stride, lbt, maxbuf, n, stride, count, (float*)out_value + 2 * first,
            out_logscale + first);
      RGS_CUDA_TRY(cudaGetLastError());
      launches += 1;
    }
  }
  if (stats) stats->launches = launches;
  return RGS_OK;
}

// ------------------------------------------------------------------------------------------------
cudaError_t scan_launch_weights(const DevVert* verts, int n, const double* U, const u64* bits, const double* fvec,
                                long long first, int count, int Bt, void* W, unsigned char* F, cudaStream_t stream) {
  scan_weights_kernel<<<(Bt + 127) / 128, 128, 0, stream>>>(verts, n, (const double2*)U, bits, (const double2*)fvec,
                                                            first, count, Bt, (double4*)W, F);
  return cudaGetLastError();
}

cudaError_t scan_launch_step(int precision, int Bt, int device, const DevStep& st, const void* Ein, void* Eout,
                             const u64* T, const void* W, const unsigned char* F, const u64* maxprev, u64* maxcur,
                             bool unit_input, cudaStream_t stream) {
  return launch_step(precision, Bt, device, stream, Ein, Eout, st, T, (const double4*)W, F, maxprev, maxcur,
                     unit_input ? 1 : 0);
}

cudaError_t scan_launch_finalize(int precision, const void* E, const u64* maxbuf, int n, int Bt, int count,
                                 void* out_value, double* out_logscale, cudaStream_t stream) {
  if (precision == RGS_PREC_C128)
    scan_finalize_kernel<double><<<(count + 127) / 128, 128, 0, stream>>>((const double*)E, maxbuf, n, Bt, count,
                                                                          (double*)out_value, out_logscale);
  else
    scan_finalize_kernel<float><<<(count + 127) / 128, 128, 0, stream>>>((const float*)E, maxbuf, n, Bt, count,
                                                                         (float*)out_value, out_logscale);
  return cudaGetLastError();
}

}  // namespace rgs
