// Exact Born sampling and conditional marginals through the scan (chain rule).
//
// For a scan order v_0..v_{n-1} and contraction vectors f_q = U_q[x_q, :], the
// environment E_S after the first k positions gives the prefix marginal
//   p(x_{v_0..v_{k-1}}) = 2^{-k} sum_c |E_S[c]|^2
// (trace out the unmeasured suffix: unitarity of each U_q, then Parseval over the
// syndrome subspace).  So p(x_v = x | prefix) = M_x / (M_0 + M_1) with M_x the squared
// norm of the table after position v with branch x.  Per position this file runs
//   chain_mass_kernel   : both branches' sum |E'|^2 per item from one read of E (no writes)
//   chain_decide_kernel : per item, exact inverse-CDF choice of x_v (or the given bit),
//                         log p(x_v | prefix), and the weights of the chosen branch
//   scan step kernel    : the chosen branch, with the usual power-of-two renormalisation
// so a sample costs one read of every table plus one scan sweep.  The final table is the
// amplitude of the drawn string, returned like rgs_scan_amplitudes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "common.hpp"
#include "chain.hpp"
#include "philox.cuh"
#include "plan.hpp"
#include "scan.hpp"
#include "scan_device.cuh"
#include "scan_row.cuh"

namespace rgs {

namespace {

constexpr int kMassBlocks = 296;  // 2 blocks (the occupancy of the mass kernel) on each of 148 SMs

// Both branches of one position, reduced to per-item sums of |E'|^2 (double).  Layout
// and geometry as scan_row_kernel; U_v rows (u0 = U_v[0,:], u1 = U_v[1,:]) are the same
// for every item, the scale 2^-e is per item.
template <typename S, typename M, int VE, int MODE, int NC, int CPL>
__global__ void __launch_bounds__(256, 2) chain_mass_kernel(const S* __restrict__ Ein, const __grid_constant__ DevStep st,
                                                            const u64* __restrict__ T, const double2* __restrict__ Uv,
                                                            const u64* __restrict__ maxprev,
                                                            double* __restrict__ partial, int lbt, int unit_input) {
  constexpr int U = RowsPerIter<NC, CPL, LoadsInFlight<S, M>::value>::value;
  constexpr int NI = CPL * VE;
  __shared__ double red[8][256][2];  // per warp, per item, per branch
  const int Bt = 1 << lbt;
  const int lC = lbt - (VE == 2 ? 1 : 0);
  const int lL = lC < 5 ? lC : 5;
  const int lR = 5 - lL;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int sub = lane >> lL;
  const int l = lane & ((1 << lL) - 1);

  // Branch weights (scaled per item): x = 0 uses (a0, a1) = u0, x = 1 uses u1.
  Cx<M> w[2][NI][2];
  for (int k = 0; k < CPL; ++k)
    for (int v = 0; v < VE; ++v) {
      const int i = k * VE + v, b = ((l + (k << lL)) * VE) + v;
      const double m2 = maxprev ? max_value<S>(maxprev[b]) : 1.0;
      const double s = ldexp(1.0, -scale_exponent(m2));
      const double4 uu[2] = {make_double4(Uv[0].x, Uv[0].y, Uv[1].x, Uv[1].y),
                             make_double4(Uv[2].x, Uv[2].y, Uv[3].x, Uv[3].y)};
      for (int x = 0; x < 2; ++x) {
        double ar = uu[x].x * s, ai = uu[x].y * s, br = uu[x].z * s, bi = uu[x].w * s;
        if (MODE == MODE_MERGE) {
          const double pr = ar + br, pim = ai + bi, mr = ar - br, mi = ai - bi;
          ar = pr;
          ai = pim;
          br = mr;
          bi = mi;
        }
        w[x][i][0] = Cx<M>{(M)ar, (M)ai};
        w[x][i][1] = Cx<M>{(M)br, (M)bi};
      }
    }

  const u64 items = (MODE == MODE_PAIR) ? (1ull << (st.r_out - 1)) : (1ull << st.r_out);
  const u64 warp = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u64 per_iter = (u64)U << lR;
  const u64 mask = (1ull << st.r_in) - 1ull;
  double acc[NI][2];
  for (int i = 0; i < NI; ++i) acc[i][0] = acc[i][1] = 0.0;

  for (u64 base = warp * per_iter; base < items; base += nwarps * per_iter) {
    u64 cc[U][NC];
    int yy[U][NC], pc[U][NC];
    bool ok[U];
    Chunk<S, VE> e[U][NC][CPL];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 it = base + ((u64)u << lR) + sub;
      ok[u] = it < items;
      const u64 ca = (MODE == MODE_PAIR) ? deposit_zero(it, st.pi) : it;
      const u64 p0 = ok[u] ? table_lookup(T, st.nbytes, ca) : 0ull;
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const u64 p = p0 ^ st.combos[k];
        cc[u][k] = p & mask;
        yy[u][k] = (int)((p >> st.r_in) & 1ull);
        pc[u][k] = __popcll(cc[u][k] & st.beta) & 1;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
          if (unit_input || !ok[u])
            e[u][k][j].unit();
          else
            e[u][k][j].load(Ein, (cc[u][k] << lC) + (u64)(l + (j << lL)));
        }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!ok[u]) continue;
#pragma unroll
      for (int j = 0; j < CPL; ++j)
#pragma unroll
        for (int v = 0; v < VE; ++v) {
          const int i = j * VE + v;
#pragma unroll
          for (int x = 0; x < 2; ++x) {
            Cx<M> oa{(M)0, (M)0}, ob{(M)0, (M)0};
#pragma unroll
            for (int k = 0; k < NC; ++k) {
              const M er = (M)e[u][k][j].re(v), ei = (M)e[u][k][j].im(v);
              const int par = pc[u][k];
              if (MODE == MODE_PAIR) {
                const int y = yy[u][k];
                Cx<M> wa = y ? w[x][i][1] : w[x][i][0];
                Cx<M> wb = y ? w[x][i][0] : w[x][i][1];
                if (y & par) {
                  wa.re = -wa.re;
                  wa.im = -wa.im;
                }
                if ((y ^ 1) & par) {
                  wb.re = -wb.re;
                  wb.im = -wb.im;
                }
                cmad(oa, er, ei, wa);
                cmad(ob, er, ei, wb);
              } else {
                cmad(oa, er, ei, par ? w[x][i][1] : w[x][i][0]);
              }
            }
            // Squared moduli of the values the step kernel would store (rounded to S).
            const S ar = (S)oa.re, ai = (S)oa.im;
            acc[i][x] += (double)norm2(ar, ai);
            if (MODE == MODE_PAIR) {
              const S br = (S)ob.re, bi = (S)ob.im;
              acc[i][x] += (double)norm2(br, bi);
            }
          }
        }
    }
  }

  // Deterministic reduction: lanes sharing items (shuffles), warps (shared memory, fixed
  // order), then one partial per block and item.
#pragma unroll
  for (int i = 0; i < NI; ++i)
#pragma unroll
    for (int x = 0; x < 2; ++x) {
      double a = acc[i][x];
      for (int off = 16; off >= (1 << lL); off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      acc[i][x] = a;
    }
  for (int b = threadIdx.x; b < Bt; b += blockDim.x)
    for (int wv = 0; wv < 8; ++wv) red[wv][b][0] = red[wv][b][1] = 0.0;
  __syncthreads();
  if (sub == 0) {
#pragma unroll
    for (int k = 0; k < CPL; ++k)
#pragma unroll
      for (int v = 0; v < VE; ++v) {
        const int i = k * VE + v, b = ((l + (k << lL)) * VE) + v;
        red[wib][b][0] = acc[i][0];
        red[wib][b][1] = acc[i][1];
      }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < Bt; b += blockDim.x) {
    double s0 = 0.0, s1 = 0.0;
    for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) {
      s0 += red[wv][b][0];
      s1 += red[wv][b][1];
    }
    partial[((size_t)blockIdx.x * Bt + b) * 2 + 0] = s0;
    partial[((size_t)blockIdx.x * Bt + b) * 2 + 1] = s1;
  }
}

// Per item: M_x = sum over blocks of the partials (fixed order); x_v drawn with the
// item's uniform (x = 0 iff u (M0 + M1) < M0) or taken from the given bits; then the
// chosen branch's weights for the step kernel, the sampled bit, log p(x_v | prefix) and
// the conditional probability p(x_v = 1 | prefix).
__global__ void chain_decide_kernel(const double* __restrict__ partial, int nblocks, int Bt, int count, int j, int v,
                                    const double2* __restrict__ U, int mode_given, u64* __restrict__ bits,
                                    long long first, const double* __restrict__ uniforms, int n, u64 seed,
                                    double4* __restrict__ Wj, double* __restrict__ logp, float* __restrict__ cond1,
                                    int* __restrict__ status) {
  // One warp per item: lanes sum strided block partials, then a fixed shuffle tree.
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= Bt) return;
  if (b >= count) {
    if (lane == 0) Wj[b] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  double m0 = 0.0, m1 = 0.0;
  for (int k = lane; k < nblocks; k += 32) {
    m0 += partial[((size_t)k * Bt + b) * 2 + 0];
    m1 += partial[((size_t)k * Bt + b) * 2 + 1];
  }
  for (int off = 16; off; off >>= 1) {
    m0 += __shfl_xor_sync(0xffffffffu, m0, off);
    m1 += __shfl_xor_sync(0xffffffffu, m1, off);
  }
  if (lane) return;
  const double tot = m0 + m1;
  const long long item = first + b;
  int x;
  if (!(tot > 0.0) || !isfinite(tot)) {
    atomicExch(status, 1);
    x = 0;
  } else if (mode_given) {
    const u64 w = bits[2 * item + (v >> 6)];
    x = (int)((w >> (v & 63)) & 1ull);
  } else {
    const double u = uniforms ? uniforms[(size_t)item * n + j] : philox_uniform(seed, (u64)item, j);
    x = (u * tot < m0) ? 0 : 1;
    if (x) bits[2 * item + (v >> 6)] |= 1ull << (v & 63);
  }
  const double2 f0 = U[(v * 2 + x) * 2 + 0], f1 = U[(v * 2 + x) * 2 + 1];
  Wj[b] = make_double4(f0.x, f0.y, f1.x, f1.y);
  if (logp) logp[item] += log((x ? m1 : m0) / tot);
  if (cond1) cond1[(size_t)item * n + j] = (float)(m1 / tot);
}

__global__ void chain_clear_bits_kernel(u64* bits, long long first, int count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < count) {
    bits[2 * (first + b)] = 0;
    bits[2 * (first + b) + 1] = 0;
  }
}

__global__ void chain_zero_kernel(double* x, long long first, int count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < count) x[first + b] = 0.0;
}

// ------------------------------------------------------------------------------- host
template <typename S, typename M, int VE, int CPL, int MODE, int NC>
cudaError_t launch_mass(dim3 grid, cudaStream_t s, const void* Ein, const DevStep& st, const u64* T,
                        const double2* Uv, const u64* mp, double* partial, int lbt, int unit) {
  chain_mass_kernel<S, M, VE, MODE, NC, CPL><<<grid, 256, 0, s>>>((const S*)Ein, st, T, Uv, mp, partial, lbt, unit);
  return cudaGetLastError();
}

template <typename S, typename M, int VE, int CPL>
cudaError_t mass_modes(dim3 grid, cudaStream_t s, const void* Ein, const DevStep& st, const u64* T,
                       const double2* Uv, const u64* mp, double* partial, int lbt, int unit) {
#define RGS_MASS(MODE, NC) launch_mass<S, M, VE, CPL, MODE, NC>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit)
  if (st.mode == MODE_PAIR) {
    if (st.ncombos == 1) return RGS_MASS(MODE_PAIR, 1);
    if (st.ncombos == 2) return RGS_MASS(MODE_PAIR, 2);
    return RGS_MASS(MODE_PAIR, 4);
  }
  if (st.ncombos == 1) return RGS_MASS(MODE_MERGE, 1);
  return RGS_MASS(MODE_MERGE, 2);
#undef RGS_MASS
}

cudaError_t launch_mass_step(int precision, int Bt, int blocks, cudaStream_t s, const void* Ein, const DevStep& st,
                             const u64* T, const double2* Uv, const u64* mp, double* partial, int unit) {
  const int lbt = __builtin_ctz((unsigned)Bt);
  const int VE = (precision != RGS_PREC_C128 && Bt >= 2) ? 2 : 1;
  const int lC = lbt - (VE == 2 ? 1 : 0);
  const int CPL = 1 << (lC - (lC < 5 ? lC : 5));
  const dim3 grid((unsigned)blocks);
  if (precision == RGS_PREC_C128) {
    if (CPL == 1) return mass_modes<double, double, 1, 1>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
    return mass_modes<double, double, 1, 2>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
  }
  if (precision == RGS_PREC_C64) {
    if (VE == 1) return mass_modes<float, double, 1, 1>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
    if (CPL == 1) return mass_modes<float, double, 2, 1>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
    return mass_modes<float, double, 2, 2>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
  }
  if (VE == 1) return mass_modes<float, float, 1, 1>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
  if (CPL == 1) return mass_modes<float, float, 2, 1>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
  return mass_modes<float, float, 2, 2>(grid, s, Ein, st, T, Uv, mp, partial, lbt, unit);
}

}  // namespace

int chain_max_tile(int precision) { return precision == RGS_PREC_C128 ? 64 : 128; }

int chain_layout(const Plan& plan, int Bt, int precision, ChainLayout& L) {
  if (Bt > chain_max_tile(precision)) return fail(RGS_ERR_ARG, "batch_tile above the chain sampler maximum");
  int rc = scan_layout(plan, Bt, precision, L.scan);
  if (rc) return rc;
  L.mass_blocks = kMassBlocks;
  L.off_partial = L.scan.total();
  L.off_status = L.off_partial + align_up((size_t)L.mass_blocks * Bt * 2 * sizeof(double), 256);
  L.total = L.off_status + 256;
  return RGS_OK;
}

int chain_run(Plan& plan, const double* U, long long count, int mode_given, u64 seed, const double* uniforms,
              int precision, unsigned long long* bits, void* out_value, double* out_logscale, double* out_logp,
              float* out_cond1, void* workspace, size_t ws_bytes, int Bt, cudaStream_t stream, bool check) {
  if (count < 0) return fail(RGS_ERR_ARG, "count must be >= 0");
  if (count == 0) return RGS_OK;
  if (!U || !bits || !out_value || !out_logscale || !workspace) return fail(RGS_ERR_ARG, "null pointer argument");
  for (auto& st : plan.steps)
    if (!st.free) return fail(RGS_ERR_UNSUPPORTED, "the chain sampler does not support fixed vertices");
  int device = 0;
  int rc = bind_device_of(workspace, &device);
  if (rc) return rc;
  ChainLayout L;
  if ((rc = chain_layout(plan, Bt, precision, L))) return rc;
  if (ws_bytes < L.total) return fail(RGS_ERR_OOM, "workspace smaller than rgs_chain_workspace_bytes()");
  if (((uintptr_t)workspace & 255) != 0) return fail(RGS_ERR_ARG, "workspace must be 256-byte aligned");
  const Plan::DeviceCopy* dc = nullptr;
  if ((rc = plan_device_copy(plan, device, &dc))) return rc;
  char* ws = (char*)workspace;
  void* buf[2] = {ws + L.scan.off_buf0, ws + L.scan.off_buf1};
  double4* W = (double4*)(ws + L.scan.off_w);
  u64* maxbuf = (u64*)(ws + L.scan.off_max);
  double* partial = (double*)(ws + L.off_partial);
  int* status = (int*)(ws + L.off_status);
  const u64* tables = (const u64*)dc->tables;
  const double2* U2 = (const double2*)U;
  RGS_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), stream));
  for (long long first = 0; first < count; first += Bt) {
    const int cnt = (int)std::min<long long>(Bt, count - first);
    if (!mode_given) chain_clear_bits_kernel<<<(cnt + 127) / 128, 128, 0, stream>>>(bits, first, cnt);
    if (out_logp) chain_zero_kernel<<<(cnt + 127) / 128, 128, 0, stream>>>(out_logp, first, cnt);
    RGS_CUDA_TRY(cudaMemsetAsync(maxbuf, 0, (size_t)plan.n * Bt * sizeof(u64), stream));
    for (int j = 0; j < plan.n; ++j) {
      const DevStep& st = plan.dev[j];
      const int v = st.v;
      RGS_CUDA_TRY(launch_mass_step(precision, Bt, L.mass_blocks, stream, buf[j & 1], st, tables + st.table_off,
                                    U2 + (size_t)v * 4, j ? maxbuf + (size_t)(j - 1) * Bt : nullptr, partial, j == 0));
      chain_decide_kernel<<<(Bt * 32 + 127) / 128, 128, 0, stream>>>(
          partial, L.mass_blocks, Bt, cnt, j, v, U2, mode_given, bits, first, uniforms, plan.n, seed,
          W + (size_t)j * Bt, out_logp, out_cond1, status);
      RGS_CUDA_TRY(cudaGetLastError());
      RGS_CUDA_TRY(scan_launch_step(precision, Bt, device, st, buf[j & 1], buf[(j + 1) & 1], tables + st.table_off,
                                    W + (size_t)j * Bt, nullptr, j ? maxbuf + (size_t)(j - 1) * Bt : nullptr,
                                    maxbuf + (size_t)j * Bt, j == 0, stream));
    }
    RGS_CUDA_TRY(scan_launch_finalize(precision, buf[plan.n & 1], maxbuf, plan.n, Bt, cnt,
                                      (char*)out_value + (size_t)first * (precision == RGS_PREC_C128 ? 16 : 8),
                                      out_logscale + first, stream));
  }
  if (check) {
    int h = 0;
    RGS_CUDA_TRY(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    RGS_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h) return fail(RGS_ERR_ZERO_NORM, "a branch pair had zero or non-finite total mass");
  }
  return RGS_OK;
}

}  // namespace rgs
