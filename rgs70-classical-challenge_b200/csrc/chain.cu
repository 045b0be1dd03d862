// Exact Born sampling and conditional marginals through the scan (chain rule).
//
// For a scan order v_0..v_{n-1} and contraction vectors f_q = U_q[x_q, :], the
// environment E_S after the first k positions gives the prefix marginal
//   p(x_{v_0..v_{k-1}}) = 2^{-k} sum_c |E_S[c]|^2
// (trace out the unmeasured suffix: unitarity of each U_q, then Parseval over the
// syndrome subspace).  So p(x_v = x | prefix) = M_x / (M_0 + M_1) with M_x the squared
// norm of the table after position v with branch x.  Per position this file runs
//   chain_gram_kernel   : a 2x2 Gram matrix per item from one read of E (no writes), from
//                         which both branch masses follow; skipped on positions whose
//                         step pairs each input row with two output rows through one
//                         combo, where M_0 and M_1 are known in closed form
//   chain_decide_kernel : per item, exact inverse-CDF choice of x_v (or the given bit),
//                         log p(x_v | prefix), and the weights of the chosen branch
//   scan step kernel    : the chosen branch, with the usual power-of-two renormalisation
// so a sample costs one scan sweep plus one read of the tables of the other positions.
// Fused pairs of the plan (positions j, j + 1): x_j as above; then one pass over j's
// input forms j's outputs in registers and accumulates the Gram matrix of position j + 1
// (scan_pair_kernel, GRAM mode, no stores, float64 sums) unless j + 1 is analytic;
// x_{j+1}; then the pair kernel writes the output of j + 1.  The table between the two
// positions never reaches memory: per pair 2 reads of j's input and 1 write instead of 1
// read, 3 passes over the intermediate table and 1 write.
// The final table is the amplitude of the drawn string, returned like rgs_scan_amplitudes.
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

constexpr int kMassBlocks = 296;   // 2 blocks (the occupancy of the Gram kernel) on each of 148 SMs
constexpr int kChainMaxTile = 128;  // largest batch tile (complex64); complex128: 64
constexpr int kDecideThreads = 128;  // threads of the per-item decision block

// Gram matrix of one position per item, from one read of the table (no writes).  Every
// output of the step is alpha f(0) + beta f(1) with f = U_v[x, :] s: in pair mode row c'
// has alpha = sum_{y=0} e, beta = sum_{y=1} (-1)^par e, and row c'^t the mirror image
// (alpha = sum_{y=1} e, beta = sum_{y=0} (-1)^par e); in merge mode alpha = sum e,
// beta = sum (-1)^par e.  Both branch masses then follow from
//   G = sum over outputs of ( |alpha|^2, |beta|^2, alpha conj(beta) ):
//   M_x / s^2 = G00 |U_x0|^2 + G11 |U_x1|^2 + 2 Re(G01 U_x0 conj(U_x1)),
// one accumulation for the two branches.  Layout and geometry as scan_row_kernel.
template <typename S, int VE, int MODE, int NC, int CPL>
__global__ void __launch_bounds__(256, 2) chain_gram_kernel(const S* __restrict__ Ein, const __grid_constant__ DevStep st,
                                                            const u64* __restrict__ T, double* __restrict__ partial,
                                                            int lbt, int unit_input) {
  constexpr int U = RowsPerIter<NC, CPL, LoadsInFlight<S, double>::value>::value;
  constexpr int NI = CPL * VE;
  __shared__ double red[8][kChainMaxTile][4];  // per warp, per item: G00, G11, Re G01, Im G01
  const int Bt = 1 << lbt;
  const int lC = lbt - (VE == 2 ? 1 : 0);
  const int lL = lC < 5 ? lC : 5;
  const int lR = 5 - lL;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int sub = lane >> lL;
  const int l = lane & ((1 << lL) - 1);

  const u64 items = (MODE == MODE_PAIR) ? (1ull << (st.r_out - 1)) : (1ull << st.r_out);
  const u64 warp = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u64 per_iter = (u64)U << lR;
  const u64 mask = (1ull << st.r_in) - 1ull;
  double g[NI][4];
#pragma unroll
  for (int i = 0; i < NI; ++i) g[i][0] = g[i][1] = g[i][2] = g[i][3] = 0.0;

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
          double aar = 0.0, aai = 0.0, bar = 0.0, bai = 0.0;  // alpha, beta of row c'
          double car = 0.0, cai = 0.0, dbr = 0.0, dbi = 0.0;  // alpha, beta of row c'^t (pair mode)
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            const double er = (double)e[u][k][j].re(v), ei = (double)e[u][k][j].im(v);
            const double sr = pc[u][k] ? -er : er, si = pc[u][k] ? -ei : ei;
            if (MODE == MODE_PAIR) {
              if (yy[u][k]) {
                car += er;
                cai += ei;
                bar += sr;
                bai += si;
              } else {
                aar += er;
                aai += ei;
                dbr += sr;
                dbi += si;
              }
            } else {
              aar += er;
              aai += ei;
              bar += sr;
              bai += si;
            }
          }
          g[i][0] = fma(aar, aar, fma(aai, aai, g[i][0]));
          g[i][1] = fma(bar, bar, fma(bai, bai, g[i][1]));
          g[i][2] = fma(aar, bar, fma(aai, bai, g[i][2]));
          g[i][3] = fma(aai, bar, fma(-aar, bai, g[i][3]));
          if (MODE == MODE_PAIR) {
            g[i][0] = fma(car, car, fma(cai, cai, g[i][0]));
            g[i][1] = fma(dbr, dbr, fma(dbi, dbi, g[i][1]));
            g[i][2] = fma(car, dbr, fma(cai, dbi, g[i][2]));
            g[i][3] = fma(cai, dbr, fma(-car, dbi, g[i][3]));
          }
        }
    }
  }

  // Deterministic reduction: lanes sharing items (shuffles), warps (shared memory, fixed
  // order), then one partial per block and item.
#pragma unroll
  for (int i = 0; i < NI; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double a = g[i][q];
      for (int off = 16; off >= (1 << lL); off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      g[i][q] = a;
    }
  for (int b = threadIdx.x; b < Bt; b += blockDim.x)
    for (int wv = 0; wv < 8; ++wv) red[wv][b][0] = red[wv][b][1] = red[wv][b][2] = red[wv][b][3] = 0.0;
  __syncthreads();
  if (sub == 0) {
#pragma unroll
    for (int k = 0; k < CPL; ++k)
#pragma unroll
      for (int v = 0; v < VE; ++v) {
        const int i = k * VE + v, b = ((l + (k << lL)) * VE) + v;
#pragma unroll
        for (int q = 0; q < 4; ++q) red[wib][b][q] = g[i][q];
      }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < Bt; b += blockDim.x) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) {
      t0 += red[wv][b][0];
      t1 += red[wv][b][1];
      t2 += red[wv][b][2];
      t3 += red[wv][b][3];
    }
    double* p = partial + ((size_t)blockIdx.x * Bt + b) * 4;
    p[0] = t0;
    p[1] = t1;
    p[2] = t2;
    p[3] = t3;
  }
}

// Per item: the Gram matrix (sum over blocks of the partials, fixed order; or, on a
// position whose step pairs every input row with two output rows through one combo,
// G = identity: there M_x = sum|E|^2 s^2 (|U_x0|^2 + |U_x1|^2) for both x -- the new
// syndrome bit is uniform, and no pass over the table is needed); the branch masses M_x;
// x_v drawn with the item's uniform (x = 0 iff u (M0 + M1) < M0) or taken from the given
// bits; then the chosen branch's weights for the step kernel, the sampled bit,
// log p(x_v | prefix) and the conditional probability p(x_v = 1 | prefix).
__global__ void chain_decide_kernel(const double* __restrict__ partial, int nblocks, int analytic, int Bt, int count,
                                    int j, int v, const double2* __restrict__ U, int mode_given, u64* __restrict__ bits,
                                    long long first, const double* __restrict__ uniforms, int n, u64 seed,
                                    double4* __restrict__ Wj, double* __restrict__ logp, float* __restrict__ cond1,
                                    int* __restrict__ status) {
  // One block per item: threads sum strided block partials, then a fixed shuffle tree
  // per warp and the warps in order (deterministic).
  __shared__ double wsum[kDecideThreads / 32][4];
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (b >= count) {
    if (threadIdx.x == 0) Wj[b] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  double g0 = 1.0, g1 = 1.0, g2 = 0.0, g3 = 0.0;
  if (!analytic) {
    g0 = g1 = 0.0;
    // The first kLoadsAhead partials of this thread are loaded before any is summed (one
    // memory round trip instead of one per partial); the sums keep the order k = t, t + 128, ...
    constexpr int kLoadsAhead = 4;
    double4 pk[kLoadsAhead];
#pragma unroll
    for (int q = 0; q < kLoadsAhead; ++q) {
      const int k = threadIdx.x + q * (int)blockDim.x;
      if (k < nblocks) pk[q] = *reinterpret_cast<const double4*>(partial + ((size_t)k * Bt + b) * 4);
    }
#pragma unroll
    for (int q = 0; q < kLoadsAhead; ++q) {
      if (threadIdx.x + q * (int)blockDim.x >= nblocks) break;
      g0 += pk[q].x;
      g1 += pk[q].y;
      g2 += pk[q].z;
      g3 += pk[q].w;
    }
    for (int k = threadIdx.x + kLoadsAhead * (int)blockDim.x; k < nblocks; k += blockDim.x) {
      const double4 p = *reinterpret_cast<const double4*>(partial + ((size_t)k * Bt + b) * 4);
      g0 += p.x;
      g1 += p.y;
      g2 += p.z;
      g3 += p.w;
    }
    for (int off = 16; off; off >>= 1) {
      g0 += __shfl_xor_sync(0xffffffffu, g0, off);
      g1 += __shfl_xor_sync(0xffffffffu, g1, off);
      g2 += __shfl_xor_sync(0xffffffffu, g2, off);
      g3 += __shfl_xor_sync(0xffffffffu, g3, off);
    }
    if (lane == 0) {
      wsum[wid][0] = g0;
      wsum[wid][1] = g1;
      wsum[wid][2] = g2;
      wsum[wid][3] = g3;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      g0 = g1 = g2 = g3 = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        g0 += wsum[w][0];
        g1 += wsum[w][1];
        g2 += wsum[w][2];
        g3 += wsum[w][3];
      }
    }
  }
  if (threadIdx.x) return;
  const double m0 = branch_mass(U + (v * 2 + 0) * 2, g0, g1, g2, g3);
  const double m1 = branch_mass(U + (v * 2 + 1) * 2, g0, g1, g2, g3);
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
template <typename S, int VE, int CPL, int MODE, int NC>
cudaError_t launch_gram(dim3 grid, cudaStream_t s, const void* Ein, const DevStep& st, const u64* T, double* partial,
                        int lbt, int unit) {
  chain_gram_kernel<S, VE, MODE, NC, CPL><<<grid, 256, 0, s>>>((const S*)Ein, st, T, partial, lbt, unit);
  return cudaGetLastError();
}

// Positions that need the Gram pass: pair mode with two or four combos, merge mode.
template <typename S, int VE, int CPL>
cudaError_t gram_modes(dim3 grid, cudaStream_t s, const void* Ein, const DevStep& st, const u64* T, double* partial,
                       int lbt, int unit) {
  if (st.mode == MODE_PAIR) {
    if (st.ncombos == 2) return launch_gram<S, VE, CPL, MODE_PAIR, 2>(grid, s, Ein, st, T, partial, lbt, unit);
    return launch_gram<S, VE, CPL, MODE_PAIR, 4>(grid, s, Ein, st, T, partial, lbt, unit);
  }
  if (st.ncombos == 1) return launch_gram<S, VE, CPL, MODE_MERGE, 1>(grid, s, Ein, st, T, partial, lbt, unit);
  return launch_gram<S, VE, CPL, MODE_MERGE, 2>(grid, s, Ein, st, T, partial, lbt, unit);
}

cudaError_t launch_gram_step(int precision, int Bt, int blocks, cudaStream_t s, const void* Ein, const DevStep& st,
                             const u64* T, double* partial, int unit) {
  const int lbt = __builtin_ctz((unsigned)Bt);
  const int VE = (precision != RGS_PREC_C128 && Bt >= 2) ? 2 : 1;
  const int lC = lbt - (VE == 2 ? 1 : 0);
  const int CPL = 1 << (lC - (lC < 5 ? lC : 5));
  const dim3 grid((unsigned)blocks);
  if (precision == RGS_PREC_C128) {
    if (CPL == 1) return gram_modes<double, 1, 1>(grid, s, Ein, st, T, partial, lbt, unit);
    return gram_modes<double, 1, 2>(grid, s, Ein, st, T, partial, lbt, unit);
  }
  if (VE == 1) return gram_modes<float, 1, 1>(grid, s, Ein, st, T, partial, lbt, unit);
  if (CPL == 1) return gram_modes<float, 2, 1>(grid, s, Ein, st, T, partial, lbt, unit);
  return gram_modes<float, 2, 2>(grid, s, Ein, st, T, partial, lbt, unit);
}

}  // namespace

int chain_max_tile(int precision) { return precision == RGS_PREC_C128 ? kChainMaxTile / 2 : kChainMaxTile; }

int chain_layout(const Plan& plan, int Bt, int precision, ChainLayout& L) {
  if (Bt > chain_max_tile(precision)) return fail(RGS_ERR_ARG, "batch_tile above the chain sampler maximum");
  int rc = scan_layout(plan, Bt, precision, L.scan);
  if (rc) return rc;
  L.mass_blocks = kMassBlocks;
  L.off_partial = L.scan.total();
  L.off_status = L.off_partial + align_up((size_t)L.mass_blocks * Bt * 4 * sizeof(double), 256);
  L.total = L.off_status + 256;
  return RGS_OK;
}

// Kernel launches of chain_run per batch tile, following its schedule: bit clearing
// (sampling) and log p zeroing (when asked), per position the Gram pass (unless analytic)
// and the decision, per single position its scan step, per fused pair the pair Gram pass
// (unless the second position is analytic) and the pair kernel, and the finalisation.
long long chain_launches_per_tile(const Plan& plan, bool mode_given, bool with_logp) {
  auto analytic = [&](int j) { return plan.dev[j].mode == MODE_PAIR && plan.dev[j].ncombos == 1; };
  const bool fuse = !plan.pair_at.empty();
  long long c = (mode_given ? 0 : 1) + (with_logp ? 1 : 0);
  for (int j = 0; j < plan.n;) {
    const int pa = fuse ? plan.pair_at[j] : -1;
    if (pa >= 0 && j + 1 < plan.n) {
      c += (analytic(j) ? 0 : 1) + 1 + (analytic(j + 1) ? 0 : 1) + 1 + 1;
      j += 2;
    } else {
      c += (analytic(j) ? 0 : 1) + 1 + 1;
      j += 1;
    }
  }
  return c + 1;
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
  // Fused pairs of positions (the plan's pairs), every precision.
  const bool fuse = !plan.pair_at.empty();
  RGS_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), stream));
  for (long long first = 0; first < count; first += Bt) {
    const int cnt = (int)std::min<long long>(Bt, count - first);
    if (!mode_given) chain_clear_bits_kernel<<<(cnt + 127) / 128, 128, 0, stream>>>(bits, first, cnt);
    if (out_logp) chain_zero_kernel<<<(cnt + 127) / 128, 128, 0, stream>>>(out_logp, first, cnt);
    RGS_CUDA_TRY(cudaMemsetAsync(maxbuf, 0, (size_t)plan.n * Bt * sizeof(u64), stream));
    // Branch masses of position j (the Gram pass over its input, unless analytic), then
    // the choice of x_{v_j} and the chosen branch's weights.
    auto decide = [&](int j, const void* in) -> cudaError_t {
      const DevStep& st = plan.dev[j];
      const int analytic = (st.mode == MODE_PAIR && st.ncombos == 1) ? 1 : 0;
      if (!analytic && in) {
        cudaError_t e = launch_gram_step(precision, Bt, L.mass_blocks, stream, in, st, tables + st.table_off, partial,
                                         j == 0);
        if (e != cudaSuccess) return e;
      }
      chain_decide_kernel<<<Bt, kDecideThreads, 0, stream>>>(
          partial, L.mass_blocks, analytic, Bt, cnt, j, st.v, U2, mode_given, bits, first, uniforms, plan.n, seed,
          W + (size_t)j * Bt, out_logp, out_cond1, status);
      return cudaGetLastError();
    };
    int seg = 0;
    for (int j = 0; j < plan.n; ++seg) {
      const void* in = buf[seg & 1];
      void* out = buf[(seg + 1) & 1];
      const int pa = fuse ? plan.pair_at[j] : -1;
      if (pa >= 0 && j + 1 < plan.n) {
        // Fused pair (j, j + 1): x_j as usual; B's branch masses from a pass over j's
        // input that forms j's outputs in registers (nothing written); x_{j+1}; then the
        // pair kernel writes B's output.  j's output table never reaches memory.
        const DevPair& P = plan.pairs[pa];
        const DevStep& sb = plan.dev[j + 1];
        const bool analytic_b = sb.mode == MODE_PAIR && sb.ncombos == 1;
        RGS_CUDA_TRY(decide(j, in));
        if (!analytic_b)
          RGS_CUDA_TRY(scan_launch_pair_gram(precision, Bt, L.mass_blocks, P, in, tables, W + (size_t)j * Bt,
                                             maxbuf + (size_t)(j - 1) * Bt, partial, stream));
        RGS_CUDA_TRY(decide(j + 1, nullptr));
        RGS_CUDA_TRY(scan_launch_pair(precision, Bt, device, P, in, out, tables, W + (size_t)j * Bt,
                                      W + (size_t)(j + 1) * Bt, maxbuf + (size_t)(j - 1) * Bt, maxbuf + (size_t)j * Bt,
                                      maxbuf + (size_t)(j + 1) * Bt, stream));
        j += 2;
      } else {
        const DevStep& st = plan.dev[j];
        RGS_CUDA_TRY(decide(j, in));
        RGS_CUDA_TRY(scan_launch_step(precision, Bt, device, st, in, out, tables + st.table_off, W + (size_t)j * Bt,
                                      nullptr, j ? maxbuf + (size_t)(j - 1) * Bt : nullptr, maxbuf + (size_t)j * Bt,
                                      j == 0, stream));
        j += 1;
      }
    }
    RGS_CUDA_TRY(scan_launch_finalize(precision, buf[seg & 1], maxbuf, plan.n, Bt, cnt,
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
