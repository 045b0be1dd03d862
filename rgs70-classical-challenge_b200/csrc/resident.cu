// Shared-memory-resident batch executor: many small instances in one persistent launch.
//
// The streaming executor (scan.cu) runs one launch per scan position because a
// rank-30 table lives in HBM.  Instances of rank <= 13 (complex64) fit in shared
// memory with room for several items, so a block keeps both ping-pong tables on chip
// and runs a whole sweep -- every position of one instance for up to 64 items -- with
// no HBM traffic besides the inputs, the byte tables (L1/L2 resident) and the outputs.
// Blocks take work units from an atomic counter (largest units first), so instances of
// different sizes and the two kinds of work share one launch:
//   kind 0: amplitudes of given bitstrings (the streaming executor's arithmetic,
//           bit for bit: same weights, same fma order, same renormalisation);
//   kind 1: exact chain-rule samples (chain.cu's algorithm: both branch masses from the
//           position's Gram matrix, one read of the table, or in closed form; inverse-CDF
//           choice with the Philox uniform of (seed, item, position); then the chosen
//           branch as one step).
// Table layout per block: E[c][b] (b fastest) for the unit's nb items.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>

#include "common.hpp"
#include "philox.cuh"
#include "plan.hpp"
#include "resident.hpp"
#include "scan_device.cuh"

namespace rgs {

ResDevice::~ResDevice() {
  if (device < 0) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  if (insts) cudaFree(insts);
  if (work) cudaFree(work);
  if (counter) cudaFree(counter);
  if (prev >= 0) cudaSetDevice(prev);
}

namespace {

template <typename S>
struct Pair2;
template <>
struct Pair2<float> {
  typedef float2 T;
};
template <>
struct Pair2<double> {
  typedef double2 T;
};

struct ItemState {
  u64 lo, hi;      // bitstring: the input (amplitudes) or the bits drawn so far (samples)
  u64 olo, ohi;    // affine syndrome offsets owed to later positions (fixed vertices)
  double m2;       // max |E|^2 after the previous position (1 before the first)
  double logp;     // sum of the log conditionals (samples)
  long long esum;  // sum of the renormalisation exponents
  int done;        // 0 running, 1 the table became zero, 2 non-finite
  int flags;       // this position: y | ov << 1
};

// Weights of one item for one position, as scan_row_kernel prepares them (s = 2^-e).
template <typename M>
__device__ __forceinline__ void branch_weights(double2 f0, double2 f1, double s, int mode, int yfix, Cx<M>& a,
                                               Cx<M>& b) {
  double ar = f0.x * s, ai = f0.y * s, br = f1.x * s, bi = f1.y * s;
  if (mode == MODE_MERGE) {
    const double pr = ar + br, pim = ai + bi, mr = ar - br, mi = ai - bi;
    ar = pr;
    ai = pim;
    br = mr;
    bi = mi;
  } else if (mode == MODE_FIXED && yfix) {
    ar = br;
    ai = bi;
  }
  a = Cx<M>{(M)ar, (M)ai};
  b = Cx<M>{(M)br, (M)bi};
}

// Both outputs (pair mode) or the one output of row `p0` for item b: the combination of
// scan_row_kernel's inner loop, combos in the same order.
template <typename S, typename M>
__device__ __forceinline__ void row_outputs(const typename Pair2<S>::T* __restrict__ Ein, const DevStep& st, u64 p0,
                                            int lnb, int b, bool unit, const Cx<M>& wA, const Cx<M>& wB, int ov,
                                            int yf, Cx<M>& oa, Cx<M>& ob) {
  const u64 mask = (1ull << st.r_in) - 1ull;
  oa = Cx<M>{(M)0, (M)0};
  ob = Cx<M>{(M)0, (M)0};
  for (int k = 0; k < st.ncombos; ++k) {
    const u64 p = p0 ^ st.combos[k];
    const u64 cc = p & mask;
    const int y = (int)((p >> st.r_in) & 1ull);
    const int par = (__popcll(cc & st.beta) & 1) ^ ov;
    M er = (M)1, ei = (M)0;
    if (!unit) {
      const typename Pair2<S>::T e = Ein[(cc << lnb) + b];
      er = (M)e.x;
      ei = (M)e.y;
    }
    if (st.mode == MODE_PAIR) {
      Cx<M> wa = y ? wB : wA;
      Cx<M> wb = y ? wA : wB;
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
    } else if (st.mode == MODE_MERGE) {
      cmad(oa, er, ei, par ? wB : wA);
    } else {
      Cx<M> w = wA;
      if (yf & par) {
        w.re = -w.re;
        w.im = -w.im;
      }
      cmad(oa, er, ei, w);
    }
  }
}

// Gram-matrix terms of row p0 for item b (chain_gram_kernel's accumulation).
template <typename S>
__device__ __forceinline__ void row_gram(const typename Pair2<S>::T* __restrict__ Ein, const DevStep& st, u64 p0,
                                         int lnb, int b, bool unit, double& g0, double& g1, double& g2, double& g3) {
  const u64 mask = (1ull << st.r_in) - 1ull;
  double aar = 0.0, aai = 0.0, bar = 0.0, bai = 0.0, car = 0.0, cai = 0.0, dbr = 0.0, dbi = 0.0;
  for (int k = 0; k < st.ncombos; ++k) {
    const u64 p = p0 ^ st.combos[k];
    const u64 cc = p & mask;
    const int y = (int)((p >> st.r_in) & 1ull);
    const int par = __popcll(cc & st.beta) & 1;
    double er = 1.0, ei = 0.0;
    if (!unit) {
      const typename Pair2<S>::T e = Ein[(cc << lnb) + b];
      er = (double)e.x;
      ei = (double)e.y;
    }
    const double sr = par ? -er : er, si = par ? -ei : ei;
    if (st.mode == MODE_PAIR && y) {
      car += er;
      cai += ei;
      bar += sr;
      bai += si;
    } else {
      aar += er;
      aai += ei;
      if (st.mode == MODE_PAIR) {
        dbr += sr;
        dbi += si;
      } else {
        bar += sr;
        bai += si;
      }
    }
  }
  g0 = fma(aar, aar, fma(aai, aai, g0));
  g1 = fma(bar, bar, fma(bai, bai, g1));
  g2 = fma(aar, bar, fma(aai, bai, g2));
  g3 = fma(aai, bar, fma(-aar, bai, g3));
  if (st.mode == MODE_PAIR) {
    g0 = fma(car, car, fma(cai, cai, g0));
    g1 = fma(dbr, dbr, fma(dbi, dbi, g1));
    g2 = fma(car, dbr, fma(cai, dbi, g2));
    g3 = fma(cai, dbr, fma(-car, dbi, g3));
  }
}

// The item's maximum |E|^2 of the last step (over the threads that own its rows), with
// the zero / non-finite bookkeeping of scan_finalize_kernel.
template <typename S>
__device__ __forceinline__ void fold_max(const u64* redm, int tid, int lnb, int slots, ItemState& s) {
  u64 m = 0;
  for (int k = 0; k < slots; ++k) {
    const u64 x = redm[tid + (k << lnb)];
    m = m > x ? m : x;
  }
  const double m2 = max_value<S>(m);
  if (!s.done) {
    if (!isfinite(m2))
      s.done = 2;
    else if (!(m2 > 0.0))
      s.done = 1;
  }
  s.m2 = m2;
}

// Per position: phase A (all threads: the Gram pass of a sample unit; item threads: the
// previous position's maximum, then the weights of an amplitude unit; thread 0: the next
// step record), a barrier, [sample units: decision and weights, a barrier], the step
// (rows of the chosen branch, per-thread maxima), a barrier.
template <typename S, typename M, int kResThreads, int kResidentSmem>
__global__ void __launch_bounds__(kResThreads, 512 / kResThreads)
    resident_kernel(const ResInstance* __restrict__ insts, const ResWork* __restrict__ work, long long nwork,
                    int* __restrict__ counter) {
  typedef typename Pair2<S>::T V;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[4][kResThreads];  // Gram partials, structure of arrays (no bank conflicts)
  __shared__ u64 redm[kResThreads];
  __shared__ Cx<M> wA[kMaxResItems], wB[kMaxResItems];
  __shared__ ItemState ist[kMaxResItems];
  __shared__ DevStep sst[2];
  __shared__ long long s_unit;
  const int tid = threadIdx.x;
  const size_t cap = (size_t)kResidentSmem / (2 * sizeof(V));
  V* const bufs[2] = {(V*)smem, (V*)smem + cap};

  for (;;) {
    if (tid == 0) s_unit = (long long)atomicAdd(counter, 1);
    __syncthreads();
    const long long w = s_unit;
    if (w >= nwork) break;
    const ResWork wk = work[w];
    const ResInstance in = insts[wk.inst];
    const double2* U2 = (const double2*)in.U;
    const int nb = in.nb, lnb = __ffs(nb) - 1;
    const bool sample = wk.kind == 1;
    const int b = tid & (nb - 1);
    const int slot = tid >> lnb, slots = kResThreads >> lnb;
    if (tid < nb) {
      ItemState s;
      s.lo = s.hi = s.olo = s.ohi = 0;
      s.m2 = 1.0;
      s.logp = 0.0;
      s.esum = 0;
      s.done = 0;
      s.flags = 0;
      if (!sample && tid < wk.num) {
        const long long item = wk.first + tid;
        s.lo = in.bits[2 * item];
        s.hi = in.bits[2 * item + 1];
      }
      ist[tid] = s;
    }
    if (tid == 0) sst[0] = in.steps[0];
    __syncthreads();
    int cur = 0;
    for (int j = 0; j < in.n; ++j) {
      const DevStep& st = sst[j & 1];
      const int mode = st.mode, v = st.v;
      const u64* T = in.tables + st.table_off;
      const V* Ein = bufs[cur];
      V* Eout = bufs[cur ^ 1];
      const bool unit = j == 0;
      const u64 rows = mode == MODE_PAIR ? (1ull << (st.r_out - 1)) : (1ull << st.r_out);
      const bool analytic = mode == MODE_PAIR && st.ncombos == 1;

      // ---- phase A
      if (sample && !analytic) {
        // Gram matrix of this position from the table (chain_gram_kernel's accumulation).
        double g0 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;
        for (u64 r = slot; r < rows; r += slots) {
          const u64 ca = mode == MODE_PAIR ? deposit_zero(r, st.pi) : r;
          row_gram<S>(Ein, st, table_lookup(T, st.nbytes, ca), lnb, b, unit, g0, g1, g2, g3);
        }
        red[0][tid] = g0;
        red[1][tid] = g1;
        red[2][tid] = g2;
        red[3][tid] = g3;
      }
      if (tid < nb) {
        ItemState& s = ist[tid];
        if (j > 0) fold_max<S>(redm, tid, lnb, slots, s);
        if (!sample) {
          // Weights of the given bit (scan_weights_kernel), with the fixed-vertex offsets.
          const DevVert vt = in.verts[j];
          const double sc = ldexp(1.0, -scale_exponent(s.m2));
          const int x = (int)((v < 64 ? (s.lo >> v) : (s.hi >> (v - 64))) & 1ull);
          const double2 f0 = U2[(v * 2 + x) * 2 + 0], f1 = U2[(v * 2 + x) * 2 + 1];
          const int ov = (int)((j < 64 ? (s.olo >> j) : (s.ohi >> (j - 64))) & 1ull);
          if (j < 64)
            s.olo &= ~(1ull << j);
          else
            s.ohi &= ~(1ull << (j - 64));
          int y = 0;
          if (vt.fixed) {
            y = hypot(f0.x, f0.y) > 1e-12 ? 0 : 1;
            if (y) {
              s.olo ^= vt.fut_lo;
              s.ohi ^= vt.fut_hi;
            }
          }
          Cx<M> wa, wb;
          branch_weights<M>(f0, f1, sc, mode, y, wa, wb);
          if (tid >= wk.num) wa = wb = Cx<M>{(M)0, (M)0};
          wA[tid] = wa;
          wB[tid] = wb;
          s.flags = y | (ov << 1);
          if (!s.done) s.esum += scale_exponent(s.m2);
        }
      }
      if (tid == 0 && j + 1 < in.n) sst[(j + 1) & 1] = in.steps[j + 1];
      __syncthreads();

      if (sample) {
        // Both branch masses (or their closed form), the decision (chain_decide_kernel).
        if (tid < nb) {
          double g0 = 1.0, g1 = 1.0, g2 = 0.0, g3 = 0.0;
          if (!analytic) {
            g0 = g1 = 0.0;
            for (int k = 0; k < slots; ++k) {
              const int q = tid + (k << lnb);
              g0 += red[0][q];
              g1 += red[1][q];
              g2 += red[2][q];
              g3 += red[3][q];
            }
          }
          const double m0 = branch_mass(U2 + (v * 2 + 0) * 2, g0, g1, g2, g3);
          const double m1 = branch_mass(U2 + (v * 2 + 1) * 2, g0, g1, g2, g3);
          ItemState& s = ist[tid];
          int x = 0;
          if (tid < wk.num) {
            const double tot = m0 + m1;
            if (!(tot > 0.0) || !isfinite(tot)) {
              atomicExch(counter + 1, 1);
            } else {
              const double u = philox_uniform(in.seed, (u64)(wk.first + tid), j);
              x = (u * tot < m0) ? 0 : 1;
              s.logp += log((x ? m1 : m0) / tot);
            }
            if (x) {
              if (v < 64)
                s.lo |= 1ull << v;
              else
                s.hi |= 1ull << (v - 64);
            }
          }
          const double sc = ldexp(1.0, -scale_exponent(s.m2));
          Cx<M> wa, wb;
          branch_weights<M>(U2[(v * 2 + x) * 2 + 0], U2[(v * 2 + x) * 2 + 1], sc, mode, 0, wa, wb);
          if (tid >= wk.num) wa = wb = Cx<M>{(M)0, (M)0};
          wA[tid] = wa;
          wB[tid] = wb;
          s.flags = 0;
          if (!s.done) s.esum += scale_exponent(s.m2);
        }
        __syncthreads();
      }

      // ---- the step: rows c' (and c'^t) of the chosen branch, per-thread maxima.
      {
        const Cx<M> wa = wA[b], wb = wB[b];
        const int fl = ist[b].flags;
        S mx = (S)0;
#pragma unroll 2
        for (u64 r = slot; r < rows; r += slots) {
          const u64 ca = mode == MODE_PAIR ? deposit_zero(r, st.pi) : r;
          Cx<M> oa, ob;
          row_outputs<S, M>(Ein, st, table_lookup(T, st.nbytes, ca), lnb, b, unit, wa, wb, (fl >> 1) & 1, fl & 1,
                            oa, ob);
          const S ar = (S)oa.re, ai = (S)oa.im;
          Eout[(ca << lnb) + b] = V{ar, ai};
          mx = fmax(mx, norm2(ar, ai));
          if (mode == MODE_PAIR) {
            const S br = (S)ob.re, bi = (S)ob.im;
            Eout[((ca ^ st.t) << lnb) + b] = V{br, bi};
            mx = fmax(mx, norm2(br, bi));
          }
        }
        redm[tid] = max_bits<S>(mx);
      }
      cur ^= 1;
      __syncthreads();
    }
    if (tid < wk.num) {
      ItemState s = ist[tid];
      fold_max<S>(redm, tid, lnb, slots, s);
      const V e = bufs[cur][tid];  // row 0 of the final table
      S re = e.x, im = e.y;
      if (s.done == 1) re = im = (S)0;
      if (s.done == 2) re = im = (S)NAN;
      const long long item = wk.first + tid;
      const double ls = (double)s.esum * 0.69314718055994530942;
      if (sample) {
        in.sample_bits[2 * item] = s.lo;
        in.sample_bits[2 * item + 1] = s.hi;
        reinterpret_cast<V*>(in.sample_value)[item] = V{re, im};
        in.sample_logscale[item] = ls;
        if (in.sample_logp) in.sample_logp[item] = s.logp;
      } else {
        reinterpret_cast<V*>(in.out_value)[item] = V{re, im};
        in.out_logscale[item] = ls;
      }
    }
    // The next unit's first barrier orders these reads before ist and s_unit are rewritten.
  }
}

template <typename S, typename M, int V>
int launch_variant(const ResDevice& dev, cudaStream_t stream, int blocks) {
  constexpr int T = kResThreadsOf[V], SM = kResSmemOf[V];
  static std::mutex mu;
  static bool attr_set[64] = {false};
  {
    std::lock_guard<std::mutex> lock(mu);
    if (dev.device >= 0 && dev.device < 64 && !attr_set[dev.device]) {
      RGS_CUDA_TRY(cudaFuncSetAttribute(resident_kernel<S, M, T, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM));
      attr_set[dev.device] = true;
    }
  }
  resident_kernel<S, M, T, SM><<<blocks, T, SM, stream>>>(dev.insts, dev.work, dev.nwork, dev.counter);
  RGS_CUDA_TRY(cudaGetLastError());
  return RGS_OK;
}

template <typename S, typename M>
int launch_kernel(const ResDevice& dev, cudaStream_t stream, int blocks) {
  if (dev.variant == 2) return launch_variant<S, M, 2>(dev, stream, blocks);
  if (dev.variant == 1) return launch_variant<S, M, 1>(dev, stream, blocks);
  return launch_variant<S, M, 0>(dev, stream, blocks);
}

size_t table_entries(int precision, int variant) {
  const size_t esize = precision == RGS_PREC_C128 ? 16 : 8;
  return (size_t)kResSmemOf[variant] / (2 * esize);
}

}  // namespace

int resident_max_rank(int precision, int variant) {
  const size_t cap = table_entries(precision, variant);
  int r = 0;
  while (((size_t)2 << r) <= cap) ++r;
  return r;
}

int resident_items(int rmax, int precision, int variant) {
  if (rmax < 0 || rmax > resident_max_rank(precision, variant)) return 0;
  const size_t cap = table_entries(precision, variant);
  int nb = kMaxResItems;
  while (nb > 1 && ((size_t)nb << rmax) > cap) nb >>= 1;
  return nb;
}

int resident_prepare(const std::vector<ResInstance>& insts_in, int precision, int variant, ResDevice& dev) {
  if (dev.device < 0) return fail(RGS_ERR_ARG, "batch has no device");
  if (variant < 0 || variant >= kResVariants) return fail(RGS_ERR_ARG, "unknown launch variant");
  std::vector<ResInstance> insts(insts_in);
  for (auto& in : insts) {
    in.nb = resident_items(in.rmax, precision, variant);
    if (in.nb < 1) return fail(RGS_ERR_UNSUPPORTED, "an instance's tables do not fit this launch variant");
  }
  std::vector<ResWork> work;
  std::vector<double> cost;
  for (size_t i = 0; i < insts.size(); ++i) {
    const ResInstance& in = insts[i];
    const double c = (double)in.n * (double)(1ull << in.rmax);
    for (int kind = 0; kind < 2; ++kind) {
      const long long total = kind ? in.nsamples : in.count;
      for (long long f = 0; f < total; f += in.nb) {
        ResWork w;
        w.inst = (int)i;
        w.kind = kind;
        w.first = f;
        w.num = (int)std::min<long long>(in.nb, total - f);
        w.pad = 0;
        work.push_back(w);
        cost.push_back(kind ? 2.0 * c : c);
      }
    }
  }
  // Largest units first: a greedy longest-processing-time order for the work counter.
  std::vector<size_t> idx(work.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
  std::vector<ResWork> sorted(work.size());
  for (size_t k = 0; k < idx.size(); ++k) sorted[k] = work[idx[k]];
  (void)precision;

  RGS_CUDA_TRY(cudaSetDevice(dev.device));
  if (!dev.counter) RGS_CUDA_TRY(cudaMalloc(&dev.counter, 2 * sizeof(int)));
  if (insts.size() > dev.insts_cap) {
    if (dev.insts) RGS_CUDA_TRY(cudaFree(dev.insts));
    dev.insts = nullptr;
    RGS_CUDA_TRY(cudaMalloc(&dev.insts, insts.size() * sizeof(ResInstance)));
    dev.insts_cap = insts.size();
  }
  if (sorted.size() > dev.work_cap) {
    if (dev.work) RGS_CUDA_TRY(cudaFree(dev.work));
    dev.work = nullptr;
    RGS_CUDA_TRY(cudaMalloc(&dev.work, sorted.size() * sizeof(ResWork)));
    dev.work_cap = sorted.size();
  }
  if (!insts.empty())
    RGS_CUDA_TRY(cudaMemcpy(dev.insts, insts.data(), insts.size() * sizeof(ResInstance), cudaMemcpyHostToDevice));
  if (!sorted.empty())
    RGS_CUDA_TRY(cudaMemcpy(dev.work, sorted.data(), sorted.size() * sizeof(ResWork), cudaMemcpyHostToDevice));
  dev.nwork = (long long)sorted.size();
  dev.variant = variant;
  return RGS_OK;
}

int resident_launch(const ResDevice& dev, int precision, cudaStream_t stream, int* blocks_out) {
  if (dev.device < 0 || !dev.counter) return fail(RGS_ERR_ARG, "batch is not prepared");
  RGS_CUDA_TRY(cudaSetDevice(dev.device));
  RGS_CUDA_TRY(cudaMemsetAsync(dev.counter, 0, 2 * sizeof(int), stream));
  const int per_sm = 512 / kResThreadsOf[dev.variant];
  const int blocks = (int)std::max<long long>(1, std::min<long long>(dev.nwork, (long long)sm_count(dev.device) * per_sm));
  if (blocks_out) *blocks_out = dev.nwork ? blocks : 0;
  if (!dev.nwork) return RGS_OK;
  if (precision == RGS_PREC_C128) return launch_kernel<double, double>(dev, stream, blocks);
  if (precision == RGS_PREC_C64_F32) return launch_kernel<float, float>(dev, stream, blocks);
  return launch_kernel<float, double>(dev, stream, blocks);
}

}  // namespace rgs
