// Scan-program compiler (host).  Algorithm of W/upstream_scan/scan_plan.py:35-152
// (whyihaveyou/rgs70-classical-challenge), restated on 128-bit masks.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <map>

namespace rgs {

std::vector<u128> future_masks(int n, const std::vector<std::pair<int, int>>& edges,
                               const std::vector<int>& order) {
  // scan_plan.py:45-55 -- later neighbours of each position, as a mask over positions.
  std::vector<int> where(n, 0);
  for (int p = 0; p < n; ++p) where[order[p]] = p;
  std::vector<u128> later(n, 0);
  for (auto& e : edges) {
    int a = where[e.first], b = where[e.second];
    if (a > b) std::swap(a, b);
    later[a] |= one_at(b);
  }
  return later;
}

namespace {

// Reduce `vec` against `rows` in insertion order (scan_plan.py:35-42).  `used`
// collects the rows added, as a mask over row indices.
inline u128 eliminate(u128 vec, const std::vector<u128>& rows, const std::vector<int>& pivots, u128& used) {
  used = 0;
  for (size_t k = 0; k < rows.size(); ++k) {
    if (bit_of(vec, pivots[k])) {
      vec ^= rows[k];
      used |= one_at((int)k);
    }
  }
  return vec;
}

std::string validate(int n, const std::vector<std::pair<int, int>>& edges, const std::vector<int>& order,
                     const std::vector<uint8_t>& fixed) {
  if (n < 1 || n > 128) return "n must be in [1, 128]";
  if ((int)order.size() != n) return "order must have n entries";
  std::vector<char> seen(n, 0);
  for (int v : order) {
    if (v < 0 || v >= n || seen[v]) return "order must be a permutation of 0..n-1";
    seen[v] = 1;
  }
  for (auto& e : edges) {
    if (e.first < 0 || e.first >= n || e.second < 0 || e.second >= n) return "edge endpoint out of range";
    if (e.first == e.second) return "self-loop in edge list";
  }
  if (!fixed.empty() && (int)fixed.size() != n) return "fixed must have n entries";
  return "";
}

// Compiles the steps; when `keep` is false only ranks are recorded.
void run_compiler(int n, const std::vector<u128>& later, const std::vector<int>& order,
                  const std::vector<uint8_t>& fixed, bool keep, std::vector<PlanStep>& steps,
                  std::vector<int>& ranks) {
  std::vector<u128> basis;
  std::vector<u128> images, rows, columns;
  std::vector<int> pivots;
  ranks.assign(n, 0);
  if (keep) steps.assign(n, PlanStep());
  for (int j = 0; j < n; ++j) {
    const int v = order[j];
    const bool is_free = fixed.empty() || !fixed[v];
    const int r_in = (int)basis.size();
    u128 beta = 0;
    for (int i = 0; i < r_in; ++i)
      if (bit_of(basis[i], j)) beta |= one_at(i);
    images.clear();
    for (auto& b : basis) images.push_back(b & ~one_at(j));
    if (is_free) images.push_back(later[j]);
    rows.clear();
    pivots.clear();
    columns.clear();
    for (auto img : images) {
      u128 used;
      u128 res = eliminate(img, rows, pivots, used);
      if (res) {
        pivots.push_back(lowest_bit(res));
        rows.push_back(res);
        used |= one_at((int)rows.size() - 1);
      }
      columns.push_back(used);
    }
    const int r_out = (int)rows.size();
    ranks[j] = r_out;
    if (keep) {
      PlanStep& st = steps[j];
      st.v = v;
      st.free = is_free;
      st.r_in = r_in;
      st.r_out = r_out;
      st.beta = beta;
      // creator[k]: first column whose highest coefficient bit is k (scan_plan.py:79-83).
      std::vector<int> creator(r_out, -1);
      for (size_t i = 0; i < columns.size(); ++i) {
        if (!columns[i]) continue;
        int top = highest_bit(columns[i]);
        if (creator[top] < 0) creator[top] = (int)i;
      }
      // Right inverse (scan_plan.py:84-91).
      st.lcols.assign(r_out, 0);
      for (int k = 0; k < r_out; ++k) {
        const int i = creator[k];
        u128 pre = one_at(i);
        for (int l = 0; l < k; ++l)
          if (bit_of(columns[i], l)) pre ^= st.lcols[l];
        st.lcols[k] = pre;
      }
      // Kernel (scan_plan.py:92-102).
      st.kernel.clear();
      for (size_t i = 0; i < columns.size(); ++i) {
        if (std::find(creator.begin(), creator.end(), (int)i) != creator.end()) continue;
        u128 vec = one_at((int)i);
        for (int k = 0; k < r_out; ++k)
          if (bit_of(columns[i], k)) vec ^= st.lcols[k];
        st.kernel.push_back(vec);
      }
      st.ycol = is_free ? columns[r_in] : 0;
      st.mcols = columns;
    }
    basis.swap(rows);
  }
}

}  // namespace

void byte_tables(const std::vector<u128>& cols, int nbits, std::vector<u128>& out, int& nbytes) {
  // scan_plan.py:133-145
  nbytes = std::max(1, (nbits + 7) / 8);
  out.assign((size_t)nbytes * 256, 0);
  for (int b = 0; b < nbytes; ++b) {
    for (int value = 0; value < 256; ++value) {
      u128 acc = 0;
      for (int t = 0; t < 8; ++t) {
        int i = 8 * b + t;
        if (i < nbits && ((value >> t) & 1)) acc ^= cols[i];
      }
      out[(size_t)b * 256 + value] = acc;
    }
  }
}

std::vector<u128> kernel_combos(const std::vector<u128>& kernel) {
  // scan_plan.py:148-152 -- span in doubling order.
  std::vector<u128> out{0};
  for (auto k : kernel) {
    size_t m = out.size();
    for (size_t i = 0; i < m; ++i) out.push_back(out[i] ^ k);
  }
  return out;
}

std::string rank_profile(int n, const std::vector<std::pair<int, int>>& edges, const std::vector<int>& order,
                         const std::vector<uint8_t>& fixed, std::vector<int>& ranks) {
  std::string err = validate(n, edges, order, fixed);
  if (!err.empty()) return err;
  std::vector<PlanStep> unused;
  run_compiler(n, future_masks(n, edges, order), order, fixed, false, unused, ranks);
  return "";
}

void small_runs(const Plan& p, int& h, int& t) {
  auto small = [&](int j) { return std::max(p.steps[j].r_in, p.steps[j].r_out) <= kSmallRank; };
  h = 0;
  while (h < p.n && small(h)) ++h;
  t = p.n;
  while (t > h && small(t - 1)) --t;
}

namespace {

u128 apply_cols(const std::vector<u128>& cols, u128 x) {
  u128 r = 0;
  for (size_t i = 0; i < cols.size(); ++i)
    if (bit_of(x, (int)i)) r ^= cols[i];
  return r;
}

// Pair code of a step as it runs in a fused pair, or -1 if the pair kernel does not
// cover it.  `basis` receives the listing basis of the step's projected combos (kappa-0
// vectors first), used when the step is B.
int pair_code(const PlanStep& st, const DevStep& d, std::vector<u128>& basis) {
  basis.clear();
  if (!st.free) return -1;
  const u128 mask = one_at(st.r_in) - 1;
  if (d.mode == MODE_MERGE) {
    if (d.ncombos != 2) return -1;
    basis.push_back((u128)d.combos[1] & mask);
    return PC_M2;
  }
  if (d.mode != MODE_PAIR) return -1;
  if (d.ncombos == 1) return PC_P1;
  if (d.ncombos == 2) {
    basis.push_back(st.kernel[0] & mask);
    return bit_of(st.kernel[0], st.r_in) ? PC_P2H : PC_P2F;
  }
  // Four combos: one kappa-0 and one kappa-1 basis vector (kappa nonzero), else unsupported.
  const u128 k1 = st.kernel[0], k2 = st.kernel[1];
  const u128 cand[3] = {k1, k2, k1 ^ k2};
  u128 zero = 0, one = 0;
  bool has0 = false, has1 = false;
  for (u128 c : cand) {
    if (!bit_of(c, st.r_in) && !has0) {
      zero = c;
      has0 = true;
    } else if (bit_of(c, st.r_in) && !has1) {
      one = c;
      has1 = true;
    }
  }
  if (!has0 || !has1) return -1;
  basis.push_back(zero & mask);
  basis.push_back(one & mask);
  return PC_P4H;
}

// Echelon pivots (highest bits, ascending) of the span of `vecs`; false if dependent.
bool pivots_of(std::vector<u128> vecs, std::vector<int>& piv) {
  piv.clear();
  for (size_t i = 0; i < vecs.size(); ++i) {
    u128 v = vecs[i];
    for (size_t k = 0; k < i; ++k)
      if (bit_of(v, highest_bit(vecs[k]))) v ^= vecs[k];
    if (!v) return false;
    vecs[i] = v;
    // keep earlier vectors free of the new pivot so later reductions stay consistent
    for (size_t k = 0; k < i; ++k)
      if (bit_of(vecs[k], highest_bit(v))) vecs[k] ^= v;
    piv.push_back(highest_bit(v));
  }
  std::sort(piv.begin(), piv.end());
  return true;
}

// The pair record of positions j, j + 1, or false when they cannot be fused.
bool make_pair(Plan& p, int j, DevPair& out, std::vector<unsigned long long>& mb_tables) {
  const PlanStep& A = p.steps[j];
  const PlanStep& B = p.steps[j + 1];
  const DevStep& dA = p.dev[j];
  const DevStep& dB = p.dev[j + 1];
  std::vector<u128> basisA, basisB;
  const int cA = pair_code(A, dA, basisA);
  const int cB = pair_code(B, dB, basisB);
  if (cA < 0 || cB < 0) return false;
  const int m = A.r_out;
  if (B.r_in != m || m < 1) return false;
  const bool pairA = cA != PC_M2;
  const u128 tA = pairA ? A.ycol : 0;
  // t_A must lie outside span(basisB) (else W is smaller than the kernel assumes).
  std::vector<u128> listing;
  if (pairA) listing.push_back(tA);
  for (u128 b : basisB) listing.push_back(b);
  std::vector<int> piv;
  if (!pivots_of(listing, piv)) return false;
  const int dw = (int)listing.size();
  if (dw > 3 || dw > m) return false;
  const int nw = 1 << dw;
  auto w_of = [&](int i) {
    u128 w = 0;
    for (int k = 0; k < dw; ++k)
      if ((i >> k) & 1) w ^= listing[k];
    return w;
  };
  DevPair d{};
  d.j = j;
  d.codeA = cA;
  d.codeB = cB;
  d.a = A.r_in;
  d.m = m;
  d.o = B.r_out;
  d.maskA = (unsigned long long)(one_at(A.r_in) - 1);
  d.betaA = (unsigned long long)A.beta;
  for (int k = 0; k < 4; ++k) d.combA[k] = dA.combos[k];
  d.betaB = (unsigned long long)B.beta;
  d.tB = (unsigned long long)(cB == PC_M2 ? 0 : B.ycol);
  const int ncb = 1 << (int)basisB.size();
  const int na = ncb;  // A-units: pairs of registers (PAIR A) or single registers (MERGE A)
  for (int u = 0; u < na; ++u) {
    const u128 w = pairA ? w_of(2 * u) : w_of(u);
    d.LAw[u] = (unsigned long long)apply_cols(A.lcols, w);
  }
  const std::vector<u128> mB(B.mcols.begin(), B.mcols.begin() + m);
  d.MB0[0] = 0;
  d.MB0[1] = pairA ? (unsigned long long)apply_cols(mB, tA) : 0;
  d.pwB = 0;
  for (int i = 0; i < nw; ++i) {
    const u128 x = w_of(i) & B.beta;
    const int par = (__builtin_popcountll((uint64_t)x) + __builtin_popcountll((uint64_t)(x >> 64))) & 1;
    d.pwB |= (unsigned)par << i;
  }
  d.dw = dw;
  for (int k = 0; k < 3; ++k) d.piv[k] = k < dw ? piv[k] : 0;
  d.tabA_off = dA.table_off;
  d.nbA = dA.nbytes;
  std::vector<u128> tab;
  int nb = 0;
  byte_tables(mB, m, tab, nb);
  if (nb != dA.nbytes) return false;
  // One 16-byte entry per (byte, value): A's table entry and M_B's, so the kernel reads
  // both maps of a group with one load per byte.
  if ((p.tables.size() + mb_tables.size()) & 1) mb_tables.push_back(0ull);
  d.tab2_off = p.tables.size() + mb_tables.size();
  d.nbMB = nb;
  for (size_t i = 0; i < tab.size(); ++i) {
    mb_tables.push_back(p.tables[dA.table_off + i]);
    mb_tables.push_back((unsigned long long)tab[i]);
  }
  out = d;
  return true;
}

// Chooses the fused pairs: non-overlapping (j, j + 1) with j >= 1, inside one of the
// leading / middle / trailing runs, maximising the intermediate entries kept out of
// HBM (2^m each); rebuilds p.pairs and p.pair_at.
void build_pairs(Plan& p) {
  p.pairs.clear();
  p.pair_at.assign(p.n, -1);
  // Drop the byte tables of an earlier pair build (they follow the step tables).
  size_t step_tables = 0;
  for (auto& d : p.dev) step_tables = std::max(step_tables, (size_t)d.table_off + ((size_t)d.nbytes << 8));
  p.tables.resize(step_tables);
  if (!p.fuse || !p.exec_ok) return;
  for (auto& st : p.steps)
    if (!st.free) return;
  int h = 0, t = 0;
  small_runs(p, h, t);
  auto region = [&](int j) { return j < h ? 0 : (j < t ? 1 : 2); };
  std::vector<DevPair> cand(p.n);
  std::vector<char> ok(p.n, 0);
  std::vector<unsigned long long> scratch;
  for (int j = 1; j + 1 < p.n; ++j) {
    if (region(j) != region(j + 1)) continue;
    scratch.clear();
    ok[j] = make_pair(p, j, cand[j], scratch) ? 1 : 0;
  }
  std::vector<double> best(p.n + 2, 0.0);
  std::vector<char> take(p.n + 1, 0);
  for (int j = p.n - 1; j >= 0; --j) {
    best[j] = best[j + 1];
    if (ok[j]) {
      const double g = std::ldexp(1.0, p.steps[j].r_out) + best[j + 2];
      if (g > best[j]) {
        best[j] = g;
        take[j] = 1;
      }
    }
  }
  std::vector<unsigned long long> mb;
  for (int j = 0; j < p.n; ++j) {
    if (!take[j]) continue;
    DevPair d;
    make_pair(p, j, d, mb);
    p.pair_at[j] = (int)p.pairs.size();
    p.pairs.push_back(d);
    ++j;
  }
  p.tables.insert(p.tables.end(), mb.begin(), mb.end());
}

// Builds the device records; fails (without error) when a step is too wide to execute.
void build_device(Plan& p) {
  p.dev.clear();
  p.tables.clear();
  p.exec_ok = true;
  for (int j = 0; j < p.n; ++j) {
    const PlanStep& st = p.steps[j];
    if (st.r_in + 1 > 62 || st.r_out > 62) {
      p.exec_ok = false;
      p.exec_reason = "rank above 61 cannot be executed";
      p.dev.clear();
      p.tables.clear();
      return;
    }
    DevStep d{};
    d.beta = (unsigned long long)st.beta;
    d.r_in = st.r_in;
    d.r_out = st.r_out;
    d.v = st.v;
    d.fixed = st.free ? 0 : 1;
    std::vector<u128> tab;
    int nbytes = 0;
    byte_tables(st.lcols, st.r_out, tab, nbytes);
    d.nbytes = nbytes;
    d.table_off = p.tables.size();
    for (auto x : tab) p.tables.push_back((unsigned long long)x);
    std::vector<u128> combos = kernel_combos(st.kernel);
    if (!st.free) {
      d.mode = MODE_FIXED;
      d.t = 0;
      d.pi = 0;
    } else if (st.ycol != 0) {
      d.mode = MODE_PAIR;
      d.t = (unsigned long long)st.ycol;
      d.pi = highest_bit(st.ycol);
      // Combos with y bit 0 first (stable): the step kernel assigns the two output rows
      // of a pair by the y bit of the row's own image alone.
      std::stable_partition(combos.begin(), combos.end(), [&](u128 c) { return !bit_of(c, st.r_in); });
    } else {
      // e_y lies in the kernel: keep one representative per y pair (the one with y bit 0).
      d.mode = MODE_MERGE;
      d.t = 0;
      d.pi = 0;
      std::vector<u128> reps;
      for (auto c : combos)
        if (!bit_of(c, st.r_in)) reps.push_back(c);
      combos.swap(reps);
    }
    d.ncombos = (int)combos.size();
    d.ng0 = 0;
    for (auto c : combos)
      if (!bit_of(c, st.r_in)) ++d.ng0;
    for (int k = 0; k < 4; ++k) d.combos[k] = k < d.ncombos ? (unsigned long long)combos[k] : 0ull;
    p.dev.push_back(d);
  }
  build_pairs(p);
}

}  // namespace

void plan_set_fusion(Plan& p, bool on) {
  p.fuse = on;
  build_pairs(p);
}

std::string compile_plan(int n, const std::vector<std::pair<int, int>>& edges, const std::vector<int>& order,
                         const std::vector<uint8_t>& fixed, Plan& out) {
  std::string err = validate(n, edges, order, fixed);
  if (!err.empty()) return err;
  out.n = n;
  out.order = order;
  out.fixed = fixed.empty() ? std::vector<uint8_t>(n, 0) : fixed;
  out.future = future_masks(n, edges, order);
  run_compiler(n, out.future, order, out.fixed, true, out.steps, out.ranks);
  out.rmax = 0;
  for (int r : out.ranks) out.rmax = std::max(out.rmax, r);
  for (auto& st : out.steps)
    if ((int)st.kernel.size() > 2) return "internal error: kernel dimension above 2";
  build_device(out);
  return "";
}

}  // namespace rgs
