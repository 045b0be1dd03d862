// Scan-program compiler (host).  Algorithm of W/upstream_scan/scan_plan.py:35-152
// (whyihaveyou/rgs70-classical-challenge), restated on 128-bit masks.
#include "plan.hpp"

#include <algorithm>
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

namespace {

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
}

}  // namespace

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
