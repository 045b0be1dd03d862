// Host GF(2) helpers of the conditional sampler (see gf2.hpp).
#include "gf2.hpp"

#include <algorithm>

namespace rgs {

namespace {
inline bool bit(u64h x, int i) { return (x >> i) & 1ull; }
inline int parity(u64h x) { return __builtin_popcountll(x) & 1; }
}  // namespace

int gf2_rank(std::vector<u64h> rows, int ncols) {
  int rank = 0;
  for (int c = 0; c < ncols && rank < (int)rows.size(); ++c) {
    int p = -1;
    for (int r = rank; r < (int)rows.size(); ++r)
      if (bit(rows[r], c)) {
        p = r;
        break;
      }
    if (p < 0) continue;
    std::swap(rows[rank], rows[p]);
    for (int r = rank + 1; r < (int)rows.size(); ++r)
      if (bit(rows[r], c)) rows[r] ^= rows[rank];
    ++rank;
  }
  return rank;
}

bool gf2_inverse(const std::vector<u64h>& rows, int m, std::vector<u64h>& inv) {
  // Gauss-Jordan on [M | I] (fourier_covariant_sampler.py:23-36); the inverse is unique.
  std::vector<u64h> a(rows), b(m);
  for (int i = 0; i < m; ++i) b[i] = 1ull << i;
  for (int col = 0; col < m; ++col) {
    int p = -1;
    for (int r = col; r < m; ++r)
      if (bit(a[r], col)) {
        p = r;
        break;
      }
    if (p < 0) return false;
    std::swap(a[col], a[p]);
    std::swap(b[col], b[p]);
    for (int r = 0; r < m; ++r)
      if (r != col && bit(a[r], col)) {
        a[r] ^= a[col];
        b[r] ^= b[col];
      }
  }
  inv.swap(b);
  return true;
}

std::vector<u64h> gf2_transpose(const std::vector<u64h>& rows, int m) {
  std::vector<u64h> t(m, 0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j)
      if (bit(rows[i], j)) t[j] |= 1ull << i;
  return t;
}

std::vector<u64h> upper_masks(const std::vector<u64h>& sym, int m) {
  std::vector<u64h> up(m, 0);
  for (int i = 0; i < m; ++i) up[i] = sym[i] & ~((2ull << i) - 1ull);
  return up;
}

void transformed_quadratic(const std::vector<u64h>& gB_sym, const std::vector<u64h>& N, int m,
                           std::vector<u64h>& Q, u64h& lin) {
  // P = N^T U N with U the strict upper triangle of g_B; q(Nz) = z^T P z.
  const std::vector<u64h> U = upper_masks(gB_sym, m);
  const std::vector<u64h> Nt = gf2_transpose(N, m);
  // UN[i] = row i of U N: XOR of rows of N selected by row i of U.
  std::vector<u64h> UN(m, 0), P(m, 0);
  for (int i = 0; i < m; ++i)
    for (int k = 0; k < m; ++k)
      if (bit(U[i], k)) UN[i] ^= N[k];
  // P[i] = row i of N^T (U N) = XOR of rows of UN selected by row i of N^T.
  for (int i = 0; i < m; ++i)
    for (int k = 0; k < m; ++k)
      if (bit(Nt[i], k)) P[i] ^= UN[k];
  lin = 0;
  Q.assign(m, 0);
  for (int i = 0; i < m; ++i) {
    if (bit(P[i], i)) lin |= 1ull << i;
    for (int j = i + 1; j < m; ++j)
      if (bit(P[i], j) ^ bit(P[j], i)) Q[i] |= 1ull << j;
  }
}

void chunk_tables(int m, int chunk_bits, const std::vector<u64h>& map_cols, const std::vector<u64h>& Q, u64h lin,
                  std::vector<u64h>& table, int& chunks) {
  chunks = (m + chunk_bits - 1) / chunk_bits;
  table.assign((size_t)chunks * (1u << chunk_bits) * 2, 0);
  const u64h all = m >= 64 ? ~0ull : ((1ull << m) - 1ull);
  for (int c = 0; c < chunks; ++c) {
    const int lo = c * chunk_bits, hi = std::min(m, (c + 1) * chunk_bits);
    const u64h above = all & ~((hi >= 64) ? ~0ull : ((1ull << hi) - 1ull));
    for (u64h code = 0; code < (1ull << (hi - lo)); ++code) {
      const u64h z = code << lo;
      u64h mapped = 0, cross = 0;
      int inner = parity(z & lin);
      for (int j = lo; j < hi; ++j) {
        if (!bit(z, j)) continue;
        if (!map_cols.empty()) mapped ^= map_cols[j];
        cross ^= Q[j] & above;
        inner ^= parity(z & Q[j]);
      }
      u64h* e = &table[((size_t)c * (1u << chunk_bits) + code) * 2];
      e[0] = mapped;
      e[1] = cross | ((u64h)inner << 63);
    }
  }
}

}  // namespace rgs
