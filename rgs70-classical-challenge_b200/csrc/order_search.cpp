// Scan-order search: simulated annealing over vertex orders for the cost sum_j 2^{r_j},
// r_j the GF(2) rank of the cut between the first j+1 vertices and the rest -- the rank
// profile of the compiled scan program, so the cost is the number of table entries a
// sweep touches.  Replaces W/order_optimization/search.cpp of
// whyihaveyou/rgs70-classical-challenge (fixed N = 70, one chain, wall-clock budget)
// with any n <= 128, an iteration budget (deterministic for a seed), and several
// independent chains on host threads whose best order wins.
//
// Moves (the reference's four kinds): swap two neighbours, move one vertex to another
// place in a window, reverse a segment, swap two vertices.  Only the prefixes inside
// the touched segment change, so a move re-ranks those cuts alone.  A candidate whose
// largest rank exceeds max_rank is rejected (the memory constraint: two tables of
// 2^max_rank entries per item).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <thread>
#include <vector>

#include "common.hpp"
#include "plan.hpp"

namespace rgs {

namespace {

struct Cuts {
  int n = 0;
  std::vector<u128> adj;
  u128 full = 0;

  // GF(2) rank of the adjacency block between `left` and its complement (the smaller
  // side is eliminated; the rank is symmetric).
  int rank(u128 left) const {
    u128 right = full & ~left;
    const int nl = __builtin_popcountll((uint64_t)left) + __builtin_popcountll((uint64_t)(left >> 64));
    if (2 * nl > n) std::swap(left, right);
    u128 piv[128];
    u128 have = 0;
    int r = 0;
    for (u128 todo = left; todo; todo &= todo - 1) {
      u128 x = adj[lowest_bit(todo)] & right;
      while (x) {
        const int p = highest_bit(x);
        if (bit_of(have, p)) {
          x ^= piv[p];
        } else {
          piv[p] = x;
          have |= one_at(p);
          ++r;
          break;
        }
      }
    }
    return r;
  }
};

struct Chain {
  std::vector<int> order, ranks;
  std::vector<u128> prefix;
  double cost = 0.0;
  int peak = 0;
};

void rerank(const Cuts& g, Chain& c, int lo, int hi) {
  u128 p = lo ? c.prefix[lo - 1] : 0;
  for (int k = lo; k <= hi; ++k) {
    p |= one_at(c.order[k]);
    c.prefix[k] = p;
  }
  for (int k = lo; k <= hi && k < g.n - 1; ++k) c.ranks[k] = g.rank(c.prefix[k]);
  c.ranks[g.n - 1] = 0;
  c.cost = 0.0;
  c.peak = 0;
  for (int r : c.ranks) {
    c.cost += std::ldexp(1.0, r);
    c.peak = std::max(c.peak, r);
  }
}

// One annealing chain: `iters` proposals, temperature falling geometrically from
// t_hi * cost to t_lo * cost over each of `cycles` cycles, each cycle restarting from the
// best order found so far (every other cycle reversed, which keeps the profile).
Chain anneal(const Cuts& g, const std::vector<int>& start, int max_rank, long long iters, uint64_t seed) {
  const int n = g.n;
  Chain cur;
  cur.order = start;
  cur.ranks.assign(n, 0);
  cur.prefix.assign(n, 0);
  rerank(g, cur, 0, n - 1);
  Chain best = cur;
  if (n < 3 || iters <= 0) return best;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> unif(0.0, 1.0);
  const int cycles = 6;
  const long long per = std::max(1ll, iters / cycles);
  const double t_hi = 0.05, t_lo = 2e-4;
  Chain cand = cur;
  for (long long it = 0; it < iters; ++it) {
    const long long cyc = it / per;
    if (it % per == 0) {
      cur = best;
      if (cyc % 2 == 1) {
        std::reverse(cur.order.begin(), cur.order.end());
        rerank(g, cur, 0, n - 1);
      }
    }
    const double phase = (double)(it % per) / (double)per;
    const double temp = cur.cost * t_hi * std::pow(t_lo / t_hi, phase);
    cand = cur;
    const int move = (int)(rng() % 4);
    int i = (int)(rng() % n), j;
    if (move == 0) {
      j = i + 1;
      if (j >= n) {
        j = i;
        i = i - 1;
      }
    } else if (rng() % 4) {
      const int w = std::max(2, std::min(n / 4, 12));
      j = std::clamp(i + (int)(rng() % (2 * w + 1)) - w, 0, n - 1);
    } else {
      j = (int)(rng() % n);
    }
    if (i == j) continue;
    if (i > j) std::swap(i, j);
    if (move == 0 || move == 3) {
      std::swap(cand.order[i], cand.order[j]);
    } else if (move == 1) {
      if (rng() & 1)
        std::rotate(cand.order.begin() + i, cand.order.begin() + i + 1, cand.order.begin() + j + 1);
      else
        std::rotate(cand.order.begin() + i, cand.order.begin() + j, cand.order.begin() + j + 1);
    } else {
      std::reverse(cand.order.begin() + i, cand.order.begin() + j + 1);
    }
    rerank(g, cand, i, j);
    if (cand.peak > max_rank) continue;
    const double d = cand.cost - cur.cost;
    if (d <= 0.0 || unif(rng) < std::exp(-d / temp)) cur = cand;
    if (cur.cost < best.cost) best = cur;
  }
  return best;
}

}  // namespace

std::string order_search(int n, const std::vector<std::pair<int, int>>& edges, const std::vector<int>& start,
                         int max_rank, long long iterations, uint64_t seed, int threads, std::vector<int>& best_order,
                         std::vector<int>& best_ranks, double& best_cost) {
  if (n < 1 || n > 128) return "n must be in [1, 128]";
  if ((int)start.size() != n) return "order must have n entries";
  std::vector<char> seen(n, 0);
  for (int v : start) {
    if (v < 0 || v >= n || seen[v]) return "order must be a permutation of 0..n-1";
    seen[v] = 1;
  }
  Cuts g;
  g.n = n;
  g.adj.assign(n, 0);
  g.full = n == 128 ? ~(u128)0 : ((u128)1 << n) - 1;
  for (auto& e : edges) {
    if (e.first < 0 || e.second < 0 || e.first >= n || e.second >= n || e.first == e.second)
      return "bad edge";
    g.adj[e.first] |= one_at(e.second);
    g.adj[e.second] |= one_at(e.first);
  }
  Chain init;
  init.order = start;
  init.ranks.assign(n, 0);
  init.prefix.assign(n, 0);
  rerank(g, init, 0, n - 1);
  if (max_rank < 0) max_rank = init.peak;
  if (init.peak > max_rank) return "the starting order already exceeds max_rank";
  if (threads < 1) threads = 1;
  std::vector<Chain> results(threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t]() {
      results[t] = anneal(g, start, max_rank, iterations, seed * 0x9E3779B97F4A7C15ull + (uint64_t)t + 1);
    });
  for (auto& th : pool) th.join();
  int bi = 0;
  for (int t = 1; t < threads; ++t)
    if (results[t].cost < results[bi].cost) bi = t;
  best_order = results[bi].order;
  best_ranks = results[bi].ranks;
  best_cost = results[bi].cost;
  return "";
}

}  // namespace rgs
