// Scan-program compiler: host side, exact GF(2) arithmetic on 128-bit masks.
//
// Compiles a vertex order of a graph with up to 128 vertices into the per-position
// scan program of whyihaveyou/rgs70-classical-challenge
// (W/upstream_scan/scan_plan.py:31-152, W/ = work/rgs_attack/): basis
// reduction in insertion order, lowest-set-bit pivots, the "first column with
// top coefficient k" right inverse and the kernel in column order.  The output is
// bit-identical to that compiler for every field it defines (v, free, r_in, r_out,
// beta, Lcols, kernel, future masks, byte tables, kernel combos); the device
// execution layout adds derived fields (see DevStep).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rgs {

using u128 = unsigned __int128;

inline int lowest_bit(u128 x) {
  uint64_t lo = (uint64_t)x;
  if (lo) return __builtin_ctzll(lo);
  return 64 + __builtin_ctzll((uint64_t)(x >> 64));
}
inline int highest_bit(u128 x) {  // x != 0
  uint64_t hi = (uint64_t)(x >> 64);
  if (hi) return 127 - __builtin_clzll(hi);
  return 63 - __builtin_clzll((uint64_t)x);
}
inline bool bit_of(u128 x, int i) { return (x >> i) & 1; }
inline u128 one_at(int i) { return (u128)1 << i; }

struct PlanStep {
  int v = 0;
  bool free = true;
  int r_in = 0, r_out = 0;
  u128 beta = 0;               // bit i: basis vector i contains this position
  std::vector<u128> lcols;     // right inverse, r_out columns of r_in+free bits
  std::vector<u128> kernel;    // null space of (c, y) -> c', at most two vectors
  u128 ycol = 0;               // image of the y unit vector in new coordinates (free steps)
};

// Execution modes of one step on the device (derived, not part of the reference plan).
enum StepMode : int {
  MODE_PAIR = 0,   // free, y image t != 0: outputs c' and c'^t read the same inputs
  MODE_MERGE = 1,  // free, y image t == 0: both y values of one input land on one output
  MODE_FIXED = 2,  // fixed vertex: y is known per bitstring
};

// Per-step record passed to the kernels by value.  Requires r_in + 1 <= 62.
struct DevStep {
  unsigned long long beta;
  unsigned long long t;          // pair partner offset (MODE_PAIR)
  unsigned long long combos[4];  // MODE_PAIR/FIXED: span(kernel); MODE_MERGE: y-bit-0 representatives
  unsigned long long table_off;  // offset (in u64) of this step's byte tables in the table blob
  int r_in, r_out, nbytes, ncombos, mode, pi, v, fixed;
  int ng0;                       // MODE_PAIR: the first ng0 combos have y bit 0 (the rest y bit 1)
};

struct Plan {
  int n = 0;
  std::vector<int> order;
  std::vector<uint8_t> fixed;        // per vertex
  std::vector<u128> future;          // per position
  std::vector<PlanStep> steps;
  std::vector<int> ranks;
  int rmax = 0;
  // Derived execution data (valid when executable()).
  std::vector<DevStep> dev;
  std::vector<unsigned long long> tables;  // concatenated byte tables
  bool exec_ok = false;
  std::string exec_reason;
  // Device copies, per device ordinal (created lazily by the executor).
  struct DeviceCopy {
    int device = -1;
    void* steps = nullptr;    // DevStep[n]
    void* tables = nullptr;   // u64[tables.size()]
    void* verts = nullptr;    // DevVert[n]
  };
  std::vector<DeviceCopy> device_copies;
  ~Plan();
};

// Vertex record for the per-bitstring weight kernel.
struct DevVert {
  unsigned long long fut_lo, fut_hi;  // future-neighbour mask of this position
  int v;
  int fixed;
};

// Returns an empty string on success, else an error message.
std::string compile_plan(int n, const std::vector<std::pair<int, int>>& edges,
                         const std::vector<int>& order, const std::vector<uint8_t>& fixed, Plan& out);

std::vector<u128> future_masks(int n, const std::vector<std::pair<int, int>>& edges,
                               const std::vector<int>& order);

// Rank profile only (no step data kept); used by the order search.
std::string rank_profile(int n, const std::vector<std::pair<int, int>>& edges, const std::vector<int>& order,
                         const std::vector<uint8_t>& fixed, std::vector<int>& ranks);

// Scan-order search (order_search.cpp): annealing over orders for sum_j 2^{r_j} under
// max r_j <= max_rank (< 0: the starting order's), `threads` independent chains of
// `iterations` proposals each; deterministic for (seed, threads, iterations).  Plans
// without fixed vertices.  Returns an empty string on success, else an error message.
std::string order_search(int n, const std::vector<std::pair<int, int>>& edges, const std::vector<int>& start,
                         int max_rank, long long iterations, uint64_t seed, int threads, std::vector<int>& best_order,
                         std::vector<int>& best_ranks, double& best_cost);

// Byte tables of one step: out[b * 256 + value] = XOR of lcols[8 b + t] over set bits t of value.
void byte_tables(const std::vector<u128>& cols, int nbits, std::vector<u128>& out, int& nbytes);

std::vector<u128> kernel_combos(const std::vector<u128>& kernel);

}  // namespace rgs

// Opaque handle of the C ABI (include/rgs_b200.h).
struct rgs_plan {
  rgs::Plan plan;
};
