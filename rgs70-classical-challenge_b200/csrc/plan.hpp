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
  std::vector<u128> mcols;     // the map (c, y) -> c' itself: image of input bit i (i < r_in + free)
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

// Two consecutive free positions A = j and B = j + 1 run as one pass (scan_pair_kernel):
// the intermediate table (A's output, B's input) stays in registers.  Rows of that
// table fall into groups, cosets q0 + W of a subspace W (dim <= 3) closed under A's
// output pairing and B's gathers; a group's inputs, its |W| intermediate rows and its
// outputs involve no row of another group.  Intermediate row i of a group is
// q0 ^ w_i, w_i = sum of listing-basis vectors by the bits of i: for PAIR A bit 0 is
// A's pair offset t_A and the higher bits (B-term index) span B's projected combos
// (kappa-0 vectors first); for MERGE A the bits span B's projected combos alone.
enum PairCode : int {
  PC_P1 = 0,   // PAIR, one combo
  PC_P2H = 1,  // PAIR, two combos, the second with y bit 1
  PC_P2F = 2,  // PAIR, two combos, both with y bit 0
  PC_P4H = 3,  // PAIR, four combos, the last two with y bit 1
  PC_M2 = 4,   // MERGE, two combos
};
constexpr int kPairCodes = 5;
struct DevPair {
  unsigned long long maskA, betaA;
  unsigned long long combA[4];   // A's combos (step order: kappa-0 first)
  unsigned long long LAw[4];     // L_A w of A-unit u's first row (with A's y bit)
  unsigned long long betaB;
  unsigned long long MB0[2];     // M_B (w | 0) of B-unit b's first row
  unsigned long long tB;         // B's output pair offset (PAIR B)
  unsigned long long tabA_off;   // A's byte tables (q -> L_A q over m bits)
  unsigned long long tab2_off;   // interleaved tables over m bits: entry (b, v) is the pair
                                 // (L_A part, M_B (. | 0) part), 16-byte aligned
  unsigned pwB;                  // bit i: parity(w_i & beta_B)
  int a;                         // r_in(A): A's y bit
  int m, o;                      // intermediate and output ranks
  int nbA, nbMB;                 // byte counts of the two tables
  int dw;                        // dim W: 2^(m - dw) groups
  int piv[3];                    // pivot bits of W (ascending): a group's q0 has zeros there
  int codeA, codeB;              // PairCode of A and B
  int j;                         // position A
};

// Positions whose input and output ranks are both at most kSmallRank run once per chunk
// of tiles (scan.cu); a fused pair never straddles the leading / middle / trailing split.
constexpr int kSmallRank = 12;

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
  // Fused pairs: pair_at[j] >= 0 when positions j and j + 1 run as pairs[pair_at[j]].
  std::vector<DevPair> pairs;
  std::vector<int> pair_at;
  bool fuse = true;                        // build fused pairs (plan_set_fusion)
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

// Leading / trailing runs of low-rank positions (input and output rank <= kSmallRank):
// positions [0, h) and [t, n) (h <= t).
void small_runs(const Plan& p, int& h, int& t);

// Turns pair fusion on or off (rebuilds the pair records; the device copies are
// refreshed by the executor).
void plan_set_fusion(Plan& p, bool on);

}  // namespace rgs

// Opaque handle of the C ABI (include/rgs_b200.h).
struct rgs_plan {
  rgs::Plan plan;
};
