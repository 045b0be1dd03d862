// Host GF(2) set-up of the conditional (Fourier-cut) sampler.
//
// For a balanced cut (A, B) with M = G[B, A] invertible over GF(2), the conditional
// state of A given x_B is (W/fourier_covariant_sampler.py:1-10, 64-74 of
// whyihaveyou/rgs70-classical-challenge, W/ = work/rgs_attack/):
//   v(z) = 2^{-m/2} (-1)^{q_B(b)} prod_j U_{B_j}[out_j, b_j],  b = N z,  N = M^{-T},
// followed by the Walsh-Hadamard transform over m bits, the phase (-1)^{q_A(z)} and
// the per-qubit unitaries U_{A_j}.  Everything index- or phase-valued here is exact
// integer arithmetic; the lookup tables follow W/init_specialization.py:53-59, 160-189.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rgs {

using u64h = unsigned long long;

// Rank over GF(2) of rows given as bitmasks over `ncols` columns.
int gf2_rank(std::vector<u64h> rows, int ncols);

// Inverse of an m x m GF(2) matrix given by row masks; false if singular.
bool gf2_inverse(const std::vector<u64h>& rows, int m, std::vector<u64h>& inv);

// Transpose of an m x m matrix of row masks.
std::vector<u64h> gf2_transpose(const std::vector<u64h>& rows, int m);

// Strict-upper-triangle row masks of a symmetric 0/1 matrix (distributed_sampler.py:57).
std::vector<u64h> upper_masks(const std::vector<u64h>& sym, int m);

// q(N z) = sum_{i<j} Q_ij z_i z_j + lin . z for q(b) = sum_{i<j} g_ij b_i b_j
// (init_specialization.py:53-59).  Returns Q as strict-upper row masks and lin.
void transformed_quadratic(const std::vector<u64h>& gB_sym, const std::vector<u64h>& N, int m,
                           std::vector<u64h>& Q, u64h& lin);

// Chunk tables over z in chunks of `chunk_bits`:
//   entry[0] = XOR of the columns of `map` selected by the chunk's set bits (0 if map empty),
//   entry[1] = (XOR over the chunk's set bits j of Q row j restricted to higher chunks)
//              | (parity of the chunk-internal quadratic and linear terms) << 63.
// parity(XOR_c entry_c[1] & (z | 1<<63)) is then q(z) mod 2 (init_specialization.py:176-188).
void chunk_tables(int m, int chunk_bits, const std::vector<u64h>& map_cols, const std::vector<u64h>& Q, u64h lin,
                  std::vector<u64h>& table, int& chunks);

}  // namespace rgs
