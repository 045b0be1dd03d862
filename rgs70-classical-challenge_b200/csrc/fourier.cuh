// Conditional (Fourier-cut) sampler: host-side plan and kernel entry points.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "gf2.hpp"

namespace rgs {

constexpr int kTileBits = 12;   // elements per tile = 2^12 (32 KiB of complex64 in shared memory)
constexpr int kLowBits = 3;     // contiguous low bits kept in strided tiles (64-byte runs)
constexpr int kChunkBits = 8;   // lookup-table chunk width over z (init_specialization.py:160)

// Per-pass tables of the init map and of a quadratic phase (see fourier.cu).
struct TileTables {
  unsigned long long mlo[64], mhi[64];
  unsigned qtab[128];
};

struct FourierPlan {
  int n = 0, m = 0;
  std::vector<int> A, B;
  bool specialized = false;      // all U_B identical: popcount weight table (init_specialization.py)
  bool deferred = true;          // terminal unitary on bit m-1 applied at draw time
  int variant = 0;               // pass-kernel launch variant (fourier_tune)
  int chunks = 0;
  std::vector<u64h> lut_z;       // [chunks][256][2] covariant map + transformed q_B
  std::vector<u64h> lut_a;       // [chunks][256][2] q_A phase (entry[0] = 0)
  std::vector<u64h> lut_cols;    // [chunks][256][2] index map of the permutation path
  std::vector<u64h> inv_rows;    // rows of N = M^{-T} (b_j = parity(N_j & z))
  std::vector<u64h> qB, qA;      // strict-upper masks of g_BB, g_AA (distributed_sampler.py:57)
  std::vector<u64h> cols;        // cols[k] = mask over B of g[A_k, B] (distributed_sampler.py:68)
  std::vector<double> uA, uB;    // complex128 [m][2][2] of the A / B sites
  // Euler factors of the A-site unitaries, U_j = diag(h_j) R(c_j, s_j) diag(g_j) with R a
  // real rotation (see fourier.cu): per-bit rotations and 8-bit-chunk tables of the two
  // diagonals (the deferred terminal bit has trivial factors).  rot_ok = false falls
  // back to general 2x2 products (a non-unitary input).
  bool rot_ok = false;
  std::vector<float> rot;        // [m][2] (k, form) of the scaled rotations (see fourier.cu)
  std::vector<float> dg, dh;     // [chunks][256][2] complex64 chunk products of g / h
  std::vector<float> rg, rh;     // [m][2] per-bit ratios g(1)/g(0), h(1)/h(0)
  TileTables tt_init{}, tt_phase{};         // pass tables of the init (pass 0) and of the q_A phase pass
  // Two-shard schedule (top bit m - 1 split over two devices, m >= 13): pass tables of the
  // shard init pass (bits 0..10 plus bit m - 1) and of its q_A phase pass.
  bool shardable = false;
  TileTables tt_init_shard{}, tt_phase_shard{};
  std::vector<unsigned long long> qsym_z, qsym_a;  // [m] rows of Q + Q^T of the two phases
  // Pass schedule (see fourier.cu).
  int ngroups = 0;               // strided target groups above the low tile
  // Device copies.
  int device = -1;
  void* d_lut_z = nullptr;
  void* d_lut_a = nullptr;
  void* d_lut_cols = nullptr;
  void* d_uA = nullptr;          // complex64 [m][2][2]
  void* d_uB = nullptr;          // complex128 [m][2][2]
  void* d_rot = nullptr;         // float2 [m]
  void* d_dg = nullptr;          // float2 [chunks][256]
  void* d_dh = nullptr;          // float2 [chunks][256]
  void* d_rg = nullptr;          // float2 [m]
  void* d_rh = nullptr;          // float2 [m]
  void* d_tt_init = nullptr;
  void* d_tt_phase = nullptr;
  void* d_tt_init_shard = nullptr;
  void* d_tt_phase_shard = nullptr;
  void* d_qsym_z = nullptr;
  void* d_qsym_a = nullptr;
  ~FourierPlan();
};

// Workspace: per-tile masses (double), per-sample weight tables, draw result.
struct FourierLayout {
  size_t off_masses = 0, off_weights = 0, off_wspecf = 0, off_result = 0, total = 0;
  long long ntiles = 0;
};

std::string fourier_build(int n, const uint8_t* graph, const double* unitaries, int m, const int* A, const int* B,
                          bool deferred, FourierPlan& p, int& status);
void fourier_layout(const FourierPlan& p, FourierLayout& L);
int fourier_upload(FourierPlan& p, int device);

struct FourierStages {
  float init_ms = 0, walsh_ms = 0, product_ms = 0;
};

// Times one compute with each pass-kernel variant (after a warm-up) and keeps the faster
// for this plan; ms[v] = milliseconds per compute (may be null).  Synchronises.
int fourier_tune(FourierPlan& p, void* state, void* ws, size_t ws_bytes, cudaStream_t s, float* ms);
// Passes of 12-bit tiles on the register-first kernel (on, default) or all passes on the
// round-per-four-axes kernel (off).  Process-wide.
int fourier_set_register_schedule(int on);
// Loading passes of the register-first kernel stage their tiles with tensor-map (TMA)
// loads in persistent blocks (on) or load them with 16-byte accesses (off, default: the
// faster on B200, where the staging buffer costs a resident block per SM).
int fourier_set_tma(int on);
// Whether a bounded wait of a TMA-staged pass gave up since the last call; clears it.
int fourier_tma_timeout(int* timed_out);

// Full conditional state for outcome mask outB (bit j = outcome of B_j), in place in
// `state` (complex64[2^m]); tile masses into the workspace.  If `stages` is given the
// call synchronises and reports device time per stage.
int fourier_compute(FourierPlan& p, uint64_t outB, void* state, void* ws, size_t ws_bytes, cudaStream_t s,
                    FourierStages* stages);
// Reference pipeline (W/distributed_sampler.py:126-144, single device): product init over
// b, WHT, index map with q_A phase into `scratch`, products; result in `scratch`.
int fourier_compute_permute(FourierPlan& p, uint64_t outB, void* state, void* scratch, void* ws, size_t ws_bytes,
                            cudaStream_t s);
// Tile masses of a state (no transform), for states produced elsewhere.
int fourier_masses(FourierPlan& p, const void* state, void* ws, cudaStream_t s);
// Two-level inverse CDF + terminal pair (deferred_global_sampler.py:65-78); synchronises.
int fourier_draw(FourierPlan& p, const void* state, void* ws, double u1, double u2, double u3, uint64_t* index,
                 double* pa, double* norm, cudaStream_t s);

// dst[z] = src[y(z)] (-1)^{q_A(z)} 2^{-m/2}, y = XOR_{k: z_k} cols[k] (distributed_sampler.py:35-41).
int fourier_index_map(FourierPlan& p, const void* src, void* dst, cudaStream_t s);
// state[z] *= (-1)^{q_A(z)} (graph_sampler.py:76-85 on the A vertices).
int fourier_quadphase(FourierPlan& p, void* state, cudaStream_t s);

// Building blocks on a state of 2^nbits complex64 values (in place).
// One half of the conditional state (top bit m - 1 == shard, shard in {0, 1}) on this
// device: 2^(m-1) values at state, the deferred terminal unitary not applied, tile masses
// of the half in the workspace.  The Walsh factor of the top bit is folded into the init
// (both halves' initial values are computed, no exchange); every other operation is local.
int fourier_compute_shard(FourierPlan& p, uint64_t outB, int shard, void* state, void* ws, size_t ws_bytes,
                          cudaStream_t s);
// Total mass of a computed shard (sum of its tile masses, fixed order).
int fourier_shard_mass(FourierPlan& p, void* ws, double* mass, cudaStream_t s);
// Two-level draw inside a computed shard (u1: tile, u2: element): the local index.
int fourier_shard_draw(FourierPlan& p, const void* state, void* ws, double u1, double u2, uint64_t* local_index,
                       cudaStream_t s);
int fwht_bits(void* state, int nbits, int lo, int hi, cudaStream_t s);
// The same butterflies with 16 x 16 Hadamard blocks on the tensor cores over `terms` (2
// or 3) BF16 parts of each value (wht_tc.cu); nbits >= 12.
int fwht_tensor_core(void* state, int nbits, int lo, int hi, int terms, cudaStream_t s);
int product_bits(void* state, int nbits, const double* u_host, int lo, int hi, cudaStream_t s);
int block_mass(const void* state, int nbits, int tile_bits, double* masses, cudaStream_t s);

}  // namespace rgs
