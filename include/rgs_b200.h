/*
 * rgs_b200 -- C ABI of the B200 graph-state probability and Born-sampling engine.
 *
 * Every entry point returns an int status (RGS_OK = 0), never throws, and
 * records a message readable with rgs_last_error().  Device buffers are owned by
 * the caller (plain device pointers); a plan owns only its small device tables.
 * `stream` is a cudaStream_t passed as void*; NULL means the legacy default stream.
 * No call synchronises the host unless its comment says so.
 *
 * Reference interfaces replaced (whyihaveyou/rgs70-classical-challenge,
 * W/ = work/rgs_attack/) are cited beside each function.  The reference exposes
 * only Python; these are the functions its Python layer would bind through
 * ctypes.
 *
 * Conventions.  Qubit/vertex q of a bitstring is bit q of a little-endian pair
 * of uint64 words (bits[2*i] holds qubits 0..63, bits[2*i+1] qubits 64..127).
 * Complex numbers are interleaved (re, im); complex128 = two doubles.
 */
#ifndef RGS_B200_H
#define RGS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define RGS_OK 0
#define RGS_ERR_ARG 1          /* bad argument: Python ValueError                     */
#define RGS_ERR_OOM 2          /* workspace or device memory too small: MemoryError    */
#define RGS_ERR_CUDA 3         /* CUDA runtime error: RuntimeError                     */
#define RGS_ERR_NONFINITE 4    /* NaN/Inf in a result: ArithmeticError                 */
#define RGS_ERR_ZERO_NORM 5    /* zero or invalid normalisation: ArithmeticError       */
#define RGS_ERR_TIMEOUT 6      /* a bounded device wait expired                        */
#define RGS_ERR_UNSUPPORTED 7  /* plan/instance outside what the executor supports     */
#define RGS_ERR_SINGULAR 8     /* GF(2) matrix not invertible (cut not full rank)      */

/* Precision of the scan executor. */
#define RGS_PREC_C64 0      /* complex64 tables, float64 weights and sums (W/upstream_scan/gpu_kernel.py:59-102) */
#define RGS_PREC_C64_F32 1  /* complex64 tables, float32 weights and sums                                        */
#define RGS_PREC_C128 2     /* complex128 tables and float64 math (W/upstream_scan/gpu_kernel_fp64.py:24-67)     */

typedef struct rgs_plan rgs_plan;

/* Library version string and the message of the last failing call in this thread. */
const char* rgs_version(void);
const char* rgs_last_error(void);
/* Number of CUDA devices visible (0 without a GPU); never fails. */
int rgs_device_count(void);

/* ---------------------------------------------------------------- scan compiler
 * Replaces make_plan / future_masks / byte_tables / kernel_combos
 * (W/upstream_scan/scan_plan.py:45-55, 58-105, 133-145, 148-152) and the
 * plan set-up of ScanOracle.__init__ (W/scan_oracle.py:12-18).
 * edges: int32[n_edges][2]; order: int32[n] (a permutation); fixed: uint8[n] or
 * NULL (vertices with deterministic y, the `fixed` argument of make_plan).
 * Host-only: needs no GPU. */
int rgs_plan_compile(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order,
                     const uint8_t* fixed, rgs_plan** out_plan);
void rgs_plan_destroy(rgs_plan* plan);

/* n, maximum rank, and whether the plan can be executed on a device (rank <= 61). */
int rgs_plan_info(const rgs_plan* plan, int32_t* n, int32_t* rmax, int32_t* executable);
/* Rank after each position: int32[n] (the profile returned by make_plan). */
int rgs_plan_ranks(const rgs_plan* plan, int32_t* ranks);
/* Future-neighbour masks: uint64[n][2] (lo, hi) (future_masks, scan_plan.py:45-55). */
int rgs_plan_future_masks(const rgs_plan* plan, uint64_t* fut);
/* Step j of the plan (Step, scan_plan.py:31-32).  Masks are 128-bit (lo, hi) pairs:
 * beta uint64[2]; lcols uint64[r_out][2]; kernel uint64[2][2] (n_kernel <= 2 used). */
int rgs_plan_step(const rgs_plan* plan, int32_t j, int32_t* v, int32_t* is_free, int32_t* r_in,
                  int32_t* r_out, uint64_t* beta, uint64_t* lcols, int32_t* n_kernel, uint64_t* kernel);
/* Byte tables of step j (byte_tables, scan_plan.py:133-145): uint64[nbytes][256][2]
 * (lo, hi); pass tables = NULL to query nbytes. */
int rgs_plan_step_tables(const rgs_plan* plan, int32_t j, uint64_t* tables, int32_t* nbytes);

/* Fused pairs (no reference counterpart: an execution choice of this engine).  The
 * compiler runs chosen consecutive free positions j, j + 1 of plans without fixed
 * vertices as one pass (scan_pair_kernel) that keeps the table between them out of
 * memory, choosing non-overlapping pairs that keep the most entries out of HBM.
 * rgs_plan_set_fusion(plan, 0) turns this off, (…, 1) back on; only before the plan's
 * first use on a device (RGS_ERR_ARG after).  Amplitudes agree to rounding either way;
 * a (value, logscale) pair of the two schedules may differ by an exact power of two. */
int rgs_plan_set_fusion(rgs_plan* plan, int32_t on);
/* Number of fused pairs and (if first_positions is not NULL) position j of each,
 * int32[count]. */
int rgs_plan_pairs(const rgs_plan* plan, int32_t* count, int32_t* first_positions);
/* Pair record k for inspection: the GF(2) data the pair kernel runs on.  Codes:
 * 0 PAIR 1 combo, 1 PAIR 2 combos (second with y bit 1), 2 PAIR 2 combos (both y bit 0),
 * 3 PAIR 4 combos (two with y bit 1), 4 MERGE 2 combos. */
typedef struct rgs_pair_info {
  int32_t j, code_a, code_b, a, m, o, dw, piv[3];
  uint32_t pw_b;
  uint64_t mask_a, beta_a, comb_a[4], la_w[4], beta_b, mb0[2], t_b;
  uint64_t la_cols[64]; /* L_A: intermediate bit i -> A input vector (y bit at a), i < m */
  uint64_t mb_cols[64]; /* M_B: intermediate bit i -> output row, i < m */
} rgs_pair_info;
int rgs_plan_pair_info(const rgs_plan* plan, int32_t k, rgs_pair_info* info);
/* Rank profile without keeping a plan (cost model sum 2^r used by order search). */
int rgs_rank_profile(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order,
                     const uint8_t* fixed, int32_t* ranks);

/* Scan-order search: simulated annealing over orders for the cost sum_j 2^{r_j} (the
 * table entries of one sweep) subject to max_j r_j <= max_rank (max_rank < 0: the
 * starting order's peak).  Replaces W/order_optimization/search.cpp:33-68 (same four move
 * kinds and peak constraint) for any n <= 128, with an iteration budget instead of a
 * wall-clock one and `threads` independent chains (the best wins); deterministic for a
 * seed.  order_out: int32[n]; ranks_out: int32[n] or NULL; cost_out or NULL.  Plans
 * without fixed vertices.  Host-only. */
int rgs_order_search(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order, int32_t max_rank,
                     int64_t iterations, uint64_t seed, int32_t threads, int32_t* order_out, int32_t* ranks_out,
                     double* cost_out);

/* ---------------------------------------------------------------- scan executor
 * Replaces GPUMixin.alloc/_sweep (W/upstream_scan/gpu_kernel.py:111-170,
 * gpu_kernel_fp64.py:76-135) and ScanOracle.amplitude (W/scan_oracle.py:25-29),
 * batched over bitstrings.  For each bitstring i:
 *     value[i] * exp(logscale[i]) * 2^(-n/2) = <x_i| (x)_q U_q |G>
 * with the same power-of-two renormalisation as the reference, computed on the
 * device (no per-step host round trip).
 *
 * Workspace: caller-owned device memory of rgs_scan_workspace_bytes(plan, batch_tile,
 * precision) bytes; batch_tile is a power of two (1..rgs_scan_max_batch_tile) =
 * bitstrings executed together in one interleaved table.  That size lets the sweep run
 * chunks of 8192 bitstrings (several tiles) with one launch per low-rank position for the
 * whole chunk; a smaller workspace (down to two tables of one tile) halves the chunk or,
 * at the least, runs tile by tile, with the same results bit for bit. */
int rgs_scan_workspace_bytes(const rgs_plan* plan, int32_t batch_tile, int32_t precision, size_t* bytes);
/* Largest batch_tile accepted for a precision (128 complex64, 256 complex64/float32 math,
 * 64 complex128). */
int rgs_scan_max_batch_tile(int32_t precision, int32_t* tile);
/* Kernel launches rgs_scan_amplitudes / rgs_scan_contract queue for `batch` items with a
 * workspace of workspace_bytes (host only, no GPU needed).  No reference counterpart: it
 * reports the launch schedule for profiling and launch-count accounting. */
int rgs_scan_launch_count(const rgs_plan* plan, int64_t batch, int32_t batch_tile, int32_t precision,
                          size_t workspace_bytes, int64_t* launches);

/* Bitstring interface: f_q = U_q[x_q, :] (W/scan_oracle.py:26).
 * unitaries: device complex128[n][2][2]; bits: device uint64[batch][2];
 * out_value: device complex64[batch] (C64 precisions) or complex128[batch] (C128);
 * out_logscale: device float64[batch]. */
int rgs_scan_amplitudes(rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t batch,
                        int32_t precision, void* out_value, double* out_logscale, void* workspace,
                        size_t workspace_bytes, int32_t batch_tile, void* stream);

/* Contraction-vector interface (the GPUMixin._sweep(f, yfix) contract):
 * fvec: device complex128[batch][n][2], f_q for every vertex of every item. */
int rgs_scan_contract(rgs_plan* plan, const double* fvec, int64_t batch, int32_t precision,
                      void* out_value, double* out_logscale, void* workspace, size_t workspace_bytes,
                      int32_t batch_tile, void* stream);

/* ---------------------------------------------------------------- chain-rule sampler over the scan
 * Exact Born sampling for any graph and order (no cut needed): the prefix marginal
 * p(x_{v_0..v_{k-1}}) = 2^{-k} sum |E_k|^2 of the scan environment gives every
 * conditional p(x_v | prefix) from one read of the table (both branches), and the
 * chosen branch is then one scan step.  Extends the reference's p(x) path
 * (W/upstream_scan/gpu_kernel.py:125-170) to sampling and conditional marginals;
 * plans with fixed vertices are not supported.  batch_tile <= 128 (64 for C128).
 * Workspace: rgs_chain_workspace_bytes().  check != 0 synchronises and reports a branch
 * pair of zero total mass as RGS_ERR_ZERO_NORM. */
int rgs_chain_workspace_bytes(const rgs_plan* plan, int32_t batch_tile, int32_t precision, size_t* bytes);
/* Kernel launches of one rgs_chain_sample (marginals = 0) or rgs_chain_marginals (1) call
 * of `count` strings, with out_logp given (with_logp = 1) or NULL: the library's own
 * schedule, counted without launching. */
int rgs_chain_launch_count(const rgs_plan* plan, int64_t count, int32_t batch_tile, int32_t marginals,
                           int32_t with_logp, int64_t* launches);
/* count exact samples.  uniforms: device float64[count][n] in scan order, or NULL for
 * Philox4x32-10 uniforms keyed by seed (counter = item, position).
 * out_bits: device uint64[count][2]; out_value/out_logscale: the amplitude of each
 * sample as rgs_scan_amplitudes; out_logp: device float64[count] = sum of log
 * conditionals = log p(x) (may be NULL); out_cond1: device float32[count][n], the
 * conditionals p(x_{v_j} = 1 | prefix) met while sampling (may be NULL). */
int rgs_chain_sample(rgs_plan* plan, const double* unitaries, int64_t count, uint64_t seed, const double* uniforms,
                     int32_t precision, uint64_t* out_bits, void* out_value, double* out_logscale, double* out_logp,
                     float* out_cond1, void* workspace, size_t workspace_bytes, int32_t batch_tile, int32_t check,
                     void* stream);
/* Conditional marginals of given bitstrings: out_cond1[i][j] = p(x_{v_j} = 1 | x_{v_0..v_{j-1}})
 * (float32, scan order), out_logp[i] = log p(x_i), plus the amplitudes. */
int rgs_chain_marginals(rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t count,
                        int32_t precision, float* out_cond1, double* out_logp, void* out_value, double* out_logscale,
                        void* workspace, size_t workspace_bytes, int32_t batch_tile, int32_t check, void* stream);

/* ---------------------------------------------------------------- resident batch of small instances
 * Many (graph, gates, order) instances -- amplitudes of given bitstrings and exact
 * chain-rule samples of each -- in ONE persistent launch: each block holds an
 * instance's whole environment table for up to 64 items in shared memory and takes
 * work units (largest first) from a device counter.  Replaces the per-instance loop
 * over ScanOracle.amplitude / the scan sweep (W/scan_oracle.py:19-28,
 * W/upstream_scan/gpu_kernel.py:125-170) for instances of rank <= rgs_batch_max_rank()
 * (13 for complex64, 12 for complex128).  Amplitudes are bitwise equal to
 * rgs_scan_amplitudes; samples use the Philox uniforms of rgs_chain_sample (same seed,
 * same item -> same uniforms).  Plans with fixed vertices: amplitudes only.
 * Every buffer of a batch lives on one device; a plan must outlive the batches that
 * use it.  Adding instances is synchronous (it uploads the plan's tables once per
 * device). */
typedef struct rgs_batch rgs_batch;
int rgs_batch_max_rank(int32_t precision, int32_t* rmax);
int rgs_batch_create(int32_t precision, rgs_batch** out);
void rgs_batch_destroy(rgs_batch* batch);
/* One instance: count amplitudes of bits (device uint64[count][2]) into out_value /
 * out_logscale (as rgs_scan_amplitudes), and nsamples samples with Philox key seed into
 * sample_bits (uint64[nsamples][2]), sample_value / sample_logscale (their amplitudes)
 * and sample_logp (log p(x) from the conditionals; may be NULL).  *index = its number. */
int rgs_batch_add(rgs_batch* batch, rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t count,
                  void* out_value, double* out_logscale, int64_t nsamples, uint64_t seed, uint64_t* sample_bits,
                  void* sample_value, double* sample_logscale, double* sample_logp, int32_t* index);
int rgs_batch_info(const rgs_batch* batch, int32_t* instances, int64_t* units);
/* Queues the whole batch on stream.  The first run after rgs_batch_add uploads the work
 * list (synchronous); later runs are two stream operations (a counter reset and one
 * kernel).  check != 0 synchronises and reports a zero-mass branch pair as
 * RGS_ERR_ZERO_NORM. */
int rgs_batch_run(rgs_batch* batch, int32_t check, void* stream);
/* Autotuning of the batch's launch: runs it with each launch variant that holds every
 * instance (one 512-thread block per SM with 192 KiB of tables, two 256-thread blocks with
 * 94 KiB, or four 128-thread blocks with 44 KiB) and keeps the fastest; *variant = the
 * chosen one, ms[3] = milliseconds per run (-1 where a variant does not fit; may be
 * NULL).  Runs the batch (outputs are written); synchronises.  No counterpart in the
 * reference (it has no batch launch). */
int rgs_batch_tune(rgs_batch* batch, void* stream, int32_t* variant, float* ms);

/* ---------------------------------------------------------------- conditional (Fourier-cut) sampler
 * Replaces DistributedSampler / FourierCovariantSampler / FusedFourierSampler /
 * DeferredGlobalMixin / SpecializedDeferredSampler (W/distributed_sampler.py:59-162,
 * W/fourier_covariant_sampler.py:97-141, W/fourier_fused_sampler.py:288-336,
 * W/deferred_global_sampler.py:40-88, W/specialized_deferred_sampler.py:204-238,
 * W/init_specialization.py:160-246) on one device.  Requires a balanced cut with
 * rank(G[B,A]) = |B| = m (RGS_ERR_SINGULAR otherwise), 4 <= m <= 40.
 * graph: host uint8[n][n]; unitaries: host complex128[n][2][2]; A, B: host int32[m].
 * deferred != 0 applies the unitary of A[m-1] at draw time (deferred_global_sampler.py:1-8).
 * The state is caller-owned device complex64[2^m]; outB bit j = outcome of B[j]. */
typedef struct rgs_fourier rgs_fourier;
int rgs_fourier_create(int32_t n, const uint8_t* graph, const double* unitaries, int32_t m, const int32_t* A,
                       const int32_t* B, int32_t deferred, rgs_fourier** out);
void rgs_fourier_destroy(rgs_fourier* plan);
/* m, whether the identical-B lookup specialisation is used, tile bits, tiles, passes. */
int rgs_fourier_info(const rgs_fourier* plan, int32_t* m, int32_t* specialized, int32_t* tile_bits,
                     int64_t* ntiles, int32_t* passes);
/* GF(2) tables for parity tests (init_specialization.py:176-188 layout):
 * lut_z uint64[chunks][256][2] (b XOR, phase mask | inner << 63) of the covariant map,
 * lut_a uint64[chunks][256][2] of q_A, lut_cols uint64[chunks][256][2] of the index map,
 * inv_rows uint64[m] rows of N = G[B,A]^{-T}.  Any pointer may be NULL. */
int rgs_fourier_tables(const rgs_fourier* plan, uint64_t* lut_z, uint64_t* lut_a, uint64_t* lut_cols,
                       uint64_t* inv_rows, int32_t* chunks);
int rgs_fourier_workspace_bytes(const rgs_fourier* plan, size_t* bytes);
/* Conditional state for outB (compute(outB), specialized_deferred_sampler.py:222-238):
 * init + WHT + q_A phase + products, tile masses into the workspace.  stage_ms: NULL, or
 * float[3] for device times of (init, walsh, product) -- then the call synchronises. */
int rgs_fourier_compute(rgs_fourier* plan, uint64_t outB, void* state, void* workspace, size_t workspace_bytes,
                        void* stream, float* stage_ms);
/* Autotuning of the pass kernels for this plan: times a compute with each launch
 * variant (3 or 4 resident blocks per SM) and keeps the faster (replaces the reference's
 * fixed fusion_bits / chunk_mib choice, W/born_production.py:34).  *variant = the chosen
 * one, ms[2] = milliseconds per compute of each (may be NULL).  Overwrites `state`;
 * synchronises. */
int rgs_fourier_tune(rgs_fourier* plan, void* state, void* workspace, size_t workspace_bytes, void* stream,
                     int32_t* variant, float* ms);
/* Pass kernel of the 12-bit tiles: register-first schedule (1, default: axes applied in
 * registers at the load and before the store, the rest in up to three shared-memory
 * rounds) or one shared-memory round per four axes (0).  Both apply the same 2x2
 * operations per axis, in a different order across axes (FP32 results agree to rounding).
 * Exists for tests and measurements.  Process-wide. */
int rgs_fourier_set_register_schedule(int32_t on);
/* Loading passes of the register-first kernel: tiles staged by tensor-map (TMA) loads in
 * persistent blocks, the next tile in flight while the current one is transformed (1), or
 * loaded by the threads with 16-byte accesses (0, default: faster on B200, where the
 * staging buffer leaves room for three resident blocks per SM instead of four).  Both
 * read the same values into the same registers (bit-identical results).  A staged pass
 * whose bounded wait gives up is reported by rgs_tensor_core_status.  Process-wide. */
int rgs_fourier_set_tma(int32_t on);
/* The reference base pipeline (distributed_sampler.py:126-144): product init over b,
 * WHT, index map with q_A phase into `scratch`, products; result in `scratch`. */
int rgs_fourier_compute_permute(rgs_fourier* plan, uint64_t outB, void* state, void* scratch, void* workspace,
                                size_t workspace_bytes, void* stream);
/* Tile masses (float64) of a state (masses(), distributed_sampler.py:145-152); synchronises. */
int rgs_fourier_masses(rgs_fourier* plan, const void* state, void* workspace, double* host_masses, double* norm,
                       void* stream);
/* Two-level inverse CDF over tile masses with uniforms u1, u2, then the deferred
 * terminal pair with u3 (draw(), deferred_global_sampler.py:72-78); synchronises.
 * Fails with RGS_ERR_ZERO_NORM when |norm - 1| > 1e-3 (distributed_sampler.py:151). */
int rgs_fourier_draw(rgs_fourier* plan, const void* state, void* workspace, double u1, double u2, double u3,
                     uint64_t* index, double* pa, double* norm, void* stream);
/* Two-shard conditional state (the top bit m - 1 split over two devices, one shard per
 * device; DeferredGlobalMixin, deferred_global_sampler.py:40-88, with the initcov_global
 * fold of the top bit's Walsh factor, :23-37).  rgs_fourier_compute_shard: this device's
 * half (top bit == shard) in `state` (complex64[2^(m-1)]), deferred terminal unitary not
 * applied, its tile masses in the workspace; needs deferred != 0 and m >= 13.  No data
 * crosses devices.  rgs_fourier_shard_mass: total mass of the computed shard
 * (synchronises).  rgs_fourier_shard_draw: two-level inverse CDF inside the shard (u1:
 * tile, u2: element), the local index (synchronises).  The draw across shards (which
 * shard, then the terminal pair U_last (v_0[l], v_1[l]) with u3) exchanges two scalars per
 * shard: see ShardedConditionalSampler. */
int rgs_fourier_compute_shard(rgs_fourier* plan, uint64_t outB, int32_t shard, void* state, void* workspace,
                              size_t workspace_bytes, void* stream);
int rgs_fourier_shard_mass(rgs_fourier* plan, void* workspace, double* mass, void* stream);
int rgs_fourier_shard_draw(rgs_fourier* plan, const void* state, void* workspace, double u1, double u2,
                           uint64_t* local_index, void* stream);
/* Index map with q_A phase (permute, distributed_sampler.py:35-41), dst != src. */
int rgs_fourier_index_map(rgs_fourier* plan, const void* src, void* dst, void* stream);
/* state[z] *= (-1)^{q_A(z)} (quadratic_phase, graph_sampler.py:76-85). */
int rgs_fourier_quadphase(rgs_fourier* plan, void* state, void* stream);

/* Building blocks on a device complex64 state of 2^nbits values (nbits >= 4), in place. */
/* Walsh-Hadamard butterflies on bits [lo, hi) (lowfwht/localfwht/fusedfwht). */
int rgs_fwht(void* state, int32_t nbits, int32_t lo, int32_t hi, void* stream);
/* The same butterflies with a precision switch: RGS_WHT_FP32 (= rgs_fwht), or 16 x 16
 * Hadamard blocks on the tensor cores (tcgen05.mma, FP32 accumulation in TMEM) over a
 * split-BF16 copy of each value with 2 or 3 terms (RGS_WHT_SPLIT_BF16X2: about 4e-6
 * relative error per 4-bit round, RGS_WHT_SPLIT_BF16X3: FP32 level).  Tensor-core
 * variants need nbits >= 12 and a 16-byte aligned state. */
#define RGS_WHT_FP32 0
#define RGS_WHT_SPLIT_BF16X2 2
#define RGS_WHT_SPLIT_BF16X3 3
int rgs_fwht_precision(void* state, int32_t nbits, int32_t lo, int32_t hi, int32_t precision, void* stream);
/* Per-qubit 2x2 products on bits [lo, hi); unitaries: device complex128[nbits][2][2]
 * (lowprod/localprod/fusedprod). */
int rgs_product(void* state, int32_t nbits, const double* unitaries, int32_t lo, int32_t hi, void* stream);
/* masses[t] = sum |state|^2 over tile t of 2^tile_bits (blockmass, distributed_sampler.py:50-54). */
int rgs_block_mass(const void* state, int32_t nbits, int32_t tile_bits, double* masses, void* stream);

/* ---------------------------------------------------------------- learned proposal (MADE)
 * No counterpart in the reference, which proposes uniformly (W/rejection_sampler.py:19);
 * these are the kernels of the masked autoregressive proposal used for rejection
 * sampling against the engine's p(x).  BF16 operands, FP32 accumulation on the tensor
 * cores (tcgen05.mma into TMEM).  All pointers are device pointers; bf16 arrays are raw
 * 16-bit values. */
/* C[M][N] = alpha * op(A) op(B) (+ bias[N]) (relu) (* mask[M][N]) (* [gate[M][N] > 0]);
 * A: [M][lda] (transA: [K][lda]); B: [K][ldb] (transB: [N][ldb]); C fp32 and/or Cb bf16. */
int rgs_gemm_bf16(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, int32_t transA, const void* B,
                  int32_t ldb, int32_t transB, float alpha, const float* bias, int32_t relu, const uint8_t* mask,
                  const void* gate, float* C, void* Cb, int32_t ldc, void* stream);
/* *timed_out = 1 if a bounded wait of a tensor-core or TMA-staged kernel (GEMM,
 * tensor-core Hadamard passes, TMA-staged Fourier passes) gave up since the last call (its
 * results are then invalid); clears the flag.
 * Synchronous. */
int rgs_tensor_core_status(int32_t* timed_out);
/* TMA loads of the GEMM's K-major operands with 16-byte aligned rows: on (1, default) or
 * off (0: every operand staged by the threads).  Both paths issue the same MMAs in the
 * same order; the switch exists for tests and measurements.  Process-wide. */
int rgs_gemm_set_tma(int32_t on);
/* Forward: x bf16[batch][n] -> h1, h2 bf16[batch][hidden] -> logits z fp32[batch][n];
 * weights bf16 W1[hidden][n], W2[hidden][hidden], W3[n][hidden] (already masked), biases fp32. */
int rgs_mlp_fwd(int32_t batch, int32_t n, int32_t hidden, const void* x, const void* w1b, const float* b1,
                const void* w2b, const float* b2, const void* w3b, const float* b3, void* h1b, void* h2b, float* z,
                void* stream);
/* Backward of the mean binary cross-entropy against soft targets (exact conditionals)
 * target fp32[batch][n]: masked weight gradients gw* fp32, bias gradients gb*, scratch
 * dz/dh2/dh1 bf16, and loss_blocks float64 partial sums of the (unscaled) loss. */
int rgs_mlp_bwd(int32_t batch, int32_t n, int32_t hidden, const void* x, const void* w2b, const void* w3b,
                const void* h1b, const void* h2b, const float* z, const float* target, const uint8_t* m1,
                const uint8_t* m2, const uint8_t* m3, void* dzb, void* dh2b, void* dh1b, float* gw1, float* gb1,
                float* gw2, float* gb2, float* gw3, float* gb3, double* loss_partials, int32_t loss_blocks,
                void* stream);
/* Adam step t (1-based) on fp32 masters w; refreshes the masked bf16 copy wb (may be NULL). */
int rgs_mlp_adam(float* w, const float* grad, float* m1, float* m2, const uint8_t* mask, void* wb, int32_t count,
                 float lr, float beta1, float beta2, float eps, int32_t t, void* stream);
/* batch autoregressive samples x bf16[batch][n] and log q(x) (n forwards, hashed uniforms). */
int rgs_mlp_sample(int32_t batch, int32_t n, int32_t hidden, const void* w1b, const float* b1, const void* w2b,
                   const float* b2, const void* w3b, const float* b3, uint64_t seed, uint64_t first, void* x,
                   double* logq, void* h1b, void* h2b, float* z, void* stream);
/* log q(x) for given x bf16[batch][n]. */
int rgs_mlp_logq(int32_t batch, int32_t n, int32_t hidden, const void* x, const void* w1b, const float* b1,
                 const void* w2b, const float* b2, const void* w3b, const float* b3, double* logq, void* h1b,
                 void* h2b, float* z, void* stream);

/* ---------------------------------------------------------------- allocation-free scan
 * No counterpart in the reference.  Same result as rgs_scan_amplitudes, for callers
 * that cannot let the library allocate device memory: hosts that give it a fixed
 * device-memory budget, and integrations whose own allocator must own every byte of
 * the GPU.  No workspace argument, and no cudaMalloc/cudaFree or allocating library
 * call: all scratch lives in one static device array of RGS_NOALLOC_SCRATCH_BYTES
 * (64 MiB) per GPU, held from library load until process exit.  It must hold the
 * plan's per-step byte tables plus one batch tile's two environment tables; plans
 * whose scratch does not fit at batch tile 1 (complex64 rank above about 21,
 * complex128 above about 20) are rejected with RGS_ERR_OOM.  "No allocation" means
 * no device allocation only: the call still makes CUDA runtime calls, takes a host
 * mutex and builds small host vectors, so never call it from a CUDA host callback
 * (cudaLaunchHostFunc) or a signal handler.  The first call on a device looks up the
 * array's address and caches it for the process; do not use the library on a device
 * after cudaDeviceReset.  Every call uploads the plan's tables from pageable host
 * memory, so a call on a stream that is being captured returns RGS_ERR_UNSUPPORTED.
 * Calls share the array: calls that overlap on the GPU race, so serialise them.
 * out_value: complex64[batch] or complex128[batch] (RGS_PREC_C128). */
#define RGS_NOALLOC_SCRATCH_BYTES (64ull << 20)
int rgs_scan_amplitudes_noalloc(rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t batch,
                                int32_t precision, void* out_value, double* out_logscale, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RGS_B200_H */
