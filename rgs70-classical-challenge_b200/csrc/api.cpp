// C ABI entry points (include/rgs_b200.h).  Thin wrappers: argument checks, error
// recording, conversion between plain arrays and the C++ plan.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "common.hpp"
#include "plan.hpp"
#include "scan.hpp"
#include "chain.hpp"

namespace rgs {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

namespace {

int read_graph(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order, const uint8_t* fixed,
               std::vector<std::pair<int, int>>& e, std::vector<int>& o, std::vector<uint8_t>& f) {
  if (n < 1 || n > 128) return fail(RGS_ERR_ARG, "n must be in [1, 128]");
  if (n_edges < 0 || (n_edges > 0 && !edges)) return fail(RGS_ERR_ARG, "bad edge list");
  if (!order) return fail(RGS_ERR_ARG, "order is required");
  e.resize(n_edges);
  for (int i = 0; i < n_edges; ++i) e[i] = {edges[2 * i], edges[2 * i + 1]};
  o.assign(order, order + n);
  if (fixed) f.assign(fixed, fixed + n);
  return RGS_OK;
}

void put128(uint64_t* dst, u128 x) {
  dst[0] = (uint64_t)x;
  dst[1] = (uint64_t)(x >> 64);
}

}  // namespace
}  // namespace rgs

using namespace rgs;

extern "C" {

const char* rgs_version(void) { return "rgs_b200 0.1 (sm_100a)"; }

const char* rgs_last_error(void) { return rgs::last_error(); }

int rgs_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

int rgs_plan_compile(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order, const uint8_t* fixed,
                     rgs_plan** out_plan) {
  if (!out_plan) return fail(RGS_ERR_ARG, "out_plan is NULL");
  *out_plan = nullptr;
  std::vector<std::pair<int, int>> e;
  std::vector<int> o;
  std::vector<uint8_t> f;
  int rc = read_graph(n, n_edges, edges, order, fixed, e, o, f);
  if (rc) return rc;
  rgs_plan* p = new (std::nothrow) rgs_plan;
  if (!p) return fail(RGS_ERR_OOM, "host allocation failed");
  std::string err = compile_plan(n, e, o, f, p->plan);
  if (!err.empty()) {
    delete p;
    return fail(RGS_ERR_ARG, err);
  }
  *out_plan = p;
  return RGS_OK;
}

void rgs_plan_destroy(rgs_plan* plan) { delete plan; }

int rgs_plan_info(const rgs_plan* plan, int32_t* n, int32_t* rmax, int32_t* executable) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  if (n) *n = plan->plan.n;
  if (rmax) *rmax = plan->plan.rmax;
  if (executable) *executable = plan->plan.exec_ok ? 1 : 0;
  return RGS_OK;
}

int rgs_plan_ranks(const rgs_plan* plan, int32_t* ranks) {
  if (!plan || !ranks) return fail(RGS_ERR_ARG, "null argument");
  for (int j = 0; j < plan->plan.n; ++j) ranks[j] = plan->plan.ranks[j];
  return RGS_OK;
}

int rgs_plan_future_masks(const rgs_plan* plan, uint64_t* fut) {
  if (!plan || !fut) return fail(RGS_ERR_ARG, "null argument");
  for (int j = 0; j < plan->plan.n; ++j) put128(fut + 2 * j, plan->plan.future[j]);
  return RGS_OK;
}

int rgs_plan_step(const rgs_plan* plan, int32_t j, int32_t* v, int32_t* is_free, int32_t* r_in, int32_t* r_out,
                  uint64_t* beta, uint64_t* lcols, int32_t* n_kernel, uint64_t* kernel) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  if (j < 0 || j >= plan->plan.n) return fail(RGS_ERR_ARG, "step index out of range");
  const PlanStep& st = plan->plan.steps[j];
  if (v) *v = st.v;
  if (is_free) *is_free = st.free ? 1 : 0;
  if (r_in) *r_in = st.r_in;
  if (r_out) *r_out = st.r_out;
  if (beta) put128(beta, st.beta);
  if (lcols)
    for (int k = 0; k < st.r_out; ++k) put128(lcols + 2 * k, st.lcols[k]);
  if (n_kernel) *n_kernel = (int32_t)st.kernel.size();
  if (kernel)
    for (size_t k = 0; k < st.kernel.size(); ++k) put128(kernel + 2 * k, st.kernel[k]);
  return RGS_OK;
}

int rgs_plan_set_fusion(rgs_plan* plan, int32_t on) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  if (!plan->plan.device_copies.empty())
    return fail(RGS_ERR_ARG, "fusion must be set before the plan's first use on a device");
  plan_set_fusion(plan->plan, on != 0);
  return RGS_OK;
}

int rgs_plan_pairs(const rgs_plan* plan, int32_t* count, int32_t* first_positions) {
  if (!plan || !count) return fail(RGS_ERR_ARG, "null argument");
  *count = (int32_t)plan->plan.pairs.size();
  if (first_positions)
    for (size_t k = 0; k < plan->plan.pairs.size(); ++k) first_positions[k] = plan->plan.pairs[k].j;
  return RGS_OK;
}

int rgs_plan_pair_info(const rgs_plan* plan, int32_t k, rgs_pair_info* info) {
  if (!plan || !info) return fail(RGS_ERR_ARG, "null argument");
  if (k < 0 || k >= (int32_t)plan->plan.pairs.size()) return fail(RGS_ERR_ARG, "pair index out of range");
  const DevPair& d = plan->plan.pairs[k];
  *info = rgs_pair_info{};
  info->j = d.j;
  info->code_a = d.codeA;
  info->code_b = d.codeB;
  info->a = d.a;
  info->m = d.m;
  info->o = d.o;
  info->dw = d.dw;
  for (int i = 0; i < 3; ++i) info->piv[i] = d.piv[i];
  info->pw_b = d.pwB;
  info->mask_a = d.maskA;
  info->beta_a = d.betaA;
  for (int i = 0; i < 4; ++i) {
    info->comb_a[i] = d.combA[i];
    info->la_w[i] = d.LAw[i];
  }
  info->beta_b = d.betaB;
  info->mb0[0] = d.MB0[0];
  info->mb0[1] = d.MB0[1];
  info->t_b = d.tB;
  const PlanStep& A = plan->plan.steps[d.j];
  const PlanStep& B = plan->plan.steps[d.j + 1];
  for (int i = 0; i < d.m && i < 64; ++i) {
    info->la_cols[i] = (uint64_t)A.lcols[i];
    info->mb_cols[i] = (uint64_t)B.mcols[i];
  }
  return RGS_OK;
}

int rgs_plan_step_tables(const rgs_plan* plan, int32_t j, uint64_t* tables, int32_t* nbytes) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  if (j < 0 || j >= plan->plan.n) return fail(RGS_ERR_ARG, "step index out of range");
  const PlanStep& st = plan->plan.steps[j];
  std::vector<u128> t;
  int nb = 0;
  byte_tables(st.lcols, st.r_out, t, nb);
  if (nbytes) *nbytes = nb;
  if (tables)
    for (size_t i = 0; i < t.size(); ++i) put128(tables + 2 * i, t[i]);
  return RGS_OK;
}

int rgs_rank_profile(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order, const uint8_t* fixed,
                     int32_t* ranks) {
  if (!ranks) return fail(RGS_ERR_ARG, "ranks is NULL");
  std::vector<std::pair<int, int>> e;
  std::vector<int> o;
  std::vector<uint8_t> f;
  int rc = read_graph(n, n_edges, edges, order, fixed, e, o, f);
  if (rc) return rc;
  std::vector<int> r;
  std::string err = rank_profile(n, e, o, f, r);
  if (!err.empty()) return fail(RGS_ERR_ARG, err);
  for (int j = 0; j < n; ++j) ranks[j] = r[j];
  return RGS_OK;
}

int rgs_order_search(int32_t n, int32_t n_edges, const int32_t* edges, const int32_t* order, int32_t max_rank,
                     int64_t iterations, uint64_t seed, int32_t threads, int32_t* order_out, int32_t* ranks_out,
                     double* cost_out) {
  std::vector<std::pair<int, int>> e;
  std::vector<int> o;
  std::vector<uint8_t> f;
  int rc = read_graph(n, n_edges, edges, order, nullptr, e, o, f);
  if (rc) return rc;
  if (!order_out) return fail(RGS_ERR_ARG, "order_out is required");
  if (iterations < 0) return fail(RGS_ERR_ARG, "iterations must be >= 0");
  std::vector<int> best, ranks;
  double cost = 0.0;
  std::string err = order_search(n, e, o, max_rank, iterations, seed, threads, best, ranks, cost);
  if (!err.empty()) return fail(RGS_ERR_ARG, err);
  for (int i = 0; i < n; ++i) order_out[i] = best[i];
  if (ranks_out)
    for (int i = 0; i < n; ++i) ranks_out[i] = ranks[i];
  if (cost_out) *cost_out = cost;
  return RGS_OK;
}

int rgs_scan_max_batch_tile(int32_t precision, int32_t* tile) {
  if (!tile) return fail(RGS_ERR_ARG, "tile is NULL");
  if (precision < RGS_PREC_C64 || precision > RGS_PREC_C128) return fail(RGS_ERR_ARG, "unknown precision");
  *tile = scan_max_tile(precision);
  return RGS_OK;
}

int rgs_scan_workspace_bytes(const rgs_plan* plan, int32_t batch_tile, int32_t precision, size_t* bytes) {
  if (!plan || !bytes) return fail(RGS_ERR_ARG, "null argument");
  ChunkLayout C;
  int rc = scan_chunk_layout(plan->plan, batch_tile, precision, scan_chunk_tiles(batch_tile), C);
  if (rc) return rc;
  *bytes = C.total;
  return RGS_OK;
}

int rgs_scan_amplitudes(rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t batch,
                        int32_t precision, void* out_value, double* out_logscale, void* workspace,
                        size_t workspace_bytes, int32_t batch_tile, void* stream) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  if (batch == 0) return RGS_OK;
  if (!unitaries || !bits) return fail(RGS_ERR_ARG, "unitaries and bits are required");
  return scan_run(plan->plan, unitaries, (const unsigned long long*)bits, nullptr, batch, precision, out_value,
                  out_logscale, workspace, workspace_bytes, batch_tile, (cudaStream_t)stream, nullptr);
}

int rgs_scan_contract(rgs_plan* plan, const double* fvec, int64_t batch, int32_t precision, void* out_value,
                      double* out_logscale, void* workspace, size_t workspace_bytes, int32_t batch_tile,
                      void* stream) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  if (batch == 0) return RGS_OK;
  if (!fvec) return fail(RGS_ERR_ARG, "fvec is required");
  return scan_run(plan->plan, nullptr, nullptr, fvec, batch, precision, out_value, out_logscale, workspace,
                  workspace_bytes, batch_tile, (cudaStream_t)stream, nullptr);
}

int rgs_scan_launch_count(const rgs_plan* plan, int64_t batch, int32_t batch_tile, int32_t precision,
                          size_t workspace_bytes, int64_t* launches) {
  if (!plan || !launches) return fail(RGS_ERR_ARG, "null argument");
  long long c = 0;
  int rc = scan_launch_count(plan->plan, batch, batch_tile, precision, workspace_bytes, &c);
  if (rc) return rc;
  *launches = c;
  return RGS_OK;
}

int rgs_chain_workspace_bytes(const rgs_plan* plan, int32_t batch_tile, int32_t precision, size_t* bytes) {
  if (!plan || !bytes) return fail(RGS_ERR_ARG, "null argument");
  ChainLayout L;
  int rc = chain_layout(plan->plan, batch_tile, precision, L);
  if (rc) return rc;
  *bytes = L.total;
  return RGS_OK;
}

int rgs_chain_launch_count(const rgs_plan* plan, int64_t count, int32_t batch_tile, int32_t marginals,
                           int32_t with_logp, int64_t* launches) {
  if (!plan || !launches) return fail(RGS_ERR_ARG, "null argument");
  if (count < 0 || batch_tile < 1) return fail(RGS_ERR_ARG, "count must be >= 0 and batch_tile >= 1");
  *launches = (count + batch_tile - 1) / batch_tile * chain_launches_per_tile(plan->plan, marginals != 0, with_logp != 0);
  return RGS_OK;
}

int rgs_chain_sample(rgs_plan* plan, const double* unitaries, int64_t count, uint64_t seed, const double* uniforms,
                     int32_t precision, uint64_t* out_bits, void* out_value, double* out_logscale, double* out_logp,
                     float* out_cond1, void* workspace, size_t workspace_bytes, int32_t batch_tile, int32_t check,
                     void* stream) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  return chain_run(plan->plan, unitaries, count, 0, seed, uniforms, precision, (unsigned long long*)out_bits,
                   out_value, out_logscale, out_logp, out_cond1, workspace, workspace_bytes, batch_tile,
                   (cudaStream_t)stream, check != 0);
}

int rgs_chain_marginals(rgs_plan* plan, const double* unitaries, const uint64_t* bits, int64_t count,
                        int32_t precision, float* out_cond1, double* out_logp, void* out_value, double* out_logscale,
                        void* workspace, size_t workspace_bytes, int32_t batch_tile, int32_t check, void* stream) {
  if (!plan) return fail(RGS_ERR_ARG, "plan is NULL");
  return chain_run(plan->plan, unitaries, count, 1, 0, nullptr, precision, (unsigned long long*)bits, out_value,
                   out_logscale, out_logp, out_cond1, workspace, workspace_bytes, batch_tile, (cudaStream_t)stream,
                   check != 0);
}

}  // extern "C"
