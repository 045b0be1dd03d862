// Host interface of the chain-rule sampler (chain.cu).
#pragma once
#include <cuda_runtime.h>

#include "plan.hpp"
#include "scan.hpp"

namespace rgs {

struct ChainLayout {
  ScanLayout scan;            // ping-pong tables, weights, maxima (as the scan executor)
  int mass_blocks = 0;        // blocks of the Gram kernel
  size_t off_partial = 0;     // per-block, per-item Gram matrices (4 float64)
  size_t off_status = 0;      // device status word
  size_t total = 0;
};

int chain_max_tile(int precision);
int chain_layout(const Plan& plan, int Bt, int precision, ChainLayout& L);
// Kernel launches of chain_run per batch tile (sampling: mode_given = false).
long long chain_launches_per_tile(const Plan& plan, bool mode_given, bool with_logp);

// mode_given = 0: draw x (Philox(seed) uniforms, or `uniforms` [count][n] in scan
// order); bits are written.  mode_given = 1: teacher forcing with the given bits.
// Outputs: final amplitude (value, logscale) of every item, and optionally log p(x) as
// the sum of log conditionals and p(x_{v_j} = 1 | prefix) per position [count][n].
int chain_run(Plan& plan, const double* U, long long count, int mode_given, unsigned long long seed,
              const double* uniforms, int precision, unsigned long long* bits, void* out_value, double* out_logscale,
              double* out_logp, float* out_cond1, void* workspace, size_t ws_bytes, int Bt, cudaStream_t stream,
              bool check);

}  // namespace rgs
