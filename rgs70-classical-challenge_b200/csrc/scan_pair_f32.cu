// scan_pair_kernel instantiations: float storage, float arithmetic.
#include "scan.hpp"
#include "scan_pair_launch.cuh"

namespace rgs {

cudaError_t launch_pair_f32(int VE, dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                            const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA,
                            u64* mc, int lbt, u64 es) {
  if (VE == 1) return launch_pair_codes<float, float, 1>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
  return launch_pair_codes<float, float, 2>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
}

// Chain-rule sampling: B's Gram partials (float64 sums) from a pass over A's input.
cudaError_t launch_pair_gram_f32(int VE, dim3 grid, cudaStream_t s, const void* Ein, const DevPair& P,
                                 const u64* tables, const double4* WA, const u64* mp, int lbt, double* partial) {
  if (VE == 1)
    return launch_pair_codes<float, float, 1, true>(grid, s, Ein, nullptr, P, tables, WA, WA, mp, nullptr, nullptr,
                                                    lbt, 0, partial);
  return launch_pair_codes<float, float, 2, true>(grid, s, Ein, nullptr, P, tables, WA, WA, mp, nullptr, nullptr,
                                                  lbt, 0, partial);
}

}  // namespace rgs
