// scan_pair_kernel instantiations: float storage, double arithmetic.
#include "scan.hpp"
#include "scan_pair_launch.cuh"

namespace rgs {

cudaError_t launch_pair_c64(int VE, dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                            const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA,
                            u64* mc, int lbt, u64 es) {
  if (VE == 1) return launch_pair_codes<float, double, 1>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
  return launch_pair_codes<float, double, 2>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
}

}  // namespace rgs
