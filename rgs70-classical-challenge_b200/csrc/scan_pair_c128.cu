// scan_pair_kernel instantiations: double storage, double arithmetic.
#include "scan.hpp"
#include "scan_pair_launch.cuh"

namespace rgs {

cudaError_t launch_pair_c128(int VE, dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                            const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA,
                            u64* mc, int lbt, u64 es) {
  (void)VE;
  return launch_pair_codes<double, double, 1>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es);
}

}  // namespace rgs
