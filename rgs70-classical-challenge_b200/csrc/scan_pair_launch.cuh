// Launch dispatch of scan_pair_kernel over the 25 (A, B) pair codes and the two index
// widths, instantiated per storage / arithmetic type in scan_pair_{c128,c64,f32}.cu.
#pragma once
#include "scan_pair.cuh"

namespace rgs {

template <typename S, typename M, int VE, int CA, int CB, typename I, bool GRAM>
cudaError_t launch_pair_one(dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                            const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA,
                            u64* mc, int lbt, u64 es, double* partial) {
  const size_t smem = GRAM ? (size_t)8 * (1u << lbt) * 4 * sizeof(double) : 0;
  scan_pair_kernel<S, M, VE, CA, CB, I, GRAM><<<grid, 256, smem, s>>>((const S*)Ein, (S*)Eout, P, tables, WA, WB, mp,
                                                                     mA, mc, lbt, es, partial);
  return cudaGetLastError();
}

template <typename S, typename M, int VE, int CA, typename I, bool GRAM>
cudaError_t launch_pair_b(dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                          const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA, u64* mc,
                          int lbt, u64 es, double* partial) {
#define RGS_PAIR_B(CB) \
  launch_pair_one<S, M, VE, CA, CB, I, GRAM>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es, partial)
  switch (P.codeB) {
    case PC_P1: return RGS_PAIR_B(PC_P1);
    case PC_P2H: return RGS_PAIR_B(PC_P2H);
    case PC_P2F: return RGS_PAIR_B(PC_P2F);
    case PC_P4H: return RGS_PAIR_B(PC_P4H);
    default: return RGS_PAIR_B(PC_M2);
  }
#undef RGS_PAIR_B
}

template <typename S, typename M, int VE, typename I, bool GRAM>
cudaError_t launch_pair_a(dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                          const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA, u64* mc,
                          int lbt, u64 es, double* partial) {
#define RGS_PAIR_A(CA) \
  launch_pair_b<S, M, VE, CA, I, GRAM>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es, partial)
  switch (P.codeA) {
    case PC_P1: return RGS_PAIR_A(PC_P1);
    case PC_P2H: return RGS_PAIR_A(PC_P2H);
    case PC_P2F: return RGS_PAIR_A(PC_P2F);
    case PC_P4H: return RGS_PAIR_A(PC_P4H);
    default: return RGS_PAIR_A(PC_M2);
  }
#undef RGS_PAIR_A
}

// 32-bit group index and chunk offset arithmetic when the pair's input (with its y bit),
// intermediate and output ranks fit in 31 bits, and so do the chunk offsets of the input
// and output rows (rank + log2 chunks per row).
template <typename S, typename M, int VE, bool GRAM = false>
cudaError_t launch_pair_codes(dim3 grid, cudaStream_t s, const void* Ein, void* Eout, const DevPair& P,
                              const u64* tables, const double4* WA, const double4* WB, const u64* mp, u64* mA,
                              u64* mc, int lbt, u64 es, double* partial = nullptr) {
  const int lC = lbt - (VE == 2 ? 1 : 0);
  if (P.a <= 30 && P.m <= 31 && P.o <= 31 && P.a + lC <= 31 && P.o + lC <= 31)
    return launch_pair_a<S, M, VE, unsigned, GRAM>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es,
                                                   partial);
  return launch_pair_a<S, M, VE, u64, GRAM>(grid, s, Ein, Eout, P, tables, WA, WB, mp, mA, mc, lbt, es, partial);
}

}  // namespace rgs
