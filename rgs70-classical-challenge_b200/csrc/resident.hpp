// Host interface of the shared-memory-resident batch executor (resident.cu): many
// small instances (amplitudes of given bitstrings and exact chain-rule samples), each
// instance's whole environment table held in shared memory, all of them in one
// persistent launch.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "plan.hpp"

namespace rgs {

constexpr int kMaxResItems = 64;              // items of one work unit (a power of two)
// Launch variants: (threads per block, dynamic shared memory per block for the two tables)
// -- one 512-thread block per SM with 192 KiB, two 256-thread blocks with 94 KiB each, or
// four 128-thread blocks with 44 KiB each (more blocks hide the per-position barriers;
// smaller tables hold fewer items).  rgs_batch_tune picks.
constexpr int kResVariants = 3;
constexpr int kResThreadsOf[kResVariants] = {512, 256, 128};
constexpr int kResSmemOf[kResVariants] = {192 * 1024, 94 * 1024, 44 * 1024};

// One instance of a batch.  Device pointers; outputs of an unused kind may be null.
struct ResInstance {
  const DevStep* steps;                  // n step records (the plan's device copy)
  const unsigned long long* tables;      // byte tables (the plan's device copy)
  const DevVert* verts;                  // vertex records (the plan's device copy)
  const double* U;                       // complex128[n][2][2]
  const unsigned long long* bits;        // amplitude inputs uint64[count][2]
  void* out_value;                       // complex64/complex128[count]
  double* out_logscale;                  // float64[count]
  unsigned long long* sample_bits;       // uint64[nsamples][2]
  void* sample_value;                    // complex[nsamples]: amplitude of each sample
  double* sample_logscale;               // float64[nsamples]
  double* sample_logp;                   // float64[nsamples] (may be null)
  long long count, nsamples;
  unsigned long long seed;               // Philox key of the samples
  int n;                                 // positions
  int nb;                                // items per work unit (power of two)
  int rmax;                              // largest table rank
  int has_fixed;                         // plan has fixed vertices (amplitudes only)
};

// One work unit: `num` consecutive items (amplitudes: kind 0, samples: kind 1) of one instance.
struct ResWork {
  int inst;
  int kind;
  long long first;
  int num;
  int pad;
};

// Device buffers of a prepared batch (owned; freed with the batch).
struct ResDevice {
  int device = -1;
  ResInstance* insts = nullptr;
  size_t insts_cap = 0;
  ResWork* work = nullptr;
  size_t work_cap = 0;
  int* counter = nullptr;  // [0]: next work unit, [1]: status (1 = a zero-mass branch pair)
  long long nwork = 0;
  int variant = 0;         // launch variant the work list was prepared for
  ~ResDevice();
};

// Largest table rank a launch variant holds in shared memory for a precision.
int resident_max_rank(int precision, int variant = 0);
// Items per work unit for an instance of rank `rmax` (0 if it does not fit).
int resident_items(int rmax, int precision, int variant = 0);
// Sets every instance's items per unit for `variant`, uploads the instance records and
// the cost-ordered work list (synchronous).
int resident_prepare(const std::vector<ResInstance>& insts, int precision, int variant, ResDevice& dev);
// Queues the persistent launch on `stream`: resets the work counter and status, then
// runs every unit.  Capturable once prepared.
int resident_launch(const ResDevice& dev, int precision, cudaStream_t stream, int* blocks_out);

}  // namespace rgs
