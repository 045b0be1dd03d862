// Status codes, error recording and small CUDA helpers shared by the library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/rgs_b200.h"

namespace rgs {

void set_error(const std::string& msg);
const char* last_error();

// Records `msg` and returns `code`.
inline int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

inline int cuda_fail(cudaError_t e, const char* where) {
  return fail(RGS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define RGS_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return ::rgs::cuda_fail(_e, #expr); \
  } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int sm_count(int device);

// The library carries its own CUDA runtime, whose current device is independent of the
// caller's runtime: make the device that owns the caller's pointer `p` current and
// return it.
int bind_device_of(const void* p, int* device);

}  // namespace rgs
