// Host loop around the reference's own GPU scan kernel (test and baseline
// infrastructure, never part of the product).  The kernel source is the reference's
// `_SRC_SCALED` string (whyihaveyou/rgs70-classical-challenge,
// work/rgs_attack/upstream_scan/gpu_kernel.py:59-102 for complex64,
// gpu_kernel_fp64.py:24-67 for complex128), extracted and compiled on this machine by
// oracle/build_ref_gpu.py into oracle/_ref/ and included before this file.  This loop
// restates GPUMixin._sweep (gpu_kernel.py:125-170, gpu_kernel_fp64.py:90-135): one
// launch per scan position on a grid of 32 x SM-count blocks of 256 threads, the
// power-of-two scale from frexp of the previous maximum modulus, and a host read of the
// maximum after every launch, as the reference does.  Free vertices only.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#ifdef REF_C128
typedef double2 ref_cplx;
typedef double ref_scale;
typedef unsigned long long ref_max;
#else
typedef float2 ref_cplx;
typedef float ref_scale;
typedef unsigned int ref_max;
#endif

extern "C" int ref_sweep(int nsteps, const int* r_in, const int* r_out, const int* nbytes, const int* ncombos,
                         const unsigned long long* beta, const long long* table_off, const long long* combo_off,
                         const unsigned long long* d_tables, const unsigned long long* d_combos, void* buf_a,
                         void* buf_b, void* d_max, const double* f, int grid, double* out_value,
                         double* out_logscale) {
  ref_cplx one;
  one.x = 1;
  one.y = 0;
  ref_cplx* A = (ref_cplx*)buf_a;
  ref_cplx* B = (ref_cplx*)buf_b;
  cudaError_t e = cudaMemcpy(A, &one, sizeof(one), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return (int)e;
  double m = 1.0, logscale = 0.0;
  for (int j = 0; j < nsteps; ++j) {
    int ex = 0;
    std::frexp(m, &ex);
    const double scale = std::ldexp(1.0, -ex);
    logscale += ex * std::log(2.0);
    if ((e = cudaMemset(d_max, 0, sizeof(ref_max))) != cudaSuccess) return (int)e;
    scan_step_scaled<<<grid, 256>>>(A, B, 1ull << r_out[j], d_tables + table_off[j], nbytes[j],
                                    d_combos + combo_off[j], ncombos[j], r_in[j], beta[j], 0ull, 1, f[4 * j],
                                    f[4 * j + 1], f[4 * j + 2], f[4 * j + 3], 0, (ref_scale)scale,
                                    (ref_max*)d_max);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    ref_cplx* t = A;
    A = B;
    B = t;
    ref_max bits = 0;
    if ((e = cudaMemcpy(&bits, d_max, sizeof(bits), cudaMemcpyDeviceToHost)) != cudaSuccess) return (int)e;
#ifdef REF_C128
    double m2;
#else
    float m2;
#endif
    std::memcpy(&m2, &bits, sizeof(m2));
    if (!(m2 > 0)) {
      out_value[0] = out_value[1] = 0.0;
      *out_logscale = logscale;
      return 0;
    }
    m = std::sqrt((double)m2);
  }
  ref_cplx v;
  if ((e = cudaMemcpy(&v, A, sizeof(v), cudaMemcpyDeviceToHost)) != cudaSuccess) return (int)e;
  out_value[0] = v.x;
  out_value[1] = v.y;
  *out_logscale = logscale;
  return 0;
}
