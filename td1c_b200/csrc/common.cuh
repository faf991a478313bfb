// common.cuh -- shared types and helpers for the td1c_b200 sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace td1c {

typedef double2 cplx;  // (re, im), same bytes as Fortran complex(c_double_complex)

__host__ __device__ __forceinline__ cplx mkc(double r, double i) { cplx c; c.x = r; c.y = i; return c; }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return mkc(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return mkc(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return mkc(a.x, -a.y); }
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return mkc(a.x * s, a.y * s); }
// conj(a) * b
__host__ __device__ __forceinline__ cplx cmulc(cplx a, cplx b) { return mkc(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
// acc += a * b
__host__ __device__ __forceinline__ void cfma(cplx& acc, cplx a, cplx b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
__host__ __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Status bits written by kernels to the device status word.
enum : int {
  ST_OK = 0,
  ST_CHOLESKY = 1,     // non-positive pivot in the Poisson band factorisation
  ST_JACOBI = 2,       // Hermitian eigensolver did not converge
  ST_NONFINITE = 4,    // non-finite value detected in an output
  ST_CUDA = 8,         // a CUDA API call failed on the host side
  ST_CONFIG = 16,      // unsupported configuration
  ST_TIMEOUT = 32,     // a bounded wait on an asynchronous copy ran out
  ST_SINGULAR = 64,    // zero pivot in the one-body propagator factorisation
};

}  // namespace td1c

#define TD1C_CUDA_CHECK(call)                                                         \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess) {                                                          \
      fprintf(stderr, "td1c_b200: CUDA error %s at %s:%d\n", cudaGetErrorString(_e), \
              __FILE__, __LINE__);                                                    \
      return (int)_e;                                                                 \
    }                                                                                 \
  } while (0)
