// Shared device helpers for the accusim_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "accusim_b200.h"

#define ACS_MAX_SPECIES 8

namespace acs {

constexpr int kBlock = 256;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// IEEE round-to-nearest FP64 operations that the compiler may not contract into FMAs. They give the
// reference's NumPy expressions bit for bit.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }

// d -= box * np.round(d / box)   (np.round: half to even == rint)
__device__ __forceinline__ double min_image(double d, double box) { return sub(d, mul(box, rint(div(d, box)))); }

// The same, bit for bit, with a multiply by 1/box in place of the division for almost every pair: t = d (1/box)
// differs from the IEEE quotient d / box by under 3e-16 |d / box|, and rint only changes at half-integers, so
// rint(t) is rint(d / box) unless t lies within 1e-9 of a half-integer (or |t| is huge); there the quotient
// decides as in the reference.
__device__ __forceinline__ double min_image(double d, double box, double inv_box) {
  const double t = d * inv_box;
  const double f = fabs(t - trunc(t));
  const double k = (fabs(f - 0.5) > 1e-9 && fabs(t) < 1e6) ? rint(t) : rint(div(d, box));
  return sub(d, mul(box, k));
}

// np.einsum("ij,ij->i") over 3 components, summed left to right without FMA.
__device__ __forceinline__ double norm2(double dx, double dy, double dz) {
  return add(add(mul(dx, dx), mul(dy, dy)), mul(dz, dz));
}

struct Box3 {
  double L[3];
  double inv[3];   // 1 / L, for min_image's multiply
  int periodic;
};

__device__ __forceinline__ void min_image3(double& dx, double& dy, double& dz, const Box3& b) {
  if (b.periodic) {
    dx = min_image(dx, b.L[0], b.inv[0]);
    dy = min_image(dy, b.L[1], b.inv[1]);
    dz = min_image(dz, b.L[2], b.inv[2]);
  }
}

// Neighbour-list slot: warp-interleaved so that a warp of consecutive atoms reads 128 contiguous bytes.
__host__ __device__ __forceinline__ int64_t nbr_slot(int64_t i, int k, int maxnb) {
  return (i >> 5) * (int64_t)maxnb * 32 + (int64_t)k * 32 + (i & 31);
}

// Deterministic block reduction of W doubles per thread into partials[blockIdx][W]; the last block to
// finish (ticket) sums the partials in block order into out[W] and resets the ticket.
template <int W>
__device__ void block_sum_finish(const double (&v)[W], double* partials, unsigned int* ticket, double* out) {
  __shared__ double sh[W][kBlock / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    double x = v[w];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[w][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      double s = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[w][k];
      partials[(int64_t)blockIdx.x * W + w] = s;
    }
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
      double s = 0.0;
      for (unsigned int b = 0; b < gridDim.x; ++b) s += ((volatile double*)partials)[(int64_t)b * W + w];
      out[w] = s;
    }
    if (threadIdx.x == 0) *ticket = 0u;
  }
}

inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

}  // namespace acs
