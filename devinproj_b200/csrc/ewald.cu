// FP64 Ewald summation on the device (accusim/forces.py:333-388): real-space erfc sum over minimum-image
// pairs inside rcut, reciprocal-space sum over the caller's k-vectors and weights, self term.
// Deterministic: every reduction runs in a fixed order.
#include <math.h>

#include <algorithm>

#include "accusim_b200_mlp.h"
#include "common.cuh"

using namespace acs;

namespace {

constexpr int kSChunks = 16;  // structure-factor partial sums per k-vector

// partial[c][k] = sum_{j in chunk c} q_j (cos, sin)(k . r_j)     (accusim/forces.py:382-383)
__global__ void k_sfac_partial(const double* __restrict__ pos, const double* __restrict__ q, int64_t n,
                               const double* __restrict__ kv, int K, double2* __restrict__ partial) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (k >= K) return;
  const int64_t per = (n + kSChunks - 1) / kSChunks;
  const int64_t j0 = c * per, j1 = min(n, j0 + per);
  const double kx = kv[3 * k], ky = kv[3 * k + 1], kz = kv[3 * k + 2];
  double re = 0.0, im = 0.0;
  for (int64_t j = j0; j < j1; ++j) {
    const double ph = pos[3 * j] * kx + pos[3 * j + 1] * ky + pos[3 * j + 2] * kz;
    double s, co;
    sincos(ph, &s, &co);
    re += q[j] * co;
    im += q[j] * s;
  }
  partial[(int64_t)c * K + k] = make_double2(re, im);
}

__global__ void k_sfac_sum(const double2* __restrict__ partial, int K, const double* __restrict__ w,
                           double2* __restrict__ S, double* __restrict__ wS2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double re = 0.0, im = 0.0;
  for (int c = 0; c < kSChunks; ++c) {
    const double2 p = partial[(int64_t)c * K + k];
    re += p.x;
    im += p.y;
  }
  S[k] = make_double2(re, im);
  wS2[k] = w[k] * (re * re + im * im);
}

struct EwaldPar {
  double L[3], a, rcut, c2a, pref_f, k;
  int K;
};

// Per atom: real-space force and energy over all minimum-image partners inside rcut, reciprocal force.
__global__ void __launch_bounds__(kBlock) k_ewald_atoms(const double* __restrict__ pos, const double* __restrict__ q,
                                                         int64_t n, const double* __restrict__ kv,
                                                         const double* __restrict__ w, const double2* __restrict__ S,
                                                         EwaldPar P, double* __restrict__ force, double* partials,
                                                         unsigned int* ticket, double* energy_real) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double u = 0.0;
  if (i < n) {
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2], qi = q[i];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double dx = min_image(sub(pos[3 * j], xi), P.L[0]);
      double dy = min_image(sub(pos[3 * j + 1], yi), P.L[1]);
      double dz = min_image(sub(pos[3 * j + 2], zi), P.L[2]);
      const double r2 = norm2(dx, dy, dz);
      const double r = sqrt(r2);
      if (!(r < P.rcut)) continue;
      const double qq = qi * q[j];
      const double er = erfc(P.a * r);
      u += 0.5 * qq * er / r;
      const double coef = qq * (er / r + P.c2a * exp(-(P.a * r) * (P.a * r))) / r2;
      fx -= coef * dx;
      fy -= coef * dy;
      fz -= coef * dz;
    }
    // reciprocal space: 4 pi / V q_i sum_k w_k Im(conj(S_k) e^{i k.r_i}) k      (accusim/forces.py:385-386)
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int k = 0; k < P.K; ++k) {
      const double kx = kv[3 * k], ky = kv[3 * k + 1], kz = kv[3 * k + 2];
      double s, co;
      sincos(xi * kx + yi * ky + zi * kz, &s, &co);
      const double2 Sk = S[k];
      const double im = Sk.x * s - Sk.y * co;
      const double t = w[k] * im;
      gx += t * kx;
      gy += t * ky;
      gz += t * kz;
    }
    force[3 * i] = P.k * (fx + P.pref_f * qi * gx);
    force[3 * i + 1] = P.k * (fy + P.pref_f * qi * gy);
    force[3 * i + 2] = P.k * (fz + P.pref_f * qi * gz);
  }
  double v[1] = {u};
  block_sum_finish<1>(v, partials, ticket, energy_real);
}

__global__ void k_sum_small(const double* __restrict__ x, int n, double* out) {
  // one block: fixed-order sum (single thread) of n values; n is the k-vector count
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += x[k];
    *out = s;
  }
}

inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

size_t acs_ewald_work_bytes(int64_t n, int32_t K) {
  const int64_t nb = ceil_div(std::max<int64_t>(n, 1), kBlock);
  return a256((size_t)kSChunks * K * 16) + a256((size_t)K * 16) + a256((size_t)K * 8) + a256(nb * 8) + 256 + 256;
}

int acs_ewald_fp64(const double* pos, const double* q, int64_t n, const double* box3, const double* kvec,
                   const double* kw, int32_t K, double alpha, double rcut, double k_coul, double* force,
                   double* energy3_dev, void* work, size_t work_bytes, void* stream) {
  if (n < 1 || !pos || !q || !box3 || !kvec || !kw || K < 1 || !force || !energy3_dev || !(rcut > 0.0) ||
      !(alpha > 0.0))
    return ACS_ERR_ARG;
  if (work_bytes < acs_ewald_work_bytes(n, K) || !work) return ACS_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)work;
  double2* partial = (double2*)w; w += a256((size_t)kSChunks * K * 16);
  double2* S = (double2*)w; w += a256((size_t)K * 16);
  double* wS2 = (double*)w; w += a256((size_t)K * 8);
  const int64_t nb = ceil_div(n, kBlock);
  double* eparts = (double*)w; w += a256(nb * 8);
  unsigned int* ticket = (unsigned int*)w;
  if (cudaMemsetAsync(ticket, 0, 4, s) != cudaSuccess) return ACS_ERR_CUDA;
  dim3 g1((K + 127) / 128, kSChunks);
  k_sfac_partial<<<g1, 128, 0, s>>>(pos, q, n, kvec, K, partial);
  k_sfac_sum<<<(K + 127) / 128, 128, 0, s>>>(partial, K, kw, S, wS2);
  k_sum_small<<<1, 32, 0, s>>>(wS2, K, energy3_dev + 1);  // sum_k w |S|^2 (scaled on the host)
  EwaldPar P;
  for (int d = 0; d < 3; ++d) P.L[d] = box3[d];
  P.a = alpha;
  P.rcut = rcut;
  P.c2a = 2.0 * alpha / sqrt(M_PI);
  const double V = box3[0] * box3[1] * box3[2];
  P.pref_f = 4.0 * M_PI / V;
  P.k = k_coul;
  P.K = K;
  k_ewald_atoms<<<(int)nb, kBlock, 0, s>>>(pos, q, n, kvec, kw, S, P, force, eparts, ticket, energy3_dev);
  return launch_status();
}

}  // extern "C"
