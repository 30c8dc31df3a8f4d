// Learned DSF->Ewald force correction: BF16 tensor-core (tcgen05) MLP forward/backward kernels and the
// radial-descriptor kernel. See umma.cuh for the operand layout and descriptor encodings.
#include <cuda_bf16.h>
#include <math.h>

#include "accusim_b200_mlp.h"
#include "common.cuh"
#include "umma.cuh"

using namespace acs;
using bf16 = __nv_bfloat16;

namespace {

__device__ __forceinline__ uint32_t pow2_cols(int n) {
  uint32_t c = 32;
  while (c < (uint32_t)n) c <<= 1;
  return c;
}

// D[128 x N] = A[128 x K] * B[N x K]^T, one CTA of 128 threads: the tensor-core primitive every MLP layer
// uses, exposed on its own so its layout and descriptors can be checked against a CUDA-core product.
__global__ void __launch_bounds__(128) k_umma_gemm_test(const bf16* __restrict__ A, const bf16* __restrict__ B,
                                                        float* __restrict__ D, int N, int K, int* status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* sA = sm;
  unsigned char* sB = sm + 128 * K * 2;
  for (int idx = threadIdx.x; idx < 128 * K; idx += blockDim.x)
    *reinterpret_cast<bf16*>(sA + umma::tile_offset(idx / K, idx % K, 128)) = A[idx];
  for (int idx = threadIdx.x; idx < N * K; idx += blockDim.x)
    *reinterpret_cast<bf16*>(sB + umma::tile_offset(idx / K, idx % K, N)) = B[idx];
  const uint32_t ncols = pow2_cols(N);
  if (threadIdx.x == 0) umma::mbar_init(&mbar, 1);
  if (warp == 0) umma::tmem_alloc(&tslot, ncols);
  umma::fence_proxy_async();
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  if (threadIdx.x == 0) {
    const uint32_t id = umma::idesc_bf16_f32(128, N);
    for (int s = 0; s < K / 16; ++s)
      umma::mma_bf16(tmem, umma::slice_desc(umma::smem_u32(sA), 128, s), umma::slice_desc(umma::smem_u32(sB), N, s),
                     id, s > 0);
    umma::commit(&mbar);
  }
  bool ok = umma::mbar_wait(&mbar, 0);
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(status, ACS_FLAG_TIMEOUT);
    umma::mbar_wait(&mbar, 0);  // give in-flight MMAs a second bounded wait before TMEM is released
  }
  umma::fence_after();
  if (ok) {
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      const int row = warp * 32 + lane;
#pragma unroll
      for (int q = 0; q < 16; ++q) D[row * N + c0 + q] = v[q];
    }
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, ncols);
}

}  // namespace

extern "C" int acs_umma_gemm_test(const void* A, const void* B, float* D, int32_t N, int32_t K, int32_t* status_dev,
                                  void* stream) {
  if (!A || !B || !D || !status_dev || N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16) return ACS_ERR_ARG;
  const size_t smem = (size_t)(128 + N) * K * 2;
  if (smem > 200 * 1024) return ACS_ERR_ARG;
  if (cudaFuncSetAttribute(k_umma_gemm_test, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return ACS_ERR_CUDA;
  k_umma_gemm_test<<<1, 128, smem, (cudaStream_t)stream>>>((const bf16*)A, (const bf16*)B, D, N, K, status_dev);
  return launch_status();
}

// ===================================================================== radial descriptors (FP32) ==
// Per ion i, for each neighbour species t and Gaussian channel k (k = lane), within rc:
//   D[i][32t + k] = sum_j g_k(r) fc(r),   V[i][32t + k] = sum_j g_k(r) fc(r) d_ij / r   (d_ij = r_j - r_i)
// g_k(r) = exp(-(r - mu_k)^2 / (2 s^2)), mu_k = r0 + k dmu, fc(r) = (cos(pi r / rc) + 1) / 2.
// X[i] = [(D - mean) / std (64), one-hot species (2), 0 ..., 1 (column 79: the layer-1 bias input)].
namespace {

struct DescPar {
  float r0, dmu, inv2s2, rc, rc2, pi_rc;
  double L[3];
  int periodic;
};

__global__ void __launch_bounds__(256) k_descriptors(const double* __restrict__ pos, const int32_t* __restrict__ sp,
                                                      int64_t n, const int32_t* __restrict__ nbr,
                                                      const int32_t* __restrict__ nnb, int maxnb, DescPar P,
                                                      const float* __restrict__ mean, const float* __restrict__ inv_std,
                                                      bf16* __restrict__ X, float* __restrict__ V) {
  const int lane = threadIdx.x & 31;
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  const float mu = P.r0 + lane * P.dmu;
  float d[2] = {0.f, 0.f}, vx[2] = {0.f, 0.f}, vy[2] = {0.f, 0.f}, vz[2] = {0.f, 0.f};
  const int m = min(nnb[i], maxnb);
  for (int k = 0; k < m; ++k) {
    const int64_t j = nbr[(i >> 5) * (int64_t)maxnb * 32 + (int64_t)k * 32 + (i & 31)];
    double dx = pos[3 * j] - xi, dy = pos[3 * j + 1] - yi, dz = pos[3 * j + 2] - zi;
    if (P.periodic) {
      dx -= P.L[0] * rint(dx / P.L[0]);
      dy -= P.L[1] * rint(dy / P.L[1]);
      dz -= P.L[2] * rint(dz / P.L[2]);
    }
    const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
    const float r2 = fx * fx + fy * fy + fz * fz;
    if (!(r2 < P.rc2)) continue;
    const float r = sqrtf(r2);
    const float fc = 0.5f * (__cosf(P.pi_rc * r) + 1.0f);
    const float t = r - mu;
    const float g = __expf(-t * t * P.inv2s2) * fc;
    const float gr = g / r;
    const int s = sp[j] & 1;
    d[s] += g;
    vx[s] += gr * fx;
    vy[s] += gr * fy;
    vz[s] += gr * fz;
  }
  bf16* xrow = X + i * 80;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int c = 32 * s + lane;
    xrow[c] = __float2bfloat16((d[s] - mean[c]) * inv_std[c]);
    float* vrow = V + (i * 64 + c) * 3;
    vrow[0] = vx[s];
    vrow[1] = vy[s];
    vrow[2] = vz[s];
  }
  if (lane < 16) {
    const int c = 64 + lane;
    float v = 0.f;
    if (lane < 2) v = (sp[i] == lane) ? 1.f : 0.f;
    if (lane == 15) v = 1.f;
    xrow[c] = __float2bfloat16(v);
  }
}

// ====================================================== fused MLP (forward, and backward when training) ==
// Layers: Z1 = X W1^T (80 -> 64, bias = column 79 of W1 on the constant input), H1 = SiLU(Z1);
// Z2 = H1 W2^T + b2, H2 = SiLU(Z2); C = H2 W3^T + b3; prediction F = sum_c C_c V_c (3-vector).
// One CTA of 128 threads per tile of 128 ions; thread t owns ion row t (TMEM lane t).
constexpr int kIn = 80, kH = 64, kOut = 64, kTile = 128;
constexpr int kGradCols = 80;  // weight-gradient GEMM width: 64 inputs + ones row (bias) + zero padding

struct MlpWeights {
  const bf16 *W1, *W2, *W3, *W2T, *W3T;  // [out x in] row-major, and the transposes of W2, W3
  const float *b2, *b3;
};

struct MlpSmem {  // byte offsets into dynamic shared memory
  static constexpr uint32_t X = 0;                              // 128 x 80 (A, layer 1)
  static constexpr uint32_t W1 = X + kTile * kIn * 2;           // 64 x 80
  static constexpr uint32_t W2 = W1 + kH * kIn * 2;             // 64 x 64
  static constexpr uint32_t W3 = W2 + kH * kH * 2;              // 64 x 64
  static constexpr uint32_t W2T = W3 + kOut * kH * 2;           // 64 x 64
  static constexpr uint32_t W3T = W2T + kH * kH * 2;            // 64 x 64
  static constexpr uint32_t H1 = W3T + kH * kOut * 2;           // 128 x 64 (A, layer 2)
  static constexpr uint32_t H2 = H1 + kTile * kH * 2;           // 128 x 64 (A, layer 3)
  static constexpr uint32_t H1T = H2 + kTile * kH * 2;          // 80 x 128 (B, dW2: rows = inputs, ones row 64)
  static constexpr uint32_t H2T = H1T + kGradCols * kTile * 2;  // 80 x 128 (B, dW3; later X^T for dW1)
  static constexpr uint32_t G = H2T + kGradCols * kTile * 2;    // 128 x 64 (A, activation gradients)
  static constexpr uint32_t GT = G + kTile * kH * 2;            // 128 x 128 (A, weight gradients; rows >= 64 zero)
  static constexpr uint32_t END = GT + kTile * kTile * 2;
};
static_assert(MlpSmem::END <= 227 * 1024, "MLP shared-memory plan exceeds 227 KB");

// Inference needs neither the transposed weights nor the gradient buffers; it stages the tile's vector
// features instead: row r (64 x 3 FP32 = 768 B) at VS + r * kVRow. The 16-byte pad makes the per-row
// 16-byte reads of 8 consecutive threads cover all 32 banks.
constexpr uint32_t kVRowBytes = kOut * 3 * 4, kVRow = kVRowBytes + 16;
struct MlpSmemInf {
  static constexpr uint32_t H1 = MlpSmem::W3 + kOut * kH * 2;   // 128 x 64
  static constexpr uint32_t H2 = H1 + kTile * kH * 2;          // 128 x 64
  static constexpr uint32_t VS = H2 + kTile * kH * 2;          // 128 rows of kVRow bytes
  static constexpr uint32_t B = VS + kTile * kVRow;            // b2, b3 (FP32, 128)
  static constexpr uint32_t FP = B + 2 * 64 * 4;               // second-half partial forces (128 x 3 FP32)
  static constexpr uint32_t END = FP + kTile * 3 * 4;
};
static_assert(MlpSmemInf::END <= 227 * 1024 && MlpSmemInf::VS % 16 == 0, "MLP inference shared-memory plan");

// TMEM columns: Z1 [0,64), Z2 [64,128), C [128,192), activation-gradient D [192,256), weight-gradient D [256,336)
constexpr uint32_t kTZ1 = 0, kTZ2 = 64, kTC = 128, kTdH = 192, kTdW = 256, kTCols = 512;

// Approximate division (MUFU reciprocal): the results are rounded to BF16 next, far coarser than its error.
// For z -> -inf, 1 + e^-z -> inf and both return 0.
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ void put(unsigned char* sm, uint32_t base, int r, int k, int R, float v) {
  *reinterpret_cast<bf16*>(sm + base + umma::tile_offset(r, k, R)) = __float2bfloat16(v);
}

// Row-major [R x K] BF16 (global, 16-byte aligned rows) -> canonical tile: each 8-element row segment of a core
// matrix is 16 contiguous bytes, moved with one asynchronous 16-byte copy (all of a thread's copies are in
// flight together; cp_async_wait() completes them). Rows >= rows_valid are zero-filled.
__device__ __forceinline__ void load_tile(unsigned char* sm, uint32_t base, const bf16* __restrict__ src, int R, int K,
                                          int rows_valid = 1 << 30) {
  const int k8n = K / 8;
  for (int c = threadIdx.x; c < R * k8n; c += blockDim.x) {
    const int r = c / k8n, k8 = c % k8n;
    const uint32_t dst = umma::smem_u32(sm + base + umma::tile_offset(r, 8 * k8, R));
    const bool in = r < rows_valid;
    const bf16* g = in ? src + (int64_t)r * K + 8 * k8 : src;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(g), "r"(in ? 16 : 0) : "memory");
  }
}

__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// One row of FP32 values (64) -> BF16 row r of a canonical tile, 16 bytes per store.
__device__ __forceinline__ void put_row64(unsigned char* sm, uint32_t base, int r, int R, const float* v) {
#pragma unroll
  for (int k8 = 0; k8 < 8; ++k8) {
    __nv_bfloat162 p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) p[q] = __floats2bfloat162_rn(v[8 * k8 + 2 * q], v[8 * k8 + 2 * q + 1]);
    *reinterpret_cast<uint4*>(sm + base + umma::tile_offset(r, 8 * k8, R)) = *reinterpret_cast<uint4*>(p);
  }
}

// Issue D(+)= A[128 x K] B[N x K]^T (one elected thread), K in 16-wide slices.
__device__ __forceinline__ void gemm(unsigned char* sm, uint32_t tmem_d, uint32_t a, uint32_t b, int N, int K,
                                     int R_b) {
  const uint32_t id = umma::idesc_bf16_f32(128, N);
  const uint32_t sa = umma::smem_u32(sm + a), sb = umma::smem_u32(sm + b);
  for (int s = 0; s < K / 16; ++s)
    umma::mma_bf16(tmem_d, umma::slice_desc(sa, 128, s), umma::slice_desc(sb, R_b, s), id, s > 0);
}

struct Sync {
  uint64_t* mbar;
  uint32_t phase;
  int* status;
  bool ok;
  // MMAs issued by thread 0 are committed; every thread waits (bounded) and orders TMEM reads after them.
  __device__ bool wait() {
    if (threadIdx.x == 0) umma::commit(mbar);
    bool done = umma::mbar_wait(mbar, phase);
    if (!done) {
      if (threadIdx.x == 0) atomicOr(status, ACS_FLAG_TIMEOUT);
      umma::mbar_wait(mbar, phase);  // second bounded wait for MMAs still in flight
    }
    phase ^= 1u;
    umma::fence_after();
    ok = ok && done;
    return done;
  }
};

__device__ __forceinline__ void smem_to_mma() {  // generic-proxy smem writes -> visible to the tensor core
  umma::fence_proxy_async();
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
}

__device__ __forceinline__ void read_row(uint32_t tmem, uint32_t col, int ncols, float* out) {
  const int warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < ncols; c0 += 16) {
    float v[16];
    umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + col + (uint32_t)c0, v);
#pragma unroll
    for (int q = 0; q < 16; ++q) out[c0 + q] = v[q];
  }
}

template <bool TRAIN>
__global__ void __launch_bounds__(128, 1) k_mlp(const bf16* __restrict__ X, const float* __restrict__ V,
                                                 const float* __restrict__ Y, int64_t n, MlpWeights W, float out_scale,
                                                 float loss_scale, float* __restrict__ Fout, float* __restrict__ gpart,
                                                 float* __restrict__ loss_part, int* status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  constexpr uint32_t kH1 = MlpSmem::H1, kH2 = MlpSmem::H2;
  const int t = threadIdx.x, warp = t >> 5;
  const int64_t row0 = (int64_t)blockIdx.x * kTile;
  const int64_t gi = row0 + t;
  const bool valid = gi < n;
  const int rows = (int)(n - row0 < kTile ? n - row0 : kTile);

  if (t == 0) umma::mbar_init(&mbar, 1);

  // operands: weights and this tile's inputs (rows past n are zero)
  load_tile(sm, MlpSmem::W1, W.W1, kH, kIn);
  load_tile(sm, MlpSmem::W2, W.W2, kH, kH);
  load_tile(sm, MlpSmem::W3, W.W3, kOut, kH);
  if (TRAIN) {
    load_tile(sm, MlpSmem::W2T, W.W2T, kH, kH);
    load_tile(sm, MlpSmem::W3T, W.W3T, kH, kOut);
  }
  load_tile(sm, MlpSmem::X, X + row0 * kIn, kTile, kIn, rows);
  if (TRAIN) {  // weight-gradient A operand: rows 64..127 stay zero
    for (int idx = t; idx < kTile * kTile; idx += blockDim.x) put(sm, MlpSmem::GT, idx / kTile, idx % kTile, kTile, 0.f);
  }
  if (warp == 0) umma::tmem_alloc(&tslot, kTCols);
  cp_async_wait();
  smem_to_mma();
  const uint32_t tm = tslot;
  Sync S{&mbar, 0u, status, true};

  float z[64], c[64];
  // ---- layer 1
  if (t == 0) gemm(sm, tm + kTZ1, MlpSmem::X, MlpSmem::W1, kH, kIn, kH);
  S.wait();
  read_row(tm, kTZ1, kH, z);
  for (int q = 0; q < kH; ++q) z[q] = silu(z[q]);
  put_row64(sm, kH1, t, kTile, z);
  if (TRAIN)
    for (int q = 0; q < kH; ++q) put(sm, MlpSmem::H1T, q, t, kGradCols, z[q]);
  if (TRAIN) {
    put(sm, MlpSmem::H1T, 64, t, kGradCols, 1.f);
    for (int q = 65; q < kGradCols; ++q) put(sm, MlpSmem::H1T, q, t, kGradCols, 0.f);
  }
  smem_to_mma();
  // ---- layer 2
  if (t == 0) gemm(sm, tm + kTZ2, kH1, MlpSmem::W2, kH, kH, kH);
  S.wait();
  read_row(tm, kTZ2, kH, z);
  for (int q = 0; q < kH; ++q) z[q] = silu(z[q] + W.b2[q]);
  put_row64(sm, kH2, t, kTile, z);
  if (TRAIN)
    for (int q = 0; q < kH; ++q) put(sm, MlpSmem::H2T, q, t, kGradCols, z[q]);
  if (TRAIN) {
    put(sm, MlpSmem::H2T, 64, t, kGradCols, 1.f);
    for (int q = 65; q < kGradCols; ++q) put(sm, MlpSmem::H2T, q, t, kGradCols, 0.f);
  }
  smem_to_mma();
  // ---- layer 3: coefficients, contraction with the vector features
  if (t == 0) gemm(sm, tm + kTC, kH2, MlpSmem::W3, kOut, kH, kOut);
  S.wait();
  read_row(tm, kTC, kOut, c);
  float F[3] = {0.f, 0.f, 0.f};
  if (valid) {
    const float* vrow = V + gi * kOut * 3;
    for (int q = 0; q < kOut; ++q) {
      c[q] += W.b3[q];
      F[0] += c[q] * vrow[3 * q];
      F[1] += c[q] * vrow[3 * q + 1];
      F[2] += c[q] * vrow[3 * q + 2];
    }
    if (Fout) {
      Fout[3 * gi] = out_scale * F[0];
      Fout[3 * gi + 1] = out_scale * F[1];
      Fout[3 * gi + 2] = out_scale * F[2];
    }
  }
  if (TRAIN) {
    // loss = loss_scale * sum |F - Y|^2 over valid rows; dF = 2 loss_scale (F - Y)
    float dF[3] = {0.f, 0.f, 0.f}, l = 0.f;
    if (valid) {
      for (int d = 0; d < 3; ++d) {
        const float r = F[d] - Y[3 * gi + d];
        l += r * r;
        dF[d] = 2.0f * loss_scale * r;
      }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((t & 31) == 0) loss_part[blockIdx.x * 4 + warp] = loss_scale * l;
    const float* vrow = V + (valid ? gi : 0) * kOut * 3;
    for (int q = 0; q < kOut; ++q) {  // dC = dF . V_c
      const float g = valid ? dF[0] * vrow[3 * q] + dF[1] * vrow[3 * q + 1] + dF[2] * vrow[3 * q + 2] : 0.f;
      put(sm, MlpSmem::G, t, q, kTile, g);
      put(sm, MlpSmem::GT, q, t, kTile, g);
    }
    smem_to_mma();
    float* gp = gpart + (int64_t)blockIdx.x * (3 * kH * kGradCols);
    // ---- dW3 (+ db3 in column 64), dH2
    if (t == 0) {
      gemm(sm, tm + kTdW, MlpSmem::GT, MlpSmem::H2T, kGradCols, kTile, kGradCols);
      gemm(sm, tm + kTdH, MlpSmem::G, MlpSmem::W3T, kH, kOut, kH);
    }
    S.wait();
    {
      float w[kGradCols];
      read_row(tm, kTdW, kGradCols, w);
      if (t < kOut)
        for (int q = 0; q < kGradCols; ++q) gp[2 * kH * kGradCols + t * kGradCols + q] = w[q];
    }
    read_row(tm, kTdH, kH, c);   // dH2
    read_row(tm, kTZ2, kH, z);   // Z2 without b2
    umma::fence_before();
    __syncthreads();
    for (int q = 0; q < kH; ++q) {
      const float g = c[q] * dsilu(z[q] + W.b2[q]);
      put(sm, MlpSmem::G, t, q, kTile, g);
      put(sm, MlpSmem::GT, q, t, kTile, g);
    }
    smem_to_mma();
    // ---- dW2 (+ db2), dH1
    if (t == 0) {
      gemm(sm, tm + kTdW, MlpSmem::GT, MlpSmem::H1T, kGradCols, kTile, kGradCols);
      gemm(sm, tm + kTdH, MlpSmem::G, MlpSmem::W2T, kH, kH, kH);
    }
    S.wait();
    {
      float w[kGradCols];
      read_row(tm, kTdW, kGradCols, w);
      if (t < kH)
        for (int q = 0; q < kGradCols; ++q) gp[1 * kH * kGradCols + t * kGradCols + q] = w[q];
    }
    read_row(tm, kTdH, kH, c);   // dH1
    read_row(tm, kTZ1, kH, z);   // Z1
    umma::fence_before();
    __syncthreads();
    for (int q = 0; q < kH; ++q) put(sm, MlpSmem::GT, q, t, kTile, c[q] * dsilu(z[q]));
    for (int k = 0; k < kIn; ++k) {  // X^T into the (now free) H2T buffer
      const bf16 v = *reinterpret_cast<const bf16*>(sm + MlpSmem::X + umma::tile_offset(t, k, kTile));
      *reinterpret_cast<bf16*>(sm + MlpSmem::H2T + umma::tile_offset(k, t, kGradCols)) = v;
    }
    smem_to_mma();
    // ---- dW1 (bias = column 79)
    if (t == 0) gemm(sm, tm + kTdW, MlpSmem::GT, MlpSmem::H2T, kGradCols, kTile, kGradCols);
    S.wait();
    {
      float w[kGradCols];
      read_row(tm, kTdW, kGradCols, w);
      if (t < kH)
        for (int q = 0; q < kGradCols; ++q) gp[t * kGradCols + q] = w[q];
    }
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tm, kTCols);
}

// Inference on one 128-ion tile with 256 threads. Warps w and w + 4 share TMEM lane quadrant w % 4 (rows
// 32 (w % 4) + lane) and split every epilogue's columns: half h = w / 4 takes [32 h, 32 h + 32). The tile's
// vector features stream into shared memory (bulk copies) behind the three layers; the two halves of the
// contraction F = sum_c C_c V_c meet in shared memory.
constexpr uint32_t kInfCols = 256;  // TMEM: Z1 [0, 64), Z2 [64, 128), C [128, 192)

__device__ __forceinline__ void read32(uint32_t tmem, int quad, uint32_t col, float* out) {
  float v[16];
  umma::tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + col, v);
#pragma unroll
  for (int q = 0; q < 16; ++q) out[q] = v[q];
  umma::tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + col + 16u, v);
#pragma unroll
  for (int q = 0; q < 16; ++q) out[16 + q] = v[q];
}

// 32 FP32 values -> BF16 columns [8 k8_0, 8 k8_0 + 32) of row r of a canonical tile, 16 bytes per store.
__device__ __forceinline__ void put_row32(unsigned char* sm, uint32_t base, int r, int R, int k8_0, const float* v) {
#pragma unroll
  for (int k8 = 0; k8 < 4; ++k8) {
    __nv_bfloat162 p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) p[q] = __floats2bfloat162_rn(v[8 * k8 + 2 * q], v[8 * k8 + 2 * q + 1]);
    *reinterpret_cast<uint4*>(sm + base + umma::tile_offset(r, 8 * (k8_0 + k8), R)) = *reinterpret_cast<uint4*>(p);
  }
}

__global__ void __launch_bounds__(256, 1) k_mlp_infer(const bf16* __restrict__ X, const float* __restrict__ V, int64_t n,
                                                      MlpWeights W, float out_scale, float* __restrict__ Fout,
                                                      int* status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t mbar, vbar;
  __shared__ uint32_t tslot;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int quad = warp & 3, half = warp >> 2;
  const int row = 32 * quad + lane;
  const int64_t row0 = (int64_t)blockIdx.x * kTile;
  const int64_t gi = row0 + row;
  const bool valid = gi < n;
  const int rows = (int)(n - row0 < kTile ? n - row0 : kTile);
  float* bias = reinterpret_cast<float*>(sm + MlpSmemInf::B);
  float* fpart = reinterpret_cast<float*>(sm + MlpSmemInf::FP);

  if (t == 0) {
    umma::mbar_init(&mbar, 1);
    umma::mbar_init(&vbar, 1);
    umma::mbar_fence_init();
  }
  __syncthreads();
  if (warp == 0) {
    if (lane == 0) umma::mbar_expect_tx(&vbar, (uint32_t)rows * kVRowBytes);
    __syncwarp();
    for (int r = lane; r < rows; r += 32)
      umma::bulk_g2s(umma::smem_u32(sm + MlpSmemInf::VS + r * kVRow), V + (row0 + r) * kOut * 3, kVRowBytes, &vbar);
  }
  load_tile(sm, MlpSmem::W1, W.W1, kH, kIn);
  load_tile(sm, MlpSmem::W2, W.W2, kH, kH);
  load_tile(sm, MlpSmem::W3, W.W3, kOut, kH);
  load_tile(sm, MlpSmem::X, X + row0 * kIn, kTile, kIn, rows);
  if (t < 128) bias[t] = t < 64 ? W.b2[t] : W.b3[t - 64];
  if (warp == 0) umma::tmem_alloc(&tslot, kInfCols);
  cp_async_wait();
  smem_to_mma();
  const uint32_t tm = tslot;
  Sync S{&mbar, 0u, status, true};
  const uint32_t col = 32u * (uint32_t)half;
  float z[32];

  if (t == 0) gemm(sm, tm + kTZ1, MlpSmem::X, MlpSmem::W1, kH, kIn, kH);
  S.wait();
  read32(tm, quad, kTZ1 + col, z);
#pragma unroll
  for (int q = 0; q < 32; ++q) z[q] = silu(z[q]);
  put_row32(sm, MlpSmemInf::H1, row, kTile, 4 * half, z);
  smem_to_mma();

  if (t == 0) gemm(sm, tm + kTZ2, MlpSmemInf::H1, MlpSmem::W2, kH, kH, kH);
  S.wait();
  read32(tm, quad, kTZ2 + col, z);
#pragma unroll
  for (int q = 0; q < 32; ++q) z[q] = silu(z[q] + bias[col + q]);
  put_row32(sm, MlpSmemInf::H2, row, kTile, 4 * half, z);
  smem_to_mma();

  if (t == 0) gemm(sm, tm + kTC, MlpSmemInf::H2, MlpSmem::W3, kOut, kH, kOut);
  S.wait();
  read32(tm, quad, kTC + col, z);
  bool have_v = umma::mbar_wait(&vbar, 0);
  if (!have_v) {
    if (t == 0) atomicOr(status, ACS_FLAG_TIMEOUT);
    umma::mbar_wait(&vbar, 0);  // second bounded wait for copies still in flight
  }
  // this half's channels q in [32 h, 32 h + 32) are the row's FP32 elements [96 h, 96 h + 96)
  float F[3] = {0.f, 0.f, 0.f};
  if (valid && have_v) {
#pragma unroll
    for (int q = 0; q < 32; ++q) z[q] += bias[64 + col + q];
    const float4* vr = reinterpret_cast<const float4*>(sm + MlpSmemInf::VS + row * kVRow) + 24 * half;
#pragma unroll
    for (int m = 0; m < 24; ++m) {
      const float4 v = vr[m];
      const float e4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) F[(4 * m + j) % 3] = fmaf(z[(4 * m + j) / 3], e4[j], F[(4 * m + j) % 3]);
    }
  }
  if (half == 1) {
    fpart[3 * row] = F[0];
    fpart[3 * row + 1] = F[1];
    fpart[3 * row + 2] = F[2];
  }
  umma::fence_before();
  __syncthreads();
  if (half == 0 && valid && have_v) {
    Fout[3 * gi] = out_scale * (F[0] + fpart[3 * row]);
    Fout[3 * gi + 1] = out_scale * (F[1] + fpart[3 * row + 1]);
    Fout[3 * gi + 2] = out_scale * (F[2] + fpart[3 * row + 2]);
  }
  if (warp == 0) umma::tmem_free(tm, kInfCols);
}

// Sum the per-tile gradient partials in tile order (deterministic) and take an Adam step on the FP32
// master parameters; refresh the BF16 operand copies (W and the transposes of W2, W3).
// Parameter vector: [W1 64x80 | W2aug 64x80 (cols 0..63 weights, 64 bias) | W3aug 64x80], FP32.
__global__ void k_adam(const float* __restrict__ gpart, int ntiles, float* __restrict__ theta,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                       float bc1, float bc2, float wd, bf16* __restrict__ W1, bf16* __restrict__ W2,
                       bf16* __restrict__ W3, bf16* __restrict__ W2T, bf16* __restrict__ W3T, float* __restrict__ bias2,
                       float* __restrict__ bias3, float* __restrict__ grad_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int P = 3 * kH * kGradCols;
  if (p >= P) return;
  const int layer = p / (kH * kGradCols), o = (p / kGradCols) % kH, col = p % kGradCols;
  const bool used = (layer == 0) ? true : (col <= 64);
  float g = 0.f;
  for (int tl = 0; tl < ntiles; ++tl) g += gpart[(int64_t)tl * P + p];
  if (grad_out) grad_out[p] = g;
  if (!used) return;
  const bool is_bias = (layer == 0) ? (col == 79) : (col == 64);
  float th = theta[p];
  const float gg = g + (is_bias ? 0.f : wd * th);
  const float mm = b1 * m[p] + (1.f - b1) * gg;
  const float vv = b2 * v[p] + (1.f - b2) * gg * gg;
  m[p] = mm;
  v[p] = vv;
  th -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
  theta[p] = th;
  const bf16 hb = __float2bfloat16(th);
  if (layer == 0) {
    W1[o * kIn + col] = hb;
  } else if (layer == 1) {
    if (col < 64) {
      W2[o * kH + col] = hb;
      W2T[col * kH + o] = hb;
    } else {
      bias2[o] = th;
    }
  } else {
    if (col < 64) {
      W3[o * kH + col] = hb;
      W3T[col * kOut + o] = hb;
    } else {
      bias3[o] = th;
    }
  }
}

}  // namespace

extern "C" {

int acs_descriptors(const double* pos, const int32_t* sp, int64_t n, const double* box3, int periodic,
                    const int32_t* nbr, const int32_t* nnb, int32_t maxnb, const float* params6, const float* mean,
                    const float* inv_std, void* X_bf16, float* V, void* stream) {
  if (n < 1 || !pos || !sp || !nbr || !nnb || maxnb < 1 || !params6 || !mean || !inv_std || !X_bf16 || !V)
    return ACS_ERR_ARG;
  DescPar P;
  P.r0 = params6[0];
  P.dmu = params6[1];
  P.inv2s2 = params6[2];
  P.rc = params6[3];
  P.rc2 = params6[3] * params6[3];
  P.pi_rc = (float)M_PI / params6[3];
  for (int d = 0; d < 3; ++d) P.L[d] = box3 ? box3[d] : 0.0;
  P.periodic = periodic && box3;
  const int64_t threads = n * 32;
  k_descriptors<<<(int)ceil_div(threads, 256), 256, 0, (cudaStream_t)stream>>>(pos, sp, n, nbr, nnb, maxnb, P, mean,
                                                                               inv_std, (bf16*)X_bf16, V);
  return launch_status();
}

size_t acs_mlp_grad_bytes(int64_t n) { return (size_t)ceil_div(n, kTile) * 3 * kH * kGradCols * 4; }
int32_t acs_mlp_param_count(void) { return 3 * kH * kGradCols; }

int acs_mlp_forward(const void* X, const float* V, int64_t n, const void* const* w5, const float* b2, const float* b3,
                    float out_scale, float* F, int32_t* status_dev, void* stream) {
  if (n < 1 || !X || !V || !w5 || !b2 || !b3 || !F || !status_dev) return ACS_ERR_ARG;
  if ((uintptr_t)V & 15) return ACS_ERR_ARG;   // rows are bulk-copied: 16-byte alignment
  const size_t smem = MlpSmemInf::END;
  // set once per device: this launch may sit inside a CUDA graph capture
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ACS_ERR_NO_DEVICE;
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return ACS_ERR_CUDA;
    attr_set[dev] = true;
  }
  MlpWeights W{(const bf16*)w5[0], (const bf16*)w5[1], (const bf16*)w5[2], (const bf16*)w5[3], (const bf16*)w5[4], b2, b3};
  k_mlp_infer<<<(int)ceil_div(n, kTile), 256, smem, (cudaStream_t)stream>>>((const bf16*)X, V, n, W, out_scale, F,
                                                                             status_dev);
  return launch_status();
}

int acs_mlp_train_step(const void* X, const float* V, const float* Y, int64_t n, void* const* w5, float* b2,
                       float* b3, float* theta, float* adam_m, float* adam_v, float lr, int32_t step, float weight_decay,
                       float* gpart, size_t gpart_bytes, float* loss_part, float* grad_out, int32_t* status_dev,
                       void* stream) {
  if (n < 1 || !X || !V || !Y || !w5 || !b2 || !b3 || !theta || !adam_m || !adam_v || !gpart || !loss_part ||
      !status_dev || step < 1)
    return ACS_ERR_ARG;
  if (gpart_bytes < acs_mlp_grad_bytes(n)) return ACS_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t smem = MlpSmem::END;
  if (cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return ACS_ERR_CUDA;
  const int ntiles = (int)ceil_div(n, kTile);
  MlpWeights W{(const bf16*)w5[0], (const bf16*)w5[1], (const bf16*)w5[2], (const bf16*)w5[3], (const bf16*)w5[4], b2, b3};
  const float loss_scale = 1.0f / (3.0f * (float)n);
  k_mlp<true><<<ntiles, 128, smem, s>>>((const bf16*)X, V, Y, n, W, 1.0f, loss_scale, nullptr, gpart, loss_part,
                                        status_dev);
  int st = launch_status();
  if (st) return st;
  if (lr > 0.f) {
    const float b1 = 0.9f, b2c = 0.999f;
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2c, (float)step);
    const int P = 3 * kH * kGradCols;
    k_adam<<<(P + 255) / 256, 256, 0, s>>>(gpart, ntiles, theta, adam_m, adam_v, lr, b1, b2c, 1e-8f, bc1, bc2,
                                           weight_decay, (bf16*)w5[0], (bf16*)w5[1], (bf16*)w5[2], (bf16*)w5[3],
                                           (bf16*)w5[4], b2, b3, grad_out);
  } else {
    const int P = 3 * kH * kGradCols;
    k_adam<<<(P + 255) / 256, 256, 0, s>>>(gpart, ntiles, theta, adam_m, adam_v, 0.f, 0.9f, 0.999f, 1e-8f, 1.f, 1.f,
                                           0.f, (bf16*)w5[0], (bf16*)w5[1], (bf16*)w5[2], (bf16*)w5[3], (bf16*)w5[4],
                                           b2, b3, grad_out);
  }
  return launch_status();
}

}  // extern "C"
