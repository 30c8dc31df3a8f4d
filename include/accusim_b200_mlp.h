/*
 * accusim_b200: Ewald summation and the learned DSF->Ewald force correction.
 *
 * acs_ewald_fp64 replaces accusim/forces.py:333-388 (Ewald.compute) on the device, FP64: the caller passes
 * the k-vectors and weights exactly as the reference builds them (accusim/forces.py:347-357), so the
 * result follows the reference's real-space, reciprocal and self terms. It labels training data for the
 * learned correction and measures its error.
 *
 * The learned correction has no counterpart in the reference: a BF16 tensor-core (tcgen05) MLP on per-ion
 * radial descriptors predicting the Ewald-minus-DSF force residual (see acs_mlp_* below).
 */
#ifndef ACCUSIM_B200_MLP_H
#define ACCUSIM_B200_MLP_H

#include "accusim_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

size_t acs_ewald_work_bytes(int64_t n, int32_t K);
/* pos (n x 3, m), q (n, C), kvec (K x 3, 1/m) and kw (K) are device arrays. force = k * f (N);
 * energy3_dev[0] = real-space pair sum (unscaled), [1] = sum_k w_k |S_k|^2 (unscaled): the host forms
 * U = k * (energy3[0] + 2 pi / V * energy3[1] - alpha / sqrt(pi) * sum q^2). */
int acs_ewald_fp64(const double* pos, const double* q, int64_t n, const double* box3, const double* kvec,
                   const double* kw, int32_t K, double alpha, double rcut, double k_coul, double* force,
                   double* energy3_dev, void* work, size_t work_bytes, void* stream);

/* Radial descriptors of n ions (positions in A, device; box3 and params6 = {r0, dmu, 1/(2 s^2), rc, 0, 0}
 * on the host) from a full neighbour list of radius >= rc in the acs_nlist_build layout: X (n x 80 BF16:
 * standardised invariants with mean/inv_std (device, 64 each), species one-hot, constant 1 in column 79)
 * and V (n x 64 x 3 FP32 vector features). Channel 32 t + k: neighbours of species t, Gaussian k. */
int acs_descriptors(const double* pos, const int32_t* sp, int64_t n, const double* box3, int periodic,
                    const int32_t* nbr, const int32_t* nnb, int32_t maxnb, const float* params6, const float* mean,
                    const float* inv_std, void* X_bf16, float* V, void* stream);
size_t acs_mlp_grad_bytes(int64_t n);
int32_t acs_mlp_param_count(void);
/* Forward pass on tcgen05: F (n x 3, FP32) = out_scale * sum_c C_c V_c with C = MLP(X). w5 = host array of
 * 5 device pointers {W1 (64x80), W2 (64x64), W3 (64x64), W2^T, W3^T} (BF16), b2, b3 FP32 (64). */
int acs_mlp_forward(const void* X, const float* V, int64_t n, const void* const* w5, const float* b2, const float* b3,
                    float out_scale, float* F, int32_t* status_dev, void* stream);
/* Forward + backward on tcgen05 for the loss sum |F - Y|^2 / (3 n), per-tile gradient partials reduced in
 * tile order, then an Adam step (lr > 0) on the FP32 parameter vector theta (3 x 64 x 80: W1 with its bias in
 * column 79, [W2 | b2], [W3 | b3]) that refreshes the BF16 operand copies and b2, b3. grad_out (optional,
 * device, 15360 floats) receives the gradient. lr = 0 computes the gradient only. */
int acs_mlp_train_step(const void* X, const float* V, const float* Y, int64_t n, void* const* w5, float* b2,
                       float* b3, float* theta, float* adam_m, float* adam_v, float lr, int32_t step, float weight_decay,
                       float* gpart, size_t gpart_bytes, float* loss_part, float* grad_out, int32_t* status_dev,
                       void* stream);

/* Tensor-core self-test: D[128 x N] = A[128 x K] * B[N x K]^T with BF16 A, B (row-major, device) and an
 * FP32 result, through the same tcgen05 path the MLP layers use. N, K multiples of 16 in [16, 256]. */
int acs_umma_gemm_test(const void* A, const void* B, float* D, int32_t N, int32_t K, int32_t* status_dev,
                       void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ACCUSIM_B200_MLP_H */
