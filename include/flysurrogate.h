/* flysurrogate.h - C ABI of the learned surrogate's GPU kernels (part of libflybrain.so).
 *
 * The surrogate is a small BF16 multilayer perceptron (1280 -> 512 -> 512 -> 10, GELU, Poisson
 * negative log-likelihood on log-rates) trained on frames the LIF engine generates; it predicts
 * the descending neurons' spike counts of a frame and pre-screens interface candidates of the
 * reference's CMA-ES calibration (flyzero/tune.py:26-166), whose full race per candidate it
 * replaces for the screening step. The reference has no surrogate: these entry points have no
 * counterpart there.
 *
 * Conventions as in flybrain.h: FB_OK / FB_ERR_* return codes, fb_last_error() for the message,
 * device pointers, work enqueued on `stream`. Matrices are row-major; bf16 is stored as uint16_t.
 */
#ifndef FLYSURROGATE_H
#define FLYSURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Epilogues of fs_gemm (C = A * B^T accumulated in FP32 on the tensor cores) */
#define FS_EPI_F32 0          /* out_f32[i][j] = C */
#define FS_EPI_BIAS_GELU 1    /* z = C + bias[j] -> out_f32 (pre-activation, kept for backward),
                                 gelu(z) -> out_bf16, and its transpose -> out_bf16_t */
#define FS_EPI_BIAS_F32 2     /* out_f32 = C + bias[j] */
#define FS_EPI_GELU_GRAD 3    /* d = C * gelu'(zin[i][j]) -> out_bf16, transpose -> out_bf16_t */

/* GEMM kinds: the BF16 m16n8k16 warp MMA; tcgen05 (one thread issues 128 x N x 16 tensor-core
 * MMAs from shared-memory descriptors, FP32 accumulator in tensor memory) with operands staged by
 * cp.async; or the same fed by TMA (2-D tensor loads with the 128-byte swizzle into a 4-stage
 * mbarrier ring; operands whose base is not 16-byte aligned take the cp.async form). Default: TMA. */
#define FS_GEMM_MMA_SYNC 0
#define FS_GEMM_TCGEN05 1
#define FS_GEMM_TCGEN05_TMA 2

/* Select the kind fs_gemm uses (-1: keep); returns the previous kind. */
int fs_gemm_kind(int32_t kind);

/* Largest K split of the TMA kind (1 .. 8; -1: keep; default 8); returns the previous limit. A GEMM
 * with few output tiles and a long K (the weight gradients: M = 512, K = the batch) splits each
 * tile's K range over a cluster of up to that many blocks, enough to fill two blocks per SM with at
 * least four 64-deep K tiles each; the FP32 partials are summed in a fixed order, so results
 * depend on the split chosen for the shape and limit, not on scheduling. A bad limit returns
 * -FB_ERR_ARG. */
int fs_gemm_split(int32_t max_split);

/* C[M x N] = A[M x K] * B[N x K]^T with bf16 A (row stride lda), bf16 B (row stride ldb), FP32
 * accumulation, then the epilogue `epi` writing rows of stride ldo (transposed outputs: stride
 * ldo_t). Any M, N, K >= 1; lda, ldb multiples of 8. */
int fs_gemm(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, int32_t lda, int32_t ldb,
            int32_t epi, const float* bias, const float* zin, float* out_f32, uint16_t* out_bf16,
            uint16_t* out_bf16_t, int32_t ldo, int32_t ldo_t, void* stream);

/* Poisson NLL on log-rates z (M x D, FP32) against counts y (M x D, FP32):
 * loss_sum[0] += sum(exp(z) - y * z) (FP64), dz = (exp(z) - y) / M as bf16 (row stride ldd >= D;
 * columns D..ldd-1 are left untouched) and its transpose (D x M). */
int fs_poisson_nll(const float* z, const float* y, int32_t M, int32_t D, double* loss_sum, uint16_t* dz,
                   int32_t ldd, uint16_t* dz_t, void* stream);

/* Column sums of a bf16 matrix (M x N, row stride ld) into FP32 grad[N] (the bias gradient). */
int fs_colsum(const uint16_t* X, int32_t M, int32_t N, int32_t ld, float* grad, void* stream);

/* Adam on FP32 master weights w[n] with FP32 moments m, v: bias-corrected with step t (>= 1);
 * writes the bf16 copy w_bf16 (same layout) and, when w_bf16_t != NULL, the transposed bf16 copy
 * of the rows x cols weight (rows * cols == n, 0 < rows <= 2,097,120) with row stride ldt >= rows. */
int fs_adam(float* w, const float* grad, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
            float eps, int32_t t, uint16_t* w_bf16, uint16_t* w_bf16_t, int32_t rows, int32_t cols, int32_t ldt,
            void* stream);

/* FP32 -> bf16 (round to nearest even); optional transposed copy of the rows x cols matrix
 * (rows * cols == n, 0 < rows <= 2,097,120) with row stride ldt >= rows. */
int fs_to_bf16(const float* x, int64_t n, uint16_t* out, uint16_t* out_t, int32_t rows, int32_t cols, int32_t ldt,
               void* stream);

#ifdef __cplusplus
}
#endif

#endif
