/*
 * surrogate_b200.h — C ABI of the learned screening surrogate's device kernels.
 *
 * No counterpart in the reference.  Its planners score every candidate
 * control sequence with the cost batch `jax.vmap(cost_fn)` inside MBD's reverse
 * diffusion step (medea_ice_ship/jax_mbd_planner.py:1363-1380).  Here a small
 * conv + MLP network predicts the ice terms of that cost (kinetic energy
 * transferred to the ice, hull impulse, bonds broken) from (costmap patch,
 * ship state, controls), so that only the best few candidates of each
 * iteration are rolled out by the DEM (dem_rollout_segment).
 *
 * All arrays are DEVICE pointers owned by the caller; bf16 arrays are
 * 16-bit bfloat16 words.  Every call is asynchronous on `stream` (a
 * cudaStream_t; NULL = default stream) and returns SG_OK or an error code for
 * a bad argument or a failed launch.  A kernel that finds a problem on the
 * device (a wait that ran past its time limit) sets *err to nonzero; no
 * kernel traps.
 */
#ifndef SURROGATE_B200_H
#define SURROGATE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_OK 0
#define SG_ERR_INVALID 1
#define SG_ERR_CUDA 2

#define SG_OUT_F32 0
#define SG_OUT_BF16 1

/* D = act(A B^T + bias) (x) [mask > 0] on the 5th-generation tensor cores
 * (tcgen05.mma, bf16 operands, fp32 accumulation in tensor memory, operand
 * tiles loaded by TMA).  A (M, K) and B (N, K) are bf16, row-major with row
 * strides lda, ldb (elements; multiples of 8, >= K), 16-byte aligned.  D (M, N)
 * row-major with row stride ldd, fp32 (SG_OUT_F32) or bf16 (SG_OUT_BF16).
 * bias (N,) fp32 or NULL; relu != 0 clamps at 0 after the bias; mask (M, ldm)
 * bf16 or NULL multiplies each entry by (mask > 0) (the ReLU derivative of a
 * forward activation).  err: one device int32, set nonzero if a wait timed out. */
int sg_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B, int32_t ldb, void* D,
            int32_t ldd, int32_t d_dtype, const float* bias, int32_t relu, const void* mask, int32_t ldm, int32_t* err,
            void* stream);

/* 3x3 convolution, stride 2, padding 1, as a GEMM over patches.  X (B, H, W, C)
 * bf16 (NHWC, H and W even) -> cols (B * H/2 * W/2, kpad) bf16, each row the
 * 3x3xC patch in (ky, kx, c) order, zero-padded from 9C to kpad columns. */
int sg_im2col(int32_t B, int32_t H, int32_t W, int32_t C, const void* X, int32_t kpad, void* cols, void* stream);

/* Adjoint of sg_im2col: dX (B, H, W, C) = sum of the patch gradients dcols
 * (B * H/2 * W/2, kpad) fp32 over every patch that holds the pixel (a gather,
 * in a fixed order), times (act > 0) where act (B, H, W, C) bf16 is given;
 * written as bf16. */
int sg_col2im(int32_t B, int32_t H, int32_t W, int32_t C, const float* dcols, int32_t kpad, const void* act,
              void* dX, void* stream);

/* out (cols, rows) = in (rows, cols)^T for bf16 matrices with row strides ld_in / ld_out. */
int sg_transpose(int32_t rows, int32_t cols, const void* in, int32_t ld_in, void* out, int32_t ld_out,
                 void* stream);

/* out[j] = sum_i in[i, j] over rows of a (rows, cols) matrix with row stride ld:
 * fp32 (in_bf16 = 0) or bf16 (in_bf16 = 1); fixed summation order. */
int sg_colsum(int32_t rows, int32_t cols, const void* in, int32_t ld, int32_t in_bf16, float* out, void* stream);

/* One Adam step (bias-corrected, step t >= 1) on n fp32 master weights p with
 * gradients g and moments m, v; also writes the bf16 copy w (rows, cols) with
 * row stride ldw (n = rows * cols, p row-major) and, if wt is not NULL, its
 * transpose (cols, rows) with row stride ldwt. */
int sg_adam(int32_t rows, int32_t cols, float* p, const float* g, float* m, float* v, float lr, float beta1,
            float beta2, float eps, int32_t t, void* w, int32_t ldw, void* wt, int32_t ldwt, void* stream);

/* Mean squared error over (rows, n_out) of pred (row stride ldp, fp32) against
 * target (row stride ldt, fp32): grad (rows, ldg) bf16 = 2 (pred - target) /
 * (rows n_out) in the first n_out columns, 0 in columns n_out .. ldg-1; loss
 * (1,) fp32 = the mean (fixed summation order). */
int sg_mse(int32_t rows, int32_t n_out, const float* pred, int32_t ldp, const float* target, int32_t ldt,
           void* grad, int32_t ldg, float* loss, void* stream);

/* MLP input rows (rows, ldx) bf16: [enc (enc_dim, bf16, row enc_row[r] of enc
 * with row stride ld_enc, or row r when enc_row is NULL) | extra (n_extra fp32,
 * row stride ld_extra) | zeros up to ldx]. */
int sg_pack_rows(int32_t rows, int32_t enc_dim, const void* enc, int32_t ld_enc, const int32_t* enc_row,
                 int32_t n_extra, const float* extra, int32_t ld_extra, void* x, int32_t ldx, void* stream);

/* The first enc_dim columns of dx (rows, ldx) bf16, times (act > 0) for act
 * (rows, enc_dim) bf16, into d_enc (rows, enc_dim) bf16. */
int sg_unpack_grad(int32_t rows, int32_t enc_dim, const void* dx, int32_t ldx, const void* act, void* d_enc,
                   void* stream);

/* out row r (row_bytes bytes, at r * ld_out_bytes) = in row idx[r] (at
 * idx[r] * ld_in_bytes); idx (rows,) int32 device array. */
int sg_gather_rows(int32_t rows, int64_t row_bytes, const void* in, int64_t ld_in_bytes, const int32_t* idx,
                   void* out, int64_t ld_out_bytes, void* stream);

/* fp32 -> bf16 (round to nearest even), n entries. */
int sg_to_bf16(int64_t n, const float* in, void* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SURROGATE_B200_H */
