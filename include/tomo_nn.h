/*
 * tomo_nn.h -- C ABI of libtomo_nn.so: the convolution kernels of the learned
 * warm start (a small U-Net that maps a 2-iteration SIRT image to a start
 * close to the converged reconstruction).  No reference counterpart: the
 * reference has no learned component.
 *
 * Layouts: activations are BF16, NHWC ([batch][H][W][C], C fastest); 3x3
 * weights are [Cout][3][3][Cin] (tap = ky*3 + kx, input channel fastest);
 * channel counts of GEMM operands are multiples of 8 (pad with zero channels).
 * All pointers are device pointers; every call is stream-ordered on `stream`
 * (a cudaStream_t passed as void*) and allocates nothing.
 *
 * Status: 0 on success, TOMO_NN_EINVAL for bad sizes or alignment (operand
 * base pointers must be 16-byte aligned), TOMO_NN_ECUDA for a launch error.
 * A tensor-core wait that gives up inside a kernel does not fault: the kernel
 * records it in a device status word that tomo_nn_status() returns.
 */
#ifndef TOMO_NN_H
#define TOMO_NN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TOMO_NN_OK 0
#define TOMO_NN_EINVAL 22
#define TOMO_NN_ETIMEDOUT 110
#define TOMO_NN_ECUDA 1000

/* C = A . B^T on the tensor cores: A [M][K] (row stride lda), B [N][K] (ldb),
 * BF16; FP32 accumulation; C written as FP32 (Cf) or BF16 (Cb), [M][N] with
 * row stride ldc, after adding bias[N] (may be NULL) and, if relu != 0, ReLU.
 * K, lda and ldb are multiples of 8. */
int tomo_nn_gemm(const void *A, int lda, const void *B, int ldb, int M, int N, int K, float *Cf, void *Cb,
                 int ldc, const float *bias, int relu, void *stream);

/* 3x3 convolution, stride 1, zero padding 1: X [batch][H][W][Cin] BF16,
 * Wt [Cout][3][3][Cin] BF16, Y [batch][H][W][Cout] as FP32 (Yf) or BF16 (Yb),
 * plus bias[Cout] (may be NULL) and optional ReLU.  Cin is a multiple of 8.
 * The input gradient of a convolution is this call on the output gradient
 * with the weights from tomo_nn_prepare_weights (Wd). */
int tomo_nn_conv3x3(const void *X, int batch, int H, int W, int Cin, const void *Wt, int Cout, float *Yf,
                    void *Yb, const float *bias, int relu, void *stream);

/* Weight and bias gradients of a convolution with `taps` = 9 (3x3, pad 1) or
 * 1 (1x1): dW [Cout][taps][Cin] = sum over pixels p of dY[p][co] x
 * im2col(X)[p][(tap, ci)], db[Cout] = sum_p dY[p][co] (db may be NULL); X
 * [batch][H][W][Cin] and dY [batch][H][W][Cout] BF16, dW and db FP32
 * (overwritten).  The pixel sum runs as a split-K tensor-core GEMM whose
 * partial tiles are added in a fixed order, so the result is deterministic.
 * `work` must hold tomo_nn_wgrad_workspace(...) bytes. */
size_t tomo_nn_wgrad_workspace(int batch, int H, int W, int Cin, int Cout, int taps);
int tomo_nn_wgrad(const void *X, const void *dY, int batch, int H, int W, int Cin, int Cout, int taps,
                  float *dW, float *db, void *work, size_t work_bytes, void *stream);

/* From FP32 master weights W [Cout][taps][Cin]: Wb = BF16 copy (forward) and,
 * if Wd != NULL, Wd [Cin][taps][Cout] BF16 with the taps reversed (the input
 * gradient's weights: a 3x3 tap (ky, kx) becomes (2-ky, 2-kx)). */
int tomo_nn_prepare_weights(const float *W, int Cout, int Cin, int taps, void *Wb, void *Wd, void *stream);

/* ReLU backward in place on BF16 arrays: dY[i] = Y[i] > 0 ? dY[i] : 0. */
int tomo_nn_relu_bwd(const void *Y, void *dY, size_t n, void *stream);

/* One Adam step on FP32 parameters p with gradient g and moments m, v
 * (step >= 1; bias-corrected; no weight decay). */
int tomo_nn_adam(float *p, const float *g, float *m, float *v, size_t n, float lr, float beta1, float beta2,
                 float eps, int step, void *stream);

/* How many times the tensor-core kernels poll a pipeline barrier (the wait
 * for the MMAs that read a shared-memory stage before it is refilled) before
 * they give up: spins >= 0 sets the limit for later launches in this process
 * (0: give up at once, which only serves to exercise the give-up path), spins
 * < 0 restores the default of 2^22.  A kernel that gives up sets bit 0 of the
 * status word, stores nothing, and before freeing its tensor memory waits for
 * its last committed MMAs with the long default limit whatever this setting. */
int tomo_nn_set_wait_limit(int spins);

/* Reads and clears the device status word of the current device (bit 0: a
 * tensor-core wait gave up); synchronises the device. */
int tomo_nn_status(unsigned *flags);

#ifdef __cplusplus
}
#endif

#endif /* TOMO_NN_H */
