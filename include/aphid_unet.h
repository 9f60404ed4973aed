/*
 * aphid_unet.h -- C ABI of the learned initial guess: a 3-D U-Net that maps
 * (log10 sigma, log10 f, source mask) on the mesh nodes to the eight real
 * channels of (Ax, Ay, Az, Phi), run and trained with BF16 tensor-core
 * (tcgen05) kernels with FP32 accumulation.  It has no counterpart in the
 * reference, whose QMR starts from zero (src/aphid_qmr.f90:230-233); its
 * output enters as the x0 of aphid_gpu_sweep / aphid_gpu_qmr and so changes
 * iteration counts, never the converged answer.
 *
 * All pointers are device pointers unless stated.  Calls launch on the
 * given stream (NULL = the legacy default stream) and return after the
 * launches.  Return APHID_UNET_OK or a negative code; the message of the
 * last failure on this host thread is in aphid_unet_last_error().
 */
#ifndef APHID_UNET_H
#define APHID_UNET_H

#ifdef __cplusplus
extern "C" {
#endif

#define APHID_UNET_OK          0
#define APHID_UNET_ERR_BADARG -1
#define APHID_UNET_ERR_CUDA   -2
#define APHID_UNET_ERR_NOMEM  -3

const char *aphid_unet_last_error(void);

/* C (op)= A B^T on the tensor cores.  A: M x K BF16 with leading dimension
 * lda, B: N x K BF16 (ldb), both K-contiguous and 16-byte aligned; C: M x N
 * (ldc).  out: 0 = C = AB^T (+bias[n]) as FP32; 1 = relu(AB^T + bias) as
 * BF16; 2 = AB^T + bias as BF16; 3 = C += AB^T, FP32, atomically (with
 * splitk > 1 the K range is split over that many CTAs).  bias may be NULL.
 * M % 128 == 0, N % 16 == 0, K % 64 == 0.  err_flag (device int, nullable)
 * is set when a bounded wait inside the kernel gave up. */
int aphid_unet_gemm_bf16(const void *A, int lda, const void *B, int ldb, void *C, int ldc, const float *bias,
                         int M, int N, int K, int out, int splitk, void *stream, int *err_flag);

#ifdef __cplusplus
}
#endif

#endif /* APHID_UNET_H */
