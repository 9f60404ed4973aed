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

/* ---- the network --------------------------------------------------------
 * 3-D U-Net: four levels of 16/32/64/128 channels, two 3x3x3 convolutions
 * with ReLU per level and side, 2x2x2 mean pooling, nearest upsampling with
 * skip concatenation, a 3x3x3 head to 8 channels.  Weights BF16 on the
 * tensor cores with FP32 master copies (Adam); activations BF16; FP32
 * accumulation.  A network object holds the buffers for one volume of
 * nodes (X, Y, Z), internally padded to multiples of 8; parameters move
 * between objects of different volumes through get/set_params.
 * Parameter layout (host, FP32): per layer W[co][tap*cin + ci], then b[co],
 * tap = ((dz+1)*3 + (dy+1))*3 + (dx+1), layers in the order
 * 3-16, 16-16, 16-32, 32-32, 32-64, 64-64, 64-128, 128-128, 192-64, 64-64,
 * 96-32, 32-32, 48-16, 16-16, 16-8.
 * Features x: [V][3] and targets / outputs [V][8] (FP32, device), voxel
 * v = i + X (j + Y k). */
typedef struct aphid_unet aphid_unet;

long long aphid_unet_param_count(void);
/* train = 0: inference buffers only.  seed: the initial He-normal weights. */
int aphid_unet_create(aphid_unet **net, int X, int Y, int Z, int train, unsigned long long seed);
int aphid_unet_destroy(aphid_unet *net);
int aphid_unet_get_params(aphid_unet *net, float *host);
int aphid_unet_set_params(aphid_unet *net, const float *host);  /* also resets the optimiser */
/* y = net(x); synchronises the stream. */
int aphid_unet_forward(aphid_unet *net, const float *x, float *y, void *stream);
/* One step on (x, target): loss = sum_v w_v sum_c (y - t)^2 / (8 sum_v w_v)
 * (weight NULL: all ones), its gradient by back-propagation, and, when
 * update != 0, one Adam step (lr; betas 0.9, 0.999).  Synchronises the
 * stream; *loss is the loss before the update. */
int aphid_unet_train_step(aphid_unet *net, const float *x, const float *target, const float *weight, float lr,
                          int update, double *loss, void *stream);
/* The parameter gradient of the last train step, in the parameter layout. */
int aphid_unet_get_grads(aphid_unet *net, float *host);

#ifdef __cplusplus
}
#endif

#endif /* APHID_UNET_H */
