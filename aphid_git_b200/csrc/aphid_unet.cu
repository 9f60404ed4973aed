// aphid_unet.cu -- the initial-guess network's device side: the tcgen05 BF16
// GEMM launcher and (below) the layers built on it.  C ABI in
// include/aphid_unet.h.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <string>

#include "../../include/aphid_unet.h"
#include "unet_gemm.cuh"

namespace aphid {
namespace unet {

namespace {

thread_local std::string g_last_error = "no error";

int set_err(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

template <int BN, int OUT>
int launch_gemm_t(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, void *C, int ldc,
                  const float *bias, int M, int N, int K, int splitk, cudaStream_t st, int *err) {
  const size_t shm = GemmShm<BN>::bytes;
  if (cudaFuncSetAttribute(k_gemm_bf16<BN, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) !=
      cudaSuccess)
    return set_err(APHID_UNET_ERR_CUDA, "cudaFuncSetAttribute (gemm)");
  const int nkb = K / kBK;
  const int per = (nkb + splitk - 1) / splitk;
  dim3 grid((unsigned)(M / kBM), (unsigned)(N / BN), (unsigned)((nkb + per - 1) / per));
  k_gemm_bf16<BN, OUT><<<grid, kGemmThreads, shm, st>>>(A, lda, B, ldb, C, ldc, bias, K, per * kBK, err);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(APHID_UNET_ERR_CUDA, std::string("gemm launch: ") + cudaGetErrorString(e));
  return APHID_UNET_OK;
}

template <int OUT>
int launch_gemm_o(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, void *C, int ldc,
                  const float *bias, int M, int N, int K, int splitk, cudaStream_t st, int *err) {
  if (N % 128 == 0) return launch_gemm_t<128, OUT>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
  if (N % 64 == 0) return launch_gemm_t<64, OUT>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
  if (N % 32 == 0) return launch_gemm_t<32, OUT>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
  return launch_gemm_t<16, OUT>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
}

}  // namespace

// C (op)= A B^T on the tensor cores; see unet_gemm.cuh for the shapes
int gemm_bf16(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, void *C, int ldc,
              const float *bias, int M, int N, int K, int out, int splitk, cudaStream_t st, int *err) {
  if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % 16 || K % kBK || lda % 8 || ldb % 8 || lda < K || ldb < K ||
      ldc < N || splitk < 1)
    return set_err(APHID_UNET_ERR_BADARG, "gemm: M % 128, N % 16, K % 64 and the leading dimensions");
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
    return set_err(APHID_UNET_ERR_BADARG, "gemm: A and B must be 16-byte aligned");
  if (splitk > 1 && out != OUT_F32_ATOMIC)
    return set_err(APHID_UNET_ERR_BADARG, "gemm: split-K needs the atomic output");
  switch (out) {
    case OUT_F32: return launch_gemm_o<OUT_F32>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
    case OUT_BF16_RELU: return launch_gemm_o<OUT_BF16_RELU>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
    case OUT_BF16: return launch_gemm_o<OUT_BF16>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
    case OUT_F32_ATOMIC: return launch_gemm_o<OUT_F32_ATOMIC>(A, lda, B, ldb, C, ldc, bias, M, N, K, splitk, st, err);
  }
  return set_err(APHID_UNET_ERR_BADARG, "gemm: unknown output operation");
}

}  // namespace unet
}  // namespace aphid

using namespace aphid::unet;

extern "C" {

const char *aphid_unet_last_error(void) { return g_last_error.c_str(); }

int aphid_unet_gemm_bf16(const void *A, int lda, const void *B, int ldb, void *C, int ldc, const float *bias, int M,
                         int N, int K, int out, int splitk, void *stream, int *err_flag) {
  return gemm_bf16(static_cast<const __nv_bfloat16 *>(A), lda, static_cast<const __nv_bfloat16 *>(B), ldb, C, ldc,
                   bias, M, N, K, out, splitk, static_cast<cudaStream_t>(stream), err_flag);
}

}  // extern "C"
