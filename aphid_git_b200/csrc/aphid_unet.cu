// aphid_unet.cu -- the initial-guess network's device side: the tcgen05 BF16
// GEMM launcher and (below) the layers built on it.  C ABI in
// include/aphid_unet.h.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

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

// cuTensorMapEncodeTiled through the runtime's driver entry point
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// a row-major BF16 matrix (rows x cols, leading dimension ld elements) as a
// 2-D tensor of box cols_box x rows_box, 128-byte swizzle
int bf16_map(CUtensorMap *m, const __nv_bfloat16 *base, int rows, int cols, int ld, int rows_box) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess || !f)
      return set_err(APHID_UNET_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = (EncodeTiledFn)f;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)rows_box}, es[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(base), dims, strides, box,
                        es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(APHID_UNET_ERR_CUDA, "cuTensorMapEncodeTiled (gemm): " + std::to_string((int)r));
  return APHID_UNET_OK;
}

template <int BN, int OUT>
int launch_gemm_t(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, void *C, int ldc,
                  const float *bias, int M, int N, int K, int splitk, cudaStream_t st, int *err) {
  const size_t shm = TmaShm<BN>::bytes;
  static bool attr = false;  // once per instantiation and process
  if (!attr) {
    if (cudaFuncSetAttribute(k_gemm_tma<BN, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) !=
        cudaSuccess)
      return set_err(APHID_UNET_ERR_CUDA, "cudaFuncSetAttribute (gemm)");
    attr = true;
  }
  CUtensorMap ma, mb;
  int rc;
  if ((rc = bf16_map(&ma, A, M, K, lda, kBM)) || (rc = bf16_map(&mb, B, N, K, ldb, BN))) return rc;
  const int nkb = K / kBK;
  const int per = (nkb + splitk - 1) / splitk;
  // 16-byte output stores where every row start is 16-byte aligned
  const size_t es = (OUT == OUT_BF16_RELU || OUT == OUT_BF16) ? 2 : 4;
  const int vec = (reinterpret_cast<uintptr_t>(C) % 16 == 0) && ((size_t)ldc * es) % 16 == 0;
  dim3 grid((unsigned)(M / kBM), (unsigned)(N / BN), (unsigned)((nkb + per - 1) / per));
  k_gemm_tma<BN, OUT><<<grid, kGemmThreads, shm, st>>>(ma, mb, C, ldc, bias, K, per * kBK, vec, err);
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


namespace aphid {
namespace unet {
namespace {

constexpr int kT = 256;  // threads of the elementwise kernels

__host__ __device__ inline long long rup(long long a, long long b) { return (a + b - 1) / b * b; }
inline unsigned nblk(long long n) { return (unsigned)std::min<long long>((n + kT - 1) / kT, 148LL * 64); }

struct Vol {
  int X, Y, Z;
  long long V, Vp;  // voxels, rows padded to 128
};

// ---------------------------------------------------------------- kernels
// features [V][3] (original volume) -> [Vp][8] BF16 on the padded volume
__global__ void k_pack_in(const float *__restrict__ x, int X, int Y, int Z, Vol v, __nv_bfloat16 *__restrict__ a) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < v.Vp * 8; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t >> 3;
    const int c = (int)(t & 7);
    float val = 0.f;
    if (r < v.V && c < 3) {
      const int px = (int)(r % v.X), py = (int)((r / v.X) % v.Y), pz = (int)(r / ((long long)v.X * v.Y));
      if (px < X && py < Y && pz < Z) val = x[(px + (long long)X * (py + (long long)Y * pz)) * 3 + c];
    }
    a[t] = __float2bfloat16_rn(val);
  }
}
// head output [Vp][16] FP32 -> [V][8] on the original volume
__global__ void k_unpack_out(const float *__restrict__ y, int X, int Y, int Z, Vol v, float *__restrict__ o) {
  const long long n = (long long)X * Y * Z * 8;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t >> 3;
    const int c = (int)(t & 7);
    const int px = (int)(r % X), py = (int)((r / X) % Y), pz = (int)(r / ((long long)X * Y));
    o[t] = y[(px + (long long)v.X * (py + (long long)v.Y * pz)) * 16 + c];
  }
}

__device__ __forceinline__ long long nb(const Vol &v, long long r, int t) {  // neighbour of r through tap t, or -1
  const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
  const int x = (int)(r % v.X) + dx, y = (int)((r / v.X) % v.Y) + dy, z = (int)(r / ((long long)v.X * v.Y)) + dz;
  if (x < 0 || y < 0 || z < 0 || x >= v.X || y >= v.Y || z >= v.Z) return -1;
  return x + (long long)v.X * (y + (long long)v.Y * z);
}

// col [Vp][kp]: col[r][t*C + c] = in[r + d_t][c] (zero outside), pads zero
__global__ void k_im2col(const __nv_bfloat16 *__restrict__ in, int C, Vol v, int kp, __nv_bfloat16 *__restrict__ col) {
  const int kc = kp / 8, used = 27 * C / 8;
  const uint4 z4 = make_uint4(0, 0, 0, 0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < v.Vp * kc; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / kc;
    const int q = (int)(t % kc);
    uint4 val = z4;
    if (q < used && r < v.V) {
      const int tap = q / (C / 8), c8 = q % (C / 8);
      const long long s = nb(v, r, tap);
      if (s >= 0) val = *reinterpret_cast<const uint4 *>(in + s * C + c8 * 8);
    }
    *reinterpret_cast<uint4 *>(col + r * kp + q * 8) = val;
  }
}
// colT [kp][Vp] (the transpose of col)
__global__ void k_im2colT(const __nv_bfloat16 *__restrict__ in, int C, Vol v, int kp, __nv_bfloat16 *__restrict__ colT) {
  const int kc = kp / 8, used = 27 * C / 8;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < v.Vp * kc; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t % v.Vp;
    const int q = (int)(t / v.Vp);
    uint4 val = make_uint4(0, 0, 0, 0);
    if (q < used && r < v.V) {
      const int tap = q / (C / 8), c8 = q % (C / 8);
      const long long s = nb(v, r, tap);
      if (s >= 0) val = *reinterpret_cast<const uint4 *>(in + s * C + c8 * 8);
    }
    const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&val);
#pragma unroll
    for (int j = 0; j < 8; j++) colT[(long long)(q * 8 + j) * v.Vp + r] = e[j];
  }
}
// gIn[u][c] += sum_t dcol[u - d_t][t*C + c]
__global__ void k_col2im(const float *__restrict__ dcol, int C, Vol v, int kp, float *__restrict__ gin) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < v.V * C; t += (long long)gridDim.x * blockDim.x) {
    const long long u = t / C;
    const int c = (int)(t % C);
    float s = 0.f;
#pragma unroll 1
    for (int tap = 0; tap < 27; tap++) {
      const long long r = nb(v, u, 26 - tap);  // u - d_tap = u + d_(26-tap)
      if (r >= 0) s += dcol[r * kp + tap * C + c];
    }
    gin[u * C + c] += s;
  }
}
// dz = g * (act > 0) (relu) or g; dZ [Vp][c64] and dZT [cn][Vp] in BF16, pads zero
__global__ void k_relu_back(const float *__restrict__ g, const __nv_bfloat16 *__restrict__ act, int C, int relu, Vol v,
                            int c64, int cn, __nv_bfloat16 *__restrict__ dZ, __nv_bfloat16 *__restrict__ dZT) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < v.Vp * c64; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / c64;
    const int c = (int)(t % c64);
    float d = 0.f;
    if (r < v.V && c < C) {
      d = g[r * C + c];
      if (relu && !(__bfloat162float(act[r * C + c]) > 0.f)) d = 0.f;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(d);
    dZ[t] = b;
    if (c < cn) dZT[(long long)c * v.Vp + r] = b;
  }
}
// gb[c] += sum_r dz[r][c] (FP32 dz, before rounding)
__global__ void k_bias_grad(const float *__restrict__ g, const __nv_bfloat16 *__restrict__ act, int C, int relu, Vol v,
                            float *__restrict__ gb) {
  const int c = blockIdx.y;
  float s = 0.f;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < v.V; r += (long long)gridDim.x * blockDim.x) {
    float d = g[r * C + c];
    if (relu && !(__bfloat162float(act[r * C + c]) > 0.f)) d = 0.f;
    s += d;
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float sh[kT / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int q = 0; q < kT / 32; q++) t += sh[q];
    atomicAdd(gb + c, t);
  }
}
// 2x2x2 mean: fine volume f -> coarse volume o
__global__ void k_pool(const __nv_bfloat16 *__restrict__ in, int C, Vol f, Vol o, __nv_bfloat16 *__restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < o.Vp * C; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / C;
    const int c = (int)(t % C);
    float s = 0.f;
    if (r < o.V) {
      const int x = (int)(r % o.X), y = (int)((r / o.X) % o.Y), z = (int)(r / ((long long)o.X * o.Y));
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const long long fr = (2 * x + (q & 1)) + (long long)f.X * ((2 * y + ((q >> 1) & 1)) + (long long)f.Y * (2 * z + (q >> 2)));
        s += __bfloat162float(in[fr * C + c]);
      }
      s *= 0.125f;
    }
    out[t] = __float2bfloat16_rn(s);
  }
}
// gf[child][c] += go[parent][c] / 8
__global__ void k_pool_back(const float *__restrict__ go, int C, Vol f, Vol o, float *__restrict__ gf) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < f.V * C; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / C;
    const int c = (int)(t % C);
    const int x = (int)(r % f.X), y = (int)((r / f.X) % f.Y), z = (int)(r / ((long long)f.X * f.Y));
    gf[t] += 0.125f * go[((x >> 1) + (long long)o.X * ((y >> 1) + (long long)o.Y * (z >> 1))) * C + c];
  }
}
// cat[r] = up(low)[r] (Cu channels) ++ skip[r] (Cs channels) on the fine volume
__global__ void k_upcat(const __nv_bfloat16 *__restrict__ low, int Cu, const __nv_bfloat16 *__restrict__ skip, int Cs,
                        Vol f, Vol o, __nv_bfloat16 *__restrict__ cat) {
  const int C = Cu + Cs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < f.Vp * C; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / C;
    const int c = (int)(t % C);
    __nv_bfloat16 val = __float2bfloat16_rn(0.f);
    if (r < f.V) {
      if (c < Cu) {
        const int x = (int)(r % f.X), y = (int)((r / f.X) % f.Y), z = (int)(r / ((long long)f.X * f.Y));
        val = low[((x >> 1) + (long long)o.X * ((y >> 1) + (long long)o.Y * (z >> 1))) * Cu + c];
      } else {
        val = skip[r * Cs + (c - Cu)];
      }
    }
    cat[t] = val;
  }
}
// the gradient of k_upcat: glow[p][c] += sum over the 8 children, gskip += tail
__global__ void k_upcat_back_low(const float *__restrict__ gcat, int Cu, int Cs, Vol f, Vol o, float *__restrict__ glow) {
  const int C = Cu + Cs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < o.V * Cu; t += (long long)gridDim.x * blockDim.x) {
    const long long p = t / Cu;
    const int c = (int)(t % Cu);
    const int x = (int)(p % o.X), y = (int)((p / o.X) % o.Y), z = (int)(p / ((long long)o.X * o.Y));
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const long long fr = (2 * x + (q & 1)) + (long long)f.X * ((2 * y + ((q >> 1) & 1)) + (long long)f.Y * (2 * z + (q >> 2)));
      s += gcat[fr * C + c];
    }
    glow[t] += s;
  }
}
__global__ void k_upcat_back_skip(const float *__restrict__ gcat, int Cu, int Cs, Vol f, float *__restrict__ gskip) {
  const int C = Cu + Cs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < f.V * Cs; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / Cs;
    const int c = (int)(t % Cs);
    gskip[t] += gcat[r * C + Cu + c];
  }
}
// weighted squared error of the head output against [V][8] targets:
// sums[0] += sum w, sums[1] += sum w r^2 (w per voxel, 8 channels each)
__global__ void k_loss_sums(const float *__restrict__ y, const float *__restrict__ tgt, const float *__restrict__ w,
                            int X, int Y, int Z, Vol v, double *__restrict__ sums) {
  const long long n = (long long)X * Y * Z;
  double sw = 0.0, se = 0.0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    const int px = (int)(r % X), py = (int)((r / X) % Y), pz = (int)(r / ((long long)X * Y));
    const long long q = px + (long long)v.X * (py + (long long)v.Y * pz);
    const float wr = w ? w[r] : 1.f;
    float e = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const float d = y[q * 16 + c] - tgt[r * 8 + c];
      e += d * d;
    }
    sw += 8.0 * wr;
    se += (double)wr * e;
  }
  for (int o = 16; o; o >>= 1) {
    sw += __shfl_xor_sync(0xffffffffu, sw, o);
    se += __shfl_xor_sync(0xffffffffu, se, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sums, sw);
    atomicAdd(sums + 1, se);
  }
}
// dy = 2 w (y - t) / sum w on the padded head output (pads zero)
__global__ void k_loss_grad(const float *__restrict__ y, const float *__restrict__ tgt, const float *__restrict__ w,
                            int X, int Y, int Z, Vol v, const double *__restrict__ sums, float *__restrict__ gy) {
  const float inv = (float)(2.0 / fmax(sums[0], 1e-30));
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < v.Vp * 16; t += (long long)gridDim.x * blockDim.x) {
    const long long q = t >> 4;
    const int c = (int)(t & 15);
    float g = 0.f;
    if (q < v.V && c < 8) {
      const int px = (int)(q % v.X), py = (int)((q / v.X) % v.Y), pz = (int)(q / ((long long)v.X * v.Y));
      if (px < X && py < Y && pz < Z) {
        const long long r = px + (long long)X * (py + (long long)Y * pz);
        g = inv * (w ? w[r] : 1.f) * (y[t] - tgt[r * 8 + c]);
      }
    }
    gy[t] = g;
  }
}
// device copies of one layer's weights: Wb [cn][kp], WTb [kp][c64]
__global__ void k_cast_w(const float *__restrict__ W, int cin, int cg, int cout, int kp, int cn, int c64,
                         __nv_bfloat16 *__restrict__ Wb, __nv_bfloat16 *__restrict__ WTb) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)kp * c64; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t / c64), co = (int)(t % c64);
    const int tap = k / cg, ci = k % cg;
    float w = 0.f;
    if (co < cout && tap < 27 && ci < cin) w = W[(long long)co * 27 * cin + tap * cin + ci];
    const __nv_bfloat16 b = __float2bfloat16_rn(w);
    WTb[t] = b;
    if (co < cn) Wb[(long long)co * kp + k] = b;
  }
}
// Adam on one layer (FP32 master weights), gradient of W from gWT [kp][cn]
__global__ void k_adam(float *__restrict__ W, float *__restrict__ m, float *__restrict__ v2, const float *__restrict__ gWT,
                       int cin, int cg, int cout, int cn, float *__restrict__ b, float *__restrict__ mb,
                       float *__restrict__ vb, const float *__restrict__ gb, float lr, float c1, float c2) {
  const long long nw = (long long)cout * 27 * cin;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nw + cout; t += (long long)gridDim.x * blockDim.x) {
    float g, *p, *pm, *pv;
    if (t < nw) {
      const int co = (int)(t / (27 * cin)), k = (int)(t % (27 * cin));
      const int tap = k / cin, ci = k % cin;
      g = gWT[(long long)(tap * cg + ci) * cn + co];
      p = W + t, pm = m + t, pv = v2 + t;
    } else {
      const int co = (int)(t - nw);
      g = gb[co];
      p = b + co, pm = mb + co, pv = vb + co;
    }
    const float mt = 0.9f * *pm + 0.1f * g, vt = 0.999f * *pv + 0.001f * g * g;
    *pm = mt;
    *pv = vt;
    *p -= lr * (mt * c1) / (sqrtf(vt * c2) + 1e-8f);
  }
}
// the gradient in the parameter layout
__global__ void k_grad_out(const float *__restrict__ gWT, const float *__restrict__ gb, int cin, int cg, int cout, int cn,
                           float *__restrict__ out) {
  const long long nw = (long long)cout * 27 * cin;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nw + cout; t += (long long)gridDim.x * blockDim.x) {
    if (t < nw) {
      const int co = (int)(t / (27 * cin)), k = (int)(t % (27 * cin));
      out[t] = gWT[(long long)((k / cin) * cg + k % cin) * cn + co];
    } else {
      out[t] = gb[t - nw];
    }
  }
}

}  // namespace

// ----------------------------------------------------------------- network
struct Layer {
  int cin, cg, cout, cn, c64, kp, level, relu;  // cg: cin rounded to 8; cn: cout rounded to 16
  float *W = nullptr, *b = nullptr, *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr;
  float *gWT = nullptr, *gb = nullptr;
  __nv_bfloat16 *Wb = nullptr, *WTb = nullptr;
  long long nparam() const { return 27LL * cin * cout + cout; }
};

// activations: index, level, channels
enum {
  A_IN, A0, S1, P1, A2, S2, P2, A4, S3, P3, A6, A7, CAT3, A8, A9, CAT2, A10, A11, CAT1, A12, A13, A_COUNT
};

}  // namespace unet
}  // namespace aphid

struct aphid_unet {
  int X, Y, Z, train;
  aphid::unet::Vol vol[4];
  std::vector<aphid::unet::Layer> L;
  __nv_bfloat16 *act[aphid::unet::A_COUNT] = {};
  float *grad[aphid::unet::A_COUNT] = {};
  int ach[aphid::unet::A_COUNT], alev[aphid::unet::A_COUNT];
  float *y = nullptr, *gy = nullptr;               // head output / its gradient [Vp][16]
  __nv_bfloat16 *col = nullptr, *colT = nullptr, *dZ = nullptr, *dZT = nullptr;
  float *dcol = nullptr;
  double *sums = nullptr;
  int *err = nullptr;
  long long step = 0;
  std::vector<void *> owned;
};

namespace aphid {
namespace unet {
namespace {

const int kLayerDef[15][4] = {  // cin, cout, level, relu
    {3, 16, 0, 1},  {16, 16, 0, 1},  {16, 32, 1, 1},  {32, 32, 1, 1},  {32, 64, 2, 1},
    {64, 64, 2, 1}, {64, 128, 3, 1}, {128, 128, 3, 1}, {192, 64, 2, 1}, {64, 64, 2, 1},
    {96, 32, 1, 1}, {32, 32, 1, 1},  {48, 16, 0, 1},  {16, 16, 0, 1},  {16, 8, 0, 0}};
// input activation and output activation of each layer (-1: head output)
const int kLayerIO[15][2] = {{A_IN, A0}, {A0, S1}, {P1, A2}, {A2, S2}, {P2, A4}, {A4, S3}, {P3, A6}, {A6, A7},
                             {CAT3, A8}, {A8, A9}, {CAT2, A10}, {A10, A11}, {CAT1, A12}, {A12, A13}, {A13, -1}};

template <class T>
int dalloc(aphid_unet *n, T **p, size_t count) {
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return set_err(APHID_UNET_ERR_NOMEM, "unet: device allocation failed");
  }
  if (cudaMemset(q, 0, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess)
    return set_err(APHID_UNET_ERR_CUDA, "unet: cudaMemset");
  n->owned.push_back(q);
  *p = static_cast<T *>(q);
  return APHID_UNET_OK;
}

#define UK(call)                                                      \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess)                                            \
      return set_err(APHID_UNET_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define UR(call)        \
  do {                  \
    int r_ = (call);    \
    if (r_) return r_;  \
  } while (0)

int cast_weights(aphid_unet *n, cudaStream_t st) {
  for (auto &l : n->L)
    k_cast_w<<<nblk((long long)l.kp * l.c64), kT, 0, st>>>(l.W, l.cin, l.cg, l.cout, l.kp, l.cn, l.c64, l.Wb, l.WTb);
  UK(cudaGetLastError());
  return APHID_UNET_OK;
}

int conv_fwd(aphid_unet *n, int li, cudaStream_t st) {
  const Layer &l = n->L[li];
  const Vol &v = n->vol[l.level];
  const __nv_bfloat16 *in = n->act[kLayerIO[li][0]];
  k_im2col<<<nblk(v.Vp * (l.kp / 8)), kT, 0, st>>>(in, l.cg, v, l.kp, n->col);
  UK(cudaGetLastError());
  if (kLayerIO[li][1] < 0)
    return gemm_bf16(n->col, l.kp, l.Wb, l.kp, n->y, 16, l.b, (int)v.Vp, l.cn, l.kp, OUT_F32, 1, st, n->err);
  return gemm_bf16(n->col, l.kp, l.Wb, l.kp, n->act[kLayerIO[li][1]], l.cn, l.b, (int)v.Vp, l.cn, l.kp,
                   OUT_BF16_RELU, 1, st, n->err);
}

// gOut: gradient of this layer's output (FP32 [Vp][cn]); adds into the input's gradient
int conv_back(aphid_unet *n, int li, const float *gout, const __nv_bfloat16 *out, cudaStream_t st) {
  const Layer &l = n->L[li];
  const Vol &v = n->vol[l.level];
  const int io = kLayerIO[li][0];
  k_relu_back<<<nblk(v.Vp * l.c64), kT, 0, st>>>(gout, out, l.cn, l.relu, v, l.c64, l.cn, n->dZ, n->dZT);
  k_bias_grad<<<dim3((unsigned)std::min<long long>((v.V + kT - 1) / kT, 64), (unsigned)l.cout), kT, 0, st>>>(
      gout, out, l.cn, l.relu, v, l.gb);
  k_im2colT<<<nblk(v.Vp * (l.kp / 8)), kT, 0, st>>>(n->act[io], l.cg, v, l.kp, n->colT);
  UK(cudaGetLastError());
  UK(cudaMemsetAsync(l.gWT, 0, (size_t)l.kp * l.cn * sizeof(float), st));
  const int tiles = (l.kp / kBM) * std::max(1, l.cn / 128);
  const int splitk = std::max(1, std::min((int)(v.Vp / kBK), 296 / tiles));
  UR(gemm_bf16(n->colT, (int)v.Vp, n->dZT, (int)v.Vp, l.gWT, l.cn, nullptr, l.kp, l.cn, (int)v.Vp, OUT_F32_ATOMIC,
               splitk, st, n->err));
  if (li == 0) return APHID_UNET_OK;  // no gradient for the input features
  UR(gemm_bf16(n->dZ, l.c64, l.WTb, l.c64, n->dcol, l.kp, nullptr, (int)v.Vp, l.kp, l.c64, OUT_F32, 1, st, n->err));
  k_col2im<<<nblk(v.V * l.cg), kT, 0, st>>>(n->dcol, l.cg, v, l.kp, n->grad[io]);
  UK(cudaGetLastError());
  return APHID_UNET_OK;
}

int forward(aphid_unet *n, const float *x, cudaStream_t st) {
  const Vol *V = n->vol;
  k_pack_in<<<nblk(V[0].Vp * 8), kT, 0, st>>>(x, n->X, n->Y, n->Z, V[0], n->act[A_IN]);
  UK(cudaGetLastError());
  auto pool = [&](int a, int b, int lev) {
    k_pool<<<nblk(V[lev + 1].Vp * n->ach[a]), kT, 0, st>>>(n->act[a], n->ach[a], V[lev], V[lev + 1], n->act[b]);
  };
  auto upcat = [&](int low, int skip, int cat, int lev) {
    k_upcat<<<nblk(V[lev].Vp * n->ach[cat]), kT, 0, st>>>(n->act[low], n->ach[low], n->act[skip], n->ach[skip], V[lev],
                                                          V[lev + 1], n->act[cat]);
  };
  UR(conv_fwd(n, 0, st));
  UR(conv_fwd(n, 1, st));
  pool(S1, P1, 0);
  UR(conv_fwd(n, 2, st));
  UR(conv_fwd(n, 3, st));
  pool(S2, P2, 1);
  UR(conv_fwd(n, 4, st));
  UR(conv_fwd(n, 5, st));
  pool(S3, P3, 2);
  UR(conv_fwd(n, 6, st));
  UR(conv_fwd(n, 7, st));
  upcat(A7, S3, CAT3, 2);
  UR(conv_fwd(n, 8, st));
  UR(conv_fwd(n, 9, st));
  upcat(A9, S2, CAT2, 1);
  UR(conv_fwd(n, 10, st));
  UR(conv_fwd(n, 11, st));
  upcat(A11, S1, CAT1, 0);
  UR(conv_fwd(n, 12, st));
  UR(conv_fwd(n, 13, st));
  UR(conv_fwd(n, 14, st));
  UK(cudaGetLastError());
  return APHID_UNET_OK;
}

int backward(aphid_unet *n, cudaStream_t st) {
  const Vol *V = n->vol;
  for (int a = 0; a < A_COUNT; a++)
    if (n->grad[a]) UK(cudaMemsetAsync(n->grad[a], 0, (size_t)V[n->alev[a]].Vp * n->ach[a] * sizeof(float), st));
  for (auto &l : n->L) UK(cudaMemsetAsync(l.gb, 0, l.cn * sizeof(float), st));
  auto back = [&](int li) {
    const int o = kLayerIO[li][1];
    return o < 0 ? conv_back(n, li, n->gy, nullptr, st) : conv_back(n, li, n->grad[o], n->act[o], st);
  };
  auto split = [&](int cat, int low, int skip, int lev) {
    const int cu = n->ach[low], cs = n->ach[skip];
    k_upcat_back_low<<<nblk(V[lev + 1].V * cu), kT, 0, st>>>(n->grad[cat], cu, cs, V[lev], V[lev + 1], n->grad[low]);
    k_upcat_back_skip<<<nblk(V[lev].V * cs), kT, 0, st>>>(n->grad[cat], cu, cs, V[lev], n->grad[skip]);
  };
  auto pool_back = [&](int pooled, int fine, int lev) {
    k_pool_back<<<nblk(V[lev].V * n->ach[fine]), kT, 0, st>>>(n->grad[pooled], n->ach[fine], V[lev], V[lev + 1],
                                                              n->grad[fine]);
  };
  UR(back(14));
  UR(back(13));
  UR(back(12));
  split(CAT1, A11, S1, 0);
  UR(back(11));
  UR(back(10));
  split(CAT2, A9, S2, 1);
  UR(back(9));
  UR(back(8));
  split(CAT3, A7, S3, 2);
  UR(back(7));
  UR(back(6));
  pool_back(P3, S3, 2);
  UR(back(5));
  UR(back(4));
  pool_back(P2, S2, 1);
  UR(back(3));
  UR(back(2));
  pool_back(P1, S1, 0);
  UR(back(1));
  UR(back(0));
  UK(cudaGetLastError());
  return APHID_UNET_OK;
}

int check_err(aphid_unet *n, cudaStream_t st) {
  int e = 0;
  UK(cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  UK(cudaStreamSynchronize(st));
  if (e) return set_err(APHID_UNET_ERR_CUDA, "unet: a bounded wait in the tensor-core GEMM gave up");
  return APHID_UNET_OK;
}

}  // namespace
}  // namespace unet
}  // namespace aphid

using namespace aphid::unet;

extern "C" {

const char *aphid_unet_last_error(void) { return g_last_error.c_str(); }

long long aphid_unet_param_count(void) {
  long long n = 0;
  for (auto &d : kLayerDef) n += 27LL * d[0] * d[1] + d[1];
  return n;
}

int aphid_unet_create(aphid_unet **out, int X, int Y, int Z, int train, unsigned long long seed) {
  if (!out || X < 1 || Y < 1 || Z < 1) return set_err(APHID_UNET_ERR_BADARG, "unet_create: bad volume");
  *out = nullptr;
  aphid_unet *n = new aphid_unet();
  n->X = X, n->Y = Y, n->Z = Z, n->train = train ? 1 : 0;
  int dims[3] = {(int)rup(X, 8), (int)rup(Y, 8), (int)rup(Z, 8)};
  for (int l = 0; l < 4; l++) {
    Vol &v = n->vol[l];
    v.X = dims[0] >> l, v.Y = dims[1] >> l, v.Z = dims[2] >> l;
    v.V = (long long)v.X * v.Y * v.Z;
    v.Vp = rup(v.V, kBM);
  }
  const int ach[A_COUNT] = {8, 16, 16, 16, 32, 32, 32, 64, 64, 64, 128, 128, 192, 64, 64, 96, 32, 32, 48, 16, 16};
  const int alev[A_COUNT] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 2, 1, 1, 1, 0, 0, 0};
  int rc = APHID_UNET_OK;
  size_t colmax = 0;
  std::mt19937_64 rng(seed);
  for (int li = 0; li < 15 && !rc; li++) {
    Layer l;
    l.cin = kLayerDef[li][0], l.cout = kLayerDef[li][1], l.level = kLayerDef[li][2], l.relu = kLayerDef[li][3];
    l.cg = (int)rup(l.cin, 8), l.cn = (int)rup(l.cout, 16), l.c64 = (int)rup(l.cout, 64);
    l.kp = (int)rup(27LL * l.cg, kBM);
    const size_t nw = 27ULL * l.cin * l.cout;
    colmax = std::max(colmax, (size_t)n->vol[l.level].Vp * l.kp);
    if ((rc = dalloc(n, &l.W, nw)) || (rc = dalloc(n, &l.b, l.cn)) || (rc = dalloc(n, &l.Wb, (size_t)l.cn * l.kp)) ||
        (rc = dalloc(n, &l.WTb, (size_t)l.kp * l.c64)))
      break;
    if (train && ((rc = dalloc(n, &l.mW, nw)) || (rc = dalloc(n, &l.vW, nw)) || (rc = dalloc(n, &l.mb, l.cout)) ||
                  (rc = dalloc(n, &l.vb, l.cout)) || (rc = dalloc(n, &l.gWT, (size_t)l.kp * l.cn)) ||
                  (rc = dalloc(n, &l.gb, l.cn))))
      break;
    // He-normal initial weights, zero biases
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (27.f * l.cin)));
    std::vector<float> h(nw);
    for (auto &w : h) w = nd(rng);
    if (cudaMemcpy(l.W, h.data(), nw * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = set_err(APHID_UNET_ERR_CUDA, "unet_create: weight upload");
      break;
    }
    n->L.push_back(l);
  }
  for (int a = 0; a < A_COUNT && !rc; a++) {
    n->ach[a] = ach[a], n->alev[a] = alev[a];
    const size_t cnt = (size_t)n->vol[alev[a]].Vp * ach[a];
    rc = dalloc(n, &n->act[a], cnt);
    if (!rc && train && a != A_IN) rc = dalloc(n, &n->grad[a], cnt);
  }
  if (!rc) rc = dalloc(n, &n->y, (size_t)n->vol[0].Vp * 16);
  if (!rc) rc = dalloc(n, &n->col, colmax);
  if (!rc) rc = dalloc(n, &n->err, 1);
  if (!rc) rc = dalloc(n, &n->sums, 2);
  if (!rc && train) {
    size_t dzmax = 0, dctmax = 0;
    for (auto &l : n->L) {
      dzmax = std::max(dzmax, (size_t)n->vol[l.level].Vp * l.c64);
      dctmax = std::max(dctmax, (size_t)n->vol[l.level].Vp * l.cn);
    }
    if (!rc) rc = dalloc(n, &n->gy, (size_t)n->vol[0].Vp * 16);
    if (!rc) rc = dalloc(n, &n->colT, colmax);
    if (!rc) rc = dalloc(n, &n->dcol, colmax);
    if (!rc) rc = dalloc(n, &n->dZ, dzmax);
    if (!rc) rc = dalloc(n, &n->dZT, dctmax);
  }
  if (!rc) rc = cast_weights(n, 0);
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = set_err(APHID_UNET_ERR_CUDA, "unet_create: initialisation");
  if (rc) {
    aphid_unet_destroy(n);
    return rc;
  }
  *out = n;
  return APHID_UNET_OK;
}

int aphid_unet_destroy(aphid_unet *n) {
  if (!n) return APHID_UNET_OK;
  for (void *p : n->owned) cudaFree(p);
  delete n;
  return APHID_UNET_OK;
}

int aphid_unet_get_params(aphid_unet *n, float *host) {
  if (!n || !host) return set_err(APHID_UNET_ERR_BADARG, "unet_get_params: null");
  size_t o = 0;
  for (auto &l : n->L) {
    const size_t nw = 27ULL * l.cin * l.cout;
    UK(cudaMemcpy(host + o, l.W, nw * sizeof(float), cudaMemcpyDeviceToHost));
    UK(cudaMemcpy(host + o + nw, l.b, l.cout * sizeof(float), cudaMemcpyDeviceToHost));
    o += nw + l.cout;
  }
  return APHID_UNET_OK;
}

int aphid_unet_set_params(aphid_unet *n, const float *host) {
  if (!n || !host) return set_err(APHID_UNET_ERR_BADARG, "unet_set_params: null");
  size_t o = 0;
  for (auto &l : n->L) {
    const size_t nw = 27ULL * l.cin * l.cout;
    UK(cudaMemcpy(l.W, host + o, nw * sizeof(float), cudaMemcpyHostToDevice));
    UK(cudaMemcpy(l.b, host + o + nw, l.cout * sizeof(float), cudaMemcpyHostToDevice));
    if (n->train) {  // a new starting point: the optimiser forgets its moments
      UK(cudaMemset(l.mW, 0, nw * sizeof(float)));
      UK(cudaMemset(l.vW, 0, nw * sizeof(float)));
      UK(cudaMemset(l.mb, 0, l.cout * sizeof(float)));
      UK(cudaMemset(l.vb, 0, l.cout * sizeof(float)));
    }
    o += nw + l.cout;
  }
  n->step = 0;
  UR(cast_weights(n, 0));
  UK(cudaDeviceSynchronize());
  return APHID_UNET_OK;
}

int aphid_unet_forward(aphid_unet *n, const float *x, float *y, void *stream) {
  if (!n || !x || !y) return set_err(APHID_UNET_ERR_BADARG, "unet_forward: null");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  UR(forward(n, x, st));
  k_unpack_out<<<nblk((long long)n->X * n->Y * n->Z * 8), kT, 0, st>>>(n->y, n->X, n->Y, n->Z, n->vol[0], y);
  UK(cudaGetLastError());
  return check_err(n, st);
}

int aphid_unet_train_step(aphid_unet *n, const float *x, const float *target, const float *weight, float lr,
                          int update, double *loss, void *stream) {
  if (!n || !x || !target) return set_err(APHID_UNET_ERR_BADARG, "unet_train_step: null");
  if (!n->train) return set_err(APHID_UNET_ERR_BADARG, "unet_train_step: created without training buffers");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  UR(forward(n, x, st));
  UK(cudaMemsetAsync(n->sums, 0, 2 * sizeof(double), st));
  k_loss_sums<<<nblk((long long)n->X * n->Y * n->Z), kT, 0, st>>>(n->y, target, weight, n->X, n->Y, n->Z, n->vol[0],
                                                                  n->sums);
  k_loss_grad<<<nblk(n->vol[0].Vp * 16), kT, 0, st>>>(n->y, target, weight, n->X, n->Y, n->Z, n->vol[0], n->sums,
                                                      n->gy);
  UK(cudaGetLastError());
  UR(backward(n, st));
  if (update) {
    n->step++;
    const float c1 = 1.f / (1.f - std::pow(0.9f, (float)n->step)), c2 = 1.f / (1.f - std::pow(0.999f, (float)n->step));
    for (auto &l : n->L)
      k_adam<<<nblk(27LL * l.cin * l.cout + l.cout), kT, 0, st>>>(l.W, l.mW, l.vW, l.gWT, l.cin, l.cg, l.cout, l.cn, l.b,
                                                                   l.mb, l.vb, l.gb, lr, c1, c2);
    UK(cudaGetLastError());
    UR(cast_weights(n, st));
  }
  double s[2] = {0, 0};
  UK(cudaMemcpyAsync(s, n->sums, sizeof(s), cudaMemcpyDeviceToHost, st));
  UR(check_err(n, st));
  if (loss) *loss = s[1] / std::max(s[0], 1e-30);
  return APHID_UNET_OK;
}

int aphid_unet_get_grads(aphid_unet *n, float *host) {
  if (!n || !host || !n->train) return set_err(APHID_UNET_ERR_BADARG, "unet_get_grads: no training buffers");
  size_t o = 0;
  float *tmp = nullptr;
  size_t maxn = 0;
  for (auto &l : n->L) maxn = std::max(maxn, (size_t)l.nparam());
  UK(cudaMalloc(&tmp, maxn * sizeof(float)));
  for (auto &l : n->L) {
    k_grad_out<<<nblk(l.nparam()), kT>>>(l.gWT, l.gb, l.cin, l.cg, l.cout, l.cn, tmp);
    if (cudaMemcpy(host + o, tmp, l.nparam() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaFree(tmp);
      return set_err(APHID_UNET_ERR_CUDA, "unet_get_grads: copy");
    }
    o += l.nparam();
  }
  cudaFree(tmp);
  return APHID_UNET_OK;
}


int aphid_unet_gemm_bf16(const void *A, int lda, const void *B, int ldb, void *C, int ldc, const float *bias, int M,
                         int N, int K, int out, int splitk, void *stream, int *err_flag) {
  return gemm_bf16(static_cast<const __nv_bfloat16 *>(A), lda, static_cast<const __nv_bfloat16 *>(B), ldb, C, ldc,
                   bias, M, N, K, out, splitk, static_cast<cudaStream_t>(stream), err_flag);
}

}  // extern "C"
