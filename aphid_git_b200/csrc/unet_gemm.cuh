// unet_gemm.cuh -- BF16 GEMM on the sm_100a tensor cores (tcgen05), the
// contraction under every convolution of the initial-guess network.
//
//   C[M x N] (op)= A[M x K] B[N x K]^T      A, B: BF16, K contiguous (K-major)
//                                           accumulation: FP32 in tensor memory
//
// One CTA of 128 threads computes a 128 x BN tile.  K is consumed in blocks
// of 64: all threads copy the A and B blocks into shared memory (cp.async,
// two buffers) in the canonical K-major, unswizzled core-matrix layout
// (8 rows x 16 bytes per core matrix); one thread issues four
// tcgen05.mma.kind::f16 (K = 16 each) per block and commits them to an
// mbarrier, whose completion frees the buffer for the block after next.
// The accumulator lives in tensor memory (lane = row, column = n); the
// epilogue reads it with tcgen05.ld (each warp its 32 lanes) and applies one
// of the output operations below.  Every wait is bounded: a wait that gives
// up sets an error flag, and the kernel still drains its own copies and
// frees its tensor memory before it returns.
//
// Requirements (checked by the host): M % 128 == 0, N % BN == 0,
// K % 64 == 0, lda, ldb multiples of 8 elements, 16-byte aligned bases.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace aphid {
namespace unet {

constexpr int kGemmThreads = 128, kBM = 128, kBK = 64;
constexpr int kGemmWait = 1 << 22;  // polls of an mbarrier before giving up

enum GemmOut {
  OUT_F32 = 0,        // C = acc (+ bias[n])                 (float)
  OUT_BF16_RELU = 1,  // C = relu(acc + bias[n])             (bf16)
  OUT_BF16 = 2,       // C = acc + bias[n]                   (bf16)
  OUT_F32_ATOMIC = 3  // C += acc, atomically (split-K)      (float)
};

__device__ __forceinline__ uint32_t gsm(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, no swizzle (layout type 0):
// start address, LBO (between the two K halves of one MMA), SBO (between
// 8-row groups), descriptor version 1, all in 16-byte units
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor of tcgen05.mma.kind::f16: FP32 accumulator, BF16 A
// and B, both K-major, shape M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void g_mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool g_mbar_wait(uint32_t bar, uint32_t phase) {
  for (int t = 0; t < kGemmWait; t++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void cp16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A: 128 x 64 block, B: BN x 64 block; element (r, k) at
// (k / 8) * (rows * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
template <int BN>
struct GemmShm {
  static constexpr uint32_t a_bytes = kBM * kBK * 2, b_bytes = BN * kBK * 2;
  static constexpr uint32_t stage = a_bytes + b_bytes;
  static constexpr size_t bytes = 2 * (size_t)stage + 64;  // + mbarriers, tmem address
};

template <int BN, int OUT>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_bf16(const __nv_bfloat16 *__restrict__ A, int lda, const __nv_bfloat16 *__restrict__ B, int ldb,
                void *C, int ldc, const float *__restrict__ bias, int K, int kchunk, int *err) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N tile");
  using SH = GemmShm<BN>;
  constexpr uint32_t kCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  extern __shared__ __align__(128) unsigned char gs[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(gs + 2 * SH::stage);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(gs + 2 * SH::stage + 16);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  // split-K: this CTA's range of K
  const int kb0 = blockIdx.z * kchunk, kb1 = min(K, kb0 + kchunk);
  const int nkb = (kb1 - kb0) / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(gsm(tslot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    g_mbar_init(gsm(&bars[0]));
    g_mbar_init(gsm(&bars[1]));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  auto load = [&](int s, int kb) {  // block kb into buffer s
    unsigned char *base = gs + s * SH::stage;
    const int k = kb0 + kb * kBK;
    for (int c = tid; c < kBM * 8; c += kGemmThreads) {
      const int r = c >> 3, kc = c & 7;
      cp16(gsm(base + kc * (kBM * 16) + (r >> 3) * 128 + (r & 7) * 16), A + (size_t)(m0 + r) * lda + k + kc * 8);
    }
    for (int c = tid; c < BN * 8; c += kGemmThreads) {
      const int r = c >> 3, kc = c & 7;
      cp16(gsm(base + SH::a_bytes + kc * (BN * 16) + (r >> 3) * 128 + (r & 7) * 16),
           B + (size_t)(n0 + r) * ldb + k + kc * 8);
    }
    cp_commit();
  };

  uint32_t phase[2] = {0, 0};
  bool ok = true;
  constexpr uint32_t idesc = idesc_bf16(kBM, BN);
  if (nkb > 0) load(0, 0);
  for (int kb = 0; kb < nkb; kb++) {
    const int s = kb & 1;
    if (kb + 1 < nkb) {
      if (kb >= 1) {  // buffer s^1 was read by the MMAs of block kb-1
        ok = g_mbar_wait(gsm(&bars[s ^ 1]), phase[s ^ 1]) && ok;
        phase[s ^ 1] ^= 1u;
      }
      load(s ^ 1, kb + 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // cp.async data -> tensor-core reads
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a = gsm(gs + s * SH::stage), b = a + SH::a_bytes;
#pragma unroll
      for (int kk = 0; kk < kBK / 16; kk++) {
        // K = 16: the two 8-element halves are core matrices 2kk and 2kk+1
        const uint64_t da = smem_desc(a + 2 * kk * (kBM * 16), kBM * 16, 128);
        const uint64_t db = smem_desc(b + 2 * kk * (BN * 16), BN * 16, 128);
        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       gsm(&bars[s]))
                   : "memory");
    }
    __syncthreads();
  }
  // the last commit covers every MMA issued before it
  if (nkb > 0) {
    const int s = (nkb - 1) & 1;
    ok = g_mbar_wait(gsm(&bars[s]), phase[s]) && ok;
    if (nkb >= 2) {  // the other buffer's last commit (block nkb-2) is complete too; consume its phase
      ok = g_mbar_wait(gsm(&bars[s ^ 1]), phase[s ^ 1]) && ok;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok && err) atomicExch(err, 1);

  // epilogue: warp w holds rows 32w .. 32w+31 (tensor-memory lanes)
  const int row = m0 + warp * 32 + (tid & 31);
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
  for (int c0 = 0; c0 < BN; c0 += 8) {
    uint32_t v[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
        : "r"(lane_base + (uint32_t)c0));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    if (nkb == 0) {
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] = 0u;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int n = n0 + c0 + q;
      float x = __uint_as_float(v[q]);
      if (OUT == OUT_F32_ATOMIC) {
        atomicAdd(reinterpret_cast<float *>(C) + (size_t)row * ldc + n, x);
        continue;
      }
      if (bias) x += __ldg(bias + n);
      if (OUT == OUT_BF16_RELU) x = fmaxf(x, 0.f);
      if (OUT == OUT_F32)
        reinterpret_cast<float *>(C)[(size_t)row * ldc + n] = x;
      else
        reinterpret_cast<__nv_bfloat16 *>(C)[(size_t)row * ldc + n] = __float2bfloat16_rn(x);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
}

}  // namespace unet
}  // namespace aphid
