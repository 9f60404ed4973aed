// unet_gemm.cuh -- BF16 GEMM on the sm_100a tensor cores (tcgen05), the
// contraction under every convolution of the initial-guess network.
//
//   C[M x N] (op)= A[M x K] B[N x K]^T      A, B: BF16, K contiguous (K-major)
//                                           accumulation: FP32 in tensor memory
//
// One CTA of 128 threads computes a 128 x BN tile (k_gemm_tma below: TMA
// producer, single-thread MMA issuer, deep shared-memory ring).  Every wait
// is bounded: a wait that gives up sets an error flag, and the kernel still
// frees its tensor memory before it returns.
//
// Requirements (checked by the host): M % 128 == 0, N % BN == 0,
// K % 64 == 0, lda, ldb multiples of 8 elements, 16-byte aligned bases.
#pragma once
#include <cuda.h>
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
// ------------------------------------------------------------------------
// k_gemm_tma: the contraction fed by the tensor-memory accelerator through
// a deep shared-memory ring.  (A first version copied each 64-wide K block
// with cp.async by all threads behind a block-wide barrier; the tensor cores
// idled through every copy, under 1% of their time busy.)  Here:
//   warp 0, one lane: producer -- for each K block, waits for its ring slot
//     to be released, then issues two TMA tile loads (A: 128 x 64, B: BN x
//     64, BF16, 128-byte swizzle) that complete on the slot's "full"
//     mbarrier;
//   warp 1, one lane: MMA issuer -- waits for "full", issues four
//     tcgen05.mma (K = 16 each) on the swizzled tiles and commits them to
//     the slot's "empty" mbarrier, which releases the slot to the producer;
//     after the last block it commits once more to "done";
//   all four warps: epilogue -- wait for "done", read the accumulator from
//   tensor memory (warp w: lanes 32w..32w+31) and apply the output
//   operation, with 16-byte stores where the output rows allow them.
// Shared-memory tiles use the canonical K-major 128-byte-swizzle layout
// (8-row, 1024-byte atoms; the K = 16 slices of a block start 32 bytes
// apart inside each 128-byte row), which is what a TMA box with a 128-byte
// inner extent and CU_TENSOR_MAP_SWIZZLE_128B writes.  No multicast: every
// load is this CTA's own.  Every wait is bounded and reports through err.
template <int BN>
struct TmaShm {
  static constexpr uint32_t a_bytes = kBM * kBK * 2, b_bytes = BN * kBK * 2;
  static constexpr uint32_t stage = a_bytes + b_bytes;
  static constexpr int stages = (int)((196u * 1024u) / stage) < 8 ? (int)((196u * 1024u) / stage) : 8;
  static constexpr size_t bytes = 1024 + (size_t)stages * stage + 256;  // alignment slack, ring, barriers
};

// shared-memory descriptor of a K-major tile in the 128-byte-swizzle layout:
// start address, LBO 16 bytes (unused for swizzled K-major), SBO 1024 bytes
// (between 8-row atoms), descriptor version 1, layout type 2 (128B swizzle)
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
__device__ __forceinline__ void g_mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void g_tma_load2(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          dst),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

template <int BN, int OUT>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_tma(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, void *C, int ldc,
               const float *__restrict__ bias, int K, int kchunk, int vec_out, int *err) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N tile");
  using SH = TmaShm<BN>;
  constexpr int S = SH::stages;
  static_assert(S >= 2, "ring");
  constexpr uint32_t kCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  extern __shared__ __align__(1024) unsigned char gs_raw[];
  // the ring starts on a 1024-byte boundary (the swizzle atom)
  unsigned char *gs = gs_raw + ((1024u - (gsm(gs_raw) & 1023u)) & 1023u);
  uint64_t *full = reinterpret_cast<uint64_t *>(gs + S * SH::stage);
  uint64_t *empty = full + S;
  uint64_t *done = empty + S;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int kb0 = blockIdx.z * kchunk, kb1 = min(K, kb0 + kchunk);
  const int nkb = (kb1 - kb0) / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(gsm(tslot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 32) {
    for (int q = 0; q < S; q++) {
      g_mbar_init(gsm(&full[q]));
      g_mbar_init(gsm(&empty[q]));
    }
    g_mbar_init(gsm(done));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  bool ok = true;

  if (warp == 0 && lane == 0 && nkb > 0) {
    // producer
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % S;
      if (kb >= S) ok = g_mbar_wait(gsm(&empty[s]), (uint32_t)((kb / S - 1) & 1)) && ok;
      const uint32_t a = gsm(gs + s * SH::stage), fb = gsm(&full[s]);
      g_mbar_expect(fb, SH::stage);
      const int k = kb0 + kb * kBK;
      g_tma_load2(a, &mapA, k, m0, fb);
      g_tma_load2(a + SH::a_bytes, &mapB, k, n0, fb);
    }
  } else if (warp == 1 && lane == 0 && nkb > 0) {
    // MMA issuer
    constexpr uint32_t idesc = idesc_bf16(kBM, BN);
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % S;
      ok = g_mbar_wait(gsm(&full[s]), (uint32_t)((kb / S) & 1)) && ok;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a = gsm(gs + s * SH::stage), b = a + SH::a_bytes;
#pragma unroll
      for (int kk = 0; kk < kBK / 16; kk++) {
        const uint64_t da = smem_desc_sw128(a + 32u * kk), db = smem_desc_sw128(b + 32u * kk);
        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       gsm(&empty[s]))
                   : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(gsm(done))
                 : "memory");
  }
  __syncwarp();
  if (nkb > 0) ok = g_mbar_wait(gsm(done), 0u) && ok;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok && err) atomicExch(err, 1);

  // epilogue: warp w holds rows 32w .. 32w+31 (tensor-memory lanes)
  const int row = m0 + warp * 32 + lane;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  if (OUT != OUT_F32_ATOMIC && BN >= 32 && vec_out) {
    // wide rows: each warp turns its 32 x 32 blocks around in shared memory
    // (the ring is free now) so that consecutive lanes store consecutive
    // 16-byte pieces of one row, instead of each lane writing its own row
    float *stg = reinterpret_cast<float *>(gs) + warp * (32 * 36);
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
#pragma unroll
      for (int h = 0; h < 32; h += 8) {
        uint32_t v[8];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
            : "r"(lane_base + (uint32_t)(c0 + h)));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        float x[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          x[q] = nkb == 0 ? 0.f : __uint_as_float(v[q]);
          if (bias) x[q] += __ldg(bias + n0 + c0 + h + q);
          if (OUT == OUT_BF16_RELU) x[q] = fmaxf(x[q], 0.f);
        }
        float4 *d = reinterpret_cast<float4 *>(stg + lane * 36 + h);
        d[0] = make_float4(x[0], x[1], x[2], x[3]);
        d[1] = make_float4(x[4], x[5], x[6], x[7]);
      }
      __syncwarp();
      if (OUT == OUT_F32) {  // 8 lanes per row, 4 rows per step
#pragma unroll
        for (int rr = 0; rr < 32; rr += 4) {
          const int r = rr + (lane >> 3), cq = (lane & 7) * 4;
          const float4 val = *reinterpret_cast<const float4 *>(stg + r * 36 + cq);
          *reinterpret_cast<float4 *>(reinterpret_cast<float *>(C) + (size_t)(m0 + warp * 32 + r) * ldc + n0 + c0 +
                                      cq) = val;
        }
      } else {  // BF16: 4 lanes per row, 8 rows per step
#pragma unroll
        for (int rr = 0; rr < 32; rr += 8) {
          const int r = rr + (lane >> 2), cq = (lane & 3) * 8;
          const float4 a = *reinterpret_cast<const float4 *>(stg + r * 36 + cq);
          const float4 b = *reinterpret_cast<const float4 *>(stg + r * 36 + cq + 4);
          uint4 u;
          u.x = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.x)) |
                ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.y)) << 16);
          u.y = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.z)) |
                ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.w)) << 16);
          u.z = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b.x)) |
                ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b.y)) << 16);
          u.w = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b.z)) |
                ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b.w)) << 16);
          *reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(C) + (size_t)(m0 + warp * 32 + r) * ldc + n0 +
                                     c0 + cq) = u;
        }
      }
      __syncwarp();
    }
  } else {
#pragma unroll 1
  for (int c0 = 0; c0 < BN; c0 += 8) {
    uint32_t v[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
        : "r"(lane_base + (uint32_t)c0));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    float x[8];
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = nkb == 0 ? 0.f : __uint_as_float(v[q]);
    const int n = n0 + c0;
    if (OUT == OUT_F32_ATOMIC) {
      float *cr = reinterpret_cast<float *>(C) + (size_t)row * ldc + n;
#pragma unroll
      for (int q = 0; q < 8; q++) atomicAdd(cr + q, x[q]);
      continue;
    }
    if (bias) {
#pragma unroll
      for (int q = 0; q < 8; q++) x[q] += __ldg(bias + n + q);
    }
    if (OUT == OUT_BF16_RELU) {
#pragma unroll
      for (int q = 0; q < 8; q++) x[q] = fmaxf(x[q], 0.f);
    }
    if (OUT == OUT_F32) {
      float *cr = reinterpret_cast<float *>(C) + (size_t)row * ldc + n;
      if (vec_out) {
        reinterpret_cast<float4 *>(cr)[0] = make_float4(x[0], x[1], x[2], x[3]);
        reinterpret_cast<float4 *>(cr)[1] = make_float4(x[4], x[5], x[6], x[7]);
      } else {
#pragma unroll
        for (int q = 0; q < 8; q++) cr[q] = x[q];
      }
    } else {
      __nv_bfloat16 *cr = reinterpret_cast<__nv_bfloat16 *>(C) + (size_t)row * ldc + n;
      if (vec_out) {
        uint4 u;
        u.x = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[0])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[1])) << 16);
        u.y = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[2])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[3])) << 16);
        u.z = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[4])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[5])) << 16);
        u.w = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[6])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[7])) << 16);
        *reinterpret_cast<uint4 *>(cr) = u;
      } else {
#pragma unroll
        for (int q = 0; q < 8; q++) cr[q] = __float2bfloat16_rn(x[q]);
      }
    }
  }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
}

}  // namespace unet
}  // namespace aphid
