// tc_gemm.cuh -- Schur updates of the mixed-precision form on 5th-generation
// tensor cores (tcgen05, sm_100a).
//
// C -= A * B for FP32 column-major operands (the trailing and Schur updates
// F22 -= L21 * U12 of src/multifrontal.jl:267-268 when the fronts are held
// in FP32).  Each operand element is split into two TF32 parts,
// x = hi + lo with hi = tf32(x) and lo = tf32(x - hi), and the product is
// accumulated in FP32 as A_hi B_hi + A_hi B_lo + A_lo B_hi, which keeps
// about 21 bits of each product (the dropped A_lo B_lo term is below FP32
// rounding of the accumulation).
//
// One CTA computes a 128 x 128 tile: the operands are converted and staged
// by all 128 threads into shared memory in the K-major 128-byte-swizzled
// layout (two stages), one elected thread issues tcgen05.mma (M=128, N=128,
// K=8, kind::tf32) with the accumulator in tensor memory and commits each
// stage to an mbarrier, and the four warps read their 32 accumulator lanes
// back with tcgen05.ld for the C -= acc epilogue.  Every mbarrier wait is
// bounded: on expiry the kernel records the failure in flags[1], frees its
// tensor memory and returns.
#pragma once

#include "common.cuh"

namespace mfgpu {

constexpr int kTcBM = 128, kTcBN = 128, kTcBK = 32;   // tile; BK = one 128-byte swizzle row of TF32
constexpr int kTcThreads = 128;
constexpr int kTcStages = 2;
constexpr int kTcOperandBytes = kTcBM * kTcBK * 4;    // 16 KB per operand part
constexpr int kTcStageBytes = 4 * kTcOperandBytes;    // A_hi, A_lo, B_hi, B_lo
constexpr size_t kTcSmem = (size_t)kTcStages * kTcStageBytes + 1024;   // + alignment slack
constexpr uint64_t kTcWaitNs = 4000000000ull;        // 4 s bound on every mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Byte offset of element (row, k) (k < 32) in a K-major, 128-byte-swizzled
// tile of 4-byte elements: 128-byte rows, 8-row groups 1024 bytes apart, the
// 16-byte chunk index XOR-ed with row % 8.
__device__ __forceinline__ uint32_t sw128_offset(int row, int k) {
  const int chunk = (k >> 2) ^ (row & 7);
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + chunk * 16 + (k & 3) * 4);
}

// UMMA shared-memory descriptor: K-major, SWIZZLE_128B, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D f32, A/B tf32, both K-major, N = 128, M = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcBN >> 3) << 17) |
                              ((uint32_t)(kTcBM >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for phase `parity` of an mbarrier: non-blocking polls until
// the phase completes (true) or kTcWaitNs of wall time pass (false).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const uint64_t start = global_ns();
  for (uint32_t i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255) == 255 && global_ns() - start > kTcWaitNs) return false;
  }
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Stage one K block (kTcBK wide) of the A tile (rows m0.., column-major lda)
// and the B tile (columns n0.., column-major ldb) as TF32 hi/lo parts.
__device__ __forceinline__ void tc_stage(uint8_t* st, const float* __restrict__ A, const float* __restrict__ B, int M,
                                         int N, int K, int lda, int ldb, int m0, int n0, int k0) {
  uint8_t* ahi = st;
  uint8_t* alo = st + kTcOperandBytes;
  uint8_t* bhi = st + 2 * kTcOperandBytes;
  uint8_t* blo = st + 3 * kTcOperandBytes;
  const int t = threadIdx.x;
  // A: thread t owns row m0+t; K is strided in memory, so 32 loads per row
#pragma unroll 8
  for (int k = 0; k < kTcBK; ++k) {
    const int m = m0 + t, kk = k0 + k;
    const float v = (m < M && kk < K) ? A[(int64_t)m + (int64_t)kk * lda] : 0.0f;
    const float h = tf32_hi(v);
    const uint32_t off = sw128_offset(t, k);
    *reinterpret_cast<float*>(ahi + off) = h;
    *reinterpret_cast<float*>(alo + off) = tf32_hi(v - h);
  }
  // B: column n is contiguous along K; thread t covers k = t % 32 of 32 columns at a time
  const int kl = t & 31, cg = t >> 5;
#pragma unroll 8
  for (int j = 0; j < kTcBN / 4; ++j) {
    const int n = cg + 4 * j;
    const int nn = n0 + n, kk = k0 + kl;
    const float v = (nn < N && kk < K) ? B[(int64_t)kk + (int64_t)nn * ldb] : 0.0f;
    const float h = tf32_hi(v);
    const uint32_t off = sw128_offset(n, kl);
    *reinterpret_cast<float*>(bhi + off) = h;
    *reinterpret_cast<float*>(blo + off) = tf32_hi(v - h);
  }
}

// Batched C -= A * B over GemmTasks whose tiles_m / tiles_n use 128 x 128.
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc(const GemmTask* __restrict__ tasks, int ntasks,
                                                           const float* __restrict__ pa, const float* __restrict__ pb,
                                                           float* __restrict__ pc, int* __restrict__ flags) {
  extern __shared__ __align__(16) uint8_t tc_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t bars[kTcStages + 1];
  __shared__ uint32_t tmem_slot;
  __shared__ int failed;

  const int t = threadIdx.x, warp = warp_id(), lane = lane_id();
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile_base <= (int64_t)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GemmTask tk = tasks[lo];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * kTcBM;
  const int n0 = (int)(local / tk.tiles_m) * kTcBN;
  const float* A = pa + tk.a;
  const float* B = pb + tk.b;
  float* C = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k;

  if (t == 0) {
    for (int s = 0; s <= kTcStages; ++s) mbar_init(&bars[s], 1);
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kTcBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  const int nk = (K + kTcBK - 1) / kTcBK;
  for (int kb = 0; kb < nk; ++kb) {
    const int st = kb % kTcStages;
    uint8_t* sbuf = smem + st * kTcStageBytes;
    if (kb >= kTcStages) {
      // stage reuse: thread 0 waits for the MMAs that read it, the block follows
      if (t == 0 && !mbar_wait(&bars[st], (uint32_t)((kb / kTcStages - 1) & 1))) failed = 1;
      __syncthreads();
      if (failed) break;
    }
    tc_stage(sbuf, A, B, M, N, K, tk.lda, tk.ldb, m0, n0, kb * kTcBK);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ahi = smem_u32(sbuf), alo = ahi + kTcOperandBytes;
      const uint32_t bhi = ahi + 2 * kTcOperandBytes, blo = ahi + 3 * kTcOperandBytes;
#pragma unroll
      for (int ks = 0; ks < kTcBK / 8; ++ks) {     // K = 8 per instruction: 32 bytes along the row
        const uint32_t ko = ks * 32;
        tc_mma_tf32(tmem, umma_desc_sw128(ahi + ko), umma_desc_sw128(bhi + ko), (kb > 0 || ks > 0) ? 1u : 0u);
        tc_mma_tf32(tmem, umma_desc_sw128(ahi + ko), umma_desc_sw128(blo + ko), 1u);
        tc_mma_tf32(tmem, umma_desc_sw128(alo + ko), umma_desc_sw128(bhi + ko), 1u);
      }
      tc_commit(&bars[st]);
    }
  }
  __syncthreads();
  if (t == 0) {
    // completes once every MMA issued above is done; also drains them after a
    // failed stage wait, before the tensor memory is freed
    tc_commit(&bars[kTcStages]);
    if (!mbar_wait(&bars[kTcStages], 0u)) failed = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!failed && nk > 0) {
    // epilogue: warp w owns accumulator lanes (rows) 32w..32w+31
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < kTcBN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int col = n0 + c0 + j;
          if (col < N) C[(int64_t)row + (int64_t)col * tk.ldc] -= __uint_as_float(v[j]);
        }
      }
    }
  } else if (failed && t == 0) {
    atomicOr(flags + 1, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcBN));
}

}  // namespace mfgpu
