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
// One CTA computes a 128 x BN tile (BN = 64 or 128) with warp
// specialisation: warps 0-3 load FP32 operands from global memory, split
// them and store the parts into a ring of STAGES shared-memory slots in the
// K-major 128-byte-swizzled layout (32 K values per slot), then arrive on the
// slot's "full" mbarrier; one thread of warp 4 waits for a full slot, issues
// the 12 tcgen05.mma (M=128, N=BN, K=8, kind::tf32) of that slot into the
// tensor-memory accumulator and commits them to the slot's "empty" mbarrier,
// which the producers wait on before they refill it.  A final commit marks
// the accumulator complete; warps 0-3 then read their 32 accumulator lanes
// with tcgen05.ld for the C -= acc epilogue.  There is no block-wide barrier
// inside the K loop, and every mbarrier wait is bounded by the handle's wait
// limit (wait_ns, 4 s unless set): on expiry the kernel records the failure
// in flags[1], waits (bounded by kTcDrainNs) for the MMAs it issued to
// complete, leaves C unwritten, frees its tensor memory and returns.
#pragma once

#include "common.cuh"

namespace mfgpu {

constexpr uint64_t kTcWaitNs = 4000000000ull;        // default bound on every mbarrier wait (4 s)
constexpr uint64_t kTcDrainNs = 4000000000ull;       // bound on the wait for issued MMAs after a failure
constexpr int kTcProducers = 128;                    // warps 0-3: operand staging, then the epilogue
constexpr int kTcThreads = kTcProducers + 32;        // warp 4: the MMA issuer

// Tile shapes: BM = 128 accumulator lanes, BN columns, BK = 32 (one 128-byte
// swizzle row of TF32), STAGES ring slots of {A_hi, A_lo, B_hi, B_lo}.
template <int BN, int STAGES>
struct TcCfg {
  static constexpr int BM = 128, BK = 32;
  static constexpr int kABytes = BM * BK * 4;
  static constexpr int kBBytes = BN * BK * 4;
  static constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;
  static constexpr size_t kSmem = (size_t)STAGES * kStageBytes + 1024;   // + alignment slack
  static constexpr int kTmemCols = BN;                                   // power of two >= 32
  // instruction descriptor: D f32, A/B tf32, both K-major, N = BN, M = 128
  static constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                     ((uint32_t)(BM >> 4) << 24);
  static_assert(BN == 64 || BN == 128, "BN must be 64 or 128");
};

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

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for phase `parity` of an mbarrier: non-blocking polls until
// the phase completes (true) or limit_ns of wall time pass (false).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
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
    if ((i & 31) == 31 && global_ns() - start > limit_ns) return false;
  }
}

// Epilogue threads: wait for the final commit (the accumulator complete).
// When that wait runs out, the failure is recorded and the thread keeps
// waiting, bounded by kTcDrainNs, for the issued MMAs to complete, so that
// the tensor memory is idle before it is freed.
__device__ __forceinline__ void tc_wait_done(uint64_t* done, uint64_t wait_ns, volatile int* failed) {
  if (!mbar_wait(done, 0u, wait_ns)) {
    *failed = 1;
    mbar_wait(done, 0u, kTcDrainNs);
  }
}

// 32 consecutive accumulator columns of this warp's 32 lanes (32x32b.x32),
// complete on return.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
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
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, float a, float b, float c, float d) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

// Split four consecutive K values of one row into TF32 hi / lo parts and
// store them as one 16-byte chunk of each swizzled operand part.
__device__ __forceinline__ void tc_put4(uint32_t hi_base, uint32_t lo_base, int row, int chunk, const float* v) {
  float h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    h[i] = tf32_hi(v[i]);
    l[i] = tf32_hi(v[i] - h[i]);
  }
  const uint32_t off = sw128_offset(row, chunk * 4);
  st_shared_v4(hi_base + off, h[0], h[1], h[2], h[3]);
  st_shared_v4(lo_base + off, l[0], l[1], l[2], l[3]);
}

// Batched C -= A * B over GemmTasks whose tiles_m / tiles_n count
// 128 x BN tiles.  flags[1] is set when a bounded wait expired.
template <int BN, int STAGES>
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc(const GemmTask* __restrict__ tasks, int ntasks,
                                                        const float* __restrict__ pa, const float* __restrict__ pb,
                                                        float* pc, int* __restrict__ flags, uint64_t wait_ns) {
  using Cfg = TcCfg<BN, STAGES>;
  constexpr int BK = Cfg::BK;
  extern __shared__ __align__(16) uint8_t tc_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done, stall;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int failed;

  const int t = threadIdx.x, warp = warp_id(), lane = lane_id();
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile_base <= (int64_t)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GemmTask tk = tasks[lo];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * Cfg::BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const int M = tk.m, N = tk.n, K = tk.k;
  const int nk = (K + BK - 1) / BK;

  if (t == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], kTcProducers);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    mbar_init(&stall, 1);   // nothing arrives on it (test hook, flags[2])
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(Cfg::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t sbase = smem_u32(smem);

  if (warp < 4) {
    // ---- producers: global FP32 -> registers -> hi/lo TF32 swizzled stages
    const float* A = pa + tk.a;
    const float* B = pb + tk.b;
    const int row = m0 + t;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES, k0 = kb * BK;
      float va[BK];
#pragma unroll
      for (int k = 0; k < BK; ++k)
        va[k] = (row < M && k0 + k < K) ? A[(int64_t)row + (int64_t)(k0 + k) * tk.lda] : 0.0f;
      constexpr int kBPer = BN * (BK / 4) / kTcProducers;    // (column, chunk) pairs per thread
      float vb[kBPer][4];
#pragma unroll
      for (int i = 0; i < kBPer; ++i) {
        const int idx = t + i * kTcProducers, n = idx >> 3, c = idx & 7;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int kk = k0 + 4 * c + j;
          vb[i][j] = (n0 + n < N && kk < K) ? B[(int64_t)kk + (int64_t)(n0 + n) * tk.ldb] : 0.0f;
        }
      }
      if (kb >= STAGES && !mbar_wait(&empty[s], (uint32_t)((kb / STAGES - 1) & 1), wait_ns)) {
        failed = 1;
        break;
      }
      const uint32_t st = sbase + s * Cfg::kStageBytes;
#pragma unroll
      for (int c = 0; c < BK / 4; ++c) tc_put4(st, st + Cfg::kABytes, t, c, va + 4 * c);
#pragma unroll
      for (int i = 0; i < kBPer; ++i) {
        const int idx = t + i * kTcProducers;
        tc_put4(st + 2 * Cfg::kABytes, st + 2 * Cfg::kABytes + Cfg::kBBytes, idx >> 3, idx & 7, vb[i]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full[s]);
      if (failed) break;
    }
  } else if (lane == 0) {
    // ---- MMA issuer: 3 TF32 products per K step into the TMEM accumulator
    if (flags[2] && !mbar_wait(&stall, 0u, wait_ns)) failed = 1;   // test hook: a wait that runs out
    int kb = 0;
    for (; kb < nk && !failed; ++kb) {
      const int s = kb % STAGES;
      if (failed || !mbar_wait(&full[s], (uint32_t)((kb / STAGES) & 1), wait_ns)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ahi = sbase + s * Cfg::kStageBytes, alo = ahi + Cfg::kABytes;
      const uint32_t bhi = ahi + 2 * Cfg::kABytes, blo = bhi + Cfg::kBBytes;
#pragma unroll
      for (int ks = 0; ks < BK / 8; ++ks) {       // K = 8 per instruction: 32 bytes along the row
        const uint32_t ko = ks * 32;
        tc_mma_tf32(tmem, umma_desc_sw128(ahi + ko), umma_desc_sw128(bhi + ko), Cfg::kIdesc,
                    (kb > 0 || ks > 0) ? 1u : 0u);
        tc_mma_tf32(tmem, umma_desc_sw128(ahi + ko), umma_desc_sw128(blo + ko), Cfg::kIdesc, 1u);
        tc_mma_tf32(tmem, umma_desc_sw128(alo + ko), umma_desc_sw128(bhi + ko), Cfg::kIdesc, 1u);
      }
      tc_commit(&empty[s]);
    }
    // completes when every MMA issued above is done (also after a failure,
    // so that the tensor memory is idle before it is freed)
    tc_commit(&done);
  }

  // the accumulator is complete (or, after a failure, every issued MMA has
  // drained) before any thread goes on; `failed` is then block-uniform
  if (warp < 4) tc_wait_done(&done, wait_ns, &failed);
  __syncthreads();
  const bool ok = !failed;
  if (warp < 4) {
    // ---- epilogue: warp w reads accumulator lanes 32w..32w+31 (rows of the tile)
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      float* C = pc + tk.c;
      const int row = m0 + warp * 32 + lane;
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        if (nk == 0) {   // K = 0: the product is zero (C = D or C = 0)
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = 0u;
        } else {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }
        if (row < M) {
          const float* D = tk.mode == kGemmFrom ? pc + tk.d : C;
          const int ldD = tk.mode == kGemmFrom ? tk.ldd : tk.ldc;
          const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
          const float sgn = tk.mode == kGemmSet ? -1.0f : 1.0f;
          float cv[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            cv[j] = (ld && col < N) ? D[(int64_t)row + (int64_t)col * ldD] : 0.0f;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            if (col < N) C[(int64_t)row + (int64_t)col * tk.ldc] = cv[j] - sgn * __uint_as_float(v[j]);
          }
        }
      }
    } else if (t == 0) {
      atomicOr(flags + 1, 1);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kTmemCols));
}

// ---------------------------------------------------------------------------
// BF16x3 variant.  Each FP32 operand is split into three bf16 parts,
// x = b1 + b2 + b3 (b1 = bf16(x), b2 = bf16(x - b1), b3 = bf16(x - b1 - b2)),
// which represents x to about 2^-24 relative -- FP32's own precision -- and
// the product keeps the six terms b_i c_j with i + j <= 4 (a1 b1, a1 b2,
// a2 b1, a1 b3, a3 b1, a2 b2), accumulated in FP32 in tensor memory by
// tcgen05.mma kind::f16 (M = 128, N = BN, K = 16).  bf16 runs at twice the
// TF32 rate, so six bf16 products cost what three TF32 products cost, with
// FP32 accuracy instead of the 2^-21 of the two-part TF32 split.
//
// The staging warps (16 in the two-stage form, 8 in the short-K form) stage
// a 64-wide K block (one 128-byte swizzle row of bf16): thread t converts
// row t % 128 over K quarter (half) t / 128 of A, and two (four) 8-value
// chunks of B; the next warp issues the MMAs; all staging warps then read
// the accumulator back (warp w: lanes 32 (w % 4).., column group w / 4).
// Sixteen staging warps keep twice the loads and conversions in flight per
// SM (the staging, not the tensor pipe, limits the one-CTA-per-SM form); the
// short-K form keeps eight so that two CTAs fit an SM's registers.
//
// The tensor core's FP32 accumulation rounds every addition towards zero,
// so over a long K its error is a bias that grows with the number of
// accumulation steps, and FP64 iterative refinement converges more slowly
// against such factors than against CUDA-core FP32 ones.  The K blocks are
// therefore spread round-robin over kAccs accumulators in tensor memory (all
// 512 columns for BN = 128): each sees a quarter of the steps and a quarter
// of the running sum, and the epilogue adds the partial sums in FP32 with
// round-to-nearest.
template <int BN, int STAGES, int ACCS = 4>
struct BxCfg {
  static constexpr int BM = 128, BK = 64;
  static constexpr int kProducers = STAGES == 1 ? 256 : 512;   // staging threads
  static constexpr int kProdWarps = kProducers / 32;
  static constexpr int kThreads = kProducers + 32;              // + the MMA-issuing warp
  static constexpr int kAPer = BM * BK / kProducers;            // A values per staging thread (one row)
  static constexpr int kABytes = BM * BK * 2;     // one bf16 part of A
  static constexpr int kBBytes = BN * BK * 2;
  static constexpr int kStageBytes = 3 * kABytes + 3 * kBBytes;
  static constexpr size_t kSmem = (size_t)STAGES * kStageBytes + 1024;
  static constexpr int kAccs = ACCS;               // accumulators, K blocks round-robin
  static constexpr int kTmemCols = kAccs * BN;     // a power of two >= 32
  // D f32, A/B bf16, both K-major, N = BN, M = 128
  static constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                     ((uint32_t)(BM >> 4) << 24);
  static_assert(BN == 64 || BN == 128, "BN must be 64 or 128");
};

// Byte offset of element (row, k) (k < 64) in a K-major, 128-byte-swizzled
// tile of 2-byte elements.
__device__ __forceinline__ uint32_t sw128_offset_b16(int row, int k) {
  const int chunk = (k >> 3) ^ (row & 7);
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + chunk * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void tc_mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// Split eight consecutive K values into three bf16 parts (x = hi + mid + lo
// exactly for FP32 x, each part rounded to nearest), packed two per word.
__device__ __forceinline__ void bx_split8(const float* v, uint32_t (&w1)[4], uint32_t (&w2)[4], uint32_t (&w3)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float x0 = v[2 * q], x1 = v[2 * q + 1];
    w1[q] = pack_bf16(x0, x1);
    const float h0 = __uint_as_float(w1[q] << 16), h1 = __uint_as_float(w1[q] & 0xFFFF0000u);
    const float r0 = x0 - h0, r1 = x1 - h1;
    w2[q] = pack_bf16(r0, r1);
    const float m0 = __uint_as_float(w2[q] << 16), m1 = __uint_as_float(w2[q] & 0xFFFF0000u);
    w3[q] = pack_bf16(r0 - m0, r1 - m1);
  }
}

// Split eight consecutive K values into three bf16 parts and store each part
// as one 16-byte chunk at byte offset `off` of its part buffer.
__device__ __forceinline__ void bx_put8(uint32_t p1, uint32_t p2, uint32_t p3, uint32_t off, const float* v) {
  uint32_t w1[4], w2[4], w3[4];
  bx_split8(v, w1, w2, w3);
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(p1 + off), "r"(w1[0]), "r"(w1[1]), "r"(w1[2]),
               "r"(w1[3]) : "memory");
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(p2 + off), "r"(w2[0]), "r"(w2[1]), "r"(w2[2]),
               "r"(w2[3]) : "memory");
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(p3 + off), "r"(w3[0]), "r"(w3[1]), "r"(w3[2]),
               "r"(w3[3]) : "memory");
}

// Batched C = f(C, A * B) (GemmTask::mode) over tasks whose tiles_m /
// tiles_n count 128 x BN tiles; flags[1] is set when a bounded wait expired.
// The short-K form (STAGES = 1, ACCS = 1: launches whose tasks all have
// K <= BK) holds one stage and one accumulator and stages one K block
// without a second register buffer, so two CTAs share an SM.
template <int BN, int STAGES, int ACCS = 4>
__global__ void __launch_bounds__(BxCfg<BN, STAGES, ACCS>::kThreads, STAGES == 1 ? 2 : 1)
    k_gemm_bx3(const GemmTask* __restrict__ tasks, int ntasks, const float* __restrict__ pa,
               const float* __restrict__ pb, float* pc, int* __restrict__ flags, uint64_t wait_ns) {
  using Cfg = BxCfg<BN, STAGES, ACCS>;
  constexpr int BK = Cfg::BK;
  extern __shared__ __align__(16) uint8_t bx_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)bx_smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done, stall;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int failed;

  const int t = threadIdx.x, warp = warp_id(), lane = lane_id();
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile_base <= (int64_t)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GemmTask tk = tasks[lo];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * Cfg::BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const int M = tk.m, N = tk.n, K = tk.k;
  const int nk = (K + BK - 1) / BK;

  if (t == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], Cfg::kProducers);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    mbar_init(&stall, 1);   // nothing arrives on it (test hook, flags[2])
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(Cfg::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t sbase = smem_u32(smem);

  constexpr int kAPer = Cfg::kAPer;
  if (warp < Cfg::kProdWarps) {
    const float* A = pa + tk.a;
    const float* B = pb + tk.b;
    const int arow = t & 127, ak = (t >> 7) * kAPer;
    const int row = m0 + arow;
    constexpr int kBPer = BN * (BK / 8) / Cfg::kProducers;   // (column, 8-chunk) pairs per thread
    // Software pipeline over K blocks: the global loads of block kb + 1 are
    // issued before block kb is split and stored, so their latency hides
    // behind that work and the wait for a free stage (two register buffers).
    auto load = [&](int kb, float (&va)[kAPer], float (&vb)[kBPer][8]) {
      const int k0 = kb * BK;
#pragma unroll
      for (int k = 0; k < kAPer; ++k) {
        const int kk = k0 + ak + k;
        va[k] = (row < M && kk < K) ? A[(int64_t)row + (int64_t)kk * tk.lda] : 0.0f;
      }
#pragma unroll
      for (int i = 0; i < kBPer; ++i) {
        const int idx = t + i * Cfg::kProducers, n = idx >> 3, c = idx & 7;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int kk = k0 + 8 * c + j;
          vb[i][j] = (n0 + n < N && kk < K) ? B[(int64_t)kk + (int64_t)(n0 + n) * tk.ldb] : 0.0f;
        }
      }
    };
    // wait for a free stage, split and store block kb, mark the stage full
    auto produce = [&](int kb, const float (&va)[kAPer], const float (&vb)[kBPer][8]) -> bool {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], (uint32_t)((kb / STAGES - 1) & 1), wait_ns)) {
        failed = 1;
        return false;
      }
      const uint32_t st = sbase + s * Cfg::kStageBytes;
#pragma unroll
      for (int c = 0; c < kAPer / 8; ++c)
        bx_put8(st, st + Cfg::kABytes, st + 2 * Cfg::kABytes, sw128_offset_b16(arow, ak + 8 * c), va + 8 * c);
      const uint32_t sb = st + 3 * Cfg::kABytes;
#pragma unroll
      for (int i = 0; i < kBPer; ++i) {
        const int idx = t + i * Cfg::kProducers;
        bx_put8(sb, sb + Cfg::kBBytes, sb + 2 * Cfg::kBBytes, sw128_offset_b16(idx >> 3, 8 * (idx & 7)), vb[i]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full[s]);
      return !failed;
    };
    if constexpr (STAGES == 1) {
      float va[kAPer], vb[kBPer][8];
      for (int kb = 0; kb < nk; ++kb) {
        load(kb, va, vb);
        if (!produce(kb, va, vb)) break;
      }
    } else {
      float va0[kAPer], vb0[kBPer][8], va1[kAPer], vb1[kBPer][8];
      if (nk > 0) load(0, va0, vb0);
      for (int kb = 0; kb < nk; kb += 2) {
        if (kb + 1 < nk) load(kb + 1, va1, vb1);
        if (!produce(kb, va0, vb0) || kb + 1 >= nk) break;
        if (kb + 2 < nk) load(kb + 2, va0, vb0);
        if (!produce(kb + 1, va1, vb1)) break;
      }
    }
  } else if (lane == 0) {
    if (flags[2] && !mbar_wait(&stall, 0u, wait_ns)) failed = 1;   // test hook: a wait that runs out
    for (int kb = 0; kb < nk && !failed; ++kb) {
      const int s = kb % STAGES;
      if (failed || !mbar_wait(&full[s], (uint32_t)((kb / STAGES) & 1), wait_ns)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a1 = sbase + s * Cfg::kStageBytes, a2 = a1 + Cfg::kABytes, a3 = a2 + Cfg::kABytes;
      const uint32_t b1 = a1 + 3 * Cfg::kABytes, b2 = b1 + Cfg::kBBytes, b3 = b2 + Cfg::kBBytes;
#pragma unroll
      for (int ks = 0; ks < BK / 16; ++ks) {      // K = 16 per instruction: 32 bytes along the row
        const uint32_t ko = ks * 32;
        // smallest terms first, into accumulator kb % kAccs
        const uint32_t acc = tmem + (uint32_t)((kb % Cfg::kAccs) * BN);
        tc_mma_bf16(acc, umma_desc_sw128(a2 + ko), umma_desc_sw128(b2 + ko), Cfg::kIdesc,
                    (kb >= Cfg::kAccs || ks > 0) ? 1u : 0u);
        tc_mma_bf16(acc, umma_desc_sw128(a3 + ko), umma_desc_sw128(b1 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a1 + ko), umma_desc_sw128(b3 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a2 + ko), umma_desc_sw128(b1 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a1 + ko), umma_desc_sw128(b2 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a1 + ko), umma_desc_sw128(b1 + ko), Cfg::kIdesc, 1u);
      }
      tc_commit(&empty[s]);
    }
    tc_commit(&done);
  }

  if (warp < Cfg::kProdWarps) tc_wait_done(&done, wait_ns, &failed);
  __syncthreads();
  const bool ok = !failed;
  if (warp < Cfg::kProdWarps) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      float* C = pc + tk.c;
      constexpr int kGroupCols = BN / (Cfg::kProdWarps / 4);   // columns per warp group
      const int q = warp & 3, grp = warp >> 2;
      const int row = m0 + q * 32 + lane;
      const float* D = tk.mode == kGemmFrom ? pc + tk.d : C;
      const int ldD = tk.mode == kGemmFrom ? tk.ldd : tk.ldc;
      const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
      const float sgn = tk.mode == kGemmSet ? -1.0f : 1.0f;
      const int nacc = nk < Cfg::kAccs ? nk : Cfg::kAccs;   // accumulators that K blocks reached
#pragma unroll 1
      for (int c0 = grp * kGroupCols; c0 < (grp + 1) * kGroupCols; c0 += 32) {
        uint32_t v[32];
        float acc[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = 0.0f;   // K = 0: the product is zero (C = D or C = 0)
        for (int b = 0; b < nacc; ++b) {
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + c0), v);
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[j] += __uint_as_float(v[j]);
        }
        if (row < M) {
          // eight columns at a time: their C (or D) values are all loaded
          // before any of them is stored
#pragma unroll
          for (int g = 0; g < 32; g += 8) {
            float cv[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int col = n0 + c0 + g + j;
              cv[j] = (ld && col < N) ? D[(int64_t)row + (int64_t)col * ldD] : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int col = n0 + c0 + g + j;
              if (col < N) C[(int64_t)row + (int64_t)col * tk.ldc] = cv[j] - sgn * acc[g + j];
            }
          }
        }
      }
    } else if (t == 0) {
      atomicOr(flags + 1, 1);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kTmemCols));
}

// ---------------------------------------------------------------------------
// Pre-split operands for the long-K updates of the FP32 fronts (the deferred
// Schur updates F22 -= L21 * U12 and the K = 256 block updates of the pivot
// blocks).  Those products are the largest of the factorization, and in
// k_gemm_bx3 every CTA of a tile row (column) splits the same A (B) tile into
// its bf16 parts again.  Here each 128 x 64 operand tile is split once, by
// k_split_planes, into three 16 KB parts laid out byte for byte as the MMA's
// shared-memory tiles (K-major, 128-byte swizzle); k_gemm_bx3p then moves
// each part into shared memory with one bulk copy (cp.async.bulk, completion
// counted on the stage's mbarrier) and issues the same six products per
// 16-wide K step into the same four round-robin accumulators, so C is
// bitwise what k_gemm_bx3 writes.
constexpr int kPlaneTile = (int)kPlaneTileBytes;   // bytes of one bf16 part of one 128 x 64 tile
constexpr int kBxpThreads = 512;           // producer lane (warp 0), MMA lane (warp 1), then 16 epilogue warps

// Split unit u of a launch's tasks: units unit_base .. of a task are its A
// tiles (row tile i, K block kb: i * kt + kb), then its B tiles (column tile
// j, K block kb).  Same split, tile mapping and zero fill as k_gemm_bx3's
// staging warps.
__global__ void __launch_bounds__(256) k_split_planes(const GemmTask* __restrict__ tasks,
                                                      const PlaneTask* __restrict__ pt, int ntasks,
                                                      const float* __restrict__ pa, const float* __restrict__ pb,
                                                      uint8_t* __restrict__ planes) {
  const int64_t u = blockIdx.x;
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pt[mid].unit_base <= u) lo = mid;
    else hi = mid - 1;
  }
  const GemmTask tk = tasks[lo];
  const PlaneTask p = pt[lo];
  const int64_t local = u - p.unit_base;
  const int64_t na = (int64_t)tk.tiles_m * p.kt;
  const int t = threadIdx.x;
  uint32_t w1[4], w2[4], w3[4];
  float v[8];
  if (local < na) {
    const int i = (int)(local / p.kt), kb = (int)(local % p.kt);
    uint8_t* dst = planes + p.a_off + (int64_t)(i * p.kt + kb) * 3 * kPlaneTile;
    const float* A = pa + tk.a;
    const int r = t & 127, row = i * 128 + r;
    for (int c = t >> 7; c < 8; c += 2) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int kk = kb * 64 + 8 * c + j;
        v[j] = (row < tk.m && kk < tk.k) ? A[(int64_t)row + (int64_t)kk * tk.lda] : 0.0f;
      }
      bx_split8(v, w1, w2, w3);
      const uint32_t off = sw128_offset_b16(r, 8 * c);
      *reinterpret_cast<uint4*>(dst + off) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
      *reinterpret_cast<uint4*>(dst + kPlaneTile + off) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
      *reinterpret_cast<uint4*>(dst + 2 * kPlaneTile + off) = make_uint4(w3[0], w3[1], w3[2], w3[3]);
    }
  } else {
    const int64_t lb = local - na;
    const int j = (int)(lb / p.kt), kb = (int)(lb % p.kt);
    uint8_t* dst = planes + p.b_off + (int64_t)(j * p.kt + kb) * 3 * kPlaneTile;
    const float* B = pb + tk.b;
    for (int q = 0; q < 4; ++q) {
      const int idx = t + q * 256, n = idx >> 3, c = idx & 7, col = j * 128 + n;
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const int kk = kb * 64 + 8 * c + jj;
        v[jj] = (col < tk.n && kk < tk.k) ? B[(int64_t)kk + (int64_t)col * tk.ldb] : 0.0f;
      }
      bx_split8(v, w1, w2, w3);
      const uint32_t off = sw128_offset_b16(n, 8 * c);
      *reinterpret_cast<uint4*>(dst + off) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
      *reinterpret_cast<uint4*>(dst + kPlaneTile + off) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
      *reinterpret_cast<uint4*>(dst + 2 * kPlaneTile + off) = make_uint4(w3[0], w3[1], w3[2], w3[3]);
    }
  }
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bulk copy (no tensor map, no multicast) of `bytes` from global memory to
// this CTA's shared memory, counted on mbarrier `bar`.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

template <int STAGES>
__global__ void __launch_bounds__(kBxpThreads, 1)
    k_gemm_bx3p(const GemmTask* __restrict__ tasks, const PlaneTask* __restrict__ pt, int ntasks,
                const uint8_t* __restrict__ planes, float* pc, int* __restrict__ flags, uint64_t wait_ns) {
  using Cfg = BxCfg<128, 2, 4>;   // tile shape, stage layout, instruction descriptor, accumulators
  constexpr int BN = 128;
  extern __shared__ __align__(16) uint8_t bxp_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)bxp_smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done, stall;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int failed;

  const int t = threadIdx.x, warp = warp_id(), lane = lane_id();
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile_base <= (int64_t)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GemmTask tk = tasks[lo];
  const PlaneTask pk = pt[lo];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int ti = (int)(local % tk.tiles_m), tj = (int)(local / tk.tiles_m);
  const int m0 = ti * Cfg::BM, n0 = tj * BN;
  const int M = tk.m, N = tk.n;
  const int nk = pk.kt;

  if (t == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    mbar_init(&stall, 1);   // nothing arrives on it (test hook, flags[2])
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(Cfg::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t sbase = smem_u32(smem);

  if (warp == 0 && lane == 0) {
    const uint8_t* a_src = planes + pk.a_off + (int64_t)ti * nk * 3 * kPlaneTile;
    const uint8_t* b_src = planes + pk.b_off + (int64_t)tj * nk * 3 * kPlaneTile;
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], (uint32_t)((kb / STAGES - 1) & 1), wait_ns)) {
        failed = 1;
        break;
      }
      if (failed) break;
      const uint32_t st = sbase + s * Cfg::kStageBytes;
      mbar_arrive_expect_tx(&full[s], 6 * kPlaneTile);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        bulk_g2s(st + q * Cfg::kABytes, a_src + (int64_t)(kb * 3 + q) * kPlaneTile, kPlaneTile, &full[s]);
        bulk_g2s(st + 3 * Cfg::kABytes + q * Cfg::kBBytes, b_src + (int64_t)(kb * 3 + q) * kPlaneTile, kPlaneTile,
                 &full[s]);
      }
      ++issued;
    }
    // copies in flight land before this CTA may end (a stage the MMA lane
    // did not consume after a wait ran out)
    for (int kb = issued > STAGES ? issued - STAGES : 0; kb < issued; ++kb)
      mbar_wait(&full[kb % STAGES], (uint32_t)((kb / STAGES) & 1), kTcDrainNs);
  } else if (warp == 1 && lane == 0) {
    if (flags[2] && !mbar_wait(&stall, 0u, wait_ns)) failed = 1;   // test hook: a wait that runs out
    for (int kb = 0; kb < nk && !failed; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full[s], (uint32_t)((kb / STAGES) & 1), wait_ns)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a1 = sbase + s * Cfg::kStageBytes, a2 = a1 + Cfg::kABytes, a3 = a2 + Cfg::kABytes;
      const uint32_t b1 = a1 + 3 * Cfg::kABytes, b2 = b1 + Cfg::kBBytes, b3 = b2 + Cfg::kBBytes;
#pragma unroll
      for (int ks = 0; ks < Cfg::BK / 16; ++ks) {
        const uint32_t ko = ks * 32;
        const uint32_t acc = tmem + (uint32_t)((kb % Cfg::kAccs) * BN);
        tc_mma_bf16(acc, umma_desc_sw128(a2 + ko), umma_desc_sw128(b2 + ko), Cfg::kIdesc,
                    (kb >= Cfg::kAccs || ks > 0) ? 1u : 0u);
        tc_mma_bf16(acc, umma_desc_sw128(a3 + ko), umma_desc_sw128(b1 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a1 + ko), umma_desc_sw128(b3 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a2 + ko), umma_desc_sw128(b1 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a1 + ko), umma_desc_sw128(b2 + ko), Cfg::kIdesc, 1u);
        tc_mma_bf16(acc, umma_desc_sw128(a1 + ko), umma_desc_sw128(b1 + ko), Cfg::kIdesc, 1u);
      }
      tc_commit(&empty[s]);
    }
    tc_commit(&done);
  }
  __syncwarp();
  // warp w owns TMEM lanes 32 (w % 4) .. (rows) at columns 32 (w / 4) ..;
  // its C (or D) values are loaded while the MMAs still run: C is neither
  // read nor written by this CTA's K loop
  float* C = pc + tk.c;
  const int q = warp & 3, c0 = (warp >> 2) * 32;
  const int row = m0 + q * 32 + lane;
  const float* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : tk.ldc;
  const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
  const float sgn = tk.mode == kGemmSet ? -1.0f : 1.0f;
  float cv[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const int col = n0 + c0 + j;
    cv[j] = (ld && row < M && col < N) ? D[(int64_t)row + (int64_t)col * ldD] : 0.0f;
  }
  tc_wait_done(&done, wait_ns, &failed);
  __syncthreads();
  const bool ok = !failed;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int nacc = nk < Cfg::kAccs ? nk : Cfg::kAccs;
    uint32_t v[32];
    float acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0f;
    for (int b = 0; b < nacc; ++b) {
      tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + c0), v);
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] += __uint_as_float(v[j]);
    }
    if (row < M) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int col = n0 + c0 + j;
        if (col < N) C[(int64_t)row + (int64_t)col * tk.ldc] = cv[j] - sgn * acc[j];
      }
    }
  } else if (t == 0) {
    atomicOr(flags + 1, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kTmemCols));
}

}  // namespace mfgpu
