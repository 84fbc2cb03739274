// common.cuh -- device helpers shared by libmfgpu's kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../plan.h"

namespace mfgpu {

// Device copies of the pattern-only plan arrays (see plan.h for meaning).
struct DevPlan {
  int64_t n, ns;
  const int32_t* c1;
  const int32_t* np;
  const int32_t* nu;
  const int32_t* nf;
  const int64_t* upd_off;
  const int64_t* front_off;
  const int64_t* colbase;
  const int32_t* child_ptr;
  const int32_t* child_idx;
  const int32_t* upd;
  const int32_t* rel;
  const int64_t* uoff;
  const int32_t* v_src;
  const int32_t* v_srow;
  const int32_t* v_frow;
  const int32_t* fc_super;
  const int32_t* fc_vbeg;
  const int32_t* fc_vend;
  const int32_t* fc_ch_ptr;
  const int32_t* fc_ch;
  const int64_t* lcolptr;
  const int64_t* ucolptr;
  const int32_t* qf;
  const int32_t* csr_ptr;
  const int32_t* csr_col;
  const int32_t* csr_src;
  const int64_t* dinv_off;   // per supernode: first 64-block of its inverted diagonal blocks (-1: small front)
  const int64_t* inv_off;    // per supernode: pool offset of inv(L11); inv(U11) follows (-1: small front)
  const int64_t* lpan_off;   // per supernode: factored first np columns (leading dimension nf)
  const int64_t* u12_off;    // per supernode: factored U12 (leading dimension lean ? np : nf)
  int32_t lean;              // panels in the compact panel pool (fronts' memory reused)
  int32_t merged;            // fronts merge original supernodes (o_* and fcu are set)
  const int32_t* seg_end;    // per column: front-local end of the rows it may pivot on
  const int32_t* col_orig;   // per column: original supernode (merged plans)
  const int32_t* o_c1;
  const int32_t* o_np;
  const int64_t* o_upd_off;
  const int32_t* o_upd;
  const int32_t* o_xpos;     // front-local column of each original update-set entry
  const int64_t* fcu_ptr;    // per front column: its U blocks
  const UBlock* fcu;
};

__device__ __forceinline__ int u12_ld(const DevPlan& P, int s) { return P.lean ? P.np[s] : P.nf[s]; }

// Per-factorization numeric state.
struct DevState {
  int32_t* ipiv;        // n: local pivot row (0-based within the supernode) of each elimination step
  int32_t* info;        // ns: first zero pivot (local), INT32_MAX if none
  int32_t* prow;        // n: V-row of each factor row
  int32_t* rowfac;      // n: factor row of each V-row
  int32_t* flags;       // [0]: speculative pivot order violated
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }

// Maximum that keeps a NaN (fmax drops it): a reduction over magnitudes
// reports a NaN anywhere in its input.  The arguments are magnitudes (fabs
// clears the sign), so a NaN result is a positive NaN, whose bit pattern
// orders above +Inf's: atomicMax on the bits keeps it too.
__device__ __forceinline__ double max_keep_nan(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }

// (|value|, index) argmax with LAPACK idamax tie-breaking: the first (lowest)
// index among equal magnitudes wins.
struct ArgMax {
  double v;
  int i;
};
__device__ __forceinline__ ArgMax better(ArgMax a, ArgMax b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}
__device__ __forceinline__ ArgMax warp_argmax(ArgMax a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ArgMax b;
    b.v = __shfl_xor_sync(0xffffffffu, a.v, o);
    b.i = __shfl_xor_sync(0xffffffffu, a.i, o);
    a = better(a, b);
  }
  return a;
}

// Block-wide argmax; `red` needs blockDim/32 entries.  All threads get the result.
__device__ __forceinline__ ArgMax block_argmax(ArgMax a, ArgMax* red) {
  a = warp_argmax(a);
  const int nw = blockDim.x >> 5;
  if (lane_id() == 0) red[warp_id()] = a;
  __syncthreads();
  if (warp_id() == 0) {
    ArgMax b = lane_id() < nw ? red[lane_id()] : ArgMax{-1.0, 0x7fffffff};
    b = warp_argmax(b);
    if (lane_id() == 0) red[0] = b;
  }
  __syncthreads();
  ArgMax r = red[0];
  __syncthreads();
  return r;
}

template <typename T>
__device__ __forceinline__ double absd(T x) {
  return fabs((double)x);
}

// ---------------------------------------------------------------------------
// ComplexF64 fronts: (re, im) pairs in Julia's ComplexF64 memory layout.  The
// factor and solve kernels are templates over the front element type, so
// they run on complex fronts through these operators.  The pivot magnitude
// is |re| + |im|, the one LAPACK's izamax (dcabs1) and so Julia's lu! on a
// ComplexF64 block use; division follows Smith's scaled formula.
// ---------------------------------------------------------------------------
struct __align__(16) zc {
  double re, im;
  zc() = default;
  __host__ __device__ constexpr zc(double r) : re(r), im(0.0) {}
  __host__ __device__ constexpr zc(double r, double i) : re(r), im(i) {}
};
__host__ __device__ __forceinline__ zc operator+(zc a, zc b) { return zc(a.re + b.re, a.im + b.im); }
__host__ __device__ __forceinline__ zc operator-(zc a, zc b) { return zc(a.re - b.re, a.im - b.im); }
__host__ __device__ __forceinline__ zc operator-(zc a) { return zc(-a.re, -a.im); }
__host__ __device__ __forceinline__ zc operator*(zc a, zc b) {
  return zc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__host__ __device__ __forceinline__ zc operator/(zc a, zc b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, d = b.re + b.im * r;
    return zc((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  }
  const double r = b.re / b.im, d = b.im + b.re * r;
  return zc((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}
__host__ __device__ __forceinline__ zc& operator+=(zc& a, zc b) { return a = a + b; }
__host__ __device__ __forceinline__ zc& operator-=(zc& a, zc b) { return a = a - b; }
__host__ __device__ __forceinline__ zc& operator*=(zc& a, zc b) { return a = a * b; }
__host__ __device__ __forceinline__ zc& operator/=(zc& a, zc b) { return a = a / b; }
__host__ __device__ __forceinline__ bool operator==(zc a, zc b) { return a.re == b.re && a.im == b.im; }
__host__ __device__ __forceinline__ bool operator!=(zc a, zc b) { return !(a == b); }
template <>
__device__ __forceinline__ double absd<zc>(zc x) {
  return fabs(x.re) + fabs(x.im);
}

// Element type of the caller's vectors and of A's values for fronts of type
// T: FP64 for the FP64 and FP32 fronts (right-hand sides, solutions,
// residuals and the values V = A[qf, qf] stay FP64), ComplexF64 for complex
// fronts.
template <typename T>
struct WideOf {
  using type = double;
};
template <>
struct WideOf<zc> {
  using type = zc;
};
template <typename T>
using Wide = typename WideOf<T>::type;
template <typename T>
constexpr bool is_complex_v = false;
template <>
constexpr bool is_complex_v<zc> = true;

// A value of V (Wide<T>) into a front of type T (FP32 fronts round it once).
template <typename T>
__device__ __forceinline__ T to_front(Wide<T> v) {
  return (T)v;
}

// 8-byte asynchronous global->shared copy with zero fill when !pred.
// Exact e / d and e % d by one 64-bit multiply and shift, for e * d < 2^32
// (m = ceil(2^32 / d): e m / 2^32 = e / d + e (m - 2^32 / d) / 2^32, whose
// second term stays below 1 / d, so the floor is e / d's).  Built once per
// divisor, it replaces the integer divisions of element loops that walk a
// block of runtime height.
struct FastDiv {
  uint64_t m;
  uint32_t d;
  // floor((2^32 - 1) / d) + 1 == ceil(2^32 / d) for every d >= 1 (one 32-bit division)
  __device__ __forceinline__ explicit FastDiv(uint32_t dd) : m((uint64_t)(0xFFFFFFFFu / dd) + 1), d(dd) {}
  __device__ __forceinline__ uint32_t div(uint32_t e) const { return (uint32_t)(((uint64_t)e * m) >> 32); }
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D += A * B on one 8x8x4 FP64 tensor-core tile (A row-major 8x4, B col-major 4x8).
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

}  // namespace mfgpu

namespace mfgpu {

// Shared-memory leading dimensions of the 64x64 tile product operands,
// chosen so DMMA fragment loads take the minimum two shared-memory wavefronts.
constexpr int kLdP = 72;   // left operand, column-major
constexpr int kLdQ = 68;   // right operand, column-major

// D = P * Q for 64x64 tiles in shared memory (P col-major ld kLdP, Q col-major
// ld kLdQ), 128 threads; D (col-major, ldd) may alias P or Q.
template <typename T>
__device__ void mm64(const T* P, const T* Q, T* D, int ldd);

template <>
__device__ __forceinline__ void mm64<double>(const double* P, const double* Q, double* D, int ldd) {
  const int lane = lane_id(), warp = warp_id();
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
  for (int kk = 0; kk < 64; kk += 4) {
    double af[4], bf[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) af[i] = P[(wm + i * 8 + (lane >> 2)) + (kk + (lane & 3)) * kLdP];
#pragma unroll
    for (int j = 0; j < 4; ++j) bf[j] = Q[(kk + (lane & 3)) + (wn + j * 8 + (lane >> 2)) * kLdQ];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        D[(wm + i * 8 + (lane >> 2)) + (wn + j * 8 + 2 * (lane & 3) + e) * ldd] = acc[i][j][e];
  __syncthreads();
}

template <>
__device__ __forceinline__ void mm64<float>(const float* P, const float* Q, float* D, int ldd) {
  const int t = threadIdx.x;
  const int tm = (t & 15) * 4, tn = (t >> 4) * 8;
  float acc[4][8] = {};
#pragma unroll 8
  for (int k = 0; k < 64; ++k) {
    float a[4], b[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = P[tm + i + k * kLdP];
#pragma unroll
    for (int j = 0; j < 8; ++j) b[j] = Q[k + (tn + j) * kLdQ];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) D[tm + i + (tn + j) * ldd] = acc[i][j];
  __syncthreads();
}

// ComplexF64 tiles on the CUDA cores (no complex tensor-core kind): the FP32
// form's thread layout, a 4 x 8 block of complex accumulators per thread.
template <>
__device__ __forceinline__ void mm64<zc>(const zc* P, const zc* Q, zc* D, int ldd) {
  const int t = threadIdx.x;
  const int tm = (t & 15) * 4, tn = (t >> 4) * 8;
  zc acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = zc(0.0);
#pragma unroll 2
  for (int k = 0; k < 64; ++k) {
    zc a[4], b[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = P[tm + i + k * kLdP];
#pragma unroll
    for (int j = 0; j < 8; ++j) b[j] = Q[k + (tn + j) * kLdQ];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) D[tm + i + (tn + j) * ldd] = acc[i][j];
  __syncthreads();
}

}  // namespace mfgpu
