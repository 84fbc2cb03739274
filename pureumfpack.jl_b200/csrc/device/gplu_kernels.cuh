// gplu_kernels.cuh -- Gilbert-Peierls left-looking sparse LU with threshold
// partial pivoting (src/gplu.jl:62-303) and the CSC triangular solves over its
// factors with the PureLU refinement (src/solve.jl:10-77,
// src/interface.jl:123-177), one warp per system.
//
// The method is a chain of n dependent column steps, each a depth-first
// reach in the graph of the partial L followed by a sparse forward solve, so a
// system cannot spread over the GPU; many systems run side by side, one warp
// each.  Inside a warp:
//   * the reach keeps the reference's depth-first order exactly (its
//     topological order fixes the order of the floating-point updates and the
//     pivot tie rule): lane 0's stack is warp-uniform state, and the scan of a
//     column of L for its next unmarked row reads 32 entries at a time, the
//     first unmarked one taken by ballot;
//   * the forward solve walks the reach in order and updates the rows of one
//     column of L per step with all lanes (a column's rows are distinct);
//   * the pivot search is a warp reduction over the reach with the first
//     position winning ties, as the reference's strict `>` scan;
//   * U's and L's new entries are appended in reach order by ballot ranks.
// The element type is Float64, Float32 or ComplexF64 (the reference's
// generic Tv).  Every product, sum, difference and quotient is rounded on its
// own (the *_rn intrinsics, never a contracted multiply-add), as the
// reference's scalar loops round them; complex values follow Julia's own
// multiplication, division and abs (GpArith), so factors and solutions are
// bit for bit the reference's restatement's.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mfgpu {

// One system of a batch.  Per-column arrays (pivot rows, workspaces, order,
// row scaling) start at col0, column pointers (n + 1 of A, of L, of U) at
// cp0, A's entries at nz0, L's entry segment at l0 (capacity lcap), U's at
// u0 (capacity ucap).
struct GpSys {
  int64_t n;
  int64_t col0;
  int64_t cp0;
  int64_t nz0;
  int64_t l0, lcap;
  int64_t u0, ucap;
};

// Per-system status besides 0 (done) and k > 0 (no nonzero pivot at column k
// under check, the reference's SingularException(k)).
constexpr int64_t kGpNotPermutation = -1;   // singular matrix factored with check = false
constexpr int64_t kGpOverflowL = -2;        // L's segment is too small: rerun with more room
constexpr int64_t kGpOverflowU = -3;
constexpr int64_t kGpPending = -4;
constexpr int64_t kGpInternal = -5;         // a depth-first search left its bounds (never expected)

constexpr unsigned kGpFull = 0xffffffffu;
constexpr int kGpWarps = 4;                  // warps (systems) per CTA of the factor kernel
constexpr int kGpScan = 4;                   // 32-row chunks of a column of L loaded together

// ComplexF64 as Julia lays it out: (re, im) doubles.
struct __align__(16) GpComplex {
  double re, im;
};

// Julia's abs(::ComplexF64) = hypot(re, im): Borges' algorithm with the
// fused-multiply-add correction, as Julia Base runs it on hardware with FMA.
__device__ __forceinline__ double gp_hypot(double x, double y) {
  double ax = fabs(x), ay = fabs(y);
  if (isinf(ax) || isinf(ay)) return __longlong_as_double(0x7ff0000000000000LL);
  if (ay > ax) {
    const double t = ax;
    ax = ay;
    ay = t;
  }
  if (ay <= __dmul_rn(ax, __dsqrt_rn(0x1p-53))) return ax;   // widely varying operands (and ay == 0)
  double scale = 0x1p-563;                                   // eps * sqrt(floatmin)
  if (ax > __dsqrt_rn(0x1.fffffffffffffp+1022)) {           // sqrt(floatmax / 2)
    ax = __dmul_rn(ax, scale);
    ay = __dmul_rn(ay, scale);
    scale = __ddiv_rn(1.0, scale);
  } else if (ay < 0x1p-511) {                                // sqrt(floatmin)
    ax = __ddiv_rn(ax, scale);
    ay = __ddiv_rn(ay, scale);
  } else {
    scale = 1.0;
  }
  double h = __dsqrt_rn(__fma_rn(ax, ax, __dmul_rn(ay, ay)));
  const double hsq = __dmul_rn(h, h), axsq = __dmul_rn(ax, ax);
  const double num = __dsub_rn(__dadd_rn(__fma_rn(-ay, ay, __dsub_rn(hsq, axsq)), __fma_rn(h, h, -hsq)),
                               __fma_rn(ax, ax, -axsq));
  h = __dsub_rn(h, __ddiv_rn(num, __dmul_rn(2.0, h)));
  return __dmul_rn(h, scale);
}

__device__ __forceinline__ double gp_cdiv2(double a, double b, double c, double d, double r, double t) {
  if (r != 0) {
    const double br = __dmul_rn(b, r);
    return br != 0 ? __dmul_rn(__dadd_rn(a, br), t) : __dadd_rn(__dmul_rn(a, t), __dmul_rn(__dmul_rn(b, t), r));
  }
  return __dmul_rn(__dadd_rn(a, __dmul_rn(d, __ddiv_rn(b, c))), t);
}

// Julia's ComplexF64 division: Smith's method with the Baudin-Smith twist
// and its overflow / underflow scaling.
__device__ __forceinline__ GpComplex gp_cdiv(GpComplex z, GpComplex w) {
  double a = z.re, b = z.im, c = w.re, d = w.im;
  const double ab = fabs(a) >= fabs(b) ? fabs(a) : fabs(b);
  const double cd = fabs(c) >= fabs(d) ? fabs(c) : fabs(d);
  const double halfov = 0x1.fffffffffffffp+1022;   // floatmax / 2
  const double twounf = 0x1p-969;                   // 2 floatmin / eps
  const double bs = 0x1p+105;                       // 2 / eps^2
  double S = 1.0;
  if (ab >= halfov) { a = 0.5 * a; b = 0.5 * b; S = 2.0 * S; }
  if (cd >= halfov) { c = 0.5 * c; d = 0.5 * d; S = 0.5 * S; }
  if (ab <= twounf) { a = __dmul_rn(a, bs); b = __dmul_rn(b, bs); S = __ddiv_rn(S, bs); }
  if (cd <= twounf) { c = __dmul_rn(c, bs); d = __dmul_rn(d, bs); S = __dmul_rn(S, bs); }
  double p, q;
  if (fabs(d) <= fabs(c)) {
    const double r = __ddiv_rn(d, c), t = __ddiv_rn(1.0, __dadd_rn(c, __dmul_rn(d, r)));
    p = gp_cdiv2(a, b, c, d, r, t);
    q = gp_cdiv2(b, -a, c, d, r, t);
  } else {
    const double r = __ddiv_rn(c, d), t = __ddiv_rn(1.0, __dadd_rn(d, __dmul_rn(c, r)));
    p = gp_cdiv2(b, a, d, c, r, t);
    q = -gp_cdiv2(a, -b, d, c, r, t);
  }
  return GpComplex{__dmul_rn(p, S), __dmul_rn(q, S)};
}

// The scalar operations of one element type, each rounded on its own as
// Julia rounds them (R: the real type of magnitudes, row scaling and tol).
template <typename T>
struct GpArith;
template <>
struct GpArith<double> {
  using R = double;
  static __device__ __forceinline__ double zero() { return 0.0; }
  static __device__ __forceinline__ double one() { return 1.0; }
  static __device__ __forceinline__ double scale(R r, double a) { return __dmul_rn(a, r); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ R mag(double a) { return fabs(a); }
  static __device__ __forceinline__ R rmul(R a, R b) { return __dmul_rn(a, b); }
};
template <>
struct GpArith<float> {
  using R = float;
  static __device__ __forceinline__ float zero() { return 0.0f; }
  static __device__ __forceinline__ float one() { return 1.0f; }
  static __device__ __forceinline__ float scale(R r, float a) { return __fmul_rn(a, r); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ R mag(float a) { return fabsf(a); }
  static __device__ __forceinline__ R rmul(R a, R b) { return __fmul_rn(a, b); }
};
template <>
struct GpArith<GpComplex> {
  using R = double;
  static __device__ __forceinline__ GpComplex zero() { return GpComplex{0.0, 0.0}; }
  static __device__ __forceinline__ GpComplex one() { return GpComplex{1.0, 0.0}; }
  static __device__ __forceinline__ GpComplex scale(R r, GpComplex a) {
    return GpComplex{__dmul_rn(a.re, r), __dmul_rn(a.im, r)};
  }
  static __device__ __forceinline__ GpComplex mul(GpComplex z, GpComplex w) {
    return GpComplex{__dsub_rn(__dmul_rn(z.re, w.re), __dmul_rn(z.im, w.im)),
                     __dadd_rn(__dmul_rn(z.re, w.im), __dmul_rn(z.im, w.re))};
  }
  static __device__ __forceinline__ GpComplex add(GpComplex a, GpComplex b) {
    return GpComplex{__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)};
  }
  static __device__ __forceinline__ GpComplex sub(GpComplex a, GpComplex b) {
    return GpComplex{__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)};
  }
  static __device__ __forceinline__ GpComplex div(GpComplex a, GpComplex b) { return gp_cdiv(a, b); }
  static __device__ __forceinline__ R mag(GpComplex a) { return gp_hypot(a.re, a.im); }
  static __device__ __forceinline__ R rmul(R a, R b) { return __dmul_rn(a, b); }
};

// Workspace of the factor kernel, per column of every system.
template <typename T>
struct GpWork {
  T* x;             // dense column being solved (zero between steps)
  int32_t* xi;      // reach in topological order (xi[top..n))
  int32_t* stack;   // depth-first stack
  int64_t* pstack;  // resume position in L of each stack entry
  int32_t* mark;    // k + 1 when a row is in column k's reach
};

// Factors being built: L's rows are A's row numbers until the finish kernel
// relabels them in pivot order; L's unit diagonal comes first in its column,
// U's diagonal last.
template <typename T>
struct GpFactors {
  int64_t* lp;      // per system n + 1, relative to the system's l0
  int32_t* li;
  T* lx;
  int64_t* up;
  int32_t* ui;
  T* ux;
  int32_t* pinv;    // row -> pivot step, -1 before it is a pivot
};

// Depth-first search from the pivot row j0 (pinv[j0] = J0 >= 0;
// gplu.jl:70-102): returns the new top; the rows it finishes go to
// xi[--top].  All lanes hold the same head, j, J, pp; lane 0 writes the
// stack and j's mark, a __syncwarp ends every step.  A row that is not yet a
// pivot has no edges: pushing it finishes it on the next step, so the scan
// finishes the unmarked ones it meets before the first unmarked pivot row at
// once, in scan order (each lane writes its own row's mark and xi slot), and
// pushes only pivot rows.  A search that would leave its n-entry stack or
// reach arrays returns -1 instead (no row is pushed or finished twice, so
// this does not happen).
__device__ __forceinline__ int64_t gp_dfs(int32_t j0, int32_t J0, int32_t stamp, int64_t top, int64_t n,
                                          const int64_t* __restrict__ lp, const int32_t* __restrict__ li,
                                          const int32_t* __restrict__ pinv, int32_t* mark, int32_t* xi,
                                          int32_t* stack, int64_t* pstack, int lane) {
  int64_t head = 0;
  int32_t j = j0, J = J0;
  int64_t pp = lp[J0];
  if (lane == 0) {
    stack[0] = j0;
    mark[j0] = stamp;
  }
  __syncwarp();
  while (head >= 0) {
    const int64_t pend = lp[J + 1];
    bool pushed = false;
    int32_t inext = -1, Jnext = -1;
    // the column is read kGpScan chunks of 32 rows at a time (their rows,
    // marks and pivot steps loaded together), then consumed chunk by chunk
    // in order; a column's rows are distinct, so finishing rows in one chunk
    // leaves the marks loaded for the next ones valid
    while (pp < pend && !pushed) {
      int32_t iv[kGpScan], jv[kGpScan];
      bool uv[kGpScan];
#pragma unroll
      for (int c = 0; c < kGpScan; ++c) {
        const int64_t p = pp + 32 * c + lane;
        iv[c] = p < pend ? li[p] : -1;
      }
#pragma unroll
      for (int c = 0; c < kGpScan; ++c)
        uv[c] = iv[c] >= 0 && iv[c] != j && mark[iv[c]] != stamp;   // j's own mark may still be in flight
#pragma unroll
      for (int c = 0; c < kGpScan; ++c) jv[c] = uv[c] ? pinv[iv[c]] : -1;
#pragma unroll
      for (int c = 0; c < kGpScan; ++c) {
        if (pushed) break;
        const unsigned bu = __ballot_sync(kGpFull, uv[c]);
        const unsigned bl = __ballot_sync(kGpFull, uv[c] && jv[c] < 0);
        const unsigned bp = bu & ~bl;
        const int f = bp ? __ffs(bp) - 1 : 32;
        const unsigned leaves = f == 32 ? bl : (bl & ((1u << f) - 1u));
        if (leaves) {
          const int cnt = __popc(leaves);
          if (top < cnt) return -1;
          if ((leaves >> lane) & 1u) {
            xi[top - 1 - __popc(leaves & ((1u << lane) - 1u))] = iv[c];
            mark[iv[c]] = stamp;
          }
          top -= cnt;
        }
        if (bp) {
          inext = __shfl_sync(kGpFull, iv[c], f);
          Jnext = __shfl_sync(kGpFull, jv[c], f);
          pp += 32 * c + f;
          pushed = true;
        }
      }
      if (!pushed) pp += 32 * kGpScan;
    }
    if (pushed) {
      if (head + 1 >= n) return -1;
      if (lane == 0) {
        pstack[head] = pp;
        stack[head + 1] = inext;
        mark[inext] = stamp;
      }
      ++head;
      j = inext;
      J = Jnext;
      pp = lp[J];
      __syncwarp();
    } else {
      if (top <= 0) return -1;
      --top;
      if (lane == 0) xi[top] = j;
      --head;
      __syncwarp();
      if (head >= 0) {
        j = stack[head];
        pp = pstack[head];
        J = pinv[j];
      }
    }
  }
  return top;
}

// gplu (gplu.jl:173-291) for the systems list[0..nlist), one warp each.
// A's rows are 0-based within the system (ascending, distinct); rs (NULL: no
// scaling) multiplies row i of A as Rs .* A does; q is the column order.
// status[s] receives 0, k + 1 or a kGp* code.  Workspaces need no clearing:
// each system clears its own at its start.
template <typename T>
__global__ void __launch_bounds__(32 * kGpWarps, 1)
    k_gplu_factor(const GpSys* __restrict__ sys, const int32_t* __restrict__ list, int64_t nlist,
                  const int64_t* __restrict__ acp, const int32_t* __restrict__ ari, const T* __restrict__ ax,
                  const typename GpArith<T>::R* __restrict__ rs, const int32_t* __restrict__ qord,
                  typename GpArith<T>::R tol, int check, GpFactors<T> F, GpWork<T> W, int64_t* __restrict__ status) {
  using O = GpArith<T>;
  using R = typename O::R;
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kGpWarps + (threadIdx.x >> 5);
  if (w >= nlist) return;
  const int64_t s = list[w];
  const GpSys d = sys[s];
  const int64_t n = d.n;
  const int64_t* cp = acp + d.cp0;
  const int32_t* ri = ari + d.nz0;
  const T* av = ax + d.nz0;
  const R* r = rs ? rs + d.col0 : nullptr;
  const int32_t* q = qord + d.col0;
  int64_t* lp = F.lp + d.cp0;
  int64_t* up = F.up + d.cp0;
  int32_t* li = F.li + d.l0;
  T* lx = F.lx + d.l0;
  int32_t* ui = F.ui + d.u0;
  T* ux = F.ux + d.u0;
  int32_t* pinv = F.pinv + d.col0;
  T* x = W.x + d.col0;
  int32_t* xi = W.xi + d.col0;
  int32_t* stack = W.stack + d.col0;
  int64_t* pstack = W.pstack + d.col0;
  int32_t* mark = W.mark + d.col0;

  for (int64_t i = lane; i < n; i += 32) {
    pinv[i] = -1;
    mark[i] = 0;
    x[i] = O::zero();
  }
  if (lane == 0) {
    lp[0] = 0;
    up[0] = 0;
  }
  __syncwarp();
  int64_t lnz = 0, unz = 0;
  for (int64_t k = 0; k < n; ++k) {
    const int32_t col = q[k];
    const int32_t stamp = (int32_t)(k + 1);
    const int64_t a0 = cp[col], a1 = cp[col + 1];
    // reach of A(:, col) in the graph of L (gplu.jl:106-122)
    int64_t top = n;
    for (int64_t pa = a0; pa < a1; ++pa) {
      const int32_t b = ri[pa];
      if (mark[b] == stamp) continue;
      const int32_t Jb = pinv[b];
      if (Jb < 0) {   // a row without edges finishes at once
        if (top <= 0) {
          top = -1;
        } else {
          --top;
          if (lane == 0) {
            mark[b] = stamp;
            xi[top] = b;
          }
          __syncwarp();
        }
      } else {
        top = gp_dfs(b, Jb, stamp, top, n, lp, li, pinv, mark, xi, stack, pstack, lane);
      }
      if (top < 0) {
        if (lane == 0) status[s] = kGpInternal;
        return;
      }
    }
    // x = A(:, col), scaled (x is zero outside the previous reaches)
    for (int64_t pa = a0 + lane; pa < a1; pa += 32) {
      const int32_t i = ri[pa];
      x[i] = r ? O::scale(r[i], av[pa]) : av[pa];
    }
    __syncwarp();
    // L x = A(:, col) over the reach in topological order (gplu.jl:226-235)
    for (int64_t base = top; base < n; base += 32) {
      const int64_t px = base + lane;
      int32_t jl = -1, Jl = -1;
      int64_t b0 = 0, b1 = 0;
      if (px < n) {
        jl = xi[px];
        Jl = pinv[jl];
        if (Jl >= 0) {
          b0 = lp[Jl] + 1;
          b1 = lp[Jl + 1];
        }
      }
      const int cnt = (int)((n - base) < 32 ? (n - base) : 32);
      for (int t = 0; t < cnt; ++t) {
        const int64_t p0 = __shfl_sync(kGpFull, b0, t), p1 = __shfl_sync(kGpFull, b1, t);
        if (p0 >= p1) continue;   // not a pivot row, or a column of L without entries below its diagonal
        const int32_t j = __shfl_sync(kGpFull, jl, t);
        const T xj = x[j];
        // four rows per lane in flight (the column's rows are distinct)
        int64_t p = p0 + lane;
        for (; p + 96 < p1; p += 128) {
          const int32_t i0 = li[p], i1 = li[p + 32], i2 = li[p + 64], i3 = li[p + 96];
          const T a0 = lx[p], a1 = lx[p + 32], a2 = lx[p + 64], a3 = lx[p + 96];
          const T y0 = x[i0], y1 = x[i1], y2 = x[i2], y3 = x[i3];
          x[i0] = O::sub(y0, O::mul(a0, xj));
          x[i1] = O::sub(y1, O::mul(a1, xj));
          x[i2] = O::sub(y2, O::mul(a2, xj));
          x[i3] = O::sub(y3, O::mul(a3, xj));
        }
        for (; p < p1; p += 32) {
          const int32_t i = li[p];
          x[i] = O::sub(x[i], O::mul(lx[p], xj));
        }
        __syncwarp();
      }
    }
    // U entries in reach order; largest unpivoted magnitude, first on ties
    // (gplu.jl:238-254)
    R best = R(-1);
    int64_t bpos = INT64_MAX;
    for (int64_t base = top; base < n; base += 32) {
      const int64_t px = base + lane;
      bool piv = false;
      int32_t pi = -1;
      T v = O::zero();
      if (px < n) {
        const int32_t i = xi[px];
        pi = pinv[i];
        v = x[i];
        piv = pi >= 0;
        if (!piv) {
          const R t = O::mag(v);
          if (t > best) {
            best = t;
            bpos = px;
          }
        }
      }
      const unsigned bal = __ballot_sync(kGpFull, piv);
      const int64_t c = __popc(bal);
      if (unz + c + 1 > d.ucap) {
        if (lane == 0) status[s] = kGpOverflowU;
        return;
      }
      if (piv) {
        const int rk = __popc(bal & ((1u << lane) - 1u));
        ui[unz + rk] = pi;
        ux[unz + rk] = v;
      }
      unz += c;
    }
    for (int off = 16; off; off >>= 1) {
      const R ob = __shfl_xor_sync(kGpFull, best, off);
      const int64_t op = __shfl_xor_sync(kGpFull, bpos, off);
      if (ob > best || (ob == best && op < bpos)) {
        best = ob;
        bpos = op;
      }
    }
    int32_t ipiv = bpos == INT64_MAX ? -1 : xi[bpos];
    if (ipiv < 0 || best <= R(0)) {   // gplu.jl:255-258
      if (check) {
        if (lane == 0) status[s] = k + 1;
        return;
      }
      if (ipiv < 0) ipiv = col;
    }
    // threshold partial pivoting: the diagonal row when it is large enough
    if (pinv[col] < 0 && O::mag(x[col]) >= O::rmul(tol, best)) ipiv = col;
    const T pivot = x[ipiv];
    if (lnz + 1 > d.lcap) {
      if (lane == 0) status[s] = kGpOverflowL;
      return;
    }
    if (lane == 0) {
      ui[unz] = (int32_t)k;
      ux[unz] = pivot;
      up[k + 1] = unz + 1;
      pinv[ipiv] = (int32_t)k;
      li[lnz] = ipiv;
      lx[lnz] = O::one();
    }
    ++unz;
    ++lnz;
    __syncwarp();
    // L's column: the unpivoted rows of the reach divided by the pivot, and
    // x cleared for the next step (gplu.jl:274-288)
    for (int64_t base = top; base < n; base += 32) {
      const int64_t px = base + lane;
      bool keep = false;
      int32_t i = -1;
      T v = O::zero();
      if (px < n) {
        i = xi[px];
        keep = pinv[i] < 0;
        v = x[i];
      }
      const unsigned bal = __ballot_sync(kGpFull, keep);
      const int64_t c = __popc(bal);
      if (lnz + c > d.lcap) {
        if (lane == 0) status[s] = kGpOverflowL;
        return;
      }
      if (keep) {
        const int rk = __popc(bal & ((1u << lane) - 1u));
        li[lnz + rk] = i;
        lx[lnz + rk] = O::div(v, pivot);
      }
      lnz += c;
      if (px < n) x[i] = O::zero();
    }
    if (lane == 0) lp[k + 1] = lnz;
    __syncwarp();
  }
  // every row must have become a pivot (the reference's invperm)
  bool missing = false;
  for (int64_t i = lane; i < n; i += 32) missing |= pinv[i] < 0;
  missing = __any_sync(kGpFull, missing);
  if (lane == 0) status[s] = missing ? kGpNotPermutation : 0;
}

// Copy the factors of the finished systems list[0..nlist) from the old
// segments to the new ones (a rerun grew other systems' room).
template <typename T>
__global__ void k_gplu_move(const GpSys* __restrict__ olds, const GpSys* __restrict__ news,
                            const int32_t* __restrict__ list, int64_t nlist, const int64_t* __restrict__ lp,
                            const int64_t* __restrict__ up, const int32_t* __restrict__ oli, const T* __restrict__ olx,
                            const int32_t* __restrict__ oui, const T* __restrict__ oux, int32_t* __restrict__ nli,
                            T* __restrict__ nlx, int32_t* __restrict__ nui, T* __restrict__ nux) {
  const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nlist) return;
  const int64_t s = list[w];
  const GpSys o = olds[s], d = news[s];
  const int64_t nl = lp[d.cp0 + d.n], nu = up[d.cp0 + d.n];
  for (int64_t e = lane; e < nl; e += 32) {
    nli[d.l0 + e] = oli[o.l0 + e];
    nlx[d.l0 + e] = olx[o.l0 + e];
  }
  for (int64_t e = lane; e < nu; e += 32) {
    nui[d.u0 + e] = oui[o.u0 + e];
    nux[d.u0 + e] = oux[o.u0 + e];
  }
}

constexpr int kGpSortStage = 1024;   // keys of a column staged in shared memory per warp

// One column's (key, value) pairs from (ki, kx) to (oi, ox): keys relabelled
// by map (NULL: as they are) and, when sorting, placed by rank (the keys of
// a column are distinct, so the rank is the sorted position; gplu.jl:383-415).
template <typename T>
__device__ __forceinline__ void gp_column_out(int64_t len, const int32_t* ki, const T* kx, const int32_t* map,
                                              bool sort, int32_t* oi, T* ox, int32_t* stage, int lane) {
  if (!sort || len <= 1) {
    for (int64_t e = lane; e < len; e += 32) {
      oi[e] = map ? map[ki[e]] : ki[e];
      ox[e] = kx[e];
    }
    return;
  }
  const bool staged = len <= kGpSortStage;
  if (staged) {
    for (int64_t e = lane; e < len; e += 32) stage[e] = map ? map[ki[e]] : ki[e];
    __syncwarp();
  }
  for (int64_t e = lane; e < len; e += 32) {
    const int32_t key = staged ? stage[e] : (map ? map[ki[e]] : ki[e]);
    int64_t rank = 0;
    if (staged) {
      for (int64_t f = 0; f < len; ++f) rank += stage[f] < key;
    } else {
      for (int64_t f = 0; f < len; ++f) rank += (map ? map[ki[f]] : ki[f]) < key;
    }
    oi[rank] = key;
    ox[rank] = kx[e];
  }
  __syncwarp();
}

// Finished factors (gplu.jl:292-302): L's rows in pivot order, both factors'
// columns sorted when sort is set, p = invperm(pinv).  One warp per column of
// every system whose status is 0.
template <typename T>
__global__ void __launch_bounds__(32 * kGpWarps)
    k_gplu_finish(const GpSys* __restrict__ sys, const int32_t* __restrict__ col_sys, int64_t ncols,
                  const int64_t* __restrict__ status, GpFactors<T> F, int sort, int32_t* __restrict__ lo_i,
                  T* __restrict__ lo_x, int32_t* __restrict__ uo_i, T* __restrict__ uo_x,
                  int32_t* __restrict__ perm) {
  __shared__ int32_t stage[kGpWarps][kGpSortStage];
  const int lane = threadIdx.x & 31;
  const int wl = threadIdx.x >> 5;
  const int64_t g = (int64_t)blockIdx.x * kGpWarps + wl;
  if (g >= ncols) return;
  const int32_t s = col_sys[g];
  if (status[s] != 0) return;
  const GpSys d = sys[s];
  const int64_t j = g - d.col0;
  const int32_t* pinv = F.pinv + d.col0;
  const int64_t* lp = F.lp + d.cp0;
  const int64_t* up = F.up + d.cp0;
  gp_column_out(lp[j + 1] - lp[j], F.li + d.l0 + lp[j], F.lx + d.l0 + lp[j], pinv, sort != 0,
                lo_i + d.l0 + lp[j], lo_x + d.l0 + lp[j], stage[wl], lane);
  gp_column_out(up[j + 1] - up[j], F.ui + d.u0 + up[j], F.ux + d.u0 + up[j], nullptr, sort != 0,
                uo_i + d.u0 + up[j], uo_x + d.u0 + up[j], stage[wl], lane);
  if (lane == 0) perm[d.col0 + pinv[j]] = (int32_t)j;
}

// The finished factors of a batch, for the solves.
template <typename T>
struct GpSolveArgs {
  const GpSys* sys;
  const int64_t* lp;
  const int32_t* li;
  const T* lx;
  const int64_t* up;
  const int32_t* ui;
  const T* ux;
  const int32_t* perm;                    // p (0-based)
  const int32_t* q;
  const typename GpArith<T>::R* rs;       // NULL: the raw GPLUFactorization solve
  const int64_t* acp;                     // unscaled A for the refinement residual
  const int32_t* ari;
  const T* ax;
};

// c = L \ c then U \ c in place (solve.jl:10-39), all lanes of the warp.
template <typename T>
__device__ __forceinline__ void gp_lu_solve(const GpSolveArgs<T>& A, const GpSys& d, T* c, int lane) {
  using O = GpArith<T>;
  const int64_t n = d.n;
  const int64_t* lp = A.lp + d.cp0;
  const int32_t* li = A.li + d.l0;
  const T* lx = A.lx + d.l0;
  const int64_t* up = A.up + d.cp0;
  const int32_t* ui = A.ui + d.u0;
  const T* ux = A.ux + d.u0;
  for (int64_t j = 0; j < n; ++j) {
    const int64_t p0 = lp[j] + 1, p1 = lp[j + 1];
    if (p0 >= p1) continue;
    const T yj = c[j];
    for (int64_t p = p0 + lane; p < p1; p += 32) {
      const int32_t i = li[p];
      c[i] = O::sub(c[i], O::mul(lx[p], yj));
    }
    __syncwarp();
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    const int64_t p0 = up[j], pd = up[j + 1] - 1;
    const T yj = O::div(c[j], ux[pd]);
    for (int64_t p = p0 + lane; p < pd; p += 32) {
      const int32_t i = ui[p];
      c[i] = O::sub(c[i], O::mul(ux[p], yj));
    }
    if (lane == 0) c[j] = yj;
    __syncwarp();
  }
}

// solve(F, b; refine) (interface.jl:123-138,170-177; solve.jl:66-77) for
// every (system, right-hand side): one warp each.  B, X and the two
// workspaces hold system s's nrhs columns at col0 * nrhs, column r at
// + r * n.  The refinement residual r = b - A x is the column-oriented
// product of the unscaled A, as SparseArrays forms it.
template <typename T>
__global__ void __launch_bounds__(128, 1)
    k_gplu_solve(GpSolveArgs<T> A, int64_t nsys, int64_t nrhs, const T* __restrict__ B, T* __restrict__ X,
                 T* __restrict__ C, T* __restrict__ R, int refine) {
  using O = GpArith<T>;
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= nsys * nrhs) return;
  const int64_t s = w / nrhs, rr = w - s * nrhs;
  const GpSys d = A.sys[s];
  const int64_t n = d.n;
  const int64_t off = d.col0 * nrhs + rr * n;
  const T* b = B + off;
  T* x = X + off;
  T* c = C + off;
  T* ax = R + off;
  const int32_t* p = A.perm + d.col0;
  const int32_t* q = A.q + d.col0;
  const auto* rs = A.rs ? A.rs + d.col0 : nullptr;
  for (int64_t k = lane; k < n; k += 32) {
    const int32_t i = p[k];
    c[k] = rs ? O::scale(rs[i], b[i]) : b[i];
  }
  __syncwarp();
  gp_lu_solve(A, d, c, lane);
  for (int64_t k = lane; k < n; k += 32) x[q[k]] = c[k];
  __syncwarp();
  const int64_t* cp = A.acp + d.cp0;
  const int32_t* ri = A.ari + d.nz0;
  const T* av = A.ax + d.nz0;
  for (int it = 0; it < refine; ++it) {
    for (int64_t i = lane; i < n; i += 32) ax[i] = O::zero();
    __syncwarp();
    for (int64_t j = 0; j < n; ++j) {
      const T xj = x[j];
      for (int64_t pa = cp[j] + lane; pa < cp[j + 1]; pa += 32) {
        const int32_t i = ri[pa];
        ax[i] = O::add(ax[i], O::mul(av[pa], xj));
      }
      __syncwarp();
    }
    for (int64_t i = lane; i < n; i += 32) ax[i] = O::sub(b[i], ax[i]);   // r = b - A x
    __syncwarp();
    for (int64_t k = lane; k < n; k += 32) {
      const int32_t i = p[k];
      c[k] = rs ? O::scale(rs[i], ax[i]) : ax[i];
    }
    __syncwarp();
    gp_lu_solve(A, d, c, lane);
    for (int64_t k = lane; k < n; k += 32) x[q[k]] = O::add(x[q[k]], c[k]);
    __syncwarp();
  }
}

}  // namespace mfgpu
