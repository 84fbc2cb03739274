// solve_kernels.cuh -- supernodal forward/backward solves on the resident fronts.
//
// Restates _solve_factor (src/interface.jl:123-138) with lsolve!/usolve!
// (src/solve.jl:10-39) over the same factors, organised by supernode instead
// of by CSC column: the unit-lower L panel [L11; L21] and the upper panel
// [U11 U12] of every supernode are read straight from its front.
//
// Forward (leaves to root, one launch group per tree level): each supernode
// gathers its right-hand-side block -- the scaled, permuted b on its pivot
// rows (c = Rs[p] .* b[p]) plus the update vectors of its children, added in
// the children's LIFO order exactly like the matrix extend-add -- solves with
// L11 and forms its own update vector w = f[np:] - L21 * y.  No atomics, so
// the result is deterministic.  Backward (root to leaves): x_piv =
// U11 \ (y - U12 * x[upd]), gathering x of the ancestors' columns.  Finally
// x[q] = x_factor (interface.jl:134-136).  Work arrays are column-major with
// one column per right-hand side.  Small supernodes (nf <= 64) substitute
// column by column in one CTA; large ones multiply by the explicit inverses
// of L11 and U11 formed after the factorization, so their solves are batched
// GEMMs (the launch sequence is built in mfgpu.cu: build_solve_schedule).
#pragma once

#include "common.cuh"
#include "factor_kernels.cuh"

namespace mfgpu {

constexpr int kSolveCols = 32;      // right-hand sides per CTA in the small-supernode kernels
constexpr int kSolveThreads = 128;
// Right-hand sides per small-supernode CTA for fronts of type T: half as
// many for ComplexF64, whose blocks take twice the shared memory.
template <typename T>
__host__ __device__ constexpr int solve_cols() {
  return sizeof(T) > 8 ? kSolveCols / 2 : kSolveCols;
}

struct SolveArgs {
  int64_t nrhs;
  const double* b;      // right-hand sides (col-major, ldb), original row order
  int64_t ldb;
  const double* rs;     // row scaling or nullptr
  int64_t ldx;          // leading dimension of x (factor order), = n
  const void* bfo;      // c = Rs[p] .* b[p] in factor order and the front type (n x nrhs, ld ldx)
};

// c = Rs[p] .* b[p] (interface.jl:127-130) in factor order, once per solve:
// bfo[k, col] = Rs[orow] * b[orow, col] with orow = qf[prow[k]].  Columns
// advance slowest over the grid, so the gathered column of b stays in L2
// while its rows are read in factor order; the fronts then read their pivot
// rows of c contiguously.  Each factor row is read by its own supernode only,
// before that supernode writes the same rows of x, so c lives in x's storage.
// The element kernels below run on a (row blocks, right-hand-side groups)
// grid: row k = blockIdx.x * blockDim.x + threadIdx.x, column groups
// blockIdx.y, blockIdx.y + gridDim.y, ... (no 64-bit division per element);
// k_rhs_factor_order and k_solve_finish take kElemCols right-hand sides per
// thread, so a row's permutation and scaling are read once for all of them.
inline dim3 grid_rows_cols(int64_t n, int64_t nrhs, int threads = 256) {
  return dim3((unsigned)((n + threads - 1) / threads), (unsigned)(nrhs < 65535 ? (nrhs > 0 ? nrhs : 1) : 65535));
}
constexpr int kElemCols = 8;
inline dim3 grid_rows_groups(int64_t n, int64_t nrhs) {
  return grid_rows_cols(n, (nrhs + kElemCols - 1) / kElemCols);
}

template <typename T>
__global__ void k_rhs_factor_order(int64_t n, int64_t nrhs, const Wide<T>* __restrict__ b, int64_t ldb,
                                   const double* __restrict__ rs, const int32_t* __restrict__ qf,
                                   const int32_t* __restrict__ prow, T* __restrict__ bfo, int64_t ldo) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int orow = qf[prow[k]];
  const double r = rs ? rs[orow] : 1.0;
  for (int64_t c0 = (int64_t)blockIdx.y * kElemCols; c0 < nrhs; c0 += (int64_t)gridDim.y * kElemCols) {
    const int cc = (int)(nrhs - c0 < kElemCols ? nrhs - c0 : kElemCols);
    Wide<T> v[kElemCols];
#pragma unroll
    for (int j = 0; j < kElemCols; ++j)
      if (j < cc) v[j] = b[orow + (c0 + j) * ldb];
#pragma unroll
    for (int j = 0; j < kElemCols; ++j)
      if (j < cc) bfo[k + (c0 + j) * ldo] = (T)(rs ? Wide<T>(r) * v[j] : v[j]);
  }
}

// Element walk of a column-major rows x cols block by n threads with one
// division per thread instead of one per element: thread t takes row
// t % rows at columns t / rows, t / rows + n / rows, ... (threads from
// (n / rows) * rows on take none).  Requires 0 < rows <= n.
struct RowWalk {
  int r, c, dc;
  bool on;
};
__device__ __forceinline__ RowWalk row_walk(int t, int n, int rows) {
  RowWalk w;
  w.dc = n / rows;
  w.r = t % rows;
  w.c = t / rows;
  w.on = w.c < w.dc;
  return w;
}

// Pivot-row value of block position a: the scaled rhs of factor row c1 + a.
template <typename T>
__device__ __forceinline__ T rhs_value(const SolveArgs& A, int c1, int a, int64_t col) {
  return static_cast<const T*>(A.bfo)[c1 + a + col * A.ldx];
}

// Block position of V-row position r (0..nf) of a child contribution: pivot
// rows are reordered by the supernode's interchanges, update rows are not.
__device__ __forceinline__ int front_pos(const DevState& S, int c1, int np, int rel) {
  return rel < np ? S.rowfac[c1 + rel] - c1 : rel;
}

// Every solve kernel is a loop-free "item" function -- one (supernode or
// block, right-hand-side chunk) per CTA -- so that the same code runs as a
// one-launch-per-step kernel (the __global__ wrappers below) and inside the
// persistent solve kernel, which walks all steps with grid barriers between
// them.  fsol and xw are written and read by different steps of one
// persistent launch, so they are never read through the non-coherent path.

// Small supernodes, forward: one CTA per (supernode bx, 32-column chunk by).
// smem: kSmallFront * kSolveCols elements.
template <typename T>
__device__ __forceinline__ void fwd_small_item(const DevPlan& P, const DevState& S, const SolveArgs& A,
                                               const int32_t* __restrict__ tasks, const T* __restrict__ pool,
                                               T* fsol, int bx, int by, T* f) {
  const int s = tasks[bx];
  const int c0 = by * solve_cols<T>();
  const int rc = min(solve_cols<T>(), (int)(A.nrhs - c0));
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int tid = threadIdx.x;
  const int64_t R = A.nrhs;
  // every thread keeps one front row (and its columns) for the whole item
  const RowWalk mf = row_walk(tid, blockDim.x, nf);
  if (mf.on)
    for (int c = mf.c; c < rc; c += mf.dc) f[mf.r + c * nf] = mf.r < np ? rhs_value<T>(A, c1, mf.r, c0 + c) : T(0);
  __syncthreads();
  for (int ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
    const int k = P.child_idx[ci];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    if (m > 0) {
      const T* w = fsol + P.colbase[k] * R + npk;
      const RowWalk mc = row_walk(tid, blockDim.x, m);
      if (mc.on) {
        const int pos = front_pos(S, c1, np, P.rel[P.upd_off[k] + mc.r]);
        for (int c = mc.c; c < rc; c += mc.dc) f[pos + c * nf] += w[mc.r + (int64_t)(c0 + c) * nfk];
      }
    }
    __syncthreads();
  }
  const T* L = pool + P.lpan_off[s];
  for (int a = 0; a < np; ++a) {
    if (mf.on && mf.r > a) {
      const T l = L[mf.r + (int64_t)a * nf];
      for (int c = mf.c; c < rc; c += mf.dc) f[mf.r + c * nf] -= l * f[a + c * nf];
    }
    __syncthreads();
  }
  T* out = fsol + P.colbase[s] * R;
  if (mf.on)
    for (int c = mf.c; c < rc; c += mf.dc) out[mf.r + (int64_t)(c0 + c) * nf] = f[mf.r + c * nf];
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kSolveThreads) k_fwd_small(DevPlan P, DevState S, SolveArgs A,
                                                             const int32_t* __restrict__ tasks,
                                                             const T* __restrict__ pool, T* fsol) {
  __shared__ T f[kSmallFront * solve_cols<T>()];
  fwd_small_item<T>(P, S, A, tasks, pool, fsol, blockIdx.x, blockIdx.y, f);
}

// Tiny supernodes (nf <= kTinyFront), the bulk of the leaf levels: one warp
// per (supernode, 32 right-hand sides), four supernodes per CTA, no block
// barriers.  The warp loads its block cooperatively (coalesced), then each
// lane runs the substitution of its own right-hand side; the arithmetic and
// its order are those of fwd_small_item / bwd_small_item.  Shared block:
// row-major, leading dimension kTinyLd (conflict-free both ways).
constexpr int kTinyFront = 32;
constexpr int kTinyLd = 33;
constexpr int kTinyWarps = 4;
// Supernodes (warps) per tiny-supernode CTA for fronts of type T (complex
// blocks take twice the shared memory).
template <typename T>
__host__ __device__ constexpr int tiny_warps() {
  return sizeof(T) > 8 ? kTinyWarps / 2 : kTinyWarps;
}

template <typename T>
__global__ void __launch_bounds__(32 * tiny_warps<T>()) k_fwd_tiny(DevPlan P, DevState S, SolveArgs A,
                                                              const int32_t* __restrict__ tasks, int ntasks,
                                                              const T* __restrict__ pool, T* fsol) {
  __shared__ T buf[tiny_warps<T>()][kTinyFront * kTinyLd];
  const int w = warp_id(), lane = lane_id();
  const int ti = blockIdx.x * tiny_warps<T>() + w;
  if (ti >= ntasks) return;                 // warp-uniform; no block barrier below
  T* f = buf[w];
  const int s = tasks[ti];
  const int c0 = blockIdx.y * 32;
  const int rc = min(32, (int)(A.nrhs - c0));
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int64_t R = A.nrhs;
  const FastDiv dnf((uint32_t)nf);
  for (int e = lane; e < nf * rc; e += 32) {
    const int c = (int)dnf.div(e), r = e - c * nf;
    f[r * kTinyLd + c] = r < np ? rhs_value<T>(A, c1, r, c0 + c) : T(0);
  }
  __syncwarp();
  for (int ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
    const int k = P.child_idx[ci];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    if (m == 0) continue;
    const T* wv = fsol + P.colbase[k] * R + npk;
    const int32_t* rl = P.rel + P.upd_off[k];
    const FastDiv dm((uint32_t)m);
    for (int e = lane; e < m * rc; e += 32) {
      const int c = (int)dm.div(e), r = e - c * m;
      f[front_pos(S, c1, np, rl[r]) * kTinyLd + c] += wv[r + (int64_t)(c0 + c) * nfk];
    }
    __syncwarp();
  }
  if (lane < rc) {
    const T* L = pool + P.lpan_off[s];
    for (int a = 0; a < np; ++a) {
      const T fa = f[a * kTinyLd + lane];
      for (int i = a + 1; i < nf; ++i) f[i * kTinyLd + lane] -= L[i + (int64_t)a * nf] * fa;
    }
  }
  __syncwarp();
  T* out = fsol + P.colbase[s] * R;
  for (int e = lane; e < nf * rc; e += 32) {
    const int c = (int)dnf.div(e), r = e - c * nf;
    out[r + (int64_t)(c0 + c) * nf] = f[r * kTinyLd + c];
  }
}

template <typename T>
__global__ void __launch_bounds__(32 * tiny_warps<T>()) k_bwd_tiny(DevPlan P, SolveArgs A,
                                                              const int32_t* __restrict__ tasks, int ntasks,
                                                              const T* __restrict__ pool, const T* fsol, T* xw) {
  __shared__ T buf[tiny_warps<T>()][kTinyFront * kTinyLd];   // rows 0..np-1: y; np..nf-1: x of the update rows
  const int w = warp_id(), lane = lane_id();
  const int ti = blockIdx.x * tiny_warps<T>() + w;
  if (ti >= ntasks) return;
  T* f = buf[w];
  const int s = tasks[ti];
  const int c0 = blockIdx.y * 32;
  const int rc = min(32, (int)(A.nrhs - c0));
  const int np = P.np[s], nu = P.nu[s], nf = P.nf[s], c1 = P.c1[s];
  const int64_t R = A.nrhs;
  const T* fs = fsol + P.colbase[s] * R;
  const int32_t* us = P.upd + P.upd_off[s];
  const FastDiv dnp((uint32_t)np);
  for (int e = lane; e < np * rc; e += 32) {
    const int c = (int)dnp.div(e), r = e - c * np;
    f[r * kTinyLd + c] = fs[r + (int64_t)(c0 + c) * nf];
  }
  if (nu > 0) {
    const FastDiv dnu((uint32_t)nu);
    for (int e = lane; e < nu * rc; e += 32) {
      const int c = (int)dnu.div(e), t = e - c * nu;
      f[(np + t) * kTinyLd + c] = xw[us[t] + (int64_t)(c0 + c) * A.ldx];
    }
  }
  __syncwarp();
  if (lane < rc) {
    const T* U = pool + P.lpan_off[s];
    const T* U12 = pool + P.u12_off[s];
    const int ldu = u12_ld(P, s);
    for (int a = 0; a < np; ++a) {
      T acc = f[a * kTinyLd + lane];
      for (int t = 0; t < nu; ++t) acc -= U12[a + (int64_t)t * ldu] * f[(np + t) * kTinyLd + lane];
      f[a * kTinyLd + lane] = acc;
    }
    for (int a = np - 1; a >= 0; --a) {
      f[a * kTinyLd + lane] /= U[a + (int64_t)a * nf];
      const T ya = f[a * kTinyLd + lane];
      for (int i = 0; i < a; ++i) f[i * kTinyLd + lane] -= U[i + (int64_t)a * nf] * ya;
    }
  }
  __syncwarp();
  for (int e = lane; e < np * rc; e += 32) {
    const int c = (int)dnp.div(e), r = e - c * np;
    xw[c1 + r + (int64_t)(c0 + c) * A.ldx] = f[r * kTinyLd + c];
  }
}

// Leaf supernodes (no children, nf <= kLeafFront), the whole bottom tree
// level, forward: one warp per (supernode, 32 right-hand sides), one lane
// per right-hand side holding its column of the block in registers (every
// register index is a compile-time constant: the loops run to kLeafFront
// with warp-uniform guards), so there is no shared memory and no index
// arithmetic per element.  Same operations, in the same order, as
// k_fwd_tiny.  (The backward pass keeps k_bwd_tiny: its gathers of x over
// the update rows coalesce across lanes along the rows, which a lane per
// right-hand side would lose.)
constexpr int kLeafFront = 16;
constexpr int kLeafWarps = 4;

template <typename T>
__global__ void __launch_bounds__(32 * kLeafWarps) k_fwd_leaf(DevPlan P, SolveArgs A, const int32_t* __restrict__ tasks,
                                                              int ntasks, const T* __restrict__ pool, T* fsol) {
  const int ti = blockIdx.x * kLeafWarps + warp_id();
  if (ti >= ntasks) return;
  const int64_t c = (int64_t)blockIdx.y * 32 + lane_id();
  if (c >= A.nrhs) return;
  const int s = tasks[ti];
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  T f[kLeafFront];
#pragma unroll
  for (int i = 0; i < kLeafFront; ++i) f[i] = i < np ? rhs_value<T>(A, c1, i, c) : T(0);
  const T* L = pool + P.lpan_off[s];
#pragma unroll
  for (int a = 0; a < kLeafFront; ++a) {
    if (a < np) {
      const T fa = f[a];
#pragma unroll
      for (int i = a + 1; i < kLeafFront; ++i)
        if (i < nf) f[i] -= L[i + (int64_t)a * nf] * fa;
    }
  }
  T* out = fsol + P.colbase[s] * A.nrhs + c * nf;
#pragma unroll
  for (int i = 0; i < kLeafFront; ++i)
    if (i < nf) out[i] = f[i];
}

// Large supernodes: gather the rhs block, one warp per right-hand side;
// item (bx, by) covers columns by * warps .. of supernode tasks[bx] (the
// persistent solve's form; the step launches use k_fwd_assemble_rows).
template <typename T>
__device__ __forceinline__ void fwd_assemble_item(const DevPlan& P, const DevState& S, const SolveArgs& A,
                                                  const int32_t* __restrict__ tasks, T* fsol, int bx, int by) {
  const int s = tasks[bx];
  const int64_t col = (int64_t)by * (blockDim.x >> 5) + warp_id();
  if (col >= A.nrhs) return;
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int lane = lane_id();
  const int64_t R = A.nrhs;
  T* f = fsol + P.colbase[s] * R + col * nf;
  for (int r = lane; r < nf; r += 32) f[r] = r < np ? rhs_value<T>(A, c1, r, col) : T(0);
  __syncwarp();
  for (int ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
    const int k = P.child_idx[ci];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    const T* w = fsol + P.colbase[k] * R + npk + col * nfk;
    const int32_t* rl = P.rel + P.upd_off[k];
    // kU rows per lane in flight: a child's rows map to distinct front
    // rows, so the loads may all precede the stores (4-byte values: twice
    // as many, they move half the bytes per access)
    constexpr int kU = sizeof(T) == 4 ? 8 : 4;
    int r = lane;
    for (; r + 32 * (kU - 1) < m; r += 32 * kU) {
      int pos[kU];
      T v[kU], o[kU];
#pragma unroll
      for (int q = 0; q < kU; ++q) {
        pos[q] = front_pos(S, c1, np, rl[r + 32 * q]);
        v[q] = w[r + 32 * q];
      }
#pragma unroll
      for (int q = 0; q < kU; ++q) o[q] = f[pos[q]];
#pragma unroll
      for (int q = 0; q < kU; ++q) f[pos[q]] = o[q] + v[q];
    }
    for (; r < m; r += 32) f[front_pos(S, c1, np, rl[r])] += w[r];
    __syncwarp();
  }
}

// Small supernodes, backward.  smem: 2 * kSmallFront * kSolveCols elements.
template <typename T>
__device__ __forceinline__ void bwd_small_item(const DevPlan& P, const SolveArgs& A,
                                               const int32_t* __restrict__ tasks, const T* __restrict__ pool,
                                               const T* fsol, T* xw, int bx, int by, T* y) {
  T* g = y + kSmallFront * solve_cols<T>();
  const int s = tasks[bx];
  const int c0 = by * solve_cols<T>();
  const int rc = min(solve_cols<T>(), (int)(A.nrhs - c0));
  const int np = P.np[s], nu = P.nu[s], nf = P.nf[s], c1 = P.c1[s];
  const int tid = threadIdx.x;
  const int64_t R = A.nrhs;
  const T* f = fsol + P.colbase[s] * R;
  const int32_t* us = P.upd + P.upd_off[s];
  const RowWalk mp = row_walk(tid, blockDim.x, np);
  if (mp.on)
    for (int c = mp.c; c < rc; c += mp.dc) y[mp.r + c * np] = f[mp.r + (int64_t)(c0 + c) * nf];
  if (nu > 0) {
    const RowWalk mu = row_walk(tid, blockDim.x, nu);
    if (mu.on) {
      const int32_t u = us[mu.r];
      for (int c = mu.c; c < rc; c += mu.dc) g[mu.r + c * nu] = xw[u + (int64_t)(c0 + c) * A.ldx];
    }
  }
  __syncthreads();
  const T* U = pool + P.lpan_off[s];
  const T* U12 = pool + P.u12_off[s];
  const int ldu = u12_ld(P, s);
  if (mp.on)
    for (int c = mp.c; c < rc; c += mp.dc) {
      T acc = y[mp.r + c * np];
      for (int t = 0; t < nu; ++t) acc -= U12[mp.r + (int64_t)t * ldu] * g[t + c * nu];
      y[mp.r + c * np] = acc;
    }
  __syncthreads();
  for (int a = np - 1; a >= 0; --a) {
    for (int c = tid; c < rc; c += blockDim.x) y[a + c * np] /= U[a + (int64_t)a * nf];
    __syncthreads();
    if (mp.on && mp.r < a) {
      const T ua = U[mp.r + (int64_t)a * nf];
      for (int c = mp.c; c < rc; c += mp.dc) y[mp.r + c * np] -= ua * y[a + c * np];
    }
    __syncthreads();
  }
  if (mp.on)
    for (int c = mp.c; c < rc; c += mp.dc) xw[c1 + mp.r + (int64_t)(c0 + c) * A.ldx] = y[mp.r + c * np];
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kSolveThreads) k_bwd_small(DevPlan P, SolveArgs A, const int32_t* __restrict__ tasks,
                                                             const T* __restrict__ pool, const T* fsol, T* xw) {
  __shared__ T y[2 * kSmallFront * solve_cols<T>()];
  bwd_small_item<T>(P, A, tasks, pool, fsol, xw, blockIdx.x, blockIdx.y, y);
}

// Large supernodes: gather x of the update columns into the w rows (the
// persistent solve's form; the step launches use k_bwd_gather_rows).
template <typename T>
__device__ __forceinline__ void bwd_gather_item(const DevPlan& P, const SolveArgs& A,
                                                const int32_t* __restrict__ tasks, T* fsol, const T* xw, int bx,
                                                int by) {
  const int s = tasks[bx];
  const int64_t col = (int64_t)by * (blockDim.x >> 5) + warp_id();
  if (col >= A.nrhs) return;
  const int np = P.np[s], nu = P.nu[s], nf = P.nf[s];
  T* f = fsol + P.colbase[s] * A.nrhs + col * nf + np;
  const int32_t* us = P.upd + P.upd_off[s];
  // independent gathers: several in flight per lane
#pragma unroll 4
  for (int t = lane_id(); t < nu; t += 32) f[t] = xw[us[t] + col * A.ldx];
}

// Row-parallel forms of the two gathers above, for the one-launch-per-step
// solve.  The per-column warps above walk a whole front per column, which
// leaves the GPU idle at the top of the tree (one front: nrhs warps).  Here
// a CTA takes four 64-row tasks (supernode s, first row r0) and kAsmCols
// right-hand sides; each thread owns one row.
constexpr int kAsmRows = 64;
constexpr int kAsmCols = 8;

struct RowTask {
  int32_t s, r0;
  int64_t pbase;          // forward: index of the front's row 0 in the pull map's row pointers
};

// Forward assembly pulled per front row.  The pull map lists, for V-row
// position v of front s (rows aptr[pbase + v] .. aptr[pbase + v + 1] of
// asrc), the (child, update row) pairs that land on v, children in the LIFO
// order of the extend-add; the thread owning v starts from the pivot row's
// rhs (or 0) and adds them in that order, so every front row gets the same
// sum, in the same order, as fwd_assemble_item, and v -> front_pos(v) is a
// bijection: no two threads write one element.
template <typename T>
__global__ void __launch_bounds__(256) k_fwd_assemble_rows(DevPlan P, DevState S, SolveArgs A,
                                                           const RowTask* __restrict__ tasks, int ntasks,
                                                           const int64_t* __restrict__ aptr,
                                                           const int2* __restrict__ asrc, T* fsol) {
  const int ti = blockIdx.x * 4 + (threadIdx.x >> 6);
  if (ti >= ntasks) return;
  const RowTask rt = tasks[ti];
  const int s = rt.s;
  const int v = rt.r0 + (threadIdx.x & 63);
  const int nf = P.nf[s];
  if (v >= nf) return;
  const int np = P.np[s], c1 = P.c1[s];
  const int p = front_pos(S, c1, np, v);
  const int64_t R = A.nrhs;
  const int64_t c0 = (int64_t)blockIdx.y * kAsmCols;
  const int cc = (int)(R - c0 < kAsmCols ? R - c0 : kAsmCols);
  T acc[kAsmCols];
#pragma unroll
  for (int c = 0; c < kAsmCols; ++c) acc[c] = (c < cc && p < np) ? rhs_value<T>(A, c1, p, c0 + c) : T(0);
  const int64_t e1 = aptr[rt.pbase + v + 1];
  for (int64_t e = aptr[rt.pbase + v]; e < e1; ++e) {
    const int2 src = asrc[e];
    const int nfk = P.nf[src.x];
    const T* w = fsol + P.colbase[src.x] * R + P.np[src.x] + src.y + c0 * nfk;
    T t[kAsmCols];
#pragma unroll
    for (int c = 0; c < kAsmCols; ++c) t[c] = c < cc ? w[(int64_t)c * nfk] : T(0);
#pragma unroll
    for (int c = 0; c < kAsmCols; ++c) acc[c] += t[c];
  }
  T* f = fsol + P.colbase[s] * R + p + c0 * nf;
#pragma unroll
  for (int c = 0; c < kAsmCols; ++c)
    if (c < cc) f[(int64_t)c * nf] = acc[c];
}

// Backward gather, one update row per thread (tasks cover 0 .. nu).
template <typename T>
__global__ void __launch_bounds__(256) k_bwd_gather_rows(DevPlan P, SolveArgs A, const RowTask* __restrict__ tasks,
                                                         int ntasks, T* fsol, const T* xw) {
  const int ti = blockIdx.x * 4 + (threadIdx.x >> 6);
  if (ti >= ntasks) return;
  const RowTask rt = tasks[ti];
  const int s = rt.s;
  const int t = rt.r0 + (threadIdx.x & 63);
  const int nu = P.nu[s];
  if (t >= nu) return;
  const int np = P.np[s], nf = P.nf[s];
  const int64_t R = A.nrhs;
  const int64_t c0 = (int64_t)blockIdx.y * kAsmCols;
  const int cc = (int)(R - c0 < kAsmCols ? R - c0 : kAsmCols);
  const T* src = xw + P.upd[P.upd_off[s] + t] + c0 * A.ldx;
  T* f = fsol + P.colbase[s] * R + np + t + c0 * nf;
  T v[kAsmCols];
#pragma unroll
  for (int c = 0; c < kAsmCols; ++c) v[c] = c < cc ? src[(int64_t)c * A.ldx] : T(0);
#pragma unroll
  for (int c = 0; c < kAsmCols; ++c)
    if (c < cc) f[(int64_t)c * nf] = v[c];
}

// Thin large supernodes, forward (nf > kSmallFront, np <= kThinNp, nu <=
// kThinNu): most of the large fronts low in the tree have a few pivots and a
// hundred or so update rows, so their forward products y = inv(L11) f[0:np]
// and w = f[np:] - L21 y have K of a few units, and as 64 x 64 GEMM tiles
// most of every tile is idle.  One CTA per (supernode, kThinCols right-hand
// sides) forms y (into x's rows c1..) and then w in place, one update row
// per thread, in a fixed order.  (With many update rows the tiled products,
// K-chunked, keep more of the GPU busy.)
constexpr int kThinNp = 64;
constexpr int kThinNu = 192;
constexpr int kThinCols = 32;
constexpr int kThinLd = kThinCols + 1;

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_thin(DevPlan P, SolveArgs A, const int32_t* __restrict__ tasks,
                                                  const T* __restrict__ pool, T* fsol, T* xw) {
  __shared__ T ys[kThinNp * kThinLd];
  const int s = tasks[blockIdx.x];
  const int64_t R = A.nrhs, c0 = (int64_t)blockIdx.y * kThinCols;
  const int cc = (int)(R - c0 < kThinCols ? R - c0 : kThinCols);
  const int np = P.np[s], nu = P.nu[s], nf = P.nf[s], c1 = P.c1[s];
  T* f = fsol + P.colbase[s] * R + c0 * nf;
  const T* Li = pool + P.inv_off[s];
  const int tid = threadIdx.x;
  for (int e = tid; e < np * cc; e += blockDim.x) {
    const int a = e % np, c = e / np;
    const T* fc = f + (int64_t)c * nf;
    T acc = T(0);
    for (int b = 0; b < np; ++b) acc += Li[a + b * np] * fc[b];
    ys[a * kThinLd + c] = acc;
    xw[c1 + a + (c0 + c) * A.ldx] = acc;
  }
  __syncthreads();
  // 64 update rows x 4 groups of 8 columns per pass
  const T* L21 = pool + P.lpan_off[s] + np;
  const int cg = (tid >> 6) * 8;
  for (int r = tid & 63; r < nu; r += 64) {
    T acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = cg + c < cc ? f[np + r + (int64_t)(cg + c) * nf] : T(0);
    for (int a = 0; a < np; ++a) {
      const T l = L21[r + (int64_t)a * nf];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] -= l * ys[a * kThinLd + cg + c];
    }
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (cg + c < cc) f[np + r + (int64_t)(cg + c) * nf] = acc[c];
  }
}

// Split-K solve products: a product with few output tiles and a long K runs
// as K chunks -- the first in the task's own mode on C, the others as plain
// products into a scratch area -- and this kernel then folds the partial
// products into C in chunk order: C += sign * P_1, C += sign * P_2, ...
// (sign -1 for the C - A*B modes and C = -(A*B), +1 for C = A*B).  One
// thread per element of C; deterministic.
struct SplitRed {
  int64_t c, p;           // C's offset (leading dimension ldc); the partial products (m x n each, ld m)
  int32_t m, n, ldc, parts;
  int32_t sign, pad;
  int64_t elem_base;      // prefix of m * n over the step's reductions
};

template <typename T>
__global__ void __launch_bounds__(256) k_split_reduce(const SplitRed* __restrict__ reds, int nreds, int64_t total,
                                                      T* base) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  int lo = 0, hi = nreds - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (reds[mid].elem_base <= e) lo = mid;
    else hi = mid - 1;
  }
  const SplitRed rd = reds[lo];
  const int64_t l = e - rd.elem_base;
  const int64_t i = l % rd.m, j = l / rd.m;
  const int64_t mn = (int64_t)rd.m * rd.n;
  T* c = base + rd.c + i + j * rd.ldc;
  const T* p = base + rd.p + l;
  T acc = *c;
  if (rd.sign < 0)
    for (int q = 0; q < rd.parts; ++q) acc -= p[q * mn];
  else
    for (int q = 0; q < rd.parts; ++q) acc += p[q * mn];
  *c = acc;
}

// x[q[k]] = x_factor[k] (interface.jl:134-136); optionally accumulate (x += d).
template <typename T>
__global__ void k_solve_finish(int64_t n, int64_t nrhs, const int32_t* __restrict__ qf, const T* __restrict__ xw,
                               int64_t ldw, Wide<T>* __restrict__ x, int64_t ldx, int accumulate) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int q = qf[k];
  for (int64_t c0 = (int64_t)blockIdx.y * kElemCols; c0 < nrhs; c0 += (int64_t)gridDim.y * kElemCols) {
    const int cc = (int)(nrhs - c0 < kElemCols ? nrhs - c0 : kElemCols);
    Wide<T> v[kElemCols], o[kElemCols];
#pragma unroll
    for (int j = 0; j < kElemCols; ++j)
      if (j < cc) {
        v[j] = (Wide<T>)xw[k + (c0 + j) * ldw];
        o[j] = accumulate ? x[q + (c0 + j) * ldx] : Wide<T>(0.0);
      }
#pragma unroll
    for (int j = 0; j < kElemCols; ++j)
      if (j < cc) x[q + (c0 + j) * ldx] = accumulate ? o[j] + v[j] : v[j];
  }
}

// r = b - A * x with the unscaled A in CSR (interface.jl:173), FP64.
constexpr int kResidualCols = 8;
inline dim3 grid_residual(int64_t n, int64_t nrhs) {
  return grid_rows_cols(n, (nrhs + kResidualCols - 1) / kResidualCols);
}
__global__ void k_residual(int64_t n, int64_t nrhs, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const int32_t* __restrict__ src, const double* __restrict__ ax,
                           const double* __restrict__ b, int64_t ldb, const double* __restrict__ x, int64_t ldx,
                           double* __restrict__ r, int64_t ldr) {
  // kResidualCols right-hand sides per thread (blockIdx.y: groups of them):
  // the row's entries are read once for all of them; each column's sum runs
  // over the row in the same order
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p0 = rp[i], p1 = rp[i + 1];
  for (int64_t c0 = (int64_t)blockIdx.y * kResidualCols; c0 < nrhs; c0 += (int64_t)gridDim.y * kResidualCols) {
    const int cc = (int)(nrhs - c0 < kResidualCols ? nrhs - c0 : kResidualCols);
    double acc[kResidualCols];
#pragma unroll
    for (int j = 0; j < kResidualCols; ++j) acc[j] = 0.0;
    for (int p = p0; p < p1; ++p) {
      const double a = ax[src[p]];
      const double* xp = x + ci[p] + c0 * ldx;
#pragma unroll
      for (int j = 0; j < kResidualCols; ++j)
        if (j < cc) acc[j] += a * xp[j * ldx];
    }
#pragma unroll
    for (int j = 0; j < kResidualCols; ++j)
      if (j < cc) r[i + (c0 + j) * ldr] = b[i + (c0 + j) * ldb] - acc[j];
  }
}

// The same for ComplexF64 A (values interleaved re, im), b, x and r.
__global__ void k_residual_z(int64_t n, int64_t nrhs, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const int32_t* __restrict__ src, const zc* __restrict__ ax, const zc* __restrict__ b,
                             int64_t ldb, const zc* __restrict__ x, int64_t ldx, zc* __restrict__ r, int64_t ldr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int64_t c = blockIdx.y; c < nrhs; c += gridDim.y) {
    zc acc(0.0);
    for (int p = rp[i]; p < rp[i + 1]; ++p) acc += ax[src[p]] * x[ci[p] + c * ldx];
    r[i + c * ldr] = b[i + c * ldb] - acc;
  }
}

// Per-column maxima of |r|, |x|, |b| for the normwise backward error: a
// 256-row slice of one column per CTA (grid: row slices x columns), reduced
// in the CTA, then one atomic per quantity and CTA.  Non-negative doubles
// order like their bit patterns, so the maxima are atomicMax on the bits; a
// NaN anywhere in a column is kept (max_keep_nan) and makes its maximum NaN.
__global__ void __launch_bounds__(256) k_bwd_error_parts(int64_t n, int64_t nrhs, const double* __restrict__ r,
                                                         int64_t ldr, const double* __restrict__ x, int64_t ldx,
                                                         const double* __restrict__ b, int64_t ldb,
                                                         unsigned long long* __restrict__ out) {
  __shared__ double red[3][8];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t c = blockIdx.y; c < nrhs; c += gridDim.y) {
    double v[3] = {0.0, 0.0, 0.0};
    if (i < n) {
      v[0] = fabs(r[i + c * ldr]);
      v[1] = fabs(x[i + c * ldx]);
      v[2] = fabs(b[i + c * ldb]);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
      for (int o = 16; o > 0; o >>= 1) v[q] = max_keep_nan(v[q], __shfl_xor_sync(0xffffffffu, v[q], o));
    if (lane_id() == 0)
      for (int q = 0; q < 3; ++q) red[q][warp_id()] = v[q];
    __syncthreads();
    if (threadIdx.x < 3) {
      double m = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = max_keep_nan(m, red[threadIdx.x][w]);
      atomicMax(out + 3 * c + threadIdx.x, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
  }
}

// max |x_i| over n doubles into out (as bits; non-negative doubles order like
// their bit patterns): grid-stride, reduced per CTA, one atomic per CTA.  A
// NaN in x gives NaN (so a NaN factor entry reads as unbounded growth).
__global__ void __launch_bounds__(256) k_abs_max(const double* __restrict__ x, int64_t n,
                                                 unsigned long long* __restrict__ out) {
  __shared__ double red[8];
  double m = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max_keep_nan(m, fabs(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = max_keep_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane_id() == 0) red[warp_id()] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = max_keep_nan(m, red[w]);
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

// row_scaling(A, kind) (src/scaling.jl:92-115) on the device from A in CSR
// (each row's entries in increasing column order, the order in which the
// column-oriented host pass accumulates them, so the result is bitwise the
// host's): SCALE_SUM 1 / sum |a_ij|, SCALE_MAX 1 / max |a_ij|, 1 for an
// empty row or SCALE_NONE.
__global__ void k_row_scaling(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ src,
                              const double* __restrict__ ax, int kind, double* __restrict__ rs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = 0.0;
  if (kind != 0)
    for (int p = rp[i]; p < rp[i + 1]; ++p) {
      const double v = fabs(ax[src[p]]);
      acc = kind == 1 ? acc + v : (v > acc ? v : acc);
    }
  rs[i] = acc > 0 ? 1.0 / acc : 1.0;
}

// ||A||_inf = max row sum of |a_ij|.
__global__ void k_norm_inf(int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ src,
                           const double* __restrict__ ax, unsigned long long* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; ++p) acc += fabs(ax[src[p]]);
  atomicMax(out, (unsigned long long)__double_as_longlong(acc));
}

}  // namespace mfgpu
