// plan_emulator.cpp -- test infrastructure: a CPU emulation of libmfgpu's
// factorization semantics over its Plan, so that the host-side plan maps
// (merged fronts, pivot segments, assembly and CSC scatter maps) can be
// checked against the oracle without a GPU.  Per front, in postorder:
//   * assembly of the original entries (v_frow) and of the children's
//     contribution blocks (rel, last child first), as k_assemble_columns and
//     k_small_fronts do;
//   * right-looking partial-pivot LU, the pivot of column k searched in rows
//     k..seg_end-1 (k_small_fronts, k_panel);
//   * _pivot_rows (k_finalize_pivots);
//   * the CSC scatter of k_scatter_csc (one front per supernode) or of
//     k_scatter_csc_merged (merged fronts).
// Built by the tests with g++ against the library's plan.cpp and
// host/symbolic.cpp; never linked into the library.
#include <cmath>
#include <complex>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "host/symbolic.h"
#include "plan.h"

using namespace mfgpu;

namespace {

typedef std::complex<double> cplx;

template <typename T>
struct ResultT {
  std::vector<int64_t> lp, li, up, ui, p, q;
  std::vector<T> lx, ux;
  int64_t stats[6] = {0, 0, 0, 0, 0, 0};
};
ResultT<double> g_result;
ResultT<cplx> g_result_c;

// Pivot magnitude: |x|, and |re| + |im| for complex values (the rule of
// LAPACK's zgetrf, which Julia's lu! on a ComplexF64 front uses).
inline double magnitude(double v) { return std::fabs(v); }
inline double magnitude(const cplx& z) { return std::fabs(z.real()) + std::fabs(z.imag()); }

// Dense LU of every front; returns the fronts (column-major, nf x nf).
template <typename T>
std::vector<std::vector<T>> factor_fronts(const Plan& P, const T* nzval, std::vector<int32_t>& ipiv) {
  std::vector<T> vx(P.nnz_a);
  for (int64_t p = 0; p < P.nnz_a; ++p) vx[p] = nzval[P.v_src[p]];
  std::vector<std::vector<T>> F(P.ns);
  for (int64_t x = 0; x < P.ns; ++x) {
    const int nf = P.nf[x], np = P.np[x], c1 = P.c1[x];
    std::vector<T>& G = F[x];
    G.assign((size_t)nf * nf, T(0));
    auto at = [&](int r, int c) -> T& { return G[r + (size_t)c * nf]; };
    for (int c = 0; c < nf; ++c) {
      const int64_t fc = P.colbase[x] + c;
      for (int p = P.fc_vbeg[fc]; p < P.fc_vend[fc]; ++p) at(P.v_frow[p], c) = vx[p];
    }
    for (int ci = P.child_ptr[x + 1] - 1; ci >= P.child_ptr[x]; --ci) {
      const int k = P.child_idx[ci];
      const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
      const int32_t* rl = P.rel.data() + P.upd_off[k];
      for (int t = 0; t < m; ++t)
        for (int r = 0; r < m; ++r) at(rl[r], rl[t]) += F[k][npk + r + (size_t)(npk + t) * nfk];
    }
    for (int k = 0; k < np; ++k) {
      const int seg = P.seg_end[c1 + k];
      int piv = k;
      double best = -1.0;
      for (int i = k; i < seg; ++i)
        if (magnitude(at(i, k)) > best) {
          best = magnitude(at(i, k));
          piv = i;
        }
      if (piv != k)
        for (int j = 0; j < nf; ++j) std::swap(at(k, j), at(piv, j));
      ipiv[c1 + k] = piv;
      const T d = at(k, k);
      for (int i = k + 1; i < nf; ++i)
        if (i >= seg || d != T(0)) at(i, k) /= d;
      for (int j = k + 1; j < nf; ++j) {
        const T u = at(k, j);
        if (u == T(0)) continue;
        for (int i = k + 1; i < nf; ++i) at(i, j) -= at(i, k) * u;
      }
    }
  }
  return F;
}

// The same factorization executed launch by launch from the plan's launch
// list (the device's sequence): small fronts, column assembly, panels
// (speculative: no interchanges and the partial-pivoting order check;
// pivoting: rows k0..seg-1 with the interchanges applied to the whole rows),
// the panel triangular solves (L rows r0.. times inv(U_kk), inv(L_kk) times
// the U rows right of the panel) and every GEMM task C -= A B.  Returns false
// when a speculative panel met a larger candidate (the device then reruns
// with the pivoting launch list).
bool run_launches(const Plan& P, const double* nzval, std::vector<double>& pool, std::vector<int32_t>& ipiv) {
  std::vector<double> vx(P.nnz_a);
  for (int64_t p = 0; p < P.nnz_a; ++p) vx[p] = nzval[P.v_src[p]];
  pool.assign((size_t)P.front_elems, 0.0);
  bool ok = true;
  auto F = [&](int s, int r, int c) -> double& { return pool[P.front_off[s] + r + (size_t)c * P.nf[s]]; };
  auto assemble = [&](int s) {
    const int nf = P.nf[s];
    for (int c = 0; c < nf; ++c)
      for (int r = 0; r < nf; ++r) F(s, r, c) = 0.0;
    for (int c = 0; c < nf; ++c) {
      const int64_t fc = P.colbase[s] + c;
      for (int p = P.fc_vbeg[fc]; p < P.fc_vend[fc]; ++p) F(s, P.v_frow[p], c) = vx[p];
    }
    for (int ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
      const int k = P.child_idx[ci], m = P.nu[k], npk = P.np[k];
      const int32_t* rl = P.rel.data() + P.upd_off[k];
      for (int t = 0; t < m; ++t)
        for (int r = 0; r < m; ++r) F(s, rl[r], rl[t]) += F(k, npk + r, npk + t);
    }
  };
  for (const Launch& l : P.launches) {
    if (l.kind == kLaunchSmall) {
      for (int64_t i = l.first; i < l.first + l.count; ++i) {
        const int s = P.small_tasks[i], nf = P.nf[s], np = P.np[s], c1 = P.c1[s];
        assemble(s);
        for (int k = 0; k < np; ++k) {
          const int seg = P.seg_end[c1 + k];
          int piv = k;
          double best = -1.0;
          for (int i2 = k; i2 < seg; ++i2)
            if (std::fabs(F(s, i2, k)) > best) {
              best = std::fabs(F(s, i2, k));
              piv = i2;
            }
          if (piv != k)
            for (int j = 0; j < nf; ++j) std::swap(F(s, k, j), F(s, piv, j));
          ipiv[c1 + k] = piv;
          const double d = F(s, k, k);
          for (int i2 = k + 1; i2 < nf; ++i2)
            if (i2 >= seg || d != 0.0) F(s, i2, k) /= d;
          for (int j = k + 1; j < nf; ++j)
            for (int i2 = k + 1; i2 < nf; ++i2) F(s, i2, j) -= F(s, i2, k) * F(s, k, j);
        }
      }
    } else if (l.kind == kLaunchAssemble) {
      int last = -1;
      for (int64_t fc = l.first; fc < l.first + l.count; ++fc)
        if (P.fc_super[fc] != last) assemble(last = P.fc_super[fc]);
    } else if (l.kind == kLaunchPanel) {
      for (int64_t i = l.first; i < l.first + l.count; ++i) {
        const PanelTask pt = P.panel_tasks[i];
        const int s = pt.s, k0 = pt.k0, nf = P.nf[s], np = P.np[s], c1 = P.c1[s];
        const int kb = std::min(kPanel, np - k0), k1 = k0 + kb;
        const bool spec = pt.mode == kPanelSpeculative;
        const int R = spec ? kb : P.seg_end[c1 + k1 - 1] - k0;
        for (int j = k0; j < k1; ++j) {
          const int seg = std::min(k0 + R, P.seg_end[c1 + j]);
          int piv = j;
          if (!spec) {
            double best = -1.0;
            for (int i2 = j; i2 < seg; ++i2)
              if (std::fabs(F(s, i2, j)) > best) {
                best = std::fabs(F(s, i2, j));
                piv = i2;
              }
            if (piv != j)
              for (int c = 0; c < nf; ++c) std::swap(F(s, j, c), F(s, piv, c));
          } else {
            for (int i2 = j + 1; i2 < seg; ++i2)
              if (std::fabs(F(s, i2, j)) > std::fabs(F(s, j, j))) ok = false;
            if (F(s, j, j) == 0.0) ok = false;
          }
          ipiv[c1 + j] = piv;   // front-local
          const double d = F(s, j, j);
          for (int i2 = j + 1; i2 < k0 + R; ++i2)
            if (d != 0.0) F(s, i2, j) /= d;
          for (int c = j + 1; c < k1; ++c)
            for (int i2 = j + 1; i2 < k0 + R; ++i2) F(s, i2, c) -= F(s, i2, j) * F(s, j, c);
        }
      }
    } else if (l.kind == kLaunchTrsm) {
      for (int64_t i = l.first; i < l.first + l.count; ++i) {
        const TrsmTask t = P.trsm_tasks[i];
        const int s = t.s, k0 = t.k0, nf = P.nf[s], np = P.np[s], c1 = P.c1[s];
        const int kb = std::min(kPanel, np - k0), k1 = k0 + kb;
        // L rows r0..nf-1: X U_kk = A  (column by column)
        for (int r = t.r0; r < nf; ++r)
          for (int j = k0; j < k1; ++j) {
            double v = F(s, r, j);
            for (int q = k0; q < j; ++q) v -= F(s, r, q) * F(s, q, j);
            F(s, r, j) = v / F(s, j, j);
            if (t.check && r < P.seg_end[c1 + j] && std::fabs(F(s, r, j)) > 1.0) ok = false;
          }
        // U rows k0..k1-1 right of the panel: L_kk X = A (unit lower)
        for (int c = k1; c < nf; ++c)
          for (int r = k0; r < k1; ++r) {
            double v = F(s, r, c);
            for (int q = k0; q < r; ++q) v -= F(s, r, q) * F(s, q, c);
            F(s, r, c) = v;
          }
      }
    } else if (l.kind == kLaunchGemm) {
      for (int64_t i = l.first; i < l.first + l.count; ++i) {
        const GemmTask& g = P.gemm_tasks[i];
        double* A = pool.data() + g.a;
        double* B = pool.data() + g.b;
        double* C = pool.data() + g.c;
        for (int c = 0; c < g.n; ++c)
          for (int k = 0; k < g.k; ++k) {
            const double b = B[k + (int64_t)c * g.ldb];
            if (b == 0.0) continue;
            for (int r = 0; r < g.m; ++r) C[r + (int64_t)c * g.ldc] -= A[r + (int64_t)k * g.lda] * b;
          }
      }
    }
  }
  return ok;
}

}  // namespace

// Run the plan's launch list (speculative, then the pivoting rerun when a
// speculative panel fails, as the device does) and return the maximum
// difference of every front against the dense emulation above, relative to
// the front's largest entry; ipiv must agree exactly (out[1] = mismatches,
// out[2] = 1 if the pivoting rerun ran, out[3] = GEMM launches).
extern "C" int emu_check_launches(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                                  const int64_t* q, int merge, double* out) {
  const SymbolicMF S = symbolic_mf(n, colptr, rowval, q);
  Plan P;
  if (merge)
    build_plan_merged(n, colptr, rowval, S.qf.data(), S.parent.data(), S.nsuper(), S.sstart.data(),
                      S.upd_ptr.data(), S.upd_idx.data(), P, kMergeMaxPivots);
  else
    build_plan(n, colptr, rowval, S.qf.data(), S.parent.data(), S.nsuper(), S.sstart.data(), S.upd_ptr.data(),
               S.upd_idx.data(), P);
  std::vector<int32_t> ipiv_ref(n), ipiv(n);
  const std::vector<std::vector<double>> F = factor_fronts(P, nzval, ipiv_ref);
  std::vector<double> pool;
  bool reran = false;
  if (!run_launches(P, nzval, pool, ipiv)) {
    build_launches(P, true);
    reran = true;
    run_launches(P, nzval, pool, ipiv);
  }
  double worst = 0;
  for (int64_t x = 0; x < P.ns; ++x) {
    const int nf = P.nf[x];
    double mx = 0, d = 0;
    for (int64_t e = 0; e < (int64_t)nf * nf; ++e) {
      mx = std::max(mx, std::fabs(F[x][e]));
      d = std::max(d, std::fabs(F[x][e] - pool[P.front_off[x] + e]));
    }
    if (mx > 0) worst = std::max(worst, d / mx);
  }
  int64_t mism = 0;
  for (int64_t j = 0; j < n; ++j) mism += ipiv[j] != ipiv_ref[j];
  int64_t ng = 0;
  for (const Launch& l : P.launches) ng += l.kind == kLaunchGemm;
  out[0] = worst;
  out[1] = (double)mism;
  out[2] = reran ? 1.0 : 0.0;
  out[3] = (double)ng;
  return 0;
}

// Factor A (0-based CSC pattern, values) with symbolic_mf(A; q) (q 0-based
// or null for AMD), merged fronts or one front per supernode.  stats: nnz_l,
// nnz_u, fronts, original supernodes, max front, max pivots.
namespace {
template <typename T>
void emulate(int64_t n, const int64_t* colptr, const int64_t* rowval, const T* nzval, const int64_t* q, int merge,
             int64_t* stats, ResultT<T>& R) {
  const SymbolicMF S = symbolic_mf(n, colptr, rowval, q);
  Plan P;
  if (merge)
    build_plan_merged(n, colptr, rowval, S.qf.data(), S.parent.data(), S.nsuper(), S.sstart.data(),
                      S.upd_ptr.data(), S.upd_idx.data(), P, kMergeMaxPivots);
  else
    build_plan(n, colptr, rowval, S.qf.data(), S.parent.data(), S.nsuper(), S.sstart.data(), S.upd_ptr.data(),
               S.upd_idx.data(), P);
  std::vector<int32_t> ipiv(n);
  const std::vector<std::vector<T>> F = factor_fronts(P, nzval, ipiv);

  std::vector<int32_t> prow(n), rowfac(n);
  for (int64_t x = 0; x < P.ns; ++x) {
    const int c1 = P.c1[x], np = P.np[x];
    for (int a = 0; a < np; ++a) prow[c1 + a] = c1 + a;
    for (int a = 0; a < np; ++a)
      if (ipiv[c1 + a] != a) std::swap(prow[c1 + a], prow[c1 + ipiv[c1 + a]]);
    for (int a = 0; a < np; ++a) rowfac[prow[c1 + a]] = c1 + a;
  }

  R.lp.assign(P.lcolptr.begin(), P.lcolptr.end());
  R.up.assign(P.ucolptr.begin(), P.ucolptr.end());
  R.li.assign(P.nnz_l, -1);
  R.lx.assign(P.nnz_l, T(NAN));
  R.ui.assign(P.nnz_u, -1);
  R.ux.assign(P.nnz_u, T(NAN));
  auto put_l = [&](int64_t at, int64_t row, T v) {
    R.li[at] = 1 + row;
    R.lx[at] = v;
  };
  auto put_u = [&](int64_t at, int64_t row, T v) {
    R.ui[at] = 1 + row;
    R.ux[at] = v;
  };
  for (int64_t fc = 0; fc < P.fc_total; ++fc) {
    const int x = P.fc_super[fc];
    const int c = (int)(fc - P.colbase[x]);
    const int np = P.np[x], nf = P.nf[x], c1 = P.c1[x];
    const T* col = F[x].data() + (size_t)c * nf;   // L column, or U12 rows 0..np-1
    if (P.merged) {
      if (c < np) {
        const int j = c1 + c, s = P.col_orig[j];
        const int a0 = P.o_c1[s] - c1, a1 = a0 + P.o_np[s];
        const int64_t lb = P.lcolptr[j];
        for (int r = 0; r < a1 - c; ++r) put_l(lb + r, c1 + c + r, r == 0 ? T(1) : col[c + r]);
        const int64_t ob = P.o_upd_off[s], on = P.o_upd_off[s + 1] - ob, lu = lb + (a1 - c);
        for (int64_t i = 0; i < on; ++i) {
          const int u = P.o_upd[ob + i], rf = rowfac[u];
          put_l(lu + i, rf, col[u < c1 + np ? rf - c1 : P.o_xpos[ob + i]]);
        }
        const int64_t ub = P.ucolptr[j + 1] - (c - a0 + 1);
        for (int b = 0; b <= c - a0; ++b) put_u(ub + b, c1 + a0 + b, col[a0 + b]);
      }
      for (int64_t e = P.fcu_ptr[fc]; e < P.fcu_ptr[fc + 1]; ++e) {
        const UBlock blk = P.fcu[e];
        for (int b = 0; b < blk.rows; ++b) put_u(blk.uoff + b, c1 + blk.row0 + b, col[blk.row0 + b]);
      }
    } else {
      const int32_t* us = P.upd.data() + P.upd_off[x];
      if (c < np) {
        const int64_t lb = P.lcolptr[c1 + c];
        for (int r = 0; r < nf - c; ++r) {
          const int fr = c + r;
          put_l(lb + r, fr < np ? c1 + fr : rowfac[us[fr - np]], r == 0 ? T(1) : col[fr]);
        }
        const int64_t ub = P.ucolptr[c1 + c + 1] - (c + 1);
        for (int b = 0; b <= c; ++b) put_u(ub + b, c1 + b, col[b]);
      } else {
        const int64_t ub = P.uoff[P.upd_off[x] + (c - np)];
        for (int a = 0; a < np; ++a) put_u(ub + a, c1 + a, col[a]);
      }
    }
  }
  R.p.resize(n);
  R.q.resize(n);
  for (int64_t k = 0; k < n; ++k) {
    R.p[k] = P.qf[prow[k]] + 1;   // p = qf[prow] (src/multifrontal.jl:355-356)
    R.q[k] = P.qf[k] + 1;
  }
  const int64_t st[6] = {P.nnz_l, P.nnz_u, P.ns, P.merged ? P.ns_orig : P.ns, P.max_nf, P.max_np};
  std::memcpy(R.stats, st, sizeof st);
  std::memcpy(stats, st, sizeof st);
}
}  // namespace

extern "C" int emu_factor(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                          const int64_t* q, int merge, int64_t* stats) {
  emulate<double>(n, colptr, rowval, nzval, q, merge, stats, g_result);
  return 0;
}

// The same for a ComplexF64 matrix, values as interleaved (re, im) doubles.
extern "C" int emu_factor_c64(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval_ri,
                              const int64_t* q, int merge, int64_t* stats) {
  std::vector<cplx> z(colptr[n]);
  for (int64_t k = 0; k < colptr[n]; ++k) z[k] = cplx(nzval_ri[2 * k], nzval_ri[2 * k + 1]);
  emulate<cplx>(n, colptr, rowval, z.data(), q, merge, stats, g_result_c);
  return 0;
}

// The last ComplexF64 factorization, 1-based, values as (re, im) pairs.
extern "C" void emu_get_c64(int64_t* lp, int64_t* li, double* lx_ri, int64_t* up, int64_t* ui, double* ux_ri,
                            int64_t* p, int64_t* q) {
  const ResultT<cplx>& R = g_result_c;
  for (size_t k = 0; k < R.lp.size(); ++k) {
    lp[k] = R.lp[k] + 1;
    up[k] = R.up[k] + 1;
  }
  std::memcpy(li, R.li.data(), R.li.size() * 8);
  std::memcpy(ui, R.ui.data(), R.ui.size() * 8);
  std::memcpy(lx_ri, R.lx.data(), R.lx.size() * 16);   // std::complex<double>: (re, im)
  std::memcpy(ux_ri, R.ux.data(), R.ux.size() * 16);
  std::memcpy(p, R.p.data(), R.p.size() * 8);
  std::memcpy(q, R.q.data(), R.q.size() * 8);
}

// The last factorization, 1-based as the library returns it.
extern "C" void emu_get(int64_t* lp, int64_t* li, double* lx, int64_t* up, int64_t* ui, double* ux, int64_t* p,
                        int64_t* q) {
  const ResultT<double>& R = g_result;
  for (size_t k = 0; k < R.lp.size(); ++k) {
    lp[k] = R.lp[k] + 1;
    up[k] = R.up[k] + 1;
  }
  std::memcpy(li, R.li.data(), R.li.size() * 8);
  std::memcpy(lx, R.lx.data(), R.lx.size() * 8);
  std::memcpy(ui, R.ui.data(), R.ui.size() * 8);
  std::memcpy(ux, R.ux.data(), R.ux.size() * 8);
  std::memcpy(p, R.p.data(), R.p.size() * 8);
  std::memcpy(q, R.q.data(), R.q.size() * 8);
}

// Build a plan from a caller's symbolic arrays (0-based), merged fronts or
// one front per supernode, as mfgpu_analyze does before anything reaches the
// device.  Returns 0 when the plan builds, 1 when the arrays are rejected as
// invalid (message in msg), 2 on any other exception.
extern "C" int emu_build_plan(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                              const int64_t* parent, int64_t ns, const int64_t* sstart, const int64_t* upd_ptr,
                              const int64_t* upd_idx, int merge, char* msg, int64_t cap) {
  auto say = [&](const char* what) {
    if (cap > 0) {
      std::strncpy(msg, what, (size_t)cap - 1);
      msg[cap - 1] = 0;
    }
  };
  try {
    Plan P;
    if (merge)
      build_plan_merged(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, P, kMergeMaxPivots);
    else
      build_plan(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, P);
    say("");
    return 0;
  } catch (const std::invalid_argument& e) {
    say(e.what());
    return 1;
  } catch (const std::exception& e) {
    say(e.what());
    return 2;
  }
}

namespace {
uint64_t fnv(const void* p, size_t n, uint64_t h) {
  const unsigned char* c = (const unsigned char*)p;
  for (size_t i = 0; i < n; ++i) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}
template <typename T>
uint64_t hash_vec(const std::vector<T>& v) {   // element types without padding
  return fnv(v.data(), v.size() * sizeof(T), 1469598103934665603ull ^ v.size());
}
uint64_t hash_gemms(const std::vector<GemmTask>& v) {   // field by field (GemmTask has padding)
  uint64_t h = 1469598103934665603ull ^ v.size();
  for (const GemmTask& g : v) {
    const int64_t a[] = {g.a, g.b, g.c, g.m, g.n, g.k, g.lda, g.ldb, g.ldc, g.tiles_m, g.tiles_n, g.mode,
                         g.tile_base, g.d, g.ldd, g.pad};
    h = fnv(a, sizeof a, h);
  }
  return h;
}
uint64_t hash_launches(const std::vector<Launch>& v) {
  uint64_t h = 1469598103934665603ull ^ v.size();
  for (const Launch& l : v) {
    const int64_t a[] = {l.kind, l.level, l.first, l.count, l.tiles, l.tiles_tc, l.rows};
    const double d[] = {l.flops, l.elems, l.extra_bytes};
    h = fnv(a, sizeof a, h);
    h = fnv(d, sizeof d, h);
  }
  return h;
}
std::string g_digest;
}  // namespace

// A digest of every field of the plan built from a caller's symbolic arrays
// (0-based), "name=hash;" per field: two plans are equal field by field when
// their digests are.
extern "C" const char* emu_plan_digest(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                                       const int64_t* parent, int64_t ns, const int64_t* sstart,
                                       const int64_t* upd_ptr, const int64_t* upd_idx, int merge) {
  Plan P;
  try {
    if (merge)
      build_plan_merged(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, P, kMergeMaxPivots);
    else
      build_plan(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, P);
  } catch (const std::exception& e) {
    g_digest = std::string("error=") + e.what() + ";";
    return g_digest.c_str();
  }
  std::string s;
  auto put = [&](const char* name, uint64_t h) { s += std::string(name) + "=" + std::to_string(h) + ";"; };
  auto num = [&](const char* name, double v) { put(name, fnv(&v, sizeof v, 0)); };
#define VEC(f) put(#f, hash_vec(P.f))
#define NUM(f) num(#f, (double)P.f)
  NUM(n); NUM(ns); NUM(nnz_a); VEC(c1); VEC(np); VEC(nu); VEC(nf); VEC(height); VEC(slot); VEC(upd_off);
  VEC(front_off); VEC(colbase); VEC(child_ptr); VEC(child_idx); VEC(parent_super); VEC(upd); VEC(rel); VEC(uoff);
  VEC(v_src); VEC(v_srow); VEC(v_frow); VEC(fc_super); VEC(fc_vbeg); VEC(fc_vend); VEC(fc_ch_ptr); VEC(fc_ch);
  NUM(fc_total); NUM(front_elems); NUM(front_elems_full); NUM(pool_elems); NUM(lean); VEC(lpan_off); VEC(u12_off);
  NUM(panel_base); NUM(panel_elems); NUM(nlevels); VEC(slot_super); VEC(level_slot); VEC(level_large);
  VEC(lcolptr); VEC(ucolptr); NUM(nnz_l); NUM(nnz_u); VEC(qf); VEC(csr_ptr); VEC(csr_col); VEC(csr_src);
  VEC(dinv_off); NUM(dinv_blocks); VEC(inv_off); NUM(inv_base); NUM(inv_elems); NUM(inv_scratch);
  NUM(inv_scratch_elems); VEC(inv_blocks); VEC(inv_steps); NUM(flops_inverse); VEC(small_tasks); VEC(panel_tasks);
  VEC(trsm_tasks); NUM(has_speculative); NUM(merged); NUM(ns_orig); VEC(seg_end); VEC(col_orig); VEC(o_c1);
  VEC(o_np); VEC(o_upd_off); VEC(o_upd); VEC(o_xpos); VEC(fcu_ptr); VEC(fcu); NUM(flops_orig); VEC(front_nv);
  NUM(flops); NUM(flops_getrf); NUM(flops_trsm); NUM(flops_gemm); NUM(assembly_bytes_per_elem); NUM(max_nf);
  NUM(max_np);
#undef VEC
#undef NUM
  put("inv_tasks", hash_gemms(P.inv_tasks));
  put("inv_tasks_tc", hash_gemms(P.inv_tasks_tc));
  put("gemm_tasks", hash_gemms(P.gemm_tasks));
  put("gemm_tasks_tc", hash_gemms(P.gemm_tasks_tc));
  put("launches", hash_launches(P.launches));
  g_digest = s;
  return g_digest.c_str();
}
