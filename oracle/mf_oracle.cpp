// mf_oracle.cpp -- CPU oracle for the multifrontal LU path of PureUMFPACK.jl.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: tests, the smoke check
// and the CPU-baseline leg of the benchmark call it to produce the reference
// answer.  The shipped library (libmfgpu.so) never links, loads or calls it.
//
// It restates, step for step, the reference's Julia algorithm:
//   row scaling            src/scaling.jl:92-126
//   AMD / COLAMD ordering  src/amd.jl:13-539   (CSparse cs_amd, order=1)
//   symbolic analysis      src/symbolic.jl:15-237
//   numeric multifrontal   src/multifrontal.jl:45-375
//   Gilbert-Peierls LU     src/gplu.jl:62-303 (the method splu uses by default),
//                          Float64, Float32 and ComplexF64
//   CSC triangular solves  src/solve.jl:10-39
//   solve + refinement     src/interface.jl:123-177
// The dense front kernels (getrf / trsm / gemm) are the same LAPACK/BLAS calls
// the reference makes through Julia's LinearAlgebra (multifrontal.jl:248,265,
// 266,268).  They are taken from numpy's bundled ILP64 OpenBLAS, loaded with
// dlopen at run time (orc_set_blas), so pivot choices follow LAPACK's partial
// pivoting exactly as Julia's OpenBLAS does.
//
// Index convention on the C ABI: 1-based int64, as SparseMatrixCSC{Float64,Int64}.
// Internally everything is 0-based.

#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

typedef int64_t i64;
using std::vector;

// ---------------------------------------------------------------------------
// BLAS / LAPACK (ILP64 Fortran interface of numpy's OpenBLAS)
// ---------------------------------------------------------------------------
typedef void (*dgetrf_fn)(const i64*, const i64*, double*, const i64*, i64*, i64*);
typedef void (*dtrsm_fn)(const char*, const char*, const char*, const char*, const i64*,
                         const i64*, const double*, const double*, const i64*, double*,
                         const i64*, size_t, size_t, size_t, size_t);
typedef void (*dgemm_fn)(const char*, const char*, const i64*, const i64*, const i64*,
                         const double*, const double*, const i64*, const double*, const i64*,
                         const double*, double*, const i64*, size_t, size_t);
// single-precision variants (Float32 factorizations)
typedef void (*sgetrf_fn)(const i64*, const i64*, float*, const i64*, i64*, i64*);
typedef void (*strsm_fn)(const char*, const char*, const char*, const char*, const i64*,
                         const i64*, const float*, const float*, const i64*, float*,
                         const i64*, size_t, size_t, size_t, size_t);
typedef void (*sgemm_fn)(const char*, const char*, const i64*, const i64*, const i64*,
                         const float*, const float*, const i64*, const float*, const i64*,
                         const float*, float*, const i64*, size_t, size_t);
// double-complex variants (ComplexF64 factorizations); Fortran COMPLEX*16 has
// std::complex<double>'s layout
typedef std::complex<double> cplx;
typedef void (*zgetrf_fn)(const i64*, const i64*, cplx*, const i64*, i64*, i64*);
typedef void (*ztrsm_fn)(const char*, const char*, const char*, const char*, const i64*,
                         const i64*, const cplx*, const cplx*, const i64*, cplx*,
                         const i64*, size_t, size_t, size_t, size_t);
typedef void (*zgemm_fn)(const char*, const char*, const i64*, const i64*, const i64*,
                         const cplx*, const cplx*, const i64*, const cplx*, const i64*,
                         const cplx*, cplx*, const i64*, size_t, size_t);
typedef void (*setthreads_fn)(int);
typedef int (*getthreads_fn)(void);

static dgetrf_fn g_dgetrf = nullptr;
static dtrsm_fn g_dtrsm = nullptr;
static dgemm_fn g_dgemm = nullptr;
static sgetrf_fn g_sgetrf = nullptr;
static strsm_fn g_strsm = nullptr;
static sgemm_fn g_sgemm = nullptr;
static zgetrf_fn g_zgetrf = nullptr;
static ztrsm_fn g_ztrsm = nullptr;
static zgemm_fn g_zgemm = nullptr;
static setthreads_fn g_setthreads = nullptr;
static getthreads_fn g_getthreads = nullptr;
static std::string g_err;

namespace {

// ---------------------------------------------------------------------------
// CSC helpers (0-based)
// ---------------------------------------------------------------------------
struct Pattern {           // CSC pattern with sorted rows
  i64 n = 0;
  vector<i64> cp;          // n+1
  vector<i64> ri;
};

// Transpose of a CSC pattern (m rows, n cols) -> (n rows, m cols); rows come
// out sorted because columns are visited in order (counting sort).
Pattern transpose_pattern(i64 m, i64 n, const i64* cp, const i64* ri) {
  Pattern t;
  t.n = m;
  t.cp.assign(m + 1, 0);
  i64 nz = cp[n];
  t.ri.resize(nz);
  for (i64 p = 0; p < nz; ++p) t.cp[ri[p] + 1]++;
  for (i64 i = 0; i < m; ++i) t.cp[i + 1] += t.cp[i];
  vector<i64> cur(t.cp.begin(), t.cp.end() - 1);
  for (i64 j = 0; j < n; ++j)
    for (i64 p = cp[j]; p < cp[j + 1]; ++p) t.ri[cur[ri[p]]++] = j;
  return t;
}

// Pattern of A + A^T with sorted rows (sparse add of two sorted CSC), diagonal
// kept or dropped.  Mirrors `Pat + copy(transpose(Pat))` (amd.jl:84-87,
// symbolic.jl:16-17) followed by the diagonal drop.
Pattern sym_pattern(i64 n, const i64* cp, const i64* ri, bool drop_diag) {
  Pattern t = transpose_pattern(n, n, cp, ri);
  Pattern s;
  s.n = n;
  s.cp.assign(n + 1, 0);
  s.ri.reserve(2 * cp[n]);
  for (i64 j = 0; j < n; ++j) {
    i64 a = cp[j], ae = cp[j + 1], b = t.cp[j], be = t.cp[j + 1];
    while (a < ae || b < be) {
      i64 r;
      if (b >= be || (a < ae && ri[a] < t.ri[b])) {
        r = ri[a++];
      } else if (a >= ae || t.ri[b] < ri[a]) {
        r = t.ri[b++];
      } else {
        r = ri[a];
        ++a;
        ++b;
      }
      if (!(drop_diag && r == j)) s.ri.push_back(r);
    }
    s.cp[j + 1] = (i64)s.ri.size();
  }
  return s;
}

// Symmetric permutation of a symmetric pattern: new column j = old column
// perm[j], rows relabelled through inv(perm) and re-sorted.
// Restates _permute_sym_csc1 (symbolic.jl:40-63).
Pattern permute_sym(const Pattern& a, const vector<i64>& perm) {
  i64 n = a.n;
  vector<i64> pinv(n);
  for (i64 k = 0; k < n; ++k) pinv[perm[k]] = k;
  Pattern b;
  b.n = n;
  b.cp.assign(n + 1, 0);
  for (i64 j = 0; j < n; ++j) b.cp[j + 1] = b.cp[j] + (a.cp[perm[j] + 1] - a.cp[perm[j]]);
  b.ri.resize(b.cp[n]);
  for (i64 j = 0; j < n; ++j) {
    i64 oj = perm[j], dst = b.cp[j];
    for (i64 p = a.cp[oj]; p < a.cp[oj + 1]; ++p) b.ri[dst++] = pinv[a.ri[p]];
    std::sort(b.ri.begin() + b.cp[j], b.ri.begin() + b.cp[j + 1]);
  }
  return b;
}

// ---------------------------------------------------------------------------
// AMD  (amd.jl:191-539; CSparse cs_amd with order = 1)
// ---------------------------------------------------------------------------
inline i64 flip(i64 x) { return -x - 2; }

i64 wclear(i64 mark, i64 lemax, i64* w, i64 n) {   // amd.jl:17-25
  if (mark < 2 || mark + lemax < 0) {
    for (i64 k = 0; k < n; ++k)
      if (w[k] != 0) w[k] = 1;
    mark = 2;
  }
  return mark;
}

i64 tdfs(i64 j, i64 k, i64* head, const i64* next, i64* post, i64* stack) {  // amd.jl:28-48
  i64 top = 0;
  stack[0] = j;
  while (top >= 0) {
    i64 p = stack[top];
    i64 i = head[p];
    if (i == -1) {
      --top;
      post[k++] = p;
    } else {
      head[p] = next[i];
      stack[++top] = i;
    }
  }
  return k;
}

// cp: n+1 column pointers (0-based), ci: row indices (diagonal dropped,
// sorted).  Returns the 0-based permutation.
vector<i64> amd_core(i64 n, const vector<i64>& cp, const vector<i64>& ci0, double dense) {
  i64 cnz = cp[n];
  i64 t = cnz + cnz / 5 + 2 * n;
  vector<i64> Ci(std::max<i64>(t, 1));
  std::copy(ci0.begin(), ci0.begin() + cnz, Ci.begin());
  double dthresh = std::max(16.0, dense * std::sqrt((double)n));
  i64 densethr = std::min<i64>(n - 2, (i64)std::floor(dthresh));

  vector<i64> len(n + 1), nv(n + 1), next(n + 1), head(n + 1), elen(n + 1), degree(n + 1),
      w(n + 1), hhead(n + 1), last(n + 1), P(n + 1), Cp(n + 1);
  for (i64 k = 0; k < n; ++k) {
    len[k] = cp[k + 1] - cp[k];
    Cp[k] = cp[k];
  }
  Cp[n] = cp[n];
  len[n] = 0;
  i64 nzmax = (i64)Ci.size();
  for (i64 i = 0; i <= n; ++i) {
    head[i] = -1;
    last[i] = -1;
    next[i] = -1;
    hhead[i] = -1;
    nv[i] = 1;
    w[i] = 1;
    elen[i] = 0;
    degree[i] = len[i];
  }
  i64 mark = wclear(0, 0, w.data(), n);
  elen[n] = -2;
  Cp[n] = -1;
  w[n] = 0;

  i64 nel = 0;
  for (i64 i = 0; i < n; ++i) {     // initialize degree lists (amd.jl:240-260)
    i64 d = degree[i];
    if (d == 0) {
      elen[i] = -2;
      ++nel;
      Cp[i] = -1;
      w[i] = 0;
    } else if (d > densethr) {
      nv[i] = 0;
      elen[i] = -1;
      ++nel;
      Cp[i] = flip(n);
      nv[n]++;
    } else {
      if (head[d] != -1) last[head[d]] = i;
      next[i] = head[d];
      head[d] = i;
    }
  }

  i64 mindeg = 0, lemax = 0;
  while (nel < n) {
    // select node of minimum approximate degree (amd.jl:267-281)
    i64 k = -1;
    for (; mindeg < n; ++mindeg) {
      k = head[mindeg];
      if (k != -1) break;
    }
    if (next[k] != -1) last[next[k]] = -1;
    head[mindeg] = next[k];
    i64 elenk = elen[k], nvk = nv[k];
    nel += nvk;

    // garbage collection (amd.jl:283-308)
    if (elenk > 0 && cnz + mindeg >= nzmax) {
      for (i64 j = 0; j < n; ++j) {
        i64 p = Cp[j];
        if (p >= 0) {
          Cp[j] = Ci[p];
          Ci[p] = flip(j);
        }
      }
      i64 q = 0, p = 0;
      while (p < cnz) {
        i64 j = flip(Ci[p++]);
        if (j >= 0) {
          Ci[q] = Cp[j];
          Cp[j] = q++;
          for (i64 k3 = 0; k3 < len[j] - 1; ++k3) Ci[q++] = Ci[p++];
        }
      }
      cnz = q;
    }

    // construct new element (amd.jl:311-356)
    i64 dk = 0;
    nv[k] = -nvk;
    i64 p = Cp[k];
    i64 pk1 = (elenk == 0) ? p : cnz;
    i64 pk2 = pk1;
    for (i64 k1 = 1; k1 <= elenk + 1; ++k1) {
      i64 e, pj, ln;
      if (k1 > elenk) {
        e = k;
        pj = p;
        ln = len[k] - elenk;
      } else {
        e = Ci[p++];
        pj = Cp[e];
        ln = len[e];
      }
      for (i64 k2 = 1; k2 <= ln; ++k2) {
        i64 i = Ci[pj++];
        i64 nvi = nv[i];
        if (nvi <= 0) continue;
        dk += nvi;
        nv[i] = -nvi;
        Ci[pk2++] = i;
        if (next[i] != -1) last[next[i]] = last[i];
        if (last[i] != -1)
          next[last[i]] = next[i];
        else
          head[degree[i]] = next[i];
      }
      if (e != k) {
        Cp[e] = flip(k);
        w[e] = 0;
      }
    }
    if (elenk != 0) cnz = pk2;
    degree[k] = dk;
    Cp[k] = pk1;
    len[k] = pk2 - pk1;
    elen[k] = -2;

    // set differences (amd.jl:359-374)
    mark = wclear(mark, lemax, w.data(), n);
    for (i64 pk = pk1; pk < pk2; ++pk) {
      i64 i = Ci[pk];
      i64 eln = elen[i];
      if (eln <= 0) continue;
      i64 nvi = -nv[i];
      i64 wnvi = mark - nvi;
      for (i64 p2 = Cp[i]; p2 <= Cp[i] + eln - 1; ++p2) {
        i64 e = Ci[p2];
        if (w[e] >= mark)
          w[e] -= nvi;
        else if (w[e] != 0)
          w[e] = degree[e] + wnvi;
      }
    }

    // degree update (amd.jl:377-432)
    for (i64 pk = pk1; pk < pk2; ++pk) {
      i64 i = Ci[pk];
      i64 p1 = Cp[i];
      i64 p2 = p1 + elen[i] - 1;
      i64 pn = p1;
      i64 h = 0, d = 0;
      for (i64 p3 = p1; p3 <= p2; ++p3) {
        i64 e = Ci[p3];
        if (w[e] != 0) {
          i64 dext = w[e] - mark;
          if (dext > 0) {
            d += dext;
            Ci[pn++] = e;
            h += e;
          } else {
            Cp[e] = flip(k);
            w[e] = 0;
          }
        }
      }
      elen[i] = pn - p1 + 1;
      i64 p3 = pn;
      i64 p4 = p1 + len[i];
      for (i64 p5 = p2 + 1; p5 < p4; ++p5) {
        i64 j = Ci[p5];
        i64 nvj = nv[j];
        if (nvj <= 0) continue;
        d += nvj;
        Ci[pn++] = j;
        h += j;
      }
      if (d == 0) {
        Cp[i] = flip(k);
        i64 nvi = -nv[i];
        dk -= nvi;
        nvk += nvi;
        nel += nvi;
        nv[i] = 0;
        elen[i] = -1;
      } else {
        degree[i] = std::min(degree[i], d);
        Ci[pn] = Ci[p3];
        Ci[p3] = Ci[p1];
        Ci[p1] = k;
        len[i] = pn - p1 + 1;
        h = h % n;
        next[i] = hhead[h];
        hhead[h] = i;
        last[i] = h;
      }
    }
    degree[k] = dk;
    lemax = std::max(lemax, dk);
    mark = wclear(mark + lemax, lemax, w.data(), n);

    // supervariable detection (amd.jl:438-474)
    for (i64 pk = pk1; pk < pk2; ++pk) {
      i64 i = Ci[pk];
      if (nv[i] >= 0) continue;
      i64 h = last[i];
      i = hhead[h];
      hhead[h] = -1;
      while (i != -1 && next[i] != -1) {
        i64 ln = len[i], eln = elen[i];
        for (i64 pp = Cp[i] + 1; pp <= Cp[i] + ln - 1; ++pp) w[Ci[pp]] = mark;
        i64 jlast = i;
        i64 j = next[i];
        while (j != -1) {
          bool ok = (len[j] == ln) && (elen[j] == eln);
          for (i64 pp = Cp[j] + 1; ok && pp <= Cp[j] + ln - 1; ++pp)
            if (w[Ci[pp]] != mark) ok = false;
          if (ok) {
            Cp[j] = flip(i);
            nv[i] += nv[j];
            nv[j] = 0;
            elen[j] = -1;
            j = next[j];
            next[jlast] = j;
          } else {
            jlast = j;
            j = next[j];
          }
        }
        i = next[i];
        ++mark;
      }
    }

    // finalize new element (amd.jl:477-504)
    p = pk1;
    for (i64 pk = pk1; pk < pk2; ++pk) {
      i64 i = Ci[pk];
      i64 nvi = -nv[i];
      if (nvi <= 0) continue;
      nv[i] = nvi;
      i64 d = degree[i] + dk - nvi;
      d = std::min(d, n - nel - nvi);
      if (head[d] != -1) last[head[d]] = i;
      next[i] = head[d];
      last[i] = -1;
      head[d] = i;
      mindeg = std::min(mindeg, d);
      degree[i] = d;
      Ci[p++] = i;
    }
    nv[k] = nvk;
    len[k] = p - pk1;
    if (len[k] == 0) {
      Cp[k] = -1;
      w[k] = 0;
    }
    if (elenk != 0) cnz = p;
  }

  // postorder the assembly tree (amd.jl:508-531)
  for (i64 i = 0; i < n; ++i) Cp[i] = flip(Cp[i]);
  for (i64 j = 0; j <= n; ++j) head[j] = -1;
  for (i64 j = n; j >= 0; --j) {
    if (nv[j] > 0) continue;
    next[j] = head[Cp[j]];
    head[Cp[j]] = j;
  }
  for (i64 e = n; e >= 0; --e) {
    if (nv[e] <= 0) continue;
    if (Cp[e] != -1) {
      next[e] = head[Cp[e]];
      head[Cp[e]] = e;
    }
  }
  i64 k = 0;
  for (i64 i = 0; i <= n; ++i)
    if (Cp[i] == -1) k = tdfs(i, k, head.data(), next.data(), P.data(), w.data());
  return vector<i64>(P.begin(), P.begin() + n);
}

vector<i64> amd_order_sym0(i64 n, const i64* cp, const i64* ri, double dense) {  // amd.jl:141-148
  if (n == 0) return {};
  if (n == 1) return {0};
  Pattern s = sym_pattern(n, cp, ri, true);
  return amd_core(n, s.cp, s.ri, dense);
}

// COLAMD = AMD on the pattern of A^T A with dense rows of A dropped
// (amd.jl:91-104, 183-188).  m = number of rows of A.
vector<i64> colamd_order0(i64 m, i64 n, const i64* cp, const i64* ri, double dense) {
  vector<i64> id(n);
  if (n <= 1) {
    for (i64 j = 0; j < n; ++j) id[j] = j;
    return id;
  }
  Pattern at = transpose_pattern(m, n, cp, ri);   // column i of AT = row i of A
  i64 densethr = (i64)std::floor(std::min((double)(n - 2), std::max(16.0, dense * std::sqrt((double)n))));
  // C = AT2 * AT2^T restricted to kept rows: C(:,j) = union over rows r of A in
  // column j (kept) of the columns of row r.
  vector<char> keep(m);
  for (i64 r = 0; r < m; ++r) keep[r] = (at.cp[r + 1] - at.cp[r]) <= densethr;
  Pattern c;
  c.n = n;
  c.cp.assign(n + 1, 0);
  vector<i64> mark(n, -1), buf;
  for (i64 j = 0; j < n; ++j) {
    buf.clear();
    for (i64 p = cp[j]; p < cp[j + 1]; ++p) {
      i64 r = ri[p];
      if (!keep[r]) continue;
      for (i64 q = at.cp[r]; q < at.cp[r + 1]; ++q) {
        i64 i = at.ri[q];
        if (mark[i] != j) {
          mark[i] = j;
          if (i != j) buf.push_back(i);
        }
      }
    }
    std::sort(buf.begin(), buf.end());
    c.ri.insert(c.ri.end(), buf.begin(), buf.end());
    c.cp[j + 1] = (i64)c.ri.size();
  }
  return amd_core(n, c.cp, c.ri, dense);
}

// ---------------------------------------------------------------------------
// Symbolic analysis (symbolic.jl:15-237)
// ---------------------------------------------------------------------------
vector<i64> etree0(const Pattern& s) {   // symbolic.jl:67-82 (nil = -1)
  i64 n = s.n;
  vector<i64> parent(n, -1), anc(n, -1);
  for (i64 k = 0; k < n; ++k) {
    for (i64 p = s.cp[k]; p < s.cp[k + 1]; ++p) {
      i64 i = s.ri[p];
      while (i != -1 && i < k) {
        i64 inext = anc[i];
        anc[i] = k;
        if (inext == -1) parent[i] = k;
        i = inext;
      }
    }
  }
  return parent;
}

vector<i64> postorder0(const vector<i64>& parent) {   // symbolic.jl:86-116
  i64 n = (i64)parent.size();
  vector<i64> head(n, -1), nextc(n, -1), post(n), stack(n);
  for (i64 j = n - 1; j >= 0; --j) {
    i64 p = parent[j];
    if (p != -1) {
      nextc[j] = head[p];
      head[p] = j;
    }
  }
  i64 k = 0;
  for (i64 j = 0; j < n; ++j) {
    if (parent[j] != -1) continue;
    i64 top = 0;
    stack[0] = j;
    while (top >= 0) {
      i64 p = stack[top];
      i64 i = head[p];
      if (i == -1) {
        --top;
        post[k++] = p;
      } else {
        head[p] = nextc[i];
        stack[++top] = i;
      }
    }
  }
  return post;
}

struct Symbolic {
  i64 n = 0;
  vector<i64> qf;                       // 0-based
  vector<i64> parent;                   // -1 = root
  vector<i64> cs_ptr, cs_idx;           // colstruct, flattened (0-based rows)
  vector<i64> sstart;                   // nsuper+1, 0-based
  vector<i64> super_of;
  vector<i64> ch_ptr, ch_idx;           // childsupers, flattened, 0-based
};

// symbolic.jl:122-160 (union rule), 167-194 (fundamental supernodes), 211-226.
Symbolic symbolic_mf0(i64 n, const i64* cp, const i64* ri, const vector<i64>* q) {
  Symbolic S;
  S.n = n;
  vector<i64> qamd = q ? *q : amd_order_sym0(n, cp, ri, 10.0);
  Pattern sym = sym_pattern(n, cp, ri, true);
  Pattern p1 = permute_sym(sym, qamd);       // == _sym_csc1(A[qamd,qamd])
  vector<i64> parent1 = etree0(p1);
  vector<i64> post = postorder0(parent1);
  S.qf.resize(n);
  for (i64 k = 0; k < n; ++k) S.qf[k] = qamd[post[k]];
  Pattern pf = permute_sym(p1, post);
  S.parent = etree0(pf);

  // column structure of L
  vector<i64> head(n, -1), nextc(n, -1), marker(n, -1), scratch(n);
  for (i64 j = n - 1; j >= 0; --j) {
    i64 p = S.parent[j];
    if (p != -1) {
      nextc[j] = head[p];
      head[p] = j;
    }
  }
  S.cs_ptr.assign(n + 1, 0);
  vector<vector<i64>> cols(n);
  for (i64 j = 0; j < n; ++j) {
    i64 cnt = 0;
    marker[j] = j;
    for (i64 p = pf.cp[j]; p < pf.cp[j + 1]; ++p) {
      i64 i = pf.ri[p];
      if (i > j && marker[i] != j) {
        marker[i] = j;
        scratch[cnt++] = i;
      }
    }
    for (i64 c = head[j]; c != -1; c = nextc[c]) {
      for (i64 i : cols[c]) {
        if (i > j && marker[i] != j) {
          marker[i] = j;
          scratch[cnt++] = i;
        }
      }
    }
    cols[j].assign(scratch.begin(), scratch.begin() + cnt);
    std::sort(cols[j].begin(), cols[j].end());
  }
  for (i64 j = 0; j < n; ++j) S.cs_ptr[j + 1] = S.cs_ptr[j] + (i64)cols[j].size();
  S.cs_idx.reserve(S.cs_ptr[n]);
  for (i64 j = 0; j < n; ++j) S.cs_idx.insert(S.cs_idx.end(), cols[j].begin(), cols[j].end());

  // fundamental supernodes
  vector<i64> nchild(n, 0);
  for (i64 j = 0; j < n; ++j)
    if (S.parent[j] != -1) nchild[S.parent[j]]++;
  S.super_of.assign(n, 0);
  i64 nsuper = 0;
  for (i64 j = 0; j < n; ++j) {
    bool cont = j > 0 && S.parent[j - 1] == j && nchild[j] == 1 &&
                (i64)cols[j - 1].size() == (i64)cols[j].size() + 1;
    if (!cont) {
      ++nsuper;
      S.sstart.push_back(j);
    }
    S.super_of[j] = nsuper - 1;
  }
  S.sstart.push_back(n);
  vector<vector<i64>> kids(nsuper);
  for (i64 sk = 0; sk < nsuper; ++sk) {
    i64 lastcol = S.sstart[sk + 1] - 1;
    i64 p = S.parent[lastcol];
    if (p != -1) kids[S.super_of[p]].push_back(sk);
  }
  S.ch_ptr.assign(nsuper + 1, 0);
  for (i64 sk = 0; sk < nsuper; ++sk) {
    S.ch_ptr[sk + 1] = S.ch_ptr[sk] + (i64)kids[sk].size();
    S.ch_idx.insert(S.ch_idx.end(), kids[sk].begin(), kids[sk].end());
  }
  return S;
}

// ---------------------------------------------------------------------------
// Numeric multifrontal (multifrontal.jl:45-375)
// ---------------------------------------------------------------------------
// Factor values of type Xv: double for Float64 and Float32 matrices (Float32
// values widen exactly), complex for ComplexF64 ones.
template <typename Xv>
struct FactorT {
  i64 n = 0;
  vector<i64> Lp, Li, Up, Ui;           // 0-based
  vector<Xv> Lx, Ux;
  vector<i64> p, q, pinv;               // 0-based
  i64 status = 0;                       // 0 ok, k>0: singular at column k (1-based)
};
using Factor = FactorT<double>;
using FactorC = FactorT<cplx>;

// A[qf,qf] as CSC (sorted rows) plus its transpose.
template <typename Xv>
struct CscT {
  i64 n = 0;
  vector<i64> cp, ri;
  vector<Xv> x;
};

template <typename Xv>
CscT<Xv> permute_csc(i64 n, const i64* cp, const i64* ri, const Xv* x, const vector<i64>& q) {
  vector<i64> pinv(n);
  for (i64 k = 0; k < n; ++k) pinv[q[k]] = k;
  CscT<Xv> v;
  v.n = n;
  v.cp.assign(n + 1, 0);
  for (i64 j = 0; j < n; ++j) v.cp[j + 1] = v.cp[j] + (cp[q[j] + 1] - cp[q[j]]);
  v.ri.resize(v.cp[n]);
  v.x.resize(v.cp[n]);
  vector<std::pair<i64, Xv>> tmp;
  for (i64 j = 0; j < n; ++j) {
    tmp.clear();
    for (i64 p = cp[q[j]]; p < cp[q[j] + 1]; ++p) tmp.push_back({pinv[ri[p]], x[p]});
    std::sort(tmp.begin(), tmp.end(),
              [](const std::pair<i64, Xv>& a, const std::pair<i64, Xv>& b) { return a.first < b.first; });
    for (size_t t = 0; t < tmp.size(); ++t) {
      v.ri[v.cp[j] + t] = tmp[t].first;
      v.x[v.cp[j] + t] = tmp[t].second;
    }
  }
  return v;
}

template <typename Xv>
CscT<Xv> transpose_csc(const CscT<Xv>& a) {
  CscT<Xv> t;
  i64 n = a.n;
  t.n = n;
  t.cp.assign(n + 1, 0);
  i64 nz = a.cp[n];
  t.ri.resize(nz);
  t.x.resize(nz);
  for (i64 p = 0; p < nz; ++p) t.cp[a.ri[p] + 1]++;
  for (i64 i = 0; i < n; ++i) t.cp[i + 1] += t.cp[i];
  vector<i64> cur(t.cp.begin(), t.cp.end() - 1);
  for (i64 j = 0; j < n; ++j)
    for (i64 p = a.cp[j]; p < a.cp[j + 1]; ++p) {
      i64 d = cur[a.ri[p]]++;
      t.ri[d] = j;
      t.x[d] = a.x[p];
    }
  return t;
}

// _factor_colptrs (multifrontal.jl:73-104), 0-based pointers.
void factor_colptrs(const Symbolic& S, vector<i64>& Lp, vector<i64>& Up) {
  i64 n = S.n, nsuper = (i64)S.sstart.size() - 1;
  Lp.assign(n + 1, 0);
  Up.assign(n + 1, 0);
  vector<i64> ucount(n, 0);
  for (i64 sk = 0; sk < nsuper; ++sk) {
    i64 c1 = S.sstart[sk], c2 = S.sstart[sk + 1] - 1, np = c2 - c1 + 1;
    i64 nu = S.cs_ptr[c2 + 1] - S.cs_ptr[c2];
    for (i64 j = c1; j <= c2; ++j) {
      Lp[j + 1] = 1 + (c2 - j) + nu;
      ucount[j] += j - c1 + 1;
    }
    for (i64 t = 0; t < nu; ++t) ucount[S.cs_idx[S.cs_ptr[c2] + t]] += np;
  }
  for (i64 j = 0; j < n; ++j) Lp[j + 1] += Lp[j];
  for (i64 j = 0; j < n; ++j) Up[j + 1] = Up[j] + ucount[j];
}

// getrf / trsm / gemm of the element type: the factorization of a Float32
// matrix runs in Float32 (the reference's generic Tv, multifrontal.jl with
// Tv = Float32: lu! / rdiv! / ldiv! / mul! on Matrix{Float32}).
template <typename T>
struct Blas;
template <>
struct Blas<double> {
  static bool ok() { return g_dgetrf && g_dtrsm && g_dgemm; }
  static void getrf(const i64* m, const i64* n, double* a, const i64* ld, i64* ipiv, i64* info) {
    g_dgetrf(m, n, a, ld, ipiv, info);
  }
  static void trsm(const char* sd, const char* ul, const char* tr, const char* dg, const i64* m, const i64* n,
                   const double* al, const double* a, const i64* lda, double* b, const i64* ldb) {
    g_dtrsm(sd, ul, tr, dg, m, n, al, a, lda, b, ldb, 1, 1, 1, 1);
  }
  static void gemm(const i64* m, const i64* n, const i64* k, const double* al, const double* a, const i64* lda,
                   const double* b, const i64* ldb, const double* be, double* c, const i64* ldc) {
    g_dgemm("N", "N", m, n, k, al, a, lda, b, ldb, be, c, ldc, 1, 1);
  }
};
template <>
struct Blas<float> {
  static bool ok() { return g_sgetrf && g_strsm && g_sgemm; }
  static void getrf(const i64* m, const i64* n, float* a, const i64* ld, i64* ipiv, i64* info) {
    g_sgetrf(m, n, a, ld, ipiv, info);
  }
  static void trsm(const char* sd, const char* ul, const char* tr, const char* dg, const i64* m, const i64* n,
                   const float* al, const float* a, const i64* lda, float* b, const i64* ldb) {
    g_strsm(sd, ul, tr, dg, m, n, al, a, lda, b, ldb, 1, 1, 1, 1);
  }
  static void gemm(const i64* m, const i64* n, const i64* k, const float* al, const float* a, const i64* lda,
                   const float* b, const i64* ldb, const float* be, float* c, const i64* ldc) {
    g_sgemm("N", "N", m, n, k, al, a, lda, b, ldb, be, c, ldc, 1, 1);
  }
};

template <>
struct Blas<cplx> {
  static bool ok() { return g_zgetrf && g_ztrsm && g_zgemm; }
  static void getrf(const i64* m, const i64* n, cplx* a, const i64* ld, i64* ipiv, i64* info) {
    g_zgetrf(m, n, a, ld, ipiv, info);
  }
  static void trsm(const char* sd, const char* ul, const char* tr, const char* dg, const i64* m, const i64* n,
                   const cplx* al, const cplx* a, const i64* lda, cplx* b, const i64* ldb) {
    g_ztrsm(sd, ul, tr, dg, m, n, al, a, lda, b, ldb, 1, 1, 1, 1);
  }
  static void gemm(const i64* m, const i64* n, const i64* k, const cplx* al, const cplx* a, const i64* lda,
                   const cplx* b, const i64* ldb, const cplx* be, cplx* c, const i64* ldc) {
    g_zgemm("N", "N", m, n, k, al, a, lda, b, ldb, be, c, ldc, 1, 1);
  }
};

// Fronts, contribution blocks and all arithmetic in T; x holds the matrix
// values in Xv (Float32 values widen exactly to double), the factor keeps Xv.
template <typename T, typename Xv = double>
int numeric_mf(i64 n, const i64* cp, const i64* ri, const Xv* x, const Symbolic& S, bool check,
               FactorT<Xv>& F) {
  if (!Blas<T>::ok()) {
    g_err = "BLAS not loaded (call orc_set_blas first)";
    return -1;
  }
  F.n = n;
  CscT<Xv> V = permute_csc(n, cp, ri, x, S.qf);
  CscT<Xv> Vt = transpose_csc(V);
  i64 nsuper = (i64)S.sstart.size() - 1;
  vector<i64> loc(n, -1), prow(n);
  for (i64 k = 0; k < n; ++k) prow[k] = k;
  i64 maxnf = 0;
  for (i64 sk = 0; sk < nsuper; ++sk) {
    i64 c2 = S.sstart[sk + 1] - 1;
    i64 nfk = (c2 + 1 - S.sstart[sk]) + (S.cs_ptr[c2 + 1] - S.cs_ptr[c2]);
    maxnf = std::max(maxnf, nfk);
  }
  vector<T> Fbuf((size_t)std::max<i64>(maxnf * maxnf, 1));
  vector<T> cbval((size_t)std::max<i64>(64, maxnf * maxnf));
  i64 cbtop = 0;
  vector<i64> cboff(nsuper, 0);
  factor_colptrs(S, F.Lp, F.Up);
  F.Li.resize(F.Lp[n]);
  F.Lx.resize(F.Lp[n]);
  F.Ui.resize(F.Up[n]);
  F.Ux.resize(F.Up[n]);
  vector<i64> Lcur(F.Lp.begin(), F.Lp.end() - 1), Ucur(F.Up.begin(), F.Up.end() - 1);
  vector<i64> ipiv;
  vector<i64> orig;
  F.status = 0;

  for (i64 sk = 0; sk < nsuper; ++sk) {
    i64 c1 = S.sstart[sk], c2 = S.sstart[sk + 1] - 1, np = c2 - c1 + 1;
    const i64* upd = S.cs_idx.data() + S.cs_ptr[c2];
    i64 nu = S.cs_ptr[c2 + 1] - S.cs_ptr[c2];
    i64 nf = np + nu;
    i64 ld = nf;
    for (i64 a = 0; a < np; ++a) loc[c1 + a] = a;
    for (i64 t = 0; t < nu; ++t) loc[upd[t]] = np + t;
    T* Fm = Fbuf.data();
    std::fill(Fm, Fm + nf * nf, T(0));
#define FE(r, c) Fm[(r) + (c) * ld]
    // assemble original entries (multifrontal.jl:217-231)
    for (i64 a = 0; a < np; ++a) {
      i64 j = c1 + a;
      for (i64 p = V.cp[j]; p < V.cp[j + 1]; ++p) {
        i64 i = V.ri[p];
        if (i >= j && loc[i] != -1) FE(loc[i], a) += (T)V.x[p];
      }
      for (i64 p = Vt.cp[j]; p < Vt.cp[j + 1]; ++p) {
        i64 k = Vt.ri[p];
        if (k > j && loc[k] != -1) FE(a, loc[k]) += (T)Vt.x[p];
      }
    }
    // extend-add children, last child first (multifrontal.jl:235-243)
    for (i64 ci = S.ch_ptr[sk + 1] - 1; ci >= S.ch_ptr[sk]; --ci) {
      i64 ck = S.ch_idx[ci];
      i64 cl = S.sstart[ck + 1] - 1;
      const i64* crows = S.cs_idx.data() + S.cs_ptr[cl];
      i64 m = S.cs_ptr[cl + 1] - S.cs_ptr[cl];
      if (m == 0) continue;
      const T* cb = cbval.data() + cboff[ck];
      for (i64 s = 0; s < m; ++s) {
        i64 cs = loc[crows[s]];
        for (i64 r = 0; r < m; ++r) FE(loc[crows[r]], cs) += cb[r + s * m];
      }
      cbtop = cboff[ck];
    }
    // getrf on the pivot block (multifrontal.jl:247-252)
    ipiv.assign(std::max<i64>(np, 1), 0);
    i64 info = 0;
    Blas<T>::getrf(&np, &np, Fm, &ld, ipiv.data(), &info);
    if (check && info != 0) {
      F.status = c1 + info;   // 1-based column, = c1 + info - 1 in 1-based c1
      return 1;
    }
    if (nu > 0) {
      for (i64 k = 0; k < np; ++k) {    // swap R12 rows (multifrontal.jl:256-263)
        i64 pk = ipiv[k] - 1;
        if (pk != k)
          for (i64 col = 0; col < nu; ++col) std::swap(FE(k, np + col), FE(pk, np + col));
      }
      const T one = 1, mone = -1;
      // L21 = A21 * U11^{-1}; U12 = L11^{-1} * A12; F22 -= L21 * U12
      Blas<T>::trsm("R", "U", "N", "N", &nu, &np, &one, Fm, &ld, &FE(np, 0), &ld);
      Blas<T>::trsm("L", "L", "N", "U", &np, &nu, &one, Fm, &ld, &FE(0, np), &ld);
      Blas<T>::gemm(&nu, &nu, &np, &mone, &FE(np, 0), &ld, &FE(0, np), &ld, &one, &FE(np, np), &ld);
    }
    // _pivot_rows (multifrontal.jl:363-375)
    orig.resize(np);
    for (i64 a = 0; a < np; ++a) orig[a] = c1 + a;
    for (i64 k = 0; k < np; ++k) {
      i64 pk = ipiv[k] - 1;
      if (pk != k) std::swap(orig[k], orig[pk]);
    }
    for (i64 a = 0; a < np; ++a) prow[c1 + a] = orig[a];
    // scatter L and U (multifrontal.jl:278-317)
    for (i64 a = 0; a < np; ++a) {
      i64 g = c1 + a;
      i64 lp = Lcur[g];
      F.Li[lp] = orig[a];
      F.Lx[lp++] = 1.0;
      for (i64 b = a + 1; b < np; ++b) {
        F.Li[lp] = orig[b];
        F.Lx[lp++] = FE(b, a);
      }
      for (i64 t = 0; t < nu; ++t) {
        F.Li[lp] = upd[t];
        F.Lx[lp++] = FE(np + t, a);
      }
      Lcur[g] = lp;
      i64 up = Ucur[g];
      for (i64 b = 0; b <= a; ++b) {
        F.Ui[up] = c1 + b;
        F.Ux[up++] = FE(b, a);
      }
      Ucur[g] = up;
    }
    for (i64 t = 0; t < nu; ++t) {
      i64 J = upd[t];
      i64 up = Ucur[J];
      for (i64 a = 0; a < np; ++a) {
        F.Ui[up] = c1 + a;
        F.Ux[up++] = FE(a, np + t);
      }
      Ucur[J] = up;
    }
    // push the Schur block (multifrontal.jl:321-332)
    if (nu > 0) {
      if ((i64)cbval.size() < cbtop + nu * nu) cbval.resize(std::max(cbtop + nu * nu, 2 * (i64)cbval.size()));
      cboff[sk] = cbtop;
      for (i64 s = 0; s < nu; ++s)
        for (i64 r = 0; r < nu; ++r) cbval[cbtop + s * nu + r] = FE(np + r, np + s);
      cbtop += nu * nu;
    }
#undef FE
    for (i64 a = 0; a < np; ++a) loc[c1 + a] = -1;
    for (i64 t = 0; t < nu; ++t) loc[upd[t]] = -1;
  }
  // relabel L rows, permutations (multifrontal.jl:347-357)
  vector<i64> rowfac(n);
  for (i64 k = 0; k < n; ++k) rowfac[prow[k]] = k;
  for (auto& r : F.Li) r = rowfac[r];
  F.q = S.qf;
  F.p.resize(n);
  F.pinv.resize(n);
  for (i64 k = 0; k < n; ++k) F.p[k] = S.qf[prow[k]];
  for (i64 k = 0; k < n; ++k) F.pinv[F.p[k]] = k;
  return 0;
}

// solve.jl:10-22 and 25-39
template <typename T, typename FT>
void lsolve(const FT& F, T* y) {
  for (i64 j = 0; j < F.n; ++j) {
    T yj = y[j];
    for (i64 p = F.Lp[j] + 1; p < F.Lp[j + 1]; ++p) y[F.Li[p]] -= (T)F.Lx[p] * yj;
  }
}
template <typename T, typename FT>
void usolve(const FT& F, T* y) {
  for (i64 j = F.n - 1; j >= 0; --j) {
    i64 pd = F.Up[j + 1] - 1;
    T yj = y[j] / (T)F.Ux[pd];
    y[j] = yj;
    for (i64 p = F.Up[j]; p < pd; ++p) y[F.Ui[p]] -= (T)F.Ux[p] * yj;
  }
}

// ---- Gilbert-Peierls left-looking LU (gplu.jl:62-303) ----------------------
// Depth-first search from row j0 in the graph of the partial L (edge j -> i
// when row j is a pivot, J = pinv[j], and row i is stored in L's column J);
// finished rows go to xi[--top], so xi[top..n) is a topological order
// (gplu.jl:70-102).
i64 gp_dfs(i64 j0, const vector<i64>& Lp, const vector<i64>& Li, const vector<i64>& pinv, i64 top,
           vector<i64>& xi, vector<i64>& stack, vector<i64>& pstack, vector<char>& marked) {
  i64 head = 0;
  stack[0] = j0;
  while (head >= 0) {
    i64 j = stack[head];
    i64 J = pinv[j];
    if (!marked[j]) {
      marked[j] = 1;
      pstack[head] = J >= 0 ? Lp[J] : 0;
    }
    bool done = true;
    if (J >= 0) {
      for (i64 p = pstack[head]; p < Lp[J + 1]; ++p) {
        i64 i = Li[p];
        if (!marked[i]) {
          pstack[head] = p;
          stack[++head] = i;
          done = false;
          break;
        }
      }
    }
    if (done) {
      --head;
      xi[--top] = j;
    }
  }
  return top;
}

// The reach of A(:, col) in the graph of L, in the order of A's stored rows
// (gplu.jl:106-122); leaves marked all clear.
i64 gp_reach(const vector<i64>& Lp, const vector<i64>& Li, const i64* cp, const i64* ri, i64 col,
             const vector<i64>& pinv, vector<i64>& xi, vector<i64>& stack, vector<i64>& pstack,
             vector<char>& marked, i64 n) {
  i64 top = n;
  for (i64 p = cp[col]; p < cp[col + 1]; ++p)
    if (!marked[ri[p]]) top = gp_dfs(ri[p], Lp, Li, pinv, top, xi, stack, pstack, marked);
  for (i64 p = top; p < n; ++p) marked[xi[p]] = 0;
  return top;
}

// Scalar arithmetic of the Gilbert-Peierls restatement for each element type,
// each operation rounded on its own as Julia evaluates it (no contraction:
// the oracle is built for baseline x86-64, which has no fused multiply-add).
// Complex values follow Julia Base: z * w = (re re - im im, re im + im re),
// z / w by the robust Smith method of Baudin and Smith with its scaling, and
// abs(z) = hypot(re, im) by Borges' fma-corrected algorithm.
double jl_hypot(double x, double y) {
  double ax = std::fabs(x), ay = std::fabs(y);
  if (std::isinf(ax) || std::isinf(ay)) return INFINITY;
  if (ay > ax) std::swap(ax, ay);
  if (ay <= ax * std::sqrt(0x1p-53)) return ax;   // widely varying operands (and ay == 0)
  double scale = 0x1p-563;                         // eps * sqrt(floatmin)
  if (ax > std::sqrt(0x1.fffffffffffffp+1022)) {   // sqrt(floatmax / 2)
    ax = ax * scale;
    ay = ay * scale;
    scale = 1.0 / scale;
  } else if (ay < 0x1p-511) {                      // sqrt(floatmin)
    ax = ax / scale;
    ay = ay / scale;
  } else {
    scale = 1.0;
  }
  double h = std::sqrt(std::fma(ax, ax, ay * ay));
  const double hsq = h * h, axsq = ax * ax;
  h = h - (std::fma(-ay, ay, hsq - axsq) + std::fma(h, h, -hsq) - std::fma(ax, ax, -axsq)) / (2.0 * h);
  return h * scale;
}
double jl_cdiv2(double a, double b, double c, double d, double r, double t) {
  if (r != 0) {
    const double br = b * r;
    return br != 0 ? (a + br) * t : a * t + (b * t) * r;
  }
  return (a + d * (b / c)) * t;
}
void jl_cdiv1(double a, double b, double c, double d, double& p, double& q) {
  const double r = d / c;
  const double t = 1.0 / (c + d * r);
  p = jl_cdiv2(a, b, c, d, r, t);
  q = jl_cdiv2(b, -a, c, d, r, t);
}
cplx jl_cdiv(cplx z, cplx w) {
  double a = z.real(), b = z.imag(), c = w.real(), d = w.imag();
  const double ab = std::fabs(a) >= std::fabs(b) ? std::fabs(a) : std::fabs(b);
  const double cd = std::fabs(c) >= std::fabs(d) ? std::fabs(c) : std::fabs(d);
  const double halfov = 0.5 * 0x1.fffffffffffffp+1023;
  const double twounf = 0x1p-1022 * 2.0 / 0x1p-52;
  const double bs = 2.0 / (0x1p-52 * 0x1p-52);
  double S = 1.0;
  if (ab >= halfov) { a = 0.5 * a; b = 0.5 * b; S = 2.0 * S; }
  if (cd >= halfov) { c = 0.5 * c; d = 0.5 * d; S = 0.5 * S; }
  if (ab <= twounf) { a = a * bs; b = b * bs; S = S / bs; }
  if (cd <= twounf) { c = c * bs; d = d * bs; S = S * bs; }
  double p, q;
  if (std::fabs(d) <= std::fabs(c)) {
    jl_cdiv1(a, b, c, d, p, q);
  } else {
    jl_cdiv1(b, a, d, c, p, q);
    q = -q;
  }
  return cplx(p * S, q * S);
}

template <typename T>
struct GpOps {   // Float64 and Float32
  using R = T;
  static T scale(R r, T a) { return a * r; }
  static T mul(T a, T b) { return a * b; }
  static T add(T a, T b) { return a + b; }
  static T sub(T a, T b) { return a - b; }
  static T div(T a, T b) { return a / b; }
  static R mag(T a) { return std::fabs(a); }
};
template <>
struct GpOps<cplx> {
  using R = double;
  static cplx scale(R r, cplx a) { return cplx(a.real() * r, a.imag() * r); }
  static cplx mul(cplx z, cplx w) {
    return cplx(z.real() * w.real() - z.imag() * w.imag(), z.real() * w.imag() + z.imag() * w.real());
  }
  static cplx add(cplx a, cplx b) { return cplx(a.real() + b.real(), a.imag() + b.imag()); }
  static cplx sub(cplx a, cplx b) { return cplx(a.real() - b.real(), a.imag() - b.imag()); }
  static cplx div(cplx a, cplx b) { return jl_cdiv(a, b); }
  static R mag(cplx a) { return jl_hypot(a.real(), a.imag()); }
};

// Each column's (row, value) pairs sorted by row (gplu.jl:383-415: the keys
// of a column are distinct, so any sort gives this order).
template <typename T>
void gp_sortcols_t(i64 n, const vector<i64>& cp, vector<i64>& ri, vector<T>& x) {
  vector<std::pair<i64, T>> tmp;
  for (i64 j = 0; j < n; ++j) {
    tmp.clear();
    for (i64 p = cp[j]; p < cp[j + 1]; ++p) tmp.emplace_back(ri[p], x[p]);
    std::sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (i64 p = cp[j]; p < cp[j + 1]; ++p) {
      ri[p] = tmp[p - cp[j]].first;
      x[p] = tmp[p - cp[j]].second;
    }
  }
}

// gplu(A; q, tol, check, sort_factors) (gplu.jl:173-303), 0-based, for
// Tv = Float64, Float32 or ComplexF64 (tol converted to real(Tv), as
// gplu.jl:213 does).  Returns 0, or -1 when the pivot rows do not form a
// permutation (a singular matrix factored with check = false: the
// reference's invperm throws there); F.status = k (1-based) when check is
// set and column k has no nonzero pivot.
template <typename T>
int gplu0(i64 n, const i64* cp, const i64* ri, const T* ax, const vector<i64>& q, typename GpOps<T>::R tol,
          bool check, bool sort_factors, FactorT<T>& F) {
  using O = GpOps<T>;
  using R = typename O::R;
  F = FactorT<T>();
  F.n = n;
  vector<T> x(n, T(0));
  vector<i64> xi(n), stack(n), pstack(n), pinv(n, -1);
  vector<char> marked(n, 0);
  F.Lp.assign(n + 1, 0);
  F.Up.assign(n + 1, 0);
  for (i64 k = 0; k < n; ++k) {
    i64 col = q[k];
    i64 top = gp_reach(F.Lp, F.Li, cp, ri, col, pinv, xi, stack, pstack, marked, n);
    for (i64 p = top; p < n; ++p) x[xi[p]] = T(0);
    for (i64 p = cp[col]; p < cp[col + 1]; ++p) x[ri[p]] = ax[p];
    for (i64 px = top; px < n; ++px) {   // L x = A(:, col), unit diagonal stored first
      i64 j = xi[px], J = pinv[j];
      if (J < 0) continue;
      T xj = x[j];
      for (i64 p = F.Lp[J] + 1; p < F.Lp[J + 1]; ++p) x[F.Li[p]] = O::sub(x[F.Li[p]], O::mul(F.Lx[p], xj));
    }
    i64 ipiv = -1;
    R a = R(-1);
    for (i64 px = top; px < n; ++px) {   // U entries in reach order; largest unpivoted row
      i64 i = xi[px];
      if (pinv[i] < 0) {
        R t = O::mag(x[i]);
        if (t > a) {
          a = t;
          ipiv = i;
        }
      } else {
        F.Ui.push_back(pinv[i]);
        F.Ux.push_back(x[i]);
      }
    }
    if (ipiv < 0 || a <= 0) {
      if (check) {
        F.status = k + 1;
        return 0;
      }
      if (ipiv < 0) ipiv = col;
    }
    if (pinv[col] < 0 && O::mag(x[col]) >= tol * a) ipiv = col;
    T pivot = x[ipiv];
    F.Ui.push_back(k);
    F.Ux.push_back(pivot);
    F.Up[k + 1] = (i64)F.Ui.size();
    pinv[ipiv] = k;
    F.Li.push_back(ipiv);
    F.Lx.push_back(T(1));
    for (i64 px = top; px < n; ++px) {
      i64 i = xi[px];
      if (pinv[i] < 0) {
        F.Li.push_back(i);
        F.Lx.push_back(O::div(x[i], pivot));
      }
      x[i] = T(0);
    }
    F.Lp[k + 1] = (i64)F.Li.size();
  }
  vector<char> seen(n, 0);
  for (i64 i = 0; i < n; ++i) {
    if (pinv[i] < 0 || seen[pinv[i]]) return -1;
    seen[pinv[i]] = 1;
  }
  for (auto& r : F.Li) r = pinv[r];
  if (sort_factors) {
    gp_sortcols_t(n, F.Lp, F.Li, F.Lx);
    gp_sortcols_t(n, F.Up, F.Ui, F.Ux);
  }
  F.q = q;
  F.pinv = pinv;
  F.p.assign(n, 0);
  for (i64 i = 0; i < n; ++i) F.p[pinv[i]] = i;
  return 0;
}

// solve(F::PureLU{ComplexF64}, b; refine) over Gilbert-Peierls factors
// (interface.jl:123-177, solve.jl:10-39) in Julia's complex arithmetic.
void gp_solve_c64(const FactorC& F, const double* Rs, i64 n, const i64* colptr, const i64* rowval,
                  const double* nzval_ri, const cplx* b, cplx* x, int refine) {
  using O = GpOps<cplx>;
  vector<cplx> c(n), r(n), ax(n);
  auto solve1 = [&](const cplx* bb, cplx* xx, bool accumulate) {
    for (i64 k = 0; k < n; ++k) c[k] = Rs ? O::scale(Rs[F.p[k]], bb[F.p[k]]) : bb[F.p[k]];
    for (i64 j = 0; j < n; ++j) {
      const cplx yj = c[j];
      for (i64 p = F.Lp[j] + 1; p < F.Lp[j + 1]; ++p) c[F.Li[p]] = O::sub(c[F.Li[p]], O::mul(F.Lx[p], yj));
    }
    for (i64 j = n - 1; j >= 0; --j) {
      const i64 pd = F.Up[j + 1] - 1;
      const cplx yj = O::div(c[j], F.Ux[pd]);
      c[j] = yj;
      for (i64 p = F.Up[j]; p < pd; ++p) c[F.Ui[p]] = O::sub(c[F.Ui[p]], O::mul(F.Ux[p], yj));
    }
    for (i64 k = 0; k < n; ++k) xx[F.q[k]] = accumulate ? O::add(xx[F.q[k]], c[k]) : c[k];
  };
  solve1(b, x, false);
  for (int it = 0; it < refine; ++it) {
    std::fill(ax.begin(), ax.end(), cplx(0.0, 0.0));
    for (i64 j = 0; j < n; ++j) {
      const cplx xj = x[j];
      for (i64 p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p)
        ax[rowval[p] - 1] = O::add(ax[rowval[p] - 1], O::mul(cplx(nzval_ri[2 * p], nzval_ri[2 * p + 1]), xj));
    }
    for (i64 i = 0; i < n; ++i) r[i] = O::sub(b[i], ax[i]);
    solve1(r.data(), x, true);
  }
}

}  // namespace

// ===========================================================================
// C ABI (ctypes).  All index arrays are 1-based int64.
// ===========================================================================
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_set_blas(const char* path) {
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) {
    g_err = dlerror();
    return -1;
  }
  g_dgetrf = (dgetrf_fn)dlsym(h, "scipy_dgetrf_64_");
  g_dtrsm = (dtrsm_fn)dlsym(h, "scipy_dtrsm_64_");
  g_dgemm = (dgemm_fn)dlsym(h, "scipy_dgemm_64_");
  g_sgetrf = (sgetrf_fn)dlsym(h, "scipy_sgetrf_64_");
  g_strsm = (strsm_fn)dlsym(h, "scipy_strsm_64_");
  g_sgemm = (sgemm_fn)dlsym(h, "scipy_sgemm_64_");
  g_zgetrf = (zgetrf_fn)dlsym(h, "scipy_zgetrf_64_");
  g_ztrsm = (ztrsm_fn)dlsym(h, "scipy_ztrsm_64_");
  g_zgemm = (zgemm_fn)dlsym(h, "scipy_zgemm_64_");
  g_setthreads = (setthreads_fn)dlsym(h, "scipy_openblas_set_num_threads64_");
  g_getthreads = (getthreads_fn)dlsym(h, "scipy_openblas_get_num_threads64_");
  if (!g_dgetrf || !g_dtrsm || !g_dgemm) {
    g_err = "missing BLAS symbols";
    return -2;
  }
  return 0;
}

int orc_blas_threads(int k) {
  if (k > 0 && g_setthreads) g_setthreads(k);
  return g_getthreads ? g_getthreads() : -1;
}

// scaling.jl:92-115.  kind: 0 NONE, 1 SUM, 2 MAX.
void orc_row_scaling(i64 n, const i64* colptr, const i64* rowval, const double* nzval, int kind, double* Rs) {
  for (i64 i = 0; i < n; ++i) Rs[i] = 1.0;
  if (kind == 0) return;
  vector<double> acc(n, 0.0);
  i64 nz = colptr[n] - 1;
  if (kind == 1) {
    for (i64 p = 0; p < nz; ++p) acc[rowval[p] - 1] += std::fabs(nzval[p]);
  } else {
    for (i64 p = 0; p < nz; ++p) {
      i64 i = rowval[p] - 1;
      double v = std::fabs(nzval[p]);
      acc[i] = v > acc[i] ? v : acc[i];
    }
  }
  for (i64 i = 0; i < n; ++i) Rs[i] = acc[i] > 0 ? 1.0 / acc[i] : 1.0;
}

static void to0(i64 n, const i64* cp1, const i64* ri1, vector<i64>& cp, vector<i64>& ri) {
  cp.resize(n + 1);
  for (i64 j = 0; j <= n; ++j) cp[j] = cp1[j] - 1;
  ri.resize(cp[n]);
  for (i64 p = 0; p < cp[n]; ++p) ri[p] = ri1[p] - 1;
}

int orc_amd_order_sym(i64 n, const i64* colptr, const i64* rowval, double dense, i64* perm) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> p = amd_order_sym0(n, cp.data(), ri.data(), dense);
  for (i64 k = 0; k < n; ++k) perm[k] = p[k] + 1;
  return 0;
}

int orc_colamd_order(i64 m, i64 n, const i64* colptr, const i64* rowval, double dense, i64* perm) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> p = colamd_order0(m, n, cp.data(), ri.data(), dense);
  for (i64 k = 0; k < n; ++k) perm[k] = p[k] + 1;
  return 0;
}

// ---- symbolic object ------------------------------------------------------
void* orc_symbolic(i64 n, const i64* colptr, const i64* rowval, const i64* q1) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q;
  if (q1) {
    q.resize(n);
    for (i64 k = 0; k < n; ++k) q[k] = q1[k] - 1;
  }
  return new Symbolic(symbolic_mf0(n, cp.data(), ri.data(), q1 ? &q : nullptr));
}
void orc_symbolic_free(void* h) { delete (Symbolic*)h; }
// sizes: [n, nsuper, nnz(colstruct), nnz(childsupers)]
void orc_symbolic_sizes(void* h, i64* out) {
  Symbolic* S = (Symbolic*)h;
  out[0] = S->n;
  out[1] = (i64)S->sstart.size() - 1;
  out[2] = S->cs_ptr.empty() ? 0 : S->cs_ptr[S->n];
  out[3] = (i64)S->ch_idx.size();
}
// 1-based copies: qf(n), parent(n; 0 = root), cs_ptr(n+1), cs_idx, sstart(nsuper+1),
// ch_ptr(nsuper+1), ch_idx.
void orc_symbolic_get(void* h, i64* qf, i64* parent, i64* cs_ptr, i64* cs_idx, i64* sstart, i64* ch_ptr,
                      i64* ch_idx) {
  Symbolic* S = (Symbolic*)h;
  i64 n = S->n, ns = (i64)S->sstart.size() - 1;
  for (i64 k = 0; k < n; ++k) {
    qf[k] = S->qf[k] + 1;
    parent[k] = S->parent[k] + 1;
  }
  for (i64 k = 0; k <= n; ++k) cs_ptr[k] = S->cs_ptr[k] + 1;
  for (size_t k = 0; k < S->cs_idx.size(); ++k) cs_idx[k] = S->cs_idx[k] + 1;
  for (i64 k = 0; k <= ns; ++k) {
    sstart[k] = S->sstart[k] + 1;
    ch_ptr[k] = S->ch_ptr[k] + 1;
  }
  for (size_t k = 0; k < S->ch_idx.size(); ++k) ch_idx[k] = S->ch_idx[k] + 1;
}

// ---- numeric factor object --------------------------------------------------
// Factor V = A (already scaled by the caller, as splu does) with optional
// caller order q1 (1-based, may be NULL).  Returns a handle; *status = 0 on
// success, k > 0 when check is set and the pivot at column k is zero, < 0 on
// error.
void* orc_multifrontal_lu(i64 n, const i64* colptr, const i64* rowval, const double* nzval, const i64* q1,
                          int check, i64* status) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q;
  if (q1) {
    q.resize(n);
    for (i64 k = 0; k < n; ++k) q[k] = q1[k] - 1;
  }
  Symbolic S = symbolic_mf0(n, cp.data(), ri.data(), q1 ? &q : nullptr);
  Factor* F = new Factor();
  int rc = numeric_mf<double>(n, cp.data(), ri.data(), nzval, S, check != 0, *F);
  *status = rc < 0 ? rc : F->status;
  return F;
}
// Numeric only, with a precomputed symbolic object (for timing the numeric
// phase separately from the symbolic one).
void* orc_numeric(void* sym, const double* nzval, const i64* colptr, const i64* rowval, int check, i64* status) {
  Symbolic* S = (Symbolic*)sym;
  vector<i64> cp, ri;
  to0(S->n, colptr, rowval, cp, ri);
  Factor* F = new Factor();
  int rc = numeric_mf<double>(S->n, cp.data(), ri.data(), nzval, *S, check != 0, *F);
  *status = rc < 0 ? rc : F->status;
  return F;
}
// gplu(A; q, tol, check, sort_factors) (gplu.jl:173-303): q1 1-based or NULL
// for the natural order.  *status as orc_multifrontal_lu (k > 0: no nonzero
// pivot at column k under check; -1: the pivot rows are not a permutation).
void* orc_gplu(i64 n, const i64* colptr, const i64* rowval, const double* nzval, const i64* q1, double tol,
               int check, int sort_factors, i64* status) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q(n);
  for (i64 k = 0; k < n; ++k) q[k] = q1 ? q1[k] - 1 : k;
  Factor* F = new Factor();
  int rc = gplu0(n, cp.data(), ri.data(), nzval, q, tol, check != 0, sort_factors != 0, *F);
  if (rc < 0) g_err = "gplu: the pivot rows are not a permutation (singular matrix, check = false)";
  *status = rc < 0 ? rc : F->status;
  return F;
}

// gplu of a Float32 matrix, all arithmetic in Float32; the factor's values
// are returned widened to Float64 (exactly), as the other Float32 entry points.
void* orc_gplu_f32(i64 n, const i64* colptr, const i64* rowval, const float* nzval, const i64* q1, double tol,
                   int check, int sort_factors, i64* status) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q(n);
  for (i64 k = 0; k < n; ++k) q[k] = q1 ? q1[k] - 1 : k;
  FactorT<float> F32;
  int rc = gplu0(n, cp.data(), ri.data(), nzval, q, (float)tol, check != 0, sort_factors != 0, F32);
  Factor* F = new Factor();
  F->n = F32.n;
  F->Lp = F32.Lp;
  F->Li = F32.Li;
  F->Up = F32.Up;
  F->Ui = F32.Ui;
  F->Lx.assign(F32.Lx.begin(), F32.Lx.end());
  F->Ux.assign(F32.Ux.begin(), F32.Ux.end());
  F->p = F32.p;
  F->q = F32.q;
  F->pinv = F32.pinv;
  F->status = F32.status;
  if (rc < 0) g_err = "gplu: the pivot rows are not a permutation (singular matrix, check = false)";
  *status = rc < 0 ? rc : F->status;
  return F;
}

// gplu of a ComplexF64 matrix (values as interleaved re, im doubles).
void* orc_gplu_c64(i64 n, const i64* colptr, const i64* rowval, const double* nzval_ri, const i64* q1, double tol,
                   int check, int sort_factors, i64* status) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q(n);
  for (i64 k = 0; k < n; ++k) q[k] = q1 ? q1[k] - 1 : k;
  vector<cplx> xz(cp[n]);
  for (i64 p = 0; p < cp[n]; ++p) xz[p] = cplx(nzval_ri[2 * p], nzval_ri[2 * p + 1]);
  FactorC* F = new FactorC();
  int rc = gplu0(n, cp.data(), ri.data(), xz.data(), q, tol, check != 0, sort_factors != 0, *F);
  if (rc < 0) g_err = "gplu: the pivot rows are not a permutation (singular matrix, check = false)";
  *status = rc < 0 ? rc : F->status;
  return F;
}

// solve(F, b; refine) over complex Gilbert-Peierls factors (Rs NULL: the raw
// F \ b, refine 0).  B, X: nrhs columns of n interleaved (re, im) doubles.
void orc_gplu_solve_c64(void* h, const double* Rs, i64 n, const i64* colptr, const i64* rowval,
                        const double* nzval_ri, i64 nrhs, const double* B, double* X, int refine) {
  const FactorC* F = (const FactorC*)h;
  vector<cplx> b(n), x(n);
  for (i64 c = 0; c < nrhs; ++c) {
    for (i64 i = 0; i < n; ++i) b[i] = cplx(B[2 * (c * n + i)], B[2 * (c * n + i) + 1]);
    gp_solve_c64(*F, Rs, n, colptr, rowval, nzval_ri, b.data(), x.data(), refine);
    for (i64 i = 0; i < n; ++i) {
      X[2 * (c * n + i)] = x[i].real();
      X[2 * (c * n + i) + 1] = x[i].imag();
    }
  }
}

void orc_factor_free(void* h) { delete (Factor*)h; }
void orc_factor_sizes(void* h, i64* out) {
  Factor* F = (Factor*)h;
  out[0] = F->n;
  out[1] = F->Lp.empty() ? 0 : F->Lp[F->n];
  out[2] = F->Up.empty() ? 0 : F->Up[F->n];
}
void orc_factor_get(void* h, i64* Lp, i64* Li, double* Lx, i64* Up, i64* Ui, double* Ux, i64* p, i64* q,
                    i64* pinv) {
  Factor* F = (Factor*)h;
  i64 n = F->n;
  for (i64 k = 0; k <= n; ++k) {
    Lp[k] = F->Lp[k] + 1;
    Up[k] = F->Up[k] + 1;
  }
  for (size_t k = 0; k < F->Li.size(); ++k) {
    Li[k] = F->Li[k] + 1;
    Lx[k] = F->Lx[k];
  }
  for (size_t k = 0; k < F->Ui.size(); ++k) {
    Ui[k] = F->Ui[k] + 1;
    Ux[k] = F->Ux[k];
  }
  for (i64 k = 0; k < n; ++k) {
    p[k] = F->p[k] + 1;
    q[k] = F->q[k] + 1;
    pinv[k] = F->pinv[k] + 1;
  }
}

// _solve_factor (interface.jl:123-138) with Rs (NULL = no scaling, as the raw
// GPLUFactorization solve at solve.jl:66-77).
void orc_solve_factor(void* h, const double* Rs, const double* b, double* x) {
  Factor* F = (Factor*)h;
  i64 n = F->n;
  vector<double> c(n);
  for (i64 k = 0; k < n; ++k) c[k] = Rs ? Rs[F->p[k]] * b[F->p[k]] : b[F->p[k]];
  lsolve(*F, c.data());
  usolve(*F, c.data());
  for (i64 k = 0; k < n; ++k) x[F->q[k]] = c[k];
}

// solve(F::PureLU, b; refine) (interface.jl:170-177).  A is the UNSCALED
// original matrix (1-based CSC), nrhs columns of b / x stored with leading
// dimension n.
void orc_solve(void* h, const double* Rs, i64 n, const i64* colptr, const i64* rowval, const double* nzval,
               i64 nrhs, const double* B, double* X, int refine) {
  vector<double> r(n), d(n);
  for (i64 c = 0; c < nrhs; ++c) {
    const double* b = B + c * n;
    double* x = X + c * n;
    orc_solve_factor(h, Rs, b, x);
    for (int it = 0; it < refine; ++it) {
      // r = b - A*x (column-oriented SpMV as SparseArrays does)
      std::vector<double> ax(n, 0.0);
      for (i64 j = 0; j < n; ++j) {
        double xj = x[j];
        for (i64 p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p) ax[rowval[p] - 1] += nzval[p] * xj;
      }
      for (i64 i = 0; i < n; ++i) r[i] = b[i] - ax[i];
      orc_solve_factor(h, Rs, r.data(), d.data());
      for (i64 i = 0; i < n; ++i) x[i] = x[i] + d[i];
    }
  }
}

// ---- Float32 (the reference's generic Tv = Float32) ---------------------------
// row_scaling in Float32 arithmetic (scaling.jl:92-115 with R = Float32).
void orc_row_scaling_f32(i64 n, const i64* colptr, const i64* rowval, const float* nzval, int kind, float* Rs) {
  for (i64 i = 0; i < n; ++i) Rs[i] = 1.0f;
  if (kind == 0) return;
  vector<float> acc(n, 0.0f);
  i64 nz = colptr[n] - 1;
  if (kind == 1) {
    for (i64 p = 0; p < nz; ++p) acc[rowval[p] - 1] += std::fabs(nzval[p]);
  } else {
    for (i64 p = 0; p < nz; ++p) {
      i64 i = rowval[p] - 1;
      float v = std::fabs(nzval[p]);
      acc[i] = v > acc[i] ? v : acc[i];
    }
  }
  for (i64 i = 0; i < n; ++i) Rs[i] = acc[i] > 0 ? 1.0f / acc[i] : 1.0f;
}

// multifrontal_lu of a Float32 matrix (already scaled by the caller): the
// whole numeric phase in Float32; the factor handle stores the Float32 values
// widened to double (exact).
void* orc_multifrontal_lu_f32(i64 n, const i64* colptr, const i64* rowval, const float* nzval, const i64* q1,
                              int check, i64* status) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q;
  if (q1) {
    q.resize(n);
    for (i64 k = 0; k < n; ++k) q[k] = q1[k] - 1;
  }
  Symbolic S = symbolic_mf0(n, cp.data(), ri.data(), q1 ? &q : nullptr);
  vector<double> xd(nzval, nzval + cp[n]);
  Factor* F = new Factor();
  int rc = numeric_mf<float>(n, cp.data(), ri.data(), xd.data(), S, check != 0, *F);
  *status = rc < 0 ? rc : F->status;
  return F;
}

// solve(F::PureLU{Float32}, b::Vector{Float32}; refine) (interface.jl:123-177)
// in Float32: scaling, triangular solves, the residual b - A x and the update.
void orc_solve_f32(void* h, const float* Rs, i64 n, const i64* colptr, const i64* rowval, const float* nzval,
                   i64 nrhs, const float* B, float* X, int refine) {
  Factor* F = (Factor*)h;
  vector<float> c(n), r(n), ax(n);
  auto solve1 = [&](const float* b, float* x) {
    for (i64 k = 0; k < n; ++k) c[k] = Rs ? Rs[F->p[k]] * b[F->p[k]] : b[F->p[k]];
    lsolve(*F, c.data());
    usolve(*F, c.data());
    for (i64 k = 0; k < n; ++k) x[F->q[k]] = c[k];
  };
  vector<float> d(n);
  for (i64 col = 0; col < nrhs; ++col) {
    const float* b = B + col * n;
    float* x = X + col * n;
    solve1(b, x);
    for (int it = 0; it < refine; ++it) {
      std::fill(ax.begin(), ax.end(), 0.0f);
      for (i64 j = 0; j < n; ++j) {
        float xj = x[j];
        for (i64 p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p) ax[rowval[p] - 1] += nzval[p] * xj;
      }
      for (i64 i = 0; i < n; ++i) r[i] = b[i] - ax[i];
      solve1(r.data(), d.data());
      for (i64 i = 0; i < n; ++i) x[i] = x[i] + d[i];
    }
  }
}


// ---- ComplexF64 (the reference's generic Tv = ComplexF64) ---------------------
// Values cross as interleaved (re, im) doubles, the memory layout of Julia's
// ComplexF64 and of std::complex<double>.  The fronts run through zgetrf /
// ztrsm / zgemm, the calls Julia's lu! / rdiv! / ldiv! / mul! make on a
// Matrix{ComplexF64} (multifrontal.jl:247-275): zgetrf chooses the pivot of
// largest |re| + |im| (LAPACK's izamax), first on ties.

// row_scaling with R = real(Tv) = Float64 and abs(z) = hypot(re, im)
// (scaling.jl:92-115).
void orc_row_scaling_c64(i64 n, const i64* colptr, const i64* rowval, const double* nzval_ri, int kind, double* Rs) {
  for (i64 i = 0; i < n; ++i) Rs[i] = 1.0;
  if (kind == 0) return;
  vector<double> acc(n, 0.0);
  i64 nz = colptr[n] - 1;
  for (i64 p = 0; p < nz; ++p) {
    i64 i = rowval[p] - 1;
    double v = std::hypot(nzval_ri[2 * p], nzval_ri[2 * p + 1]);
    if (kind == 1)
      acc[i] += v;
    else
      acc[i] = v > acc[i] ? v : acc[i];
  }
  for (i64 i = 0; i < n; ++i) Rs[i] = acc[i] > 0 ? 1.0 / acc[i] : 1.0;
}

// multifrontal_lu of a ComplexF64 matrix (already scaled by the caller).
void* orc_multifrontal_lu_c64(i64 n, const i64* colptr, const i64* rowval, const double* nzval_ri, const i64* q1,
                              int check, i64* status) {
  vector<i64> cp, ri;
  to0(n, colptr, rowval, cp, ri);
  vector<i64> q;
  if (q1) {
    q.resize(n);
    for (i64 k = 0; k < n; ++k) q[k] = q1[k] - 1;
  }
  Symbolic S = symbolic_mf0(n, cp.data(), ri.data(), q1 ? &q : nullptr);
  vector<cplx> xz(cp[n]);
  for (i64 p = 0; p < cp[n]; ++p) xz[p] = cplx(nzval_ri[2 * p], nzval_ri[2 * p + 1]);
  FactorC* F = new FactorC();
  int rc = numeric_mf<cplx, cplx>(n, cp.data(), ri.data(), xz.data(), S, check != 0, *F);
  *status = rc < 0 ? rc : F->status;
  return F;
}
void orc_factor_free_c64(void* h) { delete (FactorC*)h; }
void orc_factor_sizes_c64(void* h, i64* out) {
  FactorC* F = (FactorC*)h;
  out[0] = F->n;
  out[1] = F->Lp.empty() ? 0 : F->Lp[F->n];
  out[2] = F->Up.empty() ? 0 : F->Up[F->n];
}
void orc_factor_get_c64(void* h, i64* Lp, i64* Li, double* Lx_ri, i64* Up, i64* Ui, double* Ux_ri, i64* p, i64* q,
                        i64* pinv) {
  FactorC* F = (FactorC*)h;
  i64 n = F->n;
  for (i64 k = 0; k <= n; ++k) {
    Lp[k] = F->Lp[k] + 1;
    Up[k] = F->Up[k] + 1;
  }
  for (size_t k = 0; k < F->Li.size(); ++k) {
    Li[k] = F->Li[k] + 1;
    Lx_ri[2 * k] = F->Lx[k].real();
    Lx_ri[2 * k + 1] = F->Lx[k].imag();
  }
  for (size_t k = 0; k < F->Ui.size(); ++k) {
    Ui[k] = F->Ui[k] + 1;
    Ux_ri[2 * k] = F->Ux[k].real();
    Ux_ri[2 * k + 1] = F->Ux[k].imag();
  }
  for (i64 k = 0; k < n; ++k) {
    p[k] = F->p[k] + 1;
    q[k] = F->q[k] + 1;
    pinv[k] = F->pinv[k] + 1;
  }
}

// solve(F::PureLU{ComplexF64}, b; refine) (interface.jl:123-177): real Rs
// (NULL = none), complex b and x, the residual b - A x with the unscaled A.
void orc_solve_c64(void* h, const double* Rs, i64 n, const i64* colptr, const i64* rowval, const double* nzval_ri,
                   i64 nrhs, const double* B_ri, double* X_ri, int refine) {
  FactorC* F = (FactorC*)h;
  vector<cplx> c(n), r(n), d(n), ax(n), b(n), x(n);
  auto solve1 = [&](const cplx* bb, cplx* xx) {
    for (i64 k = 0; k < n; ++k) c[k] = Rs ? Rs[F->p[k]] * bb[F->p[k]] : bb[F->p[k]];
    lsolve(*F, c.data());
    usolve(*F, c.data());
    for (i64 k = 0; k < n; ++k) xx[F->q[k]] = c[k];
  };
  for (i64 col = 0; col < nrhs; ++col) {
    const double* bc = B_ri + 2 * col * n;
    for (i64 i = 0; i < n; ++i) b[i] = cplx(bc[2 * i], bc[2 * i + 1]);
    solve1(b.data(), x.data());
    for (int it = 0; it < refine; ++it) {
      std::fill(ax.begin(), ax.end(), cplx(0.0, 0.0));
      for (i64 j = 0; j < n; ++j) {
        const cplx xj = x[j];
        for (i64 p = colptr[j] - 1; p < colptr[j + 1] - 1; ++p)
          ax[rowval[p] - 1] += cplx(nzval_ri[2 * p], nzval_ri[2 * p + 1]) * xj;
      }
      for (i64 i = 0; i < n; ++i) r[i] = b[i] - ax[i];
      solve1(r.data(), d.data());
      for (i64 i = 0; i < n; ++i) x[i] = x[i] + d[i];
    }
    double* xc = X_ri + 2 * col * n;
    for (i64 i = 0; i < n; ++i) {
      xc[2 * i] = x[i].real();
      xc[2 * i + 1] = x[i].imag();
    }
  }
}

}  // extern "C"
