// symbolic.cpp -- ordering and symbolic analysis (host integer code).
//
// Output is identical to PureUMFPACK.jl's (see symbolic.h for the file map).
// The approximate-minimum-degree core follows the quotient-graph method of
// Amestoy, Davis & Duff as formulated in CSparse's cs_amd, which is what
// src/amd.jl:191-539 ports; its steps, tie-breaks and hash must match that
// code exactly for the permutation to be identical, so the phases below
// mirror it one for one.  Column counts use the Gilbert-Ng-Peyton skeleton
// algorithm, and the update set of each fundamental supernode is formed by a
// supernodal union, which yields the same sets as the column-by-column union
// rule of src/symbolic.jl:122-160 at a fraction of the work.

#include "symbolic.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace mfgpu {

// ---------------------------------------------------------------------------
// patterns
// ---------------------------------------------------------------------------
static Pattern transpose(idx_t m, idx_t n, const idx_t* colptr, const idx_t* rowind) {
  Pattern t;
  t.n = m;
  t.colptr.assign(m + 1, 0);
  const idx_t nz = colptr[n];
  t.rowind.resize(nz);
  for (idx_t p = 0; p < nz; ++p) ++t.colptr[rowind[p] + 1];
  for (idx_t i = 0; i < m; ++i) t.colptr[i + 1] += t.colptr[i];
  std::vector<idx_t> next(t.colptr.begin(), t.colptr.end() - 1);
  for (idx_t j = 0; j < n; ++j)
    for (idx_t p = colptr[j]; p < colptr[j + 1]; ++p) t.rowind[next[rowind[p]]++] = j;
  return t;
}

Pattern symmetrize(idx_t n, const idx_t* colptr, const idx_t* rowind, bool keep_diagonal) {
  Pattern t = transpose(n, n, colptr, rowind);
  Pattern s;
  s.n = n;
  s.colptr.resize(n + 1);
  s.rowind.reserve(2 * colptr[n]);
  s.colptr[0] = 0;
  for (idx_t j = 0; j < n; ++j) {
    const idx_t* a = rowind + colptr[j];
    const idx_t* ae = rowind + colptr[j + 1];
    const idx_t* b = t.rowind.data() + t.colptr[j];
    const idx_t* be = t.rowind.data() + t.colptr[j + 1];
    while (a != ae || b != be) {            // merge two ascending lists
      idx_t r;
      if (b == be || (a != ae && *a < *b)) r = *a++;
      else if (a == ae || *b < *a) r = *b++;
      else { r = *a++; ++b; }
      if (keep_diagonal || r != j) s.rowind.push_back(r);
    }
    s.colptr[j + 1] = (idx_t)s.rowind.size();
  }
  return s;
}

Pattern permute_symmetric(const Pattern& s, const std::vector<idx_t>& perm) {
  const idx_t n = s.n;
  std::vector<idx_t> inv(n);
  for (idx_t k = 0; k < n; ++k) inv[perm[k]] = k;
  Pattern b;
  b.n = n;
  b.colptr.resize(n + 1);
  b.colptr[0] = 0;
  for (idx_t j = 0; j < n; ++j) b.colptr[j + 1] = b.colptr[j] + (s.colptr[perm[j] + 1] - s.colptr[perm[j]]);
  b.rowind.resize(b.colptr[n]);
  for (idx_t j = 0; j < n; ++j) {
    idx_t* out = b.rowind.data() + b.colptr[j];
    idx_t cnt = 0;
    for (idx_t p = s.colptr[perm[j]]; p < s.colptr[perm[j] + 1]; ++p) out[cnt++] = inv[s.rowind[p]];
    std::sort(out, out + cnt);
  }
  return b;
}

// ---------------------------------------------------------------------------
// approximate minimum degree
// ---------------------------------------------------------------------------
namespace {

inline idx_t flipped(idx_t x) { return -x - 2; }

class MinimumDegree {
 public:
  MinimumDegree(const Pattern& g, double dense) : n_(g.n) {
    const idx_t cnz = g.colptr[n_];
    adj_.assign(std::max<idx_t>(cnz + cnz / 5 + 2 * n_, 1), 0);
    std::copy(g.rowind.begin(), g.rowind.begin() + cnz, adj_.begin());
    used_ = cnz;
    dense_limit_ = std::min<idx_t>(n_ - 2, (idx_t)std::floor(std::max(16.0, dense * std::sqrt((double)n_))));
    const size_t sz = (size_t)n_ + 1;
    len_.resize(sz); nv_.resize(sz); next_.resize(sz); head_.resize(sz); elen_.resize(sz);
    deg_.resize(sz); w_.resize(sz); hhead_.resize(sz); last_.resize(sz); ptr_.resize(sz);
    for (idx_t k = 0; k < n_; ++k) { len_[k] = g.colptr[k + 1] - g.colptr[k]; ptr_[k] = g.colptr[k]; }
    ptr_[n_] = g.colptr[n_];
    len_[n_] = 0;
  }

  std::vector<idx_t> run() {
    initialize();
    while (eliminated_ < n_) {
      const idx_t k = select_pivot();
      const idx_t elenk = elen_[k];
      idx_t nvk = nv_[k];
      eliminated_ += nvk;
      if (elenk > 0 && used_ + mindeg_ >= (idx_t)adj_.size()) compact();
      idx_t pk1, pk2, dk;
      form_element(k, elenk, nvk, pk1, pk2, dk);
      external_degrees(pk1, pk2);
      update_degrees(k, pk1, pk2, dk, nvk);
      deg_[k] = dk;
      lemax_ = std::max(lemax_, dk);
      mark_ = clear_marks(mark_ + lemax_);
      detect_supervariables(pk1, pk2);
      finalize_element(k, elenk, nvk, pk1, pk2, dk);
    }
    return assembly_postorder();
  }

 private:
  idx_t clear_marks(idx_t mark) {
    if (mark < 2 || mark + lemax_ < 0) {
      for (idx_t k = 0; k < n_; ++k)
        if (w_[k] != 0) w_[k] = 1;
      mark = 2;
    }
    return mark;
  }

  void list_insert(idx_t i, idx_t d) {      // push i onto degree list d
    if (head_[d] != -1) last_[head_[d]] = i;
    next_[i] = head_[d];
    head_[d] = i;
  }

  void initialize() {
    for (idx_t i = 0; i <= n_; ++i) {
      head_[i] = last_[i] = next_[i] = hhead_[i] = -1;
      nv_[i] = 1;
      w_[i] = 1;
      elen_[i] = 0;
      deg_[i] = len_[i];
    }
    mark_ = clear_marks(0);
    elen_[n_] = -2;
    ptr_[n_] = -1;
    w_[n_] = 0;
    for (idx_t i = 0; i < n_; ++i) {
      const idx_t d = deg_[i];
      if (d == 0) {                          // isolated: eliminate now
        elen_[i] = -2;
        ++eliminated_;
        ptr_[i] = -1;
        w_[i] = 0;
      } else if (d > dense_limit_) {         // dense: absorbed into the root
        nv_[i] = 0;
        elen_[i] = -1;
        ++eliminated_;
        ptr_[i] = flipped(n_);
        ++nv_[n_];
      } else {
        list_insert(i, d);
      }
    }
  }

  idx_t select_pivot() {
    idx_t k = -1;
    for (; mindeg_ < n_; ++mindeg_) {
      k = head_[mindeg_];
      if (k != -1) break;
    }
    if (next_[k] != -1) last_[next_[k]] = -1;
    head_[mindeg_] = next_[k];
    return k;
  }

  void compact() {                           // garbage-collect the adjacency store
    for (idx_t j = 0; j < n_; ++j) {
      const idx_t p = ptr_[j];
      if (p >= 0) { ptr_[j] = adj_[p]; adj_[p] = flipped(j); }
    }
    idx_t dst = 0, src = 0;
    while (src < used_) {
      const idx_t j = flipped(adj_[src++]);
      if (j >= 0) {
        adj_[dst] = ptr_[j];
        ptr_[j] = dst++;
        for (idx_t t = 0; t < len_[j] - 1; ++t) adj_[dst++] = adj_[src++];
      }
    }
    used_ = dst;
  }

  void form_element(idx_t k, idx_t elenk, idx_t nvk, idx_t& pk1, idx_t& pk2, idx_t& dk) {
    dk = 0;
    nv_[k] = -nvk;
    idx_t p = ptr_[k];
    pk1 = (elenk == 0) ? p : used_;
    pk2 = pk1;
    for (idx_t k1 = 1; k1 <= elenk + 1; ++k1) {
      idx_t e, pj, ln;
      if (k1 > elenk) { e = k; pj = p; ln = len_[k] - elenk; }
      else { e = adj_[p++]; pj = ptr_[e]; ln = len_[e]; }
      for (idx_t t = 0; t < ln; ++t) {
        const idx_t i = adj_[pj++];
        const idx_t nvi = nv_[i];
        if (nvi <= 0) continue;
        dk += nvi;
        nv_[i] = -nvi;
        adj_[pk2++] = i;
        if (next_[i] != -1) last_[next_[i]] = last_[i];
        if (last_[i] != -1) next_[last_[i]] = next_[i];
        else head_[deg_[i]] = next_[i];
      }
      if (e != k) { ptr_[e] = flipped(k); w_[e] = 0; }
    }
    if (elenk != 0) used_ = pk2;
    deg_[k] = dk;
    ptr_[k] = pk1;
    len_[k] = pk2 - pk1;
    elen_[k] = -2;
  }

  void external_degrees(idx_t pk1, idx_t pk2) {
    mark_ = clear_marks(mark_);
    for (idx_t pk = pk1; pk < pk2; ++pk) {
      const idx_t i = adj_[pk];
      const idx_t eln = elen_[i];
      if (eln <= 0) continue;
      const idx_t nvi = -nv_[i];
      const idx_t wnvi = mark_ - nvi;
      for (idx_t p = ptr_[i]; p <= ptr_[i] + eln - 1; ++p) {
        const idx_t e = adj_[p];
        if (w_[e] >= mark_) w_[e] -= nvi;
        else if (w_[e] != 0) w_[e] = deg_[e] + wnvi;
      }
    }
  }

  void update_degrees(idx_t k, idx_t pk1, idx_t pk2, idx_t& dk, idx_t& nvk) {
    for (idx_t pk = pk1; pk < pk2; ++pk) {
      const idx_t i = adj_[pk];
      const idx_t p1 = ptr_[i];
      const idx_t p2 = p1 + elen_[i] - 1;
      idx_t pn = p1, h = 0, d = 0;
      for (idx_t p = p1; p <= p2; ++p) {
        const idx_t e = adj_[p];
        if (w_[e] == 0) continue;
        const idx_t dext = w_[e] - mark_;
        if (dext > 0) { d += dext; adj_[pn++] = e; h += e; }
        else { ptr_[e] = flipped(k); w_[e] = 0; }     // aggressive absorption
      }
      elen_[i] = pn - p1 + 1;
      const idx_t p3 = pn;
      const idx_t p4 = p1 + len_[i];
      for (idx_t p = p2 + 1; p < p4; ++p) {
        const idx_t j = adj_[p];
        const idx_t nvj = nv_[j];
        if (nvj <= 0) continue;
        d += nvj;
        adj_[pn++] = j;
        h += j;
      }
      if (d == 0) {                                      // mass elimination
        ptr_[i] = flipped(k);
        const idx_t nvi = -nv_[i];
        dk -= nvi;
        nvk += nvi;
        eliminated_ += nvi;
        nv_[i] = 0;
        elen_[i] = -1;
      } else {
        deg_[i] = std::min(deg_[i], d);
        adj_[pn] = adj_[p3];
        adj_[p3] = adj_[p1];
        adj_[p1] = k;
        len_[i] = pn - p1 + 1;
        h %= n_;
        next_[i] = hhead_[h];
        hhead_[h] = i;
        last_[i] = h;
      }
    }
  }

  void detect_supervariables(idx_t pk1, idx_t pk2) {
    for (idx_t pk = pk1; pk < pk2; ++pk) {
      idx_t i = adj_[pk];
      if (nv_[i] >= 0) continue;
      const idx_t h = last_[i];
      i = hhead_[h];
      hhead_[h] = -1;
      for (; i != -1 && next_[i] != -1; i = next_[i], ++mark_) {
        const idx_t ln = len_[i], eln = elen_[i];
        for (idx_t p = ptr_[i] + 1; p <= ptr_[i] + ln - 1; ++p) w_[adj_[p]] = mark_;
        idx_t jlast = i;
        for (idx_t j = next_[i]; j != -1;) {
          bool same = len_[j] == ln && elen_[j] == eln;
          for (idx_t p = ptr_[j] + 1; same && p <= ptr_[j] + ln - 1; ++p) same = (w_[adj_[p]] == mark_);
          if (same) {                                    // j merges into i
            ptr_[j] = flipped(i);
            nv_[i] += nv_[j];
            nv_[j] = 0;
            elen_[j] = -1;
            j = next_[j];
            next_[jlast] = j;
          } else {
            jlast = j;
            j = next_[j];
          }
        }
      }
    }
  }

  void finalize_element(idx_t k, idx_t elenk, idx_t nvk, idx_t pk1, idx_t pk2, idx_t dk) {
    idx_t p = pk1;
    for (idx_t pk = pk1; pk < pk2; ++pk) {
      const idx_t i = adj_[pk];
      const idx_t nvi = -nv_[i];
      if (nvi <= 0) continue;
      nv_[i] = nvi;
      const idx_t d = std::min(deg_[i] + dk - nvi, n_ - eliminated_ - nvi);
      list_insert(i, d);
      last_[i] = -1;
      mindeg_ = std::min(mindeg_, d);
      deg_[i] = d;
      adj_[p++] = i;
    }
    nv_[k] = nvk;
    len_[k] = p - pk1;
    if (len_[k] == 0) { ptr_[k] = -1; w_[k] = 0; }
    if (elenk != 0) used_ = p;
  }

  std::vector<idx_t> assembly_postorder() {
    for (idx_t i = 0; i < n_; ++i) ptr_[i] = flipped(ptr_[i]);   // parent in assembly tree
    for (idx_t j = 0; j <= n_; ++j) head_[j] = -1;
    for (idx_t j = n_; j >= 0; --j) {                             // variables under their element
      if (nv_[j] > 0) continue;
      next_[j] = head_[ptr_[j]];
      head_[ptr_[j]] = j;
    }
    for (idx_t e = n_; e >= 0; --e) {                             // elements under their parent
      if (nv_[e] <= 0 || ptr_[e] == -1) continue;
      next_[e] = head_[ptr_[e]];
      head_[ptr_[e]] = e;
    }
    std::vector<idx_t> order(n_ + 1), stack(n_ + 1);
    idx_t k = 0;
    for (idx_t root = 0; root <= n_; ++root) {
      if (ptr_[root] != -1) continue;
      idx_t top = 0;
      stack[0] = root;
      while (top >= 0) {
        const idx_t p = stack[top];
        const idx_t c = head_[p];
        if (c == -1) { --top; order[k++] = p; }
        else { head_[p] = next_[c]; stack[++top] = c; }
      }
    }
    order.resize(n_);
    return order;
  }

  idx_t n_;
  std::vector<idx_t> adj_;
  idx_t used_ = 0, dense_limit_ = 0, eliminated_ = 0, mindeg_ = 0, lemax_ = 0, mark_ = 0;
  std::vector<idx_t> len_, nv_, next_, head_, elen_, deg_, w_, hhead_, last_, ptr_;
};

}  // namespace

std::vector<idx_t> amd_order(const Pattern& sym, double dense) {
  if (sym.n == 0) return {};
  if (sym.n == 1) return {0};
  MinimumDegree md(sym, dense);
  return md.run();
}

std::vector<idx_t> amd_order_sym(idx_t n, const idx_t* colptr, const idx_t* rowind, double dense) {
  if (n == 0) return {};
  if (n == 1) return {0};
  return amd_order(symmetrize(n, colptr, rowind, false), dense);
}

std::vector<idx_t> colamd_order(idx_t m, idx_t n, const idx_t* colptr, const idx_t* rowind, double dense) {
  std::vector<idx_t> order(n);
  if (n <= 1) {
    for (idx_t j = 0; j < n; ++j) order[j] = j;
    return order;
  }
  const Pattern rows = transpose(m, n, colptr, rowind);     // rows.colptr[r]: row r of A
  const idx_t limit = (idx_t)std::floor(std::min((double)(n - 2), std::max(16.0, dense * std::sqrt((double)n))));
  Pattern g;                                                // column graph of A^T A
  g.n = n;
  g.colptr.assign(n + 1, 0);
  std::vector<idx_t> seen(n, -1), col;
  for (idx_t j = 0; j < n; ++j) {
    col.clear();
    for (idx_t p = colptr[j]; p < colptr[j + 1]; ++p) {
      const idx_t r = rowind[p];
      if (rows.colptr[r + 1] - rows.colptr[r] > limit) continue;   // dense row dropped
      for (idx_t q = rows.colptr[r]; q < rows.colptr[r + 1]; ++q) {
        const idx_t i = rows.rowind[q];
        if (seen[i] == j) continue;
        seen[i] = j;
        if (i != j) col.push_back(i);
      }
    }
    std::sort(col.begin(), col.end());
    g.rowind.insert(g.rowind.end(), col.begin(), col.end());
    g.colptr[j + 1] = (idx_t)g.rowind.size();
  }
  return amd_order(g, dense);
}

// In the element type's arithmetic: R = real(Tv) accumulates (Float32 sums
// for a Float32 matrix, as the reference's generic code does).
template <typename T>
static void row_scaling_t(idx_t n, idx_t nnz, const idx_t* rowind, const T* nzval, int kind, T* rs) {
  std::fill(rs, rs + n, T(1));
  if (kind == 0) return;
  std::vector<T> acc(n, T(0));
  if (kind == 1) {
    for (idx_t p = 0; p < nnz; ++p) acc[rowind[p]] += std::fabs(nzval[p]);
  } else {
    for (idx_t p = 0; p < nnz; ++p) {
      const T v = std::fabs(nzval[p]);
      T& a = acc[rowind[p]];
      a = v > a ? v : a;
    }
  }
  for (idx_t i = 0; i < n; ++i) rs[i] = acc[i] > 0 ? T(1) / acc[i] : T(1);
}

void row_scaling(idx_t n, idx_t nnz, const idx_t* rowind, const double* nzval, int kind, double* rs) {
  row_scaling_t(n, nnz, rowind, nzval, kind, rs);
}

void row_scaling(idx_t n, idx_t nnz, const idx_t* rowind, const float* nzval, int kind, float* rs) {
  row_scaling_t(n, nnz, rowind, nzval, kind, rs);
}

// ---------------------------------------------------------------------------
// elimination tree, postorder, column counts, supernodes
// ---------------------------------------------------------------------------
static std::vector<idx_t> elimination_tree(const Pattern& s) {
  const idx_t n = s.n;
  std::vector<idx_t> parent(n, -1), ancestor(n, -1);
  for (idx_t k = 0; k < n; ++k) {
    for (idx_t p = s.colptr[k]; p < s.colptr[k + 1]; ++p) {
      for (idx_t i = s.rowind[p]; i != -1 && i < k;) {
        const idx_t up = ancestor[i];
        ancestor[i] = k;
        if (up == -1) parent[i] = k;
        i = up;
      }
    }
  }
  return parent;
}

static std::vector<idx_t> tree_postorder(const std::vector<idx_t>& parent) {
  const idx_t n = (idx_t)parent.size();
  std::vector<idx_t> first_child(n, -1), sibling(n, -1), order(n), stack(n);
  for (idx_t j = n - 1; j >= 0; --j) {       // children lists in ascending order
    const idx_t p = parent[j];
    if (p == -1) continue;
    sibling[j] = first_child[p];
    first_child[p] = j;
  }
  idx_t k = 0;
  for (idx_t root = 0; root < n; ++root) {
    if (parent[root] != -1) continue;
    idx_t top = 0;
    stack[0] = root;
    while (top >= 0) {
      const idx_t p = stack[top];
      const idx_t c = first_child[p];
      if (c == -1) { --top; order[k++] = p; }
      else { first_child[p] = sibling[c]; stack[++top] = c; }
    }
  }
  return order;
}

// Column counts of the Cholesky factor of a symmetric pattern whose
// elimination tree is already postordered (parent[j] > j).  Gilbert, Ng &
// Peyton (1994): each entry A(i,j), i > j, is in the row-subtree skeleton iff
// j is a leaf of row i's subtree; overlaps are removed at least common
// ancestors found by path-compressed union-find.  Returns |L(:,j)| - 1.
static std::vector<idx_t> column_counts(const Pattern& s, const std::vector<idx_t>& parent) {
  const idx_t n = s.n;
  std::vector<idx_t> delta(n), first(n, -1), maxfirst(n, -1), prevleaf(n, -1), ancestor(n);
  for (idx_t k = 0; k < n; ++k) {            // identity is a postorder here
    idx_t j = k;
    delta[j] = (first[j] == -1) ? 1 : 0;
    for (; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
  }
  for (idx_t i = 0; i < n; ++i) ancestor[i] = i;
  for (idx_t j = 0; j < n; ++j) {
    if (parent[j] != -1) --delta[parent[j]];
    for (idx_t p = s.colptr[j]; p < s.colptr[j + 1]; ++p) {
      const idx_t i = s.rowind[p];
      if (i <= j || first[j] <= maxfirst[i]) continue;   // j not a new leaf of row i
      maxfirst[i] = first[j];
      const idx_t jprev = prevleaf[i];
      prevleaf[i] = j;
      ++delta[j];
      if (jprev == -1) continue;                          // first leaf of row i
      idx_t q = jprev;
      while (q != ancestor[q]) q = ancestor[q];
      for (idx_t t = jprev; t != q;) {                    // path compression
        const idx_t up = ancestor[t];
        ancestor[t] = q;
        t = up;
      }
      --delta[q];
    }
    if (parent[j] != -1) ancestor[j] = parent[j];
  }
  for (idx_t j = 0; j < n; ++j)
    if (parent[j] != -1) delta[parent[j]] += delta[j];
  for (idx_t j = 0; j < n; ++j) --delta[j];                // drop the diagonal
  return delta;
}

idx_t SymbolicMF::predicted_fill() const {
  idx_t nl = n;
  for (idx_t j = 0; j < n; ++j) nl += colcount[j];
  return 2 * nl;
}

SymbolicMF symbolic_mf(idx_t n, const idx_t* colptr, const idx_t* rowind, const idx_t* q) {
  SymbolicMF S;
  S.n = n;
  const Pattern sym = symmetrize(n, colptr, rowind, false);
  std::vector<idx_t> order;
  if (q) order.assign(q, q + n);
  else order = amd_order(sym, 10.0);
  const Pattern p1 = permute_symmetric(sym, order);
  const std::vector<idx_t> post = tree_postorder(elimination_tree(p1));
  S.qf.resize(n);
  for (idx_t k = 0; k < n; ++k) S.qf[k] = order[post[k]];
  const Pattern pf = permute_symmetric(p1, post);
  S.parent = elimination_tree(pf);
  S.colcount = column_counts(pf, S.parent);

  // fundamental supernodes: j continues j-1's supernode iff j-1 is j's only
  // child and the structures nest exactly.
  std::vector<idx_t> nchild(n, 0);
  for (idx_t j = 0; j < n; ++j)
    if (S.parent[j] != -1) ++nchild[S.parent[j]];
  S.super_of.resize(n);
  for (idx_t j = 0; j < n; ++j) {
    const bool extend = j > 0 && S.parent[j - 1] == j && nchild[j] == 1 && S.colcount[j - 1] == S.colcount[j] + 1;
    if (!extend) S.sstart.push_back(j);
    S.super_of[j] = (idx_t)S.sstart.size() - 1;
  }
  S.sstart.push_back(n);
  const idx_t ns = S.nsuper();

  // child supernodes (ascending), all attached to the first column
  std::vector<idx_t> nkids(ns + 1, 0);
  for (idx_t s = 0; s < ns; ++s) {
    const idx_t p = S.parent[S.sstart[s + 1] - 1];
    if (p != -1) ++nkids[S.super_of[p] + 1];
  }
  S.child_ptr.assign(ns + 1, 0);
  for (idx_t s = 0; s < ns; ++s) S.child_ptr[s + 1] = S.child_ptr[s] + nkids[s + 1];
  S.child_idx.resize(S.child_ptr[ns]);
  {
    std::vector<idx_t> fill(S.child_ptr.begin(), S.child_ptr.end() - 1);
    for (idx_t s = 0; s < ns; ++s) {
      const idx_t p = S.parent[S.sstart[s + 1] - 1];
      if (p != -1) S.child_idx[fill[S.super_of[p]]++] = s;
    }
  }

  // update sets: rows > last column of the supernode, from the first column
  // of A and the children's update sets.
  S.upd_ptr.assign(ns + 1, 0);
  for (idx_t s = 0; s < ns; ++s) S.upd_ptr[s + 1] = S.upd_ptr[s] + S.colcount[S.sstart[s + 1] - 1];
  S.upd_idx.resize(S.upd_ptr[ns]);
  std::vector<idx_t> marker(n, -1);
  for (idx_t s = 0; s < ns; ++s) {
    const idx_t c1 = S.sstart[s], c2 = S.sstart[s + 1] - 1;
    idx_t* out = S.upd_idx.data() + S.upd_ptr[s];
    idx_t cnt = 0;
    const idx_t cap = S.upd_ptr[s + 1] - S.upd_ptr[s];
    auto take = [&](idx_t i) {
      if (i > c2 && marker[i] != s) {
        if (cnt >= cap) throw std::runtime_error("symbolic: update set exceeds its column count");
        marker[i] = s;
        out[cnt++] = i;
      }
    };
    for (idx_t j = c1; j <= c2; ++j)
      for (idx_t p = pf.colptr[j]; p < pf.colptr[j + 1]; ++p) take(pf.rowind[p]);
    for (idx_t c = S.child_ptr[s]; c < S.child_ptr[s + 1]; ++c) {
      const idx_t k = S.child_idx[c];
      for (idx_t p = S.upd_ptr[k]; p < S.upd_ptr[k + 1]; ++p) take(S.upd_idx[p]);
    }
    if (cnt != cap) throw std::runtime_error("symbolic: update set smaller than its column count");
    std::sort(out, out + cnt);
  }
  return S;
}

// Amalgamation decisions (the reference has none).  Supernodes are taken
// bottom-up; a supernode whose columns end right before its parent's (the
// parent's last child in postorder) merges into it when the merged supernode
// stays small or the logical zeros it stores stay few (thresholds in the
// style of CHOLMOD's nrelax / zrelax).  The merged supernode keeps the
// parent's update set, which contains the child's, so every merged front
// holds its children's contribution blocks.  No merged supernode exceeds
// max_pivots columns.  Returns one flag per supernode: merged into its
// parent.  Inputs 0-based: parent (etree, -1 = root) of the n columns,
// sstart (ns+1), upd_ptr (ns+1).
std::vector<char> amalgamation_marks(idx_t n, const idx_t* parent, idx_t ns, const idx_t* sstart,
                                     const idx_t* upd_ptr, idx_t max_pivots) {
  std::vector<char> merged(ns > 0 ? ns : 0, 0);
  if (ns < 2) return merged;
  std::vector<idx_t> super_of(n), sparent(ns, -1), gnp(ns), gnu(ns);
  for (idx_t s = 0; s < ns; ++s)
    for (idx_t j = sstart[s]; j < sstart[s + 1]; ++j) super_of[j] = s;
  std::vector<double> gz(ns, 0.0);
  for (idx_t s = 0; s < ns; ++s) {
    const idx_t p = parent[sstart[s + 1] - 1];
    sparent[s] = p == -1 ? -1 : super_of[p];
    gnp[s] = sstart[s + 1] - sstart[s];
    gnu[s] = upd_ptr[s + 1] - upd_ptr[s];
  }
  auto tri = [](double a, double u) { return a * (a + 1) / 2 + a * u; };
  for (idx_t s = 0; s < ns; ++s) {
    const idx_t p = sparent[s];
    if (p < 0 || sstart[s + 1] != sstart[p]) continue;   // not adjacent to the parent
    const double npc = (double)gnp[s], nuc = (double)gnu[s], npp = (double)gnp[p], nup = (double)gnu[p];
    const double extra = npc * (npp + nup - nuc);
    const double z = gz[s] + gz[p] + extra, tot = tri(npc + npp, nup);
    const double npm = npc + npp, zf = tot > 0 ? z / tot : 0.0;
    if (npm > (double)max_pivots) continue;
    const bool ok = npm <= 4 || (npm <= 16 && zf < 0.8) || (npm <= 48 && zf < 0.1) || zf < 0.05;
    if (!ok) continue;
    merged[s] = 1;
    gnp[p] += gnp[s];
    gz[p] = z;
  }
  return merged;
}

// Relaxed amalgamation (opt-in): the supernodes of amalgamation_marks become
// the factor's supernodes, so the child's columns gain explicit zeros.
void relax_supernodes(SymbolicMF& S) {
  const idx_t ns = S.nsuper();
  if (ns < 2) return;
  const std::vector<char> merged =
      amalgamation_marks(S.n, S.parent.data(), ns, S.sstart.data(), S.upd_ptr.data(), S.n);
  // rebuild the partition: a group ends at a supernode that is not merged
  std::vector<idx_t> sstart, upd_ptr{0}, upd_idx;
  std::vector<idx_t> group_of(ns);
  idx_t first = 0;
  for (idx_t s = 0; s < ns; ++s) {
    group_of[s] = (idx_t)sstart.size();
    if (merged[s]) continue;
    sstart.push_back(S.sstart[first]);
    upd_idx.insert(upd_idx.end(), S.upd_idx.begin() + S.upd_ptr[s], S.upd_idx.begin() + S.upd_ptr[s + 1]);
    upd_ptr.push_back((idx_t)upd_idx.size());
    first = s + 1;
  }
  sstart.push_back(S.n);
  const idx_t ng = (idx_t)sstart.size() - 1;
  S.sstart.swap(sstart);
  S.upd_ptr.swap(upd_ptr);
  S.upd_idx.swap(upd_idx);
  for (idx_t g = 0; g < ng; ++g) {
    const idx_t c2 = S.sstart[g + 1] - 1, nu = S.upd_ptr[g + 1] - S.upd_ptr[g];
    for (idx_t j = S.sstart[g]; j <= c2; ++j) {
      S.super_of[j] = g;
      S.colcount[j] = (c2 - j) + nu;
    }
  }
  std::vector<idx_t> nkids(ng + 1, 0);
  for (idx_t g = 0; g < ng; ++g) {
    const idx_t p = S.parent[S.sstart[g + 1] - 1];
    if (p != -1) ++nkids[S.super_of[p] + 1];
  }
  S.child_ptr.assign(ng + 1, 0);
  for (idx_t g = 0; g < ng; ++g) S.child_ptr[g + 1] = S.child_ptr[g] + nkids[g + 1];
  S.child_idx.assign(S.child_ptr[ng], 0);
  std::vector<idx_t> fill(S.child_ptr.begin(), S.child_ptr.end() - 1);
  for (idx_t g = 0; g < ng; ++g) {
    const idx_t p = S.parent[S.sstart[g + 1] - 1];
    if (p != -1) S.child_idx[fill[S.super_of[p]]++] = g;
  }
}

SymbolicMF concat_symbolic(const std::vector<SymbolicMF>& parts) {
  SymbolicMF S;
  idx_t n = 0, ns = 0, nu = 0, nc = 0;
  for (const SymbolicMF& P : parts) {
    n += P.n;
    ns += P.nsuper();
    nu += (idx_t)P.upd_idx.size();
    nc += (idx_t)P.child_idx.size();
  }
  S.n = n;
  S.qf.reserve(n);
  S.parent.reserve(n);
  S.colcount.reserve(n);
  S.super_of.reserve(n);
  S.sstart.reserve(ns + 1);
  S.upd_ptr.reserve(ns + 1);
  S.upd_idx.reserve(nu);
  S.child_ptr.reserve(ns + 1);
  S.child_idx.reserve(nc);
  idx_t co = 0, so = 0, uo = 0, ko = 0;   // column, supernode, update entry, child entry offsets
  for (const SymbolicMF& P : parts) {
    for (idx_t j = 0; j < P.n; ++j) {
      S.qf.push_back(P.qf[j] + co);
      S.parent.push_back(P.parent[j] < 0 ? -1 : P.parent[j] + co);
      S.colcount.push_back(P.colcount[j]);
      S.super_of.push_back(P.super_of[j] + so);
    }
    const idx_t pns = P.nsuper();
    for (idx_t k = 0; k < pns; ++k) {
      S.sstart.push_back(P.sstart[k] + co);
      S.upd_ptr.push_back(P.upd_ptr[k] + uo);
      S.child_ptr.push_back(P.child_ptr[k] + ko);
    }
    for (idx_t u : P.upd_idx) S.upd_idx.push_back(u + co);
    for (idx_t c : P.child_idx) S.child_idx.push_back(c + so);
    co += P.n;
    so += pns;
    uo += (idx_t)P.upd_idx.size();
    ko += (idx_t)P.child_idx.size();
  }
  S.sstart.push_back(n);
  S.upd_ptr.push_back(uo);
  S.child_ptr.push_back(ko);
  return S;
}

void factor_colptrs(const SymbolicMF& S, std::vector<idx_t>& lp, std::vector<idx_t>& up) {
  const idx_t n = S.n, ns = S.nsuper();
  lp.assign(n + 1, 0);
  up.assign(n + 1, 0);
  for (idx_t s = 0; s < ns; ++s) {
    const idx_t c1 = S.sstart[s], c2 = S.sstart[s + 1] - 1, np = c2 - c1 + 1;
    const idx_t nu = S.upd_ptr[s + 1] - S.upd_ptr[s];
    for (idx_t j = c1; j <= c2; ++j) {
      lp[j + 1] = 1 + (c2 - j) + nu;       // diagonal, pivots below, update rows
      up[j + 1] += j - c1 + 1;             // own upper triangle
    }
    for (idx_t p = S.upd_ptr[s]; p < S.upd_ptr[s + 1]; ++p) up[S.upd_idx[p] + 1] += np;
  }
  for (idx_t j = 0; j < n; ++j) {
    lp[j + 1] += lp[j];
    up[j + 1] += up[j];
  }
}

}  // namespace mfgpu
