// symbolic.h -- host-side ordering and symbolic analysis of libmfgpu.
//
// Integer host code whose output is identical to PureUMFPACK.jl's:
//   row scaling          src/scaling.jl:92-126
//   AMD / COLAMD         src/amd.jl:84-104, 141-148, 183-188, 191-539
//   symbolic_mf          src/symbolic.jl:15-226 (etree, postorder, fundamental
//                        supernodes, column structure of each supernode)
//   _factor_colptrs      src/multifrontal.jl:73-104
// All indices here are 0-based; the C ABI converts to/from 1-based.
#pragma once

#include <cstdint>
#include <vector>

namespace mfgpu {

using idx_t = int64_t;

struct Pattern {                 // CSC pattern, rows ascending in each column
  idx_t n = 0;                   // number of columns
  std::vector<idx_t> colptr;     // n+1
  std::vector<idx_t> rowind;
};

// Pattern of A + A^T, rows sorted, optionally without the diagonal.
Pattern symmetrize(idx_t n, const idx_t* colptr, const idx_t* rowind, bool keep_diagonal);
// B = S[perm, perm] for a symmetric pattern S (new column j = old column perm[j]).
Pattern permute_symmetric(const Pattern& s, const std::vector<idx_t>& perm);

// Approximate minimum degree on a symmetric pattern without diagonal.
std::vector<idx_t> amd_order(const Pattern& sym, double dense);
// AMD on A+A^T (amd_order_sym) and on the A^T A column graph (colamd_order).
std::vector<idx_t> amd_order_sym(idx_t n, const idx_t* colptr, const idx_t* rowind, double dense);
std::vector<idx_t> colamd_order(idx_t m, idx_t n, const idx_t* colptr, const idx_t* rowind, double dense);

void row_scaling(idx_t n, idx_t nnz, const idx_t* rowind, const double* nzval, int kind, double* rs);
void row_scaling(idx_t n, idx_t nnz, const idx_t* rowind, const float* nzval, int kind, float* rs);

// The symbolic factorization in supernodal form.  Column j of supernode s
// (first_col[s] <= j <= last) has the L row structure {j+1..last} followed by
// the update set upd(s) = upd_idx[upd_ptr[s] .. upd_ptr[s+1]).
struct SymbolicMF {
  idx_t n = 0;
  std::vector<idx_t> qf;         // final column order (AMD o postorder)
  std::vector<idx_t> parent;     // elimination tree of A[qf,qf]; -1 = root
  std::vector<idx_t> colcount;   // |colstruct[j]| (below-diagonal count)
  std::vector<idx_t> sstart;     // nsuper+1 supernode column boundaries
  std::vector<idx_t> super_of;   // column -> supernode
  std::vector<idx_t> upd_ptr;    // nsuper+1
  std::vector<idx_t> upd_idx;    // update set of each supernode (sorted)
  std::vector<idx_t> child_ptr;  // nsuper+1, child supernodes in ascending order
  std::vector<idx_t> child_idx;
  idx_t nsuper() const { return (idx_t)sstart.size() - 1; }
  idx_t predicted_fill() const;  // nnz(L) + nnz(U), both diagonals counted
};

// symbolic_mf(A; q): q (0-based) or nullptr for AMD.
SymbolicMF symbolic_mf(idx_t n, const idx_t* colptr, const idx_t* rowind, const idx_t* q);

// Independent systems as one block-diagonal forest: the parts' symbolic
// objects concatenated with column, supernode and update-set offsets.  This
// is the block-diagonal matrix's own symbolic_mf with the concatenated
// orders: its postorder visits the trees root by root in column order, so
// every system keeps its columns together and its own postorder, and no
// fundamental supernode spans two systems.
SymbolicMF concat_symbolic(const std::vector<SymbolicMF>& parts);

// Amalgamation decisions: flag s = supernode s merges into its parent; no
// merged supernode gets more than max_pivots columns.
std::vector<char> amalgamation_marks(idx_t n, const idx_t* parent, idx_t ns, const idx_t* sstart,
                                     const idx_t* upd_ptr, idx_t max_pivots);

// Opt-in relaxed amalgamation of the supernodes (changes the factors'
// structure: merged columns store explicit zeros).
void relax_supernodes(SymbolicMF& s);

// _factor_colptrs: 0-based Lcolptr / Ucolptr (n+1 each).
void factor_colptrs(const SymbolicMF& s, std::vector<idx_t>& lcolptr, std::vector<idx_t>& ucolptr);

}  // namespace mfgpu
