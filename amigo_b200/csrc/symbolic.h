// Host symbolic analysis for the supernodal multifrontal LDL^T.
//
// Reproduces, bit for bit, the ordering, elimination tree, fundamental and
// relaxed supernode partition and per-supernode contribution rows that the
// reference computes in SparseLDL::symbolic_analysis
// (include/sparse_ldl.h:2222-2376), so that front structures, delayed-pivot
// behaviour and inertia line up with the reference exactly.
#pragma once

#include <cstdint>
#include <vector>

namespace b200ldl {

// NestedDissection..Natural as the reference numbers them (nested
// dissection without METIS is the identity there); GraphNd is our own
// nested dissection (nd_order).
enum class Ordering : int {
  NestedDissection = 0,
  Amd = 1,
  MultiColor = 2,
  Natural = 3,
  GraphNd = 4
};

struct Symbolic {
  int n = 0;
  // ordering: iperm[original] = permuted index, perm[permuted] = original.
  // Identity for the natural ordering.
  std::vector<int> perm, iperm;
  bool permuted = false;

  // relaxed supernodes (nodes), numbered in the reference's order
  int num_nodes = 0;
  std::vector<int> node_ptr;      // [num_nodes+1]
  std::vector<int> node_to_var;   // [n], original numbering
  std::vector<int> children_ptr;  // [num_nodes+2]; roots in [num_nodes, num_nodes+1)
  std::vector<int> children;      // [num_nodes]
  std::vector<int> contrib_ptr;   // [num_nodes+1]
  std::vector<int> contrib_rows;  // original numbering, increasing permuted index
  std::vector<int> parent;        // [num_nodes], -1 for roots
};

// Ordering of the full symmetric pattern (rowp/cols: CSR with or without the
// diagonal, any column order).
void compute_ordering(Ordering order, int n, const int* rowp, const int* cols,
                      std::vector<int>& perm, std::vector<int>& iperm);

// Nested dissection of the full symmetric pattern without METIS; perm[k] =
// k-th vertex eliminated.
void nd_order(int n, const int* rowp, const int* cols, int* perm);

// Approximate minimum degree on a prepared quotient-graph CSR (diagonal
// present, sorted, unique). rowp/cols are modified. perm[k] = k-th pivot.
int amd_order(int n, int* rowp, int* cols, int* perm);

// Variable elimination tree in the permuted numbering, its postorder and the
// column counts of L (diagonal included).
void etree_postorder_colcount(int n, const int* rowp, const int* cols,
                              const int* perm, const int* iperm,
                              std::vector<int>& parent, std::vector<int>& post,
                              std::vector<int>& colcount);

// Full symbolic phase.
Symbolic analyze(Ordering order, int n, const int* rowp, const int* cols);

// Independent systems as one forest: variables, supernodes and contribution
// rows of each part shifted past the parts before it, every part's roots
// listed at the end; node_sys[k] = the part supernode k belongs to.
Symbolic merge_symbolic(const std::vector<Symbolic>& parts, std::vector<int>& node_sys);

}  // namespace b200ldl
