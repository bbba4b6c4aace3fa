/*
 * Test oracle: a C-ABI around the reference's own header-only SparseLDL
 * (include/sparse_ldl.h, include/block_amd.h, include/ordering_utils.h of
 * Mersoltane/amigo), compiled unchanged from the reference sources by
 * oracle/Makefile into oracle/_ref/liboracle_ref.so.
 *
 * This file is test infrastructure. Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load the resulting library, as the checker;
 * the product path (amigo_b200) never links or calls it.
 *
 * Private members are opened with `#define private public` so that the
 * symbolic analysis (supernode partition, children, contribution rows,
 * inverse permutation) and the per-node pivot/delay counts can be dumped and
 * compared with the product's own symbolic phase and GPU factorization.
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#define private public
#include "sparse_cholesky.h"
#include "sparse_ldl.h"
#undef private

using amigo::CSRMat;
using amigo::MemoryLocation;
using amigo::OrderingType;
using amigo::SparseLDL;
using amigo::Vector;

namespace {
struct RefHandle {
  int n = 0;
  int nnz = 0;
  std::shared_ptr<CSRMat<double>> mat;
  std::shared_ptr<Vector<double>> diag;
  std::unique_ptr<SparseLDL<double>> ldl;
  std::vector<int> rowp, cols;
};

OrderingType to_order(int order) {
  switch (order) {
    case 0:
      return OrderingType::NESTED_DISSECTION;
    case 1:
      return OrderingType::AMD;
    case 2:
      return OrderingType::MULTI_COLOR;
    default:
      return OrderingType::NATURAL;
  }
}
}  // namespace

extern "C" {

/* order: 0 nested dissection (identity without METIS), 1 AMD, 2 multicolor,
 * 3 natural. solver: 0 LDL, 1 Cholesky. */
void* oref_create(int n, int nnz, const int* rowp, const int* cols, int order,
                  int solver, double ustab, double pivot_tol,
                  double delay_growth) {
  auto* h = new RefHandle;
  h->n = n;
  h->nnz = nnz;
  h->rowp.assign(rowp, rowp + n + 1);
  h->cols.assign(cols, cols + nnz);
  h->mat = CSRMat<double>::create_from_csr_data(
      n, n, nnz, h->rowp.data(), h->cols.data(), MemoryLocation::HOST_ONLY);
  h->diag = std::make_shared<Vector<double>>(n, 0, MemoryLocation::HOST_ONLY);
  auto stype = solver == 1 ? SparseLDL<double>::SolverType::CHOLESKY
                           : SparseLDL<double>::SolverType::LDL;
  h->ldl = std::make_unique<SparseLDL<double>>(
      h->mat, stype, ustab, pivot_tol, delay_growth, to_order(order));
  return h;
}

void oref_destroy(void* p) { delete static_cast<RefHandle*>(p); }

int oref_num_nodes(void* p) {
  return static_cast<RefHandle*>(p)->ldl->num_nodes;
}

int oref_num_contrib(void* p) {
  auto* h = static_cast<RefHandle*>(p);
  return h->ldl->contrib_ptr[h->ldl->num_nodes];
}

/* Any output pointer may be null. invperm is filled with the identity when
 * the ordering is natural (the reference keeps no permutation then). */
void oref_get_symbolic(void* p, int* invperm, int* node_ptr, int* node_to_var,
                       int* children_ptr, int* children, int* contrib_ptr,
                       int* contrib_rows) {
  auto* h = static_cast<RefHandle*>(p);
  auto& s = *h->ldl;
  const int nn = s.num_nodes;
  if (invperm) {
    for (int i = 0; i < h->n; i++) invperm[i] = s.invperm ? s.invperm[i] : i;
  }
  if (node_ptr) std::copy(s.node_ptr, s.node_ptr + nn + 1, node_ptr);
  if (node_to_var) std::copy(s.node_to_var, s.node_to_var + h->n, node_to_var);
  if (children_ptr)
    std::copy(s.node_children_ptr, s.node_children_ptr + nn + 2, children_ptr);
  if (children) std::copy(s.node_children, s.node_children + nn, children);
  if (contrib_ptr) std::copy(s.contrib_ptr, s.contrib_ptr + nn + 1, contrib_ptr);
  if (contrib_rows)
    std::copy(s.contrib_rows, s.contrib_rows + s.contrib_ptr[nn], contrib_rows);
}

/* Elimination tree, its postorder and the column counts, recomputed with the
 * object's own member functions and permutation. */
void oref_etree(void* p, int* parent, int* post, int* colcount) {
  auto* h = static_cast<RefHandle*>(p);
  auto& s = *h->ldl;
  const int n = h->n;
  std::vector<int> perm, iperm, work(4 * n);
  int* pp = nullptr;
  int* ip = nullptr;
  if (s.invperm) {
    iperm.assign(s.invperm, s.invperm + n);
    perm.resize(n);
    for (int i = 0; i < n; i++) perm[iperm[i]] = i;
    pp = perm.data();
    ip = iperm.data();
  }
  std::vector<int> par(n), pst(n), cc(n);
  s.compute_etree(n, h->rowp.data(), h->cols.data(), pp, ip, par.data(),
                  work.data());
  s.post_order_etree(n, par.data(), pst.data(), work.data());
  s.count_column_nonzeros(n, h->rowp.data(), h->cols.data(), pst.data(), pp,
                          ip, par.data(), cc.data(), work.data());
  if (parent) std::copy(par.begin(), par.end(), parent);
  if (post) std::copy(pst.begin(), pst.end(), post);
  if (colcount) std::copy(cc.begin(), cc.end(), colcount);
}

/* The reference AMD permutation alone (copy_for_reorder + reorder). */
void oref_order(int n, const int* rowp, const int* cols, int order, int* perm,
                int* iperm) {
  int *rc = nullptr, *cc = nullptr, *pm = nullptr, *ipm = nullptr;
  amigo::OrderingUtils::copy_for_reorder(to_order(order), n, rowp, cols, &rc,
                                         &cc);
  amigo::OrderingUtils::reorder(to_order(order), n, rc, cc, &pm, &ipm);
  std::copy(pm, pm + n, perm);
  std::copy(ipm, ipm + n, iperm);
  delete[] rc;
  delete[] cc;
  delete[] pm;
  delete[] ipm;
}

int oref_factor(void* p, const double* data, const double* diag) {
  auto* h = static_cast<RefHandle*>(p);
  double* dst = h->mat->get_data_ptr();
  std::copy(data, data + h->nnz, dst);
  if (diag) {
    std::copy(diag, diag + h->n, h->diag->get_array());
    return h->ldl->factor(h->diag);
  }
  return h->ldl->factor(nullptr);
}

void oref_solve(void* p, int nrhs, double* x, int ldx) {
  static_cast<RefHandle*>(p)->ldl->solve(nrhs, x, ldx);
}

void oref_inertia(void* p, int* npos, int* nneg) {
  static_cast<RefHandle*>(p)->ldl->get_inertia(npos, nneg);
}

/* Per-node pivot and delayed-pivot counts of the last factorization. */
void oref_node_pivots(void* p, int* num_pivots, int* num_delayed) {
  auto* h = static_cast<RefHandle*>(p);
  auto& s = *h->ldl;
  for (int ks = 0; ks < s.num_nodes; ks++) {
    int np = 0, nd = 0;
    s.fact.get_factor(ks, &np, nullptr, &nd, nullptr, nullptr);
    if (num_pivots) num_pivots[ks] = np;
    if (num_delayed) num_delayed[ks] = nd;
  }
}

/* The reference's Hessian assembly on one rank: the CSR values zeroed, then
 * for each group, element and column j of the element's Hessian, CSRMat::
 * add_row (include/csr_matrix.h:554-567) of that column into row
 * conn[e][j] at the element's columns, the loop of ComponentGroup::
 * add_hessian_kernel (include/component_group.h:144-162) with the local and
 * global indices equal. blocks: the groups' [nelems][ncomp][ncomp] values,
 * block[e][j][i] = column j, row i. out: nnz values. */
void oref_csr_assemble(int n, int nnz, const int* rowp, const int* cols, int ngroups,
                       const int* nelems, const int* ncomp, const int* conn,
                       const double* blocks, double* out) {
  std::vector<int> rp(rowp, rowp + n + 1), cl(cols, cols + nnz);
  auto mat = CSRMat<double>::create_from_csr_data(n, n, nnz, rp.data(), cl.data(),
                                                  MemoryLocation::HOST_ONLY);
  mat->zero();
  const int* c = conn;
  const double* b = blocks;
  for (int g = 0; g < ngroups; g++) {
    const int m = ncomp[g];
    for (int e = 0; e < nelems[g]; e++, c += m) {
      for (int j = 0; j < m; j++, b += m) mat->add_row(c[j], m, c, b);
    }
  }
  std::copy(mat->get_data_ptr(), mat->get_data_ptr() + nnz, out);
}

/* The reference's SparseCholesky (include/sparse_cholesky.h): the
 * factorization of a symmetric quasi-definite matrix in natural order, the
 * first sqdef_index rows the positive definite block (sqdef_index < 0 or
 * > n: the whole matrix). */
struct RefChol {
  int n = 0;
  int nnz = 0;
  std::vector<int> rowp, cols;
  std::shared_ptr<CSRMat<double>> mat;
  std::unique_ptr<amigo::SparseCholesky<double>> chol;
};

void* oref_chol_create(int n, int nnz, const int* rowp, const int* cols, int sqdef_index) {
  auto* h = new RefChol;
  h->n = n;
  h->nnz = nnz;
  h->rowp.assign(rowp, rowp + n + 1);
  h->cols.assign(cols, cols + nnz);
  h->mat = CSRMat<double>::create_from_csr_data(n, n, nnz, h->rowp.data(), h->cols.data(),
                                                MemoryLocation::HOST_ONLY, nullptr, nullptr,
                                                sqdef_index);
  h->chol = std::make_unique<amigo::SparseCholesky<double>>(h->mat);
  return h;
}

void oref_chol_destroy(void* p) { delete static_cast<RefChol*>(p); }

int oref_chol_factor(void* p, const double* data) {
  auto* h = static_cast<RefChol*>(p);
  std::copy(data, data + h->nnz, h->mat->get_data_ptr());
  return h->chol->factor();
}

/* x (n) is overwritten with K^{-1} x. */
void oref_chol_solve(void* p, double* x) {
  auto* h = static_cast<RefChol*>(p);
  Vector<double> v(h->n, 0, MemoryLocation::HOST_ONLY);
  std::copy(x, x + h->n, v.get_array());
  h->chol->solve(&v);
  std::copy(v.get_array(), v.get_array() + h->n, x);
}

}  // extern "C"
