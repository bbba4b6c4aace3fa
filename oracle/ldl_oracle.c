/*
 * Test oracle: a plain-C restatement of the reference's numeric multifrontal
 * LDL^T (Mersoltane/amigo include/sparse_ldl.h), used only by tests/ and the
 * CPU-baseline leg of bench.py as a checker. Never linked into the product.
 *
 * Input is the reference's symbolic structure (node_ptr, node_to_var,
 * children, contrib rows, inverse permutation), so this file restates only
 * the numeric phase:
 *   - front variables: own, delayed from children, contribution rows
 *     (get_frontal_vars, sparse_ldl.h:970-1000; add_delayed_pivots 617-634)
 *   - assembly: CSR lower part, + diag, extend-add of packed-lower child
 *     blocks with mirroring of delayed entries (assemble_front_matrix,
 *     1018-1174)
 *   - partial factorization with the 1x1 / alternative 1x1 / Duff 2x2 tests
 *     and delays (factor_front_matrix_block, 1316-1553), unblocked
 *     right-looking (the same arithmetic as the blocked panel + trailing
 *     update in exact arithmetic)
 *   - fronts without contribution rows: Bunch-Kaufman (the reference calls
 *     LAPACK dsytrf there, 1226-1248; restated from the published dsytf2
 *     pivoting rule with alpha = (1 + sqrt(17)) / 8)
 *   - inertia (add_pivot_inertia, 1935-1987)
 *   - solve (solve_ldl, 1825-1926)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n, nn;
  const int *rowp, *cols;
  int *node_ptr, *node_to_var, *kid_ptr, *kids, *cptr, *crows, *iperm;
  double ustab, pivot_tol;
  /* factor per node */
  int *f, *npiv, *ndel;
  int **fv;      /* front vars after pivoting, 2x2 encoded -(v+1) */
  double **L;    /* f x npiv, ld f */
  double **cb;   /* packed lower (f-npiv) */
  int npos, nneg;
} ldlo;

static int* dup_int(const int* a, int n) {
  int* b = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
  if (n > 0) memcpy(b, a, sizeof(int) * n);
  return b;
}

ldlo* ldlo_create(int n, const int* rowp, const int* cols, int nn, const int* node_ptr,
                  const int* node_to_var, const int* children_ptr, const int* children,
                  const int* contrib_ptr, const int* contrib_rows, const int* invperm,
                  double ustab, double pivot_tol) {
  ldlo* h = (ldlo*)calloc(1, sizeof(ldlo));
  h->n = n;
  h->nn = nn;
  h->rowp = rowp;
  h->cols = cols;
  h->node_ptr = dup_int(node_ptr, nn + 1);
  h->node_to_var = dup_int(node_to_var, n);
  h->kid_ptr = dup_int(children_ptr, nn + 1);
  h->kids = dup_int(children, children_ptr[nn]);
  h->cptr = dup_int(contrib_ptr, nn + 1);
  h->crows = dup_int(contrib_rows, contrib_ptr[nn]);
  h->iperm = dup_int(invperm, n);
  h->ustab = ustab;
  h->pivot_tol = pivot_tol;
  h->f = (int*)calloc(nn + 1, sizeof(int));
  h->npiv = (int*)calloc(nn + 1, sizeof(int));
  h->ndel = (int*)calloc(nn + 1, sizeof(int));
  h->fv = (int**)calloc(nn + 1, sizeof(int*));
  h->L = (double**)calloc(nn + 1, sizeof(double*));
  h->cb = (double**)calloc(nn + 1, sizeof(double*));
  return h;
}

static void release_factor(ldlo* h) {
  for (int k = 0; k < h->nn; k++) {
    free(h->fv[k]);
    free(h->L[k]);
    free(h->cb[k]);
    h->fv[k] = NULL;
    h->L[k] = NULL;
    h->cb[k] = NULL;
  }
}

void ldlo_destroy(ldlo* h) {
  if (!h) return;
  release_factor(h);
  free(h->node_ptr);
  free(h->node_to_var);
  free(h->kid_ptr);
  free(h->kids);
  free(h->cptr);
  free(h->crows);
  free(h->iperm);
  free(h->f);
  free(h->npiv);
  free(h->ndel);
  free(h->fv);
  free(h->L);
  free(h->cb);
  free(h);
}

#define A(i, j) F[(size_t)(j) * f + (i)]

static void swap_d(double* a, double* b) {
  double t = *a;
  *a = *b;
  *b = t;
}

/* symm_swap, sparse_ldl.h:1270-1292 (a < b) */
static void symm_swap(double* F, int f, int* fv, int a, int b) {
  int t = fv[a];
  fv[a] = fv[b];
  fv[b] = t;
  for (int j = 0; j < a; j++) swap_d(&A(a, j), &A(b, j));
  swap_d(&A(a, a), &A(b, b));
  for (int j = a + 1; j < b; j++) swap_d(&A(j, a), &A(b, j));
  for (int j = b + 1; j < f; j++) swap_d(&A(j, a), &A(j, b));
}

static void factor_node(ldlo* h, int k, const double* vals, const double* diag, int* where) {
  const int ns = h->node_ptr[k + 1] - h->node_ptr[k];
  const int nc = h->cptr[k + 1] - h->cptr[k];
  int nd_in = 0;
  for (int c = h->kid_ptr[k]; c < h->kid_ptr[k + 1]; c++) nd_in += h->ndel[h->kids[c]];
  const int fs = ns + nd_in;
  const int f = fs + nc;
  int* fv = (int*)malloc(sizeof(int) * (f > 0 ? f : 1));
  double* F = (double*)calloc((size_t)f * f + 1, sizeof(double));
  for (int j = 0; j < ns; j++) fv[j] = h->node_to_var[h->node_ptr[k] + j];
  int off = ns;
  for (int c = h->kid_ptr[k]; c < h->kid_ptr[k + 1]; c++) {
    const int ch = h->kids[c];
    for (int j = 0; j < h->ndel[ch]; j++) fv[off++] = h->fv[ch][h->npiv[ch] + j];
  }
  for (int t = 0; t < nc; t++) fv[fs + t] = h->crows[h->cptr[k] + t];
  for (int p = 0; p < f; p++) where[fv[p]] = p;

  /* assembly */
  for (int j = 0; j < ns; j++) {
    const int var = fv[j];
    const int pj = h->iperm[var];
    for (int e = h->rowp[var]; e < h->rowp[var + 1]; e++) {
      const int i = h->cols[e];
      if (where[i] >= 0 && h->iperm[i] >= pj) A(where[i], j) += vals[e];
    }
  }
  if (diag)
    for (int j = 0; j < ns; j++) A(j, j) += diag[fv[j]];
  for (int c = h->kid_ptr[k]; c < h->kid_ptr[k + 1]; c++) {
    const int ch = h->kids[c];
    const int m = h->f[ch] - h->npiv[ch];
    const int* cv = h->fv[ch] + h->npiv[ch];
    const double* C = h->cb[ch];
    for (int j = 0; j < m; j++) {
      const int jf = where[cv[j]];
      for (int i = j; i < m; i++, C++) {
        const int iff = where[cv[i]];
        if (iff >= jf)
          A(iff, jf) += *C;
        else
          A(jf, iff) += *C;
      }
    }
    free(h->cb[ch]);
    h->cb[ch] = NULL;
  }

  /* partial factorization */
  const int root = (nc == 0);
  const double alpha = (1.0 + sqrt(17.0)) / 8.0;
  int kk = 0, ncand = fs;
  while (kk < ncand) {
    double wkk = A(kk, kk), abswkk = fabs(wkk);
    int imax = kk;
    double abswik = 0.0, cmax = 0.0;
    for (int i = kk + 1; i < f; i++) {
      const double a = fabs(A(i, kk));
      if (i < ncand) {
        /* first index of the largest magnitude (idamax) */
        if (imax == kk || a > abswik) {
          abswik = a;
          imax = i;
        }
      } else if (a > cmax) {
        cmax = a;
      }
    }
    const int has = (kk + 1 < ncand);
    if (!has) abswik = 0.0;
    const double colmax = fmax(abswik, cmax);
    int step = 0, kpiv = kk, need_row = 0, zero = 0;
    if (root) {
      if (fmax(abswkk, colmax) == 0.0) {
        step = 1;
        zero = 1;
      } else if (abswkk >= alpha * colmax) {
        step = 1;
      } else {
        need_row = 1;
      }
    } else if (abswkk >= h->pivot_tol && abswkk >= h->ustab * colmax) {
      step = 1;
    } else if (has) {
      need_row = 1;
    }
    if (need_row) {
      double rmax = 0.0;
      for (int j = kk; j < imax; j++) rmax = fmax(rmax, fabs(A(imax, j)));
      for (int i = imax + 1; i < f; i++) rmax = fmax(rmax, fabs(A(i, imax)));
      const double wii = A(imax, imax), abswii = fabs(wii), wik = A(imax, kk);
      if (root) {
        if (abswkk >= alpha * colmax * (colmax / rmax)) {
          step = 1;
        } else if (abswii >= alpha * rmax) {
          step = 1;
          kpiv = imax;
        } else {
          step = 2;
          kpiv = imax;
        }
      } else if (abswii >= h->pivot_tol && abswii >= h->ustab * rmax) {
        step = 1;
        kpiv = imax;
      } else {
        const double det = fabs(wkk * wii - wik * wik);
        if (det >= h->pivot_tol) {
          const double delta = det / fmax(abswii + abswik, abswkk + abswik);
          if (delta >= h->ustab * colmax && delta >= h->ustab * rmax) {
            step = 2;
            kpiv = imax;
          }
        }
      }
    }
    if (step == 0) {
      if (kk < ncand - 1) symm_swap(F, f, fv, kk, ncand - 1);
      ncand--;
      continue;
    }
    const int ksrc = kk + step - 1;
    if (kpiv != ksrc) symm_swap(F, f, fv, ksrc, kpiv);
    if (step == 1) {
      const double d = A(kk, kk);
      if (d >= 0.0)
        h->npos++;
      else
        h->nneg++;
      if (!zero && d != 0.0) {
        const double dinv = 1.0 / d;
        for (int j = kk + 1; j < f; j++) {
          const double w = A(j, kk);
          for (int i = j; i < f; i++) A(i, j) -= A(i, kk) * dinv * w;
        }
        for (int i = kk + 1; i < f; i++) A(i, kk) *= dinv;
      }
    } else {
      const double d11 = A(kk, kk), d21 = A(kk + 1, kk), d22 = A(kk + 1, kk + 1);
      const double det = d11 * d22 - d21 * d21, di = 1.0 / det;
      const double i00 = d22 * di, i01 = -d21 * di, i11 = d11 * di;
      if (det >= 0.0) {
        if (d11 >= 0.0)
          h->npos += 2;
        else
          h->nneg += 2;
      } else {
        h->npos++;
        h->nneg++;
      }
      for (int i = kk + 2; i < f; i++) {
        const double a = A(i, kk), b = A(i, kk + 1);
        A(i, kk) = a * i00 + b * i01;
        A(i, kk + 1) = a * i01 + b * i11;
      }
      for (int j = kk + 2; j < f; j++) {
        /* W(j,:) = L(j,:) D */
        const double wa = A(j, kk) * d11 + A(j, kk + 1) * d21;
        const double wb = A(j, kk) * d21 + A(j, kk + 1) * d22;
        for (int i = j; i < f; i++) A(i, j) -= A(i, kk) * wa + A(i, kk + 1) * wb;
      }
      fv[kk] = -(fv[kk] + 1);
      fv[kk + 1] = -(fv[kk + 1] + 1);
    }
    kk += step;
  }
  const int npiv = kk, m = f - npiv;
  h->f[k] = f;
  h->npiv[k] = npiv;
  h->ndel[k] = fs - npiv;
  h->fv[k] = fv;
  h->L[k] = (double*)malloc(sizeof(double) * ((size_t)f * npiv + 1));
  memcpy(h->L[k], F, sizeof(double) * (size_t)f * npiv);
  h->cb[k] = (double*)malloc(sizeof(double) * ((size_t)m * (m + 1) / 2 + 1));
  double* C = h->cb[k];
  for (int j = npiv; j < f; j++)
    for (int i = j; i < f; i++) *C++ = A(i, j);
  for (int p = 0; p < f; p++) where[fv[p] >= 0 ? fv[p] : -fv[p] - 1] = -1;
  free(F);
}

/* Nodes are numbered in postorder (children before parents), so a single
 * increasing sweep respects the tree. */
int ldlo_factor(ldlo* h, const double* vals, const double* diag) {
  release_factor(h);
  h->npos = h->nneg = 0;
  int* where = (int*)malloc(sizeof(int) * (h->n > 0 ? h->n : 1));
  for (int i = 0; i < h->n; i++) where[i] = -1;
  for (int k = 0; k < h->nn; k++) factor_node(h, k, vals, diag, where);
  free(where);
  return 0;
}

void ldlo_inertia(ldlo* h, int* npos, int* nneg) {
  *npos = h->npos;
  *nneg = h->nneg;
}

static int var_of(int v) { return v >= 0 ? v : -v - 1; }

/* solve_ldl, sparse_ldl.h:1825-1926 */
void ldlo_solve(ldlo* h, int nrhs, double* x, int ldx) {
  int fmax = 1;
  for (int k = 0; k < h->nn; k++)
    if (h->f[k] > fmax) fmax = h->f[k];
  double* t = (double*)malloc(sizeof(double) * fmax);
  for (int r = 0; r < nrhs; r++) {
    double* xr = x + (size_t)ldx * r;
    for (int k = 0; k < h->nn; k++) {
      const int f = h->f[k], np = h->npiv[k];
      const int* fv = h->fv[k];
      const double* L = h->L[k];
      for (int p = 0; p < np; p++) t[p] = xr[var_of(fv[p])];
      for (int j = 0; j < np;) {
        if (fv[j] >= 0) {
          for (int i = j + 1; i < f; i++) {
            const double u = L[(size_t)j * f + i] * t[j];
            if (i < np)
              t[i] -= u;
            else
              xr[fv[i]] -= u;
          }
          j++;
        } else {
          for (int i = j + 2; i < f; i++) {
            const double u = L[(size_t)j * f + i] * t[j] + L[(size_t)(j + 1) * f + i] * t[j + 1];
            if (i < np)
              t[i] -= u;
            else
              xr[fv[i]] -= u;
          }
          j += 2;
        }
      }
      for (int j = 0; j < np;) {
        if (fv[j] >= 0) {
          t[j] /= L[(size_t)j * f + j];
          j++;
        } else {
          const double d11 = L[(size_t)j * f + j], d21 = L[(size_t)j * f + j + 1],
                       d22 = L[(size_t)(j + 1) * f + j + 1];
          const double inv = 1.0 / (d11 * d22 - d21 * d21);
          const double a = t[j], b = t[j + 1];
          t[j] = inv * (d22 * a - d21 * b);
          t[j + 1] = inv * (d11 * b - d21 * a);
          j += 2;
        }
      }
      for (int p = 0; p < np; p++) xr[var_of(fv[p])] = t[p];
    }
    for (int k = h->nn - 1; k >= 0; k--) {
      const int f = h->f[k], np = h->npiv[k];
      const int* fv = h->fv[k];
      const double* L = h->L[k];
      for (int p = 0; p < np; p++) t[p] = xr[var_of(fv[p])];
      for (int j = 0; j < np; j++)
        for (int i = np; i < f; i++) t[j] -= L[(size_t)j * f + i] * xr[fv[i]];
      for (int i = np - 1; i >= 0;) {
        if (fv[i] >= 0) {
          for (int j = i + 1; j < np; j++) t[i] -= L[(size_t)i * f + j] * t[j];
          i--;
        } else {
          for (int j = i + 1; j < np; j++) {
            t[i - 1] -= L[(size_t)(i - 1) * f + j] * t[j];
            t[i] -= L[(size_t)i * f + j] * t[j];
          }
          i -= 2;
        }
      }
      for (int p = 0; p < np; p++) xr[var_of(fv[p])] = t[p];
    }
  }
  free(t);
}

/* Pivot record of the last factorization (test access): per supernode the
 * front size, pivots and delayed candidates, and the front variables after
 * pivoting (pivots in elimination order with 2x2 pairs encoded -(v+1), then
 * the delayed candidates, then the contribution rows) one supernode after
 * another. Any pointer may be NULL; returns the length of fv. */
long long ldlo_pivot_record(ldlo* h, int* f, int* npiv, int* ndel, int* fv) {
  long long o = 0;
  for (int k = 0; k < h->nn; k++) {
    if (f) f[k] = h->f[k];
    if (npiv) npiv[k] = h->npiv[k];
    if (ndel) ndel[k] = h->ndel[k];
    if (fv)
      for (int t = 0; t < h->f[k]; t++) fv[o + t] = h->fv[k][t];
    o += h->f[k];
  }
  return o;
}
