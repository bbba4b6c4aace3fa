// Numeric multifrontal LDL^T on sm_100a: one CTA per supernode of an
// elimination-tree level. The CTA assembles its front (CSR entries of its
// pivot columns, the diagonal vector, the children's contribution blocks),
// factors the fully summed part with threshold 1x1/2x2 pivoting (delaying
// candidates that fail, as the reference does in
// SparseLDL::factor_front_matrix_block, include/sparse_ldl.h:1316-1553) or
// with Bunch-Kaufman when the front has no contribution rows (the reference
// calls LAPACK dsytrf there, include/sparse_ldl.h:1226-1248), and writes the
// factor columns, its final front-variable order and its contribution block.
//
// Fronts up to kSmemFrontMax live in shared memory; larger ones are factored
// in place in the device pool and their factor/contribution are views into
// that storage.
#include <cfloat>
#include <climits>

#include "ldl_internal.h"

namespace b200ldl {

namespace {

constexpr int kWarps = kFactorThreads / 32;

__device__ __forceinline__ void keep_larger(double& bv, int& bi, double v, int i) {
  // larger magnitude wins; ties go to the lower index (idamax semantics)
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

// Warp-wide (argmax, max) with the result in every lane.
__device__ __forceinline__ void warp_argmax(double& bv, int& bi, double& cm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    const double om = __shfl_xor_sync(0xffffffffu, cm, o);
    keep_larger(bv, bi, ov, oi);
    cm = fmax(cm, om);
  }
}

struct Reduce {
  double v[kWarps];
  int i[kWarps];
  double m[kWarps];
};

// Block-wide (argmax, max) reduction. Result valid for all threads after the
// trailing barrier.
__device__ __forceinline__ void block_argmax(Reduce& r, double& bv, int& bi, double& cm) {
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, bv, o);
    const int oi = __shfl_down_sync(0xffffffffu, bi, o);
    const double om = __shfl_down_sync(0xffffffffu, cm, o);
    keep_larger(bv, bi, ov, oi);
    cm = fmax(cm, om);
  }
  if (lane == 0) {
    r.v[w] = bv;
    r.i[w] = bi;
    r.m[w] = cm;
  }
  __syncthreads();
  bv = r.v[0];
  bi = r.i[0];
  cm = r.m[0];
#pragma unroll
  for (int q = 1; q < kWarps; q++) {
    keep_larger(bv, bi, r.v[q], r.i[q]);
    cm = fmax(cm, r.m[q]);
  }
  __syncthreads();
}

// Symmetric interchange of rows/columns a < b of the lower-stored front,
// including the already factored columns left of a (sparse_ldl.h:1270-1292).
__device__ void symm_swap(double* F, int ld, int f, int a, int b, int* fv, int* orig) {
  const int n1 = a;              // F(a, 0:a) <-> F(b, 0:a)
  const int n2 = b - a - 1;      // F(j, a) <-> F(b, j), a < j < b
  const int n3 = f - b - 1;      // F(j, a) <-> F(j, b), j > b
  const int total = n1 + 1 + n2 + n3;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    double *p, *q;
    if (t < n1) {
      p = &F[a + (size_t)ld * t];
      q = &F[b + (size_t)ld * t];
    } else if (t == n1) {
      p = &F[a + (size_t)ld * a];
      q = &F[b + (size_t)ld * b];
    } else if (t < n1 + 1 + n2) {
      const int j = a + 1 + (t - n1 - 1);
      p = &F[j + (size_t)ld * a];
      q = &F[b + (size_t)ld * j];
    } else {
      const int j = b + 1 + (t - n1 - 1 - n2);
      p = &F[j + (size_t)ld * a];
      q = &F[j + (size_t)ld * b];
    }
    const double tmp = *p;
    *p = *q;
    *q = tmp;
  }
  if (threadIdx.x == 0) {
    int t = fv[a];
    fv[a] = fv[b];
    fv[b] = t;
    t = orig[a];
    orig[a] = orig[b];
    orig[b] = t;
  }
}

enum : int { kDelay = 0, kOne = 1, kTwo = 2, kNeedRow = 3, kZero = 4 };

__global__ void __launch_bounds__(kFactorThreads)
    factor_level_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                        const double* __restrict__ vals, const double* __restrict__ diag,
                        FactorParams prm, int fcap, int allow_big) {
  extern __shared__ __align__(16) double smem[];
  __shared__ Reduce red;
  __shared__ int sh_fail;
  __shared__ long long sh_ioff, sh_doff;

  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

  if (tid == 0) sh_fail = *((volatile int*)s.err);
  __syncthreads();
  if (sh_fail) return;

  const int ns = p.ns[node];
  const int nc = p.nc[node];
  const int kb = p.kid_ptr[node];
  const int ke = p.kid_ptr[node + 1];
  int nd_in = 0;
  for (int c = kb; c < ke; c++) nd_in += s.ndel[p.kids[c]];
  const int fs = ns + nd_in;
  const int f = fs + nc;
  const bool big = f > kSmemFrontMax;

  if (tid == 0) {
    // the launch's shared memory holds fronts up to fcap: a larger one stops
    // the factorization, which the host repeats with room for every front
    if (!big && f > fcap) {
      atomicOr(s.err, 2);
      atomicCAS(s.err + 1, -1, node);
      sh_fail = 1;
    }
    // a big front in a level the host does not prepare big fronts for stops
    // the factorization too; the host repeats it with every level prepared
    if (big && !allow_big) {
      atomicOr(s.err, 4);
      atomicCAS(s.err + 1, -1, node);
      sh_fail = 1;
    }
  }
  __syncthreads();
  if (sh_fail) return;
  if (tid == 0) {
    int fail = 0;
    const unsigned long long io = atomicAdd(s.used, 2ull * (unsigned long long)f);
    if (io + 2ull * f > s.icap) fail = 1;
    sh_ioff = (long long)io;
    if (big) {
      // the front itself plus the panel's W columns; fronts above the
      // on-chip limit also get the chained panel's W by physical row and its
      // permutation scratch
      unsigned long long need = (unsigned long long)f * f + (unsigned long long)kBigPanelMax * f;
      const unsigned long long chain =
          (unsigned long long)kBigPanelMax * f + (unsigned long long)(fs + 1) * f;
      if (prm.app && f >= prm.app_min_f) {
        // a root may finish with the chained panels: their scratch too
        need += (unsigned long long)kAppScratch + (nc == 0 ? chain : 0ull);
      } else if (f > s.cf_limit[4]) {
        need += chain;
      }
      const unsigned long long dofs = atomicAdd(s.used + 1, need);
      if (dofs + need > s.dcap) fail = 1;
      sh_doff = (long long)dofs;
    }
    if (fail) {
      atomicOr(s.err, 1);  // a pool ran out
      atomicCAS(s.err + 1, -1, node);
    }
    sh_fail = fail;
  }
  __syncthreads();
  if (sh_fail) return;

  int* fv = s.ivars + sh_ioff;
  int* orig = fv + f;
  if (big) {
    // front variables now; assembly and factorization by the big-front kernels
    const int v0b = p.var_ptr[node];
    for (int t = tid; t < ns; t += blockDim.x) fv[t] = p.node_to_var[v0b + t];
    int offb = ns;
    for (int c = kb; c < ke; c++) {
      const int ch = p.kids[c];
      const int nd = s.ndel[ch];
      const int* cfv = s.ivars + s.fv_off[ch] + s.npiv[ch];
      for (int t = tid; t < nd; t += blockDim.x) fv[offb + t] = cfv[t];
      offb += nd;
    }
    const int cb0 = p.cptr[node];
    for (int t = tid; t < nc; t += blockDim.x) fv[fs + t] = p.contrib_rows[cb0 + t];
    for (int t = tid; t < f; t += blockDim.x) orig[t] = t;
    if (tid == 0) {
      const int slot = atomicAdd(s.big_meta, 1);
      atomicMax(s.big_meta + 1, f);
      atomicMax(s.big_meta + 2, fs);
      const bool app = prm.app && f >= prm.app_min_f;
      int cls = 5;
      if (app) {
        cls = 6;
      } else {
        for (int c = 4; c >= 0; c--)
          if (f <= s.cf_limit[c]) cls = c;
      }
      if (cls == 6) {
        const int q = atomicAdd(s.big_meta + 16, 1);
        atomicMax(s.big_meta + 17, f);
        atomicMax(s.big_meta + 18, fs);
        s.class_list[(size_t)6 * p.num_nodes + q] = slot;
      } else if (cls == 5) {
        const int q = atomicAdd(s.big_meta + 3, 1);
        atomicMax(s.big_meta + 4, fs);
        atomicMax(s.big_meta + 15, f);
        s.class_list[(size_t)5 * p.num_nodes + q] = slot;
      } else {
        const int q = atomicAdd(s.big_meta + 5 + cls, 1);
        atomicMax(s.big_meta + 10 + cls, f);
        s.class_list[(size_t)cls * p.num_nodes + q] = slot;
      }
      BigFront b;
      b.node = node;
      b.f = f;
      b.fs = fs;
      b.ns = ns;
      b.nd_in = nd_in;
      b.nc = nc;
      b.k = 0;
      b.ncand = fs;
      b.kstart = 0;
      b.kw = 0;
      b.state = 0;
      b.npos = 0;
      b.nneg = 0;
      b.pad = 0;
      b.app = app ? 1 : 0;
      b.pending = -1;
      b.ioff = sh_ioff;
      b.doff = sh_doff;
      b.woff = sh_doff + (long long)f * f;
      // a-posteriori scratch after the panel's W (and, for a root, after the
      // chained panels' scratch)
      b.xoff = b.woff + (long long)kBigPanelMax * f +
               ((app && nc == 0) ? (long long)kBigPanelMax * f + (long long)(fs + 1) * f : 0ll);
      b.flops = 0.0;
      s.big[slot] = b;
    }
    return;
  }
  double* F;
  int ld;
  if (big) {
    F = s.dpool + sh_doff;
    ld = f;
  } else {
    F = smem;
    ld = f | 1;
  }

  // front variables: own, delayed from children (child order), contribution
  const int v0 = p.var_ptr[node];
  for (int t = tid; t < ns; t += blockDim.x) fv[t] = p.node_to_var[v0 + t];
  {
    int off = ns;
    for (int c = kb; c < ke; c++) {
      const int ch = p.kids[c];
      const int nd = s.ndel[ch];
      const int* cfv = s.ivars + s.fv_off[ch] + s.npiv[ch];
      for (int t = tid; t < nd; t += blockDim.x) fv[off + t] = cfv[t];
      off += nd;
    }
  }
  const int c0 = p.cptr[node];
  for (int t = tid; t < nc; t += blockDim.x) fv[fs + t] = p.contrib_rows[c0 + t];
  for (int t = tid; t < f; t += blockDim.x) orig[t] = t;

  // zero the lower triangle (whole columns, simplest coalesced pattern)
  for (int j = warp; j < f; j += kWarps) {
    double* col = F + (size_t)ld * j;
    for (int i = j + lane; i < f; i += 32) col[i] = 0.0;
  }
  __syncthreads();

  // original entries of the pivot columns
  {
    const int64_t e0 = p.scat_ptr[node];
    const int64_t e1 = p.scat_ptr[node + 1];
    for (int64_t e = e0 + tid; e < e1; e += blockDim.x) {
      int r = p.scat_row[e];
      if (r >= ns) r += nd_in;
      F[r + (size_t)ld * p.scat_col[e]] += csr_value(s, vals, p.scat_csr[e]);
    }
  }
  __syncthreads();
  if (diag) {
    for (int j = tid; j < ns; j += blockDim.x) F[j + (size_t)ld * j] += diag[fv[j]];
  }
  __syncthreads();

  // extend-add the children's contribution blocks, one child at a time
  {
    int off = ns;
    for (int c = kb; c < ke; c++) {
      const int ch = p.kids[c];
      const int nd = s.ndel[ch];
      const int m = s.f[ch] - s.npiv[ch];
      const double* cb = s.dpool + s.cb_off[ch];
      const int cld = s.cb_ld[ch];
      const int* cm = p.cmap + p.cptr[ch];
      for (int r2 = warp; r2 < m; r2 += kWarps) {
        int p2;
        if (r2 < nd) {
          p2 = off + r2;
        } else {
          p2 = cm[r2 - nd];
          if (p2 >= ns) p2 += nd_in;
        }
        const double* col = cb + (size_t)cld * r2;
        for (int r1 = r2 + lane; r1 < m; r1 += 32) {
          int p1;
          if (r1 < nd) {
            p1 = off + r1;
          } else {
            p1 = cm[r1 - nd];
            if (p1 >= ns) p1 += nd_in;
          }
          const double v = col[r1];
          if (p1 >= p2)
            F[p1 + (size_t)ld * p2] += v;
          else
            F[p2 + (size_t)ld * p1] += v;
        }
      }
      __syncthreads();
      off += nd;
    }
  }

  // partial factorization of the fully summed candidates [0, ncand).
  // Right-looking, one barrier per accepted 1x1 pivot: the warp that updates
  // the next column also produces its pivot statistics, and the scaling of
  // a pivot column into L is deferred to the next update pass (it is a
  // per-row operation, so it commutes with the row interchanges in between).
  const bool root = (nc == 0);
  const double alpha_bk = (1.0 + 4.1231056256176605) / 8.0;  // (1 + sqrt(17)) / 8
  __shared__ double st_v, st_m;
  __shared__ int st_i;
  int k = 0;
  int ncand = fs;
  int npos = 0, nneg = 0;
  double flops = 0.0;
  int pend = 0, pc = 0;
  double pd0 = 0.0, pd1 = 0.0, pd2 = 0.0;
  bool need_stats = true;

  while (k < ncand) {
    if (!prm.cholesky && need_stats) {
      if (warp == 0) {
        double bv = -1.0, cm = 0.0;
        int bi = INT_MAX;
        const double* colk = F + (size_t)ld * k;
        for (int i = k + 1 + lane; i < f; i += 32) {
          const double a = fabs(colk[i]);
          if (i < ncand)
            keep_larger(bv, bi, a, i);
          else
            cm = fmax(cm, a);
        }
        warp_argmax(bv, bi, cm);
        if (lane == 0) {
          st_v = bv;
          st_i = bi;
          st_m = cm;
        }
      }
      __syncthreads();
    }
    int step;
    int kpiv = k;
    if (prm.cholesky) {
      step = kOne;
    } else {
      const double wkk = F[k + (size_t)ld * k];
      const double abswkk = fabs(wkk);
      const bool has_cand = (k + 1 < ncand);
      const double abswik = has_cand ? st_v : 0.0;
      // st_i stays INT_MAX only if every candidate entry is NaN; keep imax a
      // valid candidate index so the rest of the step stays in bounds
      const int imax = has_cand ? (st_i < ncand ? st_i : k + 1) : k;
      const double colmax = fmax(abswik, st_m);
      if (root) {
        if (fmax(abswkk, colmax) == 0.0)
          step = kZero;
        else if (abswkk >= alpha_bk * colmax)
          step = kOne;
        else
          step = kNeedRow;
      } else if (abswkk >= prm.pivot_tol && abswkk >= prm.ustab * colmax) {
        step = kOne;
      } else {
        step = has_cand ? kNeedRow : kDelay;
      }
      if (step == kNeedRow) {
        // row/column imax off the diagonal: F(imax, k:imax), F(imax+1:, imax)
        double rv = -1.0, rmax = 0.0;
        int ri = INT_MAX;
        const int n1 = imax - k;
        const int n2 = f - imax - 1;
        for (int t = tid; t < n1 + n2; t += blockDim.x) {
          const double a = (t < n1) ? fabs(F[imax + (size_t)ld * (k + t)])
                                    : fabs(F[(imax + 1 + (t - n1)) + (size_t)ld * imax]);
          rmax = fmax(rmax, a);
        }
        block_argmax(red, rv, ri, rmax);
        const double wii = F[imax + (size_t)ld * imax];
        const double abswii = fabs(wii);
        const double wik = F[imax + (size_t)ld * k];
        if (root) {
          // Bunch-Kaufman partial pivoting (dsytf2, lower)
          if (abswkk >= alpha_bk * colmax * (colmax / rmax)) {
            step = kOne;
          } else if (abswii >= alpha_bk * rmax) {
            step = kOne;
            kpiv = imax;
          } else {
            step = kTwo;
            kpiv = imax;
          }
        } else if (abswii >= prm.pivot_tol && abswii >= prm.ustab * rmax) {
          step = kOne;
          kpiv = imax;
        } else {
          const double det = fabs(wkk * wii - wik * wik);
          step = kDelay;
          if (det >= prm.pivot_tol) {
            const double delta = det / fmax(abswii + abswik, abswkk + abswik);
            if (delta >= prm.ustab * colmax && delta >= prm.ustab * rmax) {
              step = kTwo;
              kpiv = imax;
            }
          }
        }
      }
    }

    if (step == kDelay) {
      if (k < ncand - 1) symm_swap(F, ld, f, k, ncand - 1, fv, orig);
      __syncthreads();
      ncand -= 1;
      need_stats = true;
      continue;
    }
    const int nstep = (step == kTwo) ? 2 : 1;
    const int ksrc = k + nstep - 1;
    if (kpiv != ksrc) {
      symm_swap(F, ld, f, ksrc, kpiv, fv, orig);
      __syncthreads();
    }

    // deferred scaling of the previous pivot column(s)
    if (pend == 1) {
      double* c0 = F + (size_t)ld * pc;
      for (int i = pc + 1 + tid; i < f; i += blockDim.x) c0[i] *= pd0;
    } else if (pend == 2) {
      double* c0 = F + (size_t)ld * pc;
      double* c1 = c0 + ld;
      for (int i = pc + 2 + tid; i < f; i += blockDim.x) {
        const double a = c0[i];
        const double b = c1[i];
        c0[i] = a * pd0 + b * pd1;
        c1[i] = a * pd1 + b * pd2;
      }
    }

    const double* colk = F + (size_t)ld * k;
    const int nxt = k + nstep;  // the next candidate column
    const bool want_stats = !prm.cholesky && nxt < ncand;
    if (nstep == 1) {
      const double d = colk[k];
      const double dinv = (step == kZero || (root && d == 0.0)) ? 0.0 : 1.0 / d;
      for (int j = k + 1 + warp; j < f; j += kWarps) {
        const double lj = colk[j] * dinv;
        double* colj = F + (size_t)ld * j;
        if (j == nxt && want_stats) {
          double bv = -1.0, cm = 0.0;
          int bi = INT_MAX;
          for (int i = j + lane; i < f; i += 32) {
            const double v = colj[i] - colk[i] * lj;
            colj[i] = v;
            if (i > j) {
              const double a = fabs(v);
              if (i < ncand)
                keep_larger(bv, bi, a, i);
              else
                cm = fmax(cm, a);
            }
          }
          warp_argmax(bv, bi, cm);
          if (lane == 0) {
            st_v = bv;
            st_i = bi;
            st_m = cm;
          }
        } else {
          for (int i = j + lane; i < f; i += 32) colj[i] -= colk[i] * lj;
        }
      }
      if (tid == 0) {
        if (d >= 0.0)
          npos++;
        else
          nneg++;
        const double r = (double)(f - k - 1);
        flops += r * (r + 1.0) + r;
      }
      pend = 1;
      pc = k;
      pd0 = dinv;
    } else {
      const double* colk1 = colk + ld;
      const double d11 = colk[k];
      const double d21 = colk[k + 1];
      const double d22 = colk1[k + 1];
      const double det = d11 * d22 - d21 * d21;
      const double detinv = 1.0 / det;
      const double i00 = d22 * detinv, i01 = -d21 * detinv, i11 = d11 * detinv;
      for (int j = k + 2 + warp; j < f; j += kWarps) {
        const double a = colk[j];
        const double b = colk1[j];
        const double l0 = a * i00 + b * i01;
        const double l1 = a * i01 + b * i11;
        double* colj = F + (size_t)ld * j;
        if (j == nxt && want_stats) {
          double bv = -1.0, cm = 0.0;
          int bi = INT_MAX;
          for (int i = j + lane; i < f; i += 32) {
            const double v = colj[i] - (colk[i] * l0 + colk1[i] * l1);
            colj[i] = v;
            if (i > j) {
              const double aa = fabs(v);
              if (i < ncand)
                keep_larger(bv, bi, aa, i);
              else
                cm = fmax(cm, aa);
            }
          }
          warp_argmax(bv, bi, cm);
          if (lane == 0) {
            st_v = bv;
            st_i = bi;
            st_m = cm;
          }
        } else {
          for (int i = j + lane; i < f; i += 32) colj[i] -= colk[i] * l0 + colk1[i] * l1;
        }
      }
      if (tid == 0) {
        fv[k] = -(fv[k] + 1);
        fv[k + 1] = -(fv[k + 1] + 1);
        if (det >= 0.0) {
          if (d11 >= 0.0)
            npos += 2;
          else
            nneg += 2;
        } else {
          npos++;
          nneg++;
        }
        const double r = (double)(f - k - 2);
        flops += 2.0 * r * (r + 1.0) + 6.0 * r;
      }
      pend = 2;
      pc = k;
      pd0 = i00;
      pd1 = i01;
      pd2 = i11;
    }
    __syncthreads();
    // the warp owning column nxt covered every row below it only if nxt < f
    need_stats = !(want_stats);
    k += nstep;
  }
  // last deferred scaling
  if (pend == 1) {
    double* c0 = F + (size_t)ld * pc;
    for (int i = pc + 1 + tid; i < f; i += blockDim.x) c0[i] *= pd0;
  } else if (pend == 2) {
    double* c0 = F + (size_t)ld * pc;
    double* c1 = c0 + ld;
    for (int i = pc + 2 + tid; i < f; i += blockDim.x) {
      const double a = c0[i];
      const double b = c1[i];
      c0[i] = a * pd0 + b * pd1;
      c1[i] = a * pd1 + b * pd2;
    }
  }
  __syncthreads();

  const int npiv = k;
  const int m = f - npiv;
  if (tid == 0) {
    int fail = 0;
    if (!big) {
      const unsigned long long need =
          (unsigned long long)f * npiv + (unsigned long long)m * m;
      const unsigned long long dofs = atomicAdd(s.used + 1, need);
      if (dofs + need > s.dcap) fail = 1;
      sh_doff = (long long)dofs;
    }
    if (fail) {
      atomicOr(s.err, 1);  // a pool ran out
      atomicCAS(s.err + 1, -1, node);
    }
    sh_fail = fail;
  }
  __syncthreads();
  if (sh_fail) return;

  if (!big) {
    double* L = s.dpool + sh_doff;
    double* C = L + (size_t)f * npiv;
    for (int j = warp; j < npiv; j += kWarps)
      for (int i = lane; i < f; i += 32) L[i + (size_t)f * j] = F[i + (size_t)ld * j];
    for (int j = warp; j < m; j += kWarps)
      for (int i = j + lane; i < m; i += 32)
        C[i + (size_t)m * j] = F[(npiv + i) + (size_t)ld * (npiv + j)];
  }
  if (tid == 0) {
    s.f[node] = f;
    s.fs[node] = fs;
    s.npiv[node] = npiv;
    s.ndel[node] = fs - npiv;
    s.fv_off[node] = sh_ioff;
    s.u_off[node] = (long long)atomicAdd(s.used + 2, (unsigned long long)m);
    if (big) {
      s.L_off[node] = sh_doff;
      s.L_ld[node] = f;
      s.cb_off[node] = sh_doff + (long long)npiv * (f + 1);
      s.cb_ld[node] = f;
    } else {
      s.L_off[node] = sh_doff;
      s.L_ld[node] = f;
      s.cb_off[node] = sh_doff + (long long)f * npiv;
      s.cb_ld[node] = m > 0 ? m : 1;
    }
    if (!prm.cholesky) {
      atomicAdd(s.inertia, npos);
      atomicAdd(s.inertia + 1, nneg);
    }
    atomicAdd(s.flops, flops);
  }
}

}  // namespace

size_t factor_smem_bytes(int f) {
  // the front (ld = f|1) and two columns of slack
  return ((size_t)(f | 1) * f + 2 * (size_t)f) * sizeof(double);
}

void launch_factor_level(const DevPlan& p, const DevState& s, const int* level_nodes,
                         int count, int fmax, int allow_big, const FactorParams& prm,
                         cudaStream_t stream, const double* vals, const double* diag) {
  if (count <= 0) return;
  factor_level_kernel<<<count, kFactorThreads, factor_smem_bytes(fmax), stream>>>(
      p, s, level_nodes, vals, diag, prm, fmax, allow_big);
}

cudaError_t configure_factor_kernels() {
  return cudaFuncSetAttribute(factor_level_kernel,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)factor_smem_bytes(kSmemFrontMax));
}

}  // namespace b200ldl
