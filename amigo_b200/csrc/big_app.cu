// Fronts above the shared-memory limit, factored in blocked panels with
// a-posteriori threshold tests.
//
// The reference tests one candidate at a time (SparseLDL::
// factor_front_matrix_block, include/sparse_ldl.h:1316-1553): it forms the
// candidate's column, compares the pivot with the largest entry of the
// column over every remaining row of the front, and accepts a 1x1 pivot, the
// alternative 1x1 at imax or a Duff 2x2, or delays the candidate to the
// parent. Once the candidates are arranged so that nearly every one passes
// where it stands (pivot-order reuse), that sequence of column-wide tests is
// what costs time, not arithmetic. Here a panel of up to 32 candidates is
// decided in three data-parallel passes instead:
//
//   1. app_diag_kernel (one CTA per front): the 32 x 32 diagonal block is
//      factored in shared memory with the reference's tests (one warp decides,
//      one lane per row; the CTA updates the block). A test's column maximum
//      joins the block's rows with, for the panel's first pivot, the
//      column's maximum below the block that the previous panel's trailing
//      update left behind; a candidate that fails is rotated behind the
//      block's candidates and delayed. It records, per accepted pivot, the
//      block part of the column maximum.
//   2. app_rows_kernel (many CTAs per front): every row below the block forms
//      its entries of the pivot columns, W = F21 L11^-T (the values the
//      reference's test sees), stores them for the trailing update, and the
//      column maxima over all rows below are reduced.
//   3. app_accept_kernel: the reference's tests are evaluated exactly, with
//      the column maxima over the whole front; the pivots before the first
//      failure are accepted and written as L (D on the diagonal, 2x2 blocks
//      with d21 below it, as the reference stores them). The first failing
//      pivot, and the candidates that failed in the block before it, are
//      delayed: after the trailing update
//      (big_update_kernel) app_delay_kernel moves them behind the remaining
//      candidates with the reference's symmetric interchange (symm_swap,
//      sparse_ldl.h:1270-1292), as the reference's delay does.
//
// Every accepted pivot therefore satisfies the reference's threshold test
// against its whole column, so the factorization has the reference's
// stability bound (|L| <= 1/ustab for 1x1 pivots) and, by Sylvester's law,
// its inertia; only the order in which candidates are tried differs (a
// candidate's 2x2 partner is searched within its panel's block).
//
// The front stays in HBM in logical order between passes (column-major,
// lower triangle, the layout big_chain.cu and big_update_kernel use). The
// panel's state lives in a per-front scratch area (xoff): the block's L,
// D, tests and permutation. Each pass checks that the scratch belongs to the
// current step (the step number the diagonal pass stamped), so fronts that
// finished earlier do nothing and no pass reads the front's descriptor while
// another pass of the same launch writes it.
#include <algorithm>
#include <climits>

#include "ldl_internal.h"

namespace b200ldl {

namespace {

constexpr int kBlk = 32;  // candidates per panel
constexpr int kLd = kBlk + 1;
constexpr int kRowThreads = 256;

// per-front scratch (doubles at xoff)
constexpr int kXNext = kAppNextColmax;      // [32] next panel's column maxima below (bits)
constexpr int kXL = kXNext + kBlk;          // Lb[32][33]: block rows' L entries
constexpr int kXD = kXL + kBlk * kLd;       // dd[32][3]: d | d11, d21, d22 per pivot
constexpr int kXCin = kXD + 3 * kBlk;       // block part of the column maximum
constexpr int kXRin = kXCin + kBlk;         // block part of a 2x2 partner's column maximum
constexpr int kXBelow = kXRin + kBlk;       // column maxima over the rows below (bits)
constexpr int kXInt = kXBelow + kBlk;       // ints from here
// int offsets (from kXInt as int*)
constexpr int kIPerm = 0;    // [32] block position -> block position before the panel
constexpr int kIKind = 32;   // [32] 1: 1x1, 2: first of a 2x2, 3: second of a 2x2
constexpr int kIDlt = 64;    // [32] candidates delayed in the block: pivots accepted before
constexpr int kIAcc = 96;    // pivots accepted inside the block
constexpr int kINbk = 97;    // candidates in the block
constexpr int kIK = 98;      // first position of the panel
constexpr int kIStep = 99;   // step number of the panel
constexpr int kINcand = 100;
constexpr int kIMoved = 101;  // 1 if the block permutation is not the identity
constexpr int kIDcnt = 102;   // candidates to delay after the update
constexpr int kIDpos = 103;   // [32] their positions, decreasing
constexpr int kINint = kIDpos + kBlk;
static_assert(kXInt + (kINint + 1) / 2 <= kAppScratch, "a-posteriori scratch size");

__device__ __forceinline__ double fsym(const double* F, int f, int a, int b) {
  return (a >= b) ? F[a + (size_t)f * b] : F[b + (size_t)f * a];
}

__device__ __forceinline__ int* xint(double* X) { return reinterpret_cast<int*>(X + kXInt); }
__device__ __forceinline__ const int* xint(const double* X) {
  return reinterpret_cast<const int*>(X + kXInt);
}

// largest value, lowest index on ties (idamax)
__device__ __forceinline__ void warp_argmax(double& v, int& i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (ov > v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// The reference's tests for the accepted pivots of a panel, with the column
// maxima over the whole front: number of leading pivots that pass.
__device__ int passing_prefix(const double* X, double ustab, double tol) {
  const int* xi = xint(X);
  const int acc = xi[kIAcc];
  const unsigned long long* below = reinterpret_cast<const unsigned long long*>(X + kXBelow);
  int p = 0;
  while (p < acc) {
    const int kind = xi[kIKind + p];
    const double cb = __longlong_as_double((long long)below[p]);
    if (kind == 1) {
      const double d = X[kXD + 3 * p];
      const double cm = fmax(X[kXCin + p], cb);
      if (!(fabs(d) >= tol && fabs(d) >= ustab * cm)) break;
      p += 1;
    } else {
      const double d11 = X[kXD + 3 * p], d21 = X[kXD + 3 * p + 1], d22 = X[kXD + 3 * p + 2];
      const double det = fabs(d11 * d22 - d21 * d21);
      const double ad21 = fabs(d21);
      const double delta = det / fmax(fabs(d22) + ad21, fabs(d11) + ad21);
      const double cm = fmax(X[kXCin + p], cb);
      const double rm = fmax(X[kXRin + p], __longlong_as_double((long long)below[p + 1]));
      if (!(det >= tol && delta >= ustab * cm && delta >= ustab * rm)) break;
      p += 2;
    }
  }
  return p;
}

// ---------------------------------------------------------------- pass 1

constexpr int kDiagThreads = 128;

__global__ void __launch_bounds__(kDiagThreads)
    app_diag_kernel(DevState s, FactorParams prm, const int* __restrict__ list, int step) {
  __shared__ double A[kBlk][kLd];   // the block, symmetric, factored in place
  __shared__ double A0[kBlk][kLd];  // the block before the panel
  __shared__ double Lb[kBlk][kLd];
  __shared__ int perm[kBlk], kind[kBlk], dlt[kBlk];
  __shared__ double dd[3 * kBlk], cin[kBlk], rin[kBlk], below0[kBlk];
  __shared__ int sh_t, sh_moved;
  BigFront* B = s.big + list[blockIdx.x];
  if (B->state != 0) return;  // the same in every thread
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = B->f;
  const int k = B->k;
  const int ncand = B->ncand;
  const int nbk = max(0, min(kBlk, ncand - k));
  double* F = s.dpool + B->doff;
  double* Wg = s.dpool + B->woff;
  double* X = s.dpool + B->xoff;
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;

  for (int t = tid; t < kBlk * kBlk; t += blockDim.x) {
    const int i = t % kBlk, j = t / kBlk;
    const double v = (i < nbk && j < nbk) ? fsym(F, f, k + i, k + j) : 0.0;
    A[i][j] = v;
    A0[i][j] = v;
    Lb[i][j] = 0.0;
  }
  if (tid < kBlk) {
    perm[tid] = tid;
    kind[tid] = 0;
    dlt[tid] = -1;
    cin[tid] = 0.0;
    rin[tid] = 0.0;
    dd[3 * tid] = dd[3 * tid + 1] = dd[3 * tid + 2] = 0.0;
    // the previous panel's update left these columns' maxima below the block
    below0[tid] = __longlong_as_double(
        (long long)reinterpret_cast<unsigned long long*>(X + kXNext)[tid]);
  }
  __syncthreads();

  // The reference's tests on the block's candidates in order, one warp, lane
  // r owning block row r. A test's column maximum joins the block's rows
  // (exact) with the column's maximum below the block: for the panel's first
  // pivot that is below0 (exact); after it nothing is known below, so the
  // maximum used is a lower bound. A candidate that fails a test on a lower
  // bound fails it on the true maximum as well, so it is delayed for good
  // (rotated behind the block's candidates, as the reference rotates a
  // delayed candidate), unless the a-posteriori tests reject a pivot
  // accepted before it; the accepted ones are checked with the exact maxima
  // by app_accept_kernel.
  const double u = prm.ustab, tol = prm.pivot_tol;
  if (warp == 0) {
    int t = 0, nr = nbk;
    while (t < nr) {
      const double wkk = A[t][t];
      const bool has = t + 1 < nr;
      const double at = fabs(A[lane][t]);
      double bv = (lane > t && lane < nr) ? at : -1.0;
      int bi = lane;
      warp_argmax(bv, bi);
      const double abswik = has ? bv : 0.0;
      const int imax = has ? bi : t;
      // block rows that are not candidates any more (rotated behind)
      const double cnc = warp_max((lane >= nr && lane < nbk) ? at : 0.0);
      const double col_in = fmax(abswik, cnc);
      const double colmax = fmax(col_in, t == 0 ? below0[perm[t]] : 0.0);
      int stp = 0, kpiv = t;
      double row_in = 0.0;
      // a pair that formed a 2x2 pivot in the pivot record is tried as that
      // 2x2 first (the Duff test, as below), since a 1x1 test that sees only
      // the block's rows would accept the first of them alone and the
      // a-posteriori test would then reject it
      bool hinted = false;
      if (has && s.partner) {
        const int vt = fv[k + perm[t]], vn = fv[k + perm[t + 1]];
        hinted = vt >= 0 && vn >= 0 && s.partner[vt] == vn;
      }
      if (hinted) {
        const double r2 =
            warp_max((lane >= t && lane < nbk && lane != t + 1) ? fabs(A[lane][t + 1]) : 0.0);
        const double rm2 = fmax(r2, t == 0 ? below0[perm[t + 1]] : 0.0);
        const double w21 = A[t + 1][t], w22 = A[t + 1][t + 1];
        const double det = fabs(wkk * w22 - w21 * w21);
        if (det >= tol) {
          const double delta = det / fmax(fabs(w22) + fabs(w21), fabs(wkk) + fabs(w21));
          if (delta >= u * colmax && delta >= u * rm2) {
            stp = 2;
            kpiv = t + 1;
            row_in = r2;
          }
        }
      }
      if (stp != 0) {
        // taken as recorded
      } else if (fabs(wkk) >= tol && fabs(wkk) >= u * colmax) {
        stp = 1;
      } else if (has) {
        row_in = warp_max((lane >= t && lane < nbk && lane != imax) ? fabs(A[lane][imax]) : 0.0);
        const double rowmax = fmax(row_in, t == 0 ? below0[perm[imax]] : 0.0);
        const double wii = A[imax][imax], wik = A[imax][t];
        if (fabs(wii) >= tol && fabs(wii) >= u * rowmax) {
          stp = 1;
          kpiv = imax;
        } else {
          const double det = fabs(wkk * wii - wik * wik);
          if (det >= tol) {
            const double delta = det / fmax(fabs(wii) + abswik, fabs(wkk) + abswik);
            if (delta >= u * colmax && delta >= u * rowmax) {
              stp = 2;
              kpiv = imax;
            }
          }
        }
      }
      // interchange: the accepted pivot to position t (+1), or the failing
      // candidate behind the block's candidates
      const int ksrc = (stp == 0) ? t : t + stp - 1;
      const int kdst = (stp == 0) ? nr - 1 : kpiv;
      if (ksrc != kdst) {
        {
          const double x = A[ksrc][lane];
          A[ksrc][lane] = A[kdst][lane];
          A[kdst][lane] = x;
          const double y = Lb[ksrc][lane];
          Lb[ksrc][lane] = Lb[kdst][lane];
          Lb[kdst][lane] = y;
        }
        __syncwarp();
        {
          const double x = A[lane][ksrc];
          A[lane][ksrc] = A[lane][kdst];
          A[lane][kdst] = x;
        }
        if (lane == 0) {
          int q = perm[ksrc];
          perm[ksrc] = perm[kdst];
          perm[kdst] = q;
          q = dlt[ksrc];
          dlt[ksrc] = dlt[kdst];
          dlt[kdst] = q;
        }
        __syncwarp();
      }
      if (stp == 0) {
        if (lane == 0) dlt[nr - 1] = t;
        __syncwarp();
        nr--;
        continue;
      }
      if (stp == 1) {
        const double d = A[t][t];
        const double li = A[lane][t] * (1.0 / d);
        if (lane > t && lane < nbk) Lb[lane][t] = li;
        if (lane == 0) {
          kind[t] = 1;
          dd[3 * t] = d;
          cin[t] = (kpiv == t) ? col_in : row_in;
        }
      } else {
        const double d11 = A[t][t], d21 = A[t + 1][t], d22 = A[t + 1][t + 1];
        const double di = 1.0 / (d11 * d22 - d21 * d21);
        const double i00 = d22 * di, i01 = -d21 * di, i11 = d11 * di;
        const double a = A[lane][t], b = A[lane][t + 1];
        if (lane > t + 1 && lane < nbk) {
          Lb[lane][t] = a * i00 + b * i01;
          Lb[lane][t + 1] = a * i01 + b * i11;
        }
        if (lane == 0) {
          kind[t] = 2;
          kind[t + 1] = 3;
          dd[3 * t] = d11;
          dd[3 * t + 1] = d21;
          dd[3 * t + 2] = d22;
          cin[t] = col_in;
          rin[t] = row_in;
        }
      }
      __syncwarp();
      // rank-1 or rank-2 update of the block's remaining rows and columns
      // (rotated ones included): entry (i, j) gets L(max) W(min) in both
      // triangles, the lower-triangle product of the reference's update. The
      // column loop is unrolled so that its loads are in flight together.
      const int t1 = t + stp;
      if (lane >= t1 && lane < nbk) {
#pragma unroll
        for (int c = 0; c < kBlk; c++) {
          if (c >= t1 && c < nbk) {
            const int hi = max(lane, c), lo = min(lane, c);
            double v = A[lane][c] - Lb[hi][t] * A[lo][t];
            if (stp == 2) v -= Lb[hi][t + 1] * A[lo][t + 1];
            A[lane][c] = v;
          }
        }
      }
      __syncwarp();
      t = t1;
    }
    if (lane == 0) sh_t = t;
  }
  __syncthreads();
  const int acc = sh_t;
  if (warp == 0) {
    const bool moved = (lane < nbk) && perm[lane] != lane;
    const unsigned mv = __ballot_sync(0xffffffffu, moved);
    if (lane == 0) sh_moved = mv != 0u;
  }
  __syncthreads();
  const int moved = sh_moved;

  // panel state for the next passes
  for (int t = tid; t < kBlk * kLd; t += blockDim.x) X[kXL + t] = (&Lb[0][0])[t];
  if (tid < kBlk) {
    X[kXD + 3 * tid] = dd[3 * tid];
    X[kXD + 3 * tid + 1] = dd[3 * tid + 1];
    X[kXD + 3 * tid + 2] = dd[3 * tid + 2];
    X[kXCin + tid] = cin[tid];
    X[kXRin + tid] = rin[tid];
    X[kXBelow + tid] = 0.0;
    int* xi = xint(X);
    xi[kIPerm + tid] = perm[tid];
    xi[kIKind + tid] = kind[tid];
    xi[kIDlt + tid] = dlt[tid];
  }
  if (tid == 0) {
    int* xi = xint(X);
    xi[kIAcc] = acc;
    xi[kINbk] = nbk;
    xi[kIK] = k;
    xi[kIStep] = step;
    xi[kINcand] = ncand;
    xi[kIMoved] = moved;
  }
  // the W values of the block rows for the trailing update
  for (int t = tid; t < kBlk * kBlk; t += blockDim.x) {
    const int i = t % kBlk, p = t / kBlk;
    if (p < acc && i > p && i < nbk) Wg[(size_t)p * f + k + i] = A[i][p];
  }
  if (moved) {
    // the block's rows and columns follow the interchanges: the block itself
    // and the variables here; the factor rows of earlier panels in
    // app_rows_kernel
    for (int t = tid; t < kBlk * kBlk; t += blockDim.x) {
      const int i = t % kBlk, j = t / kBlk;
      if (j <= i && i < nbk) F[(k + i) + (size_t)f * (k + j)] = A0[perm[i]][perm[j]];
    }
    int a = 0, b = 0;
    if (tid < nbk) {
      a = fv[k + perm[tid]];
      b = orig[k + perm[tid]];
    }
    __syncthreads();
    if (tid < nbk) {
      fv[k + tid] = a;
      orig[k + tid] = b;
    }
  }
}

// ---------------------------------------------------------------- pass 2

__global__ void __launch_bounds__(kRowThreads)
    app_rows_kernel(DevState s, const int* __restrict__ list, int step) {
  __shared__ double Ls[kBlk][kLd];
  __shared__ int sperm[kBlk];
  __shared__ double red[kRowThreads / 32][kBlk];
  const BigFront* B = s.big + list[blockIdx.x];
  double* X = s.dpool + B->xoff;
  const int* xi = xint(X);
  if (xi[kIStep] != step) return;  // the same in every thread
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = B->f;
  const int k = xi[kIK];
  const int nbk = xi[kINbk];
  const int acc = xi[kIAcc];
  const int moved = xi[kIMoved];
  for (int t = tid; t < kBlk * kLd; t += blockDim.x) (&Ls[0][0])[t] = X[kXL + t];
  if (tid < kBlk) sperm[tid] = xi[kIPerm + tid];
  __syncthreads();
  double* F = s.dpool + B->doff;
  double* Wg = s.dpool + B->woff;
  if (moved) {
    // the block's rows in the factor columns of earlier panels: one warp per
    // column, lane i moves row k + perm[i] to row k + i
    const int gw = blockIdx.y * (kRowThreads / 32) + warp;
    const int nw = gridDim.y * (kRowThreads / 32);
    const bool mv = lane < nbk && sperm[lane] != lane;
    for (int j = gw; j < k; j += nw) {
      const double v = mv ? F[(k + sperm[lane]) + (size_t)f * j] : 0.0;
      __syncwarp();
      if (mv) F[(k + lane) + (size_t)f * j] = v;
    }
  }
  double cm[kBlk];
#pragma unroll
  for (int p = 0; p < kBlk; p++) cm[p] = 0.0;
  const int r0 = k + nbk;
  for (int r = r0 + blockIdx.y * kRowThreads + tid; r < f; r += gridDim.y * kRowThreads) {
    double a[kBlk];
#pragma unroll
    for (int j = 0; j < kBlk; j++) a[j] = (j < nbk) ? F[r + (size_t)f * (k + sperm[j])] : 0.0;
    if (moved) {
#pragma unroll
      for (int j = 0; j < kBlk; j++)
        if (j < nbk) F[r + (size_t)f * (k + j)] = a[j];
    }
    // W = F21 L11^-T: forward substitution with the block's unit lower L
#pragma unroll
    for (int p = 0; p < kBlk; p++) {
      if (p < acc) {
        double w = a[p];
#pragma unroll
        for (int q = 0; q < p; q++) w = fma(-a[q], Ls[p][q], w);
        a[p] = w;
        Wg[(size_t)p * f + r] = w;
        cm[p] = fmax(cm[p], fabs(w));
      }
    }
  }
  // column maxima: warp, CTA, then the front (non-negative doubles compare
  // as their bit patterns)
#pragma unroll
  for (int p = 0; p < kBlk; p++) {
    const double v = warp_max(cm[p]);
    if (lane == 0) red[warp][p] = v;
  }
  __syncthreads();
  if (tid < kBlk && tid < acc) {
    double v = 0.0;
    for (int w = 0; w < kRowThreads / 32; w++) v = fmax(v, red[w][tid]);
    atomicMax(reinterpret_cast<unsigned long long*>(X + kXBelow) + tid,
              (unsigned long long)__double_as_longlong(v));
  }
}

// ---------------------------------------------------------------- pass 3

__global__ void __launch_bounds__(kRowThreads)
    app_accept_kernel(DevState s, FactorParams prm, const int* __restrict__ list, int step) {
  __shared__ double Ls[kBlk][kLd];
  __shared__ double sd[3 * kBlk], sinv[kBlk];
  __shared__ int skind[kBlk];
  __shared__ int sh_np;
  BigFront* B = s.big + list[blockIdx.x];
  double* X = s.dpool + B->xoff;
  int* xi = xint(X);
  if (xi[kIStep] != step) return;  // the same in every thread
  const int tid = threadIdx.x;
  const int f = B->f;
  const int k = xi[kIK];
  const int nbk = xi[kINbk];
  if (tid == 0) sh_np = passing_prefix(X, prm.ustab, prm.pivot_tol);
  for (int t = tid; t < kBlk * kLd; t += blockDim.x) (&Ls[0][0])[t] = X[kXL + t];
  if (tid < kBlk) {
    skind[tid] = xi[kIKind + tid];
    sd[3 * tid] = X[kXD + 3 * tid];
    sd[3 * tid + 1] = X[kXD + 3 * tid + 1];
    sd[3 * tid + 2] = X[kXD + 3 * tid + 2];
    // 1x1 pivots scale their column by 1/d, as the reference does
    sinv[tid] = (xi[kIKind + tid] == 1) ? 1.0 / X[kXD + 3 * tid] : 0.0;
  }
  __syncthreads();
  const int np = sh_np;
  double* F = s.dpool + B->doff;
  const double* Wg = s.dpool + B->woff;
  // L of the accepted pivots on the rows below the block
  for (int r = k + nbk + blockIdx.y * kRowThreads + tid; r < f; r += gridDim.y * kRowThreads) {
    for (int p = 0; p < np;) {
      if (skind[p] == 1) {
        F[r + (size_t)f * (k + p)] = Wg[(size_t)p * f + r] * sinv[p];
        p += 1;
      } else {
        const double d11 = sd[3 * p], d21 = sd[3 * p + 1], d22 = sd[3 * p + 2];
        const double di = 1.0 / (d11 * d22 - d21 * d21);
        const double a = Wg[(size_t)p * f + r], b = Wg[(size_t)(p + 1) * f + r];
        F[r + (size_t)f * (k + p)] = a * (d22 * di) + b * (-d21 * di);
        F[r + (size_t)f * (k + p + 1)] = a * (-d21 * di) + b * (d11 * di);
        p += 2;
      }
    }
  }
  if (blockIdx.y != 0) return;
  // the block's rows: D on the diagonal (d21 below a 2x2's first column), L
  for (int t = tid; t < kBlk * kBlk; t += blockDim.x) {
    const int i = t % kBlk, p = t / kBlk;
    if (p >= np || i < p || i >= nbk) continue;
    double v;
    if (i == p)
      v = (skind[p] == 3) ? sd[3 * (p - 1) + 2] : sd[3 * p];
    else if (i == p + 1 && skind[p] == 2)
      v = sd[3 * p + 1];
    else
      v = Ls[i][p];
    F[(k + i) + (size_t)f * (k + p)] = v;
  }
  if (tid != 0) return;
  // commit the panel (no other CTA reads the descriptor in this pass)
  int* fv = s.ivars + B->ioff;
  int npos = 0, nneg = 0;
  double flops = 0.0;
  for (int p = 0; p < np;) {
    if (skind[p] == 1) {
      if (sd[3 * p] >= 0.0)
        npos++;
      else
        nneg++;
      flops += 2.0 * (double)(f - k - p) * (p + 1);
      p += 1;
    } else {
      const double d11 = sd[3 * p], d21 = sd[3 * p + 1], d22 = sd[3 * p + 2];
      const double det = d11 * d22 - d21 * d21;
      if (det >= 0.0) {
        if (d11 >= 0.0)
          npos += 2;
        else
          nneg += 2;
      } else {
        npos++;
        nneg++;
      }
      fv[k + p] = -(fv[k + p] + 1);
      fv[k + p + 1] = -(fv[k + p + 1] + 1);
      flops += 4.0 * (double)(f - k - p) * (p + 2);
      p += 2;
    }
  }
  // candidates to delay: those that failed in the block while only pivots
  // that are now accepted preceded them, and the first pivot the
  // a-posteriori tests reject (positions decreasing); candidates that failed
  // after a rejected pivot are tried again
  const int acc = xi[kIAcc];
  const int ncand = xi[kINcand];
  int nd = 0;
  for (int q = nbk - 1; q >= acc; q--)
    if (xi[kIDlt + q] >= 0 && xi[kIDlt + q] <= np) xi[kIDpos + nd++] = k + q;
  if (np < acc) xi[kIDpos + nd++] = k + np;
  xi[kIDcnt] = nd;
  B->kstart = k;
  B->kw = np;
  B->k = k + np;
  B->pending = nd;
  B->npos += npos;
  B->nneg += nneg;
  B->flops += flops;
  atomicAdd(s.flops + 1, flops);
  atomicAdd(s.flops + 5, 1.0);
  if (np < acc) atomicAdd(s.flops + 6, 1.0);
  atomicAdd(s.flops + 7, (double)(nd - (np < acc ? 1 : 0)));
  // the next panel's column maxima, filled by the trailing update
  for (int j = 0; j < kBlk; j++) X[kXNext + j] = 0.0;
  B->state = (nd == 0 && k + np >= ncand) ? 1 : 0;
}

// ---------------------------------------------------------------- delay

// After the trailing update: each candidate to delay moves behind the
// remaining candidates (the reference's symm_swap with ncand - 1), largest
// position first so that no interchange moves another one still to go.
__global__ void app_delay_kernel(DevState s, const int* __restrict__ list, int step) {
  BigFront* B = s.big + list[blockIdx.x];
  double* X = s.dpool + B->xoff;
  const int* xi = xint(X);
  if (xi[kIStep] != step) return;  // the same in every thread
  const int nd = xi[kIDcnt];
  if (nd <= 0) return;
  const int f = B->f;
  const int k = B->k;
  int ncand = B->ncand;
  double* F = s.dpool + B->doff;
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;
  double* next = X + kXNext;
  for (int q = 0; q < nd; q++) {
    const int a = xi[kIDpos + q];
    const int b = ncand - 1;
    if (a < b) {
      for (int j = threadIdx.x; j < f; j += blockDim.x) {
        double *p, *r;
        if (j < a) {
          p = F + a + (size_t)f * j;
          r = F + b + (size_t)f * j;
        } else if (j == a) {
          p = F + a + (size_t)f * a;
          r = F + b + (size_t)f * b;
        } else if (j < b) {
          p = F + j + (size_t)f * a;
          r = F + b + (size_t)f * j;
        } else if (j == b) {
          continue;
        } else {
          p = F + j + (size_t)f * a;
          r = F + j + (size_t)f * b;
        }
        const double t = *p;
        *p = *r;
        *r = t;
      }
      if (threadIdx.x == 0) {
        int t = fv[a];
        fv[a] = fv[b];
        fv[b] = t;
        t = orig[a];
        orig[a] = orig[b];
        orig[b] = t;
        // columns that moved lose their estimate
        if (a - k < kBlk) next[a - k] = 0.0;
        if (b - k < kBlk) next[b - k] = 0.0;
      }
    }
    ncand--;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    B->ncand = ncand;
    B->pending = 0;
    if (B->k >= B->ncand) B->state = 2;
  }
}

__global__ void app_open_kernel(DevState s, const int* __restrict__ list, int count) {
  int open = 0, rem = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const BigFront& B = s.big[list[i]];
    if (B.state != 2) {
      open++;
      rem = max(rem, B.ncand - B.k);
    }
  }
  atomicAdd(s.big_meta + 19, open);
  atomicMax(s.big_meta + 20, rem);
}

}  // namespace

cudaError_t launch_app_panel(const DevState& s, const FactorParams& prm, int count, int max_f,
                             const int* list, int step, cudaStream_t stream) {
  static_assert(kBlk == kBigPanelMax, "panel width");
  if (count <= 0) return cudaSuccess;
  const int ych = std::max(1, std::min(64, (max_f + kRowThreads - 1) / kRowThreads));
  app_diag_kernel<<<count, 128, 0, stream>>>(s, prm, list, step);
  app_rows_kernel<<<dim3(count, ych), kRowThreads, 0, stream>>>(s, list, step);
  app_accept_kernel<<<dim3(count, ych), kRowThreads, 0, stream>>>(s, prm, list, step);
  return cudaGetLastError();
}

cudaError_t launch_app_delay(const DevState& s, int count, const int* list, int step,
                             cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  app_delay_kernel<<<count, 256, 0, stream>>>(s, list, step);
  return cudaGetLastError();
}

cudaError_t launch_app_open_count(const DevState& s, int count, const int* list,
                                  cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  app_open_kernel<<<1, 256, 0, stream>>>(s, list, count);
  return cudaGetLastError();
}

}  // namespace b200ldl
