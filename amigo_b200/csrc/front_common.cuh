// Pieces shared by the chained pivot search of the on-chip front kernel
// (cluster_front.cu) and of the big-front panel kernel (big_chain.cu).
//
// Both evaluate a chain of candidates per step: the candidate at position k
// and the ones the reference's delays would swap in from the end of the
// candidate range (SparseLDL::factor_front_matrix_block,
// include/sparse_ldl.h:1316-1553). Each member's statistics are reduced over
// the cluster, the threshold tests are applied to every member under the
// hypothesis that the members before it were delayed, and the first member
// that is accepted ends the chain.
#pragma once

#include <climits>

#include "ldl_internal.h"

namespace b200ldl {
namespace chain {

enum : int { kDelay = 0, kOne = 1, kTwo = 2, kNeedRow = 3, kZero = 4, kOneImax = 5 };

__device__ __forceinline__ void keep_larger(double& bv, int& bi, double v, int i) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

// statistics of one candidate column over one CTA's rows outside the chain
struct ColStat {
  double bv;  // largest |.| among candidate rows (0 when there is none)
  double cm;  // largest |.| among non-candidate rows
  int bi;     // logical position of bv (smallest on ties; INT_MAX if none)
  int pad;
};

// what one chain member's tests need, reduced over the cluster
struct Cand {
  double wkk, abswik, colmax;  // pivot, best candidate entry, column max
  double rmax, wii, wik;       // imax column: max off-diagonal, diagonal, entry at k
  int dec1;                    // kOne / kZero / kNeedRow / kDelay from the column alone
  int dec2;                    // kOne / kOneImax / kTwo / kDelay after the imax column
  int imaxp;                   // imax: physical row
  int mrow;                    // the member's physical row
};

// Warp-wide maximum of a non-negative double in every lane. Non-negative
// IEEE doubles order like their bit patterns, so the maximum is taken with
// two 32-bit integer reductions (high word, then low word among the lanes
// holding the highest high word): exact, and far fewer dependent steps than
// a butterfly of FP64 compares.
__device__ __forceinline__ double warp_max_nonneg(double v) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(u >> 32);
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? (unsigned)u : 0u);
  return __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
}

// warp-wide (argmax with the smallest index on ties, max) of non-negative
// values in every lane; lanes without a candidate hold (0, INT_MAX)
__device__ __forceinline__ void warp_argmax_max(double& bv, int& bi, double& cm) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(bv);
  const unsigned hi = (unsigned)(u >> 32);
  const unsigned lo = (unsigned)u;
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
  bi = __reduce_min_sync(0xffffffffu, (hi == mh && lo == ml) ? bi : INT_MAX);
  bv = __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
  cm = warp_max_nonneg(cm);
}

constexpr int kChain = 8;  // chain members per step, one per warp
constexpr double kAlphaBK = (1.0 + 4.1231056256176605) / 8.0;  // (1 + sqrt(17)) / 8

// Exchange buffers of the chained search, one copy in every CTA of the
// cluster (members push their partials into all copies). NPAR copies
// alternate with the step parity so that a CTA one step ahead never
// overwrites what a slower CTA still reads.
template <int CL, int NPAR>
struct ChainXchg {
  ColStat s1[NPAR][CL][kChain];    // per-CTA column statistics
  double s2[NPAR][CL][kChain];     // per-CTA imax-column maxima
  double V[NPAR][kChain][kChain];  // V[t][j]: column of member t at member j's row
  double P2[NPAR][kChain][2];      // (w_ii, w_ik) of member t
  Cand cand[kChain];
};

// Member t's tests from its column alone, by warp t after the first
// exchange, under the hypothesis that members 0..t-1 were delayed (they are
// non-candidates by then) and members t+1.. are still candidates at their
// own positions (ncand - j). Lane l brings CTA l's partial and the member
// entry V[t][l]; every lane takes the same decision and lane 0 records it.
template <int CL, int NPAR, typename IdxT>
__device__ __forceinline__ void decide_column(ChainXchg<CL, NPAR>& x, int par, int t, int lane,
                                              int nS, int k, int ncand, bool root,
                                              const FactorParams& prm, const IdxT* perm) {
  double bv = 0.0, cm = 0.0;
  int bi = INT_MAX;
  if (lane < CL) {
    const ColStat st = x.s1[par][lane][t];
    bv = st.bv;
    cm = st.cm;
    bi = st.bi;
  }
  if (lane < nS && lane != t) {
    const double a = fabs(x.V[par][t][lane]);
    if (lane > t)
      keep_larger(bv, bi, a, ncand - lane);
    else
      cm = fmax(cm, a);
  }
  __syncwarp();
  warp_argmax_max(bv, bi, cm);
  const int nc_t = ncand - t;
  const bool has = (k + 1 < nc_t);
  const double wkk = x.V[par][t][t];
  const double abswkk = fabs(wkk);
  const double abswik = has ? bv : 0.0;
  const int il = has ? (bi < nc_t ? bi : k + 1) : k;
  const double colmax = fmax(abswik, cm);
  int d1;
  if (prm.cholesky) {
    d1 = kOne;
  } else if (root) {
    if (fmax(abswkk, colmax) == 0.0)
      d1 = kZero;
    else if (abswkk >= kAlphaBK * colmax)
      d1 = kOne;
    else
      d1 = kNeedRow;
  } else if (abswkk >= prm.pivot_tol && abswkk >= prm.ustab * colmax) {
    d1 = kOne;
  } else {
    d1 = has ? kNeedRow : kDelay;
  }
  if (lane == 0) {
    const int mrow = (t == 0) ? (int)perm[k] : (int)perm[ncand - t];
    Cand& c = x.cand[t];
    c.wkk = wkk;
    c.abswik = abswik;
    c.colmax = colmax;
    c.dec1 = d1;
    c.dec2 = kDelay;
    // positions other than k below ncand - t hold what perm says
    c.imaxp = (il == k) ? mrow : (int)perm[il];
    c.mrow = mrow;
  }
}

// Members that need their imax column: those before the first member
// accepted from its column alone. Every warp computes the same masks.
__device__ __forceinline__ unsigned need_rows(const Cand* cand, int nS, int lane, unsigned& acc1,
                                              int& d1l) {
  d1l = (lane < nS) ? cand[lane].dec1 : kDelay;
  acc1 = __ballot_sync(0xffffffffu, d1l == kOne || d1l == kZero);
  const unsigned nrow = __ballot_sync(0xffffffffu, d1l == kNeedRow);
  return nrow & (acc1 ? (acc1 & (0u - acc1)) - 1u : 0xffffffffu);
}

// Member t's tests with its imax column, by warp t after the second
// exchange (row maximum reduced over the CTAs' partials).
template <int CL, int NPAR>
__device__ __forceinline__ void decide_row(ChainXchg<CL, NPAR>& x, int par, int t, int lane,
                                           bool root, const FactorParams& prm) {
  double rm = (lane < CL) ? x.s2[par][lane][t] : 0.0;
  __syncwarp();
  rm = warp_max_nonneg(rm);
  const Cand& c = x.cand[t];
  const double wii = x.P2[par][t][0];
  const double wik = x.P2[par][t][1];
  const double abswii = fabs(wii);
  const double abswkk = fabs(c.wkk);
  int d2;
  if (root) {
    if (abswkk >= kAlphaBK * c.colmax * (c.colmax / rm))
      d2 = kOne;
    else if (abswii >= kAlphaBK * rm)
      d2 = kOneImax;
    else
      d2 = kTwo;
  } else if (abswii >= prm.pivot_tol && abswii >= prm.ustab * rm) {
    d2 = kOneImax;
  } else {
    const double det = fabs(c.wkk * wii - wik * wik);
    d2 = kDelay;
    if (det >= prm.pivot_tol) {
      const double delta = det / fmax(abswii + c.abswik, abswkk + c.abswik);
      if (delta >= prm.ustab * c.colmax && delta >= prm.ustab * rm) d2 = kTwo;
    }
  }
  __syncwarp();
  if (lane == 0) {
    Cand& cw = x.cand[t];
    cw.rmax = rm;
    cw.wii = wii;
    cw.wik = wik;
    cw.dec2 = d2;
  }
}

// The sequential decisions replayed: the first accepted member (nS when
// every member is delayed) and how it is accepted.
__device__ __forceinline__ void replay(const Cand* cand, int nS, int lane, unsigned acc1, int d1l,
                                       int& tacc, int& kind) {
  const int d2l = (lane < nS) ? cand[lane].dec2 : kDelay;
  const unsigned acc2 = __ballot_sync(0xffffffffu, d1l == kNeedRow && d2l != kDelay);
  const unsigned accm = acc1 | acc2;
  tacc = accm ? __ffs(accm) - 1 : nS;
  kind = (tacc == nS) ? kDelay : ((acc1 >> tacc) & 1u) ? cand[tacc].dec1 : cand[tacc].dec2;
}

// The logical order after the step, by one warp: member t (t < ndelay)
// goes to ncand-1-t and what stood at ncand-ndelay comes to k (the
// reference's swaps with the last candidate, ncand shrinking by one each
// time), then the pivot interchange (imax to k for a 1x1 at imax, to k + 1
// for a 2x2).
template <typename IdxT>
__device__ __forceinline__ void reorder(const Cand* cand, IdxT* perm, IdxT* ipos, int lane, int nS,
                                        int ndelay, int k, int ncand, int kind, int nstep,
                                        int pi) {
  int xk = -1;
  if (ndelay > 0 && ncand - ndelay > k)
    xk = (ndelay < nS) ? cand[ndelay].mrow : (int)perm[ncand - ndelay];
  const int mt = (lane < ndelay) ? cand[lane].mrow : -1;
  __syncwarp();
  if (lane < ndelay) {
    perm[ncand - 1 - lane] = (IdxT)mt;
    ipos[mt] = (IdxT)(ncand - 1 - lane);
  }
  if (lane == 0 && xk >= 0) {
    perm[k] = (IdxT)xk;
    ipos[xk] = (IdxT)k;
  }
  __syncwarp();
  if (lane == 0 && (kind == kOneImax || kind == kTwo)) {
    const int a = k + nstep - 1, b = ipos[pi];
    if (a != b) {
      const IdxT pa = perm[a], pb = perm[b];
      perm[a] = pb;
      perm[b] = pa;
      ipos[pb] = (IdxT)a;
      ipos[pa] = (IdxT)b;
    }
  }
  __syncwarp();
}

}  // namespace chain
}  // namespace b200ldl
