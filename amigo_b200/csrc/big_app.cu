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
// what costs time, not arithmetic. Here a panel of up to 32 candidates of
// every front of a tree level is decided in data-parallel phases:
//
//   D. Delays left by the previous panel are applied with the reference's
//      symmetric interchange (symm_swap, sparse_ldl.h:1270-1292), by the
//      whole CTA when the level has no more fronts than CTAs, else by one
//      warp per front; the next block's column maxima below follow the
//      interchanges. Then one warp factors the 32 x 32 diagonal block with
//      the reference's tests (lane r owns block row r), left-looking: a
//      column is formed from the loaded block and the pivots taken when a
//      test reads it. A test's column maximum joins the block's rows with,
//      for the panel's first pivot, the column's exact maximum below the
//      block that the previous panel's trailing update left behind. A pair
//      that formed a 2x2 pivot in the pivot record is tried as that 2x2
//      first. A candidate that fails is rotated behind the block's
//      candidates.
//   R. (row chunks) Every row below the block forms its entries of the
//      pivot columns, W = F21 L11^-T (the values the reference's tests see),
//      stores them for the trailing update, and the column maxima over all
//      rows below are reduced. The front's last chunk to finish runs the
//      reference's tests exactly, with the column maxima over the whole
//      front, and records how many leading pivots pass.
//   A+U. The row chunks write L for the passing pivots (D on the diagonal,
//      2x2 blocks with d21 below it, as the reference stores them) and the
//      first of them commits the panel; beside them, 64 x 64 tiles give the
//      trailing matrix the rank-kw update, forming L from W as the commit
//      does. The first rejected pivot, and the candidates that failed in
//      the block while only accepted pivots preceded them, are delayed at
//      the next phase D. (In the mixed-precision mode the commit and the
//      update are separate phases: the tensor-core tiles read L from the
//      front.)
//
// Every accepted pivot therefore satisfies the reference's threshold test
// against its whole column, so the factorization has the reference's
// stability bound (|L| <= 1/ustab for 1x1 pivots) and, by Sylvester's law,
// its inertia; only the order in which candidates are tried differs (a
// candidate's 2x2 partner is searched within its panel's block). A root
// cannot delay: the candidates its tests leave are finished by the chained
// panels (Bunch-Kaufman) after the level's launch.
//
// The phases run in one cooperative launch per level, separated by grid-wide
// barriers: three per panel step. Every CTA runs the same phases and
// barriers; the loop ends for all of them on a count that the barrier makes
// visible to all, or at a cap that the progress of every step guarantees
// not to reach (each step of an active front accepts a pivot or delays a
// candidate).
//
// The front stays in HBM in logical order between steps (column-major,
// lower triangle, the layout big_chain.cu and big_update_kernel use). A
// panel's state lives in a per-front scratch area (xoff) stamped with the
// step number, so a front that finished earlier takes no part.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "ldl_internal.h"
#include "umma.cuh"

namespace cg = cooperative_groups;

namespace b200ldl {

namespace {

constexpr int kBlk = 32;  // candidates per panel
constexpr int kLd = kBlk + 1;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileU = 64;          // trailing-update tile
constexpr int kChunkFronts = 1024;  // fronts per work-item prefix

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
constexpr int kIDlt = 64;    // [32] candidates failed in the block: pivots accepted before
constexpr int kIAcc = 96;    // pivots accepted inside the block
constexpr int kINbk = 97;    // candidates in the block
constexpr int kIK = 98;      // first position of the panel
constexpr int kIStep = 99;   // step number of the panel
constexpr int kINcand = 100;
constexpr int kIMoved = 101;  // 1 if the block permutation is not the identity
constexpr int kIDcnt = 102;   // candidates to delay at the next step
constexpr int kIDpos = 103;   // [32] their positions, decreasing
constexpr int kINp = kIDpos + kBlk;  // pivots that pass the exact tests (set by phase R)
constexpr int kIRdone = kINp + 1;    // phase-R items of the panel finished
constexpr int kINint = kIRdone + 1;
static_assert(kXInt + (kINint + 1) / 2 <= kAppScratch, "a-posteriori scratch size");

__device__ __forceinline__ double fsym(const double* F, int f, int a, int b) {
  return (a >= b) ? F[a + (size_t)f * b] : F[b + (size_t)f * a];
}

__device__ __forceinline__ int* xint(double* X) { return reinterpret_cast<int*>(X + kXInt); }

// Non-negative doubles order as their bit patterns, so the warp reductions
// below are exact integer reductions (redux.sync) on the high and then the
// low 32 bits, instead of FP64 shuffle butterflies.

// Largest of the non-negative values v of the lanes with `on`, and the
// lowest lane holding it (idamax); -1 and lane 0 when no lane is on.
__device__ __forceinline__ void warp_argmax(bool on, double v, double& best, int& idx) {
  const unsigned long long b = on ? (unsigned long long)__double_as_longlong(v) : 0ull;
  // +1 keeps an active 0.0 above the inactive lanes
  const unsigned hi = on ? (unsigned)(b >> 32) + 1u : 0u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const bool cand = on && hi == mhi;
  const unsigned lo = cand ? (unsigned)b : 0u;
  const unsigned mlo = __reduce_max_sync(0xffffffffu, lo);
  const unsigned win = __ballot_sync(0xffffffffu, cand && lo == mlo);
  idx = win ? __ffs(win) - 1 : 0;
  best = mhi ? __longlong_as_double((long long)(((unsigned long long)(mhi - 1u) << 32) | mlo))
             : -1.0;
}

// largest of the lanes' non-negative values
__device__ __forceinline__ double warp_max(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  const unsigned mhi = __reduce_max_sync(0xffffffffu, (unsigned)(b >> 32));
  const unsigned mlo = __reduce_max_sync(0xffffffffu, (unsigned)(b >> 32) == mhi ? (unsigned)b : 0u);
  return __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

// The L entries (l0, l1) of a row whose W entries are (a, b) under the 2x2
// pivot d = (d11, d21, d22): (a, b) D^-1, with explicit fused multiply-adds so
// that every kernel that forms them gets the same values.
__device__ __forceinline__ void l_2x2(const double* d, double a, double b, double& l0,
                                      double& l1) {
  const double d11 = d[0], d21 = d[1], d22 = d[2];
  const double di = 1.0 / (d11 * d22 - d21 * d21);
  const double i00 = d22 * di, i01 = -d21 * di, i11 = d11 * di;
  l0 = fma(a, i00, b * i01);
  l1 = fma(a, i01, b * i11);
}

// ------------------------------------------------------------- shared memory

struct WarpDiag {  // phase D, one per warp
  double A[kBlk][kLd];  // the block, symmetric, factored in place
  double Lb[kBlk][kLd];
  double dd[3 * kBlk], cin[kBlk], rin[kBlk], below0[kBlk];
  int perm[kBlk], kind[kBlk], dlt[kBlk];
  int var[kBlk], part[kBlk];  // block candidates' variables and recorded 2x2 partners
};

struct RowsSm {  // phases R and A
  double Ls[kBlk][kLd];
  double red[kWarps][kBlk];
  double sd[3 * kBlk], sinv[kBlk];
  double scm[kBlk], srm[kBlk];  // phase A: column maxima over the front, 2x2 partner's block part
  int sperm[kBlk], skind[kBlk];
  int np;
};

// The reference's tests for the accepted pivots of a panel, with the column
// maxima over the whole front (staged in shared memory by phase A): number
// of leading pivots that pass.
__device__ int passing_prefix(const RowsSm& sm, int acc, double ustab, double tol) {
  int p = 0;
  while (p < acc) {
    const double cm = sm.scm[p];
    if (sm.skind[p] == 1) {
      const double d = sm.sd[3 * p];
      if (!(fabs(d) >= tol && fabs(d) >= ustab * cm)) break;
      p += 1;
    } else {
      const double d11 = sm.sd[3 * p], d21 = sm.sd[3 * p + 1], d22 = sm.sd[3 * p + 2];
      const double det = fabs(d11 * d22 - d21 * d21);
      const double ad21 = fabs(d21);
      const double delta = det / fmax(fabs(d22) + ad21, fabs(d11) + ad21);
      // the partner's maximum: its block part (srm) and its maximum below
      // (scm of the second position, whose block part phase D leaves at 0)
      const double rm = fmax(sm.srm[p], sm.scm[p + 1]);
      if (!(det >= tol && delta >= ustab * cm && delta >= ustab * rm)) break;
      p += 2;
    }
  }
  return p;
}

struct UpdSm {  // phase U
  double As[kBigPanelMax][kTileU];
  double Bs[kBigPanelMax][kTileU];
  double ud[3 * kBlk], usinv[kBlk];  // the panel's D, when L is formed from W
  int ukind[kBlk];
};

struct Prefix {  // work items of up to kChunkFronts fronts
  long long ptr[kChunkFronts + 1];
  long long wsum[kWarps];
};

constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
// the mixed-precision tile places the tensor-core operands after the FP64
// tiles' panels, 1 KB aligned
constexpr size_t kOpsOffset = (sizeof(UpdSm) + 1023) / 1024 * 1024;
constexpr size_t kDynSmem =
    cmax(sizeof(WarpDiag) * kWarps,
         cmax(sizeof(RowsSm), kOpsOffset + umma::kSmemFloats * sizeof(float)));

// Exclusive prefix of cnt(i) over i in [0, nl) into P.ptr (CTA-wide; nl <=
// kChunkFronts). Returns the total.
template <typename Count>
__device__ long long front_prefix(Prefix& P, int nl, Count cnt) {
  constexpr int per = kChunkFronts / kThreads;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int w = tid >> 5;
  long long c[per];
  long long mine = 0;
#pragma unroll
  for (int u = 0; u < per; u++) {
    const int i = tid * per + u;
    c[u] = (i < nl) ? cnt(i) : 0;
    mine += c[u];
  }
  long long incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) P.wsum[w] = incl;
  __syncthreads();
  long long base = 0;
  for (int q = 0; q < w; q++) base += P.wsum[q];
  long long run = base + incl - mine;
  if (tid == 0) P.ptr[0] = 0;
#pragma unroll
  for (int u = 0; u < per; u++) {
    run += c[u];
    const int i = tid * per + u;
    if (i < nl) P.ptr[i + 1] = run;
  }
  __syncthreads();
  return P.ptr[nl];
}

// front of work item t: the last i with ptr[i] <= t
__device__ __forceinline__ int item_front(const Prefix& P, int nl, long long t) {
  int lo = 0, hi = nl;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (P.ptr[mid] <= t)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------- phase D

// A front whose candidates are all decided is done, except a root with
// candidates left (delayed by the tests; a root has no parent to take them):
// they become candidates again and the root waits in `done` for the chained
// panels (Bunch-Kaufman) that run after this launch.
__device__ void finish_front(const DevState& s, BigFront* B, int* done, int* meta) {
  if (B->nc == 0 && B->k < B->fs) {
    B->ncand = B->fs;
    B->state = 3;
    done[atomicAdd(meta + 19, 1)] = (int)(B - s.big);
    atomicMax(meta + 20, B->fs - B->k);
  } else {
    B->state = 2;
  }
}

template <int NT>
__device__ __forceinline__ void group_sync() {
  if constexpr (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}

// Close the previous step of front B (trailing-update work counters, a
// finished front becomes done) and apply the delays it left, by a group of
// NT threads (a warp, or the CTA when the level has no more fronts than
// CTAs); g is the thread's index in the group. Returns 1 if the front takes
// part in this step.
template <int NT>
__device__ int phase_d_prepare(const DevState& s, BigFront* B, int* done, int* meta, int g) {
  const int f = B->f;
  double* F = s.dpool + B->doff;
  double* X = s.dpool + B->xoff;
  int* xi = xint(X);
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;
  if (g == 0 && B->kw > 0) {
    const double r = (double)(f - B->k);
    const double fl = r * (r + 1.0) * B->kw;
    B->flops += fl;
    atomicAdd(s.flops + 2, fl);
    atomicAdd(s.flops + 3, 8.0 * (r * (r + 1.0) + 2.0 * r * B->kw));
  }
  group_sync<NT>();
  if (g == 0) {
    B->kw = 0;
    if (B->state == 1) finish_front(s, B, done, meta);
  }
  group_sync<NT>();
  if (B->pending > 0 && B->state == 0) {
    // the candidates to delay move behind the remaining candidates, largest
    // position first so that no interchange moves another one still to go
    const int nd = xi[kIDcnt];
    const int k = B->k;
    int ncand = B->ncand;
    // The next panel's first test needs the exact maximum below the block
    // (rows from k + kBlk on) of every block column. An interchange of rows
    // a (in the block) and b (below it) takes row b's entry out of a
    // column's rows below and puts the entry of row a in: thread g < kBlk
    // follows column k + g, which is formed again afterwards only if the
    // entry taken out may have been its maximum, or if it is a or b.
    const int ct = k + g;
    const bool trk = g < kBlk && ct < f;
    bool stale = false;
    double mx = trk ? X[kXNext + g] : 0.0;
    for (int q = 0; q < nd; q++) {
      const int a = xi[kIDpos + q];
      const int b = ncand - 1;
      if (a < b) {
        if (trk) {
          if (ct == a || ct == b) {
            stale = true;
          } else if (b >= k + kBlk) {
            const double out = fabs(fsym(F, f, b, ct)), in = fabs(fsym(F, f, a, ct));
            if (out >= mx) stale = true;
            mx = fmax(mx, in);
          }
        }
        group_sync<NT>();  // those reads before the interchange
        // the pairs of a symmetric interchange are distinct entries: eight
        // passes of the group load theirs before any is stored back
        constexpr int kU = 8;
        for (int j0 = 0; j0 < f; j0 += NT * kU) {
          double* p[kU];
          double* r[kU];
          double vp[kU], vr[kU];
#pragma unroll
          for (int u = 0; u < kU; u++) {
            const int j = j0 + NT * u + g;
            p[u] = nullptr;
            r[u] = nullptr;
            if (j >= f || j == b) continue;
            if (j < a) {
              p[u] = F + a + (size_t)f * j;
              r[u] = F + b + (size_t)f * j;
            } else if (j == a) {
              p[u] = F + a + (size_t)f * a;
              r[u] = F + b + (size_t)f * b;
            } else if (j < b) {
              p[u] = F + j + (size_t)f * a;
              r[u] = F + b + (size_t)f * j;
            } else {
              p[u] = F + j + (size_t)f * a;
              r[u] = F + j + (size_t)f * b;
            }
          }
#pragma unroll
          for (int u = 0; u < kU; u++) {
            vp[u] = p[u] ? *p[u] : 0.0;
            vr[u] = p[u] ? *r[u] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kU; u++) {
            if (p[u]) {
              *p[u] = vr[u];
              *r[u] = vp[u];
            }
          }
        }
        if (g == 0) {
          int t = fv[a];
          fv[a] = fv[b];
          fv[b] = t;
          t = orig[a];
          orig[a] = orig[b];
          orig[b] = t;
        }
      }
      ncand--;
      group_sync<NT>();
    }
    // the block columns whose maximum below may have changed, formed again
    unsigned redo;
    if constexpr (NT == 32) {
      redo = __ballot_sync(0xffffffffu, trk && stale);
    } else {
      __shared__ unsigned redo_sh;
      if (g < 32) {
        const unsigned m = __ballot_sync(0xffffffffu, trk && stale);
        if (g == 0) redo_sh = m;
      }
      group_sync<NT>();
      redo = redo_sh;
    }
    if (trk && !stale) X[kXNext + g] = mx;
    const int lane = g & 31, wq = g >> 5;
    for (int i = wq; i < kBlk; i += NT / 32) {
      if (!((redo >> i) & 1u)) continue;
      const double* col = F + (size_t)f * (k + i);
      double m = 0.0;
      for (int r = k + kBlk + lane; r < f; r += 32) m = fmax(m, fabs(col[r]));
      m = warp_max(m);
      if (lane == 0) X[kXNext + i] = m;
    }
    group_sync<NT>();
    if (g == 0) {
      B->ncand = ncand;
      B->pending = 0;
      if (B->k >= ncand) finish_front(s, B, done, meta);
    }
    group_sync<NT>();
  }
  return B->state == 0 ? 1 : 0;
}

// Factor the next diagonal block of front B (one warp). Returns 1.
__device__ int phase_d_block(const DevState& s, const FactorParams& prm, BigFront* B, int step,
                             WarpDiag& w) {
  const int lane = threadIdx.x & 31;
  const int f = B->f;
  double* F = s.dpool + B->doff;
  double* Wg = s.dpool + B->woff;
  double* X = s.dpool + B->xoff;
  int* xi = xint(X);
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;

  const int k = B->k;
  const int ncand = B->ncand;
  const int nbk = max(0, min(kBlk, ncand - k));
  {
    // the block's lower triangle, one coalesced column per load (all loads
    // in flight before the shared-memory stores), mirrored above
    double v[kBlk];
#pragma unroll
    for (int j = 0; j < kBlk; j++)
      v[j] = (j <= lane && lane < nbk) ? F[(k + lane) + (size_t)f * (k + j)] : 0.0;
    // the candidates' variables and the partners they had in the record
    const int var = (lane < nbk) ? fv[k + lane] : -1;
    const int part = (var >= 0 && s.partner) ? s.partner[var] : -1;
    // entry (i, j) and its mirror are written by lane max(i, j) only
#pragma unroll
    for (int j = 0; j < kBlk; j++) {
      if (j <= lane) {
        w.A[lane][j] = v[j];
        w.A[j][lane] = v[j];
      }
      w.Lb[lane][j] = 0.0;
    }
    w.var[lane] = var;
    w.part[lane] = part;
  }
  w.perm[lane] = lane;
  w.kind[lane] = 0;
  w.dlt[lane] = -1;
  w.cin[lane] = 0.0;
  w.rin[lane] = 0.0;
  w.dd[3 * lane] = w.dd[3 * lane + 1] = w.dd[3 * lane + 2] = 0.0;
  w.below0[lane] = __longlong_as_double(
      (long long)reinterpret_cast<unsigned long long*>(X + kXNext)[lane]);
  // read: the trailing update of this panel fills them again for the next
  X[kXNext + lane] = 0.0;
  __syncwarp();

  // The reference's tests on the block's candidates in order. For the
  // panel's first pivot the column maximum below the block is exact
  // (below0); after it nothing is known below, so the maximum used is a
  // lower bound: a candidate that fails on a lower bound fails on the true
  // maximum as well, so it is delayed, unless the a-posteriori tests reject
  // a pivot accepted before it. Accepted pivots are checked with the exact
  // maxima in phase A.
  const double u = prm.ustab, tol = prm.pivot_tol;
  constexpr unsigned kFull = 0xffffffffu;
  int t = 0, nr = nbk;
  // Left-looking: the block keeps its entries as loaded in the columns not
  // pivoted yet, next to the pivot columns (W) and the L rows of the pivots
  // taken. A column that a test reads is formed when it is read: entry
  // (i, j) minus L(max(i, j), q) W(min(i, j), q) for each earlier pivot q in
  // order, the products and the order of the reference's lower-triangle
  // update. Lane i forms row i.
  auto form = [&](int j) -> double {
    if (lane < t || lane >= nbk) return 0.0;
    const int hi = max(lane, j), lo = min(lane, j);
    double v = w.A[lane][j];
    for (int q = 0; q < t; q++) v = fma(-w.Lb[hi][q], w.A[lo][q], v);
    return v;
  };
  while (t < nr) {
    const bool has = t + 1 < nr;
    const double ct = form(t);  // the candidate's column
    const double wkk = __shfl_sync(kFull, ct, t);
    const double at = fabs(ct);
    double bv;
    int bi;
    warp_argmax(lane > t && lane < nr, at, bv, bi);
    const double abswik = has ? bv : 0.0;
    const int imax = has ? bi : t;
    // block rows that are not candidates any more (rotated behind)
    const double cnc = (nr < nbk) ? warp_max((lane >= nr && lane < nbk) ? at : 0.0) : 0.0;
    const double col_in = fmax(abswik, cnc);
    const double colmax = fmax(col_in, t == 0 ? w.below0[w.perm[t]] : 0.0);
    int stp = 0, kpiv = t;
    double row_in = 0.0;
    double c2 = 0.0;  // the column of the partner or of imax, when formed
    // a pair that formed a 2x2 pivot in the pivot record is tried as that
    // 2x2 first (the Duff test), since a 1x1 test that sees only the block's
    // rows would accept the first of them alone and the a-posteriori test
    // would then reject it
    bool hinted = false;
    if (has) {
      const int pt = w.perm[t], vn = w.var[w.perm[t + 1]];
      hinted = w.var[pt] >= 0 && vn >= 0 && w.part[pt] == vn;
    }
    if (hinted) {
      c2 = form(t + 1);
      const double r2 = warp_max((lane >= t && lane < nbk && lane != t + 1) ? fabs(c2) : 0.0);
      const double rm2 = fmax(r2, t == 0 ? w.below0[w.perm[t + 1]] : 0.0);
      const double w21 = __shfl_sync(kFull, ct, t + 1), w22 = __shfl_sync(kFull, c2, t + 1);
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
      c2 = form(imax);
      row_in = warp_max((lane >= t && lane < nbk && lane != imax) ? fabs(c2) : 0.0);
      const double rowmax = fmax(row_in, t == 0 ? w.below0[w.perm[imax]] : 0.0);
      const double wii = __shfl_sync(kFull, c2, imax), wik = __shfl_sync(kFull, ct, imax);
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
        const double x = w.A[ksrc][lane];
        w.A[ksrc][lane] = w.A[kdst][lane];
        w.A[kdst][lane] = x;
        const double y = w.Lb[ksrc][lane];
        w.Lb[ksrc][lane] = w.Lb[kdst][lane];
        w.Lb[kdst][lane] = y;
      }
      __syncwarp();
      {
        const double x = w.A[lane][ksrc];
        w.A[lane][ksrc] = w.A[lane][kdst];
        w.A[lane][kdst] = x;
      }
      if (lane == 0) {
        int q = w.perm[ksrc];
        w.perm[ksrc] = w.perm[kdst];
        w.perm[kdst] = q;
        q = w.dlt[ksrc];
        w.dlt[ksrc] = w.dlt[kdst];
        w.dlt[kdst] = q;
      }
      __syncwarp();
    }
    if (stp == 0) {
      if (lane == 0) w.dlt[nr - 1] = t;
      __syncwarp();
      nr--;
      continue;
    }
    // the pivot columns at their positions after the interchange (rows
    // ksrc and kdst exchanged), stored as W for the later columns
    const int src = (lane == ksrc) ? kdst : (lane == kdst) ? ksrc : lane;
    const double p1 = __shfl_sync(kFull, (stp == 1 && kpiv != t) ? c2 : ct, src);
    const double p2 = __shfl_sync(kFull, c2, src);
    if (lane >= t && lane < nbk) {
      w.A[lane][t] = p1;
      if (stp == 2) w.A[lane][t + 1] = p2;
    }
    if (stp == 1) {
      const double d = __shfl_sync(kFull, p1, t);
      const double li = p1 * (1.0 / d);
      if (lane > t && lane < nbk) w.Lb[lane][t] = li;
      if (lane == 0) {
        w.kind[t] = 1;
        w.dd[3 * t] = d;
        w.cin[t] = (kpiv == t) ? col_in : row_in;
      }
    } else {
      const double d11 = __shfl_sync(kFull, p1, t), d21 = __shfl_sync(kFull, p1, t + 1),
                   d22 = __shfl_sync(kFull, p2, t + 1);
      // the expressions of the commit and of the update tiles (l_2x2)
      const double dv[3] = {d11, d21, d22};
      double l0, l1;
      l_2x2(dv, p1, p2, l0, l1);
      if (lane > t + 1 && lane < nbk) {
        w.Lb[lane][t] = l0;
        w.Lb[lane][t + 1] = l1;
      }
      if (lane == 0) {
        w.kind[t] = 2;
        w.kind[t + 1] = 3;
        w.dd[3 * t] = d11;
        w.dd[3 * t + 1] = d21;
        w.dd[3 * t + 2] = d22;
        w.cin[t] = col_in;
        w.rin[t] = row_in;
      }
    }
    __syncwarp();
    t += stp;
  }
  const int acc = t;
  const bool moved = __ballot_sync(0xffffffffu, lane < nbk && w.perm[lane] != lane) != 0u;

  // panel state for phases R and A
  for (int q = lane; q < kBlk * kLd; q += 32) X[kXL + q] = (&w.Lb[0][0])[q];
  X[kXD + 3 * lane] = w.dd[3 * lane];
  X[kXD + 3 * lane + 1] = w.dd[3 * lane + 1];
  X[kXD + 3 * lane + 2] = w.dd[3 * lane + 2];
  X[kXCin + lane] = w.cin[lane];
  X[kXRin + lane] = w.rin[lane];
  X[kXBelow + lane] = 0.0;
  xi[kIPerm + lane] = w.perm[lane];
  xi[kIKind + lane] = w.kind[lane];
  xi[kIDlt + lane] = w.dlt[lane];
  if (lane == 0) {
    xi[kIRdone] = 0;
    xi[kIAcc] = acc;
    xi[kINbk] = nbk;
    xi[kIK] = k;
    xi[kIStep] = step;
    xi[kINcand] = ncand;
    xi[kIMoved] = moved ? 1 : 0;
  }
  // the W values of the block rows for the trailing update
  for (int q = lane; q < kBlk * kBlk; q += 32) {
    const int i = q % kBlk, p = q / kBlk;
    if (p < acc && i > p && i < nbk) Wg[(size_t)p * f + k + i] = w.A[i][p];
  }
  if (moved) {
    // the block itself and the variables follow the interchanges (the factor
    // rows of earlier panels move in phase R): lane i gathers its row
    // before any lane writes
    double v[kBlk];
#pragma unroll
    for (int j = 0; j < kBlk; j++)
      v[j] = (j <= lane && lane < nbk) ? fsym(F, f, k + w.perm[lane], k + w.perm[j]) : 0.0;
    const int a = (lane < nbk) ? fv[k + w.perm[lane]] : 0;
    const int b = (lane < nbk) ? orig[k + w.perm[lane]] : 0;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kBlk; j++)
      if (j <= lane && lane < nbk) F[(k + lane) + (size_t)f * (k + j)] = v[j];
    if (lane < nbk) {
      fv[k + lane] = a;
      orig[k + lane] = b;
    }
  }
  __syncwarp();
  return 1;
}

// ---------------------------------------------------------------- phase R

__device__ __forceinline__ bool active(const DevState& s, const BigFront& B, int step) {
  return xint(s.dpool + B.xoff)[kIStep] == step;
}

// row chunks of an active front in phases R and A (at least one, which also
// carries the moves of earlier factor rows)
__device__ __forceinline__ int row_chunks(const DevState& s, const BigFront& B, int step) {
  if (!active(s, B, step)) return 0;
  const int* xi = xint(s.dpool + B.xoff);
  const int rows = B.f - (xi[kIK] + xi[kINbk]);
  return max(1, (rows + kThreads - 1) / kThreads);
}

__device__ void phase_r_item(const DevState& s, const FactorParams& prm, const BigFront& B,
                             int chunk, int nchunk, RowsSm& sm) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  double* X = s.dpool + B.xoff;
  int* xi = xint(X);
  const int f = B.f;
  const int k = xi[kIK];
  const int nbk = xi[kINbk];
  const int acc = xi[kIAcc];
  const int moved = xi[kIMoved];
  for (int t = tid; t < kBlk * kLd; t += kThreads) (&sm.Ls[0][0])[t] = X[kXL + t];
  if (tid < kBlk) sm.sperm[tid] = xi[kIPerm + tid];
  __syncthreads();
  double* F = s.dpool + B.doff;
  double* Wg = s.dpool + B.woff;
  if (moved) {
    // the block's rows in the factor columns of earlier panels: one warp per
    // column, lane i moves row k + perm[i] to row k + i
    const bool mv = lane < nbk && sm.sperm[lane] != lane;
    for (int j = chunk * kWarps + warp; j < k; j += nchunk * kWarps) {
      const double v = mv ? F[(k + sm.sperm[lane]) + (size_t)f * j] : 0.0;
      __syncwarp();
      if (mv) F[(k + lane) + (size_t)f * j] = v;
    }
  }
  double cm[kBlk];
#pragma unroll
  for (int p = 0; p < kBlk; p++) cm[p] = 0.0;
  const int r = k + nbk + chunk * kThreads + tid;
  if (r < f) {
    double a[kBlk];
#pragma unroll
    for (int j = 0; j < kBlk; j++) a[j] = (j < nbk) ? F[r + (size_t)f * (k + sm.sperm[j])] : 0.0;
    if (moved) {
#pragma unroll
      for (int j = 0; j < kBlk; j++)
        if (j < nbk) F[r + (size_t)f * (k + j)] = a[j];
    }
    // W = F21 L11^-T: forward substitution with the block's unit lower L
#pragma unroll
    for (int p = 0; p < kBlk; p++) {
      if (p < acc) {
        double wv = a[p];
#pragma unroll
        for (int q = 0; q < p; q++) wv = fma(-a[q], sm.Ls[p][q], wv);
        a[p] = wv;
        Wg[(size_t)p * f + r] = wv;
        cm[p] = fabs(wv);
      }
    }
  }
  // column maxima: warp, CTA, then the front (non-negative doubles compare
  // as their bit patterns)
#pragma unroll
  for (int p = 0; p < kBlk; p++) {
    const double v = warp_max(cm[p]);
    if (lane == 0) sm.red[warp][p] = v;
  }
  __syncthreads();
  if (tid < acc) {
    double v = 0.0;
    for (int q = 0; q < kWarps; q++) v = fmax(v, sm.red[q][tid]);
    if (v > 0.0)
      atomicMax(reinterpret_cast<unsigned long long*>(X + kXBelow) + tid,
                (unsigned long long)__double_as_longlong(v));
  }
  // the front's last item to finish has the column maxima over the whole
  // front: it runs the reference's tests on the block's pivots and records
  // how many pass (kINp), for the commit and the trailing update
  __threadfence();
  __syncthreads();
  if (tid == 0) sm.np = (atomicAdd(xi + kIRdone, 1) == nchunk - 1) ? 1 : 0;
  __syncthreads();
  if (sm.np) {
    __threadfence();
    if (tid < kBlk) {
      sm.skind[tid] = xi[kIKind + tid];
      sm.sd[3 * tid] = X[kXD + 3 * tid];
      sm.sd[3 * tid + 1] = X[kXD + 3 * tid + 1];
      sm.sd[3 * tid + 2] = X[kXD + 3 * tid + 2];
      const unsigned long long bl =
          *(reinterpret_cast<volatile unsigned long long*>(X + kXBelow) + tid);
      sm.scm[tid] = fmax(X[kXCin + tid], __longlong_as_double((long long)bl));
      sm.srm[tid] = X[kXRin + tid];
    }
    __syncthreads();
    if (tid == 0) xi[kINp] = passing_prefix(sm, acc, prm.ustab, prm.pivot_tol);
  }
  __syncthreads();
}

// ---------------------------------------------------------------- phase A


__device__ void phase_a_item(const DevState& s, const FactorParams& prm, BigFront* B, int chunk,
                             RowsSm& sm) {
  const int tid = threadIdx.x;
  double* X = s.dpool + B->xoff;
  int* xi = xint(X);
  const int f = B->f;
  const int k = xi[kIK];
  const int nbk = xi[kINbk];
  for (int t = tid; t < kBlk * kLd; t += kThreads) (&sm.Ls[0][0])[t] = X[kXL + t];
  if (tid < kBlk) {
    sm.skind[tid] = xi[kIKind + tid];
    sm.sd[3 * tid] = X[kXD + 3 * tid];
    sm.sd[3 * tid + 1] = X[kXD + 3 * tid + 1];
    sm.sd[3 * tid + 2] = X[kXD + 3 * tid + 2];
    // 1x1 pivots scale their column by 1/d, as the reference does
    sm.sinv[tid] = (xi[kIKind + tid] == 1) ? 1.0 / X[kXD + 3 * tid] : 0.0;
  }
  __syncthreads();
  const int np = xi[kINp];
  double* F = s.dpool + B->doff;
  const double* Wg = s.dpool + B->woff;
  // L of the accepted pivots on the rows below the block
  const int r = k + nbk + chunk * kThreads + tid;
  if (r < f) {
    for (int p = 0; p < np;) {
      if (sm.skind[p] == 1) {
        F[r + (size_t)f * (k + p)] = Wg[(size_t)p * f + r] * sm.sinv[p];
        p += 1;
      } else {
        double l0, l1;
        l_2x2(sm.sd + 3 * p, Wg[(size_t)p * f + r], Wg[(size_t)(p + 1) * f + r], l0, l1);
        F[r + (size_t)f * (k + p)] = l0;
        F[r + (size_t)f * (k + p + 1)] = l1;
        p += 2;
      }
    }
  }
  if (chunk == 0) {
    // the block's rows: D on the diagonal (d21 below a 2x2's first column), L
    for (int t = tid; t < kBlk * kBlk; t += kThreads) {
      const int i = t % kBlk, p = t / kBlk;
      if (p >= np || i < p || i >= nbk) continue;
      double v;
      if (i == p)
        v = (sm.skind[p] == 3) ? sm.sd[3 * (p - 1) + 2] : sm.sd[3 * p];
      else if (i == p + 1 && sm.skind[p] == 2)
        v = sm.sd[3 * p + 1];
      else
        v = sm.Ls[i][p];
      F[(k + i) + (size_t)f * (k + p)] = v;
    }
    if (tid == 0) {
      // commit the panel (the other items of this front read only the
      // scratch, never the descriptor)
      int* fv = s.ivars + B->ioff;
      int npos = 0, nneg = 0;
      double flops = 0.0;
      for (int p = 0; p < np;) {
        if (sm.skind[p] == 1) {
          if (sm.sd[3 * p] >= 0.0)
            npos++;
          else
            nneg++;
          flops += 2.0 * (double)(f - k - p) * (p + 1);
          p += 1;
        } else {
          const double d11 = sm.sd[3 * p], d21 = sm.sd[3 * p + 1], d22 = sm.sd[3 * p + 2];
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
      // candidates to delay: those that failed in the block while only
      // pivots that are now accepted preceded them, and the first pivot the
      // a-posteriori tests reject (positions decreasing); candidates that
      // failed after a rejected pivot are tried again
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
      B->state = (nd == 0 && k + np >= ncand) ? 1 : 0;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- phase U

// One 64 x 64 lower tile of front B's trailing matrix at rows i0, columns
// j0: the rank-kw update with the panel's L (columns ks..ks+kw) and W (Wg),
// in FP64; k = ks + kw is the trailing matrix's first position. L is read
// from the front's columns once committed, or (from_w) formed from W and
// the panel's D as the commit forms it.
__device__ void phase_u_tile(const DevState& s, const BigFront& B, int i0, int j0, int k, int kw,
                             int ks, bool from_w, UpdSm& sm) {
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  const int f = B.f;
  double* F = s.dpool + B.doff;
  const double* W = s.dpool + B.woff;
  if (from_w && tid < kBlk) {
    const double* X = s.dpool + B.xoff;
    const int kd = reinterpret_cast<const int*>(X + kXInt)[kIKind + tid];
    sm.ukind[tid] = kd;
    sm.ud[3 * tid] = X[kXD + 3 * tid];
    sm.ud[3 * tid + 1] = X[kXD + 3 * tid + 1];
    sm.ud[3 * tid + 2] = X[kXD + 3 * tid + 2];
    sm.usinv[tid] = (kd == 1) ? 1.0 / X[kXD + 3 * tid] : 0.0;
  }
  double cur[4][4];
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int j = j0 + ty + 16 * b;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const int i = i0 + tx + 16 * a;
      cur[a][b] = (j < f && i < f && i >= j) ? F[i + (size_t)f * j] : 0.0;
    }
  }
  {
    constexpr int kPer = kBigPanelMax * kTileU / kThreads;
    double pa[kPer], pb[kPer];
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      const int e = tid + kThreads * q;
      const int c = e / kTileU;
      const int rr = e - c * kTileU;
      pa[q] = 0.0;
      pb[q] = 0.0;
      if (c < kw) {
        if (i0 + rr < f)
          pa[q] = from_w ? W[(size_t)c * f + i0 + rr] : F[i0 + rr + (size_t)f * (ks + c)];
        if (j0 + rr < f) pb[q] = W[(size_t)c * f + j0 + rr];
      }
    }
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      const int e = tid + kThreads * q;
      const int c = e / kTileU;
      const int rr = e - c * kTileU;
      if (c < kw) {
        sm.As[c][rr] = pa[q];
        sm.Bs[c][rr] = pb[q];
      }
    }
  }
  __syncthreads();
  if (from_w) {
    // L = W D^-1 on the tile's rows, the commit's expressions
    for (int e = tid; e < kw * kTileU; e += kThreads) {
      const int c = e / kTileU, rr = e - c * kTileU;
      const int kd = sm.ukind[c];
      if (kd == 1) {
        sm.As[c][rr] = sm.As[c][rr] * sm.usinv[c];
      } else if (kd == 2) {
        double l0, l1;
        l_2x2(sm.ud + 3 * c, sm.As[c][rr], sm.As[c + 1][rr], l0, l1);
        sm.As[c][rr] = l0;
        sm.As[c + 1][rr] = l1;
      }
    }
    __syncthreads();
  }
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
  for (int c = 0; c < kw; c++) {
    double av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; a++) av[a] = sm.As[c][tx + 16 * a];
#pragma unroll
    for (int b = 0; b < 4; b++) bv[b] = sm.Bs[c][ty + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
  }
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int j = j0 + ty + 16 * b;
    if (j >= f) continue;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const int i = i0 + tx + 16 * a;
      if (i < f && i >= j) F[i + (size_t)f * j] = cur[a][b] - acc[a][b];
    }
  }
  if (j0 == k) {
    // the next panel's columns [k, k + 32): their largest magnitude over the
    // rows below the next block, for its first test (the 16 threads with
    // the same ty are one half-warp)
    unsigned long long* nxt =
        reinterpret_cast<unsigned long long*>(s.dpool + B.xoff + kAppNextColmax);
#pragma unroll
    for (int b = 0; b < 2; b++) {
      double m = 0.0;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int i = i0 + tx + 16 * a;
        if (i < f && i >= k + kBigPanelMax) m = fmax(m, fabs(cur[a][b] - acc[a][b]));
      }
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      const int j = j0 + ty + 16 * b;
      if (tx == 0 && j < f && m > 0.0)
        atomicMax(nxt + (ty + 16 * b), (unsigned long long)__double_as_longlong(m));
    }
  }
  __syncthreads();
}

__device__ __forceinline__ long long tri_tiles_rows(int rows, int tile) {
  const long long t = (rows + tile - 1) / tile;
  return t * (t + 1) / 2;
}

__device__ __forceinline__ long long tri_tiles(const BigFront& B, int tile) {
  return tri_tiles_rows(B.f - B.k, tile);
}

__device__ __forceinline__ void tri_decode(long long lt, int& I, int& J) {
  I = (int)((sqrt(8.0 * (double)lt + 1.0) - 1.0) * 0.5);
  while ((long long)(I + 1) * (I + 2) / 2 <= lt) I++;
  while ((long long)I * (I + 1) / 2 > lt) I--;
  J = (int)(lt - (long long)I * (I + 1) / 2);
}

// Mixed precision: a 128 x 128 tile (I, J) of the trailing matrix. Tiles of
// the contribution block (columns from fs on: rows that the parent
// assembles, never pivoted in this front) take the update on the tensor
// cores (umma.cuh, 3xTF32 products accumulated in FP32); the others, which
// hold the fully summed columns whose pivots are still to be decided, stay
// in FP64 as four 64 x 64 tiles. Returns 1 if a tensor-core operation did
// not complete in time.
__device__ int phase_u_tile_mixed(const DevState& s, const BigFront& B, int I, int J, UpdSm& sm,
                                  float* ops, uint64_t* mbar, uint32_t* phase, uint32_t tmem) {
  const int f = B.f, k = B.k;
  const int i0 = k + I * umma::kTileM;
  const int j0 = k + J * umma::kTileN;
  if (j0 >= B.fs) {
    double* F = s.dpool + B.doff;
    const double* W = s.dpool + B.woff;
    return umma::tile_update(F, f, F + (size_t)f * B.kstart, f, W, f, i0, j0,
                             min(umma::kTileM, f - i0), min(umma::kTileN, f - j0), B.kw, I == J,
                             ops, mbar, phase, tmem);
  }
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      const int si = i0 + a * kTileU, sj = j0 + b * kTileU;
      if (si < f && sj < f && si + kTileU - 1 >= sj)
        phase_u_tile(s, B, si, sj, B.k, B.kw, B.kstart, false, sm);
    }
  return 0;
}

// ---------------------------------------------------------------- the level

__global__ void __launch_bounds__(kThreads, 1)
    app_level_kernel(DevState s, FactorParams prm, const int* __restrict__ list, int nl,
                     int max_steps, int* done, int* meta) {
  int* counters = meta + 21;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(1024) unsigned char dsm[];
  __shared__ Prefix P;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int gwarp = blockIdx.x * kWarps + warp;
  const int nwarp = gridDim.x * kWarps;
  // mixed precision: 128 tensor-memory columns per CTA for the accumulator
  uint32_t tmem = 0, phase = 0;
  int tc_fail = 0;
  if (prm.mixed) {
    if (warp == 0) umma::tmem_alloc_128(&tmem_slot);
    if (tid == 0) umma::mbar_init(&mbar);
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    tmem = tmem_slot;
  }
  int step = 1;
  for (; step <= max_steps; step++) {
    // ---- D: one warp per front
    {
      WarpDiag& w = reinterpret_cast<WarpDiag*>(dsm)[warp];
      if (blockIdx.x == 0 && tid == 0) counters[(step + 1) & 1] = 0;
      if (nl <= (int)gridDim.x) {
        // a CTA per front: its threads apply the delays, warp 0 the block
        if ((int)blockIdx.x < nl) {
          BigFront* B = s.big + list[blockIdx.x];
          if (phase_d_prepare<kThreads>(s, B, done, meta, tid) && warp == 0) {
            phase_d_block(s, prm, B, step, w);
            if (tid == 0) atomicAdd(counters + (step & 1), 1);
          }
        }
      } else {
        for (int i = gwarp; i < nl; i += nwarp) {
          BigFront* B = s.big + list[i];
          if (phase_d_prepare<32>(s, B, done, meta, tid & 31)) {
            phase_d_block(s, prm, B, step, w);
            if ((tid & 31) == 0) atomicAdd(counters + (step & 1), 1);
          }
        }
      }
    }
    grid.sync();
    if (*((volatile int*)(counters + (step & 1))) == 0) break;  // the same in every CTA
    // ---- R: row chunks of the active fronts
    for (int c0 = 0; c0 < nl; c0 += kChunkFronts) {
      const int n = min(kChunkFronts, nl - c0);
      const long long total = front_prefix(
          P, n, [&](int i) { return (long long)row_chunks(s, s.big[list[c0 + i]], step); });
      RowsSm& sm = *reinterpret_cast<RowsSm*>(dsm);
      for (long long t = blockIdx.x; t < total; t += gridDim.x) {
        const int fi = item_front(P, n, t);
        const BigFront& B = s.big[list[c0 + fi]];
        const int nchunk = (int)(P.ptr[fi + 1] - P.ptr[fi]);
        phase_r_item(s, prm, B, (int)(t - P.ptr[fi]), nchunk, sm);
      }
      __syncthreads();
    }
    grid.sync();
    if (!prm.mixed) {
      // ---- A and U together: the row chunks that write L and commit the
      // panel, then the trailing-update tiles, which form L from W and take
      // the panel's position from the scratch, not from the descriptor that
      // the commit changes meanwhile
      for (int c0 = 0; c0 < nl; c0 += kChunkFronts) {
        const int n = min(kChunkFronts, nl - c0);
        const long long total = front_prefix(P, n, [&](int i) {
          const BigFront& B = s.big[list[c0 + i]];
          const int ra = row_chunks(s, B, step);
          if (ra == 0) return 0ll;
          const int* xi = xint(s.dpool + B.xoff);
          const int np = xi[kINp];
          return (long long)ra + (np > 0 ? tri_tiles_rows(B.f - (xi[kIK] + np), kTileU) : 0ll);
        });
        for (long long t = blockIdx.x; t < total; t += gridDim.x) {
          const int fi = item_front(P, n, t);
          BigFront* B = s.big + list[c0 + fi];
          const long long it = t - P.ptr[fi];
          const int ra = row_chunks(s, *B, step);
          if (it < ra) {
            phase_a_item(s, prm, B, (int)it, *reinterpret_cast<RowsSm*>(dsm));
          } else {
            const int* xi = xint(s.dpool + B->xoff);
            const int ks = xi[kIK], np = xi[kINp];
            int I, J;
            tri_decode(it - ra, I, J);
            phase_u_tile(s, *B, ks + np + I * kTileU, ks + np + J * kTileU, ks + np, np, ks, true,
                         *reinterpret_cast<UpdSm*>(dsm));
          }
        }
        __syncthreads();
      }
      grid.sync();
      continue;
    }
    // ---- A: the same items; the first one of a front commits the panel
    for (int c0 = 0; c0 < nl; c0 += kChunkFronts) {
      const int n = min(kChunkFronts, nl - c0);
      const long long total = front_prefix(
          P, n, [&](int i) { return (long long)row_chunks(s, s.big[list[c0 + i]], step); });
      RowsSm& sm = *reinterpret_cast<RowsSm*>(dsm);
      for (long long t = blockIdx.x; t < total; t += gridDim.x) {
        const int fi = item_front(P, n, t);
        phase_a_item(s, prm, s.big + list[c0 + fi], (int)(t - P.ptr[fi]), sm);
      }
      __syncthreads();
    }
    grid.sync();
    // ---- U (mixed precision): trailing-update tiles of the fronts that
    // accepted pivots, after the commit
    for (int c0 = 0; c0 < nl; c0 += kChunkFronts) {
      const int n = min(kChunkFronts, nl - c0);
      const long long total = front_prefix(P, n, [&](int i) {
        const BigFront& B = s.big[list[c0 + i]];
        return (active(s, B, step) && B.kw > 0) ? tri_tiles(B, umma::kTileM) : 0ll;
      });
      UpdSm& sm = *reinterpret_cast<UpdSm*>(dsm);
      for (long long t = blockIdx.x; t < total; t += gridDim.x) {
        const int fi = item_front(P, n, t);
        const BigFront& B = s.big[list[c0 + fi]];
        int I, J;
        tri_decode(t - P.ptr[fi], I, J);
        if (!tc_fail) {
          // the tensor-core operands share the dynamic shared memory with
          // the FP64 tiles' panels (a tile uses one or the other)
          float* ops = reinterpret_cast<float*>(dsm + kOpsOffset);
          tc_fail = phase_u_tile_mixed(s, B, I, J, sm, ops, &mbar, &phase, tmem);
        }
      }
      __syncthreads();
    }
    grid.sync();
  }
  // the step cap (never reached when every step makes progress)
  if (step > max_steps && blockIdx.x == 0 && tid == 0) counters[2] = 1;
  // every CTA has left the loop: the roots set aside take part in the
  // chained panels that follow
  if (blockIdx.x == 0) {
    const int nd = *((volatile int*)(meta + 19));
    for (int i = tid; i < nd; i += kThreads) s.big[done[i]].state = 0;
  }
  if (prm.mixed) {
    if (tc_fail) {
      // a tensor-core operation did not complete in time: the factorization
      // is reported failed; wait once more (bounded) before freeing TMEM
      if (tid == 0) counters[2] = 2;
      umma::mbar_wait(&mbar, phase ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) umma::tmem_free_128(tmem);
  }
}

}  // namespace

cudaError_t launch_app_level(const DevState& s, const FactorParams& prm, int count, int max_fs,
                             const int* list, int* done, int* meta, cudaStream_t stream) {
  static_assert(kBlk == kBigPanelMax, "panel width");
  if (count <= 0) return cudaSuccess;
  int dev = 0, nsm = 0, per = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, app_level_kernel, kThreads, kDynSmem);
  if (e != cudaSuccess) return e;
  if (per < 1) return cudaErrorLaunchOutOfResources;
  const int grid = nsm * per;
  // every step of an active front accepts a pivot or delays a candidate
  int max_steps = max_fs + 8;
  DevState sa = s;
  FactorParams pa = prm;
  const int* la = list;
  int na = count;
  int* da = done;
  int* ma = meta;
  void* args[] = {(void*)&sa, (void*)&pa,        (void*)&la, (void*)&na,
                  (void*)&max_steps, (void*)&da, (void*)&ma};
  return cudaLaunchCooperativeKernel((const void*)app_level_kernel, dim3(grid), dim3(kThreads),
                                     args, kDynSmem, stream);
}

cudaError_t configure_app_kernels() {
  return cudaFuncSetAttribute(app_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kDynSmem);
}

}  // namespace b200ldl
