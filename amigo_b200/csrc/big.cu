// Fronts too large for one CTA's shared memory.
//
// Each big front F (f x f, column-major, lower triangle used) lives in the
// device pool. Its fully summed candidates are factored panel by panel with
// the reference's blocked algorithm (SparseLDL::factor_front_matrix_block,
// include/sparse_ldl.h:1316-1553): within a panel the next candidate column
// is formed on the fly as F(:,k) - Lp W(k,:)^T, tested (1x1, alternative
// 1x1 at imax, Duff 2x2, or delay; Bunch-Kaufman when the front has no
// contribution rows), and accepted columns are appended to the panel; after
// the panel the trailing matrix receives one rank-kw update.
//
// B200 mapping: the panel of one front is owned by a thread-block cluster
// (4, 8 or 16 CTAs). Rows are split in contiguous blocks across the CTAs and
// each CTA keeps its rows of the panel's L and W columns in shared memory,
// so the per-column GEMV never leaves the SM. Column maxima are reduced
// across the cluster through distributed shared memory, and every CTA makes
// the same pivot decision from the same reduced values, so all CTAs run the
// same sequence of cluster barriers. The trailing update is a separate
// tiled FP64 kernel over all big fronts of the level.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "ldl_internal.h"

namespace cg = cooperative_groups;

namespace b200ldl {

namespace {

constexpr int kPanelThreads = 256;
constexpr int kPWarps = kPanelThreads / 32;
constexpr int kTile = 64;
constexpr int kUpdThreads = 256;
constexpr int kUpdMaxFronts = 1024;  // class-5 fronts per level handled by one update launch

__device__ __forceinline__ void keep_larger(double& bv, int& bi, double v, int i) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

struct Part {
  double v;  // best |.| among candidates
  int i;     // its row
  int pad;
  double m;  // max |.| among contribution rows / row max
  double x;  // a value owned by this CTA (diagonal etc.)
  double y;
};

struct BlockRed {
  double v[kPWarps];
  int i[kPWarps];
  double m[kPWarps];
};

__device__ void block_reduce(BlockRed& r, double& bv, int& bi, double& cm) {
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
  for (int q = 1; q < kPWarps; q++) {
    keep_larger(bv, bi, r.v[q], r.i[q]);
    cm = fmax(cm, r.m[q]);
  }
  __syncthreads();
}

// ---------------------------------------------------------------- assembly

// Zero the lower triangle of every big front of a level: independent of
// the assembly order, so every SM takes part (a CTA per eight columns).
__global__ void big_zero_kernel(DevState s, const int* __restrict__ list) {
  const BigFront& B = s.big[list[blockIdx.x]];
  double* F = s.dpool + B.doff;
  const int f = B.f;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int j = blockIdx.y * nw + warp; j < f; j += gridDim.y * nw) {
    double* col = F + (size_t)f * j;
    for (int i = j + lane; i < f; i += 32) col[i] = 0.0;
  }
}

// Assembly of every big front of a level in one launch, after
// big_zero_kernel: a front per cluster of CL CTAs (CL = 1: a front per CTA).
// The cluster writes Sigma on the own variables' diagonal, adds the CSR
// entries of its pivot columns, then extend-adds its children's
// contribution blocks one child after another, with a cluster barrier
// between the steps. Each entry therefore receives its terms in the order
// diag, CSR value, children in child order; since the front starts at zero
// and each position receives at most one CSR value, d + v is the same
// number as the (0 + v) + d of adding the diagonal after the values, as
// SparseLDL::assemble_front_matrix followed by factor's add_diagonal does
// (include/sparse_ldl.h:1078-1104).
template <int CL>
__device__ __forceinline__ void asm_sync() {
  if constexpr (CL == 1)
    __syncthreads();
  else
    cg::this_cluster().sync();
}

template <int CL>
__global__ void __launch_bounds__(256) big_assemble_kernel(DevPlan p, DevState s,
                                                          const double* __restrict__ vals,
                                                          const double* __restrict__ diag,
                                                          const int* __restrict__ list) {
  const BigFront& B = s.big[list[blockIdx.x / CL]];
  const int rank = (int)(blockIdx.x % CL);
  double* F = s.dpool + B.doff;
  const int f = B.f, ns = B.ns, nd_in = B.nd_in, node = B.node;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  constexpr int kW = 8;  // warps per CTA
  const int v0 = p.var_ptr[node];
  // Sigma on the diagonal of the own variables (the front is zero)
  if (diag)
    for (int j = rank * blockDim.x + threadIdx.x; j < ns; j += CL * blockDim.x)
      F[j + (size_t)f * j] = diag[p.node_to_var[v0 + j]];
  // a-posteriori panels: no column maxima for the first panel yet
  if (B.app && rank == 0 && threadIdx.x < kBigPanelMax)
    s.dpool[B.xoff + kAppNextColmax + threadIdx.x] = 0.0;
  asm_sync<CL>();
  // the CSR entries of the pivot columns (distinct positions)
  {
    const int64_t e0 = p.scat_ptr[node];
    const int64_t e1 = p.scat_ptr[node + 1];
    for (int64_t e = e0 + (int64_t)rank * blockDim.x + threadIdx.x; e < e1;
         e += (int64_t)CL * blockDim.x) {
      int r = p.scat_row[e];
      if (r >= ns) r += nd_in;
      F[r + (size_t)f * p.scat_col[e]] += csr_value(s, vals, p.scat_csr[e]);
    }
  }
  // the children's contribution blocks, one child after another
  const int kb = p.kid_ptr[node];
  const int ke = p.kid_ptr[node + 1];
  int off = ns;  // first position of this child's delayed rows
  for (int q = kb; q < ke; q++) {
    asm_sync<CL>();
    const int ch = p.kids[q];
    const int nd = s.ndel[ch];
    const int m = s.f[ch] - s.npiv[ch];
    const double* cb = s.dpool + s.cb_off[ch];
    const int cld = s.cb_ld[ch];
    const int* cm = p.cmap + p.cptr[ch];
    for (int r2 = rank * kW + warp; r2 < m; r2 += CL * kW) {
      int p2;
      if (r2 < nd) {
        p2 = off + r2;
      } else {
        p2 = cm[r2 - nd];
        if (p2 >= ns) p2 += nd_in;
      }
      const double* col = cb + (size_t)cld * r2;
      // four entries per lane pass: their loads (map, value, front) are in
      // flight together before the read-modify-writes
      for (int rb = r2 + lane; rb < m; rb += 128) {
        double* dst[4];
        double val[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int r1 = rb + 32 * u;
          dst[u] = nullptr;
          if (r1 < m) {
            int p1;
            if (r1 < nd) {
              p1 = off + r1;
            } else {
              p1 = cm[r1 - nd];
              if (p1 >= ns) p1 += nd_in;
            }
            dst[u] = (p1 >= p2) ? F + (p1 + (size_t)f * p2) : F + (p2 + (size_t)f * p1);
            val[u] = col[r1];
          }
        }
        double old[4];
#pragma unroll
        for (int u = 0; u < 4; u++) old[u] = dst[u] ? *dst[u] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (dst[u]) *dst[u] = old[u] + val[u];
      }
    }
    off += nd;
  }
}

// ------------------------------------------------------------------ panel

// Symmetric interchange of rows/columns a < b: the front in global memory
// (all CTAs of the cluster share the element range), the panel rows held in
// shared memory (exchanged by the owner of row a through DSMEM), and the
// front-variable / original-position lists. The caller barriers afterwards.
template <int CL>
__device__ void cluster_swap(cg::cluster_group& cl, int rank, double* F, int f, int* fv,
                             int* orig, int a, int b, int R, int NBP, int kw, double* Lp,
                             double* Wp, double* wc0, double* wc1) {
  const int n1 = a;
  const int n2 = b - a - 1;
  const int n3 = f - b - 1;
  const int total = n1 + 1 + n2 + n3;
  for (int t = rank * blockDim.x + threadIdx.x; t < total; t += CL * blockDim.x) {
    double *p, *q;
    if (t < n1) {
      p = &F[a + (size_t)f * t];
      q = &F[b + (size_t)f * t];
    } else if (t == n1) {
      p = &F[a + (size_t)f * a];
      q = &F[b + (size_t)f * b];
    } else if (t < n1 + 1 + n2) {
      const int j = a + 1 + (t - n1 - 1);
      p = &F[j + (size_t)f * a];
      q = &F[b + (size_t)f * j];
    } else {
      const int j = b + 1 + (t - n1 - 1 - n2);
      p = &F[j + (size_t)f * a];
      q = &F[j + (size_t)f * b];
    }
    const double tmp = *p;
    *p = *q;
    *q = tmp;
  }
  const int oa = a / R;
  const int ob = b / R;
  if (rank == oa) {
    double* La = Lp + (size_t)(a - oa * R) * NBP;
    double* Wa = Wp + (size_t)(a - oa * R) * NBP;
    double* Lb = cl.map_shared_rank(Lp, ob) + (size_t)(b - ob * R) * NBP;
    double* Wb = cl.map_shared_rank(Wp, ob) + (size_t)(b - ob * R) * NBP;
    for (int j = threadIdx.x; j < kw; j += blockDim.x) {
      double t = La[j];
      La[j] = Lb[j];
      Lb[j] = t;
      t = Wa[j];
      Wa[j] = Wb[j];
      Wb[j] = t;
    }
    if (threadIdx.x == 32) {
      double* x0 = cl.map_shared_rank(wc0, ob) + (b - ob * R);
      double* x1 = cl.map_shared_rank(wc1, ob) + (b - ob * R);
      double t = wc0[a - oa * R];
      wc0[a - oa * R] = *x0;
      *x0 = t;
      t = wc1[a - oa * R];
      wc1[a - oa * R] = *x1;
      *x1 = t;
    }
  }
  if (rank == 0 && threadIdx.x == 64) {
    int t = fv[a];
    fv[a] = fv[b];
    fv[b] = t;
    t = orig[a];
    orig[a] = orig[b];
    orig[b] = t;
  }
}

enum : int { kDelay = 0, kOne = 1, kTwo = 2, kNeedRow = 3, kZero = 4 };

// Partials are pushed: every CTA stores its partial into slot[rank] of every
// CTA of the cluster (lanes of warp 0 in parallel), then one cluster barrier,
// then every thread reduces its own CTA's slots. All CTAs reduce the same
// values in the same order, so every thread of the cluster reaches the same
// pivot decision and the same sequence of barriers.
template <int CL>
__device__ __forceinline__ void push_part(cg::cluster_group& cl, Part* slots, int rank,
                                          const Part& p) {
  if (threadIdx.x < CL) *cl.map_shared_rank(slots + rank, (unsigned)threadIdx.x) = p;
}

// One panel per launch for every front of the large class (the list
// `list`); the trailing update follows in big_update_kernel.
template <int CL>
__global__ void __launch_bounds__(kPanelThreads)
    big_panel_kernel(DevState s, FactorParams prm, int NB, const int* __restrict__ list) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  BigFront* B = s.big + list[blockIdx.x / CL];
  extern __shared__ __align__(16) double sm[];
  __shared__ Part slotA[CL], slotB[CL];
  __shared__ BlockRed red;
  __shared__ double wk[kBigPanelMax], wi[kBigPanelMax];

  const int tid = threadIdx.x;
  if (B->state != 0) return;  // same value in every CTA of the cluster
  const int f = B->f;
  const bool root = (B->nc == 0);
  int k = B->k;
  int ncand = B->ncand;
  const int NBP = NB + 1;  // odd row stride: conflict-free column access
  const int R = (f + CL - 1) / CL;
  const int r0 = rank * R;
  const int r1 = min(f, r0 + R);
  double* Lp = sm;
  double* Wp = Lp + (size_t)R * NBP;
  double* wc0 = Wp + (size_t)R * NBP;
  double* wc1 = wc0 + R;
  double* F = s.dpool + B->doff;
  double* Wg = s.dpool + B->woff;
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;
  const double alpha_bk = (1.0 + 4.1231056256176605) / 8.0;  // (1 + sqrt(17)) / 8
  int kstart = k;
  int kw = 0;
  int npos = 0, nneg = 0;
  double flops = 0.0;

  {  // one panel
  kstart = k;
  kw = 0;
  while (kw < NB - 1 && k < ncand) {
    const int ok = k / R;
    if (tid < kw) wk[tid] = cl.map_shared_rank(Wp, ok)[(size_t)(k - ok * R) * NBP + tid];
    __syncthreads();
    // candidate column k on this CTA's rows: F(:,k) - Lp W(k,:)^T
    double bv = -1.0, cm = 0.0;
    int bi = INT_MAX;
    const int lo = max(r0, k);
    for (int i = lo + tid; i < r1; i += blockDim.x) {
      double v = F[i + (size_t)f * k];
      const double* lr = Lp + (size_t)(i - r0) * NBP;
      for (int j = 0; j < kw; j++) v = fma(-lr[j], wk[j], v);
      wc0[i - r0] = v;
      const double a = fabs(v);
      if (i > k) {
        if (i < ncand)
          keep_larger(bv, bi, a, i);
        else
          cm = fmax(cm, a);
      }
    }
    block_reduce(red, bv, bi, cm);
    {
      Part P;
      P.v = bv;
      P.i = bi;
      P.pad = 0;
      P.m = cm;
      P.x = (k >= r0 && k < r1) ? wc0[k - r0] : 0.0;
      P.y = 0.0;
      push_part<CL>(cl, slotA, rank, P);
    }
    cl.sync();  // B1: column partials visible

    double gv = -1.0, gm = 0.0;
    int gi = INT_MAX;
#pragma unroll
    for (int r = 0; r < CL; r++) {
      keep_larger(gv, gi, slotA[r].v, slotA[r].i);
      gm = fmax(gm, slotA[r].m);
    }
    const double wkk = slotA[ok].x;
    const bool has = (k + 1 < ncand);
    const double abswkk = fabs(wkk);
    const double abswik = has ? gv : 0.0;
    const int imax = has ? (gi < ncand ? gi : k + 1) : k;
    const double colmax = fmax(abswik, gm);
    int step;
    int kpiv = k;
    if (prm.cholesky) {
      step = kOne;
    } else if (root) {
      if (fmax(abswkk, colmax) == 0.0)
        step = kZero;
      else if (abswkk >= alpha_bk * colmax)
        step = kOne;
      else
        step = kNeedRow;
    } else if (abswkk >= prm.pivot_tol && abswkk >= prm.ustab * colmax) {
      step = kOne;
    } else {
      step = has ? kNeedRow : kDelay;
    }
    double wii = 0.0, wik = 0.0;
    if (step == kNeedRow) {
      const int oi = imax / R;
      if (tid < kw) wi[tid] = cl.map_shared_rank(Wp, oi)[(size_t)(imax - oi * R) * NBP + tid];
      __syncthreads();
      double rm = 0.0, dummy = -1.0;
      int di = INT_MAX;
      for (int i = lo + tid; i < r1; i += blockDim.x) {
        double v = (i < imax) ? F[imax + (size_t)f * i] : F[i + (size_t)f * imax];
        const double* lr = Lp + (size_t)(i - r0) * NBP;
        for (int j = 0; j < kw; j++) v = fma(-lr[j], wi[j], v);
        wc1[i - r0] = v;
        if (i != imax) rm = fmax(rm, fabs(v));
      }
      block_reduce(red, dummy, di, rm);
      {
        Part P;
        const bool own = (imax >= r0 && imax < r1);
        P.v = 0.0;
        P.i = 0;
        P.pad = 0;
        P.m = rm;
        P.x = own ? wc1[imax - r0] : 0.0;
        P.y = own ? wc0[imax - r0] : 0.0;
        push_part<CL>(cl, slotB, rank, P);
      }
      cl.sync();  // B2: row partials visible
      double rmax = 0.0;
#pragma unroll
      for (int r = 0; r < CL; r++) rmax = fmax(rmax, slotB[r].m);
      wii = slotB[oi].x;
      wik = slotB[oi].y;
      const double abswii = fabs(wii);
      if (root) {
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

    if (step == kDelay) {
      if (k < ncand - 1)
        cluster_swap<CL>(cl, rank, F, f, fv, orig, k, ncand - 1, R, NBP, kw, Lp, Wp, wc0,
                         wc1);
      ncand -= 1;
      cl.sync();  // B3: swap visible
      continue;
    }
    const int nstep = (step == kTwo) ? 2 : 1;
    const int ksrc = k + nstep - 1;
    // the pivot columns: 1x1 at k -> wc0; 1x1 at imax -> wc1; 2x2 -> wc0, wc1
    const bool use1 = (step != kTwo) && (kpiv != k);
    if (kpiv != ksrc) {
      cluster_swap<CL>(cl, rank, F, f, fv, orig, ksrc, kpiv, R, NBP, kw, Lp, Wp, wc0, wc1);
      cl.sync();  // B3
    }
    const double* colA = use1 ? wc1 : wc0;
    if (nstep == 1) {
      // pivot value known from the reduced partials: wkk (at k) or wii (at imax)
      const double d = use1 ? wii : wkk;
      const bool zero = (step == kZero) || (root && d == 0.0);
      const double dinv = zero ? 0.0 : 1.0 / d;
      for (int i = lo + tid; i < r1; i += blockDim.x) {
        const double w = colA[i - r0];
        double* lr = Lp + (size_t)(i - r0) * NBP;
        double* wr = Wp + (size_t)(i - r0) * NBP;
        if (i == k) {
          lr[kw] = d;
          wr[kw] = d;
          F[k + (size_t)f * k] = d;
        } else {
          const double l = w * dinv;
          lr[kw] = l;
          wr[kw] = w;
          F[i + (size_t)f * k] = l;
        }
      }
      if (rank == 0 && tid == 0) {
        if (d >= 0.0)
          npos++;
        else
          nneg++;
        flops += 2.0 * (double)(f - k) * (kw + 1);
      }
    } else {
      // 2x2 at (k, k+1) after moving imax to k+1: D = [wkk wik; wik wii]
      const double d11 = wkk, d21 = wik, d22 = wii;
      const double det = d11 * d22 - d21 * d21;
      const double detinv = 1.0 / det;
      const double i00 = d22 * detinv, i01 = -d21 * detinv, i11 = d11 * detinv;
      for (int i = lo + tid; i < r1; i += blockDim.x) {
        double* lr = Lp + (size_t)(i - r0) * NBP;
        double* wr = Wp + (size_t)(i - r0) * NBP;
        const double a = wc0[i - r0];
        const double b = wc1[i - r0];
        if (i == k) {
          lr[kw] = d11;
          lr[kw + 1] = 0.0;
          wr[kw] = a;
          wr[kw + 1] = b;
          F[k + (size_t)f * k] = d11;
        } else if (i == k + 1) {
          lr[kw] = d21;
          lr[kw + 1] = d22;
          wr[kw] = a;
          wr[kw + 1] = b;
          F[k + 1 + (size_t)f * k] = d21;
          F[k + 1 + (size_t)f * (k + 1)] = d22;
        } else {
          const double l0 = a * i00 + b * i01;
          const double l1 = a * i01 + b * i11;
          lr[kw] = l0;
          lr[kw + 1] = l1;
          wr[kw] = a;
          wr[kw + 1] = b;
          F[i + (size_t)f * k] = l0;
          F[i + (size_t)f * (k + 1)] = l1;
        }
      }
      if (rank == 0 && tid == 0) {
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
        flops += 4.0 * (double)(f - k) * (kw + 2);
      }
    }
    k += nstep;
    kw += nstep;
    cl.sync();  // B4: new panel columns visible
  }

  {
    // W columns of the panel for the trailing update (rows >= k)
    for (int j = 0; j < kw; j++) {
      const int lo2 = max(r0, k);
      for (int i = lo2 + tid; i < r1; i += blockDim.x)
        Wg[(size_t)j * f + i] = Wp[(size_t)(i - r0) * NBP + j];
    }
  }
  }  // one panel
  if (rank == 0 && tid == 0) {
    B->k = k;
    B->ncand = ncand;
    B->kstart = kstart;
    B->kw = kw;
    B->npos += npos;
    B->nneg += nneg;
    B->flops += flops;
    atomicAdd(s.flops + 1, flops);
    if (k >= ncand) B->state = 1;
  }
}

// --------------------------------------------------------- trailing update

// One launch per panel for all class-5 fronts of the level (list5, nl of
// them): lower-triangular 64x64 tiles of each front's trailing matrix in one
// tile space; every CTA forms the prefix of tile counts itself. The last CTA
// to finish closes the panel (work counters, kw = 0, finished fronts done).
__global__ void __launch_bounds__(kUpdThreads, 2)
    big_update_kernel(DevState s, const int* __restrict__ list5, int nl) {
  __shared__ double As[kBigPanelMax][kTile];
  __shared__ double Bs[kBigPanelMax][kTile];
  __shared__ long long tptr[kUpdMaxFronts + 1];
  __shared__ long long wsum[kUpdThreads / 32];
  __shared__ int last;
  const int tid = threadIdx.x;
  {
    // tile counts of the fronts (kUpdMaxFronts / kUpdThreads per thread,
    // contiguous), then an exclusive scan over the CTA
    constexpr int per = kUpdMaxFronts / kUpdThreads;
    long long cnt[per];
    long long mine = 0;
#pragma unroll
    for (int u = 0; u < per; u++) {
      const int i = tid * per + u;
      cnt[u] = 0;
      if (i < nl) {
        const BigFront& B = s.big[list5[i]];
        if (B.state != 2 && B.kw > 0) {
          const long long t = (B.f - B.k + kTile - 1) / kTile;
          cnt[u] = t * (t + 1) / 2;
        }
      }
      mine += cnt[u];
    }
    const int lane = tid & 31;
    const int w = tid >> 5;
    long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    long long base = 0;
    for (int q = 0; q < w; q++) base += wsum[q];
    long long run = base + incl - mine;
    if (tid == 0) tptr[0] = 0;
#pragma unroll
    for (int u = 0; u < per; u++) {
      run += cnt[u];
      const int i = tid * per + u;
      if (i < nl) tptr[i + 1] = run;
    }
  }
  __syncthreads();
  const long long total = tptr[nl];
  const int tx = tid & 15;
  const int ty = tid >> 4;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    // the front: last fi with tptr[fi] <= t
    int lo = 0, hi = nl;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (tptr[mid] <= t)
        lo = mid;
      else
        hi = mid;
    }
    const BigFront& B = s.big[list5[lo]];
    const long long lt = t - tptr[lo];
    int I = (int)((sqrt(8.0 * (double)lt + 1.0) - 1.0) * 0.5);
    while ((long long)(I + 1) * (I + 2) / 2 <= lt) I++;
    while ((long long)I * (I + 1) / 2 > lt) I--;
    const int J = (int)(lt - (long long)I * (I + 1) / 2);
    const int f = B.f;
    const int k = B.k;
    const int kw = B.kw;
    const int ks = B.kstart;
    const double* F0 = s.dpool + B.doff;
    double* F = s.dpool + B.doff;
    const double* W = s.dpool + B.woff;
    const int i0 = k + I * kTile;
    const int j0 = k + J * kTile;
    // this thread's 4x4 entries of the trailing tile, loaded first so that
    // their latency overlaps the panel loads and the products
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
    __syncthreads();
    {
      // the panel's rows of L and W for this tile: every load of the thread
      // is issued before the first shared-memory store, so that the tile
      // waits on HBM once rather than once per column
      constexpr int kPer = kBigPanelMax * kTile / kUpdThreads;
      static_assert(kPer * kUpdThreads == kBigPanelMax * kTile, "panel split");
      double pa[kPer], pb[kPer];
#pragma unroll
      for (int u = 0; u < kPer; u++) {
        const int q = tid + kUpdThreads * u;
        const int c = q / kTile;
        const int r = q - c * kTile;
        pa[u] = 0.0;
        pb[u] = 0.0;
        if (c < kw) {
          if (i0 + r < f) pa[u] = F0[i0 + r + (size_t)f * (ks + c)];
          if (j0 + r < f) pb[u] = W[(size_t)c * f + j0 + r];
        }
      }
#pragma unroll
      for (int u = 0; u < kPer; u++) {
        const int q = tid + kUpdThreads * u;
        const int c = q / kTile;
        const int r = q - c * kTile;
        if (c < kw) {
          As[c][r] = pa[u];
          Bs[c][r] = pb[u];
        }
      }
    }
    __syncthreads();
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
    for (int c = 0; c < kw; c++) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; a++) av[a] = As[c][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; b++) bv[b] = Bs[c][ty + 16 * b];
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
  }
  // close the panel once every CTA is done with the fronts' fields
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(reinterpret_cast<unsigned*>(s.err + 2), 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int i = tid; i < nl; i += blockDim.x) {
    BigFront& B = s.big[list5[i]];
    if (B.state == 2) continue;
    if (B.kw > 0) {
      const double r = (double)(B.f - B.k);
      const double fl = r * (r + 1.0) * B.kw;
      B.flops += fl;
      atomicAdd(s.flops + 2, fl);
      // trailing lower triangle read and written, panel L and W rows read
      atomicAdd(s.flops + 3, 8.0 * (r * (r + 1.0) + 2.0 * r * B.kw));
    }
    B.kw = 0;
    if (B.state == 1) B.state = 2;
  }
  if (tid == 0) s.err[2] = 0;
}

__global__ void big_finalize_kernel(DevState s, int nbig, int cholesky) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbig) return;
  const BigFront& B = s.big[i];
  const int node = B.node;
  const int npiv = B.k;
  const int m = B.f - npiv;
  s.f[node] = B.f;
  s.fs[node] = B.fs;
  s.npiv[node] = npiv;
  s.ndel[node] = B.fs - npiv;
  s.fv_off[node] = B.ioff;
  s.L_off[node] = B.doff;
  s.L_ld[node] = B.f;
  if (B.pad == 1) {  // factored on chip: contribution block after L, ld m
    s.cb_off[node] = B.doff + (long long)B.f * npiv;
    s.cb_ld[node] = m > 0 ? m : 1;
  } else {  // factored in place in the pool
    s.cb_off[node] = B.doff + (long long)npiv * (B.f + 1);
    s.cb_ld[node] = B.f;
  }
  s.u_off[node] = (long long)atomicAdd(s.used + 2, (unsigned long long)m);
  if (!cholesky) {
    atomicAdd(s.inertia, B.npos);
    atomicAdd(s.inertia + 1, B.nneg);
  }
  atomicAdd(s.flops, B.flops);
}

template <int CL>
cudaError_t launch_panel(const DevState& s, const FactorParams& prm, int count, int NB,
                         size_t smem, const int* list, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(count * CL, 1, 1);
  cfg.blockDim = dim3(kPanelThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, big_panel_kernel<CL>, s, prm, NB, list);
}

constexpr size_t kPanelSmemMax = 224 * 1024;

template <int CL>
cudaError_t launch_assemble_cl(const DevPlan& p, const DevState& s, const int* list, int nl,
                               const double* vals, const double* diag, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nl * CL), 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = CL > 1 ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, big_assemble_kernel<CL>, p, s, vals, diag, list);
}

// One launch for the level's fronts in `list`: a CTA per front when they
// fill the GPU, otherwise a cluster of 4 or 16 CTAs per front.
cudaError_t assemble_big(const DevPlan& p, const DevState& s, const int* list, int nl,
                         int max_f, const double* vals, const double* diag, cudaStream_t stream,
                         Prof& prof) {
  if (nl <= 0) return cudaSuccess;
  prof.begin(stream);
  big_zero_kernel<<<dim3(nl, std::max(1, std::min(256, (max_f + 7) / 8))), 256, 0, stream>>>(s,
                                                                                        list);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (nl >= 148)
    e = launch_assemble_cl<1>(p, s, list, nl, vals, diag, stream);
  else if (nl >= 37)
    e = launch_assemble_cl<4>(p, s, list, nl, vals, diag, stream);
  else
    e = launch_assemble_cl<16>(p, s, list, nl, vals, diag, stream);
  prof.end(kPhBigAsm, stream, 2);
  return e;
}

// Panels and trailing updates of the fronts in `list` from their current
// position (B.k), at most `max_left` candidates left per front: a chained
// panel per launch where the front fits the chained kernel, else the
// per-pivot panel kernel.
cudaError_t run_big_panels(const DevState& s, const FactorParams& prm, const int* list, int count,
                           int max_f, int max_left, cudaStream_t stream, Prof& prof) {
  const int CL = max_f > 1600 ? 16 : 8;
  const int R = (max_f + CL - 1) / CL;
  int NB = kBigPanelMax;
  while (NB > 4 && (size_t)R * (2 * (NB + 1) + 2) * sizeof(double) > kPanelSmemMax) NB >>= 1;
  const size_t smem = (size_t)R * (2 * (NB + 1) + 2) * sizeof(double);
  const int upd_grid = 148 * 4;
  const int cnb = big_chain_panel_width(max_f);
  const bool chained = cnb > 0;
  const int nsteps = chained ? (max_left + cnb - 2) / (cnb - 1) + 1
                             : (max_left + (NB - 2)) / (NB - 1) + 1;
  for (int st = 0; st < nsteps; st++) {
    cudaError_t e;
    prof.begin(stream);
    if (chained)
      e = launch_big_chain_panel(s, prm, count, max_f, cnb, list, stream);
    else if (CL == 16)
      e = launch_panel<16>(s, prm, count, NB, smem, list, stream);
    else
      e = launch_panel<8>(s, prm, count, NB, smem, list, stream);
    if (e != cudaSuccess) return e;
    prof.end(kPhBigPanel, stream, 1);
    prof.begin(stream);
    for (int c0 = 0; c0 < count; c0 += kUpdMaxFronts) {
      const int nl = std::min(kUpdMaxFronts, count - c0);
      big_update_kernel<<<upd_grid, kUpdThreads, 0, stream>>>(s, list + c0, nl);
    }
    prof.end(kPhBigUpd, stream, (count + kUpdMaxFronts - 1) / kUpdMaxFronts);
  }
  return cudaGetLastError();
}

// Class-6 fronts: blocked panels with a-posteriori tests (big_app.cu), all
// of the level's panel steps in one cooperative launch. Roots among them
// whose panels left candidates (failed tests cannot be delayed past a root)
// finish with the chained panels, Bunch-Kaufman as for every root.
cudaError_t app_level(const DevPlan& p, const DevState& s, const BigLevelInfo& info,
                      const FactorParams& prm, const double* vals,
                      const double* diag, cudaStream_t stream, Prof& prof) {
  const int nl = info.count_app;
  const int* list6 = s.class_list + (size_t)6 * p.num_nodes;
  cudaError_t e = assemble_big(p, s, list6, nl, info.max_f_app, vals, diag, stream, prof);
  if (e != cudaSuccess) return e;
  prof.begin(stream);
  int* list7 = s.class_list + (size_t)7 * p.num_nodes;
  e = launch_app_level(s, prm, nl, info.max_fs_app, list6, list7, s.big_meta, stream);
  if (e != cudaSuccess) return e;
  prof.end(kPhBigPanel, stream, 1);
  int meta[5] = {0, 0, 0, 0, 0};  // big_meta[19..23]
  e = cudaMemcpyAsync(meta, s.big_meta + 19, sizeof(meta), cudaMemcpyDeviceToHost, stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return e;
  if (meta[4]) return cudaErrorUnknown;  // the step cap or a tensor-core timeout
  if (meta[0] > 0) return run_big_panels(s, prm, list7, meta[0], info.max_f_app, meta[1], stream, prof);
  return cudaSuccess;
}

}  // namespace

cudaError_t configure_big_kernels() {
  cudaError_t e;
  e = cudaFuncSetAttribute(big_panel_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kPanelSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(big_panel_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kPanelSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(big_panel_kernel<16>,
                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(big_assemble_kernel<16>,
                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  e = configure_big_chain_kernel();
  if (e != cudaSuccess) return e;
  return configure_cluster_front_kernels();
}

cudaError_t launch_big_level(const DevPlan& p, const DevState& s, const BigLevelInfo& info,
                             const FactorParams& prm, const double* vals,
                             const double* diag, cudaStream_t stream, Prof& prof) {
  const int nb = info.count;
  if (nb <= 0) return cudaSuccess;
  prof.begin(stream);

  // fronts that fit in a cluster's distributed shared memory
  {
    cudaError_t e = launch_cluster_fronts(p, s, info.class_count, info.class_maxf, vals, diag,
                                          prm, stream, p.num_nodes);
    if (e != cudaSuccess) return e;
  }
  prof.end(kPhCluster, stream, info.cluster_launches);
  if (info.count_app > 0) {
    cudaError_t e = app_level(p, s, info, prm, vals, diag, stream, prof);
    if (e != cudaSuccess) return e;
  }
  if (info.count_large == 0) {
    prof.begin(stream);
    big_finalize_kernel<<<(nb + 255) / 256, 256, 0, stream>>>(s, nb, prm.cholesky);
    prof.end(kPhBigAsm, stream, 1);
    return cudaGetLastError();
  }
  // larger fronts: a cluster per front, one panel per launch over the front
  // in global memory
  const int* list5 = s.class_list + (size_t)5 * p.num_nodes;
  {
    cudaError_t e =
        assemble_big(p, s, list5, info.count_large, info.max_f_large, vals, diag, stream, prof);
    if (e != cudaSuccess) return e;
    e = run_big_panels(s, prm, list5, info.count_large, info.max_f_large, info.max_fs_large,
                       stream, prof);
    if (e != cudaSuccess) return e;
  }
  prof.begin(stream);
  big_finalize_kernel<<<(nb + 255) / 256, 256, 0, stream>>>(s, nb, prm.cholesky);
  prof.end(kPhBigAsm, stream, 1);
  return cudaGetLastError();
}

}  // namespace b200ldl
