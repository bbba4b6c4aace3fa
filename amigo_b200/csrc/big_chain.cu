// Big fronts (too large for one cluster's shared memory), one panel per
// launch with the chained pivot search.
//
// The front F (f x f, column-major, lower triangle) stays in HBM in logical
// order at panel boundaries. A cluster of 16 CTAs owns one front: CTA r
// holds the rows [k0 + r R, k0 + r R + R) of the panel's L in shared memory
// (k0 the panel's first pivot, R = (f - k0) / 16 rounded up), and the
// panel's W columns go to HBM by physical row. Inside the panel the logical
// order (the reference's symm_swap, SparseLDL::factor_front_matrix_block,
// include/sparse_ldl.h:1316-1553) is a permutation in shared memory, so a
// delay or a pivot interchange moves no data; candidate columns are formed
// as F(:,c) - Lp W(c,:)^T (sparse_ldl.h:1337-1344) from the untouched F.
// Each step evaluates a chain of up to 8 candidates (one per warp) with the
// decisions of front_common.cuh. At the end of the panel the permutation is
// applied to the rows and columns of F that moved (gathered into a scratch
// buffer, then scattered back), the panel's L is written into its logical
// columns and the W columns in logical order for the tiled trailing update
// (big_update_kernel).
#include <cooperative_groups.h>

#include <climits>

#include "front_common.cuh"
#include "ldl_internal.h"

namespace cg = cooperative_groups;

namespace b200ldl {

namespace {

using namespace chain;

constexpr int kBcCL = 16;
constexpr int kBcThreads = 256;
constexpr int kBcWarps = kBcThreads / 32;
static_assert(kChain == kBcWarps, "one chain member per warp");

// panel width NB: 32 where the panel state fits, 16 for the largest fronts
template <int NB>
struct BcShared {
  ChainXchg<kBcCL, 2> x;
  int piv[NB];  // physical rows of the panel's pivots
  int scan[kBcWarps];
  double Wm[kChain][NB + 1];           // W(pc_m, :) of the columns being formed
  int pcs[kChain];                     // their physical columns
  ColStat red[kBcWarps][kChain];       // per-warp column statistics
  double red2[kBcWarps][kChain];       // per-warp imax-column maxima
};

// Shared-memory layout (bytes): the panel's L for own rows [R][NB + 1]
// doubles (odd row stride), the chain's columns over own rows
// [2][2][kChain][R] doubles, then perm and ipos [f] as 16-bit indices and
// the moved positions [f].
template <int NB>
__host__ __device__ __forceinline__ size_t bc_smem(int f) {
  const size_t R = (size_t)(f + kBcCL - 1) / kBcCL;
  return R * (NB + 1) * 8 + (size_t)4 * kChain * R * 8 + (size_t)3 * f * 2 + 16;
}

template <typename T>
__device__ __forceinline__ T* at_rank(cg::cluster_group& cl, T* ptr, int r, int rank) {
  return (r == rank) ? ptr : cl.map_shared_rank(ptr, (unsigned)r);
}

// F(a, b) of the symmetric front from its lower triangle
__device__ __forceinline__ double fsym(const double* F, int f, int a, int b) {
  return (a >= b) ? F[a + (size_t)f * b] : F[b + (size_t)f * a];
}

// d(8x8) += a(8x4) b(4x8) on the FP64 tensor cores. Fragments: lane l
// holds a(l / 4, l % 4), b(l % 4, l / 4) and d(l / 4, 2 (l % 4) + {0, 1}).
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Columns pc_m (m in mask, up to 8) of the panel's Schur complement on this
// CTA's rows, v(r, m) = F(r, pc_m) - Lp(r, :) W(pc_m, :)^T, by all warps
// together. Rows go in tiles of 8 over the warps. The product of a tile with
// the 8 columns is one 8x8 FP64 tensor-core tile per 4 panel columns, so
// Lp is read once for all the columns. The F entries of a whole sweep of
// tiles are loaded before the products, so that their latencies overlap.
// Chunk x of the panel columns holds columns 16 (x / 4) + (x % 4) + 4 j,
// j = 0..3. With the odd row stride of Lp, the 8x4 A fragment then falls
// on distinct banks. Columns at and beyond the panel's width are zero in
// Lp and in Wm; chunks entirely beyond it are skipped (exact). emit(m, q,
// pos, pc, v) is called for every own row q with position pos >= k.
constexpr int kSweepTiles = 8;
template <int NB, typename Emit>
__device__ __forceinline__ void panel_columns(const double* F, int f, const double* Lp,
                                              const double* Wm, const int* pcs, unsigned mask,
                                              const unsigned short* ipos, int r0, int Q, int k,
                                              int kwn, int warp, int lane, Emit emit) {
  constexpr int kNBP = NB + 1;
  constexpr int kChunks = NB / 4;
  const int g = lane >> 2;
  const int tig = lane & 3;
  const int m0 = 2 * tig;
  const int m1 = m0 + 1;
  const bool h0 = (mask >> m0) & 1u;
  const bool h1 = (mask >> m1) & 1u;
  const int pc0 = h0 ? pcs[m0] : 0;
  const int pc1 = h1 ? pcs[m1] : 0;
  double bf[kChunks];
#pragma unroll
  for (int x = 0; x < kChunks; x++) bf[x] = Wm[g * kNBP + 16 * (x / 4) + (x % 4) + 4 * tig];
  const int ntiles = (Q + 7) >> 3;
  for (int i0 = warp; i0 < ntiles; i0 += kBcWarps * kSweepTiles) {
    double f0[kSweepTiles], f1[kSweepTiles];
    int pos[kSweepTiles];
#pragma unroll
    for (int u = 0; u < kSweepTiles; u++) {
      const int q = 8 * (i0 + kBcWarps * u) + g;
      pos[u] = -1;
      f0[u] = 0.0;
      f1[u] = 0.0;
      if (q < Q) {
        const int r = r0 + q;
        pos[u] = ipos[r];
        if (pos[u] >= k) {
          if (h0) f0[u] = fsym(F, f, r, pc0);
          if (h1) f1[u] = fsym(F, f, r, pc1);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kSweepTiles; u++) {
      const int tile = i0 + kBcWarps * u;
      if (tile >= ntiles) break;  // the same in every lane
      // rows of the last tile beyond Q read the next shared array (never used)
      const double* arow = Lp + (size_t)(8 * tile + g) * kNBP + 4 * tig;
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int x = 0; x < kChunks; x++) {
        if (16 * (x / 4) >= kwn) break;  // the same in every lane
        dmma(c0, c1, arow[16 * (x / 4) + (x % 4)], bf[x]);
      }
      if (pos[u] >= k) {
        const int q = 8 * tile + g;
        if (h0) emit(m0, q, pos[u], pc0, f0[u] - c0);
        if (h1) emit(m1, q, pos[u], pc1, f1[u] - c1);
      }
      __syncwarp();
    }
  }
}

template <int NB>
__global__ void __launch_bounds__(kBcThreads)
    big_chain_panel_kernel(DevState s, FactorParams prm, const int* __restrict__ list) {
  constexpr int kNB = NB;
  constexpr int kNBP = NB + 1;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  BigFront* B = s.big + list[blockIdx.x / kBcCL];
  extern __shared__ __align__(16) double sm[];
  __shared__ BcShared<NB> sh;
  if (B->state != 0) return;  // the same in every CTA of the cluster

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = B->f;
  const bool root = (B->nc == 0);
  const bool single = root || prm.cholesky;  // no delays: chains of one
  int k = B->k;
  int ncand = B->ncand;
  const int kstart = k;
  // rows before kstart are eliminated, and after the previous panel's
  // permutation pass the remaining ones are exactly [kstart, f): only those
  // are split over the CTAs, so the per-step work shrinks as the front
  // progresses
  const int R = (f - kstart + kBcCL - 1) / kBcCL;
  const int r0 = kstart + rank * R;
  const int Q = max(0, min(f, r0 + R) - r0);
  double* Lp = sm;                               // [R][kNBP]
  double* colbuf = Lp + (size_t)R * kNBP;        // [2][2][kChain][R]
  unsigned short* perm = reinterpret_cast<unsigned short*>(colbuf + (size_t)4 * kChain * R);
  unsigned short* ipos = perm + f;
  unsigned short* mlist = ipos + f;
  double* F = s.dpool + B->doff;
  double* Wg = s.dpool + B->woff;                 // [NB][f] logical, for the trailing update
  double* Wph = Wg + (size_t)kBigPanelMax * f;    // [NB][f] by physical row, inside the panel
  double* T = Wph + (size_t)kBigPanelMax * f;     // permutation scratch [fs + 1][f]
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;

  for (int t = tid; t < R * kNBP; t += kBcThreads) Lp[t] = 0.0;
  for (int t = tid; t < 4 * kChain * R; t += kBcThreads) colbuf[t] = 0.0;
  for (int p = tid; p < f; p += kBcThreads) {
    perm[p] = (unsigned short)p;
    ipos[p] = (unsigned short)p;
  }
  __syncthreads();

  int kw = 0;
  int npos = 0, nneg = 0;
  double flops = 0.0;
  int stepno = 0;
  // the previous step's accepted columns: W(., c) for c >= kw_prev was
  // written to HBM by its owner after the last barrier, so members read it
  // from the owner's column buffers (written before that barrier) instead
  int prev_n = 0;
  const double* prevA = nullptr;
  const double* prevB = nullptr;

  while (kw < kNB - 1 && k < ncand) {
    const int par = stepno & 1;
    stepno++;
    const int nS = single ? 1 : min(kChain, ncand - k);
    double* cb0 = colbuf + (size_t)(par * 2) * kChain * R;
    double* cb1 = cb0 + (size_t)kChain * R;
    const int kw_safe = kw - prev_n;

    // ---- exchange 1: the chain members' columns. Warp t brings member t's
    // W row; then all warps form all members' columns over row tiles.
    if (warp < nS) {
      const int t = warp;
      const int pc = (t == 0) ? perm[k] : perm[ncand - t];
      double wl = 0.0;
      if (lane < kw_safe) {
        wl = __ldcg(Wph + (size_t)lane * f + pc);
      } else if (lane < kw) {
        const int o = (pc - kstart) / R;
        const double* src = (lane == kw_safe) ? prevA : prevB;
        wl = at_rank(cl, src, o, rank)[pc - kstart - o * R];
      }
      if (lane < kNB) sh.Wm[t][lane] = wl;
      if (lane == 0) sh.pcs[t] = pc;
    }
    __syncthreads();
    {
      double bv[2] = {0.0, 0.0}, cm[2] = {0.0, 0.0};
      int bi[2] = {INT_MAX, INT_MAX};
      panel_columns<NB>(F, f, Lp, &sh.Wm[0][0], sh.pcs, (1u << nS) - 1u, ipos, r0, Q, k, kw,
                        warp, lane, [&](int m, int q, int pos, int, double v) {
                          cb0[(size_t)m * R + q] = v;
                          int j = -1;
                          if (pos == k)
                            j = 0;
                          else if (pos > ncand - nS && pos < ncand)
                            j = ncand - pos;
                          if (j >= 0) {
                            for (int d = 0; d < kBcCL; d++)
                              *at_rank(cl, &sh.x.V[par][m][j], d, rank) = v;
                          } else if (pos < ncand) {
                            keep_larger(bv[m & 1], bi[m & 1], fabs(v), pos);
                          } else {
                            cm[m & 1] = fmax(cm[m & 1], fabs(v));
                          }
                        });
      // the 8 lanes with the same lane % 4 hold the same two members
#pragma unroll
      for (int i = 0; i < 2; i++) {
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, bv[i], o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi[i], o);
          keep_larger(bv[i], bi[i], ov, oi);
          cm[i] = fmax(cm[i], __shfl_xor_sync(0xffffffffu, cm[i], o));
        }
      }
      if (lane < 4) {
#pragma unroll
        for (int i = 0; i < 2; i++) {
          ColStat st;
          st.bv = bv[i];
          st.cm = cm[i];
          st.bi = bi[i];
          st.pad = 0;
          sh.red[warp][2 * lane + i] = st;
        }
      }
    }
    __syncthreads();
    if (warp < nS) {
      const int t = warp;
      double bv = 0.0, cm = 0.0;
      int bi = INT_MAX;
      if (lane < kBcWarps) {
        const ColStat st = sh.red[lane][t];
        bv = st.bv;
        cm = st.cm;
        bi = st.bi;
      }
      warp_argmax_max(bv, bi, cm);
      if (lane < kBcCL) {
        ColStat st;
        st.bv = bv;
        st.cm = cm;
        st.bi = bi;
        st.pad = 0;
        *at_rank(cl, &sh.x.s1[par][rank][t], lane, rank) = st;
      }
    }
    cl.sync();  // B1

    if (warp < nS) decide_column<kBcCL, 2>(sh.x, par, warp, lane, nS, k, ncand, root, prm, perm);
    __syncthreads();

    unsigned acc1;
    int d1l;
    const unsigned need2 = need_rows(sh.x.cand, nS, lane, acc1, d1l);
    if (need2) {
      // ---- exchange 2: the imax columns of the members that need them (every
      // W column is in HBM by now), formed like the member columns
      if (need2 & (1u << warp)) {
        const int t = warp;
        const int pc = sh.x.cand[t].imaxp;
        if (lane < kNB) sh.Wm[t][lane] = (lane < kw) ? __ldcg(Wph + (size_t)lane * f + pc) : 0.0;
        if (lane == 0) sh.pcs[t] = pc;
      }
      __syncthreads();
      {
        double rm[2] = {0.0, 0.0};
        panel_columns<NB>(F, f, Lp, &sh.Wm[0][0], sh.pcs, need2, ipos, r0, Q, k, kw, warp, lane,
                          [&](int m, int q, int, int pc, double v) {
                            cb1[(size_t)m * R + q] = v;
                            if (r0 + q == pc) {
                              const double wik = cb0[(size_t)m * R + q];
                              for (int d = 0; d < kBcCL; d++) {
                                double* dst = at_rank(cl, &sh.x.P2[par][m][0], d, rank);
                                dst[0] = v;
                                dst[1] = wik;
                              }
                            } else {
                              rm[m & 1] = fmax(rm[m & 1], fabs(v));
                            }
                          });
#pragma unroll
        for (int i = 0; i < 2; i++) {
#pragma unroll
          for (int o = 4; o < 32; o <<= 1)
            rm[i] = fmax(rm[i], __shfl_xor_sync(0xffffffffu, rm[i], o));
        }
        if (lane < 4) {
          sh.red2[warp][2 * lane] = rm[0];
          sh.red2[warp][2 * lane + 1] = rm[1];
        }
      }
      __syncthreads();
      if (need2 & (1u << warp)) {
        const int t = warp;
        const double rm = warp_max_nonneg((lane < kBcWarps) ? sh.red2[lane][t] : 0.0);
        if (lane < kBcCL) *at_rank(cl, &sh.x.s2[par][rank][t], lane, rank) = rm;
      }
      cl.sync();  // B2
      if (need2 & (1u << warp)) decide_row<kBcCL, 2>(sh.x, par, warp, lane, root, prm);
      __syncthreads();
    }

    int tacc, kind;
    replay(sh.x.cand, nS, lane, acc1, d1l, tacc, kind);
    const int ndelay = tacc;
    const int nstep = (kind == kTwo) ? 2 : 1;
    const int pi = (tacc < nS) ? sh.x.cand[tacc].imaxp : -1;
    if (warp == 0) reorder(sh.x.cand, perm, ipos, lane, nS, ndelay, k, ncand, kind, nstep, pi);
    if (tacc == nS) {
      ncand -= ndelay;
      prev_n = 0;
      __syncthreads();
      continue;
    }
    const Cand& ca = sh.x.cand[tacc];
    const int pk = ca.mrow;
    const double* colA = ((kind == kOneImax) ? cb1 : cb0) + (size_t)tacc * R;
    const double* colB = cb1 + (size_t)tacc * R;
    const int p0 = (kind == kOneImax) ? pi : pk;
    // W columns (HBM, physical rows) and L columns of own rows
    if (nstep == 1) {
      const double d = (kind == kOneImax) ? ca.wii : ca.wkk;
      const double dinv = (kind == kZero || (root && d == 0.0)) ? 0.0 : 1.0 / d;
      for (int q = tid; q < Q; q += kBcThreads) {
        const int r = r0 + q;
        const double a = colA[q];
        Wph[(size_t)kw * f + r] = a;
        Lp[(size_t)q * kNBP + kw] = (r == p0) ? d : a * dinv;
      }
      if (tid == 0) {
        sh.piv[kw] = p0;
        if (rank == 0) {
          if (d >= 0.0)
            npos++;
          else
            nneg++;
          flops += 2.0 * (double)(f - k) * (kw + 1);
        }
      }
    } else {
      const double d11 = ca.wkk, d21 = ca.wik, d22 = ca.wii;
      const double det = d11 * d22 - d21 * d21;
      const double detinv = 1.0 / det;
      const double i00 = d22 * detinv, i01 = -d21 * detinv, i11 = d11 * detinv;
      for (int q = tid; q < Q; q += kBcThreads) {
        const int r = r0 + q;
        const double a = colA[q], b = colB[q];
        Wph[(size_t)kw * f + r] = a;
        Wph[(size_t)(kw + 1) * f + r] = b;
        double* lr = Lp + (size_t)q * kNBP;
        if (r == pk) {
          lr[kw] = d11;
          lr[kw + 1] = 0.0;
        } else if (r == pi) {
          lr[kw] = d21;
          lr[kw + 1] = d22;
        } else {
          lr[kw] = a * i00 + b * i01;
          lr[kw + 1] = a * i01 + b * i11;
        }
      }
      if (tid == 0) {
        sh.piv[kw] = pk;
        sh.piv[kw + 1] = pi;
        if (rank == 0) {
          fv[pk] = -(fv[pk] + 1);
          fv[pi] = -(fv[pi] + 1);
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
    }
    prev_n = nstep;
    prevA = colA;
    prevB = colB;
    ncand -= ndelay;
    k += nstep;
    kw += nstep;
    __syncthreads();  // L, W and the order visible to every warp
  }

  // ---- the positions that moved: F's rows and columns follow them
  {
    const int per = (f - kstart + kBcThreads - 1) / kBcThreads;
    const int a0 = kstart + tid * per;
    const int a1 = min(f, a0 + per);
    int cnt = 0;
    for (int p = a0; p < a1; p++) cnt += (perm[p] != p);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) sh.scan[warp] = incl;
    __syncthreads();
    int base = 0, total = 0;
    for (int w2 = 0; w2 < kBcWarps; w2++) {
      if (w2 < warp) base += sh.scan[w2];
      total += sh.scan[w2];
    }
    int idx = base + incl - cnt;
    for (int p = a0; p < a1; p++)
      if (perm[p] != p) mlist[idx++] = (unsigned short)p;
    __syncthreads();
    const int nm = total;  // the same in every CTA
    if (nm > 0) {
      // gather: T[m][x] = F(perm[p_m], x), 256-column chunks over the cluster
      const int nch = (f + kBcThreads - 1) / kBcThreads;
      for (int c = rank; c < nm * nch; c += kBcCL) {
        const int m = c / nch;
        const int x = (c - m * nch) * kBcThreads + tid;
        if (x < f) T[(size_t)m * f + x] = fsym(F, f, perm[mlist[m]], x);
      }
      cl.sync();
      // scatter: F(p_m, b) = old F(perm[p_m], perm[b]) = T[m][perm[b]]
      for (int c = rank; c < nm * nch; c += kBcCL) {
        const int m = c / nch;
        const int b = (c - m * nch) * kBcThreads + tid;
        if (b < f) {
          const int p = mlist[m];
          const double v = __ldcg(T + (size_t)m * f + perm[b]);
          if (b >= p)
            F[b + (size_t)f * p] = v;
          else
            F[p + (size_t)f * b] = v;
        }
      }
    }
    cl.sync();
  }

  // ---- the panel's L (and D) into its logical columns; W in logical order
  // for the trailing update
  for (int c = 0; c < kw; c++) {
    for (int q = tid; q < Q; q += kBcThreads) {
      const int r = r0 + q;
      const int pos = ipos[r];
      if (pos >= kstart + c) F[pos + (size_t)f * (kstart + c)] = Lp[(size_t)q * kNBP + c];
      if (pos >= k) Wg[(size_t)c * f + pos] = Wph[(size_t)c * f + r];
    }
  }
  if (rank == 0) {
    // the variables in logical order (T is free now)
    int* tv = reinterpret_cast<int*>(T);
    for (int p = kstart + tid; p < f; p += kBcThreads) {
      tv[p] = fv[perm[p]];
      tv[f + p] = orig[perm[p]];
    }
    __syncthreads();
    for (int p = kstart + tid; p < f; p += kBcThreads) {
      fv[p] = tv[p];
      orig[p] = tv[f + p];
    }
  }
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
  cl.sync();
}

template <int NB>
bool fits(int f) {
  return f <= 65535 && bc_smem<NB>(f) + sizeof(BcShared<NB>) + 1024 <= 232448;
}

template <int NB>
cudaError_t configure_nb() {
  cudaError_t e = cudaFuncSetAttribute(big_chain_panel_kernel<NB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(232448 - sizeof(BcShared<NB>) - 1024));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(big_chain_panel_kernel<NB>,
                              cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

template <int NB>
cudaError_t launch_nb(const DevState& s, const FactorParams& prm, int count, int max_f,
                      const int* list, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(count * kBcCL, 1, 1);
  cfg.blockDim = dim3(kBcThreads, 1, 1);
  cfg.dynamicSmemBytes = bc_smem<NB>(max_f);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kBcCL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, big_chain_panel_kernel<NB>, s, prm, list);
}

}  // namespace

int big_chain_panel_width(int f) {
  if (fits<32>(f)) return 32;
  if (fits<16>(f)) return 16;
  return 0;
}

cudaError_t configure_big_chain_kernel() {
  cudaError_t e = configure_nb<16>();
  if (e != cudaSuccess) return e;
  return configure_nb<32>();
}

cudaError_t launch_big_chain_panel(const DevState& s, const FactorParams& prm, int count,
                                   int max_f, int nb, const int* list, cudaStream_t stream) {
  return nb == 32 ? launch_nb<32>(s, prm, count, max_f, list, stream)
                  : launch_nb<16>(s, prm, count, max_f, list, stream);
}

}  // namespace b200ldl
