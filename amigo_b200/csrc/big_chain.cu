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

// Column pc of the panel's Schur complement on this CTA's rows, by one
// warp; w holds W(pc, :) (zero beyond the panel's width). kRowsPerLane rows
// per lane pass so that their HBM loads are in flight together (more rows
// in flight measured slower: the strided loads of the row part queue up).
constexpr int kRowsPerLane = 4;
template <int NB, typename Use>
__device__ __forceinline__ void big_member_column(const double* F, int f, const double* Lp,
                                                  const unsigned short* ipos, int r0, int Q,
                                                  int pc, int k, int kwn, int lane,
                                                  const double* w, double* out, Use use) {
  constexpr int kNB = NB;
  constexpr int kNBP = NB + 1;
  for (int qb = lane; qb < Q; qb += 32 * kRowsPerLane) {
    double fv4[kRowsPerLane];
    int pos4[kRowsPerLane];
#pragma unroll
    for (int u = 0; u < kRowsPerLane; u++) {
      const int q = qb + 32 * u;
      pos4[u] = -1;
      fv4[u] = 0.0;
      if (q < Q) {
        const int r = r0 + q;
        pos4[u] = ipos[r];
        if (pos4[u] >= k) fv4[u] = fsym(F, f, r, pc);
      }
    }
#pragma unroll
    for (int u = 0; u < kRowsPerLane; u++) {
      if (pos4[u] < k) continue;
      const int q = qb + 32 * u;
      const double* lr = Lp + (size_t)q * kNBP;
      double a0 = 0.0, a1 = 0.0;
      // columns at and beyond the panel's width are zero: skip them in
      // groups of 8 (exact, the skipped products are zeros)
#pragma unroll
      for (int c8 = 0; c8 < kNB; c8 += 8) {
        if (c8 >= kwn) break;
#pragma unroll
        for (int c = c8; c < c8 + 8; c += 2) {
          a0 = fma(lr[c], w[c], a0);
          a1 = fma(lr[c + 1], w[c + 1], a1);
        }
      }
      const double v = fv4[u] - (a0 + a1);
      out[q] = v;
      use(q, r0 + q, pos4[u], v);
    }
  }
  __syncwarp();
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

    // ---- exchange 1: warp t forms the column of chain member t
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
      double w[kNB];
#pragma unroll
      for (int c = 0; c < kNB; c++) w[c] = __shfl_sync(0xffffffffu, wl, c);
      double bv = 0.0, cm = 0.0;
      int bi = INT_MAX;
      double* out = cb0 + (size_t)t * R;
      big_member_column<NB>(F, f, Lp, ipos, r0, Q, pc, k, kw, lane, w, out,
                        [&](int q, int r, int pos, double v) {
                          int j = -1;
                          if (pos == k)
                            j = 0;
                          else if (pos > ncand - nS && pos < ncand)
                            j = ncand - pos;
                          if (j >= 0) {
                            for (int d = 0; d < kBcCL; d++)
                              *at_rank(cl, &sh.x.V[par][t][j], d, rank) = v;
                          } else if (pos < ncand) {
                            keep_larger(bv, bi, fabs(v), pos);
                          } else {
                            cm = fmax(cm, fabs(v));
                          }
                        });
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
      // ---- exchange 2: warp t forms the imax column of member t (every W
      // column is in HBM by now)
      if (need2 & (1u << warp)) {
        const int t = warp;
        const int pc = sh.x.cand[t].imaxp;
        const double wl = (lane < kw) ? __ldcg(Wph + (size_t)lane * f + pc) : 0.0;
        double w[kNB];
#pragma unroll
        for (int c = 0; c < kNB; c++) w[c] = __shfl_sync(0xffffffffu, wl, c);
        double rm = 0.0;
        double* out = cb1 + (size_t)t * R;
        const double* colk = cb0 + (size_t)t * R;
        big_member_column<NB>(F, f, Lp, ipos, r0, Q, pc, k, kw, lane, w, out,
                          [&](int q, int r, int pos, double v) {
                            if (r == pc) {
                              const double wik = colk[q];
                              for (int d = 0; d < kBcCL; d++) {
                                double* dst = at_rank(cl, &sh.x.P2[par][t][0], d, rank);
                                dst[0] = v;
                                dst[1] = wik;
                              }
                            } else {
                              rm = fmax(rm, fabs(v));
                            }
                          });
        rm = warp_max_nonneg(rm);
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
