// Fronts resident in a thread-block cluster's distributed shared memory.
//
// A front of size f (145 <= f <= cluster_front_limit(4)) is held entirely on
// chip: its lower triangle is split row-cyclically over the CL CTAs of a
// cluster (physical row r on CTA r % CL, rows stored packed, row-major), so
// every CTA holds about f^2 / (2 CL) doubles. The front is assembled
// straight into DSMEM (CSR entries, the diagonal vector, the children's
// contribution blocks), factored with the reference's threshold 1x1 / 2x2 /
// delay tests (SparseLDL::factor_front_matrix_block,
// include/sparse_ldl.h:1316-1553; Bunch-Kaufman when there are no
// contribution rows, as LAPACK dsytrf there), and only the factor columns
// and the contribution block leave the chip.
//
// Symmetric interchanges are never carried out on the data. The logical
// order of the front (what the reference's symm_swap produces) is kept as a
// permutation perm / ipos replicated in every CTA, and element {i, j} is
// read from the physical lower-triangle slot of {perm[i], perm[j]}. A delay
// or a pivot interchange is a two-entry update of perm. The factor columns
// and the contribution block are written out in logical order at the end.
//
// Speculative delay chains. A delay leaves the Schur complement unchanged,
// so the candidates the reference would test after t delays in a row
// (position k, then the ones swapped in from ncand-1, ncand-2, ...) are
// known in advance and have the same columns. Each step therefore forms the
// columns of a chain of up to 8 candidates at once (one per warp), reduces
// their statistics in one cluster exchange, forms the imax columns the
// tests need in a second exchange, and then replays the reference's
// sequential decisions on those values: the first member that is accepted
// ends the chain, the ones before it are delayed. The decisions are the
// ones the one-candidate-at-a-time algorithm takes.
//
// Blocked: accepted pivot columns are collected in panels of up to 16.
// Inside a panel the front is left untouched: a candidate column is
// F(:,c) - Lp W(c,:)^T with the panel's L on the owner's rows and a copy of
// the panel's W rows in every CTA (the reference's W formulation,
// sparse_ldl.h:1337-1344). After the panel each CTA applies one
// register-tiled rank-kw update to its own remaining rows from its own
// shared memory.
#include <cooperative_groups.h>

#include <climits>

#include "front_common.cuh"
#include "ldl_internal.h"

namespace cg = cooperative_groups;

namespace b200ldl {

namespace {

using namespace chain;

constexpr int kCfThreads = 256;
constexpr int kCfWarps = kCfThreads / 32;
constexpr int kNB = 16;           // panel width (pivot columns per trailing update)
constexpr int kNBP = kNB + 1;     // odd row stride of the panel arrays
static_assert(kChain == kCfWarps, "one chain member per warp");

// offset of physical row r inside its owner's packed storage (owner r % CL,
// local row q = r / CL): q (o + 1) + CL q (q - 1) / 2 with o = r % CL
template <int CL>
__host__ __device__ __forceinline__ long long row_off(int r) {
  const long long q = r / CL;
  const long long o = r - q * CL;
  return q * (o + 1) + (long long)CL * q * (q - 1) / 2;
}

// packed length of CTA `rank`'s rows for a front of size f
template <int CL>
__host__ __device__ __forceinline__ long long tri_len(int f, int rank) {
  const long long Q = (f - rank + CL - 1) / CL;
  return Q * (rank + 1) + (long long)CL * Q * (Q - 1) / 2;
}

// the same shared-memory object in CTA r of the cluster
template <int CL, typename T>
__device__ __forceinline__ T* at_rank(cg::cluster_group& cl, T* ptr, int r, int rank) {
  if constexpr (CL == 1) {
    return ptr;
  } else {
    return (r == rank) ? ptr : cl.map_shared_rank(ptr, (unsigned)r);
  }
}

template <int CL>
__device__ __forceinline__ double* row_ptr(cg::cluster_group& cl, double* tri, int rank, int r) {
  return at_rank<CL>(cl, tri, r % CL, rank) + row_off<CL>(r);
}

template <int CL>
__device__ __forceinline__ void csync(cg::cluster_group& cl) {
  if constexpr (CL == 1)
    __syncthreads();
  else
    cl.sync();
}

template <int CL>
struct CfShared {
  static constexpr int NPAR = (CL == 1) ? 1 : 2;  // exchange buffers by step parity
  ChainXchg<CL, NPAR> x;
  int piv[kNB];  // physical rows of the panel's pivots
  int scan[kCfWarps];
};

// Shared-memory layout of one CTA (in doubles), the same in every CTA of the
// cluster so that a DSMEM address maps to the same array in each: packed
// own rows of the front (sized for the CTA with the longest share), the
// panel's W for all physical rows [f][kNBP], the panel's L for own rows
// [Qmax][kNBP], the chain's columns over own rows [NPAR][2][kChain][Qmax],
// then perm, ipos, rem and rpos ([f] ints each).
template <int CL>
__host__ __device__ __forceinline__ long long cf_layout(int f, long long* oW, long long* oL,
                                                        long long* oC, long long* oI) {
  long long t = 0;
  for (int r = 0; r < CL; r++) {
    const long long tr = tri_len<CL>(f, r);
    t = tr > t ? tr : t;
  }
  const long long Qmax = (f + CL - 1) / CL;
  *oW = t;
  *oL = *oW + (long long)f * kNBP;
  *oC = *oL + Qmax * kNBP;
  *oI = *oC + (long long)CfShared<CL>::NPAR * 2 * kChain * Qmax;
  return *oI + (4LL * f + 1) / 2;
}

// Column pc of the current Schur complement on this CTA's rows, for one
// warp: v(r) = F_sym(r, pc) - Lp(r,:) W(pc,:)^T, two rows per lane pass.
// Rows already eliminated (logical position < k) are skipped; for the
// others the value is stored in out[q] and handed to use(q, r, pos, v).
template <int CL, typename Use>
__device__ __forceinline__ void member_column(cg::cluster_group& cl, double* tri,
                                              const double* Lp, const double* Wall,
                                              const int* ipos, int rank, int Q, int pc, int k,
                                              int kwn, int lane, double* out, Use use) {
  double w[kNB];
  const double* wr = Wall + (size_t)pc * kNBP;
#pragma unroll
  for (int c = 0; c < kNB; c++) w[c] = wr[c];
  const double* rowc = row_ptr<CL>(cl, tri, rank, pc);
  for (int q0 = lane; q0 < Q; q0 += 64) {
    const int q1 = q0 + 32;
    const bool h1 = q1 < Q;
    const int r0 = rank + q0 * CL;
    const int r1 = rank + (h1 ? q1 : q0) * CL;
    const int pos0 = ipos[r0];
    const int pos1 = h1 ? ipos[r1] : -1;
    const double f0 = (r0 >= pc) ? tri[row_off<CL>(r0) + pc] : rowc[r0];
    const double f1 = (r1 >= pc) ? tri[row_off<CL>(r1) + pc] : rowc[r1];
    const double* l0 = Lp + (size_t)q0 * kNBP;
    const double* l1 = Lp + (size_t)(h1 ? q1 : q0) * kNBP;
    double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
    // columns at and beyond the panel's width are zero: skip them in
    // groups of 8 (exact, the skipped products are zeros)
#pragma unroll
    for (int c8 = 0; c8 < kNB; c8 += 8) {
      if (c8 >= kwn) break;
#pragma unroll
      for (int c = c8; c < c8 + 8; c += 2) {
        a0 = fma(l0[c], w[c], a0);
        a1 = fma(l0[c + 1], w[c + 1], a1);
        b0 = fma(l1[c], w[c], b0);
        b1 = fma(l1[c + 1], w[c + 1], b1);
      }
    }
    const double v0 = f0 - (a0 + a1);
    const double v1 = f1 - (b0 + b1);
    if (pos0 >= k) {
      out[q0] = v0;
      use(q0, r0, pos0, v0);
    }
    if (h1 && pos1 >= k) {
      out[q1] = v1;
      use(q1, r1, pos1, v1);
    }
  }
  __syncwarp();  // reconverge before the caller's warp reductions
}

template <int CL>
__global__ void __launch_bounds__(kCfThreads)
    cluster_front_kernel(DevPlan p, DevState s, const int* __restrict__ list,
                         const double* __restrict__ vals, const double* __restrict__ diag,
                         FactorParams prm) {
  constexpr int NPAR = CfShared<CL>::NPAR;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  BigFront* B = s.big + list[blockIdx.x / CL];
  extern __shared__ __align__(16) double sm[];
  __shared__ CfShared<CL> sh;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int gt = rank * kCfThreads + tid;  // thread id in the cluster
  const int gw = rank * kCfWarps + warp;   // warp id in the cluster
  const int f = B->f;
  const int fs = B->fs;
  const int ns = B->ns;
  const int nd_in = B->nd_in;
  const int node = B->node;
  const bool root = (B->nc == 0);
  long long oW, oL, oC, oI;
  cf_layout<CL>(f, &oW, &oL, &oC, &oI);
  const int Qmax = (f + CL - 1) / CL;
  const int Q = (f - rank + CL - 1) / CL;  // own physical rows r = rank + q CL
  double* tri = sm;
  double* Wall = sm + oW;
  double* Lp = sm + oL;
  double* colbuf = sm + oC;
  int* perm = reinterpret_cast<int*>(sm + oI);
  int* ipos = perm + f;
  int* rem = ipos + f;
  int* rpos = rem + f;
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;

  // ---- zero the front and the panel arrays, identity order
  for (long long t = tid; t < oI; t += kCfThreads) sm[t] = 0.0;
  for (int r = tid; r < f; r += kCfThreads) {
    perm[r] = r;
    ipos[r] = r;
  }
  csync<CL>(cl);

  // ---- assembly straight into distributed shared memory (physical order is
  // the front's initial variable order)
  {
    const int64_t e0 = p.scat_ptr[node];
    const int64_t e1 = p.scat_ptr[node + 1];
    for (int64_t e = e0 + gt; e < e1; e += CL * kCfThreads) {
      int r = p.scat_row[e];
      if (r >= ns) r += nd_in;
      double* dst = row_ptr<CL>(cl, tri, rank, r) + p.scat_col[e];
      *dst += csr_value(s, vals, p.scat_csr[e]);
    }
  }
  csync<CL>(cl);
  if (diag) {
    const int v0 = p.var_ptr[node];
    for (int j = gt; j < ns; j += CL * kCfThreads) {
      double* dst = row_ptr<CL>(cl, tri, rank, j) + j;
      *dst += diag[p.node_to_var[v0 + j]];
    }
    csync<CL>(cl);
  }
  {
    const int kb = p.kid_ptr[node];
    const int ke = p.kid_ptr[node + 1];
    int off = ns;
    for (int c = kb; c < ke; c++) {
      const int ch = p.kids[c];
      const int nd = s.ndel[ch];
      const int m = s.f[ch] - s.npiv[ch];
      const double* cb = s.dpool + s.cb_off[ch];
      const int cld = s.cb_ld[ch];
      const int* cm = p.cmap + p.cptr[ch];
      for (int r2 = gw; r2 < m; r2 += CL * kCfWarps) {
        int p2;
        if (r2 < nd) {
          p2 = off + r2;
        } else {
          p2 = cm[r2 - nd];
          if (p2 >= ns) p2 += nd_in;
        }
        const double* col = cb + (size_t)cld * r2;
        // four entries per lane pass: their loads are issued before the
        // read-modify-writes into the front
        for (int rb = r2 + lane; rb < m; rb += 128) {
          int p1[4];
          double v[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int r1 = rb + 32 * u;
            p1[u] = -1;
            if (r1 < m) {
              int pp;
              if (r1 < nd) {
                pp = off + r1;
              } else {
                pp = cm[r1 - nd];
                if (pp >= ns) pp += nd_in;
              }
              p1[u] = pp;
              v[u] = col[r1];
            }
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            if (p1[u] < 0) continue;
            const int hi = p1[u] >= p2 ? p1[u] : p2;
            const int lo = p1[u] >= p2 ? p2 : p1[u];
            double* dst = row_ptr<CL>(cl, tri, rank, hi) + lo;
            *dst += v[u];
          }
        }
      }
      csync<CL>(cl);
      off += nd;
    }
  }

  // ---- partial factorization of the candidates [0, ncand)
  const bool single = root || prm.cholesky;  // no delays: chains of one
  int k = 0;
  int ncand = fs;
  int npos = 0, nneg = 0;
  double flops = 0.0;
  int stepno = 0;

  while (k < ncand) {
    const int kstart = k;
    int kw = 0;
    while (kw < kNB - 1 && k < ncand) {
      const int par = (NPAR == 1) ? 0 : (stepno & 1);
      stepno++;
      const int nS = single ? 1 : min(kChain, ncand - k);
      // chain member t sits at logical position k (t = 0) or ncand - t
      double* cb0 = colbuf + (size_t)(par * 2) * kChain * Qmax;
      double* cb1 = cb0 + (size_t)kChain * Qmax;

      // ---- exchange 1: warp t forms the column of chain member t
      if (warp < nS) {
        const int t = warp;
        const int pc = (t == 0) ? perm[k] : perm[ncand - t];
        double bv = 0.0, cm = 0.0;
        int bi = INT_MAX;
        double* out = cb0 + (size_t)t * Qmax;
        member_column<CL>(cl, tri, Lp, Wall, ipos, rank, Q, pc, k, kw, lane, out,
                          [&](int q, int r, int pos, double v) {
                            int j = -1;
                            if (pos == k)
                              j = 0;
                            else if (pos > ncand - nS && pos < ncand)
                              j = ncand - pos;
                            if (j >= 0) {
                              for (int d = 0; d < CL; d++)
                                *at_rank<CL>(cl, &sh.x.V[par][t][j], d, rank) = v;
                            } else if (pos < ncand) {
                              keep_larger(bv, bi, fabs(v), pos);
                            } else {
                              cm = fmax(cm, fabs(v));
                            }
                          });
        warp_argmax_max(bv, bi, cm);
        if (lane < CL) {
          ColStat st;
          st.bv = bv;
          st.cm = cm;
          st.bi = bi;
          st.pad = 0;
          *at_rank<CL>(cl, &sh.x.s1[par][rank][t], lane, rank) = st;
        }
      }
      csync<CL>(cl);  // B1: statistics and chain entries visible everywhere

      // member tests from the columns alone
      if (warp < nS)
        decide_column<CL, NPAR>(sh.x, par, warp, lane, nS, k, ncand, root, prm, perm);
      __syncthreads();

      unsigned acc1;
      int d1l;
      const unsigned need2 = need_rows(sh.x.cand, nS, lane, acc1, d1l);
      if (need2) {
        // ---- exchange 2: warp t forms the imax column of member t
        if (need2 & (1u << warp)) {
          const int t = warp;
          const int pc = sh.x.cand[t].imaxp;
          double rm = 0.0;
          double* out = cb1 + (size_t)t * Qmax;
          const double* colk = cb0 + (size_t)t * Qmax;
          member_column<CL>(cl, tri, Lp, Wall, ipos, rank, Q, pc, k, kw, lane, out,
                            [&](int q, int r, int pos, double v) {
                              if (r == pc) {
                                const double wik = colk[q];
                                for (int d = 0; d < CL; d++) {
                                  double* dst = at_rank<CL>(cl, &sh.x.P2[par][t][0], d, rank);
                                  dst[0] = v;
                                  dst[1] = wik;
                                }
                              } else {
                                rm = fmax(rm, fabs(v));
                              }
                            });
          rm = warp_max_nonneg(rm);
          if (lane < CL) *at_rank<CL>(cl, &sh.x.s2[par][rank][t], lane, rank) = rm;
        }
        csync<CL>(cl);  // B2
        if (need2 & (1u << warp)) decide_row<CL, NPAR>(sh.x, par, warp, lane, root, prm);
        __syncthreads();
      }

      // ---- replay the sequential decisions: delays up to the first
      // accepted member; the logical order by warp 0
      int tacc, kind;
      replay(sh.x.cand, nS, lane, acc1, d1l, tacc, kind);
      const int ndelay = tacc;  // members before tacc (all nS when none accepted)
      const int nstep = (kind == kTwo) ? 2 : 1;
      const int pi_acc = (tacc < nS) ? sh.x.cand[tacc].imaxp : -1;
      if (warp == 0) reorder(sh.x.cand, perm, ipos, lane, nS, ndelay, k, ncand, kind, nstep, pi_acc);
      if (tacc == nS) {
        ncand -= ndelay;
        __syncthreads();
        continue;
      }
      const Cand& ca = sh.x.cand[tacc];
      const int pk = ca.mrow;
      const int pi = pi_acc;
      // accepted columns: the member's column at k, or the imax column at k
      // (1x1 at imax); a 2x2 takes both
      const double* colA = ((kind == kOneImax) ? cb1 : cb0) + (size_t)tacc * Qmax;
      const double* colB = cb1 + (size_t)tacc * Qmax;
      const int p0 = (kind == kOneImax) ? pi : pk;
      // W columns: every CTA gathers the accepted columns from their owners
      // (entries of eliminated rows are gathered too and never read)
      for (int r0 = tid; r0 < f; r0 += 4 * kCfThreads) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int r = r0 + u * kCfThreads;
          if (r < f) {
            a[u] = at_rank<CL>(cl, colA, r % CL, rank)[r / CL];
            if (nstep == 2) b[u] = at_rank<CL>(cl, colB, r % CL, rank)[r / CL];
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int r = r0 + u * kCfThreads;
          if (r < f) {
            Wall[(size_t)r * kNBP + kw] = a[u];
            if (nstep == 2) Wall[(size_t)r * kNBP + kw + 1] = b[u];
          }
        }
      }
      // L columns on own rows; the pivot rows keep D
      if (nstep == 1) {
        const double d = (kind == kOneImax) ? ca.wii : ca.wkk;
        const double dinv = (kind == kZero || (root && d == 0.0)) ? 0.0 : 1.0 / d;
        for (int q = tid; q < Q; q += kCfThreads) {
          const int r = rank + q * CL;
          Lp[(size_t)q * kNBP + kw] = (r == p0) ? d : colA[q] * dinv;
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
        for (int q = tid; q < Q; q += kCfThreads) {
          const int r = rank + q * CL;
          double* lr = Lp + (size_t)q * kNBP;
          if (r == pk) {
            lr[kw] = d11;
            lr[kw + 1] = 0.0;
          } else if (r == pi) {
            lr[kw] = d21;
            lr[kw + 1] = d22;
          } else {
            const double a = colA[q], b = colB[q];
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
      ncand -= ndelay;
      k += nstep;
      kw += nstep;
      __syncthreads();  // W, L and the order visible to every warp
    }

    if (kw > 0) {
      // the panel's L (and D) into the front's slots: row r, panel column c
      // (pivot row pc, logical position kstart + c) goes to slot {r, pc};
      // logical-lower entries only
      for (int q = warp; q < Q; q += kCfWarps) {
        const int r = rank + q * CL;
        const int pos = ipos[r];
        if (pos < kstart) continue;
        const double* lr = Lp + (size_t)q * kNBP;
        const long long ro = row_off<CL>(r);
        for (int c = lane; c < kw; c += 32) {
          if (pos < kstart + c) continue;
          const int pc = sh.piv[c];
          if (r >= pc)
            tri[ro + pc] = lr[c];
          else
            row_ptr<CL>(cl, tri, rank, pc)[r] = lr[c];
        }
      }
      // remaining physical rows, sorted: rem[0..nrem), rpos[r] = index
      {
        const int per = (f + kCfThreads - 1) / kCfThreads;
        const int a0 = tid * per;
        const int a1 = min(f, a0 + per);
        int cnt = 0;
        for (int r = a0; r < a1; r++) cnt += (ipos[r] >= k);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        if (lane == 31) sh.scan[warp] = incl;
        __syncthreads();
        int base = 0;
        for (int w2 = 0; w2 < warp; w2++) base += sh.scan[w2];
        int idx = base + incl - cnt;
        for (int r = a0; r < a1; r++) {
          if (ipos[r] >= k) {
            rem[idx] = r;
            rpos[r] = idx;
            idx++;
          }
        }
        __syncthreads();
      }
      // rank-kw trailing update of own remaining rows over remaining
      // columns (physical c <= r); two rows per warp pass share the W loads
      for (int qa = warp; qa < Q; qa += 2 * kCfWarps) {
        const int qb = qa + kCfWarps;
        const int ra = rank + qa * CL;
        const int rb = rank + qb * CL;
        const bool aon = ipos[ra] >= k;
        const bool bon = (qb < Q) && ipos[rb] >= k;
        if (!aon && !bon) continue;
        const int ja = aon ? rpos[ra] : -1;
        const int jb = bon ? rpos[rb] : -1;
        const int jmax = ja > jb ? ja : jb;
        double la[kNB], lb[kNB];
        const double* lra = Lp + (size_t)qa * kNBP;
        const double* lrb = Lp + (size_t)(bon ? qb : qa) * kNBP;
#pragma unroll
        for (int c = 0; c < kNB; c++) {
          la[c] = aon ? lra[c] : 0.0;
          lb[c] = bon ? lrb[c] : 0.0;
        }
        double* ta = tri + row_off<CL>(ra);
        double* tb = tri + row_off<CL>(bon ? rb : ra);
        for (int j = lane; j <= jmax; j += 32) {
          const int c = rem[j];
          const double* wc = Wall + (size_t)c * kNBP;
          double acca = 0.0, accb = 0.0;
#pragma unroll
          for (int cc = 0; cc < kNB; cc++) {
            const double wv = wc[cc];
            acca = fma(la[cc], wv, acca);
            accb = fma(lb[cc], wv, accb);
          }
          if (j <= ja) ta[c] -= acca;
          if (j <= jb) tb[c] -= accb;
        }
      }
      if (rank == 0 && tid == 0) {
        const double r = (double)(f - k);
        flops += r * (r + 1.0) * kw;
      }
      __syncthreads();
      for (int t = tid; t < Q * kNBP; t += kCfThreads) Lp[t] = 0.0;
      csync<CL>(cl);  // updates and L slots visible before the next panel
    }
  }

  // ---- write the factor columns (f x npiv, ld f) and the contribution
  // block ((f-npiv)^2, ld f-npiv) in logical order into the pool region
  const int npiv = k;
  const int m = f - npiv;
  double* Lg = s.dpool + B->doff;
  double* Cg = Lg + (size_t)f * npiv;
  for (int j = rank + CL * warp; j < f; j += CL * kCfWarps) {
    const int pj = perm[j];
    for (int i = j + lane; i < f; i += 32) {
      const int pi = perm[i];
      const int hi = pi >= pj ? pi : pj;
      const int lo = pi >= pj ? pj : pi;
      const double v = row_ptr<CL>(cl, tri, rank, hi)[lo];
      if (j < npiv)
        Lg[i + (size_t)f * j] = v;
      else
        Cg[(i - npiv) + (size_t)m * (j - npiv)] = v;
    }
  }
  if (rank == 0) {
    // the front's variables in logical order (rem / rpos are free now)
    for (int i = tid; i < f; i += kCfThreads) {
      rem[i] = fv[perm[i]];
      rpos[i] = orig[perm[i]];
    }
    __syncthreads();
    for (int i = tid; i < f; i += kCfThreads) {
      fv[i] = rem[i];
      orig[i] = rpos[i];
    }
  }
  if (rank == 0 && tid == 0) {
    B->k = npiv;
    B->ncand = ncand;
    B->kw = 0;
    B->npos += npos;
    B->nneg += nneg;
    B->flops += flops;
    atomicAdd(s.flops + 4, flops);
    B->pad = 1;  // packed output layout: CB after L with ld m
    B->state = 2;
  }
  csync<CL>(cl);  // no CTA leaves while others read its shared memory
}

template <int CL>
cudaError_t launch_cf(const DevPlan& p, const DevState& s, const int* list, int count,
                      const double* vals, const double* diag, const FactorParams& prm,
                      size_t smem, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(count * CL, 1, 1);
  cfg.blockDim = dim3(kCfThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, cluster_front_kernel<CL>, p, s, list, vals, diag, prm);
}

template <int CL>
size_t cf_smem(int fmax) {
  long long oW, oL, oC, oI;
  return (size_t)cf_layout<CL>(fmax, &oW, &oL, &oC, &oI) * sizeof(double);
}

// dynamic shared memory available next to the kernel's static arrays
// (227 KB per CTA on sm_100, minus those and a small margin)
template <int CL>
constexpr size_t cf_dyn_max() {
  return 232448 - sizeof(CfShared<CL>) - 1024;
}

}  // namespace

// Largest front each cluster size can hold (shared memory per CTA).
int cluster_front_limit(int cl_index) {
  static int lim[5] = {0, 0, 0, 0, 0};
  if (lim[0] == 0) {
    int f;
    for (f = kSmemFrontMax; cf_smem<1>(f + 1) <= cf_dyn_max<1>(); f++) {}
    lim[0] = f;
    for (f = lim[0]; cf_smem<2>(f + 1) <= cf_dyn_max<2>(); f++) {}
    lim[1] = f;
    for (f = lim[1]; cf_smem<4>(f + 1) <= cf_dyn_max<4>(); f++) {}
    lim[2] = f;
    for (f = lim[2]; cf_smem<8>(f + 1) <= cf_dyn_max<8>(); f++) {}
    lim[3] = f;
    for (f = lim[3]; cf_smem<16>(f + 1) <= cf_dyn_max<16>(); f++) {}
    lim[4] = f;
  }
  return lim[cl_index];
}

cudaError_t configure_cluster_front_kernels() {
  cudaError_t e;
  e = cudaFuncSetAttribute(cluster_front_kernel<1>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cf_dyn_max<1>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<2>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cf_dyn_max<2>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<4>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cf_dyn_max<4>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<8>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cf_dyn_max<8>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<16>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cf_dyn_max<16>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(cluster_front_kernel<16>,
                              cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

// one launch per cluster size; class c holds fronts in
// (limit(c-1), limit(c)] and uses CL = 1 << c
cudaError_t launch_cluster_fronts(const DevPlan& p, const DevState& s, const int* counts,
                                  const int* maxf, const double* vals, const double* diag,
                                  const FactorParams& prm, cudaStream_t stream, int nn) {
  for (int c = 0; c < 5; c++) {
    if (counts[c] <= 0) continue;
    const int* list = s.class_list + (size_t)c * nn;
    cudaError_t e;
    switch (c) {
      case 0:
        e = launch_cf<1>(p, s, list, counts[c], vals, diag, prm, cf_smem<1>(maxf[c]), stream);
        break;
      case 1:
        e = launch_cf<2>(p, s, list, counts[c], vals, diag, prm, cf_smem<2>(maxf[c]), stream);
        break;
      case 2:
        e = launch_cf<4>(p, s, list, counts[c], vals, diag, prm, cf_smem<4>(maxf[c]), stream);
        break;
      case 3:
        e = launch_cf<8>(p, s, list, counts[c], vals, diag, prm, cf_smem<8>(maxf[c]), stream);
        break;
      default:
        e = launch_cf<16>(p, s, list, counts[c], vals, diag, prm, cf_smem<16>(maxf[c]),
                          stream);
        break;
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace b200ldl
