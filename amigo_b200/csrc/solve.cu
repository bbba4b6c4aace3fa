// Level-scheduled supernodal solves with the stored multifrontal factor.
//
// Forward (leaves to roots): each supernode assembles a front vector from the
// right-hand side at its own variables and the update vectors of its
// children, applies its unit-lower pivot block (1x1 and 2x2 pivots) down the
// whole front, writes D^{-1} t to the solution at its pivot variables and
// leaves the rest of the front as its own update vector for the parent. No
// two supernodes of a level write the same location, so the sweep is
// deterministic and needs no atomics.
//
// Backward (roots to leaves): gather the final solution at the delayed and
// contribution rows, subtract L21^T x2, back-substitute L11^T and scatter to
// the pivot variables.
//
// Same arithmetic as the reference's solve_ldl (include/sparse_ldl.h:
// 1825-1926: solve_pivot_lower, L21 product, scatter_subtract,
// solve_pivot_diagonal, and the transposed sweep), reorganised so that the
// descendants' contributions travel as update vectors instead of
// scatter-subtracts into the shared solution vector, and blocked: one warp
// solves each diagonal block of up to 33 pivots while the whole CTA applies
// the block to the rows below, with all right-hand sides of a chunk at once.
#include "ldl_internal.h"

namespace b200ldl {

namespace {

constexpr int kSWarps = kSolveThreads / 32;
constexpr int kBlk = 32;

constexpr int kMaxRhs = 8;  // right-hand sides per launch

// v[r][j] -= sum_{i in [i0, i1)} L(i, j) v[r][i] for r < nr, by one warp
__device__ __forceinline__ void gemv_t_col(const double* L, int ldl, int j, int i0, int i1,
                                           double* v, int f, int nr, int lane) {
  const double* lj = L + (size_t)ldl * j;
  double acc[kMaxRhs];
#pragma unroll
  for (int r = 0; r < kMaxRhs; r++) acc[r] = 0.0;
  // four rows per lane pass: their loads are in flight together
  for (int ib = i0 + lane; ib < i1; ib += 128) {
    double l4[4];
#pragma unroll
    for (int u = 0; u < 4; u++) l4[u] = (ib + 32 * u < i1) ? lj[ib + 32 * u] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int i = ib + 32 * u;
      if (i >= i1) break;
#pragma unroll
      for (int r = 0; r < kMaxRhs; r++)
        if (r < nr) acc[r] += l4[u] * v[(size_t)r * f + i];
    }
  }
#pragma unroll
  for (int r = 0; r < kMaxRhs; r++) {
    if (r < nr) {
      double a = acc[r];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) v[(size_t)r * f + j] -= a;
    }
  }
}

// end of the pivot block starting at jb: at most 32 pivots, and 2x2 pairs
// never straddle two blocks
__device__ __forceinline__ int block_end(const int* fv, int jb, int npiv) {
  int j = jb;
  while (j < npiv) {
    const int st = (fv[j] >= 0) ? 1 : 2;
    if (j + st - jb > kBlk) break;
    j += st;
  }
  return j;
}

// Bit t set if position jb + t is the second row of a 2x2 pivot. Blocks
// start on a pair boundary, so inside a run of negative (2x2-marked) entries
// the odd offsets are the second rows.
__device__ __forceinline__ unsigned second_rows(const int* fv, int jb, int je, int lane) {
  const bool neg = (jb + lane < je) && fv[jb + lane] < 0;
  const unsigned negm = __ballot_sync(0xffffffffu, neg);
  const unsigned below = lane == 0 ? 0u : (~negm) & ((1u << lane) - 1u);
  const int start = below ? (32 - __clz(below)) : 0;
  return __ballot_sync(0xffffffffu, neg && ((lane - start) & 1));
}

// Warp 0: forward substitution with the unit-lower diagonal block (rows and
// columns [jb, je), at most 32) held in registers (lane t owns row jb + t),
// then D^{-1} to the solution at the block's pivot variables.
__device__ __forceinline__ void fwd_block(const double* L, int ldl, const int* fv, int jb,
                                          int je, double* v, int f, int nr, double* x,
                                          int ldx, int r0, int lane) {
  const int nb = je - jb;
  const unsigned sec = second_rows(fv, jb, je, lane);
  const bool mine = lane < nb;
  double Lrow[kBlk];
#pragma unroll
  for (int j = 0; j < kBlk; j++)
    Lrow[j] = (mine && j < nb) ? L[(jb + lane) + (size_t)ldl * (jb + j)] : 0.0;
  double vr[kMaxRhs];
#pragma unroll
  for (int r = 0; r < kMaxRhs; r++) vr[r] = (mine && r < nr) ? v[(size_t)r * f + jb + lane] : 0.0;
#pragma unroll
  for (int j = 0; j < kBlk; j++) {
    if (j < nb) {
      const bool first = j + 1 < nb && ((sec >> (j + 1)) & 1u);
      const bool upd = lane > j && !(first && lane == j + 1);
#pragma unroll
      for (int r = 0; r < kMaxRhs; r++) {
        const double vj = __shfl_sync(0xffffffffu, vr[r], j);
        if (upd && r < nr) vr[r] = fma(-Lrow[j], vj, vr[r]);
      }
    }
  }
  // D^{-1}: 1x1 pivots divide; 2x2 pairs exchange values with the partner
  const bool is_sec = (sec >> lane) & 1u;
  const bool is_first = lane + 1 < 32 && ((sec >> (lane + 1)) & 1u) && lane + 1 < nb;
  const double dd = mine ? L[(jb + lane) + (size_t)ldl * (jb + lane)] : 1.0;
  const double dsub = (mine && is_sec) ? L[(jb + lane) + (size_t)ldl * (jb + lane - 1)] : 0.0;
  const double dd_up = __shfl_down_sync(0xffffffffu, dd, 1);
  const double dsub_up = __shfl_down_sync(0xffffffffu, dsub, 1);
  const double dd_dn = __shfl_up_sync(0xffffffffu, dd, 1);
  const int var = mine ? fv[jb + lane] : 0;
  const int vi = var >= 0 ? var : -var - 1;
#pragma unroll
  for (int r = 0; r < kMaxRhs; r++) {
    const double up = __shfl_down_sync(0xffffffffu, vr[r], 1);
    const double dn = __shfl_up_sync(0xffffffffu, vr[r], 1);
    if (mine && r < nr) {
      double y;
      if (is_first) {
        const double d11 = dd, d21 = dsub_up, d22 = dd_up;
        y = (d22 * vr[r] - d21 * up) / (d11 * d22 - d21 * d21);
      } else if (is_sec) {
        const double d11 = dd_dn, d21 = dsub, d22 = dd;
        y = (d11 * vr[r] - d21 * dn) / (d11 * d22 - d21 * d21);
      } else {
        y = vr[r] / dd;
      }
      x[(size_t)ldx * (r0 + r) + vi] = y;
      v[(size_t)r * f + jb + lane] = vr[r];
    }
  }
}

// Warp 0: back substitution with the transposed block L11^T (lane t owns
// row jb + t and keeps column jb + t of the block in registers).
__device__ __forceinline__ void bwd_block(const double* L, int ldl, const int* fv, int jb,
                                          int je, double* v, int f, int nr, int lane) {
  const int nb = je - jb;
  const unsigned sec = second_rows(fv, jb, je, lane);
  const bool mine = lane < nb;
  double Lcol[kBlk];
  const double* col = L + (size_t)ldl * (jb + lane) + jb;
#pragma unroll
  for (int q = 0; q < kBlk; q++) Lcol[q] = (mine && q < nb) ? col[q] : 0.0;
  double vr[kMaxRhs];
#pragma unroll
  for (int r = 0; r < kMaxRhs; r++) vr[r] = (mine && r < nr) ? v[(size_t)r * f + jb + lane] : 0.0;
#pragma unroll
  for (int jj = kBlk - 1; jj >= 0; jj--) {
    if (jj < nb) {
      const bool upd = lane < jj && !(((sec >> jj) & 1u) && lane == jj - 1);
#pragma unroll
      for (int r = 0; r < kMaxRhs; r++) {
        const double vj = __shfl_sync(0xffffffffu, vr[r], jj);
        if (upd && r < nr) vr[r] = fma(-Lcol[jj], vj, vr[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kMaxRhs; r++)
    if (mine && r < nr) v[(size_t)r * f + jb + lane] = vr[r];
}

__global__ void __launch_bounds__(kSolveThreads, 2)
    forward_level_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                         double* __restrict__ x, int ldx, int nrhs, int r0, int nr,
                         double* __restrict__ upool) {
  extern __shared__ __align__(16) double sm[];
  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = s.f[node];
  const int fs = s.fs[node];
  const int npiv = s.npiv[node];
  const int ns = p.ns[node];
  const int m = f - npiv;
  const int nd_in = fs - ns;
  const int* fv = s.ivars + s.fv_off[node];
  const int* orig = fv + f;
  const double* L = s.dpool + s.L_off[node];
  const int ldl = s.L_ld[node];
  const int kb = p.kid_ptr[node];
  const int ke = p.kid_ptr[node + 1];
  double* v = sm;                          // [nr][f], post-pivot order
  int* post_of = (int*)(sm + (size_t)nr * f);  // [f]

  for (int q = tid; q < f; q += blockDim.x) post_of[q < fs ? orig[q] : q] = q;
  for (int q = tid; q < nr * f; q += blockDim.x) v[q] = 0.0;
  __syncthreads();
  const int v0 = p.var_ptr[node];
  for (int q = tid; q < nr * ns; q += blockDim.x) {
    const int r = q / ns;
    const int t = q - r * ns;
    v[(size_t)r * f + post_of[t]] = x[(size_t)ldx * (r0 + r) + p.node_to_var[v0 + t]];
  }
  __syncthreads();
  int off = ns;
  for (int c = kb; c < ke; c++) {
    const int ch = p.kids[c];
    const int nd = s.ndel[ch];
    const int mc = s.f[ch] - s.npiv[ch];
    const double* uc = upool + s.u_off[ch] * nrhs + (size_t)r0 * mc;
    const int* cm = p.cmap + p.cptr[ch];
    for (int t = tid; t < mc; t += blockDim.x) {
      int q;
      if (t < nd) {
        q = off + t;
      } else {
        q = cm[t - nd];
        if (q >= ns) q += nd_in;
      }
      q = post_of[q];
      for (int r = 0; r < nr; r++) v[(size_t)r * f + q] += uc[(size_t)r * mc + t];
    }
    __syncthreads();
    off += nd;
  }

  // blocked unit-lower solve: warp 0 solves the diagonal block in registers
  // and writes D^{-1} t to the solution; then the CTA updates the rows below
  for (int jb = 0; jb < npiv;) {
    const int je = block_end(fv, jb, npiv);
    if (warp == 0) fwd_block(L, ldl, fv, jb, je, v, f, nr, x, ldx, r0, lane);
    __syncthreads();
    for (int i = je + tid; i < f; i += blockDim.x) {
      double acc[kMaxRhs];
#pragma unroll
      for (int r = 0; r < kMaxRhs; r++) acc[r] = 0.0;
      // the row's block entries are all loaded before the products, so that
      // their HBM latency is paid once per row, not once per column
      // (two halves of 16 columns keep the registers for two CTAs per SM)
#pragma unroll
      for (int h = 0; h < kBlk; h += 16) {
        if (jb + h >= je) break;
        double lv[16];
#pragma unroll
        for (int j = 0; j < 16; j++)
          lv[j] = (jb + h + j < je) ? L[i + (size_t)ldl * (jb + h + j)] : 0.0;
#pragma unroll
        for (int j = 0; j < 16; j++) {
          if (jb + h + j >= je) break;
#pragma unroll
          for (int r = 0; r < kMaxRhs; r++)
            if (r < nr) acc[r] = fma(lv[j], v[(size_t)r * f + jb + h + j], acc[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < kMaxRhs; r++)
        if (r < nr) v[(size_t)r * f + i] -= acc[r];
    }
    __syncthreads();
    jb = je;
  }
  double* uo = upool + s.u_off[node] * nrhs + (size_t)r0 * m;
  for (int q = tid; q < nr * m; q += blockDim.x) {
    const int r = q / m;
    const int t = q - r * m;
    uo[(size_t)r * m + t] = v[(size_t)r * f + npiv + t];
  }
}

__global__ void __launch_bounds__(kSolveThreads)
    backward_level_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                          double* __restrict__ x, int ldx, int r0, int nr) {
  extern __shared__ __align__(16) double sm[];
  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = s.f[node];
  const int npiv = s.npiv[node];
  const int* fv = s.ivars + s.fv_off[node];
  const double* L = s.dpool + s.L_off[node];
  const int ldl = s.L_ld[node];
  double* v = sm;                           // [nr][f]
  int* bst = (int*)(sm + (size_t)nr * f);   // block starts

  for (int q = tid; q < nr * f; q += blockDim.x) {
    const int r = q / f;
    const int t = q - r * f;
    const int var = fv[t];
    v[q] = x[(size_t)ldx * (r0 + r) + (var >= 0 ? var : -var - 1)];
  }
  __shared__ int nblk;
  if (tid == 0) {
    int nb = 0;
    for (int jb = 0; jb < npiv;) {
      bst[nb++] = jb;
      jb = block_end(fv, jb, npiv);
    }
    bst[nb] = npiv;
    nblk = nb;
  }
  __syncthreads();
  // t1 -= L21^T x2, one warp per pivot column, all RHS per L read
  if (npiv < f) {
    for (int j = warp; j < npiv; j += kSWarps) gemv_t_col(L, ldl, j, npiv, f, v, f, nr, lane);
    __syncthreads();
  }
  // L11^T back substitution, block by block from the last
  for (int b = nblk - 1; b >= 0; b--) {
    const int jb = bst[b];
    const int je = bst[b + 1];
    if (je < npiv) {
      for (int j = jb + warp; j < je; j += kSWarps) gemv_t_col(L, ldl, j, je, npiv, v, f, nr, lane);
      __syncthreads();
    }
    if (warp == 0) bwd_block(L, ldl, fv, jb, je, v, f, nr, lane);
    __syncthreads();
  }
  for (int q = tid; q < nr * npiv; q += blockDim.x) {
    const int r = q / npiv;
    const int t = q - r * npiv;
    const int var = fv[t];
    x[(size_t)ldx * (r0 + r) + (var >= 0 ? var : -var - 1)] = v[(size_t)r * f + t];
  }
}

}  // namespace

constexpr size_t kSolveSmemMax = 224 * 1024;

cudaError_t configure_solve_kernels() {
  cudaError_t e = cudaFuncSetAttribute(forward_level_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSolveSmemMax);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(backward_level_kernel,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSolveSmemMax);
}

// right-hand sides per launch so that [nr][fmax] doubles + fmax ints fit
int solve_rhs_chunk(int fmax, int nrhs) {
  const size_t per = (size_t)fmax * sizeof(double);
  const size_t fixed = (size_t)fmax * sizeof(int) + 64;
  if (fixed + per > kSolveSmemMax) return 0;
  int c = (int)((kSolveSmemMax - fixed) / per);
  if (c > kMaxRhs) c = kMaxRhs;
  return c < nrhs ? c : nrhs;
}

int launch_forward_level(const DevPlan& p, const DevState& s, const int* level_nodes,
                         int count, double* x, int ldx, int nrhs, double* upool,
                         int fmax, cudaStream_t stream) {
  if (count <= 0) return 0;
  const int c = solve_rhs_chunk(fmax, nrhs);
  int n = 0;
  for (int r0 = 0; r0 < nrhs; r0 += c) {
    const int nr = (nrhs - r0 < c) ? nrhs - r0 : c;
    const size_t smem = (size_t)nr * fmax * sizeof(double) + (size_t)fmax * sizeof(int);
    forward_level_kernel<<<count, kSolveThreads, smem, stream>>>(p, s, level_nodes, x, ldx,
                                                                 nrhs, r0, nr, upool);
    n++;
  }
  return n;
}

int launch_backward_level(const DevPlan& p, const DevState& s, const int* level_nodes,
                          int count, double* x, int ldx, int nrhs, int fmax,
                          cudaStream_t stream) {
  if (count <= 0) return 0;
  const int c = solve_rhs_chunk(fmax, nrhs);
  int n = 0;
  for (int r0 = 0; r0 < nrhs; r0 += c) {
    const int nr = (nrhs - r0 < c) ? nrhs - r0 : c;
    const size_t smem = (size_t)nr * fmax * sizeof(double) + (size_t)fmax * sizeof(int);
    backward_level_kernel<<<count, kSolveThreads, smem, stream>>>(p, s, level_nodes, x, ldx,
                                                                  r0, nr);
    n++;
  }
  return n;
}

}  // namespace b200ldl
