// Solves with the supernodes of large fronts, one thread-block cluster of
// 16 CTAs per supernode.
//
// A single CTA streams the whole factor block of a large supernode from HBM
// at the bandwidth of one SM; the cluster splits the front's rows (multiples
// of 32 rows per CTA) so that the factor is read by 16 SMs, and moves the
// solved values between CTAs through distributed shared memory. The
// arithmetic is the reference's solve_ldl (include/sparse_ldl.h:1825-1926):
// forward unit-lower solve with the pivot block, D^{-1}, backward solve with
// the transposed block, with the 2x2 pivots' off-diagonal D entry (stored in
// the L slot below the first row of the pair) excluded from the triangular
// sweeps.
//
// Forward, per 32-row pivot tile: the CTA owning the tile solves it in
// registers (one warp), one cluster barrier, then every CTA pulls the tile's
// values and updates its own rows below it. Backward, per tile from the
// last: every CTA forms L(rows below, tile)^T x on its own rows and pushes
// the partial sums to the tile's owner, one cluster barrier, then the owner
// subtracts them and back-substitutes the tile in registers.
#include <cooperative_groups.h>

#include "ldl_internal.h"

namespace cg = cooperative_groups;

namespace b200ldl {

namespace {

constexpr int kSbCL = 16;
constexpr int kSbThreads = 256;
constexpr int kSbWarps = kSbThreads / 32;
constexpr int kTileR = 32;
constexpr int kSbRhs = 8;  // right-hand sides per launch
static_assert(4 * kSbWarps == kTileR, "backward: four tile columns per warp");

template <typename T>
__device__ __forceinline__ T* at_rank(cg::cluster_group& cl, T* ptr, int r, int rank) {
  return (r == rank) ? ptr : cl.map_shared_rank(ptr, (unsigned)r);
}

// rows per CTA: a multiple of the tile height so that no tile is split
__host__ __device__ __forceinline__ int sb_rows(int f) {
  const int per = (f + kSbCL - 1) / kSbCL;
  return ((per + kTileR - 1) / kTileR) * kTileR;
}

// Bit t of secw[w]: position 32 w + t < npiv is the second row of a 2x2
// pivot. Inside a run of 2x2-marked positions the pairs start at the run's
// first position, so the second rows are the odd offsets into the run.
__device__ void second_row_bits(const int* fv, int npiv, unsigned* secw, int lane) {
  int carry = 0;  // parity of the run length entering the chunk
  for (int w = 0; w * 32 < npiv; w++) {
    const int p = 32 * w + lane;
    const bool neg = p < npiv && fv[p] < 0;
    const unsigned negm = __ballot_sync(0xffffffffu, neg);
    const unsigned nonneg_below = (~negm) & ((1u << lane) - 1u);
    const int ridx = nonneg_below ? lane - 32 + __clz(nonneg_below) : lane + carry;
    const unsigned secm = __ballot_sync(0xffffffffu, neg && (ridx & 1));
    if (lane == 0) secw[w] = secm;
    const int r31 = __shfl_sync(0xffffffffu, ridx, 31);
    carry = ((negm >> 31) & 1u) ? ((r31 + 1) & 1) : 0;
  }
}

__device__ __forceinline__ bool is_second(const unsigned* secw, int p) {
  return (secw[p >> 5] >> (p & 31)) & 1u;
}

__global__ void __launch_bounds__(kSbThreads, 1)
    forward_big_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                       double* __restrict__ x, int ldx, int nrhs, int r0rhs, int nr,
                       double* __restrict__ upool) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int node = nodes[blockIdx.x / kSbCL];
  extern __shared__ __align__(16) double sm[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int gt = rank * kSbThreads + tid;
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
  const int R = sb_rows(f);
  const int rb = rank * R;        // first own row
  const int re = min(f, rb + R);  // end of own rows
  double* v = sm;                                               // [nr][R] own rows, post-pivot order
  double* tb = v + (size_t)nr * R;                              // [kTileR][kSbRhs] pulled tile
  int* post_of = reinterpret_cast<int*>(tb + kTileR * kSbRhs);  // [f]
  unsigned* secw = reinterpret_cast<unsigned*>(post_of + f);    // [npiv / 32 + 1]

  for (int q = tid; q < f; q += kSbThreads) post_of[q < fs ? orig[q] : q] = q;
  for (int q = tid; q < nr * R; q += kSbThreads) v[q] = 0.0;
  if (warp == 0) second_row_bits(fv, npiv, secw, lane);
  cl.sync();
  // right-hand side at the supernode's own variables, into the owners' rows
  const int v0 = p.var_ptr[node];
  for (int t = gt; t < ns; t += kSbCL * kSbThreads) {
    const int q = post_of[t];
    const int o = q / R;
    double* dst = at_rank(cl, v, o, rank) + (q - o * R);
    const int var = p.node_to_var[v0 + t];
    for (int r = 0; r < nr; r++) dst[(size_t)r * R] = x[(size_t)ldx * (r0rhs + r) + var];
  }
  cl.sync();
  // children's update vectors, one child at a time (fixed summation order).
  // Every CTA reads each child's entries and adds the ones that land in its
  // own rows, so no two CTAs write a row and a CTA barrier separates the
  // children
  {
    const int kb = p.kid_ptr[node];
    const int ke = p.kid_ptr[node + 1];
    int off = ns;
    for (int c = kb; c < ke; c++) {
      const int ch = p.kids[c];
      const int nd = s.ndel[ch];
      const int mc = s.f[ch] - s.npiv[ch];
      const double* uc = upool + s.u_off[ch] * nrhs + (size_t)r0rhs * mc;
      const int* cm = p.cmap + p.cptr[ch];
#pragma unroll 1
      for (int t = tid; t < mc; t += kSbThreads) {
        int q;
        if (t < nd) {
          q = off + t;
        } else {
          q = cm[t - nd];
          if (q >= ns) q += nd_in;
        }
        q = post_of[q];
        if (q / R == rank) {
          double* dst = v + (q - rank * R);
#pragma unroll 1
          for (int r = 0; r < nr; r++) dst[(size_t)r * R] += uc[(size_t)r * mc + t];
        }
      }
      __syncthreads();
      off += nd;
    }
  }

  // unit-lower solve, tile by tile
  const int ntile = (npiv + kTileR - 1) / kTileR;
  // a tile's entries of this thread's first row below it: loaded a tile
  // ahead (they do not depend on the solved values), so that their HBM
  // latency overlaps the previous tile's update, barrier and solve
  double lvn[kTileR];
  auto prefetch = [&](int tb_) {
    const int jb_ = tb_ * kTileR;
    const int nb_ = min(jb_ + kTileR, npiv) - jb_;
    const int i_ = max(jb_ + nb_, rb) + tid;
    const double* li_ = L + i_ + (size_t)ldl * jb_;
#pragma unroll
    for (int j = 0; j < kTileR; j++) lvn[j] = (i_ < re && j < nb_) ? li_[(size_t)ldl * j] : 0.0;
  };
  if (ntile > 0) prefetch(0);
  for (int b = 0; b < ntile; b++) {
    const int jb = b * kTileR;
    const int je = min(jb + kTileR, npiv);
    const int nb = je - jb;
    const int ob = jb / R;
    if (rank == ob && warp == 0) {
      // the tile in registers: lane t owns row jb + t
      const bool mine = lane < nb;
      const unsigned sec = secw[jb >> 5];  // tiles are 32-aligned
      double Lrow[kTileR];
#pragma unroll
      for (int j = 0; j < kTileR; j++)
        Lrow[j] = (mine && j < nb) ? L[(jb + lane) + (size_t)ldl * (jb + j)] : 0.0;
      double vr[kSbRhs];
      double* vrow = v + (jb - rb) + lane;
#pragma unroll
      for (int r = 0; r < kSbRhs; r++) vr[r] = (mine && r < nr) ? vrow[(size_t)r * R] : 0.0;
#pragma unroll
      for (int j = 0; j < kTileR; j++) {
        if (j < nb) {
          // the L slot below the first row of a 2x2 pair holds D, not L
          const bool skip = (j + 1 < kTileR) && ((sec >> (j + 1)) & 1u) && lane == j + 1;
          const bool upd = lane > j && !skip;
#pragma unroll
          for (int r = 0; r < kSbRhs; r++) {
            const double vj = __shfl_sync(0xffffffffu, vr[r], j);
            if (upd && r < nr) vr[r] = fma(-Lrow[j], vj, vr[r]);
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kSbRhs; r++)
        if (mine && r < nr) vrow[(size_t)r * R] = vr[r];
    }
    cl.sync();  // the tile's solved values visible to the cluster
    // pull them, then update own rows below the tile
    {
      const double* src = at_rank(cl, v, ob, rank) + (jb - ob * R);
      for (int q = tid; q < nb * nr; q += kSbThreads) {
        const int r = q / nb;
        const int j = q - r * nb;
        tb[j * kSbRhs + r] = src[(size_t)r * R + j];
      }
    }
    __syncthreads();
    // a 2x2 pair across the tile boundary: its D slot (je, je - 1) is skipped
    const int skip_i = (je < npiv && is_second(secw, je)) ? je : -1;
    double lv0[kTileR];
#pragma unroll
    for (int j = 0; j < kTileR; j++) lv0[j] = lvn[j];
    if (b + 1 < ntile) prefetch(b + 1);
    for (int i = max(je, rb) + tid; i < re; i += kSbThreads) {
      double acc[kSbRhs];
#pragma unroll
      for (int r = 0; r < kSbRhs; r++) acc[r] = 0.0;
      const double* li = L + i + (size_t)ldl * jb;
      // the row's tile entries are all loaded before the products, so that
      // their HBM latency is paid once per row, not once per column (the
      // first row's were loaded a tile ahead)
      const bool first = i < max(je, rb) + kSbThreads;
      double lv[kTileR];
#pragma unroll
      for (int j = 0; j < kTileR; j++) lv[j] = first ? lv0[j] : (j < nb) ? li[(size_t)ldl * j] : 0.0;
#pragma unroll
      for (int j = 0; j < kTileR; j++) {
        const double l = (i == skip_i && j == nb - 1) ? 0.0 : lv[j];
#pragma unroll
        for (int r = 0; r < kSbRhs; r++)
          if (r < nr) acc[r] = fma(l, tb[j * kSbRhs + r], acc[r]);
      }
#pragma unroll
      for (int r = 0; r < kSbRhs; r++)
        if (r < nr) v[(size_t)r * R + (i - rb)] -= acc[r];
    }
    __syncthreads();
  }
  cl.sync();

  // D^{-1} at the pivots (a 2x2 pair reads its partner, possibly in another
  // CTA), the solution at the pivot variables; the rest is the update vector
  for (int i = rb + tid; i < min(re, npiv); i += kSbThreads) {
    const bool sec = is_second(secw, i);
    const bool first = (i + 1 < npiv) && is_second(secw, i + 1);
    const int var = fv[i];
    const int vi = var >= 0 ? var : -var - 1;
    const double dd = L[i + (size_t)ldl * i];
    int pp = -1;
    double d11 = 0.0, d21 = 0.0, d22 = 0.0;
    if (first) {
      pp = i + 1;
      d11 = dd;
      d21 = L[(i + 1) + (size_t)ldl * i];
      d22 = L[(i + 1) + (size_t)ldl * (i + 1)];
    } else if (sec) {
      pp = i - 1;
      d11 = L[(i - 1) + (size_t)ldl * (i - 1)];
      d21 = L[i + (size_t)ldl * (i - 1)];
      d22 = dd;
    }
    const double* vp = nullptr;
    if (pp >= 0) {
      const int op = pp / R;
      vp = at_rank(cl, v, op, rank) + (pp - op * R);
    }
    for (int r = 0; r < nr; r++) {
      const double t = v[(size_t)r * R + (i - rb)];
      double y;
      if (first) {
        const double u = vp[(size_t)r * R];
        y = (d22 * t - d21 * u) / (d11 * d22 - d21 * d21);
      } else if (sec) {
        const double u = vp[(size_t)r * R];
        y = (d11 * t - d21 * u) / (d11 * d22 - d21 * d21);
      } else {
        y = t / dd;
      }
      x[(size_t)ldx * (r0rhs + r) + vi] = y;
    }
  }
  double* uo = upool + s.u_off[node] * nrhs + (size_t)r0rhs * m;
  for (int i = max(rb, npiv) + tid; i < re; i += kSbThreads)
    for (int r = 0; r < nr; r++) uo[(size_t)r * m + (i - npiv)] = v[(size_t)r * R + (i - rb)];
  cl.sync();  // partners read through DSMEM are done
}

__global__ void __launch_bounds__(kSbThreads)
    backward_big_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                        double* __restrict__ x, int ldx, int r0rhs, int nr) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int node = nodes[blockIdx.x / kSbCL];
  extern __shared__ __align__(16) double sm[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = s.f[node];
  const int npiv = s.npiv[node];
  const int* fv = s.ivars + s.fv_off[node];
  const double* L = s.dpool + s.L_off[node];
  const int ldl = s.L_ld[node];
  const int R = sb_rows(f);
  const int rb = rank * R;
  const int re = min(f, rb + R);
  double* v = sm;                     // [nr][R]
  double* part = v + (size_t)nr * R;  // [2][kSbCL][kTileR][kSbRhs]
  unsigned* secw = reinterpret_cast<unsigned*>(part + 2 * kSbCL * kTileR * kSbRhs);

  for (int q = tid; q < nr * R; q += kSbThreads) {
    const int r = q / R;
    const int i = rb + (q - r * R);
    double val = 0.0;
    if (i < re) {
      const int var = fv[i];
      val = x[(size_t)ldx * (r0rhs + r) + (var >= 0 ? var : -var - 1)];
    }
    v[q] = val;
  }
  if (warp == 0) second_row_bits(fv, npiv, secw, lane);
  __syncthreads();

  const int ntile = (npiv + kTileR - 1) / kTileR;
  for (int b = ntile - 1; b >= 0; b--) {
    const int jb = b * kTileR;
    const int je = min(jb + kTileR, npiv);
    const int nb = je - jb;
    const int ob = jb / R;
    const int par = b & 1;
    const int skip_i = (je < npiv && is_second(secw, je)) ? je : -1;
    // partial sums of L(i, j) x(i) over own rows i >= je: warp w takes
    // columns jb + 4w .. jb + 4w + 3
    {
      const int j0 = 4 * warp;
      double acc[4][kSbRhs];
#pragma unroll
      for (int c = 0; c < 4; c++)
#pragma unroll
        for (int r = 0; r < kSbRhs; r++) acc[c][r] = 0.0;
      // four rows per lane pass: their 16 HBM loads are in flight together
      for (int ib = max(je, rb) + lane; ib < re; ib += 128) {
        double lv[4][4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int i = ib + 32 * u;
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int j = j0 + c;
            lv[u][c] = (i < re && j < nb && !(i == skip_i && j == nb - 1))
                           ? L[i + (size_t)ldl * (jb + j)]
                           : 0.0;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int i = ib + 32 * u;
          if (i >= re) continue;
#pragma unroll
          for (int r = 0; r < kSbRhs; r++) {
            const double xr = (r < nr) ? v[(size_t)r * R + (i - rb)] : 0.0;
#pragma unroll
            for (int c = 0; c < 4; c++) acc[c][r] = fma(lv[u][c], xr, acc[c][r]);
          }
        }
      }
      __syncwarp();
#pragma unroll
      for (int c = 0; c < 4; c++)
#pragma unroll
        for (int r = 0; r < kSbRhs; r++) {
          double a = acc[c][r];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
          acc[c][r] = a;
        }
      // lane (c, r) pushes one value to the tile's owner
      const int c = lane / kSbRhs;
      const int r = lane - c * kSbRhs;
      double val = 0.0;
#pragma unroll
      for (int cc = 0; cc < 4; cc++)
#pragma unroll
        for (int rr = 0; rr < kSbRhs; rr++)
          if (cc == c && rr == r) val = acc[cc][rr];
      double* dst = at_rank(cl, part, ob, rank);
      dst[((size_t)(par * kSbCL + rank) * kTileR + (j0 + c)) * kSbRhs + r] = val;
    }
    cl.sync();  // partials at the owner
    if (rank == ob && warp == 0) {
      const bool mine = lane < nb;
      const unsigned sec = secw[jb >> 5];
      double Lcol[kTileR];
      const double* col = L + (size_t)ldl * (jb + lane) + jb;
#pragma unroll
      for (int q = 0; q < kTileR; q++) Lcol[q] = (mine && q < nb) ? col[q] : 0.0;
      double vr[kSbRhs];
      double* vrow = v + (jb - rb) + lane;
#pragma unroll
      for (int r = 0; r < kSbRhs; r++) {
        double a = 0.0;
        if (mine && r < nr) {
          a = vrow[(size_t)r * R];
          for (int c = 0; c < kSbCL; c++)
            a -= part[((size_t)(par * kSbCL + c) * kTileR + lane) * kSbRhs + r];
        }
        vr[r] = a;
      }
#pragma unroll
      for (int jj = kTileR - 1; jj >= 0; jj--) {
        if (jj < nb) {
          const bool upd = lane < jj && !(((sec >> jj) & 1u) && lane == jj - 1);
#pragma unroll
          for (int r = 0; r < kSbRhs; r++) {
            const double vj = __shfl_sync(0xffffffffu, vr[r], jj);
            if (upd && r < nr) vr[r] = fma(-Lcol[jj], vj, vr[r]);
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kSbRhs; r++)
        if (mine && r < nr) vrow[(size_t)r * R] = vr[r];
    }
    __syncthreads();
  }
  for (int q = tid; q < nr * R; q += kSbThreads) {
    const int r = q / R;
    const int i = rb + (q - r * R);
    if (i < min(re, npiv)) {
      const int var = fv[i];
      x[(size_t)ldx * (r0rhs + r) + (var >= 0 ? var : -var - 1)] = v[q];
    }
  }
  cl.sync();
}

size_t fwd_big_smem(int fmax) {
  const size_t R = (size_t)sb_rows(fmax);
  return (R * kSbRhs + kTileR * kSbRhs) * sizeof(double) + (size_t)fmax * sizeof(int) +
         ((size_t)fmax / 32 + 2) * sizeof(unsigned) + 16;
}

size_t bwd_big_smem(int fmax) {
  const size_t R = (size_t)sb_rows(fmax);
  return (R * kSbRhs + (size_t)2 * kSbCL * kTileR * kSbRhs) * sizeof(double) +
         ((size_t)fmax / 32 + 2) * sizeof(unsigned) + 16;
}

cudaLaunchConfig_t cluster_cfg(int count, size_t smem, cudaStream_t st, cudaLaunchAttribute* a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(count * kSbCL, 1, 1);
  cfg.blockDim = dim3(kSbThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = kSbCL;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  cfg.attrs = a;
  cfg.numAttrs = 1;
  return cfg;
}

constexpr size_t kSbSmemMax = 200 * 1024;

}  // namespace

bool solve_big_fits(int f) {
  return fwd_big_smem(f) <= kSbSmemMax && bwd_big_smem(f) <= kSbSmemMax;
}

cudaError_t configure_solve_big_kernels() {
  cudaError_t e = cudaFuncSetAttribute(forward_big_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSbSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(forward_big_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed,
                           1);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(backward_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kSbSmemMax);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(backward_big_kernel,
                              cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

int launch_forward_big(const DevPlan& p, const DevState& s, const int* nodes, int count,
                       double* x, int ldx, int nrhs, double* upool, int fmax,
                       cudaStream_t stream, cudaError_t* err) {
  if (count <= 0) return 0;
  int n = 0;
  for (int r0 = 0; r0 < nrhs; r0 += kSbRhs) {
    const int nr = (nrhs - r0 < kSbRhs) ? nrhs - r0 : kSbRhs;
    cudaLaunchAttribute a[1];
    cudaLaunchConfig_t cfg = cluster_cfg(count, fwd_big_smem(fmax), stream, a);
    const cudaError_t e =
        cudaLaunchKernelEx(&cfg, forward_big_kernel, p, s, nodes, x, ldx, nrhs, r0, nr, upool);
    if (e != cudaSuccess) {
      *err = e;
      return n;
    }
    n++;
  }
  return n;
}

int launch_backward_big(const DevPlan& p, const DevState& s, const int* nodes, int count,
                        double* x, int ldx, int nrhs, int fmax, cudaStream_t stream,
                        cudaError_t* err) {
  if (count <= 0) return 0;
  int n = 0;
  for (int r0 = 0; r0 < nrhs; r0 += kSbRhs) {
    const int nr = (nrhs - r0 < kSbRhs) ? nrhs - r0 : kSbRhs;
    cudaLaunchAttribute a[1];
    cudaLaunchConfig_t cfg = cluster_cfg(count, bwd_big_smem(fmax), stream, a);
    const cudaError_t e =
        cudaLaunchKernelEx(&cfg, backward_big_kernel, p, s, nodes, x, ldx, r0, nr);
    if (e != cudaSuccess) {
      *err = e;
      return n;
    }
    n++;
  }
  return n;
}

}  // namespace b200ldl
