// Fronts resident in a thread-block cluster's distributed shared memory.
//
// A front of size f (145 <= f <= kClusterFrontMax) is held entirely on chip:
// its lower triangle is split row-cyclically over the CL CTAs of a cluster
// (row i on CTA i % CL, rows stored packed, row-major), so every CTA holds
// about f^2 / (2 CL) doubles and the work per CTA is balanced. The front is
// assembled straight into DSMEM (CSR entries, the diagonal vector, the
// children's contribution blocks), factored right-looking with the
// reference's threshold 1x1 / 2x2 / delay tests (SparseLDL::
// factor_front_matrix_block, include/sparse_ldl.h:1316-1553; Bunch-Kaufman
// when there are no contribution rows, as LAPACK dsytrf there), and only the
// factor columns and the contribution block leave the chip.
//
// Per accepted 1x1 pivot: every CTA reduces the pivot column over its rows,
// pushes its partial into every CTA's slot through DSMEM, one cluster
// barrier, every thread reduces the slots (identical decisions everywhere),
// each CTA gathers the pivot column from its owners and applies the rank-1
// update to its own rows. No global memory is touched inside the loop.
#include <cooperative_groups.h>

#include <climits>

#include "ldl_internal.h"

namespace cg = cooperative_groups;

namespace b200ldl {

namespace {

constexpr int kCfThreads = 256;
constexpr int kCfWarps = kCfThreads / 32;

struct CfPart {
  double v;
  int i;
  int pad;
  double m;
  double x;
  double y;
};

struct CfRed {
  double v[kCfWarps];
  int i[kCfWarps];
  double m[kCfWarps];
};

__device__ __forceinline__ void keep_larger(double& bv, int& bi, double v, int i) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

__device__ void cf_reduce(CfRed& r, double& bv, int& bi, double& cm) {
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
  for (int q = 1; q < kCfWarps; q++) {
    keep_larger(bv, bi, r.v[q], r.i[q]);
    cm = fmax(cm, r.m[q]);
  }
  __syncthreads();
}

// offset of row i inside its owner's packed storage (owner i % CL, local
// row q = i / CL): q (r + 1) + CL q (q - 1) / 2
template <int CL>
__device__ __forceinline__ long long row_off(int i) {
  const long long q = i / CL;
  const long long r = i - q * CL;
  return q * (r + 1) + (long long)CL * q * (q - 1) / 2;
}

template <int CL>
__device__ __forceinline__ double* row_ptr(cg::cluster_group& cl, double* tri, int rank, int i) {
  const int o = i % CL;
  double* base = (o == rank) ? tri : cl.map_shared_rank(tri, o);
  return base + row_off<CL>(i);
}

// packed length of CTA `rank`'s rows for a front of size f
template <int CL>
__host__ __device__ __forceinline__ long long tri_len(int f, int rank) {
  const long long Q = (f - rank + CL - 1) / CL;
  return Q * (rank + 1) + (long long)CL * Q * (Q - 1) / 2;
}

template <int CL>
__device__ __forceinline__ void push(cg::cluster_group& cl, CfPart* slots, int rank,
                                     const CfPart& p) {
  if (threadIdx.x < CL) *cl.map_shared_rank(slots + rank, (unsigned)threadIdx.x) = p;
}

// symmetric interchange of rows/columns a < b of the distributed triangle;
// every element pair is exchanged by exactly one thread of the cluster
template <int CL>
__device__ void tri_swap(cg::cluster_group& cl, double* tri, int rank, int f, int a, int b,
                         int* fv, int* orig) {
  const int n1 = a;
  const int n2 = b - a - 1;
  const int n3 = f - b - 1;
  const int total = n1 + 1 + n2 + n3;
  double* ra = row_ptr<CL>(cl, tri, rank, a);
  double* rb = row_ptr<CL>(cl, tri, rank, b);
  for (int t = rank * blockDim.x + threadIdx.x; t < total; t += CL * blockDim.x) {
    double *p, *q;
    if (t < n1) {
      p = ra + t;
      q = rb + t;
    } else if (t == n1) {
      p = ra + a;
      q = rb + b;
    } else if (t < n1 + 1 + n2) {
      const int j = a + 1 + (t - n1 - 1);
      p = row_ptr<CL>(cl, tri, rank, j) + a;
      q = rb + j;
    } else {
      const int j = b + 1 + (t - n1 - 1 - n2);
      double* rj = row_ptr<CL>(cl, tri, rank, j);
      p = rj + a;
      q = rj + b;
    }
    const double tmp = *p;
    *p = *q;
    *q = tmp;
  }
  if (rank == 0 && threadIdx.x == 0) {
    int t = fv[a];
    fv[a] = fv[b];
    fv[b] = t;
    t = orig[a];
    orig[a] = orig[b];
    orig[b] = t;
  }
}

enum : int { kDelay = 0, kOne = 1, kTwo = 2, kNeedRow = 3, kZero = 4 };

template <int CL>
__global__ void __launch_bounds__(kCfThreads)
    cluster_front_kernel(DevPlan p, DevState s, const int* __restrict__ list,
                         const double* __restrict__ vals, const double* __restrict__ diag,
                         FactorParams prm) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  BigFront* B = s.big + list[blockIdx.x / CL];
  extern __shared__ __align__(16) double sm[];
  // slotA is double-buffered by iteration parity: a CTA may push the next
  // column partial before a slower CTA has finished reading this one
  __shared__ CfPart slotA[2][CL], slotB[CL];
  __shared__ CfRed red;

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
  double* tri = sm;
  const long long tl = tri_len<CL>(f, rank);
  double* col0 = tri + tl;
  double* col1 = col0 + f;
  int* fv = s.ivars + B->ioff;
  int* orig = fv + f;
  // own rows: i = rank + q * CL for q < Q
  const int Q = (f - rank + CL - 1) / CL;

  // ---- assembly straight into distributed shared memory
  for (long long t = tid; t < tl; t += kCfThreads) tri[t] = 0.0;
  cl.sync();
  {
    const int64_t e0 = p.scat_ptr[node];
    const int64_t e1 = p.scat_ptr[node + 1];
    for (int64_t e = e0 + gt; e < e1; e += CL * kCfThreads) {
      int r = p.scat_row[e];
      if (r >= ns) r += nd_in;
      double* dst = row_ptr<CL>(cl, tri, rank, r) + p.scat_col[e];
      *dst += vals[p.scat_csr[e]];
    }
  }
  cl.sync();
  if (diag) {
    const int v0 = p.var_ptr[node];
    for (int j = gt; j < ns; j += CL * kCfThreads) {
      double* dst = row_ptr<CL>(cl, tri, rank, j) + j;
      *dst += diag[p.node_to_var[v0 + j]];
    }
    cl.sync();
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
        for (int r1 = r2 + lane; r1 < m; r1 += 32) {
          int p1;
          if (r1 < nd) {
            p1 = off + r1;
          } else {
            p1 = cm[r1 - nd];
            if (p1 >= ns) p1 += nd_in;
          }
          const int hi = p1 >= p2 ? p1 : p2;
          const int lo = p1 >= p2 ? p2 : p1;
          double* dst = row_ptr<CL>(cl, tri, rank, hi) + lo;
          *dst += col[r1];
        }
      }
      cl.sync();
      off += nd;
    }
  }

  // ---- partial factorization of the candidates [0, ncand)
  const double alpha_bk = (1.0 + 4.1231056256176605) / 8.0;  // (1 + sqrt(17)) / 8
  int k = 0;
  int ncand = fs;
  int npos = 0, nneg = 0;
  double flops = 0.0;
  int pend = 0, pc = 0;
  double pd0 = 0.0, pd1 = 0.0, pd2 = 0.0;

  int it = 0;
  while (k < ncand) {
    CfPart* sA = slotA[it & 1];
    it++;
    // pivot column k over own rows i > k
    double bv = -1.0, cmx = 0.0;
    int bi = INT_MAX;
    {
      const int q0 = (k + 1 - rank + CL - 1) / CL > 0 ? (k + 1 - rank + CL - 1) / CL : 0;
      for (int q = q0 + tid; q < Q; q += kCfThreads) {
        const int i = rank + q * CL;
        const double a = fabs(tri[row_off<CL>(i) + k]);
        if (i < ncand)
          keep_larger(bv, bi, a, i);
        else
          cmx = fmax(cmx, a);
      }
    }
    cf_reduce(red, bv, bi, cmx);
    {
      CfPart P;
      P.v = bv;
      P.i = bi;
      P.pad = 0;
      P.m = cmx;
      P.x = (k % CL == rank) ? tri[row_off<CL>(k) + k] : 0.0;
      P.y = 0.0;
      push<CL>(cl, sA, rank, P);
    }
    cl.sync();  // B1

    double gv = -1.0, gm = 0.0;
    int gi = INT_MAX;
#pragma unroll
    for (int r = 0; r < CL; r++) {
      keep_larger(gv, gi, sA[r].v, sA[r].i);
      gm = fmax(gm, sA[r].m);
    }
    const double wkk = sA[k % CL].x;
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
      // column imax below it, and row imax from k to imax (on its owner)
      double rm = 0.0, dummy = -1.0;
      int di = INT_MAX;
      const int q0 = (imax + 1 - rank + CL - 1) / CL > 0 ? (imax + 1 - rank + CL - 1) / CL : 0;
      for (int q = q0 + tid; q < Q; q += kCfThreads) {
        const int i = rank + q * CL;
        rm = fmax(rm, fabs(tri[row_off<CL>(i) + imax]));
      }
      const bool own = (imax % CL == rank);
      if (own) {
        const double* ri = tri + row_off<CL>(imax);
        for (int j = k + tid; j < imax; j += kCfThreads) rm = fmax(rm, fabs(ri[j]));
      }
      cf_reduce(red, dummy, di, rm);
      {
        CfPart P;
        P.v = 0.0;
        P.i = 0;
        P.pad = 0;
        P.m = rm;
        P.x = own ? tri[row_off<CL>(imax) + imax] : 0.0;
        P.y = own ? tri[row_off<CL>(imax) + k] : 0.0;
        push<CL>(cl, slotB, rank, P);
      }
      cl.sync();  // B2
      double rmax = 0.0;
#pragma unroll
      for (int r = 0; r < CL; r++) rmax = fmax(rmax, slotB[r].m);
      wii = slotB[imax % CL].x;
      wik = slotB[imax % CL].y;
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
      if (k < ncand - 1) {
        tri_swap<CL>(cl, tri, rank, f, k, ncand - 1, fv, orig);
        cl.sync();  // B3
      }
      ncand -= 1;
      continue;
    }
    const int nstep = (step == kTwo) ? 2 : 1;
    const int ksrc = k + nstep - 1;
    if (kpiv != ksrc) {
      tri_swap<CL>(cl, tri, rank, f, ksrc, kpiv, fv, orig);
      cl.sync();  // B3
    }

    // deferred scaling of the previous pivot column(s) (every CTA gathered
    // them before the barrier above; swaps since then commute with it)
    if (pend) {
      const int from = pc + pend;
      const int q0 = (from - rank + CL - 1) / CL > 0 ? (from - rank + CL - 1) / CL : 0;
      for (int q = q0 + tid; q < Q; q += kCfThreads) {
        double* ri = tri + row_off<CL>(rank + q * CL);
        if (pend == 1) {
          ri[pc] *= pd0;
        } else {
          const double a = ri[pc], b = ri[pc + 1];
          ri[pc] = a * pd0 + b * pd1;
          ri[pc + 1] = a * pd1 + b * pd2;
        }
      }
    }
    // gather the pivot column(s) below the pivot block from their owners
    const int k1 = k + nstep;  // first row below the pivot block
    for (int j = k1 + tid; j < f; j += kCfThreads) {
      const double* rj = row_ptr<CL>(cl, tri, rank, j);
      col0[j] = rj[k];
      if (nstep == 2) col1[j] = rj[k + 1];
    }
    __syncthreads();
    // rank-1 / rank-2 update of own rows i >= k1, columns j in [k1, i]
    double dinv = 0.0, i00 = 0.0, i01 = 0.0, i11 = 0.0;
    double d11 = 0.0, d21 = 0.0, d22 = 0.0;
    if (nstep == 1) {
      const double d = (kpiv != k) ? wii : wkk;
      dinv = (step == kZero || (root && d == 0.0)) ? 0.0 : 1.0 / d;
      if (rank == 0 && tid == 0) {
        if (d >= 0.0)
          npos++;
        else
          nneg++;
        const double r = (double)(f - k - 1);
        flops += r * (r + 1.0) + r;
      }
    } else {
      d11 = wkk;
      d21 = wik;
      d22 = wii;
      const double det = d11 * d22 - d21 * d21;
      const double detinv = 1.0 / det;
      i00 = d22 * detinv;
      i01 = -d21 * detinv;
      i11 = d11 * detinv;
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
        const double r = (double)(f - k - 2);
        flops += 2.0 * r * (r + 1.0) + 6.0 * r;
      }
    }
    {
      const int q0 = (k1 - rank + CL - 1) / CL > 0 ? (k1 - rank + CL - 1) / CL : 0;
      for (int q = q0 + warp; q < Q; q += kCfWarps) {
        const int i = rank + q * CL;
        double* ri = tri + row_off<CL>(i);
        if (nstep == 1) {
          const double li = ri[k] * dinv;
          for (int j = k1 + lane; j <= i; j += 32) ri[j] = fma(-li, col0[j], ri[j]);
        } else {
          const double a = ri[k], b = ri[k + 1];
          const double l0 = a * i00 + b * i01;
          const double l1 = a * i01 + b * i11;
          for (int j = k1 + lane; j <= i; j += 32)
            ri[j] = fma(-l0, col0[j], fma(-l1, col1[j], ri[j]));
        }
      }
    }
    pend = nstep;
    pc = k;
    if (nstep == 1) {
      pd0 = dinv;
    } else {
      pd0 = i00;
      pd1 = i01;
      pd2 = i11;
    }
    k += nstep;
    // the next step reads only this CTA's own rows before its barrier
    __syncthreads();
  }
  cl.sync();  // all gathers of the last pivot column are done
  if (pend) {
    const int from = pc + pend;
    const int q0 = (from - rank + CL - 1) / CL > 0 ? (from - rank + CL - 1) / CL : 0;
    for (int q = q0 + tid; q < Q; q += kCfThreads) {
      double* ri = tri + row_off<CL>(rank + q * CL);
      if (pend == 1) {
        ri[pc] *= pd0;
      } else {
        const double a = ri[pc], b = ri[pc + 1];
        ri[pc] = a * pd0 + b * pd1;
        ri[pc + 1] = a * pd1 + b * pd2;
      }
    }
  }
  __syncthreads();

  // ---- write the factor columns (f x npiv, ld f) and the contribution
  // block ((f-npiv)^2, ld f-npiv) into the front's pool region
  const int npiv = k;
  const int m = f - npiv;
  double* Lg = s.dpool + B->doff;
  double* Cg = Lg + (size_t)f * npiv;
  for (int q = warp; q < Q; q += kCfWarps) {
    const int i = rank + q * CL;
    const double* ri = tri + row_off<CL>(i);
    const int jl = i + 1 < npiv ? i + 1 : npiv;
    for (int j = lane; j < jl; j += 32) Lg[i + (size_t)f * j] = ri[j];
    if (i >= npiv) {
      const int pp = i - npiv;
      for (int qq = lane; qq <= pp; qq += 32) Cg[pp + (size_t)m * qq] = ri[npiv + qq];
    }
  }
  if (rank == 0 && tid == 0) {
    B->k = npiv;
    B->ncand = ncand;
    B->kw = 0;
    B->npos += npos;
    B->nneg += nneg;
    B->flops += flops;
    B->pad = 1;  // packed output layout: CB after L with ld m
    B->state = 2;
  }
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
  long long worst = 0;
  for (int r = 0; r < CL; r++) {
    const long long t = tri_len<CL>(fmax, r);
    if (t > worst) worst = t;
  }
  return (size_t)(worst + 2LL * fmax) * sizeof(double);
}

constexpr size_t kCfSmemMax = 224 * 1024;

}  // namespace

// Largest front each cluster size can hold (shared memory per CTA).
int cluster_front_limit(int cl_index) {
  static int lim[5] = {0, 0, 0, 0, 0};
  if (lim[0] == 0) {
    int f;
    for (f = kSmemFrontMax; cf_smem<1>(f + 1) <= kCfSmemMax; f++) {}
    lim[0] = f;
    for (f = lim[0]; cf_smem<2>(f + 1) <= kCfSmemMax; f++) {}
    lim[1] = f;
    for (f = lim[1]; cf_smem<4>(f + 1) <= kCfSmemMax; f++) {}
    lim[2] = f;
    for (f = lim[2]; cf_smem<8>(f + 1) <= kCfSmemMax; f++) {}
    lim[3] = f;
    for (f = lim[3]; cf_smem<16>(f + 1) <= kCfSmemMax; f++) {}
    lim[4] = f;
  }
  return lim[cl_index];
}

cudaError_t configure_cluster_front_kernels() {
  cudaError_t e;
  e = cudaFuncSetAttribute(cluster_front_kernel<1>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCfSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<2>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCfSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<4>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCfSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<8>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCfSmemMax);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_front_kernel<16>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCfSmemMax);
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
