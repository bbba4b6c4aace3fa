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
// scatter-subtracts into the shared solution vector.
#include "ldl_internal.h"

namespace b200ldl {

namespace {

constexpr int kSWarps = kSolveThreads / 32;

__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int q = 0; q < kSWarps; q++) t += red[q];
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(kSolveThreads)
    forward_level_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                         double* __restrict__ x, int ldx, int nrhs,
                         double* __restrict__ upool) {
  extern __shared__ __align__(16) double sm[];
  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x;
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
  double* w = sm;      // pre-pivot order
  double* v = sm + f;  // post-pivot order

  for (int r = 0; r < nrhs; r++) {
    double* xr = x + (size_t)ldx * r;
    const int v0 = p.var_ptr[node];
    for (int t = tid; t < f; t += blockDim.x)
      w[t] = (t < ns) ? xr[p.node_to_var[v0 + t]] : 0.0;
    __syncthreads();
    int off = ns;
    for (int c = kb; c < ke; c++) {
      const int ch = p.kids[c];
      const int nd = s.ndel[ch];
      const int mc = s.f[ch] - s.npiv[ch];
      const double* uc = upool + s.u_off[ch] * nrhs + (size_t)r * mc;
      const int* cm = p.cmap + p.cptr[ch];
      for (int t = tid; t < mc; t += blockDim.x) {
        int q;
        if (t < nd) {
          q = off + t;
        } else {
          q = cm[t - nd];
          if (q >= ns) q += nd_in;
        }
        w[q] += uc[t];
      }
      __syncthreads();
      off += nd;
    }
    for (int t = tid; t < f; t += blockDim.x) v[t] = (t < fs) ? w[orig[t]] : w[t];
    __syncthreads();

    for (int j = 0; j < npiv;) {
      if (fv[j] >= 0) {
        const double vj = v[j];
        const double* lj = L + (size_t)ldl * j;
        for (int i = j + 1 + tid; i < f; i += blockDim.x) v[i] -= lj[i] * vj;
        if (tid == 0) xr[fv[j]] = vj / lj[j];
        __syncthreads();
        j += 1;
      } else {
        const double a = v[j];
        const double b = v[j + 1];
        const double* l0 = L + (size_t)ldl * j;
        const double* l1 = l0 + ldl;
        for (int i = j + 2 + tid; i < f; i += blockDim.x) v[i] -= l0[i] * a + l1[i] * b;
        if (tid == 0) {
          const double d11 = l0[j], d21 = l0[j + 1], d22 = l1[j + 1];
          const double inv = 1.0 / (d11 * d22 - d21 * d21);
          xr[-fv[j] - 1] = inv * (d22 * a - d21 * b);
          xr[-fv[j + 1] - 1] = inv * (d11 * b - d21 * a);
        }
        __syncthreads();
        j += 2;
      }
    }
    double* uo = upool + s.u_off[node] * nrhs + (size_t)r * m;
    for (int t = tid; t < m; t += blockDim.x) uo[t] = v[npiv + t];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSolveThreads)
    backward_level_kernel(DevPlan p, DevState s, const int* __restrict__ nodes,
                          double* __restrict__ x, int ldx, int nrhs) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[kSWarps];
  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int f = s.f[node];
  const int npiv = s.npiv[node];
  const int* fv = s.ivars + s.fv_off[node];
  const double* L = s.dpool + s.L_off[node];
  const int ldl = s.L_ld[node];
  double* v = sm;

  for (int r = 0; r < nrhs; r++) {
    double* xr = x + (size_t)ldx * r;
    for (int t = tid; t < f; t += blockDim.x) {
      const int var = fv[t];
      v[t] = xr[var >= 0 ? var : -var - 1];
    }
    __syncthreads();
    // t1 -= L21^T x2, one warp per pivot column
    for (int j = warp; j < npiv; j += kSWarps) {
      const double* lj = L + (size_t)ldl * j;
      double acc = 0.0;
      for (int i = npiv + lane; i < f; i += 32) acc += lj[i] * v[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0) v[j] -= acc;
    }
    __syncthreads();
    // L11^T back substitution
    for (int j = npiv - 1; j >= 0;) {
      if (fv[j] >= 0) {
        const double* lj = L + (size_t)ldl * j;
        double acc = 0.0;
        for (int i = j + 1 + tid; i < npiv; i += blockDim.x) acc += lj[i] * v[i];
        acc = block_sum(acc, red);
        if (tid == 0) v[j] -= acc;
        __syncthreads();
        j -= 1;
      } else {
        const double* l0 = L + (size_t)ldl * (j - 1);
        const double* l1 = l0 + ldl;
        double a0 = 0.0, a1 = 0.0;
        for (int i = j + 1 + tid; i < npiv; i += blockDim.x) {
          a0 += l0[i] * v[i];
          a1 += l1[i] * v[i];
        }
        a0 = block_sum(a0, red);
        a1 = block_sum(a1, red);
        if (tid == 0) {
          v[j - 1] -= a0;
          v[j] -= a1;
        }
        __syncthreads();
        j -= 2;
      }
    }
    for (int t = tid; t < npiv; t += blockDim.x) {
      const int var = fv[t];
      xr[var >= 0 ? var : -var - 1] = v[t];
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t configure_solve_kernels() {
  const int bytes = 2 * kSolveSmemFront * (int)sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(forward_level_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(backward_level_kernel,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

void launch_forward_level(const DevPlan& p, const DevState& s, const int* level_nodes,
                          int count, double* x, int ldx, int nrhs, double* upool,
                          int fmax, cudaStream_t stream) {
  if (count <= 0) return;
  const size_t smem = 2 * (size_t)fmax * sizeof(double);
  forward_level_kernel<<<count, kSolveThreads, smem, stream>>>(p, s, level_nodes, x, ldx,
                                                               nrhs, upool);
}

void launch_backward_level(const DevPlan& p, const DevState& s, const int* level_nodes,
                           int count, double* x, int ldx, int nrhs, int fmax,
                           cudaStream_t stream) {
  if (count <= 0) return;
  const size_t smem = (size_t)fmax * sizeof(double);
  backward_level_kernel<<<count, kSolveThreads, smem, stream>>>(p, s, level_nodes, x, ldx,
                                                                nrhs);
}

}  // namespace b200ldl
