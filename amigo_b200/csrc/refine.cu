// FP64 residuals and iterative refinement against the CSR KKT matrix.
//
// berr = ||b - K x||_inf / (||K||_inf ||x||_inf + ||b||_inf), per right-hand
// side, with K the full symmetric CSR plus the diagonal vector (what the
// factorization assembles, sparse_ldl.h:1099-1104). The reference has no
// refinement; its plugin's comment asks for one (newton_direction.py:6-8).
#include <algorithm>
#include <cuda_runtime.h>

#include "ldl_internal.h"

namespace b200ldl {

namespace {

constexpr int kMaxR = 8;

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(addr), __double_as_longlong(v));
}

// r = b - (K + diag) x for nr columns; one warp per row
__global__ void residual_kernel(int n, const int* __restrict__ rowp, const int* __restrict__ cols,
                                const double* __restrict__ vals, const double* __restrict__ diag,
                                const double* __restrict__ x, int ldx,
                                const double* __restrict__ b, int ldb, double* __restrict__ r,
                                int ldr, int nr) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  double acc[kMaxR];
#pragma unroll
  for (int c = 0; c < kMaxR; c++) acc[c] = 0.0;
  for (int e = rowp[row] + lane; e < rowp[row + 1]; e += 32) {
    const double v = vals[e];
    const int j = cols[e];
#pragma unroll
    for (int c = 0; c < kMaxR; c++)
      if (c < nr) acc[c] = fma(v, x[(size_t)ldx * c + j], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < kMaxR; c++) {
    if (c < nr) {
      double a = acc[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) {
        if (diag) a = fma(diag[row], x[(size_t)ldx * c + row], a);
        r[(size_t)ldr * c + row] = b[(size_t)ldb * c + row] - a;
      }
    }
  }
}

// out[c] = max_i |v[i + ld c]|  (out zeroed by the caller)
__global__ void colmax_kernel(int n, const double* __restrict__ v, int ld, int nr, double* out) {
  for (int c = 0; c < nr; c++) {
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      m = fmax(m, fabs(v[(size_t)ld * c + i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out + c, m);
  }
}

// ||K + diag||_inf
__global__ void infnorm_kernel(int n, const int* __restrict__ rowp, const int* __restrict__ cols,
                               const double* __restrict__ vals, const double* __restrict__ diag,
                               double* out) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double s = 0.0;
  if (row < n) {
    const double dg = diag ? diag[row] : 0.0;
    for (int e = rowp[row] + lane; e < rowp[row + 1]; e += 32)
      s += fabs(cols[e] == row ? vals[e] + dg : vals[e]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0 && row < n) atomic_max_nonneg(out, s);
}

__global__ void axpy_kernel(int n, int nr, const double* __restrict__ d, int ldd,
                            double* __restrict__ x, int ldx) {
  const size_t total = (size_t)n * nr;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / n);
    const int i = (int)(t - (size_t)c * n);
    x[(size_t)ldx * c + i] += d[(size_t)ldd * c + i];
  }
}

__global__ void copy_cols_kernel(int n, int nr, const double* __restrict__ src, int lds,
                                 double* __restrict__ dst, int ldd) {
  const size_t total = (size_t)n * nr;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / n);
    const int i = (int)(t - (size_t)c * n);
    dst[(size_t)ldd * c + i] = src[(size_t)lds * c + i];
  }
}

// Derivative of a scalar loss with respect to the CSR values and the
// diagonal, given the solution x of K x = b and the adjoint lam = K^{-1} g
// (g = dloss/dx): dloss/dK(i,j) = -sum_r lam(i,r) x(j,r), one warp per row.
__global__ void value_gradient_kernel(int n, const int* __restrict__ rowp,
                                      const int* __restrict__ cols,
                                      const double* __restrict__ lam, int ldl,
                                      const double* __restrict__ x, int ldx, int nr,
                                      double* __restrict__ gvals, double* __restrict__ gdiag) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  double li[kMaxR];
#pragma unroll
  for (int c = 0; c < kMaxR; c++) li[c] = (c < nr) ? lam[(size_t)ldl * c + row] : 0.0;
  for (int e = rowp[row] + lane; e < rowp[row + 1]; e += 32) {
    const int j = cols[e];
    double g = 0.0;
#pragma unroll
    for (int c = 0; c < kMaxR; c++)
      if (c < nr) g = fma(li[c], x[(size_t)ldx * c + j], g);
    gvals[e] = -g;
  }
  if (gdiag && lane == 0) {
    double g = 0.0;
#pragma unroll
    for (int c = 0; c < kMaxR; c++)
      if (c < nr) g = fma(li[c], x[(size_t)ldx * c + row], g);
    gdiag[row] = -g;
  }
}

// The regularized diagonal of one inertia-correction attempt:
// out[i] = diag[i] (+ dx on primal rows when dx > 0) (- dc on constraint
// rows when dc > 0), the additions in that order, as
// InertiaCorrector._compute_perturbation makes them
// (amigo/algorithm/solvers/inertia_correction.py:293-306).
__global__ void perturb_diag_kernel(int n, const double* __restrict__ diag,
                                    const unsigned char* __restrict__ cls, double dx, double dc,
                                    double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = diag ? diag[i] : 0.0;
    const unsigned char c = cls[i];
    if (dx > 0.0 && (c & 1)) v += dx;
    if (dc > 0.0 && (c & 2)) v += -dc;
    out[i] = v;
  }
}

}  // namespace

void launch_perturb_diag(int n, const double* diag, const unsigned char* cls, double dx,
                         double dc, double* out, cudaStream_t st) {
  const int threads = 256;
  const int blocks = std::max(1, std::min((n + threads - 1) / threads, 148 * 8));
  perturb_diag_kernel<<<blocks, threads, 0, st>>>(n, diag, cls, dx, dc, out);
}

void launch_value_gradient(int n, const int* rowp, const int* cols, const double* lam, int ldl,
                           const double* x, int ldx, int nr, double* gvals, double* gdiag,
                           cudaStream_t st) {
  const int threads = 256;
  const int blocks = (int)(((long long)n * 32 + threads - 1) / threads);
  value_gradient_kernel<<<blocks, threads, 0, st>>>(n, rowp, cols, lam, ldl, x, ldx, nr, gvals,
                                                    gdiag);
}

int refine_max_rhs() { return kMaxR; }

void launch_residual(int n, const int* rowp, const int* cols, const double* vals,
                     const double* diag, const double* x, int ldx, const double* b, int ldb,
                     double* r, int ldr, int nr, cudaStream_t st) {
  const int threads = 256;
  const int blocks = (int)(((long long)n * 32 + threads - 1) / threads);
  residual_kernel<<<blocks, threads, 0, st>>>(n, rowp, cols, vals, diag, x, ldx, b, ldb, r, ldr,
                                              nr);
}

void launch_colmax(int n, const double* v, int ld, int nr, double* out, cudaStream_t st) {
  colmax_kernel<<<296, 256, 0, st>>>(n, v, ld, nr, out);
}

void launch_infnorm(int n, const int* rowp, const int* cols, const double* vals,
                    const double* diag, double* out, cudaStream_t st) {
  const int threads = 256;
  const int blocks = (int)(((long long)n * 32 + threads - 1) / threads);
  infnorm_kernel<<<blocks, threads, 0, st>>>(n, rowp, cols, vals, diag, out);
}

void launch_axpy(int n, int nr, const double* d, int ldd, double* x, int ldx, cudaStream_t st) {
  axpy_kernel<<<592, 256, 0, st>>>(n, nr, d, ldd, x, ldx);
}

void launch_copy_cols(int n, int nr, const double* src, int lds, double* dst, int ldd,
                      cudaStream_t st) {
  copy_cols_kernel<<<592, 256, 0, st>>>(n, nr, src, lds, dst, ldd);
}

}  // namespace b200ldl
