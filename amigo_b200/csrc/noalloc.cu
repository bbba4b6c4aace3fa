// Allocation-free dense symmetric-indefinite factor + solve.
//
// Who needs this: callers that must not allocate device memory once they are
// running. Examples are a real-time controller that re-solves the same small
// KKT system every few milliseconds, where an allocation has unbounded
// latency and may synchronize the device, and a plugin inside an
// application whose framework has already reserved nearly all device memory
// for its own pool, so a library cudaMalloc can fail. Such callers hand over
// inputs and outputs only.
//
// This entry point is a variant of the front factorization for a front
// without contribution rows (Bunch-Kaufman 1x1/2x2 pivoting, as the reference
// uses LAPACK dsytrf there). The working matrix lives in a file-scope device
// array of fixed size instead of the handle's pool, so nothing is allocated:
// no cudaMalloc, no cudaFree, no allocating library routine.
//
// Limits and sharing: n <= kNoAllocMaxN (512). Every GPU that loads the
// library keeps this array (2 MiB) until the process exits. All calls on a
// device share it and it keeps the previous call's contents; each call
// rewrites every entry it reads before reading it. Calls whose kernels
// overlap on the GPU (different streams, no ordering between them) race on
// the array and give wrong results; order them on one stream. The first
// call on each device looks up the array's device address (with that device
// current); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>

#include "../../include/b200ldl.h"

namespace {

constexpr int kNoAllocMaxN = 512;
constexpr int kNoAllocThreads = 512;
constexpr int kNoAllocWarps = kNoAllocThreads / 32;

// n x n working matrix, then n ints of front variables (as doubles' room)
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxN * kNoAllocMaxN +
                                                          kNoAllocMaxN];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {nullptr};

__device__ __forceinline__ void keep_larger(double& bv, int& bi, double v, int i) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

struct NaRed {
  double v[kNoAllocWarps];
  int i[kNoAllocWarps];
  double m[kNoAllocWarps];
};

__device__ void na_reduce(NaRed& r, double& bv, int& bi, double& cm) {
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
  for (int q = 1; q < kNoAllocWarps; q++) {
    keep_larger(bv, bi, r.v[q], r.i[q]);
    cm = fmax(cm, r.m[q]);
  }
  __syncthreads();
}

__device__ void na_swap(double* F, int n, int* fv, int a, int b) {
  const int n1 = a, n2 = b - a - 1, n3 = n - b - 1;
  const int total = n1 + 1 + n2 + n3;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    double *p, *q;
    if (t < n1) {
      p = &F[a + (size_t)n * t];
      q = &F[b + (size_t)n * t];
    } else if (t == n1) {
      p = &F[a + (size_t)n * a];
      q = &F[b + (size_t)n * b];
    } else if (t < n1 + 1 + n2) {
      const int j = a + 1 + (t - n1 - 1);
      p = &F[j + (size_t)n * a];
      q = &F[b + (size_t)n * j];
    } else {
      const int j = b + 1 + (t - n1 - 1 - n2);
      p = &F[j + (size_t)n * a];
      q = &F[j + (size_t)n * b];
    }
    const double tmp = *p;
    *p = *q;
    *q = tmp;
  }
  if (threadIdx.x == 0) {
    const int t = fv[a];
    fv[a] = fv[b];
    fv[b] = t;
  }
}

__global__ void __launch_bounds__(kNoAllocThreads)
    noalloc_dense_kernel(int n, const double* __restrict__ a, int lda, double* __restrict__ b,
                         int ldb, int nrhs, int* __restrict__ inertia, double* scratch) {
  __shared__ NaRed red;
  __shared__ double t[kNoAllocMaxN];
  double* F = scratch;                                  // n x n, ld n
  int* fv = (int*)(scratch + (size_t)kNoAllocMaxN * kNoAllocMaxN);  // [n]
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

  // every entry read below is written here first (lower triangle + fv)
  for (int j = warp; j < n; j += kNoAllocWarps)
    for (int i = j + lane; i < n; i += 32) F[i + (size_t)n * j] = a[i + (size_t)lda * j];
  for (int i = tid; i < n; i += blockDim.x) fv[i] = i;
  __syncthreads();

  const double alpha = (1.0 + 4.1231056256176605) / 8.0;  // (1 + sqrt(17)) / 8
  int npos = 0, nneg = 0;
  for (int k = 0; k < n;) {
    double bv = -1.0, cm = 0.0;
    int bi = INT_MAX;
    for (int i = k + 1 + tid; i < n; i += blockDim.x) keep_larger(bv, bi, fabs(F[i + (size_t)n * k]), i);
    na_reduce(red, bv, bi, cm);
    const double akk = F[k + (size_t)n * k];
    const double absakk = fabs(akk);
    const double colmax = (k + 1 < n) ? bv : 0.0;
    const int imax = (k + 1 < n) ? (bi < n ? bi : k + 1) : k;
    int step = 1, kp = k;
    bool zero = false;
    if (fmax(absakk, colmax) == 0.0) {
      zero = true;
    } else if (absakk < alpha * colmax) {
      double rv = -1.0, rmax = 0.0;
      int ri = INT_MAX;
      const int n1 = imax - k, n2 = n - imax - 1;
      for (int q = tid; q < n1 + n2; q += blockDim.x) {
        const double x = (q < n1) ? fabs(F[imax + (size_t)n * (k + q)])
                                  : fabs(F[(imax + 1 + (q - n1)) + (size_t)n * imax]);
        rmax = fmax(rmax, x);
      }
      na_reduce(red, rv, ri, rmax);
      const double absaii = fabs(F[imax + (size_t)n * imax]);
      if (absakk >= alpha * colmax * (colmax / rmax)) {
        step = 1;
      } else if (absaii >= alpha * rmax) {
        step = 1;
        kp = imax;
      } else {
        step = 2;
        kp = imax;
      }
    }
    const int ksrc = k + step - 1;
    if (kp != ksrc) {
      na_swap(F, n, fv, ksrc, kp);
      __syncthreads();
    }
    double* c0 = F + (size_t)n * k;
    if (step == 1) {
      const double d = c0[k];
      const double dinv = (zero || d == 0.0) ? 0.0 : 1.0 / d;
      for (int j = k + 1 + warp; j < n; j += kNoAllocWarps) {
        const double lj = c0[j] * dinv;
        double* cj = F + (size_t)n * j;
        for (int i = j + lane; i < n; i += 32) cj[i] -= c0[i] * lj;
      }
      __syncthreads();
      for (int i = k + 1 + tid; i < n; i += blockDim.x) c0[i] *= dinv;
      if (d >= 0.0)
        npos++;
      else
        nneg++;
    } else {
      double* c1 = c0 + n;
      const double d11 = c0[k], d21 = c0[k + 1], d22 = c1[k + 1];
      const double det = d11 * d22 - d21 * d21;
      const double di = 1.0 / det;
      const double i00 = d22 * di, i01 = -d21 * di, i11 = d11 * di;
      for (int j = k + 2 + warp; j < n; j += kNoAllocWarps) {
        const double x0 = c0[j], x1 = c1[j];
        const double l0 = x0 * i00 + x1 * i01, l1 = x0 * i01 + x1 * i11;
        double* cj = F + (size_t)n * j;
        for (int i = j + lane; i < n; i += 32) cj[i] -= c0[i] * l0 + c1[i] * l1;
      }
      __syncthreads();
      for (int i = k + 2 + tid; i < n; i += blockDim.x) {
        const double x0 = c0[i], x1 = c1[i];
        c0[i] = x0 * i00 + x1 * i01;
        c1[i] = x0 * i01 + x1 * i11;
      }
      if (tid == 0) {
        fv[k] = -(fv[k] + 1);
        fv[k + 1] = -(fv[k + 1] + 1);
      }
      if (det >= 0.0) {
        if (d11 >= 0.0)
          npos += 2;
        else
          nneg += 2;
      } else {
        npos++;
        nneg++;
      }
    }
    __syncthreads();
    k += step;
  }
  if (inertia && tid == 0) {
    inertia[0] = npos;
    inertia[1] = nneg;
  }

  // solve with L D L^T for each right-hand side
  for (int r = 0; r < nrhs; r++) {
    double* br = b + (size_t)ldb * r;
    for (int p = tid; p < n; p += blockDim.x) {
      const int v = fv[p];
      t[p] = br[v >= 0 ? v : -v - 1];
    }
    __syncthreads();
    for (int j = 0; j < n;) {
      const double* c0 = F + (size_t)n * j;
      if (fv[j] >= 0) {
        const double tj = t[j];
        for (int i = j + 1 + tid; i < n; i += blockDim.x) t[i] -= c0[i] * tj;
        __syncthreads();
        j += 1;
      } else {
        const double* c1 = c0 + n;
        const double t0 = t[j], t1 = t[j + 1];
        for (int i = j + 2 + tid; i < n; i += blockDim.x) t[i] -= c0[i] * t0 + c1[i] * t1;
        __syncthreads();
        j += 2;
      }
    }
    if (tid == 0) {
      for (int j = 0; j < n;) {
        const double* c0 = F + (size_t)n * j;
        if (fv[j] >= 0) {
          t[j] = c0[j] != 0.0 ? t[j] / c0[j] : 0.0;
          j += 1;
        } else {
          const double d11 = c0[j], d21 = c0[j + 1], d22 = c0[n + j + 1];
          const double inv = 1.0 / (d11 * d22 - d21 * d21);
          const double x0 = t[j], x1 = t[j + 1];
          t[j] = inv * (d22 * x0 - d21 * x1);
          t[j + 1] = inv * (d11 * x1 - d21 * x0);
          j += 2;
        }
      }
    }
    __syncthreads();
    for (int j = n - 1; j >= 0;) {
      if (fv[j] >= 0) {
        const double* c0 = F + (size_t)n * j;
        double m = 0.0;
        for (int i = j + 1 + tid; i < n; i += blockDim.x) m += c0[i] * t[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m += __shfl_down_sync(0xffffffffu, m, o);
        if (lane == 0) red.m[warp] = m;
        __syncthreads();
        if (tid == 0) {
          double s = 0.0;
          for (int q = 0; q < kNoAllocWarps; q++) s += red.m[q];
          t[j] -= s;
        }
        __syncthreads();
        j -= 1;
      } else {
        const double* c0 = F + (size_t)n * (j - 1);
        const double* c1 = c0 + n;
        double a0 = 0.0, a1 = 0.0;
        for (int i = j + 1 + tid; i < n; i += blockDim.x) {
          a0 += c0[i] * t[i];
          a1 += c1[i] * t[i];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          a0 += __shfl_down_sync(0xffffffffu, a0, o);
          a1 += __shfl_down_sync(0xffffffffu, a1, o);
        }
        if (lane == 0) {
          red.m[warp] = a0;
          red.v[warp] = a1;
        }
        __syncthreads();
        if (tid == 0) {
          double s0 = 0.0, s1 = 0.0;
          for (int q = 0; q < kNoAllocWarps; q++) {
            s0 += red.m[q];
            s1 += red.v[q];
          }
          t[j - 1] -= s0;
          t[j] -= s1;
        }
        __syncthreads();
        j -= 2;
      }
    }
    for (int p = tid; p < n; p += blockDim.x) {
      const int v = fv[p];
      br[v >= 0 ? v : -v - 1] = t[p];
    }
    __syncthreads();
  }
}

// device address of the scratch array for the current device (looked up once)
double* scratch_for_current_device(int* status) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *status = -3;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      *status = -3;
      return nullptr;
    }
    g_scratch_addr[dev] = static_cast<double*>(ptr);
  }
  *status = 0;
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int b200ldl_dense_solve_noalloc(int n, const double* a, int lda, double* b, int ldb,
                                           int nrhs, int* inertia, void* stream) {
  if (n < 0 || nrhs < 0) return -1;
  if (n > kNoAllocMaxN) return -6;  // larger than the fixed scratch array
  if (n == 0) return 0;
  if (!a || lda < n || (nrhs > 0 && (!b || ldb < n))) return -1;
  int st = 0;
  double* scratch = scratch_for_current_device(&st);
  if (st != 0) return st;
  noalloc_dense_kernel<<<1, kNoAllocThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, a, lda, b, ldb, nrhs, inertia, scratch);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
