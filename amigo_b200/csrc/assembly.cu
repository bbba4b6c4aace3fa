// KKT assembly: element Hessian blocks into the values of the fixed CSR
// pattern, on the device, deterministically.
//
// The reference zeroes the matrix and, for each component group in turn,
// each element in turn and each column j of the element's Hessian, adds
// the column into CSR row conn[e][j] at the columns conn[e][i], dropping
// entries outside the pattern (OptimizationProblem::hessian,
// include/optimization_problem.h:1063-1088; ComponentGroup::
// add_hessian_kernel, include/component_group.h:144-162; CSRMat::add_row,
// include/csr_matrix.h:554-567). Its GPU backend scatters the same values
// with atomicAdd through a per-entry position table
// (include/cuda/component_group_backend.cuh:157-190), so its sums come in
// an order that changes from run to run.
//
// Here the scatter is inverted once per pattern on the host: for every CSR
// entry, the positions of its contributions in the concatenated element
// blocks, in the reference's sequential order (group, element, j, i). The
// kernel then gathers: one thread per CSR entry, summing from zero in that
// order, so the values are bit-identical to the reference's CPU assembly
// and need no atomics. Traffic: the block values and one 8-byte source
// index per contribution read once, the values written once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/b200ldl.h"
#include "ldl_internal.h"

namespace {

__global__ void csr_gather_kernel(int nnz, const long long* __restrict__ ptr,
                                  const long long* __restrict__ src,
                                  const double* __restrict__ blocks, double* __restrict__ vals) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x) {
    double v = 0.0;
    const long long e = ptr[p + 1];
    for (long long s = ptr[p]; s < e; s++) v += blocks[src[s]];
    vals[p] = v;
  }
}

template <typename T>
struct DevArr {
  T* ptr = nullptr;
  size_t count = 0;
  ~DevArr() {
    if (ptr) cudaFree(ptr);
  }
};

}  // namespace

struct b200ldl_assembly {
  int n = 0, nnz = 0;
  long long nvals = 0;    // block values expected (sum over groups of nelem * ncomp^2)
  long long dropped = 0;  // contributions outside the pattern
  std::vector<long long> ptr, src;  // the plan, host copy
  DevArr<long long> d_ptr, d_src;
  bool uploaded = false;
  std::string last_error;
};

namespace {

int afail(b200ldl_assembly* a, int code, const char* fmt, ...) {
  if (a) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    a->last_error = buf;
  }
  return code;
}

// CSR index of (row, col), or -1 when the pattern has no such entry
inline long long find_entry(const int* rowp, const int* cols, int row, int col) {
  const int* b = cols + rowp[row];
  const int* e = cols + rowp[row + 1];
  const int* it = std::lower_bound(b, e, col);
  return (it != e && *it == col) ? (long long)(it - cols) : -1;
}

int upload(b200ldl_assembly* a) {
  if (a->uploaded) return 0;
  const size_t np = a->ptr.size(), ns = std::max<size_t>(1, a->src.size());
  cudaError_t e = cudaMalloc(&a->d_ptr.ptr, np * sizeof(long long));
  if (e == cudaSuccess) e = cudaMalloc(&a->d_src.ptr, ns * sizeof(long long));
  if (e == cudaSuccess)
    e = cudaMemcpy(a->d_ptr.ptr, a->ptr.data(), np * sizeof(long long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !a->src.empty())
    e = cudaMemcpy(a->d_src.ptr, a->src.data(), a->src.size() * sizeof(long long),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return afail(a, -3, "CUDA error: %s", cudaGetErrorString(e));
  a->uploaded = true;
  return 0;
}

}  // namespace

extern "C" {

int b200ldl_assembly_create(b200ldl_assembly_t* out, int n, const int* rowp, const int* cols,
                            int ngroups, const int* nelems, const int* ncomp, const int* conn) {
  if (!out) return -1;
  *out = nullptr;
  auto* a = new b200ldl_assembly;
  *out = a;
  if (n < 0 || !rowp || (n > 0 && !cols) || ngroups < 0 || (ngroups > 0 && (!nelems || !ncomp)))
    return afail(a, -1, "bad arguments");
  if (rowp[0] != 0) return afail(a, -1, "rowp[0] must be 0");
  for (int r = 0; r < n; r++) {
    if (rowp[r + 1] < rowp[r]) return afail(a, -1, "rowp must be non-decreasing");
    for (int t = rowp[r] + 1; t < rowp[r + 1]; t++)
      if (cols[t] <= cols[t - 1]) return afail(a, -1, "columns of row %d not sorted", r);
  }
  a->n = n;
  a->nnz = rowp[n];
  long long nconn = 0;
  for (int g = 0; g < ngroups; g++) {
    if (nelems[g] < 0 || ncomp[g] < 0) return afail(a, -1, "group %d: negative size", g);
    nconn += (long long)nelems[g] * ncomp[g];
    a->nvals += (long long)nelems[g] * ncomp[g] * ncomp[g];
  }
  if (nconn > 0 && !conn) return afail(a, -1, "conn is null");
  for (long long t = 0; t < nconn; t++)
    if (conn[t] < 0 || conn[t] >= n)
      return afail(a, -1, "connectivity entry %lld = %d out of range", t, conn[t]);
  // pass 1: contributions per CSR entry; pass 2: their sources, in order
  std::vector<long long> cnt((size_t)a->nnz + 1, 0);
  for (int pass = 0; pass < 2; pass++) {
    const int* c = conn;
    long long off = 0;  // first block value of the group
    for (int g = 0; g < ngroups; g++) {
      const int m = ncomp[g];
      for (int e = 0; e < nelems[g]; e++, c += m) {
        for (int j = 0; j < m; j++) {
          for (int i = 0; i < m; i++) {
            const long long p = find_entry(rowp, cols, c[j], c[i]);
            if (p < 0) {
              if (pass == 0) a->dropped++;
              continue;
            }
            if (pass == 0)
              cnt[p + 1]++;
            else
              a->src[cnt[p]++] = off + ((long long)e * m + j) * m + i;
          }
        }
      }
      off += (long long)nelems[g] * m * m;
    }
    if (pass == 0) {
      for (int p = 0; p < a->nnz; p++) cnt[p + 1] += cnt[p];
      a->ptr = cnt;
      a->src.assign((size_t)cnt[a->nnz], 0);
    }
  }
  return 0;
}

int b200ldl_assembly_values(b200ldl_assembly_t a, const double* blocks, double* vals,
                            void* stream) {
  if (!a) return -1;
  if (a->nnz > 0 && !vals) return afail(a, -1, "vals is null");
  if (!a->src.empty() && !blocks) return afail(a, -1, "blocks is null");
  if (a->nnz == 0) return 0;
  const int st = upload(a);
  if (st != 0) return st;
  const int threads = 256;
  const int grid = std::max(1, std::min((a->nnz + threads - 1) / threads, 148 * 8));
  csr_gather_kernel<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(
      a->nnz, a->d_ptr.ptr, a->d_src.ptr, blocks, vals);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return afail(a, -3, "CUDA error: %s", cudaGetErrorString(e));
  return 0;
}

int b200ldl_assembly_info(b200ldl_assembly_t a, long long* out, int nout) {
  if (!a || !out) return -1;
  const long long v[4] = {(long long)a->src.size(), a->dropped, a->nvals, (long long)a->nnz};
  for (int t = 0; t < nout && t < 4; t++) out[t] = v[t];
  return 0;
}

int b200ldl_assembly_plan(b200ldl_assembly_t a, long long* ptr, long long* src) {
  if (!a) return -1;
  if (ptr) std::copy(a->ptr.begin(), a->ptr.end(), ptr);
  if (src) std::copy(a->src.begin(), a->src.end(), src);
  return 0;
}

const char* b200ldl_assembly_last_error(b200ldl_assembly_t a) {
  return a ? a->last_error.c_str() : "null handle";
}

void b200ldl_assembly_destroy(b200ldl_assembly_t a) { delete a; }

}  // extern "C"

namespace b200ldl {

int assembly_device_plan(const ::b200ldl_assembly* a, int* n, int* nnz, const long long** ptr,
                         const long long** src) {
  if (!a || !a->d_ptr.ptr) return -1;
  *n = a->n;
  *nnz = a->nnz;
  *ptr = a->d_ptr.ptr;
  *src = a->d_src.ptr;
  return 0;
}

}  // namespace b200ldl
