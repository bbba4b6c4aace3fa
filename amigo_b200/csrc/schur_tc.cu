// Dense Schur-complement update on the tensor cores, C -= A B^T (optionally
// its lower triangle only), FP64 in and out, the products as 3xTF32 on
// tcgen05 with the accumulator in tensor memory (umma.cuh). The mixed-
// precision factorization applies the same tile update to the contribution
// blocks of big fronts; this entry point exposes it on its own.
#include <cuda_runtime.h>

#include "../../include/b200ldl.h"
#include "umma.cuh"

namespace {

using namespace b200ldl;

__device__ int g_schur_tc_status;

__global__ void __launch_bounds__(128)
    schur_tc_kernel(int m, int n, int k, const double* __restrict__ A, int lda,
                    const double* __restrict__ B, int ldb, double* C, int ldc, int lower) {
  extern __shared__ __align__(1024) float ops[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x;
  if ((tid >> 5) == 0) umma::tmem_alloc_128(&tmem_slot);
  if (tid == 0) umma::mbar_init(&mbar);
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t tmem = tmem_slot;
  uint32_t phase = 0;
  const long long i0 = (long long)blockIdx.x * umma::kTileM;
  const long long j0 = (long long)blockIdx.y * umma::kTileN;
  // tiles wholly above the diagonal have nothing to update (the same in
  // every thread)
  if (!(lower && j0 > i0 + umma::kTileM - 1)) {
    const int mr = (int)(m - i0 < umma::kTileM ? m - i0 : umma::kTileM);
    const int nc = (int)(n - j0 < umma::kTileN ? n - j0 : umma::kTileN);
    const int st = umma::tile_update(C, ldc, A, lda, B, ldb, i0, j0, mr, nc, k, lower != 0, ops,
                                     &mbar, &phase, tmem);
    if (st && tid == 0) atomicExch(&g_schur_tc_status, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if ((tid >> 5) == 0) umma::tmem_free_128(tmem);
}

constexpr size_t kSmem = umma::kSmemFloats * sizeof(float);

}  // namespace

extern "C" int b200ldl_schur_update_tc(int m, int n, int k, const double* a, int lda,
                                       const double* b, int ldb, double* c, int ldc, int lower,
                                       void* stream) {
  if (m < 0 || n < 0 || k < 0) return -1;
  if (m == 0 || n == 0 || k == 0) return 0;
  if (!a || !b || !c || lda < m || ldb < n || ldc < m) return -1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaFuncSetAttribute(schur_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmem);
  if (e != cudaSuccess) return -3;
  const int zero = 0;
  e = cudaMemcpyToSymbolAsync(g_schur_tc_status, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return -3;
  dim3 grid((m + umma::kTileM - 1) / umma::kTileM, (n + umma::kTileN - 1) / umma::kTileN);
  schur_tc_kernel<<<grid, 128, kSmem, st>>>(m, n, k, a, lda, b, ldb, c, ldc, lower);
  e = cudaGetLastError();
  if (e != cudaSuccess) return -3;
  int status = 0;
  e = cudaMemcpyFromSymbolAsync(&status, g_schur_tc_status, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                st);
  if (e != cudaSuccess) return -3;
  if (cudaStreamSynchronize(st) != cudaSuccess) return -3;
  return status ? 1 : 0;
}
