// Blackwell (sm_100a) tensor-core tile update for the Schur complement:
//
//   C(i, j) -= sum_c A(i, c) B(j, c)      for the 128 x 128 tile at (i0, j0)
//
// with A, B and C in FP64 in global memory (column-major) and the products
// on the 5th-generation tensor cores (tcgen05.mma, kind::tf32) with the
// accumulator in tensor memory (TMEM). Each FP64 operand is split into two
// TF32 parts, hi = tf32(x) and lo = tf32(x - hi), and the tile is
// accumulated as A_hi B_hi + A_hi B_lo + A_lo B_hi (the 3xTF32 scheme), so
// that the products carry about 21 significant bits before the FP32
// accumulation; the FP32 sum is subtracted from the FP64 C.
//
// Shared-memory operand layout: K-major, no swizzle, in 8-row x 16-byte core
// matrices (the canonical UMMA K-major layout): element (m, k) of a 128 x 32
// operand is at float index (k / 4) * 512 + (m / 8) * 32 + (m % 8) * 4 + k % 4,
// so the 8-row groups are 128 bytes apart (stride byte offset) and the two
// 16-byte halves of one instruction's K = 8 are 2048 bytes apart (leading
// byte offset). One instruction covers M = 128, N = 128, K = 8.
//
// Protocol: one CTA of 128 or 256 threads. The caller allocates 128 TMEM
// columns (tmem_alloc_128) and initialises one mbarrier (mbar_init) once;
// every call waits for its own MMAs through the mbarrier with a bounded spin
// (status != 0 when the bound is reached; nothing is then left in flight
// that the caller could not wait for with the same bound).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace b200ldl {
namespace umma {

constexpr int kTileM = 128;
constexpr int kTileN = 128;
constexpr int kChunkK = 32;                       // K staged per round
constexpr int kOpFloats = kTileM * kChunkK;       // one staged operand
constexpr int kSmemFloats = 4 * kOpFloats;        // A_hi, A_lo, B_hi, B_lo (64 KB)
constexpr long long kSpinLimit = 1ll << 26;       // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, K-major without swizzle (Blackwell
// version field = 1): start address, leading and stride byte offsets, all in
// 16-byte units.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1u) << 46;
  return d;
}

// instruction descriptor: D in FP32, A and B in TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
  asm volatile("fence.mbarrier_init.release.cluster;" ::);
}

// wait for the phase with parity `parity` to complete; false after the bound
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kSpinLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity));
    if (done) return true;
  }
  return false;
}

// one warp: 128 TMEM columns, their base address written to *dst (shared)
__device__ __forceinline__ void tmem_alloc_128(uint32_t* dst) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(
      smem_u32(dst)));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

// the same warp that allocated
__device__ __forceinline__ void tmem_free_128(uint32_t base) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(base));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
        "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
      smem_u32(bar)));
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::);
#pragma unroll
  for (int q = 0; q < 32; q++) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ int op_index(int m, int k) {
  return (k >> 2) * 512 + (m >> 3) * 32 + (m & 7) * 4 + (k & 3);
}

// C(i0 + r, j0 + c) -= sum_{q < kk} A(i0 + r, q) B(j0 + c, q) for r < mrows, c < ncols,
// and only where lower(i0 + r, j0 + c) holds (i >= j when lower_only).
// A(i, q) = A[i + lda q], B(j, q) = B[j + ldb q], C(i, j) = C[i + ldc j]. The
// whole CTA calls it (blockDim.x = 128 or 256). ops: kSmemFloats floats of
// shared memory aligned to 128 bytes. *phase tracks the mbarrier's parity.
// Returns 0, or 1 if an MMA did not complete within the spin bound.
__device__ __noinline__ static int tile_update(double* C, long long ldc, const double* A, long long lda,
                           const double* B, long long ldb, long long i0, long long j0, int mrows,
                           int ncols, int kk, bool lower_only, float* ops, uint64_t* mbar,
                           uint32_t* phase, uint32_t tmem) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  float* a_hi = ops;
  float* a_lo = ops + kOpFloats;
  float* b_hi = ops + 2 * kOpFloats;
  float* b_lo = ops + 3 * kOpFloats;
  constexpr uint32_t kIdesc = idesc_tf32(kTileM, kTileN);
  int status = 0;
  for (int k0 = 0; k0 < kk; k0 += kChunkK) {
    const int kc = min(kChunkK, kk - k0);
    // stage this K chunk: FP64 -> (tf32 hi, tf32 lo), zero beyond the tile
    for (int e = tid; e < kTileM * kChunkK; e += nthr) {
      const int m = e % kTileM, q = e / kTileM;
      double va = 0.0, vb = 0.0;
      if (q < kc) {
        if (m < mrows) va = A[(i0 + m) + lda * (k0 + q)];
        if (m < ncols) vb = B[(j0 + m) + ldb * (k0 + q)];
      }
      const float ha = to_tf32(static_cast<float>(va));
      const float hb = to_tf32(static_cast<float>(vb));
      const int o = op_index(m, q);
      a_hi[o] = ha;
      a_lo[o] = to_tf32(static_cast<float>(va - static_cast<double>(ha)));
      b_hi[o] = hb;
      b_lo[o] = to_tf32(static_cast<float>(vb - static_cast<double>(hb)));
    }
    // generic-proxy stores become visible to the tensor cores' async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::);
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::);
      const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
      const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
      for (int s = 0; s < kChunkK / 8; s++) {
        const uint32_t off = s * 2 * 2048;  // two 16-byte K halves per instruction
        const uint32_t first = (k0 == 0 && s == 0) ? 0u : 1u;
        mma_tf32(tmem, smem_desc(ah + off, 2048, 128), smem_desc(bh + off, 2048, 128), kIdesc,
                 first);
        mma_tf32(tmem, smem_desc(ah + off, 2048, 128), smem_desc(bl + off, 2048, 128), kIdesc, 1u);
        mma_tf32(tmem, smem_desc(al + off, 2048, 128), smem_desc(bh + off, 2048, 128), kIdesc, 1u);
      }
      mma_commit(mbar);
    }
    // the operands may be overwritten only after the MMAs that read them
    const bool ok = mbar_wait(mbar, *phase);
    *phase ^= 1u;
    if (__syncthreads_or(!ok)) {  // the same verdict in every thread
      status = 1;
      break;
    }
  }
  if (status || kk <= 0) {
    __syncthreads();
    return status;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (the tile's rows),
  // warps 4..7 (when present) the second half of the columns
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int row = (warp & 3) * 32 + lane;
  const int nquarters = (nthr >= 256) ? 2 : 4;  // 32-column loads per warp
  const int cbase = (nthr >= 256) ? (warp >> 2) * 64 : 0;
  for (int qq = 0; qq < nquarters; qq++) {
    const int c0 = cbase + qq * 32;
    float v[32];
    tmem_ld32(tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16) + c0, v);
    if (row < mrows) {
      const long long i = i0 + row;
#pragma unroll
      for (int q = 0; q < 32; q++) {
        const int c = c0 + q;
        const long long j = j0 + c;
        if (c < ncols && (!lower_only || i >= j)) C[i + ldc * j] -= static_cast<double>(v[q]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  return 0;
}

}  // namespace umma
}  // namespace b200ldl
