// umma.cuh -- BF16 tensor-core GEMM on sm_100a (tcgen05 / TMEM) with
// pluggable epilogues, for the surrogate network.
//
//   C[M x N] = A[M x K] * B[N x K]^T      A, B bf16, K-major (row-major with
//                                          K contiguous), FP32 accumulate
//
// One CTA (4 warps) owns a 128-row tile of C and all N <= 512 columns.  K is
// consumed in 64-wide chunks: the warps stage the A and B chunks in shared
// memory in the canonical no-swizzle K-major layout (8-row x 16-byte core
// matrices; the two 16-byte K halves of an MMA sit LBO bytes apart, 8-row
// groups SBO = 128 bytes apart), one elected thread issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N <= 256 per instruction,
// K = 16) into a TMEM accumulator and commits to an mbarrier, and the
// epilogue reads the accumulator back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = rows of the tile).  Every wait is bounded: on timeout
// the kernel records an error code and releases its TMEM.
#ifndef POFD_UMMA_CUH
#define POFD_UMMA_CUH

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pofd {
namespace umma {

constexpr int kRows = 128;      // M tile (TMEM lanes)
constexpr int kKChunk = 64;     // K per shared-memory stage
constexpr int kMaxN = 512;      // TMEM columns
constexpr int kThreads = 128;
constexpr unsigned kSpinLimit = 1u << 24;  // bounded mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100 layout: start >> 4 in [0,14),
// LBO >> 4 in [16,30), SBO >> 4 in [32,46), version 1 in [46,48),
// layout type 0 = no swizzle in [61,64)).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo,
                                              uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  return d;
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major,
// N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc,
                                         uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct GemmShape {
  int M, N, K;                       // N multiple of 16 (<= 512), K multiple of 16
  const __nv_bfloat16* A; int lda;   // [M][K]
  const __nv_bfloat16* B; int ldb;   // [N][K]
  int* err;                          // error code (0 = ok)
};

__host__ __device__ constexpr int tmem_cols(int n) {
  return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512;
}

// Shared memory bytes of the main loop for N columns.
__host__ __device__ constexpr size_t smem_bytes(int n) {
  return static_cast<size_t>(kRows + n) * kKChunk * 2 + 64;
}

// Stage a [R x kw] bf16 chunk (rows r0.., columns k0..k0+kw) into the
// canonical layout: 16-byte cell (r, kg) at kg * R * 16 + r * 16.  Rows at or
// beyond nrows are zero.
__device__ __forceinline__ void stage_chunk(const __nv_bfloat16* __restrict__ g, int ld,
                                            int r0, int nrows, int R, int k0, int kw,
                                            uint8_t* s) {
  const int kgs = kw >> 3;
  for (int c = threadIdx.x; c < R * kgs; c += kThreads) {
    const int r = c % R, kg = c / R;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r0 + r < nrows)
      v = *reinterpret_cast<const uint4*>(g + static_cast<size_t>(r0 + r) * ld + k0 + kg * 8);
    *reinterpret_cast<uint4*>(s + (static_cast<size_t>(kg) * R + r) * 16) = v;
  }
}

// Main loop: accumulates the CTA's 128 x N tile into TMEM and returns the
// TMEM base address (or 0xFFFFFFFF after a timeout, err set).  Must be called
// by all kThreads threads; smem points at smem_bytes(N) dynamic bytes.
__device__ __forceinline__ uint32_t mainloop(const GemmShape& g, int m0, uint8_t* smem,
                                             uint32_t* tslot, uint64_t* bar, int* abort) {
  uint8_t* sA = smem;
  uint8_t* sB = smem + kRows * kKChunk * 2;
  const int ncols = tmem_cols(g.N);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (threadIdx.x < 32) tmem_alloc(tslot, ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const int nchunks = (g.K + kKChunk - 1) / kKChunk;
  for (int kc = 0; kc < nchunks; ++kc) {
    const int k0 = kc * kKChunk;
    const int kw = min(kKChunk, g.K - k0);
    stage_chunk(g.A, g.lda, m0, g.M, kRows, k0, kw, sA);
    stage_chunk(g.B, g.ldb, 0, g.N, g.N, k0, kw, sB);
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      for (int s = 0; s < kw / 16; ++s) {
        const uint32_t a = smem_u32(sA) + static_cast<uint32_t>(2 * s * kRows * 16);
        const uint64_t ad = smem_desc(a, kRows * 16, 128);
        for (int n0 = 0; n0 < g.N; n0 += 256) {
          const int nn = min(256, g.N - n0);
          const uint32_t b = smem_u32(sB) + static_cast<uint32_t>((2 * s * g.N + n0) * 16);
          const uint64_t bd = smem_desc(b, static_cast<uint32_t>(g.N) * 16, 128);
          mma_bf16(tbase + static_cast<uint32_t>(n0), ad, bd, instr_desc(kRows, nn),
                   (kc > 0 || s > 0) ? 1u : 0u);
        }
      }
      mma_commit(bar);
    }
    // all threads wait for the MMAs before the chunk buffers are reused
    const bool ok = mbar_wait(bar, static_cast<uint32_t>(kc & 1));
    if (!ok) atomicExch(abort, 1);
    __syncthreads();
    if (*abort) break;
  }
  tc_fence_after();
  if (*abort) {
    if (threadIdx.x == 0 && g.err) atomicCAS(g.err, 0, 1);
    return 0xFFFFFFFFu;
  }
  return tbase;
}

__device__ __forceinline__ void release(uint32_t* tslot, int ncols) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  __syncwarp();
  if (threadIdx.x < 32) tmem_dealloc(*tslot, static_cast<uint32_t>(ncols));
}

}  // namespace umma
}  // namespace pofd
#endif
