// umma.cuh -- BF16 tensor-core GEMM on sm_100a (TMA + tcgen05 / TMEM) with
// pluggable epilogues, for the surrogate network.
//
//   C[M x N] = A[M x K] * B[N x K]^T      A, B bf16, K-major (row-major with
//                                          K contiguous), FP32 accumulate
//
// One CTA (4 warps) owns a 128 x ntile tile of C (ntile <= 128 divides N).
// K is consumed in 64-wide chunks through a 3-stage shared-memory ring: one
// thread (warp 0) issues TMA tile loads (cp.async.bulk.tensor, 3-D tensor
// maps that view a row-major [rows][K] matrix as [K/8][rows][8], so the
// copy lands directly in the canonical no-swizzle K-major layout: 8-row x
// 16-byte core matrices, K halves LBO = rows * 16 bytes apart, 8-row groups
// SBO = 128 bytes apart), signalling a "full" mbarrier with the byte count;
// one thread (warp 1) waits on it and issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = ntile, K = 16) into a
// TMEM accumulator, committing to the stage's "empty" mbarrier so the
// producer can refill it; the last commit releases the epilogue, which reads
// the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 =
// rows of the tile).  Every wait is bounded: on timeout the kernel records
// an error code, stops issuing work and releases its TMEM.
#ifndef POFD_UMMA_CUH
#define POFD_UMMA_CUH

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pofd {
namespace umma {

constexpr int kRows = 128;      // M tile (TMEM lanes)
constexpr int kKChunk = 64;     // K per shared-memory stage
constexpr int kStages = 3;      // shared-memory ring depth
constexpr int kMaxNTile = 128;  // N per CTA
constexpr int kMaxN = 512;      // N per GEMM
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

// Bounded wait for the phase with the given parity (at most `limit`
// try_wait rounds); false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          unsigned limit = kSpinLimit) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < limit; ++it) {
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

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes),
               "r"(smem_u32(bar))
               : "memory");
}

// 3-D tiled TMA load into this CTA's shared memory, completing on bar.
__device__ __forceinline__ void tma_load3(void* dst, const CUtensorMap* map, int c0, int c1,
                                          int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
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
  int M, N, K;   // N multiple of 16 (<= 512), K multiple of 16
  int ntile;     // N per CTA (16, 32, 64 or 128; divides N)
  int* err;      // error code (0 = ok)
};

__host__ __device__ constexpr int tmem_cols(int n) {
  return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512;
}

__host__ __device__ constexpr int pick_ntile(int n) {
  return (n % 128 == 0) ? 128 : (n % 64 == 0) ? 64 : (n % 32 == 0) ? 32 : 16;
}

__host__ __device__ constexpr size_t stage_bytes(int ntile) {
  return static_cast<size_t>(kRows + ntile) * kKChunk * 2;
}

// Dynamic shared memory of the main loop (ring + 1 KB alignment slack).
__host__ __device__ constexpr size_t smem_bytes(int ntile) {
  return kStages * stage_bytes(ntile) + 1024;
}

struct Barriers {
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t done;
  uint32_t tslot;
  int abort;
};

// Main loop: accumulates the CTA's 128 x ntile tile (rows m0.., columns
// n0..) into TMEM and returns the TMEM base address, or 0xFFFFFFFF after a
// timeout (err set).  Called by all kThreads threads.
__device__ __forceinline__ uint32_t mainloop(const GemmShape& g, const CUtensorMap* tmA,
                                             const CUtensorMap* tmB, int m0, int n0,
                                             uint8_t* smem_raw, Barriers& bs) {
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~static_cast<uintptr_t>(1023));
  const int nt = g.ntile;
  const size_t sbytes = stage_bytes(nt);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&bs.full[s], 1);
      mbar_init(&bs.empty[s], 1);
    }
    mbar_init(&bs.done, 1);
    bs.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) tmem_alloc(&bs.tslot, static_cast<uint32_t>(tmem_cols(nt)));
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = bs.tslot;
  const int nk = (g.K + kKChunk - 1) / kKChunk;
  const uint32_t tx = static_cast<uint32_t>(sbytes);
  if (warp == 0 && lane == 0) {
    // producer: TMA loads into the ring
    for (int kc = 0; kc < nk; ++kc) {
      const int s = kc % kStages;
      if (kc >= kStages && !mbar_wait(&bs.empty[s], static_cast<uint32_t>((kc / kStages - 1) & 1))) {
        atomicExch(&bs.abort, 1);
        break;
      }
      uint8_t* sa = smem + s * sbytes;
      mbar_expect_tx(&bs.full[s], tx);
      tma_load3(sa, tmA, 0, m0, kc * (kKChunk / 8), &bs.full[s]);
      tma_load3(sa + kRows * kKChunk * 2, tmB, 0, n0, kc * (kKChunk / 8), &bs.full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = instr_desc(kRows, nt);
    bool ok = true;
    for (int kc = 0; kc < nk; ++kc) {
      const int s = kc % kStages;
      if (!mbar_wait(&bs.full[s], static_cast<uint32_t>((kc / kStages) & 1))) {
        atomicExch(&bs.abort, 1);
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(smem + s * sbytes);
      const uint32_t sb = sa + static_cast<uint32_t>(kRows * kKChunk * 2);
      const int kw = min(kKChunk, g.K - kc * kKChunk);
      for (int q = 0; q < kw / 16; ++q) {
        const uint64_t ad = smem_desc(sa + static_cast<uint32_t>(2 * q * kRows * 16), kRows * 16, 128);
        const uint64_t bd = smem_desc(sb + static_cast<uint32_t>(2 * q * nt * 16),
                                      static_cast<uint32_t>(nt) * 16, 128);
        mma_bf16(tbase, ad, bd, idesc, (kc > 0 || q > 0) ? 1u : 0u);
      }
      mma_commit(&bs.empty[s]);
    }
    if (ok) mma_commit(&bs.done);
  }
  __syncwarp();
  const bool fin = mbar_wait(&bs.done, 0u);
  if (!fin) atomicExch(&bs.abort, 1);
  tc_fence_after();
  __syncthreads();
  if (bs.abort) {
    if (threadIdx.x == 0 && g.err) atomicCAS(g.err, 0, 1);
    return 0xFFFFFFFFu;
  }
  return tbase;
}

__device__ __forceinline__ void release(Barriers& bs, int ntile) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  __syncwarp();
  if (threadIdx.x < 32) tmem_dealloc(bs.tslot, static_cast<uint32_t>(tmem_cols(ntile)));
}

}  // namespace umma
}  // namespace pofd
#endif
