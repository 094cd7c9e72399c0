// surrogate.cu -- BF16 tensor-core MLP surrogate of the log-likelihood:
// forward, backward and Adam on sm_100a (tcgen05 / TMEM GEMMs from
// umma.cuh), trained online on exact (theta, logL) pairs.
//
// Network: x (free parameters, standardised, zero-padded to 16 inputs)
//   -> 3 hidden layers of H SiLU units -> 1 output, the standardised
//   logL - running max.  BF16 weights and activations, FP32 accumulation,
//   FP32 master weights and Adam moments.
#include "surrogate.cuh"

#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>

#include "setup.hh"
#include "umma.cuh"

namespace pofd {

namespace {

using bf16 = __nv_bfloat16;
constexpr int NT = umma::kThreads;

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << what << ": " << cudaGetErrorString(e);
    throw Error(e == cudaErrorMemoryAllocation ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}

template <class T>
T* dal(size_t n) {
  void* p = nullptr;
  ck(cudaMalloc(&p, (n ? n : 1) * sizeof(T)), "cudaMalloc");
  ck(cudaMemset(p, 0, (n ? n : 1) * sizeof(T)), "cudaMemset");
  return static_cast<T*>(p);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// ------------------------------------------------------------ GEMM kernels
#define UMMA_PROLOGUE                                                         \
  extern __shared__ __align__(1024) uint8_t smem[];                          \
  __shared__ umma::Barriers bs;                                               \
  const int m0 = blockIdx.x * umma::kRows, n0 = blockIdx.y * g.ntile;         \
  const uint32_t tb = umma::mainloop(g, &tmA, &tmB, m0, n0, smem, bs);        \
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;                 \
  const int row = m0 + warp * 32 + lane;                                      \
  const uint32_t tlane = static_cast<uint32_t>(warp * 32) << 16;

__device__ __forceinline__ void st_bf16x16(bf16* dst, const float* v) {
  __align__(16) bf16 h[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) h[j] = __float2bfloat16_rn(v[j]);
  reinterpret_cast<uint4*>(dst)[0] = reinterpret_cast<const uint4*>(h)[0];
  reinterpret_cast<uint4*>(dst)[1] = reinterpret_cast<const uint4*>(h)[1];
}

// Plain product C = A B^T in FP32 (a checkable entry point of the tensor-core
// main loop).
__global__ void __launch_bounds__(NT) k_gemm_f32(const __grid_constant__ CUtensorMap tmA,
                                                 const __grid_constant__ CUtensorMap tmB,
                                                 umma::GemmShape g, float* __restrict__ C,
                                                 int ldc) {
  UMMA_PROLOGUE
  if (tb != 0xFFFFFFFFu) {
    for (int c0 = 0; c0 < g.ntile; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tb + tlane + c0, v);
      if (row < g.M)
        for (int j = 0; j < 16; ++j) C[static_cast<size_t>(row) * ldc + n0 + c0 + j] = v[j];
    }
  }
  umma::release(bs, g.ntile);
}

// Hidden layer forward: z = A W^T + b, h = silu(z); writes h (bf16,
// [M][ldh]) and, when given, z (fp32 [M][N]) and h^T (bf16 [N][ldt]).  The
// last hidden layer also writes this column tile's part of the network
// output, ypart[tile][row] = h . w4 (+ b4 in tile 0).
__global__ void __launch_bounds__(NT) k_fwd(const __grid_constant__ CUtensorMap tmA,
                                            const __grid_constant__ CUtensorMap tmB,
                                            umma::GemmShape g, const float* __restrict__ bias,
                                            bf16* __restrict__ h, int ldh,
                                            float* __restrict__ z, bf16* __restrict__ ht,
                                            int ldt, const float* __restrict__ w4,
                                            const float* __restrict__ b4,
                                            float* __restrict__ ypart) {
  UMMA_PROLOGUE
  if (tb != 0xFFFFFFFFu) {
    float yacc = 0.0f;
    for (int c0 = 0; c0 < g.ntile; c0 += 16) {
      float v[16], hv[16];
      umma::tmem_ld16(tb + tlane + c0, v);
      const int cb = n0 + c0;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        v[j] += bias[cb + j];
        hv[j] = silu(v[j]);
      }
      if (row < g.M) {
        st_bf16x16(h + static_cast<size_t>(row) * ldh + cb, hv);
        if (z) {
          float4* zp = reinterpret_cast<float4*>(z + static_cast<size_t>(row) * g.N + cb);
#pragma unroll
          for (int q = 0; q < 4; ++q) zp[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const bf16 hb = __float2bfloat16_rn(hv[j]);
          if (ht) ht[static_cast<size_t>(cb + j) * ldt + row] = hb;
          if (w4) yacc += __bfloat162float(hb) * w4[cb + j];
        }
      }
    }
    if (w4 && row < g.M)
      ypart[static_cast<size_t>(blockIdx.y) * g.M + row] = yacc + (blockIdx.y == 0 ? b4[0] : 0.0f);
  }
  umma::release(bs, g.ntile);
}

// Backward through a hidden layer: dh = dZ_next W_next (this GEMM, with B =
// W_next^T), dz = dh * silu'(z); writes dz (bf16 [M][N]) and dz^T (bf16
// [N][ldt]).
__global__ void __launch_bounds__(NT) k_bwd_dx(const __grid_constant__ CUtensorMap tmA,
                                               const __grid_constant__ CUtensorMap tmB,
                                               umma::GemmShape g, const float* __restrict__ z,
                                               bf16* __restrict__ dz, bf16* __restrict__ dzt,
                                               int ldt) {
  UMMA_PROLOGUE
  if (tb != 0xFFFFFFFFu) {
    for (int c0 = 0; c0 < g.ntile; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tb + tlane + c0, v);
      const int cb = n0 + c0;
      if (row < g.M) {
        const float4* zp = reinterpret_cast<const float4*>(z + static_cast<size_t>(row) * g.N + cb);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 zz = zp[q];
          v[4 * q] *= dsilu(zz.x);
          v[4 * q + 1] *= dsilu(zz.y);
          v[4 * q + 2] *= dsilu(zz.z);
          v[4 * q + 3] *= dsilu(zz.w);
        }
        st_bf16x16(dz + static_cast<size_t>(row) * g.N + cb, v);
#pragma unroll
        for (int j = 0; j < 16; ++j)
          dzt[static_cast<size_t>(cb + j) * ldt + row] = __float2bfloat16_rn(v[j]);
      }
    }
  }
  umma::release(bs, g.ntile);
}

struct AdamArgs {
  float lr, b1, b2, eps, bc1, bc2;  // bc = 1 - beta^t
};

// Weight gradient G = dZ^T X (this GEMM: A = dZ^T [Nout x M], B = X^T
// [Nin x M]) followed by the Adam step of W [Nout][Nin]; writes the bf16
// copies W (row-major) and W^T.  grad_out, when given, receives G instead
// of the update (gradient checks).
__global__ void __launch_bounds__(NT) k_wgrad_adam(const __grid_constant__ CUtensorMap tmA,
                                                   const __grid_constant__ CUtensorMap tmB,
                                                   umma::GemmShape g, AdamArgs ad,
                                                   float* __restrict__ W, float* __restrict__ m,
                                                   float* __restrict__ v, bf16* __restrict__ Wb,
                                                   int ldwb, bf16* __restrict__ Wt, int ldwt,
                                                   float* __restrict__ grad_out) {
  UMMA_PROLOGUE
  if (tb != 0xFFFFFFFFu) {
    for (int c0 = 0; c0 < g.ntile; c0 += 16) {
      float gv[16];
      umma::tmem_ld16(tb + tlane + c0, gv);
      const int cb = n0 + c0;
      if (row >= g.M) continue;
      const size_t i0 = static_cast<size_t>(row) * g.N + cb;
      if (grad_out) {
        float4* gp = reinterpret_cast<float4*>(grad_out + i0);
#pragma unroll
        for (int q = 0; q < 4; ++q) gp[q] = make_float4(gv[4 * q], gv[4 * q + 1], gv[4 * q + 2], gv[4 * q + 3]);
        continue;
      }
      float w[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const size_t i = i0 + j;
        const float mm = ad.b1 * m[i] + (1.0f - ad.b1) * gv[j];
        const float vv = ad.b2 * v[i] + (1.0f - ad.b2) * gv[j] * gv[j];
        m[i] = mm;
        v[i] = vv;
        w[j] = W[i] - ad.lr * (mm / ad.bc1) / (sqrtf(vv / ad.bc2) + ad.eps);
        W[i] = w[j];
      }
      st_bf16x16(Wb + static_cast<size_t>(row) * ldwb + cb, w);
      if (Wt)
        for (int j = 0; j < 16; ++j)
          Wt[static_cast<size_t>(cb + j) * ldwt + row] = __float2bfloat16_rn(w[j]);
    }
  }
  umma::release(bs, g.ntile);
}

// ------------------------------------------------------ elementwise kernels
// Whitened, zero-padded bf16 inputs x [Mp][16] and x^T [16][Mp] from theta
// rows (free parameters only): x = W (theta_free - mu), W [16][16] row-major
// (lower triangular); rows >= M are zero.
__global__ void k_pack_inputs(int M, int Mp, const float* __restrict__ theta, int npar,
                              const int* __restrict__ idx, int nin,
                              const float* __restrict__ mu, const float* __restrict__ wm,
                              const int* __restrict__ rows, bf16* __restrict__ x,
                              bf16* __restrict__ xt) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Mp) return;
  const int src = (r < M) ? (rows ? rows[r] : r) : -1;
  float d[Surrogate::kInPad];
#pragma unroll
  for (int j = 0; j < Surrogate::kInPad; ++j)
    d[j] = (src >= 0 && j < nin) ? theta[static_cast<size_t>(src) * npar + idx[j]] - mu[j] : 0.0f;
#pragma unroll
  for (int k = 0; k < Surrogate::kInPad; ++k) {
    float v = 0.0f;
#pragma unroll
    for (int j = 0; j < Surrogate::kInPad; ++j) v = fmaf(wm[k * Surrogate::kInPad + j], d[j], v);
    const bf16 b = __float2bfloat16_rn(v);
    x[static_cast<size_t>(r) * Surrogate::kInPad + k] = b;
    if (xt) xt[static_cast<size_t>(k) * Mp + r] = b;
  }
}

// Network output y = sum of the column-tile parts, the loss and
// dy = 2 (y - t) / M.
__global__ void k_out_loss(int M, int Mp, int ntiles, const float* __restrict__ ypart,
                           const float* __restrict__ t, float* __restrict__ y,
                           float* __restrict__ dy_out, float* __restrict__ loss) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Mp) return;
  float yy = 0.0f;
  for (int k = 0; k < ntiles; ++k) yy += ypart[static_cast<size_t>(k) * Mp + r];
  y[r] = yy;
  const float d = (r < M) ? (yy - t[r]) : 0.0f;
  dy_out[r] = 2.0f * d / static_cast<float>(M);
  if (r < M) atomicAdd(loss, d * d / static_cast<float>(M));
}

// dz3 = dy w4 * silu'(z3), one thread per (16-column chunk, row).
__global__ void k_out_dz(int Mp, int H, const float* __restrict__ dy,
                         const float* __restrict__ w4, const float* __restrict__ z3,
                         bf16* __restrict__ dz3, bf16* __restrict__ dz3t) {
  const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<long long>(Mp) * (H / 16)) return;
  const int r = static_cast<int>(e % Mp), c0 = static_cast<int>(e / Mp) * 16;
  const float d = dy[r];
  const float4* zp = reinterpret_cast<const float4*>(z3 + static_cast<size_t>(r) * H + c0);
  float v[16];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float4 zz = zp[q];
    v[4 * q] = d * w4[c0 + 4 * q] * dsilu(zz.x);
    v[4 * q + 1] = d * w4[c0 + 4 * q + 1] * dsilu(zz.y);
    v[4 * q + 2] = d * w4[c0 + 4 * q + 2] * dsilu(zz.z);
    v[4 * q + 3] = d * w4[c0 + 4 * q + 3] * dsilu(zz.w);
  }
  st_bf16x16(dz3 + static_cast<size_t>(r) * H + c0, v);
#pragma unroll
  for (int j = 0; j < 16; ++j) dz3t[static_cast<size_t>(c0 + j) * Mp + r] = __float2bfloat16_rn(v[j]);
}

// Gradients of w4 (sum_r dy h3[r]), b4 (sum dy) and the hidden biases
// (column sums of dz), then their Adam steps; one block per vector entry.
struct BiasArgs {
  int Mp, H;
  const float* dy;
  const bf16* h3;
  const bf16* dz[3];
  float* p[5];   // b1, b2, b3, w4, b4
  float* m[5];
  float* v[5];
  float* grad_out[5];
};

__global__ void k_bias_adam(BiasArgs a, AdamArgs ad) {
  __shared__ float sh[32];
  const int H = a.H;
  const int e = blockIdx.x;  // 0..3H: b1, b2, b3, w4 entries; 4H: b4
  int which, c;
  if (e < 3 * H) { which = e / H; c = e - which * H; }
  else if (e < 4 * H) { which = 3; c = e - 3 * H; }
  else { which = 4; c = 0; }
  float s = 0.0f;
  for (int r = threadIdx.x; r < a.Mp; r += blockDim.x) {
    if (which < 3) s += __bfloat162float(a.dz[which][static_cast<size_t>(r) * H + c]);
    else if (which == 3) s += a.dy[r] * __bfloat162float(a.h3[static_cast<size_t>(r) * H + c]);
    else s += a.dy[r];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float g = 0.0f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) g += sh[w];
    if (a.grad_out[which]) {
      a.grad_out[which][c] = g;
      return;
    }
    float* p = a.p[which];
    float* m = a.m[which];
    float* v = a.v[which];
    const float mm = ad.b1 * m[c] + (1.0f - ad.b1) * g;
    const float vv = ad.b2 * v[c] + (1.0f - ad.b2) * g * g;
    m[c] = mm;
    v[c] = vv;
    p[c] -= ad.lr * (mm / ad.bc1) / (sqrtf(vv / ad.bc2) + ad.eps);
  }
}

// Minibatch rows: Philox-free LCG hash of (iteration, slot) over the pairs
// held (uniform with replacement).
__global__ void k_pick_rows(int Mb, unsigned n, unsigned long long it,
                            unsigned long long seed, int* __restrict__ rows) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= Mb) return;
  unsigned long long x = seed ^ (it * 0x9E3779B97F4A7C15ull) ^ (static_cast<unsigned long long>(r) *
                                                                 0xBF58476D1CE4E5B9ull);
  // splitmix64 finaliser (Steele, Lea & Flood 2014)
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  rows[r] = static_cast<int>((x >> 32) * static_cast<unsigned long long>(n) >> 32);
}

// Targets (logL - ymax, floored at -clip) / ys.
__global__ void k_gather_targets(int M, const int* __restrict__ rows,
                                 const double* __restrict__ logl, double ymax, double clip,
                                 double iys, float* __restrict__ t) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  const double d = logl[rows ? rows[r] : r] - ymax;
  t[r] = static_cast<float>((d < -clip ? -clip : d) * iys);
}

// Network output to log-likelihood units: logL = ymax + ys * y.
__global__ void k_unscale(int M, int Mp, int ntiles, const float* __restrict__ ypart,
                          double ymax, double ys, double* __restrict__ out,
                          int* __restrict__ status) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  float yy = 0.0f;
  for (int k = 0; k < ntiles; ++k) yy += ypart[static_cast<size_t>(k) * Mp + r];
  out[r] = ymax + ys * static_cast<double>(yy);
  if (status) status[r] = POFD_OK;
}

// Appends the valid rows (status OK, finite logL) to the pair ring in row
// order: one block walks the rows in chunks, a ballot prefix gives each
// valid row its slot, so the ring's contents -- and every minibatch drawn
// from it -- depend only on the inputs (ranks that train on the same pairs
// train the same network).
__global__ void k_append_pairs(int n, const float* __restrict__ theta, int npar,
                               const double* __restrict__ logl, const int* __restrict__ status,
                               float* __restrict__ ptheta, double* __restrict__ plogl,
                               unsigned* __restrict__ counters, unsigned cap) {
  // counters[0] = pairs written (ring), counters[1] = pairs held
  __shared__ unsigned wsum[32];
  __shared__ unsigned base;
  if (threadIdx.x == 0) base = counters[0];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int r = c0 + static_cast<int>(threadIdx.x);
    const bool ok = r < n && (!status || status[r] == POFD_OK) && isfinite(logl[r]);
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    unsigned off = base;
    for (int k = 0; k < wid; ++k) off += wsum[k];
    if (ok) {
      const unsigned slot = (off + __popc(bal & ((1u << lane) - 1u))) % cap;
      for (int p = 0; p < npar; ++p)
        ptheta[static_cast<size_t>(slot) * npar + p] = theta[static_cast<size_t>(r) * npar + p];
      plogl[slot] = logl[r];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
      for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) tot += wsum[k];
      base += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    counters[0] = base;
    counters[1] = min(max(counters[1], base), cap);
  }
}

// ----------------------------------------------------------- tensor maps
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    ck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q),
       "cuTensorMapEncodeTiled entry point");
    if (q != cudaDriverEntryPointSuccess || !p) throw Error(POFD_E_CUDA, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeFn>(p);
  }
  return fn;
}

// A row-major bf16 matrix [rows][K] (leading dimension ld elements) viewed
// as [K/8][rows][8] so that a {8, box_rows, 8} box lands in the canonical
// no-swizzle K-major layout; rows and K beyond the matrix read as zero.
CUtensorMap kmajor_map(const bf16* base, int rows, int K, int ld, int box_rows) {
  if (reinterpret_cast<uintptr_t>(base) % 16 || ld % 8 || K % 16)
    throw Error(POFD_E_ARG, "tensor map: base 16-byte aligned, ld multiple of 8, K multiple of 16");
  CUtensorMap m;
  const cuuint64_t dims[3] = {8, static_cast<cuuint64_t>(rows), static_cast<cuuint64_t>(K / 8)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(ld) * 2, 16};
  // the box is always {8, box_rows, 8}: rows and K groups past the matrix
  // are zero-filled, so every stage holds exactly stage_bytes() and keeps the
  // layout the MMA descriptors assume
  const cuuint32_t box[3] = {8, static_cast<cuuint32_t>(box_rows), 8};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(base),
                                 dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(POFD_E_CUDA, "cuTensorMapEncodeTiled failed");
  return m;
}

struct Gemm {
  umma::GemmShape g;
  CUtensorMap a, b;
  dim3 grid;
  size_t smem;
};

// N tile of a GEMM: the widest of 128, 64, 32 dividing N that still gives at
// least one CTA per SM, else 16.  The surrogate's GEMMs are small (a few
// hundred rows); narrower tiles spread them -- and the fused epilogues, the
// Adam update of the weight gradient above all -- over more SMs.
int ntile_for(int M, int N) {
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0)
      nsm = 148;
  }
  const int rt = (M + umma::kRows - 1) / umma::kRows;
  for (int nt : {128, 64, 32})
    if (N % nt == 0 && rt * (N / nt) >= nsm) return nt;
  return 16;
}

// C[M x N] = A[M x K] B[N x K]^T with A (lda) and B (ldb) row-major bf16.
Gemm plan_gemm(int M, int N, int K, const bf16* A, int lda, const bf16* B, int ldb, int* err) {
  if (M <= 0 || N < 16 || N > umma::kMaxN || N % 16 || K < 16 || K % 16)
    throw Error(POFD_E_ARG, "gemm: need N in [16, 512] and K >= 16, both multiples of 16");
  Gemm q;
  const int nt = ntile_for(M, N);
  q.g = umma::GemmShape{M, N, K, nt, err};
  q.a = kmajor_map(A, M, K, lda, umma::kRows);
  q.b = kmajor_map(B, N, K, ldb, nt);
  q.grid = dim3(static_cast<unsigned>((M + umma::kRows - 1) / umma::kRows),
                static_cast<unsigned>(N / nt));
  q.smem = umma::smem_bytes(nt);
  return q;
}

void set_gemm_attributes() {
  static bool done = false;
  if (done) return;
  const int sm = static_cast<int>(umma::smem_bytes(umma::kMaxNTile));
  ck(cudaFuncSetAttribute(k_gemm_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  ck(cudaFuncSetAttribute(k_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  ck(cudaFuncSetAttribute(k_bwd_dx, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  ck(cudaFuncSetAttribute(k_wgrad_adam, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  done = true;
}

}  // namespace

// ===================================================================== host

Surrogate::Surrogate(int device, cudaStream_t stream, unsigned npar, const int* free_idx,
                     unsigned nin, unsigned hidden, unsigned capacity, uint64_t seed)
    : device_(device), stream_(stream), npar_(npar), nin_(nin), H_(hidden), cap_(capacity),
      seed_(seed) {
  if (device < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  if (nin == 0 || nin > static_cast<unsigned>(kInPad)) throw Error(POFD_E_ARG, "1..16 inputs");
  if (hidden < 16 || hidden > 512 || hidden % 16) throw Error(POFD_E_ARG, "hidden width must be a multiple of 16 in [16, 512]");
  if (capacity < 128) throw Error(POFD_E_ARG, "capacity must be >= 128");
  for (unsigned i = 0; i < nin; ++i)
    if (free_idx[i] < 0 || static_cast<unsigned>(free_idx[i]) >= npar) throw Error(POFD_E_ARG, "input index out of range");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  idx_ = dal<int>(kInPad);
  ck(cudaMemcpy(idx_, free_idx, nin * sizeof(int), cudaMemcpyHostToDevice), "upload");
  mu_ = dal<float>(kInPad);
  wm_ = dal<float>(kInPad * kInPad);
  std::vector<float> eye(kInPad * kInPad, 0.0f);
  for (int k = 0; k < kInPad; ++k) eye[k * kInPad + k] = 1.0f;
  ck(cudaMemcpy(wm_, eye.data(), eye.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
  const size_t H = H_;
  const size_t sz[kNumTensors] = {H * kInPad, H, H * H, H, H * H, H, H, 1};
  for (int t = 0; t < kNumTensors; ++t) {
    size_[t] = sz[t];
    p_[t] = dal<float>(sz[t]);
    m_[t] = dal<float>(sz[t]);
    v_[t] = dal<float>(sz[t]);
  }
  w1b_ = dal<bf16>(H * kInPad);
  w2b_ = dal<bf16>(H * H);
  w3b_ = dal<bf16>(H * H);
  w2t_ = dal<bf16>(H * H);
  w3t_ = dal<bf16>(H * H);
  ptheta_ = dal<float>(static_cast<size_t>(cap_) * npar_);
  plogl_ = dal<double>(cap_);
  counters_ = dal<unsigned>(4);
  err_ = dal<int>(1);
  set_gemm_attributes();
  init_weights();
}

Surrogate::~Surrogate() {
  cudaSetDevice(device_);
  for (int t = 0; t < kNumTensors; ++t) {
    cudaFree(p_[t]);
    cudaFree(m_[t]);
    cudaFree(v_[t]);
  }
  void* q[] = {idx_, mu_, wm_, w1b_, w2b_, w3b_, w2t_, w3t_, ptheta_, plogl_, counters_, err_,
               ws_.x, ws_.xt, ws_.h[0], ws_.h[1], ws_.h[2], ws_.ht[0], ws_.ht[1], ws_.ht[2],
               ws_.z[0], ws_.z[1], ws_.z[2], ws_.dz[0], ws_.dz[1], ws_.dz[2], ws_.dzt[0],
               ws_.dzt[1], ws_.dzt[2], ws_.y, ws_.ypart, ws_.t, ws_.dy, ws_.rows, ws_.loss};
  for (void* p : q)
    if (p) cudaFree(p);
}

// He-style uniform initialisation (fan-in) from a seeded host generator.
void Surrogate::init_weights() {
  uint64_t s = seed_ ? seed_ : 0x1234567ull;
  auto next = [&s]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
  };
  const int fan[kNumTensors] = {static_cast<int>(nin_), 1, static_cast<int>(H_), 1,
                                static_cast<int>(H_), 1, static_cast<int>(H_), 1};
  std::vector<std::vector<float>> host(kNumTensors);
  for (int t = 0; t < kNumTensors; ++t) {
    host[t].assign(size_[t], 0.0f);
    if (t == 1 || t == 3 || t == 5 || t == 7) continue;  // biases start at 0
    const double a = std::sqrt(6.0 / fan[t]) * (t == 6 ? 0.5 : 1.0);
    for (size_t i = 0; i < size_[t]; ++i) {
      if (t == 0 && (i % kInPad) >= nin_) continue;  // padded inputs
      host[t][i] = static_cast<float>((2.0 * next() - 1.0) * a);
    }
  }
  set_params_host(host);
}

void Surrogate::set_params_host(const std::vector<std::vector<float>>& host) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  for (int t = 0; t < kNumTensors; ++t) {
    ck(cudaMemcpy(p_[t], host[t].data(), size_[t] * sizeof(float), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemset(m_[t], 0, size_[t] * sizeof(float)), "memset");
    ck(cudaMemset(v_[t], 0, size_[t] * sizeof(float)), "memset");
  }
  step_ = 0;
  refresh_bf16(host);
}

void Surrogate::refresh_bf16(const std::vector<std::vector<float>>& host) {
  const size_t H = H_;
  std::vector<bf16> a(H * kInPad), b(H * H), bt(H * H), c(H * H), ct(H * H);
  for (size_t i = 0; i < H * kInPad; ++i) a[i] = __float2bfloat16_rn(host[0][i]);
  for (size_t r = 0; r < H; ++r)
    for (size_t k = 0; k < H; ++k) {
      b[r * H + k] = __float2bfloat16_rn(host[2][r * H + k]);
      bt[k * H + r] = b[r * H + k];
      c[r * H + k] = __float2bfloat16_rn(host[4][r * H + k]);
      ct[k * H + r] = c[r * H + k];
    }
  ck(cudaMemcpy(w1b_, a.data(), a.size() * sizeof(bf16), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(w2b_, b.data(), b.size() * sizeof(bf16), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(w2t_, bt.data(), bt.size() * sizeof(bf16), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(w3b_, c.data(), c.size() * sizeof(bf16), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(w3t_, ct.data(), ct.size() * sizeof(bf16), cudaMemcpyHostToDevice), "upload");
}

void Surrogate::get_params_host(std::vector<std::vector<float>>& host) const {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  host.resize(kNumTensors);
  for (int t = 0; t < kNumTensors; ++t) {
    host[t].resize(size_[t]);
    ck(cudaMemcpy(host[t].data(), p_[t], size_[t] * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
  }
}

void Surrogate::ensure_work(int Mp) {
  if (Mp <= ws_.Mp) return;
  void* q[] = {ws_.x, ws_.xt, ws_.h[0], ws_.h[1], ws_.h[2], ws_.ht[0], ws_.ht[1], ws_.ht[2],
               ws_.z[0], ws_.z[1], ws_.z[2], ws_.dz[0], ws_.dz[1], ws_.dz[2], ws_.dzt[0],
               ws_.dzt[1], ws_.dzt[2], ws_.y, ws_.ypart, ws_.t, ws_.dy, ws_.rows, ws_.loss};
  for (void* p : q)
    if (p) cudaFree(p);
  ws_ = Work{};
  const size_t M = static_cast<size_t>(Mp), H = H_;
  ws_.Mp = Mp;
  ws_.x = dal<bf16>(M * kInPad);
  ws_.xt = dal<bf16>(M * kInPad);
  for (int l = 0; l < 3; ++l) {
    ws_.h[l] = dal<bf16>(M * H);
    ws_.ht[l] = dal<bf16>(M * H);
    ws_.z[l] = dal<float>(M * H);
    ws_.dz[l] = dal<bf16>(M * H);
    ws_.dzt[l] = dal<bf16>(M * H);
  }
  ws_.y = dal<float>(M);
  ws_.ypart = dal<float>(M * (umma::kMaxN / 16));
  ws_.t = dal<float>(M);
  ws_.dy = dal<float>(M);
  ws_.rows = dal<int>(M);
  ws_.loss = dal<float>(1);
}

// Forward of M rows of theta (optionally gathered through rows) into
// ws_.y; keeps z, h and h^T when train.
void Surrogate::forward(int M, const float* theta, int npar, const int* rows, bool train,
                        cudaStream_t st) {
  const int Mp = (M + umma::kRows - 1) / umma::kRows * umma::kRows;
  ensure_work(Mp);
  const int H = static_cast<int>(H_);
  k_pack_inputs<<<(Mp + 127) / 128, 128, 0, st>>>(M, Mp, theta, npar, idx_, static_cast<int>(nin_),
                                                  mu_, wm_, rows, ws_.x, train ? ws_.xt : nullptr);
  const bf16* Ws[3] = {w1b_, w2b_, w3b_};
  const bf16* in = ws_.x;
  int ldin = kInPad;
  for (int l = 0; l < 3; ++l) {
    const int K = (l == 0) ? kInPad : H;
    const Gemm q = plan_gemm(Mp, H, K, in, ldin, Ws[l], K, err_);
    const bool last = (l == 2);
    k_fwd<<<q.grid, NT, q.smem, st>>>(q.a, q.b, q.g, p_[2 * l + 1], ws_.h[l], H,
                                      train ? ws_.z[l] : nullptr, train ? ws_.ht[l] : nullptr, Mp,
                                      last ? p_[6] : nullptr, last ? p_[7] : nullptr, ws_.ypart);
    in = ws_.h[l];
    ldin = H;
  }
  ck(cudaGetLastError(), "surrogate forward");
}

void Surrogate::predict(unsigned n, const float* theta, unsigned npar, double* out, int* status,
                        cudaStream_t st) {
  if (n == 0) return;
  if (npar < npar_) throw Error(POFD_E_ARG, "Not enough elements in params");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (!st) st = stream_;
  forward(static_cast<int>(n), theta, static_cast<int>(npar), nullptr, false, st);
  const int Mp = (static_cast<int>(n) + umma::kRows - 1) / umma::kRows * umma::kRows;
  const int ntiles = static_cast<int>(H_) / ntile_for(Mp, static_cast<int>(H_));
  k_unscale<<<(n + 127) / 128, 128, 0, st>>>(static_cast<int>(n), Mp, ntiles, ws_.ypart, ymax_, ys_,
                                             out, status);
  ck(cudaGetLastError(), "k_unscale");
}

void Surrogate::add_pairs(unsigned n, const float* theta, unsigned npar, const double* logl,
                          const int* status, cudaStream_t st) {
  if (n == 0) return;
  if (npar != npar_) throw Error(POFD_E_ARG, "parameter count differs from the surrogate's");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (!st) st = stream_;
  k_append_pairs<<<1, 1024, 0, st>>>(static_cast<int>(n), theta, static_cast<int>(npar), logl,
                                     status, ptheta_, plogl_, counters_, cap_);
  ck(cudaGetLastError(), "k_append_pairs");
}

unsigned Surrogate::npairs() const {
  unsigned c[4];
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  ck(cudaMemcpy(c, counters_, sizeof(c), cudaMemcpyDeviceToHost), "D2H");
  return c[1];
}

void Surrogate::pairs_host(unsigned n, float* theta, double* logl) const {
  if (n > npairs()) throw Error(POFD_E_ARG, "more pairs asked for than are held");
  if (n == 0) return;
  if (theta)
    ck(cudaMemcpy(theta, ptheta_, static_cast<size_t>(n) * npar_ * sizeof(float),
                  cudaMemcpyDeviceToHost), "D2H pairs");
  if (logl) ck(cudaMemcpy(logl, plogl_, n * sizeof(double), cudaMemcpyDeviceToHost), "D2H pairs");
}

// Standardisation of the inputs (mean, 1/sd of the free parameters) and of
// the target (running max, sd of logL) from the pairs held.
void Surrogate::refresh_scaling() {
  const unsigned n = npairs();
  if (n < 2) throw Error(POFD_E_ARG, "need at least two training pairs");
  std::vector<float> th(static_cast<size_t>(n) * npar_);
  std::vector<double> ll(n);
  ck(cudaMemcpy(th.data(), ptheta_, th.size() * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
  ck(cudaMemcpy(ll.data(), plogl_, n * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
  std::vector<int> idx(kInPad, 0);
  ck(cudaMemcpy(idx.data(), idx_, kInPad * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
  // inputs standardised over the pairs whose target is not clipped (the
  // region the sampler explores once burnt in), when there are enough of
  // them; far-off burn-in points then sit at large |x| instead of setting
  // the scale
  double lmax = -std::numeric_limits<double>::infinity();
  for (double v : ll) lmax = std::max(lmax, v);
  const double clip0 = 25.0 + 2.5 * nin_;
  std::vector<unsigned> use;
  for (unsigned i = 0; i < n; ++i)
    if (ll[i] - lmax > -clip0) use.push_back(i);
  if (use.size() < std::max<size_t>(2 * nin_, 64)) {
    use.resize(n);
    for (unsigned i = 0; i < n; ++i) use[i] = i;
  }
  // Whitening: mean and covariance of the inputs over those pairs, W = L^-1
  // with L L^T the covariance (Cholesky), so that the network sees
  // decorrelated unit-variance inputs (the knot values of a P(D) posterior
  // are strongly correlated).  A covariance that is not positive definite
  // falls back to the diagonal (1/sd) scaling.
  const double nu = static_cast<double>(use.size());
  const unsigned K = nin_;
  std::vector<double> mean_in(K, 0.0), cov(K * K, 0.0);
  for (unsigned k = 0; k < K; ++k) {
    double s = 0;
    for (unsigned i : use) s += th[static_cast<size_t>(i) * npar_ + idx[k]];
    mean_in[k] = s / nu;
  }
  for (unsigned i : use) {
    double d[kInPad];
    for (unsigned k = 0; k < K; ++k) d[k] = th[static_cast<size_t>(i) * npar_ + idx[k]] - mean_in[k];
    for (unsigned a = 0; a < K; ++a)
      for (unsigned b = 0; b <= a; ++b) cov[a * K + b] += d[a] * d[b];
  }
  for (unsigned a = 0; a < K; ++a)
    for (unsigned b = 0; b <= a; ++b) cov[a * K + b] /= nu;
  std::vector<double> L(K * K, 0.0), Winv(K * K, 0.0);
  bool chol = true;
  for (unsigned a = 0; a < K && chol; ++a) {
    for (unsigned b = 0; b <= a; ++b) {
      double v = cov[a * K + b];
      for (unsigned c = 0; c < b; ++c) v -= L[a * K + c] * L[b * K + c];
      if (a == b) {
        if (!(v > 1e-12 * std::fabs(cov[a * K + a])) || !(v > 0)) {
          chol = false;
          break;
        }
        L[a * K + a] = std::sqrt(v);
      } else {
        L[a * K + b] = v / L[b * K + b];
      }
    }
  }
  if (chol) {
    // inverse of the lower-triangular factor, column by column
    for (unsigned c = 0; c < K; ++c)
      for (unsigned a = c; a < K; ++a) {
        double v = (a == c) ? 1.0 : 0.0;
        for (unsigned b = c; b < a; ++b) v -= L[a * K + b] * Winv[b * K + c];
        Winv[a * K + c] = v / L[a * K + a];
      }
  } else {
    for (unsigned k = 0; k < K; ++k) {
      const double sd = std::sqrt(std::max(cov[k * K + k], 0.0));
      Winv[k * K + k] = sd > 0 ? 1.0 / sd : 1.0;
    }
  }
  std::vector<float> mu(kInPad, 0.0f), wm(kInPad * kInPad, 0.0f);
  for (unsigned a = 0; a < K; ++a) {
    mu[a] = static_cast<float>(mean_in[a]);
    for (unsigned b = 0; b < K; ++b) wm[a * kInPad + b] = static_cast<float>(Winv[a * K + b]);
  }
  whitened_ = chol;
  // target: logL - max, floored at -clip so that far-off burn-in points do
  // not set the scale; the floor grows with the number of inputs (a
  // chi-square of nin degrees of freedom sits near -nin/2)
  double mx = -std::numeric_limits<double>::infinity();
  for (double v : ll) mx = std::max(mx, v);
  const double clip = 25.0 + 2.5 * nin_;
  double s = 0, s2 = 0;
  for (double v : ll) s += std::max(v - mx, -clip);
  const double m = s / n;
  for (double v : ll) {
    const double d = std::max(v - mx, -clip) - m;
    s2 += d * d;
  }
  const double sd = std::sqrt(s2 / n);
  ymax_ = mx;
  clip_ = clip;
  ys_ = (sd > 0) ? sd : 1.0;
  ck(cudaMemcpy(mu_, mu.data(), kInPad * sizeof(float), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(wm_, wm.data(), wm.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
  scaled_ = true;
}

// One training iteration on Mb rows (rows of the pair buffer, or the first
// Mb pairs when rows is null).  grads (8 tensors), when given, receive the
// loss gradients and the weights are not updated.
float Surrogate::iteration(int Mb, const int* rows, float lr, float** grads, cudaStream_t st) {
  const int Mp = (Mb + umma::kRows - 1) / umma::kRows * umma::kRows;
  const int H = static_cast<int>(H_);
  forward(Mb, ptheta_, static_cast<int>(npar_), rows, true, st);
  k_gather_targets<<<(Mb + 127) / 128, 128, 0, st>>>(Mb, rows, plogl_, ymax_, clip_, 1.0 / ys_,
                                                     ws_.t);
  ck(cudaMemsetAsync(ws_.loss, 0, sizeof(float), st), "memset");
  const int ntiles = H / ntile_for(Mp, H);
  k_out_loss<<<(Mp + 127) / 128, 128, 0, st>>>(Mb, Mp, ntiles, ws_.ypart, ws_.t, ws_.y, ws_.dy,
                                               ws_.loss);
  {
    const long long ne = static_cast<long long>(Mp) * (H / 16);
    k_out_dz<<<static_cast<unsigned>((ne + 127) / 128), 128, 0, st>>>(Mp, H, ws_.dy, p_[6],
                                                                     ws_.z[2], ws_.dz[2],
                                                                     ws_.dzt[2]);
  }
  ++step_;
  AdamArgs ad{lr, 0.9f, 0.999f, 1e-8f, 1.0f - std::pow(0.9f, static_cast<float>(step_)),
              1.0f - std::pow(0.999f, static_cast<float>(step_))};
  const bf16* Wt[3] = {nullptr, w2t_, w3t_};
  bf16* Wb[3] = {w1b_, w2b_, w3b_};
  bf16* Wtw[3] = {nullptr, w2t_, w3t_};
  for (int l = 2; l >= 0; --l) {
    if (l > 0) {
      // dh_{l-1} = dz_l W_l: A = dz_l [Mp x H], B = W_l^T [H x H]
      const Gemm q = plan_gemm(Mp, H, H, ws_.dz[l], H, Wt[l], H, err_);
      k_bwd_dx<<<q.grid, NT, q.smem, st>>>(q.a, q.b, q.g, ws_.z[l - 1], ws_.dz[l - 1],
                                           ws_.dzt[l - 1], Mp);
    }
    // G_l = dz_l^T X_l: A = dz_l^T [H x Mp], B = X_l^T [Nin x Mp]
    const int nin = (l == 0) ? kInPad : H;
    const bf16* XT = (l == 0) ? ws_.xt : ws_.ht[l - 1];
    const Gemm q = plan_gemm(H, nin, Mp, ws_.dzt[l], Mp, XT, Mp, err_);
    k_wgrad_adam<<<q.grid, NT, q.smem, st>>>(q.a, q.b, q.g, ad, p_[2 * l], m_[2 * l], v_[2 * l],
                                             Wb[l], nin, Wtw[l], H,
                                             grads ? grads[2 * l] : nullptr);
  }
  BiasArgs ba{};
  ba.Mp = Mp;
  ba.H = H;
  ba.dy = ws_.dy;
  ba.h3 = ws_.h[2];
  for (int l = 0; l < 3; ++l) ba.dz[l] = ws_.dz[l];
  const int map[5] = {1, 3, 5, 6, 7};
  for (int q = 0; q < 5; ++q) {
    ba.p[q] = p_[map[q]];
    ba.m[q] = m_[map[q]];
    ba.v[q] = v_[map[q]];
    ba.grad_out[q] = grads ? grads[map[q]] : nullptr;
  }
  k_bias_adam<<<4 * H + 1, 256, 0, st>>>(ba, ad);
  ck(cudaGetLastError(), "surrogate training");
  return 0.0f;
}

void Surrogate::train(unsigned iters, unsigned batch, float lr, float* last_loss) {
  if (batch == 0 || batch > 65536) throw Error(POFD_E_ARG, "batch must be in [1, 65536]");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  refresh_scaling();
  const unsigned n = npairs();
  const int Mb = static_cast<int>(batch);
  ensure_work((Mb + umma::kRows - 1) / umma::kRows * umma::kRows);
  ck(cudaMemset(err_, 0, sizeof(int)), "memset");
  for (unsigned it = 0; it < iters; ++it) {
    k_pick_rows<<<(Mb + 127) / 128, 128, 0, stream_>>>(Mb, n, static_cast<unsigned long long>(step_) + 1,
                                                     seed_, ws_.rows);
    iteration(Mb, ws_.rows, lr, nullptr, stream_);
  }
  ck(cudaStreamSynchronize(stream_), "synchronize");
  check_err();
  if (last_loss) ck(cudaMemcpy(last_loss, ws_.loss, sizeof(float), cudaMemcpyDeviceToHost), "D2H");
}

void Surrogate::gradients(unsigned n, float** grads_dev, float* loss) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (!scaled_) refresh_scaling();
  if (n == 0 || n > npairs()) throw Error(POFD_E_ARG, "rows beyond the pairs held");
  ensure_work((static_cast<int>(n) + umma::kRows - 1) / umma::kRows * umma::kRows);
  ck(cudaMemset(err_, 0, sizeof(int)), "memset");
  const unsigned s0 = step_;
  iteration(static_cast<int>(n), nullptr, 0.0f, grads_dev, stream_);
  step_ = s0;
  ck(cudaStreamSynchronize(stream_), "synchronize");
  check_err();
  if (loss) ck(cudaMemcpy(loss, ws_.loss, sizeof(float), cudaMemcpyDeviceToHost), "D2H");
}

void Surrogate::check_err() {
  int e = 0;
  ck(cudaMemcpy(&e, err_, sizeof(int), cudaMemcpyDeviceToHost), "D2H err");
  if (e) {
    ck(cudaMemset(err_, 0, sizeof(int)), "memset");
    throw Error(POFD_E_CUDA, "tensor-core wait timed out");
  }
}

void Surrogate::scaling(double* out) const {
  std::vector<float> mu(kInPad), wm(kInPad * kInPad);
  ck(cudaMemcpy(mu.data(), mu_, kInPad * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
  ck(cudaMemcpy(wm.data(), wm_, wm.size() * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
  for (int k = 0; k < kInPad; ++k) out[k] = mu[k];
  for (int k = 0; k < kInPad * kInPad; ++k) out[kInPad + k] = wm[k];
  const int o = kInPad + kInPad * kInPad;
  out[o] = ymax_;
  out[o + 1] = ys_;
  out[o + 2] = clip_;
  out[o + 3] = whitened_ ? 1.0 : 0.0;
}

// The tensor-core main loop on its own: C = A B^T (fp32).
void bf16_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C,
               int ldc, int* err, cudaStream_t st) {
  set_gemm_attributes();
  const Gemm q = plan_gemm(M, N, K, static_cast<const bf16*>(A), lda, static_cast<const bf16*>(B),
                           ldb, err);
  k_gemm_f32<<<q.grid, NT, q.smem, st>>>(q.a, q.b, q.g, C, ldc);
  ck(cudaGetLastError(), "k_gemm_f32");
}

}  // namespace pofd
