// engine1d.cu -- 1D P(D) likelihood: sm_100a kernels and the batched engine.
//
// Reference path restated (aconley/pofd_affine 0.5.1):
//   numberCountsKnotsSpline::setParams / getR  numberCountsKnotsSpline.cc:265-274, 436-529
//   PDFactory::initRInterp / initR             PDFactory.cc:426-527, 541-620
//   PDFactory::getMeanVarFromR                 PDFactory.cc:625-679
//   PDFactory::initPD (FFT, exp, shift)        PDFactory.cc:1031-1141
//   PDFactory::getPD (noise, inverse FFT)      PDFactory.cc:1154-1243
//   PDFactory::findSplitPoint / unwrap         PDFactory.cc:691-1009
//   PD::normalize / getMean / applyLog         PD.cc:146-184, 245-274
//   PD::getLogLikeBinned / Unbinned            PD.cc:557-677
//   calcLikeSingle::getLogLike / calcLike      calcLike.cc:389-443, 884-955
//
// Layout in HBM (P proposals, B beam sets, D datasets, n FFT size, NI
// interpolation nodes, nc = n/2+1):
//   nodes [P][B][2][NI]        R at the nodes (pos/neg side)
//   spl   [P][B][2][NI][4]     node spline (y, b, c, d) per interval
//   rbuf  [P][B][2*nc]         R grid (x dflux), then its D2Z spectrum in place
//   pbuf  [P][D][2*nc]         per-dataset spectrum, then its Z2D P(D) in place
//   ppart/pmidx [P][D][nchunk] chunk reductions of the P(D)
//   pinfo [P][D]               split, normalisation, mean, log-likelihood
// Each proposal's R and P(D) rows are contiguous so the D2Z/Z2D run as two
// batched cuFFT calls over P*B and P*D rows.
#include "engine1d.cuh"

#include <algorithm>
#include <cstring>
#include <sstream>

#include "common.cuh"
#include "fft1d.cuh"

namespace pofd {

namespace {

constexpr int NT = 256;           // threads per block for the streaming kernels
constexpr int kMaxTilesPer = 4;   // smallest R-fill tile: NT * 4 grid points
constexpr int CHUNK = NT * 16;    // P(D) elements per reduction block
constexpr int kSplineThreads = 1024;  // threads per node-spline block
constexpr int KMAX = Engine1::KMAX;
constexpr int MAXTERMS = 4096;    // beam terms held in shared memory

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << what << ": " << cudaGetErrorString(e);
    throw Error(e == cudaErrorMemoryAllocation ? POFD_E_NOMEM : POFD_E_CUDA,
                s.str());
  }
}
void cufft_check(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) {
    std::ostringstream s;
    s << what << ": cuFFT error " << static_cast<int>(r);
    throw Error(r == CUFFT_ALLOC_FAILED ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}

// ------------------------------------------------------------- kernels

// Model set-up for one proposal: log2 knot values from the float parameters
// and the natural cubic spline through (log2 S_k, log2 n_k), stored per
// interval as (y, b, c, d) exactly as the spline library forms them at
// evaluation (numberCountsKnotsSpline.cc:265-274).  Returns the status.
__device__ int model_solve(const Model1Dev& m, const float* __restrict__ th,
                           double logfac, double* __restrict__ out,
                           double* __restrict__ wk /* 8*KMAX */) {
  const int K = m.K;
  double* y = wk;
  double* c = y + KMAX;
  double* g = c + KMAX;
  double* diag = g + KMAX;
  double* off = diag + KMAX;
  double* alp = off + KMAX;
  double* gam = alp + KMAX;
  double* z = gam + KMAX;
  for (int k = 0; k < K; ++k) {
    y[k] = logfac * static_cast<double>(th[k]);
    if (isnan(y[k])) return POFD_E_INVALID_MODEL;
  }
  const double* x = m.logknots;
  for (int k = 0; k < K; ++k) c[k] = 0.0;
  const int N = K - 2;
  for (int i = 0; i < N; ++i) {
    const double h_i = x[i + 1] - x[i], h_ip1 = x[i + 2] - x[i + 1];
    const double g_i = (h_i != 0.0) ? 1.0 / h_i : 0.0;
    const double g_ip1 = (h_ip1 != 0.0) ? 1.0 / h_ip1 : 0.0;
    off[i] = h_ip1;
    diag[i] = 2.0 * (h_ip1 + h_i);
    g[i] = 3.0 * ((y[i + 2] - y[i + 1]) * g_ip1 - (y[i + 1] - y[i]) * g_i);
  }
  if (N == 1) {
    c[1] = g[0] / diag[0];
  } else if (N > 1) {
    // symmetric tridiagonal L D L^T solve
    alp[0] = diag[0];
    gam[0] = off[0] / alp[0];
    for (int i = 1; i < N - 1; ++i) {
      alp[i] = diag[i] - off[i - 1] * gam[i - 1];
      gam[i] = off[i] / alp[i];
    }
    alp[N - 1] = diag[N - 1] - off[N - 2] * gam[N - 2];
    z[0] = g[0];
    for (int i = 1; i < N; ++i) z[i] = g[i] - gam[i - 1] * z[i - 1];
    for (int i = 0; i < N; ++i) z[i] = z[i] / alp[i];
    c[N] = z[N - 1];
    for (int i = N - 2; i >= 0; --i) c[1 + i] = z[i] - gam[i] * c[2 + i];
  }
  for (int i = 0; i < K - 1; ++i) {
    const double dx = x[i + 1] - x[i];
    const double dy = y[i + 1] - y[i];
    out[4 * i + 0] = y[i];
    out[4 * i + 1] = (dy / dx) - dx * (c[i + 1] + 2.0 * c[i]) / 3.0;
    out[4 * i + 2] = c[i];
    out[4 * i + 3] = (c[i + 1] - c[i]) / (3.0 * dx);
  }
  return POFD_OK;
}

// Knot spline of every proposal: one block per proposal, thread 0 solving
// in shared memory.  Publishes the model status and the sigma multiplier.
__global__ void k_model1(Model1Dev m, const float* __restrict__ theta,
                         int npar, double logfac, double* __restrict__ cnt,
                         int* __restrict__ mstatus,
                         double* __restrict__ sigmult) {
  __shared__ double wk[8 * KMAX];
  __shared__ double cs[4 * KMAX];
  const int w = blockIdx.x;
  const float* th = theta + static_cast<size_t>(w) * npar;
  if (threadIdx.x == 0) {
    const int st = model_solve(m, th, logfac, cs, wk);
    mstatus[w] = st;
    sigmult[w] = static_cast<double>(th[m.K]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * (m.K - 1); i += blockDim.x)
    cnt[static_cast<size_t>(w) * 4 * KMAX + i] = cs[i];
}

// R at the interpolation nodes, one node per thread, terms summed in the
// beam's order (numberCountsKnotsSpline.cc:495-526).  log2(x * ieta) is
// formed as log2|x| + log2(ieta) from host-computed logs; the range test uses
// the product itself, as the reference does.
__global__ void k_rnodes1(const BSet1Dev* __restrict__ bsets, Model1Dev m,
                          int B, int NI, int maxterms,
                          const double* __restrict__ cnt,
                          const int* __restrict__ mstatus,
                          double* __restrict__ nodes) {
  extern __shared__ double sm[];
  const int row = blockIdx.y;  // (w*B + b)*2 + side
  const int side = row & 1;
  const int wb = row >> 1;
  const int w = wb / B, b = wb - w * B;
  const BSet1Dev& bs = bsets[b];
  const Side1Dev& sd = bs.side[side];
  if (!sd.nodes || mstatus[w] != 0) return;
  const int K = m.K;
  double* s_lk = sm;
  double* s_cs = s_lk + KMAX;
  double* s_w = s_cs + 4 * KMAX;
  double* s_le = s_w + maxterms;
  double* s_ie = s_le + maxterms;
  const double* cs = cnt + static_cast<size_t>(w) * 4 * KMAX;
  for (int i = threadIdx.x; i < K; i += blockDim.x) s_lk[i] = m.logknots[i];
  for (int i = threadIdx.x; i < 4 * (K - 1); i += blockDim.x) s_cs[i] = cs[i];
  const int nt = sd.nterms;
  for (int i = threadIdx.x; i < nt; i += blockDim.x) {
    s_w[i] = sd.w[i];
    s_le[i] = sd.lie[i];
    s_ie[i] = sd.ieta[i];
  }
  __shared__ dev::Exp2Table e2;
  e2.load();
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NI) return;
  const double f = sd.x[i];
  const double lf = sd.lxa[i];
  double workval = 0.0;
  const bool posb = (f > 0 && bs.haspos && f <= bs.rr_hi);
  const bool negb = !posb && (bs.hasneg && f < 0 && f >= bs.rr_lo);
  if (posb || negb) {
    // the knot interval and the range test of every term at this node come
    // from the host-built table (the reference searches them per call);
    // terms outside the node's first-to-last in-range span are not visited
    const unsigned char* __restrict__ kt = sd.kidx + i;
    const int2 jr = sd.jrange[i];
    for (int j = jr.x; j < jr.y; ++j) {
      const int k = kt[static_cast<size_t>(j) * NI];
      if (k == 255) continue;
      const double delx = (lf + s_le[j]) - s_lk[k];
      const double* q = s_cs + 4 * k;
      const double cts =
          dev::exp2_tab(q[0] + delx * (q[1] + delx * (q[2] + delx * q[3])), e2.t);
      if (cts > 0) workval += s_w[j] * cts * s_ie[j];
    }
  }
  nodes[static_cast<size_t>(row) * NI + i] = bs.prefac * workval;
}

// Natural cubic spline through (x_i, log2 R_i) over the NI nodes: RHS of
// the tridiagonal system, forward and back substitution against the
// precomputed LDL^T factors as two block-wide affine-map scans, then the
// per-interval (y, b, c, d) (PDFactory.cc:466-474, 522).
template <int RT>
__global__ void __launch_bounds__(RT, 2048 / RT)
k_rspline1(const BSet1Dev* __restrict__ bsets, int B, int NI,
           const int* __restrict__ mstatus, const double* __restrict__ nodes,
           double* __restrict__ spl) {
  extern __shared__ double sm[];
  const int row = blockIdx.x;
  const int side = row & 1;
  const int wb = row >> 1;
  const int w = wb / B, b = wb - w * B;
  const Side1Dev& sd = bsets[b].side[side];
  if (!sd.nodes || mstatus[w] != 0) return;
  double* y = sm;             // NI
  double* c = y + NI;         // NI (full second-derivative/2 array)
  double* scr = c + NI;       // 64
  const double* R = nodes + static_cast<size_t>(row) * NI;
  for (int i = threadIdx.x; i < NI; i += RT) {
    const double v = R[i];
    y[i] = (v > 0) ? log2(v) : dev::kSmallLogVal;
  }
  __syncthreads();
  const int N = NI - 2;
  const int E = (N + RT - 1) / RT;
  const int s0 = threadIdx.x * E;
  const int s1 = min(s0 + E, N);
  const double* ih = sd.ih;
  const double* al = sd.alpha;
  const double* ga = sd.gamma;
  // forward: z_i = g_i - gamma_{i-1} z_{i-1}, z_0 = g_0; stored in c[1+i]
  double A = 1.0, Bv = 0.0;
  for (int i = s0; i < s1; ++i) {
    const double gi = 3.0 * ((y[i + 2] - y[i + 1]) * ih[i + 1] - (y[i + 1] - y[i]) * ih[i]);
    c[1 + i] = gi;
    const double a = (i == 0) ? 0.0 : -ga[i - 1];
    Bv = a * Bv + gi;
    A = a * A;
  }
  // exclusive prefix: the previous thread's composed map at z = 0
  const double zin = dev::block_affine_scan_w<RT>(A, Bv, scr);
  {
    double z = zin;
    for (int i = s0; i < s1; ++i) {
      const double gi = c[1 + i];
      z = (i == 0) ? gi : gi - ga[i - 1] * z;
      c[1 + i] = z / al[i];  // cc_i
    }
  }
  __syncthreads();
  // back: c_i = cc_i - gamma_i c_{i+1}, c_{N-1} = cc_{N-1}
  A = 1.0;
  Bv = 0.0;
  for (int i = s1 - 1; i >= s0; --i) {
    const double a = (i == N - 1) ? 0.0 : -ga[i];
    Bv = a * Bv + c[1 + i];
    A = a * A;
  }
  const double cin = dev::block_affine_rscan_w<RT>(A, Bv, scr);
  {
    double cn = cin;
    for (int i = s1 - 1; i >= s0; --i) {
      const double cc = c[1 + i];
      cn = (i == N - 1) ? cc : cc - ga[i] * cn;
      c[1 + i] = cn;
    }
  }
  if (threadIdx.x == 0) {
    c[0] = 0.0;
    c[NI - 1] = 0.0;
  }
  __syncthreads();
  // one 32-byte record (y, b, c, d) per interval
  double2* out = reinterpret_cast<double2*>(spl + static_cast<size_t>(row) * 4 * NI);
  const double* x = sd.x;
  for (int i = threadIdx.x; i < NI - 1; i += RT) {
    const double dx = x[i + 1] - x[i];
    const double dy = y[i + 1] - y[i];
    out[2 * i] = make_double2(y[i], (dy / dx) - dx * (c[i + 1] + 2.0 * c[i]) / 3.0);
    out[2 * i + 1] = make_double2(c[i], (c[i + 1] - c[i]) / (3.0 * dx));
  }
}

// The wrapped R grid: 2^spline(flux) * dflux inside each side's covered
// index range, zero elsewhere (PDFactory.cc:556-613), plus the first and
// second flux moments (PDFactory.cc:634-665).  The node interval of every
// grid point is parameter-independent and comes from a host-built table
// (gidx, -1 outside the covered ranges).
struct GridFill1 {
  double dflux, minflux_R, off0, off1;
  int wrap, NI;
  const double* __restrict__ x0;
  const double* __restrict__ x1;
  const double* __restrict__ S0;   // this row's node spline [2][NI][4]
  const double* __restrict__ e2;   // exp2 table in shared memory

  __device__ __forceinline__ GridFill1(const BSet1Dev& bs, const double* spl_row, int ni,
                                       const double* tab)
      : dflux(bs.dflux), minflux_R(bs.minflux_R), off0(bs.side[0].grid_off),
        off1(bs.side[1].grid_off), wrap(bs.wrapRidx), NI(ni), x0(bs.side[0].x),
        x1(bs.side[1].x), S0(spl_row), e2(tab) {}

  // R at grid index i (di = i as a double) with node interval q (< 0: not
  // covered), and its moment terms added to mn, var: weight 0 at i = 0 (its
  // flux is 0), 1/2 at the positive edge, 1 elsewhere
  __device__ __forceinline__ double point(int i, double di, int q, double& mn,
                                          double& var) const {
    const bool neg = i > wrap;
    const double pd = __dmul_rn(di, dflux);
    double r = 0.0;
    if (q >= 0) {
      const double cflux = __dadd_rn(pd, neg ? off1 : off0);
      const double2* S = reinterpret_cast<const double2*>(S0 + (neg ? 4 * NI : 0)) + 2 * q;
      const double2 yb = S[0], cd = S[1];
      const double delx = cflux - (neg ? x1 : x0)[q];
      const double v = yb.x + delx * (yb.y + delx * (cd.x + delx * cd.y));
      r = dev::exp2_tab(v, e2) * dflux;
    }
    const double cf = neg ? static_cast<double>(i - wrap - 1) * dflux + minflux_R : pd;
    double prod = cf * r;
    if (i == wrap) prod *= 0.5;
    mn += prod;
    var += cf * prod;
    return r;
  }

  // R at the len (<= 16) consecutive grid indices of one run (i0, q) --
  // points of one covered node interval q on one side of the wrap -- into
  // the shared tile at out[pad(o + k)], with their moment terms.  The cubic
  // exponent v(t) of point i0 + t has constant third differences, so 2^v
  // follows from three running products: R(t+1) = R(t) E1(t), E1(t+1) =
  // E1(t) E2(t), E2(t+1) = E2(t) E3, with E1(0) = 2^(v(1) - v(0)), E2(0) =
  // 2^(second difference), E3 = 2^(third difference), the differences taken
  // analytically from the cubic: four exp2 per run instead of one per
  // point, and no per-point cubic or table lookup.  The products add at
  // most ~16^3/6 roundings (< 1e-13 relative) to each value.  A run whose
  // exponents leave the safe range goes point by point.
  __device__ __forceinline__ void run_products(int i0, int len, int q, double* out, int o,
                                               double& mn, double& var) const {
    const bool neg = i0 > wrap;
    const double2* S = reinterpret_cast<const double2*>(S0 + (neg ? 4 * NI : 0)) + 2 * q;
    const double2 yb = S[0], cd = S[1];
    const double h = dflux;
    const double d0 = __dadd_rn(__dmul_rn(static_cast<double>(i0), dflux), neg ? off1 : off0) -
                      (neg ? x1 : x0)[q];
    const double v0 = yb.x + d0 * (yb.y + d0 * (cd.x + d0 * cd.y));
    const double D1 = h * (yb.y + cd.x * (2.0 * d0 + h) + cd.y * (3.0 * d0 * (d0 + h) + h * h));
    const double D2 = h * h * (2.0 * cd.x + 6.0 * cd.y * (d0 + h));
    const double D3 = 6.0 * cd.y * h * h * h;
    if (fabs(v0) < 500.0 && fabs(D1) < 16.0 && fabs(D2) < 4.0 && fabs(D3) < 2.0) {
      double R = dev::exp2_tab(v0, e2) * dflux;
      double E1 = dev::exp2_tab(D1, e2), E2 = dev::exp2_tab(D2, e2);
      const double E3 = dev::exp2_tab(D3, e2);
      const double cb = neg ? minflux_R : 0.0;
      const int ib = neg ? wrap + 1 : 0;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (k >= len) break;
        const int i = i0 + k;
        out[pad(o + k)] = R;
        const double cf = neg ? static_cast<double>(i - ib) * dflux + cb
                              : __dmul_rn(static_cast<double>(i), dflux);
        double prod = cf * R;
        if (i == wrap) prod *= 0.5;
        mn += prod;
        var += cf * prod;
        R *= E1;
        E1 *= E2;
        E2 *= E3;
      }
      return;
    }
    for (int k = 0; k < len; ++k) {
      const int i = i0 + k;
      out[pad(o + k)] = point(i, static_cast<double>(i), q, mn, var);
    }
  }
  // shared tile index of span offset j: one pad word per 16 values, so that
  // threads starting runs ~16 values apart do not share a bank
  __device__ __forceinline__ static int pad(int j) { return j + (j >> 4); }
};

// The R grid materialised (cuFFT path, and the own path when the fill is
// not fused into the forward pass A), with block partial moment sums.
template <int PER>
__global__ void __launch_bounds__(NT)
k_rfill1(const BSet1Dev* __restrict__ bsets, int B, int n, int NI,
         int nc2, int ntile, const int* __restrict__ mstatus,
         const double* __restrict__ spl, double* __restrict__ rbuf,
         double* __restrict__ rpart) {
  __shared__ double shr[32];
  __shared__ dev::Exp2Table e2;
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  e2.load();
  __syncthreads();
  const BSet1Dev& bs = bsets[b];
  const GridFill1 rg(bs, spl + static_cast<size_t>(wb) * 2 * 4 * NI, NI, e2.t);
  const int* __restrict__ gidx = bs.gidx;
  double* R = rbuf + static_cast<size_t>(wb) * nc2;
  const int base = blockIdx.x * (NT * PER) + threadIdx.x;
  int q[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int i = base + k * NT;
    q[k] = (i < n) ? gidx[i] : -2;
  }
  double mn = 0.0, var = 0.0;
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int i = base + k * NT;
    if (q[k] == -2) break;
    R[i] = rg.point(i, static_cast<double>(i), q[k], mn, var);
  }
  mn = dev::block_sum<NT>(mn, shr);
  var = dev::block_sum<NT>(var, shr);
  if (threadIdx.x == 0) {
    double* o = rpart + (static_cast<size_t>(wb) * ntile + blockIdx.x) * 2;
    o[0] = mn;
    o[1] = var;
  }
}

// The R grid materialised by running products over static runs (mode 2):
// each beam set's grid is cut, at set-up, into runs of at most 16
// consecutive points that share one node interval and one side of the wrap
// (bs.runs: x = first index, y = (q + 1) << 8 | len << 2 | kind; kind 0:
// uncovered, R = 0; 1: shorter than four points, evaluated point by point;
// 2: running products, GridFill1::run_products).  Block k takes runs
// [k NT, k NT + NT) of its row -- one per thread, so no thread's run crosses
// an interval and warps do not diverge on interval changes -- stages their
// contiguous span of the grid (at most 16 NT values) in shared memory and
// writes it out coalesced; block partial moment sums (zero for blocks past
// the row's runs).
__global__ void __launch_bounds__(NT)
k_rfill1_run(const BSet1Dev* __restrict__ bsets, int B, int NI, int nc2, int ntile,
             const int* __restrict__ mstatus, const double* __restrict__ spl,
             double* __restrict__ rbuf, double* __restrict__ rpart) {
  __shared__ double tile[NT * 17];
  __shared__ double shr[32];
  __shared__ dev::Exp2Table e2;
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  e2.load();
  __syncthreads();
  const BSet1Dev& bs = bsets[b];
  const int r0 = blockIdx.x * NT;
  double mn = 0.0, var = 0.0;
  if (r0 < bs.nruns) {
    const GridFill1 rg(bs, spl + static_cast<size_t>(wb) * 2 * 4 * NI, NI, e2.t);
    const int r1 = min(r0 + NT, bs.nruns);
    const int span0 = __ldg(&bs.runs[r0].x);
    const int2 last = __ldg(&bs.runs[r1 - 1]);
    const int span = last.x + ((last.y >> 2) & 31) - span0;
    const int r = r0 + threadIdx.x;
    if (r < r1) {
      const int2 d = __ldg(&bs.runs[r]);
      const int len = (d.y >> 2) & 31, kind = d.y & 3, q = (d.y >> 8) - 1;
      const int o = d.x - span0;
      if (kind == 2) {
        rg.run_products(d.x, len, q, tile, o, mn, var);
      } else if (kind == 1) {
        for (int k = 0; k < len; ++k) {
          const int i = d.x + k;
          tile[GridFill1::pad(o + k)] = rg.point(i, static_cast<double>(i), q, mn, var);
        }
      } else {
        for (int k = 0; k < len; ++k) tile[GridFill1::pad(o + k)] = 0.0;
      }
    }
    __syncthreads();
    double* R = rbuf + static_cast<size_t>(wb) * nc2 + span0;
    for (int j = threadIdx.x; j < span; j += NT) R[j] = tile[GridFill1::pad(j)];
  }
  mn = dev::block_sum<NT>(mn, shr);
  var = dev::block_sum<NT>(var, shr);
  if (threadIdx.x == 0) {
    double* o = rpart + (static_cast<size_t>(wb) * ntile + blockIdx.x) * 2;
    o[0] = mn;
    o[1] = var;
  }
}

// R-fill launch with PER grid points per thread (an autotuned knob), or
// (seg) by running products over the static runs.
void launch_rfill(int per, bool seg, dim3 grid, cudaStream_t st, const BSet1Dev* bsets, int B,
                  int n, int NI, int nc2, int ntile, const int* mstatus, const double* spl,
                  double* rbuf, double* rpart) {
  if (seg) {
    k_rfill1_run<<<grid, NT, 0, st>>>(bsets, B, NI, nc2, ntile, mstatus, spl, rbuf, rpart);
    return;
  }
  switch (per) {
    case 4: k_rfill1<4><<<grid, NT, 0, st>>>(bsets, B, n, NI, nc2, ntile, mstatus, spl, rbuf, rpart); break;
    case 16: k_rfill1<16><<<grid, NT, 0, st>>>(bsets, B, n, NI, nc2, ntile, mstatus, spl, rbuf, rpart); break;
    default: k_rfill1<8><<<grid, NT, 0, st>>>(bsets, B, n, NI, nc2, ntile, mstatus, spl, rbuf, rpart); break;
  }
}

// Moments, sigma estimate and the shift decision (PDFactory.cc:660-679,
// 1067-1076), one thread per (proposal, beam set).
// Noise cut-off of the half-length spectrum (own-FFT path): with noise sigma
// the factor exp(-sigma^2 w_k^2 / 2) is below e^-760 -- exactly 0 in double
// precision, whose exp underflows below -745.2 -- for every bin k with
// min(k, m - k) > kc, kc = ceil(sqrt(1520) / (sigma * 2 pi / (n dflux))) + 1.
// Returns m (no bin is cut) without noise.
__device__ __forceinline__ int noise_cut(double sigma, double dflux, int n) {
  const int m = n / 2;
  if (!(sigma > 0.0)) return m;
  const double iflux = dev::kTwoPi / (static_cast<double>(n) * dflux);
  const double x = sqrt(1520.0) / (sigma * iflux);
  return (x >= static_cast<double>(m)) ? m : static_cast<int>(ceil(x)) + 1;
}

// Rows of 256 bins (row a: bins [256 a, 256 a + 256) of the m1 x 256 view)
// whose bins all lie beyond the cut-off.
__device__ __forceinline__ bool row_cut(int a, int m, int kc) {
  return min(256 * a, m - 256 * a - 255) > kc;
}

__global__ void k_moments1(const BSet1Dev* __restrict__ bsets,
                           const DSet1Dev* __restrict__ dsets, int B, int D, int n,
                           int nc2, int ntile, int nrow,
                           const int* __restrict__ mstatus,
                           const double* __restrict__ sigmult,
                           const double* __restrict__ rbuf,
                           const double* __restrict__ rpart,
                           double* __restrict__ mom, int* __restrict__ kcut_set,
                           int* __restrict__ kcut_ds) {
  const int wb = blockIdx.x * blockDim.x + threadIdx.x;
  if (wb >= nrow) return;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  const BSet1Dev& bs = bsets[b];
  if (kcut_set) {
    // bins the spectrum kernel reads: the widest cut-off of the set's
    // datasets; per dataset for the inverse transform's input
    int kmax = 0;
    for (int dd = 0; dd < bs.nds; ++dd) {
      const int d = bs.ds_begin + dd;
      const int kc = noise_cut(sigmult[w] * dsets[d].sigma_base, bs.dflux, n);
      kcut_ds[static_cast<size_t>(w) * D + d] = kc;
      kmax = max(kmax, kc);
    }
    kcut_set[wb] = (bs.nds > 0) ? kmax : n / 2;
  }
  double mn = 0.0, var = 0.0;
  const double* p = rpart + static_cast<size_t>(wb) * ntile * 2;
  for (int t = 0; t < ntile; ++t) {
    mn += p[2 * t];
    var += p[2 * t + 1];
  }
  const int wrap = bs.wrapRidx;
  if (wrap < n - 1) {
    const double cf = bs.minflux_R;
    const double prod = 0.5 * cf * rbuf[static_cast<size_t>(wb) * nc2 + (wrap - 1)];
    mn -= prod;
    var -= cf * prod;
  }
  const double sg = sqrt(var);
  const bool doshift = (sg > bs.dflux) && (fabs(mn) > bs.dflux);
  double* o = mom + static_cast<size_t>(wb) * 4;
  o[0] = mn;
  o[1] = var;
  o[2] = doshift ? -mn : 0.0;
  o[3] = doshift ? 1.0 : 0.0;
}

// exp(R~ - R~0) with the mean shift, then one noise-multiplied copy per
// dataset of the beam set (PDFactory.cc:1106-1132, 1174-1188).  The
// self-conjugate Nyquist bin keeps only its real part, which is what the
// c2r transform uses of it.  Where every dataset's noise exponent is below
// -750, exp() underflows to exactly 0 and the reference's product is 0: those
// bins are written as 0 without evaluating exp/sincos of the R spectrum.
__global__ void __launch_bounds__(NT)
k_spectrum1(const BSet1Dev* __restrict__ bsets,
            const DSet1Dev* __restrict__ dsets, int B, int D, int n, int nc,
            const int* __restrict__ mstatus, const double* __restrict__ sigmult,
            const double* __restrict__ mom, const double* __restrict__ rbuf,
            double* __restrict__ pbuf) {
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  const int k = blockIdx.x * NT + threadIdx.x;
  if (k >= nc) return;
  const BSet1Dev& bs = bsets[b];
  const double dflux = bs.dflux;
  const double iflux = dev::kTwoPi / (static_cast<double>(n) * dflux);
  const double sm = sigmult[w];
  const double wv = iflux * static_cast<double>(k);
  bool all_zero = k > 0;
  for (int dd = 0; dd < bs.nds && all_zero; ++dd) {
    const double sigma = sm * dsets[bs.ds_begin + dd].sigma_base;
    if (!(sigma > 0)) { all_zero = false; break; }
    const double sigfac = -0.5 * sigma * sigma;
    if (!(sigfac * wv * wv < -750.0)) all_zero = false;
  }
  if (all_zero) {
    for (int dd = 0; dd < bs.nds; ++dd)
      reinterpret_cast<double2*>(pbuf + (static_cast<size_t>(w) * D + bs.ds_begin + dd) * 2 * nc)[k] =
          make_double2(0.0, 0.0);
    return;
  }
  const double2* Rt = reinterpret_cast<const double2*>(rbuf + static_cast<size_t>(wb) * 2 * nc);
  const double* mo = mom + static_cast<size_t>(wb) * 4;
  const bool doshift = mo[3] != 0.0;
  double2 p;
  if (k == 0) {
    p = make_double2(1.0, 0.0);
  } else {
    const double r0 = Rt[0].x;
    const double2 v = Rt[k];
    const double expfac = exp(v.x - r0);
    const double ival = doshift ? v.y - (mo[2] * iflux) * static_cast<double>(k) : v.y;
    double s, c;
    sincos(ival, &s, &c);
    p = make_double2(expfac * c, expfac * s);
  }
  if ((n & 1) == 0 && k == n / 2) p.y = 0.0;
  for (int dd = 0; dd < bs.nds; ++dd) {
    const int d = bs.ds_begin + dd;
    const double sigma = sm * dsets[d].sigma_base;
    double2 o = p;
    if (sigma > 0 && k > 0) {
      const double sigfac = -0.5 * sigma * sigma;
      const double ef = exp(sigfac * wv * wv);
      o = make_double2(ef * p.x, ef * p.y);
    }
    reinterpret_cast<double2*>(pbuf + (static_cast<size_t>(w) * D + d) * 2 * nc)[k] = o;
  }
}

// ------------------------------------------------------------------
// Own FFT path (power-of-two n = 2m, m = m1 * 256, m1 in [8, 512]): the
// four-step real transform of fft1d.cuh with the R grid fill fused into the
// forward pass A, the real-transform split / merge fused into the spectrum
// kernel, and the inverse written straight into the P(D) rows.
constexpr int FRB = 16;   // rows per pass-B block

// Pass A: L1*L2-point DFTs down CB = 256/L2 columns of the m1 x 256 view
// (one DFT per thread in each stage), times W_m^{c b}, stored as rows
// Y[c][b].  Input rows are complex: for the forward transform the R grid
// itself, whose real values R_{2j}, R_{2j+1} are z_j.
template <int L1, int L2, int S>
__global__ void __launch_bounds__(256, 3)
k_fftA(int rowsz, int nrows_per_w, const int* __restrict__ mstatus,
       const double2* __restrict__ in, double2* __restrict__ out,
       const double2* __restrict__ WH, const double2* __restrict__ WL,
       const int* __restrict__ kcut) {
  constexpr int M1 = L1 * L2;
  constexpr int M2 = 256;
  constexpr int m = M1 * M2;
  constexpr int CB = 256 / L2;
  constexpr int NH = m / 128;
  extern __shared__ double2 fs[];  // [(n2 * L1 + k1) * CB + b], then H, L, T
  double2* Hs = fs + 256 * L1;
  const double2* Ls = Hs + NH;
  double2* Ts = Hs + NH + 128;  // inter-stage twiddles W_m^{(m / M1) n2 k1}
  const int row = blockIdx.y;
  if (mstatus[row / nrows_per_w] != 0) return;
  const int b0 = blockIdx.x * CB;
  const int t = threadIdx.x;
  const double2* src = in + static_cast<size_t>(row) * rowsz;
  double2* dst = out + static_cast<size_t>(row) * rowsz;
  double2 v[L1];
  {
    const int b = t % CB, n2 = t / CB;
    // inverse input: rows beyond the noise cut-off are zero and not read
    const int kc = kcut ? kcut[row] : m;
#pragma unroll
    for (int n1 = 0; n1 < L1; ++n1) {
      const int a = L2 * n1 + n2;
      v[n1] = row_cut(a, m, kc) ? make_double2(0.0, 0.0) : src[a * M2 + b0 + b];
    }
    fft::load_tw2(Hs, WH, WL, NH, t, 256);
    if (L2 > 1 && t < L1 * L2) Ts[t] = fft::tw2<S>(WH, WL, (m / M1) * (t / L1) * (t % L1));
    __syncthreads();
    fft::dft<L1, S>(v);
    if (L2 > 1) {
#pragma unroll
      for (int k1 = 0; k1 < L1; ++k1) {
        if (n2 * k1) v[k1] = fft::cmul(v[k1], Ts[n2 * L1 + k1]);
        fs[(n2 * L1 + k1) * CB + b] = v[k1];
      }
    } else {
#pragma unroll
      for (int k1 = 0; k1 < L1; ++k1) {
        const int bb = b0 + b;
        dst[k1 * M2 + bb] = (k1 * bb) ? fft::cmul(v[k1], fft::tw2<S>(Hs, Ls, k1 * bb)) : v[k1];
      }
    }
  }
  if (L2 > 1) {
    __syncthreads();
#pragma unroll
    for (int it = 0; it < L1 / L2; ++it) {
      const int e = t + 256 * it;
      const int b = e % CB, k1 = e / CB;
      double2 u[L2 > 1 ? L2 : 1];
#pragma unroll
      for (int n2 = 0; n2 < L2; ++n2) u[n2] = fs[(n2 * L1 + k1) * CB + b];
      fft::dft<L2, S>(u);
#pragma unroll
      for (int k2 = 0; k2 < L2; ++k2) {
        const int c = k1 + L1 * k2;
        const int bb = b0 + b;
        dst[c * M2 + bb] = (c * bb) ? fft::cmul(u[k2], fft::tw2<S>(Hs, Ls, c * bb)) : u[k2];
      }
    }
  }
}

// Forward pass A with the R grid fill fused in: each thread evaluates the
// R values of its inputs z_j = R_{2j} + i R_{2j+1} (GridFill1::point, as
// k_rfill1 does) straight into the registers of its first DFT, so the R grid
// is neither written to nor read back from memory.  Block partial moment
// sums go to rpart[row][blockIdx.x] (L2 tiles per row); R at grid index
// wrap - 1, which k_moments1 needs for its edge term, is stored at its place
// in rbuf -- pass B overwrites rbuf with the spectrum only after
// k_moments1 has read it.

template <int L1, int L2, bool RUNS>
__global__ void __launch_bounds__(256, RUNS ? 3 : 2)
k_fftAR(const BSet1Dev* __restrict__ bsets, int B, int NI, int rowsz,
        const int* __restrict__ mstatus, const double* __restrict__ spl,
        double* __restrict__ rbuf, double* __restrict__ rpart,
        double2* __restrict__ out, const double2* __restrict__ WH,
        const double2* __restrict__ WL) {
  constexpr int M1 = L1 * L2;
  constexpr int M2 = 256;
  constexpr int m = M1 * M2;
  constexpr int CB = 256 / L2;
  constexpr int NH = m / 128;
  extern __shared__ double2 fs[];  // [(n2 * L1 + k1) * CB + b], then H, L
  __shared__ dev::Exp2Table e2;
  __shared__ double shr[32];
  double2* Hs = fs + 256 * L1;
  const double2* Ls = Hs + NH;
  double2* Ts = Hs + NH + 128;  // inter-stage twiddles W_m^{(m / M1) n2 k1}
  const int row = blockIdx.y;
  const int w = row / B, bset = row - w * B;
  if (mstatus[w] != 0) return;
  const int b0 = blockIdx.x * CB;
  const int t = threadIdx.x;
  e2.load();
  if (!RUNS) {
    fft::load_tw2(Hs, WH, WL, NH, t, 256);
    if (L2 > 1 && t < L1 * L2) Ts[t] = fft::tw2<-1>(WH, WL, (m / M1) * (t / L1) * (t % L1));
  }
  __syncthreads();
  const BSet1Dev& bs = bsets[bset];
  const GridFill1 rg(bs, spl + static_cast<size_t>(row) * 2 * 4 * NI, NI, e2.t);
  const int* __restrict__ gidx = bs.gidx;
  const int iw = bs.wrapRidx - 1;
  double* Rrow = rbuf + static_cast<size_t>(row) * 2 * rowsz;
  double2* dst = out + static_cast<size_t>(row) * rowsz;
  double mn = 0.0, var = 0.0;
  double2 v[L1];
  {
    const int b = t % CB, n2 = t / CB;
    if (RUNS) {
      // the block's inputs are M1 row segments of 2 CB consecutive grid
      // points (segment r: [2 (256 r + b0), 2 (256 r + b0 + CB))); the
      // static runs covering them (bs.aruns, this block's slice) are
      // evaluated by running products into the padded staging area, which
      // spans the exchange buffer and the twiddle tables (loaded after)
      double* stage = reinterpret_cast<double*>(fs);
      const int* __restrict__ toff = bs.arun_off + blockIdx.x * 257;
      const int k1 = toff[t + 1];
      for (int k = toff[t]; k < k1; ++k) {
        const int2 d = __ldg(bs.aruns + k);
        const int len = (d.y >> 2) & 31, kind = d.y & 3, q = (d.y >> 8) - 1;
        const int o = (d.x >> 9) * (2 * CB) + (d.x & 511) - 2 * b0;
        if (kind == 2) {
          rg.run_products(d.x, len, q, stage, o, mn, var);
        } else if (kind == 1) {
          for (int e = 0; e < len; ++e) {
            const int i = d.x + e;
            stage[GridFill1::pad(o + e)] = rg.point(i, static_cast<double>(i), q, mn, var);
          }
        } else {
          for (int e = 0; e < len; ++e) stage[GridFill1::pad(o + e)] = 0.0;
        }
        if (iw >= d.x && iw < d.x + len) Rrow[iw] = stage[GridFill1::pad(o + iw - d.x)];
      }
      __syncthreads();
#pragma unroll
      for (int n1 = 0; n1 < L1; ++n1) {
        const int p = (L2 * n1 + n2) * (2 * CB) + 2 * b;
        v[n1] = make_double2(stage[GridFill1::pad(p)], stage[GridFill1::pad(p + 1)]);
      }
      __syncthreads();
      fft::load_tw2(Hs, WH, WL, NH, t, 256);
      if (L2 > 1 && t < L1 * L2) Ts[t] = fft::tw2<-1>(WH, WL, (m / M1) * (t / L1) * (t % L1));
      __syncthreads();
    } else {
#pragma unroll
      for (int n1 = 0; n1 < L1; ++n1) {
        const int i = 2 * ((L2 * n1 + n2) * M2 + b0 + b);
        const int2 q = __ldg(reinterpret_cast<const int2*>(gidx + i));
        const double di = static_cast<double>(i);
        const double r0 = rg.point(i, di, q.x, mn, var);
        const double r1 = rg.point(i + 1, di + 1.0, q.y, mn, var);
        if (i == iw) Rrow[i] = r0;
        if (i + 1 == iw) Rrow[i + 1] = r1;
        v[n1] = make_double2(r0, r1);
      }
    }
    fft::dft<L1, -1>(v);
    if (L2 > 1) {
#pragma unroll
      for (int k1 = 0; k1 < L1; ++k1) {
        if (n2 * k1) v[k1] = fft::cmul(v[k1], Ts[n2 * L1 + k1]);
        fs[(n2 * L1 + k1) * CB + b] = v[k1];
      }
    } else {
#pragma unroll
      for (int k1 = 0; k1 < L1; ++k1) {
        const int bb = b0 + b;
        dst[k1 * M2 + bb] = (k1 * bb) ? fft::cmul(v[k1], fft::tw2<-1>(Hs, Ls, k1 * bb)) : v[k1];
      }
    }
  }
  if (L2 > 1) {
    __syncthreads();
#pragma unroll
    for (int it = 0; it < L1 / L2; ++it) {
      const int e = t + 256 * it;
      const int b = e % CB, k1 = e / CB;
      double2 u[L2 > 1 ? L2 : 1];
#pragma unroll
      for (int n2 = 0; n2 < L2; ++n2) u[n2] = fs[(n2 * L1 + k1) * CB + b];
      fft::dft<L2, -1>(u);
#pragma unroll
      for (int k2 = 0; k2 < L2; ++k2) {
        const int c = k1 + L1 * k2;
        const int bb = b0 + b;
        dst[c * M2 + bb] = (c * bb) ? fft::cmul(u[k2], fft::tw2<-1>(Hs, Ls, c * bb)) : u[k2];
      }
    }
  }
  mn = dev::block_sum<256>(mn, shr);
  var = dev::block_sum<256>(var, shr);
  if (t == 0) {
    double* o = rpart + (static_cast<size_t>(row) * L2 + blockIdx.x) * 2;
    o[0] = mn;
    o[1] = var;
  }
}

// Pass B: 256-point DFTs along rows c0..c0+15 of Y (16 x 16 split), stored
// in natural order Z[c + m1 d].
template <int S>
__global__ void __launch_bounds__(256, 2)
k_fftB(int m1, int rowsz, int nrows_per_w, const int* __restrict__ mstatus,
       const double2* __restrict__ in, double2* __restrict__ out,
       const double2* __restrict__ WH, const double2* __restrict__ WL,
       const int* __restrict__ kcut) {
  extern __shared__ double2 fs[];  // [(k1 * 16 + n2) * 17 + r], then T
  double2* Ts = fs + 16 * 16 * 17;  // inter-stage twiddles W_256^{n2 k1} (symmetric)
  // blocks take the rows last-written-first: the tail of pass A's output is
  // still in L2 when this pass starts (and the P(D) scan after the inverse,
  // in natural order, then starts on this pass's last-written rows)
  const int row = gridDim.y - 1 - blockIdx.y;
  if (mstatus[row / nrows_per_w] != 0) return;
  const int rb = min(FRB, m1);
  const int c0 = (gridDim.x - 1 - blockIdx.x) * rb;
  const int m = m1 * 256;
  const int t = threadIdx.x;
  const double2* src = in + static_cast<size_t>(row) * rowsz;
  double2* dst = out + static_cast<size_t>(row) * rowsz;
  const int kc = kcut ? kcut[row] : m;
  double2 v[16];
  if (t < 16 * rb) {
    const int n2 = t & 15, r = t >> 4;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) v[n1] = src[(c0 + r) * 256 + 16 * n1 + n2];
  }
  Ts[t] = fft::tw2<S>(WH, WL, (m / 256) * (t >> 4) * (t & 15));
  __syncthreads();
  if (t < 16 * rb) {
    const int n2 = t & 15, r = t >> 4;
    fft::dft<16, S>(v);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
      if (n2 * k1) v[k1] = fft::cmul(v[k1], Ts[k1 * 16 + n2]);
      fs[(k1 * 16 + n2) * 17 + r] = v[k1];
    }
  }
  __syncthreads();
  if (t < 16 * rb) {
    const int r = t % rb, k1 = t / rb;
    double2 u[16];
#pragma unroll
    for (int n2 = 0; n2 < 16; ++n2) u[n2] = fs[(k1 * 16 + n2) * 17 + r];
    fft::dft<16, S>(u);
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
      // bins beyond the noise cut-off are never read (forward transform)
      const int k = (c0 + r) + m1 * (k1 + 16 * k2);
      if (min(k, m - k) <= kc) dst[k] = u[k2];
    }
  }
}

// The spectrum on bin pairs (q, m - q): the real-transform split X from Z,
// exp(X - X_0) with the mean shift, the noise factor per dataset (bins whose
// noise exponent is below -750 for every dataset are exactly 0, as in the
// reference), and the merge Z' of the inverse real transform, written into
// each dataset's row.  Wn[k] = e^{-2 pi i k / n}, k in [0, m].
__device__ __forceinline__ bool spec_all_zero(const BSet1Dev& bs, const DSet1Dev* dsets,
                                              double sm, double wv, int k) {
  if (k == 0) return false;
  for (int dd = 0; dd < bs.nds; ++dd) {
    const double sigma = sm * dsets[bs.ds_begin + dd].sigma_base;
    if (!(sigma > 0)) return false;
    const double sigfac = -0.5 * sigma * sigma;
    if (!(sigfac * wv * wv < -750.0)) return false;
  }
  return true;
}

__device__ __forceinline__ double2 spec_p(double2 X, double r0, int k, int m, bool doshift,
                                          double shiftw) {
  if (k == 0) return make_double2(1.0, 0.0);
  const double expfac = exp(X.x - r0);
  const double ival = doshift ? X.y - shiftw * static_cast<double>(k) : X.y;
  double s, c;
  sincos(ival, &s, &c);
  double2 p = make_double2(expfac * c, expfac * s);
  if (k == m) p.y = 0.0;
  return p;
}

__global__ void __launch_bounds__(NT, 4)
k_spectrum1f(const BSet1Dev* __restrict__ bsets, const DSet1Dev* __restrict__ dsets, int B,
             int D, int n, int rowsz, const int* __restrict__ mstatus,
             const double* __restrict__ sigmult, const double* __restrict__ mom,
             const double2* __restrict__ zbuf, double2* __restrict__ pbuf,
             const double2* __restrict__ Wn, const int* __restrict__ kcut_set,
             const int* __restrict__ kcut_ds) {
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  const int m = n / 2;
  const BSet1Dev& bs = bsets[b];
  const double iflux = dev::kTwoPi / (static_cast<double>(n) * bs.dflux);
  const double sm = sigmult[w];
  const double* mo = mom + static_cast<size_t>(wb) * 4;
  const bool doshift = mo[3] != 0.0;
  const double shiftw = mo[2] * iflux;
  const double2* Z = zbuf + static_cast<size_t>(wb) * rowsz;
  // pairs up to the widest cut-off of the set plus one row of 256 bins cover
  // every bin of a row the inverse transform reads (at either end)
  const int qmax = min(m / 2, kcut_set[wb] + 256);
  for (int q = blockIdx.x * NT + threadIdx.x; q <= qmax; q += gridDim.x * NT) {
    const int ka = q, kb = (q == 0) ? m : m - q;  // bins of the pair
    const bool za = spec_all_zero(bs, dsets, sm, iflux * ka, ka);
    const bool zb = spec_all_zero(bs, dsets, sm, iflux * kb, kb);
    double2 pa = make_double2(0.0, 0.0), pb = make_double2(0.0, 0.0);
    if (!(za && zb)) {
      const double2 z0 = Z[0];
      const double r0 = z0.x + z0.y;  // X_0
      double2 Xa, Xb;
      if (q == 0) {
        Xa = make_double2(r0, 0.0);
        Xb = make_double2(z0.x - z0.y, 0.0);  // X_m
      } else {
        const double2 a = Z[q], c = Z[m - q];
        // E_k = (Z_k + conj Z_{m-k}) / 2, O_k = (Z_k - conj Z_{m-k}) / (2i)
        const double2 Ea = make_double2(0.5 * (a.x + c.x), 0.5 * (a.y - c.y));
        const double2 Oa = make_double2(0.5 * (a.y + c.y), -0.5 * (a.x - c.x));
        const double2 Eb = make_double2(Ea.x, -Ea.y);
        const double2 Ob = make_double2(0.5 * (c.y + a.y), -0.5 * (c.x - a.x));
        Xa = fft::cadd(Ea, fft::cmul(__ldg(Wn + q), Oa));
        Xb = fft::cadd(Eb, fft::cmul(__ldg(Wn + m - q), Ob));
      }
      if (!za) pa = spec_p(Xa, r0, ka, m, doshift, shiftw);
      if (!zb) pb = spec_p(Xb, r0, kb, m, doshift, shiftw);
    }
    for (int dd = 0; dd < bs.nds; ++dd) {
      const int d = bs.ds_begin + dd;
      const double sigma = sm * dsets[d].sigma_base;
      double2 Pa = pa, Pb = pb;
      if (sigma > 0) {
        const double sigfac = -0.5 * sigma * sigma;
        if (ka > 0) {
          const double wv = iflux * ka;
          const double ef = exp(sigfac * wv * wv);
          Pa = make_double2(ef * pa.x, ef * pa.y);
        }
        const double wv = iflux * kb;
        const double ef = exp(sigfac * wv * wv);
        Pb = make_double2(ef * pb.x, ef * pb.y);
      }
      double2* out = pbuf + static_cast<size_t>(w * D + d) * rowsz;
      // rows the inverse transform does not read (every bin beyond the noise
      // cut-off, hence zero) are not written
      const int kc = kcut_ds[static_cast<size_t>(w) * D + d];
      // Z'_k = (P_k + conj P_{m-k}) + i (P_k - conj P_{m-k}) e^{+2 pi i k / n}
      if (!row_cut(ka >> 8, m, kc)) {
        const double2 e = make_double2(Pa.x + Pb.x, Pa.y - Pb.y);
        const double2 o = fft::cmul(make_double2(Pa.x - Pb.x, Pa.y + Pb.y), fft::conj(__ldg(Wn + ka)));
        out[ka] = make_double2(e.x - o.y, e.y + o.x);
      }
      if (q != 0 && kb != ka && !row_cut(kb >> 8, m, kc)) {
        const double2 e = make_double2(Pb.x + Pa.x, Pb.y - Pa.y);
        const double2 o = fft::cmul(make_double2(Pb.x - Pa.x, Pb.y + Pa.y), fft::conj(__ldg(Wn + kb)));
        out[kb] = make_double2(e.x - o.y, e.y + o.x);
      }
    }
  }
}

struct SplitParams {
  double sgpos, sgneg, n1sigpos, n1signeg;
  long long botidx, topidx;
};

constexpr int kSearchPer = 8;  // values per thread per window of the split search

__device__ __forceinline__ long long to_index(double v) {
  // (int) conversion of the reference, saturated so that huge values stay
  // out of range instead of wrapping.
  if (!(v < 9.0e15)) return 0x7fffffffffffLL;
  if (!(v > -9.0e15)) return -0x7fffffffffffLL;
  return static_cast<long long>(v);
}

__device__ __forceinline__ SplitParams split_params(const BSet1Dev& bs,
                                                    double var, double sigma) {
  SplitParams sp;
  sp.sgpos = sqrt(var + sigma * sigma);
  sp.sgneg = (9 * sigma * sigma > var) ? sigma : sp.sgpos;
  sp.n1sigpos = 2.5 * sp.sgpos;
  sp.n1signeg = 2.5 * sp.sgneg;
  sp.botidx = to_index(sp.n1sigpos / bs.dflux);
  if (sp.n1sigpos > fabs(bs.minflux_R))
    sp.topidx = bs.wrapRidx;
  else
    sp.topidx = to_index(-(sp.n1signeg + bs.minflux_R) / bs.dflux + bs.wrapRidx + 1);
  return sp;
}

__device__ __forceinline__ double clip0(double v) { return (v < 0) ? 0.0 : v; }

// Chunk reductions over the P(D) after the inverse transform: peak, sum,
// index-weighted sum and the minimum inside the split search window
// (PDFactory.cc:779-815, PD.cc:123-140, 245-274).
__global__ void __launch_bounds__(NT)
k_pscan1(const BSet1Dev* __restrict__ bsets, const DSet1Dev* __restrict__ dsets,
         int B, int D, int n, int nc2, int nchunk,
         const int* __restrict__ mstatus, const double* __restrict__ sigmult,
         const double* __restrict__ mom, const double* __restrict__ pbuf,
         double* __restrict__ ppart, int* __restrict__ pmidx) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  const int wd = blockIdx.y;
  const int w = wd / D, d = wd - w * D;
  if (mstatus[w] != 0) return;
  const DSet1Dev& ds = dsets[d];
  const BSet1Dev& bs = bsets[ds.bs];
  const double var = mom[(static_cast<size_t>(w) * B + ds.bs) * 4 + 1];
  const SplitParams sp = split_params(bs, var, sigmult[w] * ds.sigma_base);
  const double* p = pbuf + static_cast<size_t>(wd) * nc2;
  const int base = blockIdx.x * CHUNK;
  constexpr int PER2 = CHUNK / NT / 2;  // double2 loads per thread
  double2 v[PER2];
#pragma unroll
  for (int k = 0; k < PER2; ++k) {
    const int i = base + 2 * (k * NT + threadIdx.x);
    v[k] = (i < n) ? *reinterpret_cast<const double2*>(p + i) : make_double2(-1.0, -1.0);
  }
  double mx = 0.0, sum = 0.0, wsum = 0.0, mnv = 1.0e308;
  int mni = 0x7fffffff;
  bool any = false;
#pragma unroll
  for (int k = 0; k < PER2; ++k) {
    const int li = 2 * (k * NT + threadIdx.x);
    const int i = base + li;
    if (i >= n) break;
    const double xa = clip0(v[k].x);
    if (!any || xa > mx) mx = xa;
    any = true;
    sum += xa;
    wsum += static_cast<double>(li) * xa;
    if (i >= sp.botidx && i <= sp.topidx) dev::argmin_merge(mnv, mni, xa, i);
    if (i + 1 < n) {  // odd n: the row's last pair has one element
      const double xb = clip0(v[k].y);
      if (xb > mx) mx = xb;
      sum += xb;
      wsum += static_cast<double>(li + 1) * xb;
      if (i + 1 >= sp.botidx && i + 1 <= sp.topidx) dev::argmin_merge(mnv, mni, xb, i + 1);
    }
  }
  if (!any) mx = -1.0e308;
  // the four block reductions in one shared-memory round, each with the
  // butterfly trees of dev::block_max / block_sum / block_argmin (the same
  // results, one barrier instead of a dozen)
  for (int o = 16; o > 0; o >>= 1) {
    mx = dev::dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    const double v2 = __shfl_xor_sync(0xffffffffu, mnv, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, mni, o);
    dev::argmin_merge(mnv, mni, v2, i2);
  }
  const int wp = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    shd[wp] = mx;
    shd[8 + wp] = sum;
    shd[16 + wp] = wsum;
    shd[24 + wp] = mnv;
    shi[wp] = mni;
  }
  __syncthreads();
  if (wp == 0) {
    static_assert(NT / 32 <= 8, "one shared slot per warp");
    const bool in = l < NT / 32;
    mx = in ? shd[l] : -1.0e308;
    sum = in ? shd[8 + l] : 0.0;
    wsum = in ? shd[16 + l] : 0.0;
    mnv = in ? shd[24 + l] : 1.0e308;
    mni = in ? shi[l] : 0x7fffffff;
    for (int o = 16; o > 0; o >>= 1) {
      mx = dev::dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
      wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
      const double v2 = __shfl_xor_sync(0xffffffffu, mnv, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, mni, o);
      dev::argmin_merge(mnv, mni, v2, i2);
    }
    if (l == 0) {
      double* o = ppart + (static_cast<size_t>(wd) * nchunk + blockIdx.x) * 4;
      o[0] = mx;
      o[1] = sum;
      o[2] = wsum;
      o[3] = mnv;
      pmidx[static_cast<size_t>(wd) * nchunk + blockIdx.x] = mni;
    }
  }
}

__device__ __forceinline__ double logp_at(const double* __restrict__ p, int n,
                                          int split, double itot, int j) {
  int s = j + split;
  if (s >= n) s -= n;
  const double v = clip0(p[s]) * itot;
  return (v > 0.0) ? log2(v) : dev::kSmallLogVal;
}

// Split point, unwrap, normalisation, mean and the log-likelihood of one
// (proposal, dataset): PDFactory.cc:691-1009, PD.cc:146-274, 557-677,
// calcLike.cc:419-425.
__global__ void __launch_bounds__(NT)
k_pfinish1(const BSet1Dev* __restrict__ bsets,
           const DSet1Dev* __restrict__ dsets, int B, int D, int n, int nc2,
           int nchunk, double log2toe, const int* __restrict__ mstatus,
           const double* __restrict__ sigmult, const double* __restrict__ mom,
           const double* __restrict__ pbuf, const double* __restrict__ ppart,
           const int* __restrict__ pmidx, PDInfo1* __restrict__ pinfo) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  __shared__ int s_state;   // 0 need search, 1 done, <0 error
  __shared__ int s_split;
  __shared__ double s_jitter;
  const int wd = blockIdx.x;
  const int w = wd / D, d = wd - w * D;
  PDInfo1& info = pinfo[wd];
  if (mstatus[w] != 0) {
    if (threadIdx.x == 0) info.status = mstatus[w];
    return;
  }
  const DSet1Dev& ds = dsets[d];
  const BSet1Dev& bs = bsets[ds.bs];
  const double var = mom[(static_cast<size_t>(w) * B + ds.bs) * 4 + 1];
  const SplitParams sp = split_params(bs, var, sigmult[w] * ds.sigma_base);
  const double* p = pbuf + static_cast<size_t>(wd) * nc2;
  const double dflux = bs.dflux;
  const double* pp = ppart + static_cast<size_t>(wd) * nchunk * 4;
  const int* pm = pmidx + static_cast<size_t>(wd) * nchunk;

  if (threadIdx.x == 0) {
    int st = 0;
    int split = -1;
    double jitter = 0.0;
    const double fluxrange = n * dflux;
    double peak = -1.0e308, minval = 1.0e308;
    int minidx = 0x7fffffff;
    for (int c = 0; c < nchunk; ++c) {
      if (pp[4 * c] > peak) peak = pp[4 * c];
      dev::argmin_merge(minval, minidx, pp[4 * c + 3], pm[c]);
    }
    const long long botidx = sp.botidx, topidx = sp.topidx;
    if (sp.sgpos <= 0 || sp.sgneg <= 0) st = POFD_E_SPLIT_RANGE;
    else if (fluxrange < (sp.n1sigpos + sp.n1signeg)) st = POFD_E_SPLIT_RANGE;
    // a NaN peak (non-finite P(D)) is reported here too, where the
    // reference would carry the NaN on to its un-shift check
    else if (!(peak > 0.0)) st = POFD_E_SPLIT_PEAK;
    else if (botidx >= n || topidx >= n || botidx < 0 || topidx < 0) st = POFD_E_SPLIT_LOGIC;
    if (st == 0) {
      if (botidx > topidx) {
        minidx = static_cast<int>(botidx);
        minval = clip0(p[minidx]);
      }
      if (minidx < 0 || minidx >= n) st = POFD_E_SPLIT_MIN;  // no finite minimum
      else if (minval > 1e-5 * peak) st = POFD_E_SPLIT_MIN;
    }
    if (st == 0) {
      const int pre = 17;
      bool found = false;
      if (minidx > pre) {
        bool mono = true;
        const int initidx = minidx - pre;
        double prevval = clip0(p[initidx]);
        jitter = prevval;
        for (int i = initidx + 1; i < minidx; ++i) {
          const double cv = clip0(p[i]);
          if (cv >= prevval) mono = false;
          jitter += cv;
          prevval = cv;
        }
        if (mono) { split = minidx; found = true; }
        else {
          jitter += minval;
          jitter = 1.1 * jitter / static_cast<double>(pre + 1);
        }
      } else {
        jitter = 5e-14 * peak;
        if (minval > jitter) { split = minidx; found = true; }
      }
      if (!found) {
        if (minval <= 0.0) {
          const int nminup = 3;
          long long bi, ti;
          if (minidx < botidx) bi = botidx; else bi = minidx - nminup;
          if (minidx > topidx - nminup) ti = topidx - nminup; else ti = minidx + nminup;
          if (bi < 0) bi = 0;
          for (long long i = bi; i < ti; ++i) {
            const double cv = clip0(p[i]);
            if (cv > minval) minval = cv;
          }
        }
        if (minval > 0) jitter = (5.0 * minval) < jitter ? (5.0 * minval) : jitter;
        if (botidx >= topidx) st = POFD_E_SPLIT_LOGIC;
        else if (clip0(p[topidx]) < jitter) st = POFD_E_SPLIT_TOP;
      }
      if (st == 0 && found) { s_state = 1; s_split = split; }
      else if (st == 0) { s_state = 0; s_jitter = jitter; }
    }
    if (st != 0) s_state = st;
  }
  __syncthreads();
  int state = s_state;
  if (state == 0) {
    // search down from topidx-1 for the first value below the jitter level:
    // windows of kSearchPer * NT values from the top, each thread's loads
    // issued together; the highest hit of the first window with one is the
    // first hit of the element-by-element search
    const double jitter = s_jitter;
    int found = -1;
    for (long long top = sp.topidx - 1; top >= sp.botidx; top -= NT * kSearchPer) {
      double pv[kSearchPer];
#pragma unroll
      for (int k = 0; k < kSearchPer; ++k) {
        const long long i = top - threadIdx.x - static_cast<long long>(NT) * k;
        pv[k] = (i >= sp.botidx) ? p[i] : 1.0e308;
      }
      int hit = -1;
#pragma unroll
      for (int k = kSearchPer - 1; k >= 0; --k) {
        const long long i = top - threadIdx.x - static_cast<long long>(NT) * k;
        if (i >= sp.botidx && clip0(pv[k]) < jitter) hit = static_cast<int>(i);
      }
      const int m = dev::block_max_int<NT>(hit, shi);
      if (m >= 0) { found = m; break; }
    }
    if (found >= 0) { state = 1; if (threadIdx.x == 0) s_split = found + 1; }
    else state = POFD_E_SPLIT_NONE;
    __syncthreads();
  }
  if (state < 0) {
    if (threadIdx.x == 0) {
      info.status = state;
      info.ll = 0.0;
    }
    return;
  }
  const int split = s_split;
  // Sum below the split: whole chunks from the partials, the rest read.
  const int cfull = split / CHUNK;
  double part = 0.0;
  for (int i = cfull * CHUNK + threadIdx.x; i < split; i += NT) part += clip0(p[i]);
  part = dev::block_sum<NT>(part, shd);
  double S = 0.0, W = 0.0, T = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    S += pp[4 * c + 1];
    W += static_cast<double>(c) * CHUNK * pp[4 * c + 1] + pp[4 * c + 2];
    if (c < cfull) T += pp[4 * c + 1];
  }
  T += part;
  const double q0 = clip0(p[split]);
  const double qlast = clip0(p[split == 0 ? n - 1 : split - 1]);
  const double tot = (S - 0.5 * q0 - 0.5 * qlast) * dflux;
  const double itot = 1.0 / tot;
  const double srot = W - static_cast<double>(split) * S + static_cast<double>(n) * T;
  const double msum = itot * (srot - 0.5 * static_cast<double>(n - 1) * qlast);
  const double tmn = msum * dflux * dflux;
  if (isinf(tmn) || isnan(tmn)) {
    if (threadIdx.x == 0) { info.status = POFD_E_UNSHIFT; info.ll = 0.0; }
    return;
  }
  const double minflux = -tmn;
  const double maxflux = minflux + static_cast<double>(n - 1) * dflux;
  const double maxfluxval = maxflux - dflux;
  const double idflux = 1.0 / dflux;
  double ll = 0.0;
  if (ds.binned) {
    for (int e = threadIdx.x; e < ds.nnz; e += NT) {
      const double cnt = ds.nzcnt[e];
      const double cflux = ds.bincent0 + static_cast<double>(ds.nzidx[e]) * ds.bindelta;
      double v;
      if (cflux < minflux) v = cnt * logp_at(p, n, split, itot, 0);
      else if (cflux > maxfluxval) v = cnt * logp_at(p, n, split, itot, n - 1);
      else {
        const double delt = (cflux - minflux) * idflux;
        const int idx = static_cast<int>(delt);
        const double t = delt - static_cast<double>(idx);
        v = ((1.0 - t) * logp_at(p, n, split, itot, idx) +
             t * logp_at(p, n, split, itot, idx + 1)) * cnt;
      }
      ll += v;
    }
  } else {
    for (int e = threadIdx.x; e < ds.nnz; e += NT) {
      const double cflux = ds.flux[e];
      double v;
      if (cflux <= minflux) v = logp_at(p, n, split, itot, 0);
      else if (cflux >= maxfluxval) v = logp_at(p, n, split, itot, n - 1);
      else {
        const double delt = (cflux - minflux) * idflux;
        const int idx = static_cast<int>(delt);
        const double t = delt - static_cast<double>(idx);
        v = (1.0 - t) * logp_at(p, n, split, itot, idx) +
            t * logp_at(p, n, split, itot, idx + 1);
      }
      ll += v;
    }
  }
  ll = dev::block_sum<NT>(ll, shd);
  if (threadIdx.x == 0) {
    info.status = 0;
    info.split = split;
    info.itot = itot;
    info.minflux = minflux;
    info.sgpos = sp.sgpos;
    info.sgneg = sp.sgneg;
    info.ll = (log2toe * ll - ds.like_offset) / ds.like_norm;
  }
}

// Per-proposal sum over beam sets and datasets in the reference's order;
// a negative sigma multiplier gives bad_like for the beam set
// (calcLike.cc:404, 916-920).
__global__ void k_reduce1(const BSet1Dev* __restrict__ bsets, int B, int D,
                          int nprop, const int* __restrict__ mstatus,
                          const double* __restrict__ sigmult,
                          const PDInfo1* __restrict__ pinfo, Prior1 pr,
                          const double* __restrict__ bonus,
                          double* __restrict__ logl, int* __restrict__ status) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nprop) return;
  if (mstatus[w] != 0) {
    logl[w] = __longlong_as_double(0x7ff8000000000000LL);
    status[w] = mstatus[w];
    return;
  }
  const double sm = sigmult[w];
  double LogLike = 0.0;
  int st = 0;
  for (int b = 0; b < B; ++b) {
    const BSet1Dev& bs = bsets[b];
    if (bs.maxsb * sm < 0.0) { LogLike += 1e25; continue; }
    double s = 0.0;
    for (int dd = 0; dd < bs.nds; ++dd) {
      const PDInfo1& in = pinfo[static_cast<size_t>(w) * D + bs.ds_begin + dd];
      if (in.status != 0 && st == 0) st = in.status;
      s += in.ll;
    }
    LogLike += s;
  }
  // priors, once for all data sets (calcLike.cc:918-952)
  constexpr double half_log_2pi = 0.918938517570495605469;
  if (pr.has_sigma) {
    const double val = (sm - 1.0) / pr.sigma_width;
    LogLike -= half_log_2pi + pr.log_sigma_width + 0.5 * val * val;
  }
  if (pr.has_cfirb) {
    const double val = (pr.cfirb_mean - bonus[4 * static_cast<size_t>(w)]) / pr.cfirb_sigma;
    LogLike -= half_log_2pi + pr.log_cfirb_sigma + 0.5 * val * val;
  }
  if (pr.has_poisson) {
    const double val = (pr.poisson_mean - bonus[4 * static_cast<size_t>(w) + 1]) / pr.poisson_sigma;
    LogLike -= half_log_2pi + pr.log_poisson_sigma + 0.5 * val * val;
  }
  if (pr.alpha > 0.0) LogLike += pr.alpha * bonus[4 * static_cast<size_t>(w) + 2];
  status[w] = st;
  logl[w] = (st == 0) ? LogLike : __longlong_as_double(0x7ff8000000000000LL);
}

// Bonus integrals and the slope penalty of each proposal's knot model, one
// block per proposal.  <S> and <S^2> are the integrals of S dN/dS and
// S^2 dN/dS over [S_0, S_{K-1}) (numberCountsKnotsSpline.cc:300-343, the
// integrand of numberCountsKnotsSpline.cc:646-670), by Gauss-Legendre
// quadrature in u = log2 S on host-built nodes: the integrand
// s^{a+1} 2^{spline(u)} is smooth inside each knot interval.  The penalty is
// minus the sum of squared deviations of the log2-log2 knot slopes from their
// mean (numberCountsKnotsSpline.cc:540-559), before the factor alpha.
// out[w][4] = {<S>, <S^2>, penalty, 0}, NaN for an invalid model.  With cnt
// the spline comes from the model kernel of the same batch; without it the
// block solves it.  fill_at >= 0 also stores <S>, <S^2> as floats in
// theta[w][fill_at .. fill_at + 1] (fillBonusParams, calcLike.cc:958-980).
constexpr int kBonusThreads = 256;
__global__ void __launch_bounds__(kBonusThreads)
k_bonus1(Model1Dev m, float* theta, int npar, double logfac,
         const double* __restrict__ cnt, const int* __restrict__ mstatus,
         const double* __restrict__ qu, const double* __restrict__ qs,
         const double* __restrict__ qw, int nper, double* __restrict__ out,
         int fill_at) {
  __shared__ double cs[4 * KMAX];
  __shared__ double lk[KMAX];
  __shared__ double wk[8 * KMAX];
  __shared__ double red[2][kBonusThreads / 32];
  __shared__ int sst;
  const int w = blockIdx.x;
  const int K = m.K;
  const float* th = theta + static_cast<size_t>(w) * npar;
  for (int i = threadIdx.x; i < K; i += blockDim.x) lk[i] = m.logknots[i];
  if (threadIdx.x == 0) sst = cnt ? mstatus[w] : model_solve(m, th, logfac, cs, wk);
  __syncthreads();
  if (cnt && sst == 0)
    for (int i = threadIdx.x; i < 4 * (K - 1); i += blockDim.x)
      cs[i] = cnt[static_cast<size_t>(w) * 4 * KMAX + i];
  __syncthreads();
  double s1 = 0.0, s2 = 0.0;
  if (sst == 0) {
    const int nq = (K - 1) * nper;
    for (int j = threadIdx.x; j < nq; j += blockDim.x) {
      const int k = j / nper;
      const double d = qu[j] - lk[k];
      const double* q = cs + 4 * k;
      const double S = qs[j];
      const double a = qw[j] * S * S * exp2(q[0] + d * (q[1] + d * (q[2] + d * q[3])));
      s1 += a;
      s2 += a * S;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = s1;
    red[1][threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double qnan = __longlong_as_double(0x7ff8000000000000LL);
  double t1 = 0.0, t2 = 0.0, pen = 0.0;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) {
    t1 += red[0][i];
    t2 += red[1][i];
  }
  if (sst != 0 || K < 2) {
    t1 = t2 = qnan;
    pen = (sst != 0) ? qnan : 0.0;
  } else {
    double mean_deriv = 0.0;
    for (int i = 1; i < K; ++i)
      mean_deriv += (logfac * static_cast<double>(th[i]) -
                     logfac * static_cast<double>(th[i - 1])) / (lk[i] - lk[i - 1]);
    mean_deriv /= static_cast<double>(K - 1);
    for (int i = 1; i < K; ++i) {
      const double dl = (logfac * static_cast<double>(th[i]) -
                         logfac * static_cast<double>(th[i - 1])) / (lk[i] - lk[i - 1]) -
                        mean_deriv;
      pen -= dl * dl;
    }
  }
  if (out) {
    double* o = out + 4 * static_cast<size_t>(w);
    o[0] = t1;
    o[1] = t2;
    o[2] = pen;
    o[3] = 0.0;
  }
  if (fill_at >= 0) {
    float* tw = theta + static_cast<size_t>(w) * npar;
    tw[fill_at] = static_cast<float>(t1);
    tw[fill_at + 1] = static_cast<float>(t2);
  }
}

// The unwrapped, normalised (optionally log2) P(D) of one row.
__global__ void k_pdwrite1(const double* __restrict__ p, int n, int split,
                           double itot, int setlog, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = i + split;
  if (s >= n) s -= n;
  const double v = clip0(p[s]) * itot;
  out[i] = setlog ? ((v > 0.0) ? log2(v) : dev::kSmallLogVal) : v;
}

template <class T>
T* dalloc(size_t n) {
  void* p = nullptr;
  cuda_check(cudaMalloc(&p, n * sizeof(T) + 16), "cudaMalloc");
  return static_cast<T*>(p);
}

}  // namespace

// ===================================================================== host

namespace {
// exchange (256 L1 entries) plus the twiddle tables: H has m / 128 = 2 m1
// entries, L 128, the inter-stage table L1 L2 = m1; and at least the padded
// staging area of the run-based fill, which spans the exchange buffer and
// the tables (512 L1 values, one pad word per 16: 544 L1 doubles).  73.7 KB
// at m1 = 128: three blocks per SM fit.
constexpr size_t kFftASmemMax = (256 * 16 + 2 * 256 + 128 + 256) * sizeof(double2);
inline size_t fftA_smem(int m1) {
  const size_t l1 = static_cast<size_t>(m1 < 16 ? m1 : 16);
  const size_t tables = (256 * l1 + 2 * static_cast<size_t>(m1) + 128 + m1) * sizeof(double2);
  const size_t staging = 544 * l1 * sizeof(double);
  return tables > staging ? tables : staging;
}

template <int S>
void launch_fftA(int m1, int rows, cudaStream_t st, int rowsz, int nrw, const int* mstatus,
                 const double2* in, double2* out, const double2* WH, const double2* WL,
                 const int* kcut) {
#define POFD_FFTA(L1, L2)                                                              \
  k_fftA<L1, L2, S><<<dim3(L2, rows), 256, fftA_smem(m1), st>>>(rowsz, nrw, mstatus, in, out, \
                                                                WH, WL, kcut)
  switch (m1) {
    case 8: POFD_FFTA(8, 1); break;
    case 16: POFD_FFTA(16, 1); break;
    case 32: POFD_FFTA(16, 2); break;
    case 64: POFD_FFTA(16, 4); break;
    case 128: POFD_FFTA(16, 8); break;
    case 256: POFD_FFTA(16, 16); break;
    default: throw Error(POFD_E_ARG, "own FFT: unsupported size");
  }
#undef POFD_FFTA
}

// Fused R fill + forward pass A; returns the tiles per row (partial
// moment sums per row in rpart).
int launch_fftAR(int m1, bool runs, int rows, cudaStream_t st, const BSet1Dev* bsets, int B,
                 int NI, int rowsz, const int* mstatus, const double* spl, double* rbuf,
                 double* rpart, double2* out, const double2* WH, const double2* WL) {
#define POFD_FFTAR(L1, L2)                                                                  \
  if (runs)                                                                                 \
    k_fftAR<L1, L2, true><<<dim3(L2, rows), 256, fftA_smem(m1), st>>>(                      \
        bsets, B, NI, rowsz, mstatus, spl, rbuf, rpart, out, WH, WL);                       \
  else                                                                                      \
    k_fftAR<L1, L2, false><<<dim3(L2, rows), 256, fftA_smem(m1), st>>>(                     \
        bsets, B, NI, rowsz, mstatus, spl, rbuf, rpart, out, WH, WL);                       \
  return L2
  switch (m1) {
    case 8: POFD_FFTAR(8, 1);
    case 16: POFD_FFTAR(16, 1);
    case 32: POFD_FFTAR(16, 2);
    case 64: POFD_FFTAR(16, 4);
    case 128: POFD_FFTAR(16, 8);
    case 256: POFD_FFTAR(16, 16);
    default: throw Error(POFD_E_ARG, "own FFT: unsupported size");
  }
#undef POFD_FFTAR
}

template <bool RUNS>
void fftAR_attr_runs() {
  const int sm = static_cast<int>(kFftASmemMax);
  // the run-based fill fits three blocks per SM (80 registers, 73.7 KB of
  // dynamic shared memory at m1 = 128) when the carve-out is all shared
  if (RUNS) {
    const int c = cudaSharedmemCarveoutMaxShared;
    cuda_check(cudaFuncSetAttribute(k_fftAR<16, 8, RUNS>, cudaFuncAttributePreferredSharedMemoryCarveout, c), "attr");
    cuda_check(cudaFuncSetAttribute(k_fftAR<16, 4, RUNS>, cudaFuncAttributePreferredSharedMemoryCarveout, c), "attr");
    cuda_check(cudaFuncSetAttribute(k_fftAR<16, 2, RUNS>, cudaFuncAttributePreferredSharedMemoryCarveout, c), "attr");
  }
  cuda_check(cudaFuncSetAttribute(k_fftAR<8, 1, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftAR<16, 1, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftAR<16, 2, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftAR<16, 4, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftAR<16, 8, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftAR<16, 16, RUNS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
}

void fftAR_attr() {
  fftAR_attr_runs<false>();
  fftAR_attr_runs<true>();
}

template <int S>
void fftA_attr() {
  const int sm = static_cast<int>(kFftASmemMax);
  {
    const int c = cudaSharedmemCarveoutMaxShared;
    cuda_check(cudaFuncSetAttribute(k_fftA<16, 8, S>, cudaFuncAttributePreferredSharedMemoryCarveout, c), "attr");
    cuda_check(cudaFuncSetAttribute(k_fftA<16, 4, S>, cudaFuncAttributePreferredSharedMemoryCarveout, c), "attr");
    cuda_check(cudaFuncSetAttribute(k_fftA<16, 2, S>, cudaFuncAttributePreferredSharedMemoryCarveout, c), "attr");
  }
  cuda_check(cudaFuncSetAttribute(k_fftA<8, 1, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftA<16, 1, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftA<16, 2, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftA<16, 4, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftA<16, 8, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
  cuda_check(cudaFuncSetAttribute(k_fftA<16, 16, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr");
}

constexpr size_t kFftBSmemMax = (16 * 16 * 17 + 256) * sizeof(double2);

// pass B: the exchange and the inter-stage table (its twiddles are W_256
// powers only)
inline size_t fftB_smem(int) { return kFftBSmemMax; }
}  // namespace


Engine1::Engine1(int device, cudaStream_t stream)
    : device_(device), stream_(stream) {}

Engine1::~Engine1() {
  if (device_ < 0) return;  // host-only: nothing was allocated on a GPU
  cudaSetDevice(device_);
  drop_graphs();
  for (auto& kv : plans_) {
    if (kv.second.fwd) { fftwork_.forget(kv.second.fwd); cufftDestroy(kv.second.fwd); }
    if (kv.second.inv) { fftwork_.forget(kv.second.inv); cufftDestroy(kv.second.inv); }
  }
  free_work();
  free_static();
}

void Engine1::configure(unsigned nknots, const double* knotpos,
                        unsigned fftsize, unsigned ninterp, bool bin_data,
                        unsigned nbins) {
  if (nknots < 3 || nknots > static_cast<unsigned>(KMAX))
    throw Error(POFD_E_ARG, "nknots must be in [3, 64]");
  for (unsigned i = 0; i < nknots; ++i)
    if (!(knotpos[i] > 0) || (i > 0 && !(knotpos[i] > knotpos[i - 1])))
      throw Error(POFD_E_ARG, "knot positions must be positive and increasing");
  if (fftsize < 64) throw Error(POFD_E_ARG, "fftsize must be >= 64");
  if (ninterp < 4 || ninterp > 8192) throw Error(POFD_E_ARG, "ninterp must be in [4, 8192]");
  knots_.assign(knotpos, knotpos + nknots);
  n_ = fftsize;
  ninterp_ = ninterp;
  bin_data_ = bin_data;
  nbins_ = nbins;
  static_ok_ = false;
}

int Engine1::add_beamset(const Beam1& bm, double exp_conf) {
  HostSet s;
  s.bm = bm;
  s.exp_conf = exp_conf;
  sets_.push_back(std::move(s));
  static_ok_ = false;
  return static_cast<int>(sets_.size()) - 1;
}

void Engine1::refresh_set(HostSet& s) {
  s.maxsb = s.sb[0];
  for (size_t i = 1; i < s.sb.size(); ++i)
    if (s.sb[i] > s.maxsb) s.maxsb = s.sb[i];
  for (size_t i = 0; i < s.data.size(); ++i) {
    const double var = s.sb[i] * s.sb[i] + s.exp_conf * s.exp_conf;
    if (var > 0) {
      const double ndd = static_cast<double>(s.data[i].count());
      s.lo[i] = -0.5 * ndd * (std::log(kTwoPi * var) + 1.0);
    }
  }
  auto mm = s.data[0].minmax();
  s.minDF = mm.first;
  s.maxDF = mm.second;
  for (size_t i = 1; i < s.data.size(); ++i) {
    mm = s.data[i].minmax();
    if (mm.first < s.minDF) s.minDF = mm.first;
    if (mm.second > s.maxDF) s.maxDF = mm.second;
  }
  s.rr_set = false;
}

void Engine1::add_dataset(int bs, const double* data, size_t nd, bool meansub,
                          double sigma_base, double like_norm) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  if (nd == 0) throw Error(POFD_E_ARG, "No pixels in data");
  HostSet& s = sets_[bs];
  Data1 d;
  d.data.assign(data, data + nd);
  if (meansub) d.meanSubtract();
  if (bin_data_) d.applyBinning(nbins_);
  s.data.push_back(std::move(d));
  s.sb.push_back(sigma_base);
  s.lo.push_back(0.0);
  s.ln.push_back(like_norm);
  refresh_set(s);
  static_ok_ = false;
}

// A dataset whose pixels are in device memory: mean subtraction and binning
// on the GPU (ingest_bin1, bit-identical to the host path), only the counts
// come back.  Unbinned likelihoods take the (mean-subtracted) pixels back.
void Engine1::add_dataset_device(int bs, double* data_dev, size_t nd, bool meansub,
                                 double sigma_base, double like_norm) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  if (nd == 0) throw Error(POFD_E_ARG, "No pixels in data");
  if (device_ < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  HostSet& s = sets_[bs];
  Data1 d;
  if (bin_data_) {
    unsigned* bins = nullptr;
    cuda_check(cudaMalloc(&bins, nbins_ * sizeof(unsigned)), "cudaMalloc");
    double info[3];
    try {
      ingest_bin1(data_dev, nd, meansub, nbins_, bins, info, stream_);
      d.bins.resize(nbins_);
      cuda_check(cudaMemcpy(d.bins.data(), bins, nbins_ * sizeof(unsigned),
                            cudaMemcpyDeviceToHost), "D2H bins");
    } catch (...) {
      cudaFree(bins);
      throw;
    }
    cudaFree(bins);
    d.binned = true;
    d.nbins = nbins_;
    d.bincent0 = info[1];
    d.bindelta = info[2];
    d.npix = nd;
  } else {
    d.data.resize(nd);
    cuda_check(cudaMemcpy(d.data.data(), data_dev, nd * sizeof(double), cudaMemcpyDeviceToHost),
               "D2H data");
    if (meansub) d.meanSubtract();
  }
  s.data.push_back(std::move(d));
  s.sb.push_back(sigma_base);
  s.lo.push_back(0.0);
  s.ln.push_back(like_norm);
  refresh_set(s);
  static_ok_ = false;
}

// calcLikeSingle::setRRange (calcLike.cc:346-371), for every beam set.
void Engine1::set_rranges(const float* theta, unsigned npar) {
  if (npar < knots_.size()) throw Error(POFD_E_ARG, "Number of knot values different than expected");
  for (size_t k = 0; k < knots_.size(); ++k)
    if (std::isnan(static_cast<double>(theta[k])))
      throw Error(POFD_E_INVALID_MODEL, "Model is not valid");
  const double safetyfac = 1.05;
  for (auto& s : sets_) {
    if (s.data.empty()) throw Error(POFD_E_ARG, "Data not loaded");
    const auto raw = rrange_knots(knots_.back(), s.bm);
    const double sigma = std::sqrt(s.exp_conf * s.exp_conf + s.maxsb * s.maxsb);
    s.minR = safetyfac * raw.first;
    s.maxR = safetyfac * raw.second + kNZeroPad * sigma;
    if (s.minDF < s.minR && s.bm.hasneg) s.minR = s.minDF;
    if (s.maxDF > s.maxR && s.bm.haspos) s.maxR = s.maxDF;
    s.rr_set = true;
  }
  static_ok_ = false;
}

// A dataset without pixels whose noise level is set per call: the P(D)
// factory path (getPD(sigma)) runs through the same kernels with it.
void Engine1::add_virtual_dataset(int bs, double sigma_base) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  HostSet& s = sets_[bs];
  Data1 d;
  d.binned = true;
  d.nbins = 0;
  s.data.push_back(std::move(d));
  s.sb.push_back(sigma_base);
  s.lo.push_back(0.0);
  s.ln.push_back(1.0);
  s.maxsb = sigma_base;
  static_ok_ = false;
}

void Engine1::set_virtual_sigma(int bs, double sigma) {
  HostSet& s = sets_.at(bs);
  s.sb.back() = sigma;
  s.maxsb = sigma;
  if (!static_ok_) return;
  const int d = h_bsets_[bs].ds_begin + h_bsets_[bs].nds - 1;
  h_dsets_[d].sigma_base = sigma;
  h_bsets_[bs].maxsb = sigma;
  cuda_check(cudaMemcpy(d_dsets_ + d, &h_dsets_[d], sizeof(DSet1Dev), cudaMemcpyHostToDevice), "upload");
  cuda_check(cudaMemcpy(d_bsets_ + bs, &h_bsets_[bs], sizeof(BSet1Dev), cudaMemcpyHostToDevice), "upload");
}

void Engine1::set_rrange_explicit(int bs, double minR, double maxR) {
  HostSet& s = sets_.at(bs);
  s.minR = minR;
  s.maxR = maxR;
  s.rr_set = true;
  static_ok_ = false;
}

std::pair<double, double> Engine1::rrange(int bs) const {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  return {sets_[bs].minR, sets_[bs].maxR};
}

void Engine1::dataset_info(int bs, int ds, double* o, uint32_t* bins) const {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  const HostSet& s = sets_[bs];
  if (ds < 0 || ds >= static_cast<int>(s.data.size()))
    throw Error(POFD_E_ARG, "invalid dataset index");
  const Data1& d = s.data[ds];
  if (o) {
    o[0] = static_cast<double>(d.count());
    o[1] = d.nbins;
    o[2] = d.bincent0;
    o[3] = d.bindelta;
    o[4] = s.lo[ds];
    o[5] = s.sb[ds];
    o[6] = s.ln[ds];
    o[7] = s.minDF;
    o[8] = s.maxDF;
  }
  if (bins && d.binned) std::memcpy(bins, d.bins.data(), d.bins.size() * sizeof(uint32_t));
}

void Engine1::free_static() {
  for (void* p : static_allocs_) cudaFree(p);
  static_allocs_.clear();
  d_bsets_ = nullptr;
  d_dsets_ = nullptr;
  static_ok_ = false;
}

// Upload the parameter-independent data: beam terms, interpolation nodes
// and their spline factorisation, grid ranges, binned data.
unsigned Engine1::fill_tiles() const {
  const unsigned pts = NT * static_cast<unsigned>(tune_.rfill_per);
  return tune_.rfill_mode >= 2 ? runblk_ : (n_ + pts - 1) / pts;
}

void Engine1::build_static() {
  if (device_ < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  free_static();
  if (sets_.empty()) throw Error(POFD_E_ARG, "no beam sets");
  runblk_ = 0;
  auto up = [&](const std::vector<double>& v) -> const double* {
    double* p = dalloc<double>(v.size() ? v.size() : 1);
    static_allocs_.push_back(p);
    if (!v.empty())
      cuda_check(cudaMemcpy(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
    return p;
  };
  auto upi = [&](const std::vector<int>& v) -> const int* {
    int* p = dalloc<int>(v.size() ? v.size() : 1);
    static_allocs_.push_back(p);
    if (!v.empty())
      cuda_check(cudaMemcpy(p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice), "upload");
    return p;
  };
  const unsigned K = static_cast<unsigned>(knots_.size());
  std::vector<double> lk(K);
  for (unsigned i = 0; i < K; ++i) lk[i] = std::log2(knots_[i]);
  model_.K = static_cast<int>(K);
  model_.logknots = up(lk);
  model_.minknot = knots_.front();
  model_.maxknot = knots_.back();
  {
    // 64 panels of 20 points per knot interval
    KnotQuadrature kq;
    kq.build(lk.data(), static_cast<int>(K), 64, 20);
    d_qu_ = up(kq.u);
    d_qs_ = up(kq.s);
    d_qw_ = up(kq.w);
    qper_ = kq.nper;
  }

  cuda_check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device_),
             "SM count");
  B_ = static_cast<unsigned>(sets_.size());
  maxterms_ = 1;
  h_bsets_.assign(B_, BSet1Dev{});
  h_dsets_.clear();
  const unsigned NI = ninterp_;
  const double ininterpm1 = 1.0 / static_cast<double>(NI - 1);
  const double subedgemult = 1e-5;  // PDFactory.h:30
  for (unsigned b = 0; b < B_; ++b) {
    HostSet& s = sets_[b];
    if (!s.rr_set) throw Error(POFD_E_ARG, "R range not set");
    if (s.data.empty()) throw Error(POFD_E_ARG, "Data not loaded");
    const double maxflux = s.maxR, minflux = s.minR;
    if (maxflux <= 0.0) throw Error(POFD_E_ARG, "Invalid (non-positive) maxflux");
    if (minflux == maxflux) throw Error(POFD_E_ARG, "Invalid (0) range between min/max flux");
    RGrid1 g;
    g.init(n_, minflux, maxflux);
    BSet1Dev& bd = h_bsets_[b];
    double prefac = s.bm.pixsize / 3600.0;
    prefac = prefac * prefac;
    bd.prefac = prefac;
    const auto rr = rrange_knots(knots_.back(), s.bm);
    bd.rr_lo = rr.first;
    bd.rr_hi = rr.second;
    bd.haspos = s.bm.haspos;
    bd.hasneg = s.bm.hasneg;
    bd.dflux = g.dflux;
    bd.minflux_R = g.minflux_R;
    bd.wrapRidx = static_cast<int>(g.wrapRidx);
    bd.maxsb = s.maxsb;
    std::vector<int> gidx(n_, -1);
    for (int side = 0; side < 2; ++side) {
      Side1Dev& sd = bd.side[side];
      sd.nodes = 0;
      sd.grid_lo = 1;
      sd.grid_hi = 0;
      sd.grid_off = 0.0;
      const bool has = side == 0 ? s.bm.haspos : s.bm.hasneg;
      if (!has) continue;
      std::vector<double> x(NI);
      if (side == 0) {
        const double mini = knots_.front() * subedgemult;
        double maxi = knots_.back() * s.bm.maxpos();
        const double dinterp = 0.001 * (maxi - mini) * ininterpm1;
        maxi -= dinterp;
        const double dif = (std::log2(maxi / mini)) * ininterpm1;
        for (unsigned i = 0; i < NI; ++i) x[i] = mini * std::exp2(static_cast<double>(i) * dif);
      } else {
        double maxi = -knots_.front() * subedgemult;
        double mini = -knots_.back() * s.bm.maxneg();
        const double dinterp = 0.001 * (maxi - mini) * ininterpm1;
        mini += dinterp;
        maxi -= dinterp;
        const double dif = (std::log2(mini / maxi)) * ininterpm1;
        for (unsigned i = 0; i < NI; ++i)
          x[i] = maxi * std::exp2(static_cast<double>(NI - i - 1) * dif);
      }
      SplineSystem sys;
      sys.factor(x);
      std::vector<double> tw, tie;
      s.bm.terms(side == 1, tw, tie);
      if (tie.size() > static_cast<size_t>(MAXTERMS))
        throw Error(POFD_E_ARG, "beam has too many terms; histogram it");
      std::vector<double> lxa(NI), lie(tie.size());
      for (unsigned i = 0; i < NI; ++i) lxa[i] = std::log2(std::fabs(x[i]));
      for (size_t j = 0; j < tie.size(); ++j) lie[j] = std::log2(tie[j]);
      sd.lxa = up(lxa);
      sd.lie = up(lie);
      {
        // knot interval of every (term, node): parameter independent, as
        // the range test on |x| / eta and log2|x| + log2(1/eta) are
        const size_t nt = tie.size();
        std::vector<double> lk(knots_.size());
        for (size_t k = 0; k < knots_.size(); ++k) lk[k] = std::log2(knots_[k]);
        const int K = static_cast<int>(knots_.size());
        std::vector<unsigned char> kt(nt * NI, 255);
        for (size_t j = 0; j < nt; ++j)
          for (unsigned i = 0; i < NI; ++i) {
            const double currarg = std::fabs(sys.x[i]) * tie[j];
            if (currarg < knots_.front() || currarg >= knots_.back()) continue;
            const double u = lxa[i] + lie[j];
            int ilo = 0, ihi = K - 1;
            while (ihi > ilo + 1) {
              const int mid = (ihi + ilo) >> 1;
              if (lk[mid] > u) ihi = mid; else ilo = mid;
            }
            kt[j * NI + i] = static_cast<unsigned char>(ilo);
          }
        unsigned char* d = nullptr;
        cuda_check(cudaMalloc(&d, kt.size() + 16), "cudaMalloc");
        static_allocs_.push_back(d);
        cuda_check(cudaMemcpy(d, kt.data(), kt.size(), cudaMemcpyHostToDevice), "upload");
        sd.kidx = d;
        // per node, the first and one past the last term inside the knot
        // range: the only terms the node's sum visits
        std::vector<int2> jr(NI, make_int2(0, 0));
        for (unsigned i = 0; i < NI; ++i) {
          int lo = -1, hi = -1;
          for (size_t j = 0; j < nt; ++j)
            if (kt[j * NI + i] != 255) {
              if (lo < 0) lo = static_cast<int>(j);
              hi = static_cast<int>(j) + 1;
            }
          if (lo >= 0) jr[i] = make_int2(lo, hi);
        }
        int2* dj = nullptr;
        cuda_check(cudaMalloc(&dj, jr.size() * sizeof(int2) + 16), "cudaMalloc");
        static_allocs_.push_back(dj);
        cuda_check(cudaMemcpy(dj, jr.data(), jr.size() * sizeof(int2), cudaMemcpyHostToDevice),
                   "upload");
        sd.jrange = dj;
      }
      sd.nodes = 1;
      sd.nterms = static_cast<int>(tie.size());
      if (sd.nterms > maxterms_) maxterms_ = sd.nterms;
      sd.w = up(tw);
      sd.ieta = up(tie);
      sd.x = up(sys.x);
      sd.ih = up(sys.ih);
      sd.alpha = up(sys.alpha);
      sd.gamma = up(sys.gamma);
      // grid ranges (PDFactory.cc:563-606)
      if (side == 0 && maxflux > 0) {
        const double minI = x[0], maxI = x[NI - 1];
        const unsigned lo = static_cast<unsigned>(minI / g.dflux + 0.9999999999999999);
        unsigned hi = static_cast<unsigned>(maxI / g.dflux);
        if (hi > g.wrapRidx) hi = g.wrapRidx;
        sd.grid_lo = static_cast<int>(lo);
        sd.grid_hi = static_cast<int>(hi);
        sd.grid_off = 0.0;
      }
      if (side == 1 && minflux < 0 && g.wrapRidx > 0) {
        const double minI = x[0], maxI = x[NI - 1];
        unsigned lo = static_cast<unsigned>((minI - g.minflux_R) / g.dflux + g.wrapRidx + 1 + 0.9999999999999999);
        if (lo <= g.wrapRidx) lo = g.wrapRidx + 1;
        unsigned hi = static_cast<unsigned>((maxI - g.minflux_R) / g.dflux + g.wrapRidx + 1);
        if (hi > n_ - 1) hi = n_ - 1;
        sd.grid_lo = static_cast<int>(lo);
        sd.grid_hi = static_cast<int>(hi);
        sd.grid_off = g.minflux_R - static_cast<double>(g.wrapRidx + 1) * g.dflux;
      }
      // interval of every covered grid point (gsl-style bisection)
      for (int i = sd.grid_lo; i <= sd.grid_hi; ++i) {
        const double cflux = static_cast<double>(i) * g.dflux + sd.grid_off;
        size_t lo = 0, hi = NI - 1;
        while (hi > lo + 1) {
          const size_t mid = (hi + lo) / 2;
          if (x[mid] > cflux) hi = mid; else lo = mid;
        }
        gidx[i] = static_cast<int>(lo);
      }
    }
    bd.gidx = upi(gidx);
    {
      // runs for the running-product fill: cut at interval and side
      // changes and after 16 points
      std::vector<int> runs;
      const int wrap = static_cast<int>(g.wrapRidx);
      const int n = static_cast<int>(n_);
      for (int i = 0; i < n;) {
        const int q = gidx[i];
        const bool neg = i > wrap;
        int j = i + 1;
        while (j < n && j - i < 16 && gidx[j] == q && (j > wrap) == neg) ++j;
        const int len = j - i;
        const int kind = q < 0 ? 0 : (len >= 4 ? 2 : 1);
        runs.push_back(i);
        runs.push_back(((q + 1) << 8) | (len << 2) | kind);
        i = j;
      }
      bd.nruns = static_cast<int>(runs.size() / 2);
      bd.runs = reinterpret_cast<const int2*>(upi(runs));
      const unsigned nb = (static_cast<unsigned>(bd.nruns) + NT - 1) / NT;
      if (nb > runblk_) runblk_ = nb;
      // the same cut, per block of the own FFT's forward pass A (R fill
      // mode 3): block bx's inputs are its M1 row segments of 2 CB
      // consecutive grid points, [2 (256 r + bx CB), 2 (256 r + bx CB + CB))
      bd.aruns = nullptr;
      bd.arun_off = nullptr;
      if (n >= 4096 && n <= 131072 && (n & (n - 1)) == 0) {
        const int m1 = n / 512;
        const int L2 = (m1 == 8) ? 1 : m1 / 16, CB = 256 / L2;
        // each block's runs are dealt to its 256 threads longest first onto
        // the least loaded thread (estimated cost: a running-product run
        // ~100 instructions + 12 per point, a point-by-point run 60 per
        // point, a zero run 2 per point), then stored in thread order:
        // thread t of block bx takes aruns[arun_off[bx * 257 + t] ..
        // arun_off[bx * 257 + t + 1])
        std::vector<int> ar, off(static_cast<size_t>(L2) * 257);
        for (int bx = 0; bx < L2; ++bx) {
          std::vector<std::pair<int, int>> blk;  // (first index, packed)
          for (int r = 0; r < m1; ++r) {
            const int s0 = 2 * (256 * r + bx * CB), s1 = s0 + 2 * CB;
            for (int i = s0; i < s1;) {
              const int q = gidx[i];
              const bool neg = i > wrap;
              int j = i + 1;
              while (j < s1 && j - i < 16 && gidx[j] == q && (j > wrap) == neg) ++j;
              const int len = j - i;
              blk.push_back({i, ((q + 1) << 8) | (len << 2) | (q < 0 ? 0 : (len >= 4 ? 2 : 1))});
              i = j;
            }
          }
          auto cost = [](int packed) {
            const int len = (packed >> 2) & 31, kind = packed & 3;
            return kind == 2 ? 100 + 12 * len : (kind == 1 ? 60 * len : 2 * len);
          };
          std::vector<int> order(blk.size());
          for (size_t k = 0; k < order.size(); ++k) order[k] = static_cast<int>(k);
          std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return cost(blk[a].second) > cost(blk[b].second);
          });
          std::vector<std::vector<int>> per(256);
          std::vector<long> load(256, 0);
          for (int k : order) {
            int tmin = 0;
            for (int t2 = 1; t2 < 256; ++t2)
              if (load[t2] < load[tmin]) tmin = t2;
            per[tmin].push_back(k);
            load[tmin] += cost(blk[k].second);
          }
          for (int t2 = 0; t2 < 256; ++t2) {
            off[static_cast<size_t>(bx) * 257 + t2] = static_cast<int>(ar.size() / 2);
            for (int k : per[t2]) {
              ar.push_back(blk[k].first);
              ar.push_back(blk[k].second);
            }
          }
          off[static_cast<size_t>(bx) * 257 + 256] = static_cast<int>(ar.size() / 2);
        }
        bd.aruns = reinterpret_cast<const int2*>(upi(ar));
        bd.arun_off = upi(off);
      }
    }
    bd.ds_begin = static_cast<int>(h_dsets_.size());
    bd.nds = static_cast<int>(s.data.size());
    for (size_t i = 0; i < s.data.size(); ++i) {
      const Data1& d = s.data[i];
      DSet1Dev dd{};
      dd.bs = static_cast<int>(b);
      dd.sigma_base = s.sb[i];
      dd.like_offset = s.lo[i];
      dd.like_norm = s.ln[i];
      dd.binned = d.binned ? 1 : 0;
      if (d.binned) {
        std::vector<int> idx;
        std::vector<double> cnt;
        for (unsigned k = 0; k < d.nbins; ++k)
          if (d.bins[k]) { idx.push_back(static_cast<int>(k)); cnt.push_back(static_cast<double>(d.bins[k])); }
        dd.nnz = static_cast<int>(idx.size());
        dd.nzidx = upi(idx);
        dd.nzcnt = up(cnt);
        dd.flux = nullptr;
        dd.bincent0 = d.bincent0;
        dd.bindelta = d.bindelta;
      } else {
        dd.nnz = static_cast<int>(d.data.size());
        dd.flux = up(d.data);
        dd.nzidx = nullptr;
        dd.nzcnt = nullptr;
      }
      h_dsets_.push_back(dd);
    }
  }
  D_ = static_cast<unsigned>(h_dsets_.size());
  d_bsets_ = dalloc<BSet1Dev>(B_);
  static_allocs_.push_back(d_bsets_);
  cuda_check(cudaMemcpy(d_bsets_, h_bsets_.data(), B_ * sizeof(BSet1Dev), cudaMemcpyHostToDevice), "upload");
  d_dsets_ = dalloc<DSet1Dev>(D_);
  static_allocs_.push_back(d_dsets_);
  cuda_check(cudaMemcpy(d_dsets_, h_dsets_.data(), D_ * sizeof(DSet1Dev), cudaMemcpyHostToDevice), "upload");
  ntile_ = fill_tiles();
  nchunk_ = (n_ + CHUNK - 1) / CHUNK;
  // own FFT: n = 2m, m = m1 * 256 with m1 a power of two in [8, 256].  By
  // default (no FFT mode set) from n = 8192: at n = 4096 batched cuFFT is
  // ~5 % faster on the B200, above it the own FFT is faster (1.6x at
  // n = 65536 and 131072); on request (set_fft_mode(0)) from n = 4096.
  own_fft_ = (fft_mode_ == 0 || (fft_mode_ < 0 && n_ >= 8192)) && n_ >= 4096 && n_ <= 131072 &&
             (n_ & (n_ - 1)) == 0;
  tune_.own_fft = own_fft_ ? 1 : 0;
  if (own_fft_) {
    const size_t m = n_ / 2;
    std::vector<double2> wh(m / 128), wl(128), wn(m + 1);
    const long double tau = 6.283185307179586476925286766559005768L;
    for (size_t j = 0; j < m / 128; ++j) {
      const long double a = -tau * static_cast<long double>(128 * j) / static_cast<long double>(m);
      wh[j] = make_double2(static_cast<double>(cosl(a)), static_cast<double>(sinl(a)));
    }
    for (size_t i = 0; i < 128; ++i) {
      const long double a = -tau * static_cast<long double>(i) / static_cast<long double>(m);
      wl[i] = make_double2(static_cast<double>(cosl(a)), static_cast<double>(sinl(a)));
    }
    for (size_t k = 0; k <= m; ++k) {
      const long double a = -tau * static_cast<long double>(k) / static_cast<long double>(n_);
      wn[k] = make_double2(static_cast<double>(cosl(a)), static_cast<double>(sinl(a)));
    }
    d_wh_ = dalloc<double2>(m / 128);
    static_allocs_.push_back(d_wh_);
    d_wl_ = dalloc<double2>(128);
    static_allocs_.push_back(d_wl_);
    d_wn_ = dalloc<double2>(m + 1);
    static_allocs_.push_back(d_wn_);
    cuda_check(cudaMemcpy(d_wh_, wh.data(), wh.size() * sizeof(double2), cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemcpy(d_wl_, wl.data(), wl.size() * sizeof(double2), cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemcpy(d_wn_, wn.data(), (m + 1) * sizeof(double2), cudaMemcpyHostToDevice), "upload");
  }
  static_ok_ = true;
  // shapes changed: old plans/graphs/work space no longer match
  drop_graphs();
  for (auto& kv : plans_) {
    if (kv.second.fwd) { fftwork_.forget(kv.second.fwd); cufftDestroy(kv.second.fwd); }
    if (kv.second.inv) { fftwork_.forget(kv.second.inv); cufftDestroy(kv.second.inv); }
  }
  plans_.clear();
  const unsigned P = ws_.P;
  free_work();
  if (P) reserve(P);
}

void Engine1::drop_graphs() {
  for (auto& kv : plans_) {
    for (auto& g : kv.second.graphs) cudaGraphExecDestroy(g.second);
    kv.second.graphs.clear();
    if (kv.second.host_graph) cudaGraphExecDestroy(kv.second.host_graph);
    kv.second.host_graph = nullptr;
  }
}

// Times each stage of one launch sequence with CUDA events, reps times.
void Engine1::profile_stages(unsigned nprop, const float* theta, unsigned npar,
                             int reps, double* stage_ms) {
  double ll;
  std::vector<double> lls(nprop);
  std::vector<int> sts(nprop);
  eval_host(nprop, theta, npar, lls.data(), sts.data());  // staging + warm
  cudaEvent_t ev[kNumStages + 1];
  for (auto& e : ev) cuda_check(cudaEventCreate(&e), "event create");
  for (int k = 0; k < kNumStages; ++k) stage_ms[k] = 0.0;
  (void)ll;
  for (int r = 0; r < reps; ++r) {
    launch_all(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_, ev);
    cuda_check(cudaStreamSynchronize(stream_), "synchronize");
    for (int k = 0; k < kNumStages; ++k) {
      float ms = 0.f;
      cuda_check(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]), "elapsed");
      stage_ms[k] += ms / reps;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
}

// Mean time of one launch sequence for these rows, as the caller's graph
// replays it (the first evaluation stages the rows and captures the graph).
double Engine1::time_sequence(unsigned nprop, const float* theta, unsigned npar, int reps) {
  std::vector<double> ll(nprop);
  std::vector<int> st(nprop);
  eval_host(nprop, theta, npar, ll.data(), st.data());
  enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);  // warm
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event create");
  cuda_check(cudaEventCreate(&e1), "event create");
  cuda_check(cudaEventRecord(e0, stream_), "event record");
  for (int r = 0; r < reps; ++r) enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);
  cuda_check(cudaEventRecord(e1, stream_), "event record");
  cuda_check(cudaEventSynchronize(e1), "event sync");
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return static_cast<double>(ms) / reps;
}

void Engine1::set_tuning(const Tune1& t) {
  if (t.rfill_per != 4 && t.rfill_per != 8 && t.rfill_per != 16)
    throw Error(POFD_E_ARG, "rfill_per must be 4, 8 or 16");
  if (t.rnodes_threads != 64 && t.rnodes_threads != 128 && t.rnodes_threads != 256)
    throw Error(POFD_E_ARG, "rnodes_threads must be 64, 128 or 256");
  if (t.spec_blocks < 1 || t.spec_blocks > 64) throw Error(POFD_E_ARG, "spec_blocks must be in [1, 64]");
  if (t.rfill_mode < 0 || t.rfill_mode > 3) throw Error(POFD_E_ARG, "rfill_mode must be 0 ... 3");
  const bool fft_changed = (t.own_fft != 0) != (tune_.own_fft != 0);
  tune_ = t;
  tune_.own_fft = t.own_fft ? 1 : 0;
  if (fft_changed) set_fft_mode(tune_.own_fft ? 0 : 1);  // rebuilds tables, plans, work space
  if (static_ok_) ntile_ = fill_tiles();
  drop_graphs();
}

// Coordinate descent over the knobs, one pass, each candidate timed on the
// captured graph of the whole sequence.  The FFT choice is tried only where
// the own FFT supports the size.
void Engine1::autotune(unsigned nprop, const float* theta, unsigned npar, int reps, double* out7) {
  NvtxRange nvtx_range("pofd like1 autotune");
  if (nprop == 0 || reps < 1) throw Error(POFD_E_ARG, "autotune needs rows and reps >= 1");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  const double t_untuned = time_sequence(nprop, theta, npar, reps);
  Tune1 best = tune_;
  double best_ms = t_untuned;
  auto trial = [&](const Tune1& t) {
    set_tuning(t);
    const double ms = time_sequence(nprop, theta, npar, reps);
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  };
  const bool own_possible = n_ >= 4096 && n_ <= 131072 && (n_ & (n_ - 1)) == 0;
  if (own_possible) {
    Tune1 t = best;
    t.own_fft = best.own_fft ? 0 : 1;
    trial(t);
  }
  for (int per : {4, 8, 16}) {
    if (per == best.rfill_per) continue;
    Tune1 t = best;
    t.rfill_per = per;
    trial(t);
  }
  for (int th : {64, 128, 256}) {
    if (th == best.rnodes_threads) continue;
    Tune1 t = best;
    t.rnodes_threads = th;
    trial(t);
  }
  if (best.own_fft && own_possible) {
    for (int rf : {0, 1, 2, 3}) {
      if (rf == best.rfill_mode) continue;
      Tune1 t = best;
      t.rfill_mode = rf;
      trial(t);
    }
  }
  if (best.own_fft && own_possible) {
    for (int sb : {2, 4, 8, 16, 32}) {
      if (sb == best.spec_blocks) continue;
      Tune1 t = best;
      t.spec_blocks = sb;
      trial(t);
    }
  }
  set_tuning(best);
  if (out7) {
    out7[0] = best.own_fft;
    out7[1] = best.rfill_per;
    out7[2] = best.rnodes_threads;
    out7[3] = best.spec_blocks;
    out7[4] = best.rfill_mode;
    out7[5] = best_ms;
    out7[6] = t_untuned;
  }
}

const char* Engine1::stage_name(int i) const {
  static const char* lib[kNumStages] = {
      "k_model1+k_rnodes1", "k_rspline1", "k_rfill1", "k_moments1",
      "cufft_d2z", "k_spectrum1", "cufft_z2d", "k_pscan1", "k_pfinish1",
      "k_reduce1"};
  static const char* own[kNumStages] = {
      "k_model1+k_rnodes1", "k_rspline1", "k_rfill1", "k_moments1",
      "k_fftA1+k_fftB1", "k_spectrum1f", "k_fftA1+k_fftB1_inv", "k_pscan1", "k_pfinish1",
      "k_reduce1"};
  static const char* fused[kNumStages] = {
      "k_model1+k_rnodes1", "k_rspline1", "k_fftAR1", "k_moments1",
      "k_fftB1", "k_spectrum1f", "k_fftA1+k_fftB1_inv", "k_pscan1", "k_pfinish1",
      "k_reduce1"};
  if (i < 0 || i >= kNumStages) return "";
  if (!own_fft_) return lib[i];
  return fused_fill() ? fused[i] : own[i];
}

// Prior setters (calcLike.h:251-269, calcLike.cc:839-877).  The prior
// values are launch arguments of the reduction kernel, so captured graphs
// are dropped.
void Engine1::set_sigma_prior(bool on, double width) {
  if (on && !(width > 0.0)) throw Error(POFD_E_ARG, "Invalid (non-positive) sigma prior width");
  prior_.has_sigma = on ? 1 : 0;
  if (on) {
    prior_.sigma_width = width;
    prior_.log_sigma_width = std::log(width);
  }
  drop_graphs();
}

void Engine1::set_cfirb_prior(bool on, double mean, double sigma) {
  if (on) {
    if (mean < 0.0) throw Error(POFD_E_ARG, "Invalid (negative) CFIRB mean");
    if (!(sigma > 0.0)) throw Error(POFD_E_ARG, "Invalid (non-positive) CFIRB sigma");
    prior_.cfirb_mean = mean;
    prior_.cfirb_sigma = sigma;
    prior_.log_cfirb_sigma = std::log(sigma);
  }
  prior_.has_cfirb = on ? 1 : 0;
  drop_graphs();
}

void Engine1::set_poisson_prior(bool on, double mean, double sigma) {
  if (on) {
    if (mean < 0.0) throw Error(POFD_E_ARG, "Invalid (negative) Poisson prior mean");
    if (!(sigma > 0.0)) throw Error(POFD_E_ARG, "Invalid (non-positive) Poisson prior sigma");
    prior_.poisson_mean = mean;
    prior_.poisson_sigma = sigma;
    prior_.log_poisson_sigma = std::log(sigma);
  }
  prior_.has_poisson = on ? 1 : 0;
  drop_graphs();
}

void Engine1::set_regularization(double alpha) {
  if (!(alpha >= 0.0)) throw Error(POFD_E_ARG, "Invalid (negative) regularization alpha");
  prior_.alpha = alpha;
  drop_graphs();
}

void Engine1::bonus_host(unsigned nprop, const float* theta, unsigned npar, double* out) {
  if (nprop == 0) return;
  if (npar < knots_.size()) throw Error(POFD_E_ARG, "Not enough elements in paramSet");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  const size_t nb = static_cast<size_t>(nprop) * npar * sizeof(float);
  float* d = nullptr;
  cuda_check(cudaMalloc(&d, nb), "cudaMalloc");
  cudaError_t e = cudaMemcpyAsync(d, theta, nb, cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) {
    k_bonus1<<<nprop, kBonusThreads, 0, stream_>>>(model_, d, static_cast<int>(npar),
                                                   std::log2(10.0), nullptr, nullptr, d_qu_,
                                                   d_qs_, d_qw_, qper_, ws_.bonus, -1);
    e = cudaGetLastError();
  }
  std::vector<double> o(static_cast<size_t>(nprop) * 4);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(o.data(), ws_.bonus, o.size() * sizeof(double), cudaMemcpyDeviceToHost,
                        stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  cudaFree(d);
  cuda_check(e, "bonus evaluation");
  for (unsigned i = 0; i < nprop; ++i) {
    out[2 * i] = o[4 * i];
    out[2 * i + 1] = o[4 * i + 1];
  }
}

void Engine1::fill_bonus(unsigned nprop, float* theta_dev, unsigned npar, cudaStream_t st) {
  if (nprop == 0) return;
  const unsigned K = static_cast<unsigned>(knots_.size());
  if (npar < K + 3) throw Error(POFD_E_ARG, "Not enough room to fill");
  if (!static_ok_) reserve(std::max(nprop, ws_.P));
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (!st) st = stream_;
  k_bonus1<<<nprop, kBonusThreads, 0, st>>>(model_, theta_dev, static_cast<int>(npar),
                                            std::log2(10.0), nullptr, nullptr, d_qu_, d_qs_,
                                            d_qw_, qper_, nullptr, static_cast<int>(K + 1));
  cuda_check(cudaGetLastError(), "k_bonus1");
}

void Engine1::set_fft_mode(int mode) {
  if (mode != 0 && mode != 1) throw Error(POFD_E_ARG, "fft mode must be 0 (own) or 1 (cuFFT)");
  tune_.own_fft = (mode == 0) ? 1 : 0;
  if (mode == fft_mode_) return;
  fft_mode_ = mode;
  static_ok_ = false;  // rebuilds tables, plans, graphs and work space
}

void Engine1::free_work() {
  void* ptrs[] = {ws_.cnt, ws_.mstatus, ws_.sigmult, ws_.nodes, ws_.spl,
                  ws_.rbuf, ws_.rpart, ws_.mom, ws_.pbuf, ws_.ppart,
                  ws_.pmidx, ws_.pinfo, ws_.pdout, ws_.theta_in, ws_.logl,
                  ws_.tmp, ws_.bonus, ws_.kcut_set, ws_.kcut_ds};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ws_.h_theta) cudaFreeHost(ws_.h_theta);
  if (ws_.h_logl) cudaFreeHost(ws_.h_logl);  // h_status lies in the same block
  ws_ = Workspace1{};
}

void Engine1::reserve(unsigned P) {
  if (P == 0) throw Error(POFD_E_ARG, "max_batch must be > 0");
  if (!static_ok_) {
    ws_.P = std::max(ws_.P, P);
    build_static();  // calls reserve again with the stored capacity
    return;
  }
  if (ws_.P >= P && ws_.rbuf) return;
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  free_work();
  drop_graphs();
  const size_t nc2 = 2 * (static_cast<size_t>(n_) / 2 + 1);
  const size_t NI = ninterp_;
  ws_.P = P;
  ws_.cnt = dalloc<double>(static_cast<size_t>(P) * 4 * KMAX);
  ws_.mstatus = dalloc<int>(P);
  ws_.sigmult = dalloc<double>(P);
  ws_.bonus = dalloc<double>(static_cast<size_t>(P) * 4);
  ws_.nodes = dalloc<double>(static_cast<size_t>(P) * B_ * 2 * NI);
  ws_.spl = dalloc<double>(static_cast<size_t>(P) * B_ * 2 * 4 * NI);
  ws_.rbuf = dalloc<double>(static_cast<size_t>(P) * B_ * nc2);
  // room for the smallest tile the autotuner may pick, or the run blocks
  ws_.rpart = dalloc<double>(
      static_cast<size_t>(P) * B_ *
      std::max<size_t>((n_ + NT * kMaxTilesPer - 1) / (NT * kMaxTilesPer), runblk_) * 2);
  if (own_fft_) {
    ws_.tmp = dalloc<double>(static_cast<size_t>(P) * std::max(B_, D_) * nc2);
    fftA_attr<-1>();
    fftA_attr<1>();
    fftAR_attr();
    cuda_check(cudaFuncSetAttribute(k_fftB<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(kFftBSmemMax)), "attr");
    cuda_check(cudaFuncSetAttribute(k_fftB<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(kFftBSmemMax)), "attr");
  }
  ws_.mom = dalloc<double>(static_cast<size_t>(P) * B_ * 4);
  ws_.kcut_set = dalloc<int>(static_cast<size_t>(P) * B_);
  ws_.kcut_ds = dalloc<int>(static_cast<size_t>(P) * D_);
  ws_.pbuf = dalloc<double>(static_cast<size_t>(P) * D_ * nc2);
  ws_.ppart = dalloc<double>(static_cast<size_t>(P) * D_ * nchunk_ * 4);
  ws_.pmidx = dalloc<int>(static_cast<size_t>(P) * D_ * nchunk_);
  ws_.pinfo = dalloc<PDInfo1>(static_cast<size_t>(P) * D_);
  ws_.pdout = dalloc<double>(n_);
  // logL [P] then status [P] in one allocation: one download per call
  ws_.logl = dalloc<double>(P + (P + 1) / 2);
  ws_.status = reinterpret_cast<int*>(ws_.logl + P);
  cuda_check(cudaFuncSetAttribute(k_rnodes1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>((KMAX + 4 * KMAX + 3 * MAXTERMS) * sizeof(double))),
             "smem attribute");
  cuda_check(cudaFuncSetAttribute(k_rspline1<kSplineThreads>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>((2 * 8192 + 64) * sizeof(double))),
             "smem attribute");
  cuda_check(cudaMemset(ws_.nodes, 0, static_cast<size_t>(P) * B_ * 2 * NI * sizeof(double)), "memset");
}

void Engine1::ensure_plans(unsigned nprop) {
  auto it = plans_.find(nprop);
  if (it != plans_.end() && (it->second.fwd || own_fft_)) return;
  Plans pl;
  if (own_fft_) {  // the own FFT needs no cuFFT plans; the entry holds graphs
    plans_[nprop] = pl;
    return;
  }
  int n = static_cast<int>(n_);
  const int nc = n / 2 + 1;
  int inemb[1] = {2 * nc}, onemb[1] = {nc};
  bool grew = fftwork_.make(&pl.fwd, 1, &n, inemb, 2 * nc, onemb, nc, CUFFT_D2Z,
                            static_cast<int>(nprop * B_));
  int inemb2[1] = {nc}, onemb2[1] = {2 * nc};
  grew |= fftwork_.make(&pl.inv, 1, &n, inemb2, nc, onemb2, 2 * nc, CUFFT_Z2D,
                        static_cast<int>(nprop * D_));
  if (grew) drop_graphs();  // captured transforms used the old work area
  plans_[nprop] = pl;
}


void Engine1::launch_all(unsigned nprop, const float* theta, unsigned npar,
                         double* logl, int* status, cudaStream_t st,
                         cudaEvent_t* ev) {
  // ev (optional): kNumStages+1 events recorded between the stages
  auto mark = [&](int i) {
    if (ev) cuda_check(cudaEventRecord(ev[i], st), "event record");
  };
  const int NI = static_cast<int>(ninterp_);
  const int n = static_cast<int>(n_);
  const int nc = n / 2 + 1;
  const int nc2 = 2 * nc;
  const int P = static_cast<int>(nprop);
  const int B = static_cast<int>(B_), D = static_cast<int>(D_);
  Plans& pl = plans_.at(nprop);

  mark(0);
  k_model1<<<P, 32, 0, st>>>(model_, theta, static_cast<int>(npar), std::log2(10.0),
                             ws_.cnt, ws_.mstatus, ws_.sigmult);
  if (prior_.needs_bonus())
    k_bonus1<<<P, kBonusThreads, 0, st>>>(model_, const_cast<float*>(theta), static_cast<int>(npar),
                                          std::log2(10.0), ws_.cnt, ws_.mstatus, d_qu_, d_qs_,
                                          d_qw_, qper_, ws_.bonus, -1);
  {
    const size_t smem = (KMAX + 4 * KMAX + 3 * static_cast<size_t>(maxterms_)) * sizeof(double);
    const int th = tune_.rnodes_threads;
    dim3 grid((NI + th - 1) / th, P * B * 2);
    k_rnodes1<<<grid, th, smem, st>>>(d_bsets_, model_, B, NI, maxterms_,
                                      ws_.cnt, ws_.mstatus, ws_.nodes);
  }
  mark(1);
  {
    const size_t smem = (2 * static_cast<size_t>(NI) + 64) * sizeof(double);
    k_rspline1<kSplineThreads><<<P * B * 2, kSplineThreads, smem, st>>>(d_bsets_, B, NI, ws_.mstatus,
                                            ws_.nodes, ws_.spl);
  }
  mark(2);
  if (own_fft_) {
    const int m = n / 2, m1 = m / 256;
    const int rowsz = nc;  // double2 per row
    double2* tmp = reinterpret_cast<double2*>(ws_.tmp);
    double2* rb = reinterpret_cast<double2*>(ws_.rbuf);
    double2* pb = reinterpret_cast<double2*>(ws_.pbuf);
    const bool fused = fused_fill();
    int ntile = static_cast<int>(ntile_);
    if (fused) {
      // R fill inside the forward pass A: the grid goes straight into tmp
      ntile = launch_fftAR(m1, tune_.rfill_mode == 3, P * B, st, d_bsets_, B, NI, rowsz,
                           ws_.mstatus, ws_.spl, ws_.rbuf, ws_.rpart, tmp, d_wh_, d_wl_);
    } else {
      dim3 grid(ntile_, P * B);
      launch_rfill(tune_.rfill_per, tune_.rfill_mode >= 2, grid, st, d_bsets_, B, n, NI, nc2, static_cast<int>(ntile_),
                   ws_.mstatus, ws_.spl, ws_.rbuf, ws_.rpart);
    }
    mark(3);
    k_moments1<<<(P * B + 127) / 128, 128, 0, st>>>(d_bsets_, d_dsets_, B, D, n, nc2,
                                                    ntile, P * B,
                                                    ws_.mstatus, ws_.sigmult, ws_.rbuf, ws_.rpart,
                                                    ws_.mom, ws_.kcut_set, ws_.kcut_ds);
    mark(4);
    const int rb_rows = m1 < FRB ? m1 : FRB;
    if (!fused)
      launch_fftA<-1>(m1, P * B, st, rowsz, B, ws_.mstatus, rb, tmp, d_wh_, d_wl_, nullptr);
    k_fftB<-1><<<dim3(m1 / rb_rows, P * B), 256, fftB_smem(m1), st>>>(
        m1, rowsz, B, ws_.mstatus, tmp, rb, d_wh_, d_wl_, ws_.kcut_set);
    mark(5);
    {
      // a few blocks per row loop over the pairs up to the row's cut-off
      dim3 grid(std::min((m / 2 + 1 + NT - 1) / NT, tune_.spec_blocks), P * B);
      k_spectrum1f<<<grid, NT, 0, st>>>(d_bsets_, d_dsets_, B, D, n, rowsz, ws_.mstatus,
                                        ws_.sigmult, ws_.mom, rb, pb, d_wn_, ws_.kcut_set,
                                        ws_.kcut_ds);
    }
    mark(6);
    launch_fftA<1>(m1, P * D, st, rowsz, D, ws_.mstatus, pb, tmp, d_wh_, d_wl_, ws_.kcut_ds);
    k_fftB<1><<<dim3(m1 / rb_rows, P * D), 256, fftB_smem(m1), st>>>(
        m1, rowsz, D, ws_.mstatus, tmp, pb, d_wh_, d_wl_, nullptr);
  } else {
    {
      dim3 grid(ntile_, P * B);
      launch_rfill(tune_.rfill_per, tune_.rfill_mode >= 2, grid, st, d_bsets_, B, n, NI, nc2, static_cast<int>(ntile_),
                   ws_.mstatus, ws_.spl, ws_.rbuf, ws_.rpart);
    }
    mark(3);
    k_moments1<<<(P * B + 127) / 128, 128, 0, st>>>(d_bsets_, d_dsets_, B, D, n, nc2,
                                                    static_cast<int>(ntile_), P * B,
                                                    ws_.mstatus, ws_.sigmult, ws_.rbuf,
                                                    ws_.rpart, ws_.mom, nullptr, nullptr);
    mark(4);
    cufft_check(cufftSetStream(pl.fwd, st), "cufftSetStream");
    cufft_check(cufftExecD2Z(pl.fwd, ws_.rbuf, reinterpret_cast<cufftDoubleComplex*>(ws_.rbuf)),
                "cufftExecD2Z");
    mark(5);
    {
      dim3 grid((nc + NT - 1) / NT, P * B);
      k_spectrum1<<<grid, NT, 0, st>>>(d_bsets_, d_dsets_, B, D, n, nc, ws_.mstatus,
                                       ws_.sigmult, ws_.mom, ws_.rbuf, ws_.pbuf);
    }
    mark(6);
    cufft_check(cufftSetStream(pl.inv, st), "cufftSetStream");
    cufft_check(cufftExecZ2D(pl.inv, reinterpret_cast<cufftDoubleComplex*>(ws_.pbuf), ws_.pbuf),
                "cufftExecZ2D");
  }
  mark(7);
  {
    dim3 grid(nchunk_, P * D);
    k_pscan1<<<grid, NT, 0, st>>>(d_bsets_, d_dsets_, B, D, n, nc2,
                                  static_cast<int>(nchunk_), ws_.mstatus,
                                  ws_.sigmult, ws_.mom, ws_.pbuf, ws_.ppart,
                                  ws_.pmidx);
  }
  mark(8);
  k_pfinish1<<<P * D, NT, 0, st>>>(d_bsets_, d_dsets_, B, D, n, nc2,
                                   static_cast<int>(nchunk_), std::log(2.0),
                                   ws_.mstatus, ws_.sigmult, ws_.mom, ws_.pbuf,
                                   ws_.ppart, ws_.pmidx, ws_.pinfo);
  mark(9);
  k_reduce1<<<(P + 127) / 128, 128, 0, st>>>(d_bsets_, B, D, P, ws_.mstatus,
                                            ws_.sigmult, ws_.pinfo, prior_, ws_.bonus,
                                            logl, status);
  mark(10);
  cuda_check(cudaGetLastError(), "kernel launch");
}

// Replays a CUDA graph of the whole launch sequence for these pointers,
// captured on the first call that sees them.  If the caller's stream is
// itself being captured, the launches are recorded into the caller's graph.
void Engine1::enqueue(unsigned nprop, const float* theta_dev, unsigned npar,
                      double* logl_dev, int* status_dev, cudaStream_t st) {
  NvtxRange nvtx_range("pofd like1 enqueue");
  if (nprop == 0) return;
  if (npar < knots_.size() + 1) throw Error(POFD_E_ARG, "Not enough elements in paramSet");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  ensure_plans(nprop);
  if (!st) st = stream_;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cuda_check(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing");
  if (cs != cudaStreamCaptureStatusNone) {
    launch_all(nprop, theta_dev, npar, logl_dev, status_dev, st, nullptr);
    return;
  }
  cudaGraphExec_t g = graph_for(nprop, theta_dev, npar, logl_dev, status_dev);
  if (g) cuda_check(cudaGraphLaunch(g, st), "graph launch");
  else launch_all(nprop, theta_dev, npar, logl_dev, status_dev, st, nullptr);
}

cudaGraphExec_t Engine1::graph_for(unsigned nprop, const float* theta,
                                   unsigned npar, double* logl, int* status) {
  Plans& pl = plans_.at(nprop);
  if (pl.no_graph) return nullptr;
  const GraphKey key{theta, npar, logl, status};
  for (auto& kv : pl.graphs)
    if (kv.first == key) return kv.second;
  if (!pl.warmed) {  // first use of this batch size runs eagerly
    pl.warmed = true;
    return nullptr;
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    bool threw = false;
    try {
      launch_all(nprop, theta, npar, logl, status, stream_, nullptr);
    } catch (...) {
      threw = true;
    }
    const cudaError_t ec = cudaStreamEndCapture(stream_, &g);
    if (threw || ec != cudaSuccess || !g || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
      ge = nullptr;
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
  if (!ge) {
    pl.no_graph = true;  // cannot be captured: always run eagerly
    return nullptr;
  }
  if (pl.graphs.size() >= 8) {
    cudaGraphExecDestroy(pl.graphs.front().second);
    pl.graphs.erase(pl.graphs.begin());
  }
  pl.graphs.push_back({key, ge});
  return ge;
}

// The upload of theta, the launch sequence and the download of logL and
// status, captured together for each batch size after its first (eager) use.
cudaGraphExec_t Engine1::host_graph_for(unsigned nprop, unsigned npar) {
  Plans& pl = plans_.at(nprop);
  if (pl.no_graph || !pl.warmed) return nullptr;
  if (pl.host_graph && pl.host_npar == npar) return pl.host_graph;
  if (pl.host_graph) {
    cudaGraphExecDestroy(pl.host_graph);
    pl.host_graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    bool threw = false;
    try {
      cuda_check(cudaMemcpyAsync(ws_.theta_in, ws_.h_theta,
                                 static_cast<size_t>(nprop) * npar * sizeof(float),
                                 cudaMemcpyHostToDevice, stream_), "H2D theta");
      launch_all(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_, nullptr);
      cuda_check(cudaMemcpyAsync(ws_.h_logl, ws_.logl,
                                 ws_.P * sizeof(double) + nprop * sizeof(int),
                                 cudaMemcpyDeviceToHost, stream_), "D2H results");
    } catch (...) {
      threw = true;
    }
    const cudaError_t ec = cudaStreamEndCapture(stream_, &g);
    if (threw || ec != cudaSuccess || !g || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
      ge = nullptr;
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
  if (ge) {
    pl.host_graph = ge;
    pl.host_npar = npar;
  }
  return ge;
}

void Engine1::eval_host(unsigned nprop, const float* theta, unsigned npar,
                        double* logl, int* status) {
  NvtxRange nvtx_range("pofd like1 eval_batch");
  if (nprop == 0) return;
  if (npar < knots_.size() + 1) throw Error(POFD_E_ARG, "Not enough elements in paramSet");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (!ws_.theta_in || ws_.h_npar < npar) {
    if (ws_.theta_in) cudaFree(ws_.theta_in);
    if (ws_.h_theta) cudaFreeHost(ws_.h_theta);
    ws_.theta_in = dalloc<float>(static_cast<size_t>(ws_.P) * npar);
    cuda_check(cudaMallocHost(&ws_.h_theta, static_cast<size_t>(ws_.P) * npar * sizeof(float)), "cudaMallocHost");
    ws_.h_npar = npar;
    drop_graphs();
  }
  if (!ws_.h_logl) {
    // logL [P] then status [P], as on the device
    cuda_check(cudaMallocHost(&ws_.h_logl, ws_.P * (sizeof(double) + sizeof(int))),
               "cudaMallocHost");
    ws_.h_status = reinterpret_cast<int*>(ws_.h_logl + ws_.P);
  }
  std::memcpy(ws_.h_theta, theta, static_cast<size_t>(nprop) * npar * sizeof(float));
  ensure_plans(nprop);
  cudaGraphExec_t g = host_graph_for(nprop, npar);
  if (g) {
    cuda_check(cudaGraphLaunch(g, stream_), "graph launch");
  } else {
    cuda_check(cudaMemcpyAsync(ws_.theta_in, ws_.h_theta,
                               static_cast<size_t>(nprop) * npar * sizeof(float),
                               cudaMemcpyHostToDevice, stream_), "H2D theta");
    enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);
    cuda_check(cudaMemcpyAsync(ws_.h_logl, ws_.logl, ws_.P * sizeof(double) + nprop * sizeof(int),
                               cudaMemcpyDeviceToHost, stream_), "D2H results");
  }
  cuda_check(cudaStreamSynchronize(stream_), "synchronize");
  std::memcpy(logl, ws_.h_logl, nprop * sizeof(double));
  std::memcpy(status, ws_.h_status, nprop * sizeof(int));
}

int Engine1::pd_host(int bs, int ds, const float* theta, unsigned npar,
                     bool setlog, double* pd_out, double* info12) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  if (ds < 0 || ds >= static_cast<int>(sets_[bs].data.size())) throw Error(POFD_E_ARG, "invalid dataset index");
  double ll;
  int st;
  eval_host(1, theta, npar, &ll, &st);
  const int d = h_bsets_[bs].ds_begin + ds;
  PDInfo1 info;
  cuda_check(cudaMemcpy(&info, ws_.pinfo + d, sizeof(PDInfo1), cudaMemcpyDeviceToHost), "D2H info");
  double mom[4] = {0, 0, 0, 0};
  cuda_check(cudaMemcpy(mom, ws_.mom + static_cast<size_t>(bs) * 4, sizeof(mom), cudaMemcpyDeviceToHost), "D2H mom");
  if (info12) {
    const BSet1Dev& b = h_bsets_[bs];
    info12[0] = b.dflux; info12[1] = b.minflux_R; info12[2] = b.wrapRidx;
    info12[3] = mom[0]; info12[4] = mom[1]; info12[5] = mom[3]; info12[6] = mom[2];
    info12[7] = info.split; info12[8] = info.sgpos; info12[9] = info.sgneg;
    info12[10] = info.minflux; info12[11] = 0.0;
  }
  const int bst = info.status;
  if (bst != 0) return bst;
  const size_t nc2 = 2 * (static_cast<size_t>(n_) / 2 + 1);
  k_pdwrite1<<<(n_ + 255) / 256, 256, 0, stream_>>>(ws_.pbuf + static_cast<size_t>(d) * nc2,
                                                    static_cast<int>(n_), info.split, info.itot,
                                                    setlog ? 1 : 0, ws_.pdout);
  cuda_check(cudaGetLastError(), "pdwrite");
  cuda_check(cudaMemcpyAsync(pd_out, ws_.pdout, n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H pd");
  cuda_check(cudaStreamSynchronize(stream_), "synchronize");
  return 0;
}

void Engine1::rnodes_host(int bs, int side, const float* theta, unsigned npar,
                          double* x_out, double* r_out) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  double ll;
  int st;
  eval_host(1, theta, npar, &ll, &st);
  const Side1Dev& sd = h_bsets_[bs].side[side & 1];
  if (!sd.nodes) throw Error(POFD_E_ARG, "beam has no such side");
  const size_t NI = ninterp_;
  cuda_check(cudaMemcpy(x_out, sd.x, NI * sizeof(double), cudaMemcpyDeviceToHost), "D2H x");
  cuda_check(cudaMemcpy(r_out, ws_.nodes + (static_cast<size_t>(bs) * 2 + (side & 1)) * NI,
                        NI * sizeof(double), cudaMemcpyDeviceToHost), "D2H R");
}

void Engine1::rgrid_host(int bs, const float* theta, unsigned npar, double* out) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  if (!static_ok_ || ws_.P < 1) reserve(std::max(1u, ws_.P));
  if (!ws_.theta_in || ws_.h_npar < npar) {
    double ll;
    int st;
    eval_host(1, theta, npar, &ll, &st);  // allocates staging
  }
  cuda_check(cudaMemcpy(ws_.theta_in, theta, npar * sizeof(float), cudaMemcpyHostToDevice), "H2D");
  const int NI = static_cast<int>(ninterp_), n = static_cast<int>(n_);
  const int nc2 = 2 * (n / 2 + 1);
  const int B = static_cast<int>(B_);
  k_model1<<<1, 32, 0, stream_>>>(model_, ws_.theta_in, static_cast<int>(npar),
                                  std::log2(10.0), ws_.cnt, ws_.mstatus, ws_.sigmult);
  k_rnodes1<<<dim3((NI + 127) / 128, B * 2), 128,
              (KMAX + 4 * KMAX + 3 * static_cast<size_t>(maxterms_)) * sizeof(double), stream_>>>(
      d_bsets_, model_, B, NI, maxterms_, ws_.cnt, ws_.mstatus, ws_.nodes);
  k_rspline1<kSplineThreads><<<B * 2, kSplineThreads, (2 * static_cast<size_t>(NI) + 64) * sizeof(double), stream_>>>(
      d_bsets_, B, NI, ws_.mstatus, ws_.nodes, ws_.spl);
  launch_rfill(tune_.rfill_per, tune_.rfill_mode >= 2, dim3(ntile_, B), stream_, d_bsets_, B, n,
               NI, nc2, static_cast<int>(ntile_), ws_.mstatus, ws_.spl, ws_.rbuf, ws_.rpart);
  cuda_check(cudaGetLastError(), "rgrid kernels");
  cuda_check(cudaMemcpyAsync(out, ws_.rbuf + static_cast<size_t>(bs) * nc2, n_ * sizeof(double),
                             cudaMemcpyDeviceToHost, stream_), "D2H R grid");
  cuda_check(cudaStreamSynchronize(stream_), "synchronize");
}

}  // namespace pofd
