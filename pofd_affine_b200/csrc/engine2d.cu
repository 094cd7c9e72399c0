// engine2d.cu -- 2D (two-band) P(D) likelihood: sm_100a kernels + engine.
//
// Reference path restated (aconley/pofd_affine 0.5.1):
//   numberCountsDoubleLogNormal::setParams / sigma / offset
//                          numberCountsDoubleLogNormal.cc:1010-1052, 1172-1193
//   numberCountsDoubleLogNormal::getR (row precompute + column loop)
//                          numberCountsDoubleLogNormal.cc:1788-2007
//   PDFactoryDouble::initRFlux / initR (edge integrals) / getRStats
//                          PDFactoryDouble.cc:18-49, 313-722
//   PDFactoryDouble::initPD / getPD                PDFactoryDouble.cc:1145-1499
//   PDFactoryDouble::findSplitPoint / unwrap       PDFactoryDouble.cc:784-1118
//   PDDouble::normalize / getMeans / applyLog / getLogLikeBinned
//                          PDDouble.cc:142-447, 1103-1222
//   calcLikeDoubleSingle::getLogLike / calcLikeDouble::getLogLike
//                          calcLikeDouble.cc:553-616, 1195-1277
//
// HBM layout (P proposals, B beam sets, D datasets, n grid, nc = n/2+1,
// T terms per row slot):
//   rw    [P][B][n + nedge][T][3]  per-row colour terms (c0, c1, c2)
//   rbuf  [P][B][n][2nc]           R grid (x dflux1 dflux2), then its 2D
//                                  spectrum in place
//   pbuf  [P][D][n][2nc]           per-dataset spectrum, then the P(D)
//   rowpart/colpart                marginal partial sums of the P(D)
#include "engine2d.cuh"

#include <cstring>
#include <sstream>

#include "common.cuh"
#include "fft1d.cuh"

namespace pofd {

namespace {

constexpr int NT = 256;
constexpr int RB_MIN = 2;    // fewest R-grid rows per block (sizes the partials)
constexpr int RTILE = 32;    // P(D) rows per scan block
constexpr int GCH = 1024;    // data bins per gather block
constexpr int KMAX = Engine2::KMAX;
constexpr int MAXT = 2048;   // colour terms per row slot (a sanity limit on raw beams)
constexpr int SNT = 1024;    // threads of the split kernel

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << what << ": " << cudaGetErrorString(e);
    throw Error(e == cudaErrorMemoryAllocation ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}
void fk(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) {
    std::ostringstream s;
    s << what << ": cuFFT error " << static_cast<int>(r);
    throw Error(r == CUFFT_ALLOC_FAILED ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}
template <class T>
T* dal(size_t n) {
  void* p = nullptr;
  ck(cudaMalloc(&p, n * sizeof(T) + 16), "cudaMalloc");
  return static_cast<T*>(p);
}

__device__ __forceinline__ long long sat_index(double v) {
  if (!(v < 9.0e15)) return 0x7fffffffffffLL;
  if (!(v > -9.0e15)) return -0x7fffffffffffLL;
  return static_cast<long long>(v);
}
__device__ __forceinline__ double clip0(double v) { return (v < 0) ? 0.0 : v; }

// ------------------------------------------------------------- model
// Natural cubic spline through (x, y), written per interval as (y,b,c,d);
// out[4*(n-1)] holds y[n-1].
__device__ void nat_spline(const double* x, const double* y, int n,
                           double* out, double* wk) {
  double* c = wk;
  double* g = c + KMAX;
  double* diag = g + KMAX;
  double* off = diag + KMAX;
  double* alp = off + KMAX;
  double* gam = alp + KMAX;
  for (int k = 0; k < n; ++k) c[k] = 0.0;
  const int N = n - 2;
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
    alp[0] = diag[0];
    gam[0] = off[0] / alp[0];
    for (int i = 1; i < N - 1; ++i) {
      alp[i] = diag[i] - off[i - 1] * gam[i - 1];
      gam[i] = off[i] / alp[i];
    }
    alp[N - 1] = diag[N - 1] - off[N - 2] * gam[N - 2];
    for (int i = 1; i < N; ++i) g[i] = g[i] - gam[i - 1] * g[i - 1];
    for (int i = 0; i < N; ++i) g[i] = g[i] / alp[i];
    c[N] = g[N - 1];
    for (int i = N - 2; i >= 0; --i) c[1 + i] = g[i] - gam[i] * c[2 + i];
  }
  for (int i = 0; i < n - 1; ++i) {
    const double dx = x[i + 1] - x[i];
    const double dy = y[i + 1] - y[i];
    out[4 * i + 0] = y[i];
    out[4 * i + 1] = (dy / dx) - dx * (c[i + 1] + 2.0 * c[i]) / 3.0;
    out[4 * i + 2] = c[i];
    out[4 * i + 3] = (c[i + 1] - c[i]) / (3.0 * dx);
  }
  out[4 * (n - 1)] = y[n - 1];
}

// Knot counts (log2-log2 natural spline), sigma and offset curves of one
// proposal (numberCountsDoubleLogNormal.cc:1010-1052): cnt layout
// [0,4K) counts, [4K,8K) sigma, [8K,12K) offset; values of 1- or 2-knot
// curves sit at stride 4.
__global__ void k_model2(Model2Dev m, const float* __restrict__ theta,
                         int npar, double logfac, double* __restrict__ cnt,
                         int* __restrict__ mstatus,
                         double* __restrict__ sigmult) {
  __shared__ double wk[6 * KMAX];
  __shared__ double y[KMAX];
  __shared__ double o[12 * KMAX];
  const int w = blockIdx.x;
  const float* th = theta + static_cast<size_t>(w) * npar;
  if (threadIdx.x == 0) {
    int st = 0;
    const int K = m.K, ns = m.ns, no = m.no;
    for (int k = 0; k < K; ++k) {
      y[k] = logfac * static_cast<double>(th[k]);
      if (isnan(y[k])) st = POFD_E_INVALID_MODEL;
    }
    if (st == 0) nat_spline(m.logknots, y, K, o, wk);
    for (int k = 0; k < ns; ++k) {
      const double v = static_cast<double>(th[K + k]);
      if (isnan(v) || isinf(v)) st = POFD_E_INVALID_MODEL;
      y[k] = v;
    }
    if (st == 0) {
      if (ns > 2) nat_spline(m.sk, y, ns, o + 4 * KMAX, wk);
      else for (int k = 0; k < ns; ++k) o[4 * KMAX + 4 * k] = y[k];
    }
    for (int k = 0; k < no; ++k) {
      const double v = static_cast<double>(th[K + ns + k]);
      if (isnan(v)) st = POFD_E_INVALID_MODEL;
      y[k] = v;
    }
    if (st == 0) {
      if (no > 2) nat_spline(m.ok, y, no, o + 8 * KMAX, wk);
      else for (int k = 0; k < no; ++k) o[8 * KMAX + 4 * k] = y[k];
    }
    mstatus[w] = st;
    sigmult[2 * w] = static_cast<double>(th[K + ns + no]);
    sigmult[2 * w + 1] = static_cast<double>(th[K + ns + no + 1]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 12 * KMAX; i += blockDim.x)
    cnt[static_cast<size_t>(w) * 12 * KMAX + i] = o[i];
}

__device__ __forceinline__ double spline_at(const double* x, const double* s,
                                            int n, double v) {
  const int k = dev::bsearch_lo(x, v, 0, n - 1);
  const double dl = v - x[k];
  const double* q = s + 4 * k;
  return q[0] + dl * (q[1] + dl * (q[2] + dl * q[3]));
}

// getSigmaInner / getOffsetInner: constant (1 knot), linear (2), natural
// cspline (>= 3), clamped outside the knots; sigma floored at min_sigma
// inside the knot range only.
__device__ __forceinline__ double curve_at(const double* x, const double* s,
                                           int n, double v, bool floor_sig,
                                           double min_sigma) {
  if (n == 1) return s[0];
  if (v <= x[0]) return s[0];
  if (v >= x[n - 1]) return s[4 * (n - 1)];
  double val;
  if (n == 2) val = s[0] + (v - x[0]) / (x[1] - x[0]) * (s[4] - s[0]);
  else val = spline_at(x, s, n, v);
  if (floor_sig) val = (val < min_sigma) ? min_sigma : val;
  return val;
}

// One colour term of a row (numberCountsDoubleLogNormal.cc:1883-1963):
// c0 = weight * counts / sigma * prefac (0: the term is skipped), c1 =
// log f1 + offset - log(beam1/beam2), c2 = -1/(2 ln2 sigma^2).
__device__ __forceinline__ double3 row_term(const BSet2Dev& bs, const Model2Dev& m,
                                            const double* __restrict__ cs, int r, int sgn,
                                            int j, double ilog2toe, const double* tab) {
  double c0 = 0.0, c1 = 0.0, c2 = 0.0;
  const Sign2Dev& sg = bs.sg[sgn];
  const double f1val = fabs(bs.rowflux[r]);
  if (f1val < sg.maxf1) {
    const double ieta1 = sg.ieta1[j];
    const double f1prod = f1val * ieta1;
    if (f1prod >= m.minknot && f1prod < m.maxknot) {
      const double cts = dev::exp2_tab(spline_at(m.logknots, cs, m.K, log2(f1prod)), tab);
      if (cts > 0) {
        const double isigma =
            1.0 / curve_at(m.sk, cs + 4 * KMAX, m.ns, f1prod, true, m.min_sigma);
        if (sg.ishist) c0 = sg.w[j] * ieta1 * isigma * cts * bs.prefac;
        else c0 = cts * ieta1 * isigma * bs.prefac;
        c1 = bs.rowlog[r] + curve_at(m.ok, cs + 8 * KMAX, m.no, f1prod, false, 0.0) -
             sg.logratio[j];
        c2 = -0.5 * isigma * isigma * ilog2toe;
      }
    }
  }
  return make_double3(c0, c1, c2);
}

// Per-row colour terms, one warp per row: the row's terms of the positive
// band-2 sign component, then those of the negative one, each list with
// its zero terms dropped and its order kept, written as (c0, c1, c2)
// triples at rw[row][0 .. npos + nneg); rcnt[row] = (npos, nneg).  The R
// grid kernels read these lists directly (the same values for every lane
// of a warp), with no per-block staging.
constexpr int ROWS_PER_BLOCK = NT / 32;
__global__ void __launch_bounds__(NT)
k_rows2(const BSet2Dev* __restrict__ bsets, Model2Dev m, int B,
        double ilog2toe, const int* __restrict__ mstatus,
        const double* __restrict__ cnt, double* __restrict__ rw,
        int2* __restrict__ rcnt) {
  __shared__ dev::Exp2Table e2;
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  e2.load();
  __syncthreads();
  const BSet2Dev& bs = bsets[b];
  const int r = blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= bs.nrows) return;
  double* out = rw + (static_cast<size_t>(wb) * bs.nrows + r) * bs.Ts * 3;
  const int sgn1 = bs.rowsgn[r];
  int np = 0, nn = 0;
  if (sgn1 >= 0) {
    np = bs.hassign[sgn1] ? bs.sg[sgn1].nt : 0;
    nn = bs.hassign[sgn1 + 1] ? bs.sg[sgn1 + 1].nt : 0;
  }
  const double* cs = cnt + static_cast<size_t>(w) * 12 * KMAX;
  int npos = 0, nneg = 0;
  for (int half = 0; half < 2; ++half) {
    const int k0 = half ? np : 0, k1 = half ? np + nn : np;
    const int sgn = sgn1 + half;
    int put = half ? npos : 0;
    for (int kb = k0; kb < k1; kb += 32) {
      const int k = kb + lane;
      double3 t = make_double3(0.0, 0.0, 0.0);
      if (k < k1) t = row_term(bs, m, cs, r, sgn, k - k0, ilog2toe, e2.t);
      const bool keep = (k < k1) && t.x != 0.0;
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        double* q = out + 3 * (put + __popc(bal & ((1u << lane) - 1u)));
        q[0] = t.x;
        q[1] = t.y;
        q[2] = t.z;
      }
      put += __popc(bal);
    }
    if (half) nneg = put - npos;
    else npos = put;
  }
  if (lane == 0) rcnt[static_cast<size_t>(wb) * bs.nrows + r] = make_int2(npos, nneg);
}

// Main R grid, rows 1..n-1 x columns 1..n-1 (row 0 and column 0 are the
// edge cells), times dflux1*dflux2, with block partial sums of the
// trapezoid moments of getRStats (PDFactoryDouble.cc:593-722).  A block
// covers RG_COLS = RG_CPT * NT columns and RB rows; thread t owns columns
// base + t + NT q (q < RG_CPT: each store of a warp stays coalesced) and
// reads their flux constants once.  Per row the sign, the term counts and
// the list address are read once per thread, and each colour term's
// (c0, c1, c2) once for all the thread's columns of that term's band-2 sign
// component: the terms of a cell are summed in the list's order
// (numberCountsDoubleLogNormal.cc:1972-2002), the columns giving the
// independent exp2 chains.
constexpr int RG_CPT = 4;
constexpr int RG_COLS = RG_CPT * NT;
template <int RB>
__global__ void __launch_bounds__(NT, 4)
k_rgrid2(const BSet2Dev* __restrict__ bsets, int B, int n, int nc2,
         const int* __restrict__ mstatus, const double* __restrict__ rw,
         const int2* __restrict__ rcnt, double* __restrict__ rbuf,
         double* __restrict__ rpart) {
  __shared__ double shr[32];
  const int wb = blockIdx.z;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  __shared__ dev::Exp2Table e2;
  e2.load();
  __syncthreads();
  const BSet2Dev& bs = bsets[b];
  const int nrows = bs.nrows, ts3 = 3 * bs.Ts;
  const int* __restrict__ rowsgn = bs.rowsgn;
  const double* __restrict__ rowflux = bs.rowflux;
  const int j0 = blockIdx.x * RG_COLS + threadIdx.x;
  double if2[RG_CPT], lf2[RG_CPT], cf2[RG_CPT];
  unsigned cpos = 0, cneg = 0;  // columns (bits q) in each band-2 sign component
#pragma unroll
  for (int q = 0; q < RG_CPT; ++q) {
    const int j = j0 + q * NT;
    if2[q] = 0.0;
    lf2[q] = 0.0;
    cf2[q] = 0.0;
    if (j >= 1 && j < n) {
      if2[q] = bs.colinv[j];
      lf2[q] = bs.collog[j];
      cf2[q] = bs.rflux2[j];
      if (if2[q] != 0.0) {
        if (bs.colsgn[j]) cneg |= 1u << q;
        else cpos |= 1u << q;
      }
    }
  }
  const unsigned hsm = (bs.hassign[0] ? 1u : 0u) | (bs.hassign[1] ? 2u : 0u) |
                       (bs.hassign[2] ? 4u : 0u) | (bs.hassign[3] ? 8u : 0u);
  const double fluxfac = bs.dflux1 * bs.dflux2;
  double m1 = 0.0, v1 = 0.0, m2 = 0.0, v2 = 0.0;
  for (int rr = 0; rr < RB; ++rr) {
    const int r = 1 + blockIdx.y * RB + rr;
    if (r >= n) break;
    const int sgn1 = rowsgn[r];
    const size_t ri = static_cast<size_t>(wb) * nrows + r;
    double acc[RG_CPT];
#pragma unroll
    for (int q = 0; q < RG_CPT; ++q) acc[q] = 0.0;
    if (sgn1 >= 0) {
      const int2 nt = rcnt[ri];
      const double* __restrict__ L = rw + ri * ts3;
#pragma unroll
      for (int fs = 0; fs < 2; ++fs) {
        const unsigned cols = fs ? cneg : cpos;
        if (!cols || !((hsm >> (sgn1 + fs)) & 1u)) continue;
        const double* __restrict__ T = fs ? L + 3 * nt.x : L;
        const int cnt = fs ? nt.y : nt.x;
        for (int k = 0; k < cnt; ++k) {
          const double c0 = __ldg(T + 3 * k), c1 = __ldg(T + 3 * k + 1),
                       c2 = __ldg(T + 3 * k + 2);
#pragma unroll
          for (int q = 0; q < RG_CPT; ++q) {
            if (!((cols >> q) & 1u)) continue;
            const double t = lf2[q] - c1;
            acc[q] += c0 * dev::exp2_tab(t * t * c2, e2.t);
          }
        }
      }
    }
    const double cf1 = rowflux[r];
    const double rw1 = (r == n - 1) ? 0.5 : 1.0;
    double* Rrow = rbuf + (static_cast<size_t>(wb) * n + r) * nc2;
#pragma unroll
    for (int q = 0; q < RG_CPT; ++q) {
      const int j = j0 + q * NT;
      if (j < 1 || j >= n) continue;
      const double R = acc[q] * if2[q] * fluxfac;
      Rrow[j] = R;
      const double cR = rw1 * R;
      const double wc = (j == n - 1) ? 0.5 : 1.0;
      const double p1 = wc * cf1 * cR;
      const double p2 = wc * cf2[q] * cR;
      m1 += p1;
      v1 += cf1 * p1;
      m2 += p2;
      v2 += cf2[q] * p2;
    }
  }
  m1 = dev::block_sum<NT>(m1, shr);
  v1 = dev::block_sum<NT>(v1, shr);
  m2 = dev::block_sum<NT>(m2, shr);
  v2 = dev::block_sum<NT>(v2, shr);
  if (threadIdx.x == 0) {
    double* o = rpart + ((static_cast<size_t>(wb) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * 4;
    o[0] = m1; o[1] = v1; o[2] = m2; o[3] = v2;
  }
}

// Edge rows (band-1 fluxes below the first grid step) against every main and
// edge column, weighted by the log-trapezoid factors of the band-1 edge
// integral (PDFactoryDouble.cc:426-514).  One block per (tile of RG_COLS
// columns, group of ER edge rows, proposal x beam set), the columns spread
// over the threads as in k_rgrid2 so that each row's terms are read once per
// thread for its RG_CPT columns; the group partials are summed in
// k_rfinish2 into Rx (main columns) and the double integral r[0,0] (edge
// columns).
constexpr int ER_MIN = 4;    // fewest edge rows per group (sizes the partials)
template <int ER>
__global__ void __launch_bounds__(NT, 4)
k_redge2(const BSet2Dev* __restrict__ bsets, int B, int n, int nedge,
         const int* __restrict__ mstatus, const double* __restrict__ rw,
         const int2* __restrict__ rcnt, double* __restrict__ epart) {
  const int wb = blockIdx.z;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  __shared__ dev::Exp2Table e2;
  e2.load();
  __syncthreads();
  const BSet2Dev& bs = bsets[b];
  const int ncol = n + nedge;
  const int nrows = bs.nrows, ts3 = 3 * bs.Ts;
  const int j0 = blockIdx.x * RG_COLS + threadIdx.x;
  double if2[RG_CPT], lf2[RG_CPT], acc[RG_CPT];
  unsigned cpos = 0, cneg = 0;
#pragma unroll
  for (int q = 0; q < RG_CPT; ++q) {
    const int j = j0 + q * NT;
    if2[q] = 0.0;
    lf2[q] = 0.0;
    acc[q] = 0.0;
    if (j < ncol) {
      if2[q] = bs.colinv[j];
      lf2[q] = bs.collog[j];
      if (if2[q] != 0.0) {
        if (bs.colsgn[j]) cneg |= 1u << q;
        else cpos |= 1u << q;
      }
    }
  }
  const unsigned hsm = (bs.hassign[0] ? 1u : 0u) | (bs.hassign[1] ? 2u : 0u) |
                       (bs.hassign[2] ? 4u : 0u) | (bs.hassign[3] ? 8u : 0u);
  for (int rr = 0; rr < ER; ++rr) {
    const int i = blockIdx.y * ER + rr;
    if (i >= nedge) break;
    const int r = n + i;
    const int sgn1 = bs.rowsgn[r];
    if (sgn1 < 0) continue;
    const size_t ri = static_cast<size_t>(wb) * nrows + r;
    const int2 nt = rcnt[ri];
    const double* __restrict__ L = rw + ri * ts3;
    const double wr = ((i == 0 || i == nedge - 1) ? 0.5 : 1.0) * bs.e1[i];
    double rs[RG_CPT];
#pragma unroll
    for (int q = 0; q < RG_CPT; ++q) rs[q] = 0.0;
#pragma unroll
    for (int fs = 0; fs < 2; ++fs) {
      const unsigned cols = fs ? cneg : cpos;
      if (!cols || !((hsm >> (sgn1 + fs)) & 1u)) continue;
      const double* __restrict__ T = fs ? L + 3 * nt.x : L;
      const int cnt = fs ? nt.y : nt.x;
      for (int k = 0; k < cnt; ++k) {
        const double a0 = __ldg(T + 3 * k), a1 = __ldg(T + 3 * k + 1), a2 = __ldg(T + 3 * k + 2);
#pragma unroll
        for (int q = 0; q < RG_CPT; ++q) {
          if (!((cols >> q) & 1u)) continue;
          const double t = lf2[q] - a1;
          rs[q] += a0 * dev::exp2_tab(t * t * a2, e2.t);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < RG_CPT; ++q) acc[q] += wr * (rs[q] * if2[q]);
  }
#pragma unroll
  for (int q = 0; q < RG_CPT; ++q) {
    const int j = j0 + q * NT;
    if (j < ncol) epart[(static_cast<size_t>(wb) * gridDim.y + blockIdx.y) * ncol + j] = acc[q];
  }
}

// Edge integral along band 2 for column 0 (PDFactoryDouble.cc:518-550):
// one warp per main row (NT / 32 rows per block, so that the exp2 table is
// built once for several rows), each lane taking edge columns lane, lane +
// 32, ...: the row's sign, term counts and each term's (c0, c1, c2) are read
// once per lane for all its columns of one band-2 sign component; a warp
// reduction gives the row's sum.
constexpr int RY_ROWS = NT / 32;
constexpr int RY_CPL = 8;  // edge columns per lane held at once
__global__ void __launch_bounds__(NT, 4)
k_ry2(const BSet2Dev* __restrict__ bsets, int B, int n, int nedge,
      const int* __restrict__ mstatus, const double* __restrict__ rw,
      const int2* __restrict__ rcnt, double* __restrict__ redge) {
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  __shared__ dev::Exp2Table e2;
  e2.load();
  __syncthreads();
  const BSet2Dev& bs = bsets[b];
  const int lane = threadIdx.x & 31;
  const int r = 1 + blockIdx.x * RY_ROWS + (threadIdx.x >> 5);  // main rows 1..n-1
  if (r >= n) return;
  const int sgn1 = bs.rowsgn[r];
  const size_t ri = static_cast<size_t>(wb) * bs.nrows + r;
  const double* __restrict__ row = rw + ri * bs.Ts * 3;
  const int2 nt = rcnt[ri];
  const unsigned hsm = (bs.hassign[0] ? 1u : 0u) | (bs.hassign[1] ? 2u : 0u) |
                       (bs.hassign[2] ? 4u : 0u) | (bs.hassign[3] ? 8u : 0u);
  double tot = 0.0;
  for (int c0 = 0; c0 < nedge; c0 += 32 * RY_CPL) {
    double lf2[RY_CPL], if2[RY_CPL], acc[RY_CPL];
    unsigned cpos = 0, cneg = 0;
#pragma unroll
    for (int q = 0; q < RY_CPL; ++q) {
      const int jj = c0 + lane + 32 * q;
      lf2[q] = 0.0;
      if2[q] = 0.0;
      acc[q] = 0.0;
      if (jj < nedge) {
        const int j = n + jj;
        if2[q] = bs.colinv[j];
        lf2[q] = bs.collog[j];
        if (if2[q] != 0.0) {
          if (bs.colsgn[j]) cneg |= 1u << q;
          else cpos |= 1u << q;
        }
      }
    }
    if (sgn1 >= 0) {
#pragma unroll
      for (int fs = 0; fs < 2; ++fs) {
        const unsigned cols = fs ? cneg : cpos;
        if (!cols || !((hsm >> (sgn1 + fs)) & 1u)) continue;
        const double* __restrict__ T = fs ? row + 3 * nt.x : row;
        const int cnt = fs ? nt.y : nt.x;
        for (int k = 0; k < cnt; ++k) {
          const double a0 = __ldg(T + 3 * k), a1 = __ldg(T + 3 * k + 1), a2 = __ldg(T + 3 * k + 2);
#pragma unroll
          for (int q = 0; q < RY_CPL; ++q) {
            if (!((cols >> q) & 1u)) continue;
            const double t = lf2[q] - a1;
            acc[q] += a0 * dev::exp2_tab(t * t * a2, e2.t);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < RY_CPL; ++q) {
      const int jj = c0 + lane + 32 * q;
      if (jj >= nedge) continue;
      const double R = acc[q] * if2[q];
      tot += (jj == 0 || jj == nedge - 1) ? 0.5 * R : R;
    }
  }
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if (lane == 0) redge[static_cast<size_t>(wb) * (2 * n + 1) + n + r] = tot * bs.iRynorm;
}

// Edge cells into the grid (times dflux1*dflux2), the remaining moment
// contributions and the shift decisions (PDFactoryDouble.cc:560-585,
// 1198-1213).
__global__ void __launch_bounds__(NT)
k_rfinish2(const BSet2Dev* __restrict__ bsets, int B, int n, int nc2,
           int edge, int nedge, int ngr, int nparts,
           const int* __restrict__ mstatus, const double* __restrict__ redge,
           const double* __restrict__ epart, const double* __restrict__ rpart,
           double* __restrict__ rbuf, double* __restrict__ fpart) {
  // Edge cells of row 0 and column 0 (all but r[0,0]) for NT columns/rows
  // per block, their moment contributions plus a slice of k_rgrid2's
  // partials; r[0,0] and the final sums are k_rfinal2's.
  __shared__ double shr[32];
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  const BSet2Dev& bs = bsets[b];
  const double fluxfac = bs.dflux1 * bs.dflux2;
  const double* E = redge + static_cast<size_t>(wb) * (2 * n + 1);
  double* R = rbuf + static_cast<size_t>(wb) * n * nc2;
  const int ncol = n + nedge;
  const double* ep = epart + static_cast<size_t>(wb) * ngr * ncol;
  double m1 = 0.0, v1 = 0.0, m2 = 0.0, v2 = 0.0;
  const int j = blockIdx.x * NT + threadIdx.x;  // row-0 column / column-0 row
  if (j >= 1 && j < n) {
    // row 0 (row factor 1/2)
    double val = 0.0;
    if (edge) {
      double c = 0.0;
      for (int g = 0; g < ngr; ++g) c += ep[static_cast<size_t>(g) * ncol + j];
      val = c * bs.iRxnorm * fluxfac;
    }
    R[j] = val;
    const double cf1r0 = bs.rowflux[0];
    const double cR = 0.5 * val;
    const double wc = (j == n - 1) ? 0.5 : 1.0;
    const double cf2 = bs.rflux2[j];
    const double p1 = wc * cf1r0 * cR, p2 = wc * cf2 * cR;
    m1 += p1; v1 += cf1r0 * p1; m2 += p2; v2 += cf2 * p2;
    // column 0 (column factor 1/2), row j
    const double cv = edge ? E[n + j] * fluxfac : 0.0;
    R[static_cast<size_t>(j) * nc2] = cv;
    const double cR2 = (j == n - 1) ? 0.5 * cv : cv;
    const double cf1 = bs.rowflux[j], cf20 = bs.rflux2[0];
    const double q1 = 0.5 * cf1 * cR2, q2 = 0.5 * cf20 * cR2;
    m1 += q1; v1 += cf1 * q1; m2 += q2; v2 += cf20 * q2;
  }
  const double* pp = rpart + static_cast<size_t>(wb) * nparts * 4;
  for (int k = j; k < nparts; k += gridDim.x * NT) {
    m1 += pp[4 * k]; v1 += pp[4 * k + 1]; m2 += pp[4 * k + 2]; v2 += pp[4 * k + 3];
  }
  m1 = dev::block_sum<NT>(m1, shr);
  v1 = dev::block_sum<NT>(v1, shr);
  m2 = dev::block_sum<NT>(m2, shr);
  v2 = dev::block_sum<NT>(v2, shr);
  if (threadIdx.x == 0) {
    double* o = fpart + (static_cast<size_t>(wb) * gridDim.x + blockIdx.x) * 4;
    o[0] = m1; o[1] = v1; o[2] = m2; o[3] = v2;
  }
}

// r[0,0] (the double edge integral, PDFactoryDouble.cc:426-467), its cell
// and moment term, the moment sums and the shift decisions
// (PDFactoryDouble.cc:560-585, 1198-1213); one block per proposal and beam
// set.
__global__ void __launch_bounds__(NT)
k_rfinal2(const BSet2Dev* __restrict__ bsets, int B, int n, int nc2, int edge,
          int nedge, int ngr, int nfp, const int* __restrict__ mstatus,
          const double* __restrict__ epart, const double* __restrict__ fpart,
          double* __restrict__ rbuf, double* __restrict__ mom) {
  __shared__ double shr[32];
  const int wb = blockIdx.x;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  const BSet2Dev& bs = bsets[b];
  const double fluxfac = bs.dflux1 * bs.dflux2;
  const int ncol = n + nedge;
  const double* ep = epart + static_cast<size_t>(wb) * ngr * ncol;
  double r00 = 0.0;
  if (edge) {
    for (int jj = threadIdx.x; jj < nedge; jj += NT) {
      double c = 0.0;
      for (int g = 0; g < ngr; ++g) c += ep[static_cast<size_t>(g) * ncol + n + jj];
      r00 += (jj == 0 || jj == nedge - 1) ? 0.5 * c : c;
    }
    r00 = dev::block_sum<NT>(r00, shr) * bs.iR00norm;
  }
  double m1 = 0.0, v1 = 0.0, m2 = 0.0, v2 = 0.0;
  const double* fp = fpart + static_cast<size_t>(wb) * nfp * 4;
  for (int k = threadIdx.x; k < nfp; k += NT) {
    m1 += fp[4 * k]; v1 += fp[4 * k + 1]; m2 += fp[4 * k + 2]; v2 += fp[4 * k + 3];
  }
  m1 = dev::block_sum<NT>(m1, shr);
  v1 = dev::block_sum<NT>(v1, shr);
  m2 = dev::block_sum<NT>(m2, shr);
  v2 = dev::block_sum<NT>(v2, shr);
  if (threadIdx.x == 0) {
    const double val = edge ? r00 * fluxfac : 0.0;
    rbuf[static_cast<size_t>(wb) * n * nc2] = val;
    // cell (0, 0): row factor 1/2, column weight 1/2
    const double cf1 = bs.rowflux[0], cf2 = bs.rflux2[0];
    const double p1 = 0.5 * cf1 * 0.5 * val, p2 = 0.5 * cf2 * 0.5 * val;
    m1 += p1; v1 += cf1 * p1; m2 += p2; v2 += cf2 * p2;
    const double s1 = sqrt(v1), s2 = sqrt(v2);
    const bool d1 = (s1 > bs.dflux1) && (fabs(m1) > bs.dflux1);
    const bool d2 = (s2 > bs.dflux2) && (fabs(m2) > bs.dflux2);
    double* o = mom + static_cast<size_t>(wb) * 8;
    o[0] = m1; o[1] = m2; o[2] = v1; o[3] = v2;
    o[4] = d1 ? -m1 : 0.0; o[5] = d2 ? -m2 : 0.0;
    o[6] = d1 ? 1.0 : 0.0; o[7] = d2 ? 1.0 : 0.0;
  }
}

// Exponent a = Re R~ - R~00 and phase (cos, sin) of the shifted imaginary
// part at bin (i1, i2).
struct PVal2 {
  double a, c, s;
};
__device__ __forceinline__ PVal2 pval2(const double2* Rt, int nc, int n, int i1, int i2,
                                       double r0, const double* mo, double sf1,
                                       double sf2) {
  const double2 v = Rt[static_cast<size_t>(i1) * nc + i2];
  double ival = v.y;
  if (mo[6] != 0.0) {
    const double sp1 = (i1 < nc) ? sf1 * static_cast<double>(i1)
                                 : -sf1 * static_cast<double>(n - i1);
    ival = ival - sp1;
  }
  if (mo[7] != 0.0) ival = ival - sf2 * static_cast<double>(i2);
  PVal2 r;
  r.a = v.x - r0;
  sincos(ival, &r.s, &r.c);
  return r;
}

// The self-conjugate columns (i2 = 0 and n/2, two of nc): the Hermitian
// part p = (p(i1) + conj p(n - i1)) / 2, or the real part where the row is
// its own mirror, times each dataset's noise factor.
__device__ __forceinline__ void spectrum2_selfconj(const BSet2Dev& bs, const DSet2Dev* dsets,
                                                int n, int nc, int i1, int i2,
                                                const double2* Rt, double r0, const double* mo,
                                                double sf1, double sf2, double sm1, double sm2,
                                                double iflux1, double iflux2, double didx1,
                                                double didx2, double2* out, size_t dstride) {
  const PVal2 pv = pval2(Rt, nc, n, i1, i2, r0, mo, sf1, sf2);
  // (a mirror at the origin would need i1 = 0 and i2 = 0: the origin itself)
  const int j1 = (n - i1) % n;
  const bool self = (j1 == i1);
  PVal2 qv{0.0, 1.0, 0.0};
  if (!self) qv = pval2(Rt, nc, n, j1, i2, r0, mo, sf1, sf2);
  for (int dd = 0; dd < bs.nds; ++dd) {
    const int d = bs.ds_begin + dd;
    const DSet2Dev& ds = dsets[d];
    const double s1 = sm1 * ds.sb1, s2 = sm2 * ds.sb2;
    double nz = 0.0;
    if (s1 > 0 || s2 > 0) {
      const double sf1n = -0.5 * s1 * s1 * iflux1 * iflux1;
      const double sf2n = -0.5 * s2 * s2 * iflux2 * iflux2;
      nz = sf1n * didx1 * didx1 + sf2n * didx2 * didx2;
    }
    const double ep = exp(pv.a + nz);
    double2 o;
    if (self) {
      o = make_double2(ep * pv.c, 0.0);
    } else {
      const double eq = exp(qv.a + nz);
      o = make_double2(0.5 * (ep * pv.c + eq * qv.c), 0.5 * (ep * pv.s - eq * qv.s));
    }
    out[static_cast<size_t>(d) * dstride] = o;
  }
}

// exp(R~ - R~00) with the shifts, the Hermitian part of the self-conjugate
// columns (0 and n/2), then one noise product per dataset
// (PDFactoryDouble.cc:1241-1342, 1383-1437).  The noise exponent of a
// dataset is added to the exponent of exp(R~ - R~00) -- one exp per bin and
// dataset for the reference's two, the same product rounded once.  Bins
// where every dataset's noise exponent is below -750 are exactly 0 in the
// reference and are written as 0 directly.
__global__ void __launch_bounds__(NT, 5)
k_spectrum2(const BSet2Dev* __restrict__ bsets,
            const DSet2Dev* __restrict__ dsets, int B, int D, int n, int nc,
            const int* __restrict__ mstatus, const double* __restrict__ sigmult,
            const double* __restrict__ mom, const double* __restrict__ rbuf,
            double* __restrict__ pbuf) {
  const int wb = blockIdx.y;
  const int w = wb / B, b = wb - w * B;
  if (mstatus[w] != 0) return;
  const long long e = static_cast<long long>(blockIdx.x) * NT + threadIdx.x;
  if (e >= static_cast<long long>(n) * nc) return;
  const int i1 = static_cast<int>(e / nc), i2 = static_cast<int>(e - static_cast<long long>(i1) * nc);
  const BSet2Dev& bs = bsets[b];
  const double iflux1 = dev::kTwoPi / (static_cast<double>(n) * bs.dflux1);
  const double iflux2 = dev::kTwoPi / (static_cast<double>(n) * bs.dflux2);
  const double sm1 = sigmult[2 * w], sm2 = sigmult[2 * w + 1];
  const double didx1 = (i1 < nc) ? static_cast<double>(i1) : static_cast<double>(n - i1);
  const double didx2 = static_cast<double>(i2);
  bool all_zero = (i1 != 0 || i2 != 0);
  for (int dd = 0; dd < bs.nds && all_zero; ++dd) {
    const DSet2Dev& ds = dsets[bs.ds_begin + dd];
    const double s1 = sm1 * ds.sb1, s2 = sm2 * ds.sb2;
    if (!(s1 > 0 || s2 > 0)) { all_zero = false; break; }
    const double sf1 = -0.5 * s1 * s1 * iflux1 * iflux1;
    const double sf2 = -0.5 * s2 * s2 * iflux2 * iflux2;
    if (!(sf1 * didx1 * didx1 + sf2 * didx2 * didx2 < -750.0)) all_zero = false;
  }
  double2* out0 = reinterpret_cast<double2*>(pbuf) + static_cast<size_t>(w) * D * n * nc;
  if (all_zero) {
    for (int dd = 0; dd < bs.nds; ++dd)
      out0[static_cast<size_t>(bs.ds_begin + dd) * n * nc + e] = make_double2(0.0, 0.0);
    return;
  }
  const double2* Rt = reinterpret_cast<const double2*>(rbuf + static_cast<size_t>(wb) * n * 2 * nc);
  const double* mo = mom + static_cast<size_t>(wb) * 8;
  const double r0 = Rt[0].x;
  const double sf1 = mo[4] * iflux1, sf2 = mo[5] * iflux2;
  if (i1 == 0 && i2 == 0) {
    for (int dd = 0; dd < bs.nds; ++dd)
      out0[static_cast<size_t>(bs.ds_begin + dd) * n * nc + e] = make_double2(1.0, 0.0);
    return;
  }
  if (i2 == 0 || ((n & 1) == 0 && i2 == n / 2)) {
    spectrum2_selfconj(bs, dsets, n, nc, i1, i2, Rt, r0, mo, sf1, sf2, sm1, sm2, iflux1,
                       iflux2, didx1, didx2, out0 + e, static_cast<size_t>(n) * nc);
    return;
  }
  const PVal2 pv = pval2(Rt, nc, n, i1, i2, r0, mo, sf1, sf2);
  for (int dd = 0; dd < bs.nds; ++dd) {
    const int d = bs.ds_begin + dd;
    const DSet2Dev& ds = dsets[d];
    const double s1 = sm1 * ds.sb1, s2 = sm2 * ds.sb2;
    double nz = 0.0;
    if (s1 > 0 || s2 > 0) {
      const double sf1n = -0.5 * s1 * s1 * iflux1 * iflux1;
      const double sf2n = -0.5 * s2 * s2 * iflux2 * iflux2;
      nz = sf1n * didx1 * didx1 + sf2n * didx2 * didx2;
    }
    const double ep = exp(pv.a + nz);
    out0[static_cast<size_t>(d) * n * nc + e] = make_double2(ep * pv.c, ep * pv.s);
  }
}

// Marginal partial sums of the clipped P(D): per (row tile, column) and per
// (row, column tile).
__global__ void __launch_bounds__(NT)
k_pscan2(int D, int n, int nc2, const int* __restrict__ mstatus,
         const double* __restrict__ pbuf, double* __restrict__ rowpart,
         double* __restrict__ colpart) {
  __shared__ double srow[RTILE][NT / 32];
  const int wd = blockIdx.z;
  const int w = wd / D;
  if (mstatus[w] != 0) return;
  const int c = blockIdx.x * NT + threadIdx.x;
  const int r0 = blockIdx.y * RTILE;
  const double* p = pbuf + static_cast<size_t>(wd) * n * nc2;
  double cs = 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int rr = 0; rr < RTILE; ++rr) {
    const int r = r0 + rr;
    double v = 0.0;
    if (r < n && c < n) v = clip0(p[static_cast<size_t>(r) * nc2 + c]);
    cs += v;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) srow[rr][warp] = v;
  }
  if (c < n) colpart[(static_cast<size_t>(wd) * gridDim.y + blockIdx.y) * n + c] = cs;
  __syncthreads();
  if (threadIdx.x < RTILE) {
    const int r = r0 + threadIdx.x;
    double s = 0.0;
    for (int k = 0; k < NT / 32; ++k) s += srow[threadIdx.x][k];
    if (r < n) rowpart[(static_cast<size_t>(wd) * n + r) * gridDim.x + blockIdx.x] = s;
  }
}

// PDFactoryDouble::findSplitPoint (PDFactoryDouble.cc:784-968) on a
// marginal held in shared memory, block-wide.  Returns the status; the
// split index lands in *out.
__device__ int split_marginal(const double* data, int n, double dflux,
                              double sgpos, double sgneg, double* shd,
                              int* shi, int* out, int* s_state,
                              double* s_jit) {
  const double n1 = 2.25, f1 = 5e-14, f2 = 1.5e-5, f3 = 5;
  if (sgpos <= 0 || sgneg <= 0) return POFD_E_SPLIT_RANGE;
  const double n1sigpos = n1 * sgpos, n1signeg = n1 * sgneg;
  if (n * dflux < (n1sigpos + n1signeg)) return POFD_E_SPLIT_RANGE;
  double mx = -1.0e308;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = dev::dmax(mx, data[i]);
  const double peak = dev::block_max<SNT>(mx, shd);
  if (!(peak > 0.0)) return POFD_E_SPLIT_PEAK;
  const long long top = static_cast<long long>(n) - sat_index(n1signeg / dflux) - 1;
  const long long bot = sat_index(n1sigpos / dflux);
  if (top >= n || bot < 0 || bot > top) return POFD_E_SPLIT_LOGIC;
  double mv = 1.0e308;
  int mi = 0x7fffffff;
  for (long long i = bot + threadIdx.x; i <= top; i += blockDim.x)
    dev::argmin_merge(mv, mi, data[i], static_cast<int>(i));
  dev::block_argmin<SNT>(mv, mi, shd, shi);
  if (mv > f2 * peak) return POFD_E_SPLIT_MIN;
  if (threadIdx.x == 0) {
    int st = 0;
    double minval = mv, jitter = 0.0;
    const int minidx = mi;
    bool found = false;
    const int pre = 17;
    if (minidx > pre) {
      bool mono = true;
      double prev = data[minidx - pre];
      jitter = prev;
      for (int i = minidx - pre + 1; i < minidx; ++i) {
        const double cv = data[i];
        if (cv >= prev) mono = false;
        jitter += cv;
        prev = cv;
      }
      if (mono) { *out = minidx; found = true; }
      else jitter = 1.1 * (jitter + minval) / static_cast<double>(pre + 1);
    } else {
      jitter = f1 * peak;
      if (minval > jitter) { *out = minidx; found = true; }
    }
    if (!found) {
      if (minval <= 0.0) {
        long long bi, ti;
        if (minidx < bot) bi = bot; else bi = (minidx >= 3) ? (minidx - 3) : minidx;
        if (minidx > top - 3) ti = top - 3; else ti = minidx + 3;
        ti = (ti >= n) ? (n - 1) : ti;
        for (long long i = bi; i < ti; ++i)
          if (data[i] > minval) minval = data[i];
      }
      if (minval > 0) jitter = (f3 * minval) < jitter ? (f3 * minval) : jitter;
      if (bot >= top) st = POFD_E_SPLIT_LOGIC;
      else if (data[top] < jitter) st = POFD_E_SPLIT_TOP;
    }
    *s_state = (st != 0) ? st : (found ? 1 : 0);
    *s_jit = jitter;
  }
  __syncthreads();
  const int state = *s_state;
  if (state != 0) return (state == 1) ? 0 : state;
  const double jitter = *s_jit;
  for (long long t = top - 1; t >= bot; t -= blockDim.x) {
    const long long i = t - threadIdx.x;
    int hit = -1;
    if (i >= bot && data[i] < jitter) hit = static_cast<int>(i);
    const int m = dev::block_max_int<SNT>(hit, shi);
    if (m >= 0) {
      if (threadIdx.x == 0) *out = m + 1;
      __syncthreads();
      return 0;
    }
  }
  return POFD_E_SPLIT_NONE;
}

// Marginals, split points, normalisation and means of one (proposal,
// dataset) (PDFactoryDouble.cc:978-1118, PDDouble.cc:142-208, 355-447).
__global__ void __launch_bounds__(SNT)
k_psplit2(const BSet2Dev* __restrict__ bsets,
          const DSet2Dev* __restrict__ dsets, int B, int D, int n, int nc2,
          int nct, int nrt, const int* __restrict__ mstatus,
          const double* __restrict__ sigmult, const double* __restrict__ mom,
          const double* __restrict__ pbuf, const double* __restrict__ rowpart,
          const double* __restrict__ colpart, PDInfo2* __restrict__ pinfo) {
  extern __shared__ double sm[];
  __shared__ double shd[64];
  __shared__ int shi[64];
  __shared__ int s_state, s_s1, s_s2;
  __shared__ double s_jit;
  const int wd = blockIdx.x;
  const int w = wd / D, d = wd - w * D;
  PDInfo2& info = pinfo[wd];
  if (mstatus[w] != 0) {
    if (threadIdx.x == 0) info.status = mstatus[w];
    return;
  }
  const DSet2Dev& ds = dsets[d];
  const BSet2Dev& bs = bsets[ds.bs];
  const double* mo = mom + (static_cast<size_t>(w) * B + ds.bs) * 8;
  const double sigma1 = sigmult[2 * w] * ds.sb1, sigma2 = sigmult[2 * w + 1] * ds.sb2;
  const double var1 = mo[2], var2 = mo[3];
  const double sg1pos = sqrt(var1 + sigma1 * sigma1);
  const double sg2pos = sqrt(var2 + sigma2 * sigma2);
  const double sg1neg = (9 * sigma1 * sigma1 > var1) ? sigma1 : sg1pos;
  const double sg2neg = (9 * sigma2 * sigma2 > var2) ? sigma2 : sg2pos;
  const double* p = pbuf + static_cast<size_t>(wd) * n * nc2;
  double* Srow = sm;
  double* Scol = sm + n;
  double* marg = sm + 2 * n;
  const double* rp = rowpart + static_cast<size_t>(wd) * n * nct;
  const double* cp = colpart + static_cast<size_t>(wd) * nrt * n;
  for (int i = threadIdx.x; i < n; i += SNT) {
    double s = 0.0;
    for (int k = 0; k < nct; ++k) s += rp[static_cast<size_t>(i) * nct + k];
    Srow[i] = s;
    double c = 0.0;
    for (int k = 0; k < nrt; ++k) c += cp[static_cast<size_t>(k) * n + i];
    Scol[i] = c;
  }
  __syncthreads();
  // band-1 marginal: trapezoid over columns of each row
  for (int i = threadIdx.x; i < n; i += SNT)
    marg[i] = Srow[i] - 0.5 * clip0(p[static_cast<size_t>(i) * nc2]) -
              0.5 * clip0(p[static_cast<size_t>(i) * nc2 + n - 1]);
  __syncthreads();
  int st = split_marginal(marg, n, bs.dflux1, sg1pos, sg1neg, shd, shi, &s_s1,
                          &s_state, &s_jit);
  __syncthreads();
  if (st == 0) {
    for (int j = threadIdx.x; j < n; j += SNT)
      marg[j] = Scol[j] - 0.5 * clip0(p[j]) -
                0.5 * clip0(p[static_cast<size_t>(n - 1) * nc2 + j]);
    __syncthreads();
    st = split_marginal(marg, n, bs.dflux2, sg2pos, sg2neg, shd, shi, &s_s2,
                        &s_state, &s_jit);
    __syncthreads();
  }
  if (st != 0) {
    if (threadIdx.x == 0) info.status = st;
    return;
  }
  const int s1 = s_s1, s2 = s_s2;
  const int s1m = (s1 == 0) ? n - 1 : s1 - 1;
  const int s2m = (s2 == 0) ? n - 1 : s2 - 1;
  auto P = [&](int i, int j) { return clip0(p[static_cast<size_t>(i) * nc2 + j]); };
  // total, rotated-row trapezoid (mean1) and rotated-column trapezoid (mean2)
  double tot = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = threadIdx.x; i < n; i += SNT) {
    tot += Srow[i];
    const int a = (i - s1 + n) % n;
    const double rowtrap = Srow[i] - 0.5 * (P(i, s2) + P(i, s2m));
    a1 += ((a == n - 1) ? 0.5 : 1.0) * static_cast<double>(a) * rowtrap;
    const int bb = (i - s2 + n) % n;
    const double coltrap = Scol[i] - 0.5 * (P(s1, i) + P(s1m, i));
    a2 += ((bb == n - 1) ? 0.5 : 1.0) * static_cast<double>(bb) * coltrap;
  }
  tot = dev::block_sum<SNT>(tot, shd);
  a1 = dev::block_sum<SNT>(a1, shd);
  a2 = dev::block_sum<SNT>(a2, shd);
  if (threadIdx.x == 0) {
    const double iraw = tot - 0.5 * (Srow[s1] + Srow[s1m]) - 0.5 * (Scol[s2] + Scol[s2m]) +
                        0.25 * (P(s1, s2) + P(s1, s2m) + P(s1m, s2) + P(s1m, s2m));
    const double itot = 1.0 / (iraw * bs.dflux1 * bs.dflux2);
    const double mean1 = itot * a1 * (bs.dflux1 * bs.dflux1 * bs.dflux2);
    const double mean2 = itot * a2 * (bs.dflux1 * bs.dflux2 * bs.dflux2);
    if (isinf(mean1) || isnan(mean1) || isinf(mean2) || isnan(mean2)) {
      info.status = POFD_E_UNSHIFT;
    } else {
      info.status = 0;
      info.s1 = s1;
      info.s2 = s2;
      info.itot = itot;
      info.minflux1 = -mean1;
      info.minflux2 = -mean2;
      info.sg1pos = sg1pos; info.sg1neg = sg1neg;
      info.sg2pos = sg2pos; info.sg2neg = sg2neg;
    }
  }
}

// Reference-order sums (opt-in): PDDouble::getIntegral, normalize and
// getMeans (PDDouble.cc:142-208, 355-447) as one sequential chain each over
// the rotated, clipped P(D) in row-major order, every product and sum
// rounded separately (no fused multiply-add), as the reference's host build
// evaluates them.  Overwrites itot and the two minflux values k_psplit2 left
// in pinfo; the split indices are kept.  One block per (proposal, dataset):
// the block stages one rotated row in shared memory and thread 0 walks it.
// The tree sums of k_psplit2 are exact to ~1e-16 relative; the sequential
// chain is not (its rounding grows with n^2), and at n = 2048 the
// difference moves a log-likelihood over millions of pixels by ~1e-5.  Slow
// (a 2n^2-long dependent chain per dataset): for parity checks, not for
// sampling.
__global__ void __launch_bounds__(NT)
k_pseq2(const BSet2Dev* __restrict__ bsets, const DSet2Dev* __restrict__ dsets,
        int D, int n, int nc2, const int* __restrict__ mstatus,
        const double* __restrict__ pbuf, PDInfo2* __restrict__ pinfo) {
  extern __shared__ double row[];
  __shared__ double s_itot;
  const int wd = blockIdx.x;
  const int w = wd / D, d = wd - w * D;
  if (mstatus[w] != 0) return;
  PDInfo2& info = pinfo[wd];
  if (info.status != 0) return;
  const BSet2Dev& bs = bsets[dsets[d].bs];
  const double d1 = bs.dflux1, d2 = bs.dflux2;
  const int s1 = info.s1, s2 = info.s2;
  const double* p = pbuf + static_cast<size_t>(wd) * n * nc2;
  auto stage = [&](int a) {
    int i = a + s1;
    if (i >= n) i -= n;
    const double* r = p + static_cast<size_t>(i) * nc2;
    for (int b = threadIdx.x; b < n; b += NT) {
      int j = b + s2;
      if (j >= n) j -= n;
      row[b] = clip0(r[j]);
    }
  };
  // getIntegral
  double tot = 0.0;
  for (int a = 0; a < n; ++a) {
    __syncthreads();
    stage(a);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (a == 0) {
        tot = __dmul_rn(0.5, row[0]);
        for (int j = 1; j < n - 1; ++j) tot = __dadd_rn(tot, row[j]);
        tot = __dadd_rn(tot, __dmul_rn(0.5, row[n - 1]));
        tot = __dmul_rn(tot, 0.5);
      } else if (a < n - 1) {
        tot = __dadd_rn(tot, __dmul_rn(0.5, row[0]));
        for (int j = 1; j < n - 1; ++j) tot = __dadd_rn(tot, row[j]);
        tot = __dadd_rn(tot, __dmul_rn(0.5, row[n - 1]));
      } else {
        tot = __dadd_rn(tot, __dmul_rn(0.25, row[0]));
        for (int j = 1; j < n - 1; ++j) tot = __dadd_rn(tot, __dmul_rn(0.5, row[j]));
        tot = __dadd_rn(tot, __dmul_rn(0.25, row[n - 1]));
      }
    }
  }
  if (threadIdx.x == 0) s_itot = 1.0 / __dmul_rn(__dmul_rn(tot, d1), d2);
  __syncthreads();
  const double itot = s_itot;
  // getMeans on the normalised array (each element stored as p * itot)
  double mean1 = 0.0, mean2 = 0.0;
  const double nm1 = static_cast<double>(n - 1);
  for (int a = 0; a < n; ++a) {
    __syncthreads();
    stage(a);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (a == 0) {
        for (int j = 1; j < n - 1; ++j)
          mean2 = __dadd_rn(mean2, __dmul_rn(static_cast<double>(j), __dmul_rn(row[j], itot)));
        mean2 = __dadd_rn(mean2, __dmul_rn(__dmul_rn(0.5, nm1), __dmul_rn(row[n - 1], itot)));
        mean2 = __dmul_rn(mean2, 0.5);
      } else if (a < n - 1) {
        double xsum = __dmul_rn(0.5, __dmul_rn(row[0], itot));
        for (int j = 1; j < n - 1; ++j) {
          const double pv = __dmul_rn(row[j], itot);
          xsum = __dadd_rn(xsum, pv);
          mean2 = __dadd_rn(mean2, __dmul_rn(static_cast<double>(j), pv));
        }
        const double pl = __dmul_rn(row[n - 1], itot);
        xsum = __dadd_rn(xsum, __dmul_rn(0.5, pl));
        mean1 = __dadd_rn(mean1, __dmul_rn(xsum, static_cast<double>(a)));
        mean2 = __dadd_rn(mean2, __dmul_rn(__dmul_rn(0.5, nm1), pl));
      } else {
        double xsum = __dmul_rn(0.5, __dmul_rn(row[0], itot));
        for (int j = 1; j < n - 1; ++j) {
          const double pv = __dmul_rn(row[j], itot);
          xsum = __dadd_rn(xsum, pv);
          mean2 = __dadd_rn(mean2, __dmul_rn(__dmul_rn(0.5, static_cast<double>(j)), pv));
        }
        const double pl = __dmul_rn(row[n - 1], itot);
        xsum = __dadd_rn(xsum, __dmul_rn(0.5, pl));
        mean1 = __dadd_rn(mean1, __dmul_rn(__dmul_rn(0.5, xsum), nm1));
        mean2 = __dadd_rn(mean2, __dmul_rn(__dmul_rn(0.25, nm1), pl));
      }
    }
  }
  if (threadIdx.x == 0) {
    mean1 = __dmul_rn(mean1, __dmul_rn(__dmul_rn(d1, d1), d2));
    mean2 = __dmul_rn(mean2, __dmul_rn(__dmul_rn(d1, d2), d2));
    if (isinf(mean1) || isnan(mean1) || isinf(mean2) || isnan(mean2)) {
      info.status = POFD_E_UNSHIFT;
    } else {
      info.itot = itot;
      info.minflux1 = -mean1;
      info.minflux2 = -mean2;
    }
  }
}

__device__ __forceinline__ double lq2(const double* __restrict__ p, int n,
                                      int nc2, int s1, int s2, double itot,
                                      int a, int b) {
  int i = a + s1; if (i >= n) i -= n;
  int j = b + s2; if (j >= n) j -= n;
  const double v = clip0(p[static_cast<size_t>(i) * nc2 + j]) * itot;
  return (v <= 0.0) ? dev::kSmallLogVal : log2(v);
}

// Bilinear log2 P(D) at the non-zero data bins (PDDouble.cc:1103-1172),
// block partial sums.  The reference reads one cell past the grid when a
// bin centre falls in the last row or column; here the last cell is used.
__global__ void __launch_bounds__(NT)
k_pgather2(const BSet2Dev* __restrict__ bsets,
           const DSet2Dev* __restrict__ dsets, int D, int n, int nc2,
           int gchunks, const int* __restrict__ mstatus,
           const double* __restrict__ pbuf, const PDInfo2* __restrict__ pinfo,
           double* __restrict__ gpart) {
  __shared__ double shr[32];
  const int wd = blockIdx.y;
  const int w = wd / D, d = wd - w * D;
  if (mstatus[w] != 0) return;
  const PDInfo2 in = pinfo[wd];
  double acc = 0.0;
  const DSet2Dev& ds = dsets[d];
  if (in.status == 0) {
    const BSet2Dev& bs = bsets[ds.bs];
    const double* p = pbuf + static_cast<size_t>(wd) * n * nc2;
    const double mf1 = in.minflux1, mf2 = in.minflux2;
    const double d1 = bs.dflux1, d2 = bs.dflux2;
    const double maxflux1 = mf1 + static_cast<double>(n - 1) * d1;
    const double maxflux2 = mf2 + static_cast<double>(n - 1) * d2;
    const double id1 = 1.0 / d1, id2 = 1.0 / d2;
    const int s1 = in.s1, s2 = in.s2;
    const double itot = in.itot;
    const int e1 = min(ds.nnz, (blockIdx.x + 1) * GCH);
    if (!ds.binned) {
      // PDDouble::getLogLikeUnbinned (PDDouble.cc:994-1051): per pixel,
      // inclusive edge tests
      for (int e = blockIdx.x * GCH + threadIdx.x; e < e1; e += NT) {
        const double cflux1 = ds.f1[e], cflux2 = ds.f2[e];
        const double delt1 = (cflux1 - mf1) * id1, delt2 = (cflux2 - mf2) * id2;
        const int idx1 = static_cast<int>(delt1), idx2 = static_cast<int>(delt2);
        double iv;
        if (cflux1 <= mf1) {
          if (cflux2 <= mf2) iv = lq2(p, n, nc2, s1, s2, itot, 0, 0);
          else if (cflux2 >= maxflux2) iv = lq2(p, n, nc2, s1, s2, itot, 0, n - 1);
          else iv = lq2(p, n, nc2, s1, s2, itot, 0, idx2);
        } else if (cflux1 >= maxflux1) {
          if (cflux2 <= mf2) iv = lq2(p, n, nc2, s1, s2, itot, n - 1, 0);
          else if (cflux2 >= maxflux2) iv = lq2(p, n, nc2, s1, s2, itot, n - 1, n - 1);
          else iv = lq2(p, n, nc2, s1, s2, itot, n - 1, idx2);
        } else if (cflux2 <= mf2) {
          iv = lq2(p, n, nc2, s1, s2, itot, idx1, 0);
        } else if (cflux2 >= maxflux2) {
          iv = lq2(p, n, nc2, s1, s2, itot, idx1, n - 1);
        } else {
          const double t = delt1 - static_cast<double>(idx1);
          const double u = delt2 - static_cast<double>(idx2);
          const int i1 = min(idx1, n - 2), i2 = min(idx2, n - 2);
          const double omu = 1.0 - u, omt = 1.0 - t;
          iv = omt * (omu * lq2(p, n, nc2, s1, s2, itot, i1, i2) +
                      u * lq2(p, n, nc2, s1, s2, itot, i1, i2 + 1)) +
               t * (omu * lq2(p, n, nc2, s1, s2, itot, i1 + 1, i2) +
                    u * lq2(p, n, nc2, s1, s2, itot, i1 + 1, i2 + 1));
        }
        acc += iv;
      }
    } else {
      for (int e = blockIdx.x * GCH + threadIdx.x; e < e1; e += NT) {
        const double cnt = ds.nzcnt[e];
        const double cflux1 = ds.bc1 + static_cast<double>(ds.nzi1[e]) * ds.bd1;
        const double cflux2 = ds.bc2 + static_cast<double>(ds.nzi2[e]) * ds.bd2;
        const int idx1 = static_cast<int>((cflux1 - mf1) * id1);
        const int idx2 = static_cast<int>((cflux2 - mf2) * id2);
        double iv;
        if (cflux1 < mf1) {
          if (cflux2 < mf2) iv = lq2(p, n, nc2, s1, s2, itot, 0, 0);
          else if (cflux2 > maxflux2) iv = lq2(p, n, nc2, s1, s2, itot, 0, n - 1);
          else iv = lq2(p, n, nc2, s1, s2, itot, 0, idx2);
        } else if (cflux1 > maxflux1) {
          if (cflux2 < mf2) iv = lq2(p, n, nc2, s1, s2, itot, n - 1, 0);
          else if (cflux2 > maxflux2) iv = lq2(p, n, nc2, s1, s2, itot, n - 1, n - 1);
          else iv = lq2(p, n, nc2, s1, s2, itot, n - 1, idx2);
        } else if (cflux2 < mf2) {
          iv = lq2(p, n, nc2, s1, s2, itot, idx1, 0);
        } else if (cflux2 > maxflux2) {
          iv = lq2(p, n, nc2, s1, s2, itot, idx1, n - 1);
        } else {
          double t = (cflux1 - mf1) * id1 - static_cast<double>(idx1);
          double u = (cflux2 - mf2) * id2 - static_cast<double>(idx2);
          int i1 = idx1, i2 = idx2;
          if (i1 > n - 2) { i1 = n - 2; t = 1.0; }
          if (i2 > n - 2) { i2 = n - 2; u = 1.0; }
          const double omu = 1.0 - u, omt = 1.0 - t;
          iv = omt * (omu * lq2(p, n, nc2, s1, s2, itot, i1, i2) +
                      u * lq2(p, n, nc2, s1, s2, itot, i1, i2 + 1)) +
               t * (omu * lq2(p, n, nc2, s1, s2, itot, i1 + 1, i2) +
                    u * lq2(p, n, nc2, s1, s2, itot, i1 + 1, i2 + 1));
        }
        acc += cnt * iv;
      }
    }
  }
  acc = dev::block_sum<NT>(acc, shr);
  if (threadIdx.x == 0) gpart[static_cast<size_t>(wd) * gchunks + blockIdx.x] = acc;
}

// Per-proposal sum over beam sets and datasets; a negative sigma multiplier
// gives bad_like for the beam set (calcLikeDouble.cc:571-576, 1219-1224).
__global__ void k_reduce2(const BSet2Dev* __restrict__ bsets,
                          const DSet2Dev* __restrict__ dsets, int B, int D,
                          int nprop, int gchunks, double log2toe,
                          const int* __restrict__ mstatus,
                          const double* __restrict__ sigmult,
                          const PDInfo2* __restrict__ pinfo,
                          const double* __restrict__ gpart, Prior2 pr,
                          const double* __restrict__ bonus,
                          double* __restrict__ logl, int* __restrict__ status) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nprop) return;
  const double qnan = __longlong_as_double(0x7ff8000000000000LL);
  if (mstatus[w] != 0) {
    logl[w] = qnan;
    status[w] = mstatus[w];
    return;
  }
  const double sm1 = sigmult[2 * w], sm2 = sigmult[2 * w + 1];
  double LogLike = 0.0;
  int st = 0;
  for (int b = 0; b < B; ++b) {
    const BSet2Dev& bs = bsets[b];
    if (bs.maxsb1 * sm1 < 0.0 || bs.maxsb2 * sm2 < 0.0) { LogLike += 1e25; continue; }
    double s = 0.0;
    for (int dd = 0; dd < bs.nds; ++dd) {
      const int d = bs.ds_begin + dd;
      const PDInfo2& in = pinfo[static_cast<size_t>(w) * D + d];
      if (in.status != 0) {
        if (st == 0) st = in.status;
        continue;
      }
      double ll = 0.0;
      const double* g = gpart + (static_cast<size_t>(w) * D + d) * gchunks;
      for (int c = 0; c < gchunks; ++c) ll += g[c];
      s += (log2toe * ll - dsets[d].like_offset) / dsets[d].like_norm;
    }
    LogLike += s;
  }
  // priors, once for all data sets (calcLikeDouble.cc:1236-1276)
  constexpr double half_log_2pi = 0.918938517570495605469;
  const double sm[2] = {sm1, sm2};
  const double* bn = bonus + 8 * static_cast<size_t>(w);
  for (int b = 0; b < 2; ++b)
    if (pr.has_sigma[b]) {
      const double val = (sm[b] - 1.0) / pr.sigma_width[b];
      LogLike -= half_log_2pi + pr.log_sigma_width[b] + 0.5 * val * val;
    }
  for (int b = 0; b < 2; ++b)
    if (pr.has_cfirb[b]) {
      const double val = (pr.cfirb_mean[b] - bn[b]) / pr.cfirb_sigma[b];
      LogLike -= half_log_2pi + pr.log_cfirb_sigma[b] + 0.5 * val * val;
    }
  for (int b = 0; b < 2; ++b)
    if (pr.has_poisson[b]) {
      const double val = (pr.poisson_mean[b] - bn[2 + b]) / pr.poisson_sigma[b];
      LogLike -= half_log_2pi + pr.log_poisson_sigma[b] + 0.5 * val * val;
    }
  if (pr.alpha > 0.0) LogLike += pr.alpha * bn[4];
  status[w] = st;
  logl[w] = (st == 0) ? LogLike : qnan;
}

// Bonus integrals and the band-1 slope penalty of each proposal's model,
// one block per proposal.  numberCountsDoubleLogNormal::splineInt(a, b)
// (numberCountsDoubleLogNormal.cc:1549-1631) integrates
// S1^(a+b) n1(S1) exp(b mu(S1) + b^2/2 sigma^2(S1)) over [S_0, S_{K-1})
// (the integrand of numberCountsDoubleLogNormal.cc:2424-2512, sigma floored
// at min_sigma in every branch there); here by Gauss-Legendre quadrature in
// u = log2 S1 on host-built nodes that also break at the colour-curve
// knots.  out[w][8] = {<S1>, <S2>, <S1^2>, <S2^2>, penalty, 0, 0, 0}, NaN for
// an invalid model; the penalty is differenceRegularize of the band-1 knots
// (numberCountsDoubleLogNormal.cc:2154-2173) before the factor alpha.
// fill_at >= 0 stores the four integrals as floats at theta[w][fill_at..].
// ------------------------------------------------------------------
// Column transforms fused with the spectrum (FFT mode 1).  After batched 1D
// row transforms of the R grid (cuFFT D2Z on its n rows), the row-
// transformed grid Y[i1][i2] (n x nc, row stride nc) goes down its columns
// here: each block takes C = 256 / M adjacent columns (M = n / 16 threads
// per column) into shared memory, runs the forward n-point DFT of every
// column, forms per bin exp(R~ - R~00) with the shifts and one dataset's
// noise (the work of k_spectrum2, same formulas), runs the inverse column
// DFT and writes the columns of that dataset's half spectrum, which batched
// 1D Z2D row transforms then take to the P(D).  So the spectrum costs no
// HBM round trip of its own and the column passes of both 2D transforms
// read and write the grid once.
//
// Column DFT, n = 16 M, M = 16 M3 (n in [512, 4096]): with n = n1 M + u,
// u = m M3 + s and k = k1 + 16 (k2 + 16 k3),
//   stage 1: 16-point register DFTs over n1, times W_n^{u k1};
//   stage 2: 16-point register DFTs over m, times W_M^{s k2};
//   stage 3: M3-point register DFTs over s.
// The forward output stays in the stage-3 slots, position
// (16 k1 + k2)(M3 + 1) + k3 (a padded stride, free of bank conflicts); the
// spectrum works slot by slot, and the inverse runs the transposed stages
// in reverse order (M3-point DFTs over k3, twiddle W_M^{-s k2}, 16-point
// DFTs over k2, twiddle W_n^{-u k1}, 16-point DFTs over k1), which read
// those slots and end in natural order.  Twiddles W_n^j, j < n, come from
// two shared tables H[j >> 5] L[j & 31] built on the host in long double.
constexpr int CS_THREADS = 256;

__host__ __device__ constexpr int cs_slots(int n) { return 256 * (n / 256 + 1); }
inline size_t colspec_smem(int n) {
  const int C = CS_THREADS / (n / 16);
  return (static_cast<size_t>(C) * cs_slots(n) + n / 32 + 32) * sizeof(double2);
}

template <int S>
__device__ __forceinline__ double2 cs_tw(const double2* H, const double2* L, int j) {
  const double2 h = H[j >> 5];
  const int lo = j & 31;
  const double2 w = lo ? fft::cmul(h, L[lo]) : h;
  return (S < 0) ? w : make_double2(w.x, -w.y);
}

// forward column DFT of the C columns in buf (natural order in, stage-3
// slots out)
template <int N>
__device__ __forceinline__ void cs_forward(double2* buf, const double2* H, const double2* L,
                                           int c, int u) {
  constexpr int M = N / 16, M3 = N / 256, SL = cs_slots(N), PP = 16 / M3;
  double2* b = buf + c * SL;
  double2 v[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = b[n1 * M + u];
  fft::dft<16, -1>(v);
#pragma unroll
  for (int k1 = 1; k1 < 16; ++k1)
    if (u) v[k1] = fft::cmul(v[k1], cs_tw<-1>(H, L, u * k1));
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) b[k1 * M + u] = v[k1];
  __syncthreads();
  {
    const int k1 = u / M3, s = u % M3;
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = b[k1 * M + m * M3 + s];
    fft::dft<16, -1>(v);
#pragma unroll
    for (int k2 = 1; k2 < 16; ++k2)
      if (s) v[k2] = fft::cmul(v[k2], cs_tw<-1>(H, L, 16 * s * k2));
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) b[(k1 * 16 + k2) * (M3 + 1) + s] = v[k2];
    __syncthreads();
  }
#pragma unroll
  for (int pp = 0; pp < PP; ++pp) {
    const int pr = pp * M + u;
    double2 z[M3];
#pragma unroll
    for (int s2 = 0; s2 < M3; ++s2) z[s2] = b[pr * (M3 + 1) + s2];
    fft::dft<M3, -1>(z);
#pragma unroll
    for (int k3 = 0; k3 < M3; ++k3) b[pr * (M3 + 1) + k3] = z[k3];
  }
  __syncthreads();
}

// inverse column DFT: stage-3 slots in, natural order out (into b[i1])
template <int N>
__device__ __forceinline__ void cs_inverse(double2* buf, const double2* H, const double2* L,
                                           int c, int u) {
  constexpr int M = N / 16, M3 = N / 256, SL = cs_slots(N), PP = 16 / M3;
  double2* b = buf + c * SL;
#pragma unroll
  for (int pp = 0; pp < PP; ++pp) {
    const int pr = pp * M + u;
    const int k2 = pr & 15;
    double2 z[M3];
#pragma unroll
    for (int k3 = 0; k3 < M3; ++k3) z[k3] = b[pr * (M3 + 1) + k3];
    fft::dft<M3, 1>(z);
#pragma unroll
    for (int s2 = 0; s2 < M3; ++s2)
      b[pr * (M3 + 1) + s2] = (s2 * k2) ? fft::cmul(z[s2], cs_tw<1>(H, L, 16 * s2 * k2)) : z[s2];
  }
  __syncthreads();
  double2 v[16];
  {
    const int k1 = u / M3, s = u % M3;
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) v[k2] = b[(k1 * 16 + k2) * (M3 + 1) + s];
    fft::dft<16, 1>(v);
    __syncthreads();
    // Z_{k1}[m M3 + s], times W_n^{-u' k1} for u' = m M3 + s
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int up = m * M3 + s;
      b[k1 * M + up] = (up * k1) ? fft::cmul(v[m], cs_tw<1>(H, L, up * k1)) : v[m];
    }
    __syncthreads();
  }
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) v[k1] = b[k1 * M + u];
  fft::dft<16, 1>(v);
  __syncthreads();
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) b[n1 * M + u] = v[n1];
  __syncthreads();
}

// Sum of the row-transformed grid's column 0 over the rows: R~00 (the DC
// bin of the 2D transform), one block per (proposal, beam set).
__global__ void __launch_bounds__(NT)
k_r0sum2(int n, int nc, const int* __restrict__ mstatus, int B,
         const double* __restrict__ rbuf, double* __restrict__ r0) {
  __shared__ double shr[32];
  const int wb = blockIdx.x;
  if (mstatus[wb / B] != 0) return;
  const double2* Y = reinterpret_cast<const double2*>(rbuf) + static_cast<size_t>(wb) * n * nc;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) acc += Y[static_cast<size_t>(i) * nc].x;
  acc = dev::block_sum<NT>(acc, shr);
  if (threadIdx.x == 0) r0[wb] = acc;
}

template <int N>
__global__ void __launch_bounds__(CS_THREADS, 2)
k_colspec2(const BSet2Dev* __restrict__ bsets, const DSet2Dev* __restrict__ dsets, int B,
           int D, const int* __restrict__ mstatus, const double* __restrict__ sigmult,
           const double* __restrict__ mom, const double* __restrict__ r0buf,
           const double* __restrict__ rbuf, double* __restrict__ pbuf,
           const double2* __restrict__ WH, const double2* __restrict__ WL) {
  constexpr int M = N / 16, M3 = N / 256, SL = cs_slots(N);
  constexpr int C = CS_THREADS / M;
  constexpr int nc = N / 2 + 1;
  extern __shared__ double2 csm[];
  double2* buf = csm;                 // [C][SL]
  double2* Hs = csm + C * SL;         // N / 32
  double2* Ls = Hs + N / 32;          // 32
  const int wb = blockIdx.y;
  const int w = wb / B, bsi = wb - w * B;
  if (mstatus[w] != 0) return;
  const int t = threadIdx.x;
  for (int i = t; i < N / 32 + 32; i += CS_THREADS)
    Hs[i] = (i < N / 32) ? WH[i] : WL[i - N / 32];
  const int c0 = blockIdx.x * C;      // first column of the block
  const int c = t / M, u = t % M;
  const BSet2Dev& bs = bsets[bsi];
  const double2* Y = reinterpret_cast<const double2*>(rbuf) + static_cast<size_t>(wb) * N * nc;
  const double iflux1 = dev::kTwoPi / (static_cast<double>(N) * bs.dflux1);
  const double iflux2 = dev::kTwoPi / (static_cast<double>(N) * bs.dflux2);
  const double sm1 = sigmult[2 * w], sm2 = sigmult[2 * w + 1];
  const double* mo = mom + static_cast<size_t>(wb) * 8;
  const double r0 = r0buf[wb];
  const double sf1 = mo[4] * iflux1, sf2 = mo[5] * iflux2;
  const bool sh1 = mo[6] != 0.0, sh2 = mo[7] != 0.0;
  for (int dd = 0; dd < bs.nds; ++dd) {
    const int d = bs.ds_begin + dd;
    const DSet2Dev& ds = dsets[d];
    // load the C columns (a warp covers 32 / C rows of C adjacent columns)
    for (int e = t; e < C * N; e += CS_THREADS) {
      const int i1 = e / C, cc = e % C;
      const int i2 = c0 + cc;
      buf[cc * SL + i1] = (i2 < nc) ? Y[static_cast<size_t>(i1) * nc + i2] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    cs_forward<N>(buf, Hs, Ls, c, u);
    // spectrum, slot by slot and in place; the self-conjugate columns
    // (i2 = 0 and n/2) go by mirror pairs (i1, n - i1), each pair owned by
    // one thread: their Hermitian parts are conjugates of each other
    const double s1 = sm1 * ds.sb1, s2 = sm2 * ds.sb2;
    const bool noisy = (s1 > 0 || s2 > 0);
    const double sf1n = -0.5 * s1 * s1 * iflux1 * iflux1;
    const double sf2n = -0.5 * s2 * s2 * iflux2 * iflux2;
#pragma unroll 4
    for (int q = t; q < C * SL; q += CS_THREADS) {
      const int cc = q / SL, pos = q % SL;
      const int pr = pos / (M3 + 1), k3 = pos % (M3 + 1);
      const int i2 = c0 + cc;
      if (k3 == M3 || i2 >= nc || i2 == 0 || i2 == N / 2) continue;
      const int i1 = (pr >> 4) + 16 * ((pr & 15) + 16 * k3);
      const double didx1 = (i1 < nc) ? static_cast<double>(i1) : static_cast<double>(N - i1);
      const double didx2 = static_cast<double>(i2);
      const double nz = noisy ? sf1n * didx1 * didx1 + sf2n * didx2 * didx2 : 0.0;
      if (noisy && nz < -750.0) {  // exactly 0 in the reference
        buf[q] = make_double2(0.0, 0.0);
        continue;
      }
      const double2 X = buf[q];
      double ival = X.y;
      if (sh1) ival -= (i1 < nc) ? sf1 * static_cast<double>(i1) : -sf1 * static_cast<double>(N - i1);
      if (sh2) ival -= sf2 * static_cast<double>(i2);
      double sn, cs;
      sincos(ival, &sn, &cs);
      const double ep = exp((X.x - r0) + nz);
      buf[q] = make_double2(ep * cs, ep * sn);
    }
    for (int cc = 0; cc < C; ++cc) {
      const int i2 = c0 + cc;
      if (i2 != 0 && i2 != N / 2) continue;
      double2* b = buf + cc * SL;
      const double didx2 = static_cast<double>(i2);
#pragma unroll 1
      for (int i1 = t; i1 <= N / 2; i1 += CS_THREADS) {
        const int j1 = (N - i1) % N;
        const int si = ((i1 & 15) * 16 + ((i1 >> 4) & 15)) * (M3 + 1) + (i1 >> 8);
        const int sj = ((j1 & 15) * 16 + ((j1 >> 4) & 15)) * (M3 + 1) + (j1 >> 8);
        if (i1 == 0 && i2 == 0) {
          b[si] = make_double2(1.0, 0.0);
          continue;
        }
        const double didx1 = static_cast<double>(i1);
        const double nz = noisy ? sf1n * didx1 * didx1 + sf2n * didx2 * didx2 : 0.0;
        if (noisy && nz < -750.0) {
          b[si] = make_double2(0.0, 0.0);
          if (j1 != i1) b[sj] = make_double2(0.0, 0.0);
          continue;
        }
        const double2 X = b[si];
        double ival = X.y;
        if (sh1) ival -= sf1 * static_cast<double>(i1);
        if (sh2) ival -= sf2 * didx2;
        double sn, cs;
        sincos(ival, &sn, &cs);
        const double ep = exp((X.x - r0) + nz);
        if (j1 == i1) {
          b[si] = make_double2(ep * cs, 0.0);
        } else {
          const double2 Xq = b[sj];
          double iq = Xq.y;
          if (sh1) iq -= -sf1 * static_cast<double>(N - j1);
          if (sh2) iq -= sf2 * didx2;
          double sq, cq;
          sincos(iq, &sq, &cq);
          const double eq = exp((Xq.x - r0) + nz);
          const double2 o = make_double2(0.5 * (ep * cs + eq * cq), 0.5 * (ep * sn - eq * sq));
          b[si] = o;
          b[sj] = make_double2(o.x, -o.y);
        }
      }
    }
    __syncthreads();
    cs_inverse<N>(buf, Hs, Ls, c, u);
    double2* Pd = reinterpret_cast<double2*>(pbuf) + (static_cast<size_t>(w) * D + d) * N * nc;
    for (int e = t; e < C * N; e += CS_THREADS) {
      const int i1 = e / C, cc = e % C;
      const int i2 = c0 + cc;
      if (i2 < nc) Pd[static_cast<size_t>(i1) * nc + i2] = buf[cc * SL + i1];
    }
    __syncthreads();
  }
}

constexpr int kBonus2Threads = 256;
__global__ void __launch_bounds__(kBonus2Threads)
k_bonus2(Model2Dev m, float* theta, int npar, double logfac,
         const double* __restrict__ cnt, const int* __restrict__ mstatus,
         const double* __restrict__ qu, const double* __restrict__ qs,
         const double* __restrict__ qw, const int* __restrict__ qk, int nq,
         double* __restrict__ out, int fill_at) {
  __shared__ double cs[12 * KMAX];
  __shared__ double lk[KMAX], sk[KMAX], okn[KMAX];
  __shared__ double red[4][kBonus2Threads / 32];
  const int w = blockIdx.x;
  const int K = m.K;
  const int st = mstatus[w];
  for (int i = threadIdx.x; i < K; i += blockDim.x) lk[i] = m.logknots[i];
  for (int i = threadIdx.x; i < m.ns; i += blockDim.x) sk[i] = m.sk[i];
  for (int i = threadIdx.x; i < m.no; i += blockDim.x) okn[i] = m.ok[i];
  for (int i = threadIdx.x; i < 12 * KMAX; i += blockDim.x)
    cs[i] = cnt[static_cast<size_t>(w) * 12 * KMAX + i];
  __syncthreads();
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  if (st == 0) {
    for (int j = threadIdx.x; j < nq; j += blockDim.x) {
      const int k = qk[j];
      const double d = qu[j] - lk[k];
      const double* q = cs + 4 * k;
      const double S = qs[j];
      const double base = qw[j] * S * S * exp2(q[0] + d * (q[1] + d * (q[2] + d * q[3])));
      const double mu = curve_at(okn, cs + 8 * KMAX, m.no, S, false, 0.0);
      double sg = curve_at(sk, cs + 4 * KMAX, m.ns, S, false, 0.0);
      if (sg < m.min_sigma) sg = m.min_sigma;
      a[0] += base;
      a[1] += base * exp(mu + 0.5 * sg * sg);
      a[2] += base * S;
      a[3] += base * S * exp(2.0 * mu + 2.0 * sg * sg);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[c] += __shfl_down_sync(0xffffffffu, a[c], o);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 4; ++c) red[c][threadIdx.x >> 5] = a[c];
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double qnan = __longlong_as_double(0x7ff8000000000000LL);
  double t[4] = {0.0, 0.0, 0.0, 0.0}, pen = 0.0;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i)
    for (int c = 0; c < 4; ++c) t[c] += red[c][i];
  const float* th = theta + static_cast<size_t>(w) * npar;
  if (st != 0) {
    for (int c = 0; c < 4; ++c) t[c] = qnan;
    pen = qnan;
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
    double* o = out + 8 * static_cast<size_t>(w);
    o[0] = t[0];
    o[1] = t[1];
    o[2] = t[2];
    o[3] = t[3];
    o[4] = pen;
    o[5] = o[6] = o[7] = 0.0;
  }
  if (fill_at >= 0) {
    float* tw = theta + static_cast<size_t>(w) * npar;
    for (int c = 0; c < 4; ++c) tw[fill_at + c] = static_cast<float>(t[c]);
  }
}

// The unwrapped, normalised (optionally log2) 2D P(D) of one row.
__global__ void k_pdwrite2(const double* __restrict__ p, int n, int nc2,
                           int s1, int s2, double itot, int setlog,
                           double* __restrict__ out) {
  const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<long long>(n) * n) return;
  const int a = static_cast<int>(e / n), b = static_cast<int>(e - static_cast<long long>(a) * n);
  int i = a + s1; if (i >= n) i -= n;
  int j = b + s2; if (j >= n) j -= n;
  const double v = clip0(p[static_cast<size_t>(i) * nc2 + j]) * itot;
  out[e] = setlog ? ((v <= 0.0) ? dev::kSmallLogVal : log2(v)) : v;
}

}  // namespace

// ===================================================================== host

Engine2::Engine2(int device, cudaStream_t stream)
    : device_(device), stream_(stream) {}

Engine2::~Engine2() {
  if (device_ < 0) return;
  cudaSetDevice(device_);
  drop_graphs();
  for (auto& kv : plans_) {
    if (kv.second.fwd) { fftwork_.forget(kv.second.fwd); cufftDestroy(kv.second.fwd); }
    if (kv.second.inv) { fftwork_.forget(kv.second.inv); cufftDestroy(kv.second.inv); }
  }
  free_work();
  free_static();
}

void Engine2::configure(unsigned nknots, const double* knotpos,
                        unsigned nsigma, const double* sigmapos,
                        unsigned noffset, const double* offsetpos,
                        unsigned fftsize, unsigned nedge, bool edge_integ,
                        bool bin_data, unsigned nbins) {
  auto incr = [](unsigned n, const double* v, const char* what) {
    for (unsigned i = 0; i < n; ++i)
      if (!(v[i] > 0) || (i > 0 && !(v[i] > v[i - 1])))
        throw Error(POFD_E_ARG, std::string(what) + " positions must be positive and increasing");
  };
  if (nknots < 3 || nknots > static_cast<unsigned>(KMAX))
    throw Error(POFD_E_ARG, "nknots must be in [3, 64]");
  if (nsigma < 1 || nsigma > static_cast<unsigned>(KMAX) || noffset < 1 ||
      noffset > static_cast<unsigned>(KMAX))
    throw Error(POFD_E_ARG, "sigma and offset knots must number 1..64");
  incr(nknots, knotpos, "knot");
  incr(nsigma, sigmapos, "sigma knot");
  incr(noffset, offsetpos, "offset knot");
  if (fftsize < 16 || fftsize > 8192) throw Error(POFD_E_ARG, "fftsize must be in [16, 8192]");
  if (edge_integ && (nedge < 2 || nedge > fftsize))
    throw Error(POFD_E_ARG, "Nedge is less than R fill size");
  if (nbins == 0) throw Error(POFD_E_ARG, "Trying to bin with no bins");
  knots_.assign(knotpos, knotpos + nknots);
  sigk_.assign(sigmapos, sigmapos + nsigma);
  offk_.assign(offsetpos, offsetpos + noffset);
  n_ = fftsize;
  nedge_ = nedge;
  edge_ = edge_integ;
  bin_data_ = bin_data;
  nbins_ = nbins;
  static_ok_ = false;
}

int Engine2::add_beamset(const Beam2& bm, double ec1, double ec2) {
  HostSet s;
  s.bm = bm;
  s.ec1 = ec1;
  s.ec2 = ec2;
  sets_.push_back(std::move(s));
  static_ok_ = false;
  return static_cast<int>(sets_.size()) - 1;
}

// calcLikeDoubleSingle::setSigmaBase1/2 (calcLikeDouble.cc:377-487) and the
// data flux range of the beam set.
void Engine2::refresh_set(HostSet& s) {
  s.maxsb1 = s.sb1[0];
  s.maxsb2 = s.sb2[0];
  for (size_t i = 1; i < s.sb1.size(); ++i) {
    if (s.sb1[i] > s.maxsb1) s.maxsb1 = s.sb1[i];
    if (s.sb2[i] > s.maxsb2) s.maxsb2 = s.sb2[i];
  }
  for (size_t i = 0; i < s.data.size(); ++i) {
    const double v1 = s.sb1[i] * s.sb1[i] + s.ec1 * s.ec1;
    const double v2 = s.sb2[i] * s.sb2[i] + s.ec2 * s.ec2;
    const double sp = std::sqrt(v1 * v2);
    if (sp > 0) {
      const double ndd = static_cast<double>(s.data[i].count());
      s.lo[i] = -ndd * (std::log(kTwoPi * sp) + 1.0);
    }
  }
  double mm[4];
  s.data[0].minmax(mm);
  for (int k = 0; k < 4; ++k) s.mdf[k] = mm[k];
  for (size_t i = 1; i < s.data.size(); ++i) {
    s.data[i].minmax(mm);
    if (mm[0] < s.mdf[0]) s.mdf[0] = mm[0];
    if (mm[1] > s.mdf[1]) s.mdf[1] = mm[1];
    if (mm[2] < s.mdf[2]) s.mdf[2] = mm[2];
    if (mm[3] > s.mdf[3]) s.mdf[3] = mm[3];
  }
  s.rr_set = false;
}

void Engine2::add_dataset(int bs, const double* d1, const double* d2,
                          size_t nd, bool meansub, double sigma1,
                          double sigma2, double like_norm) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  if (nd == 0) throw Error(POFD_E_ARG, "No pixels in data");
  HostSet& s = sets_[bs];
  Data2 d;
  d.d1.assign(d1, d1 + nd);
  d.d2.assign(d2, d2 + nd);
  if (meansub) d.meanSubtract();
  if (bin_data_) d.applyBinning(nbins_, nbins_);
  s.data.push_back(std::move(d));
  s.sb1.push_back(sigma1);
  s.sb2.push_back(sigma2);
  s.lo.push_back(0.0);
  s.ln.push_back(like_norm);
  refresh_set(s);
  static_ok_ = false;
}

// A two-band dataset whose pixels are in device memory: mean subtraction
// and binning on the GPU (ingest_bin2, bit-identical to the host path).
void Engine2::add_dataset_device(int bs, double* d1_dev, double* d2_dev, size_t nd, bool meansub,
                                 double sigma1, double sigma2, double like_norm) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size()))
    throw Error(POFD_E_ARG, "invalid beam set index");
  if (nd == 0) throw Error(POFD_E_ARG, "No pixels in data");
  if (device_ < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  HostSet& s = sets_[bs];
  Data2 d;
  if (bin_data_) {
    const size_t nb = static_cast<size_t>(nbins_) * nbins_;
    unsigned* bins = nullptr;
    ck(cudaMalloc(&bins, nb * sizeof(unsigned)), "cudaMalloc");
    double info[6];
    try {
      ingest_bin2(d1_dev, d2_dev, nd, meansub, nbins_, nbins_, bins, info, stream_);
      d.bins.resize(nb);
      ck(cudaMemcpy(d.bins.data(), bins, nb * sizeof(unsigned), cudaMemcpyDeviceToHost),
         "D2H bins");
    } catch (...) {
      cudaFree(bins);
      throw;
    }
    cudaFree(bins);
    d.binned = true;
    d.nbins1 = d.nbins2 = nbins_;
    d.bc1 = info[2];
    d.bd1 = info[3];
    d.bc2 = info[4];
    d.bd2 = info[5];
    d.npix = nd;
  } else {
    d.d1.resize(nd);
    d.d2.resize(nd);
    ck(cudaMemcpy(d.d1.data(), d1_dev, nd * sizeof(double), cudaMemcpyDeviceToHost), "D2H data");
    ck(cudaMemcpy(d.d2.data(), d2_dev, nd * sizeof(double), cudaMemcpyDeviceToHost), "D2H data");
    if (meansub) d.meanSubtract();
  }
  s.data.push_back(std::move(d));
  s.sb1.push_back(sigma1);
  s.sb2.push_back(sigma2);
  s.lo.push_back(0.0);
  s.ln.push_back(like_norm);
  refresh_set(s);
  static_ok_ = false;
}

// calcLikeDoubleSingle::setRRange (calcLikeDouble.cc:496-534).
void Engine2::set_rranges(const float* theta, unsigned npar) {
  if (npar < nparams()) throw Error(POFD_E_ARG, "Not enough parameters present to set");
  Model2Host m;
  m.set(knots_, sigk_, offk_, theta);
  const double safetyfac = 1.1;
  for (auto& s : sets_) {
    if (s.data.empty()) throw Error(POFD_E_ARG, "Data not loaded");
    double raw[4];
    m.rrange(s.bm, raw);
    const double sg1 = std::sqrt(s.ec1 * s.ec1 + s.maxsb1 * s.maxsb1);
    const double sg2 = std::sqrt(s.ec2 * s.ec2 + s.maxsb2 * s.maxsb2);
    s.rr[0] = safetyfac * raw[0];
    s.rr[1] = safetyfac * raw[1] + kNZeroPad * sg1;
    s.rr[2] = safetyfac * raw[2];
    s.rr[3] = safetyfac * raw[3] + kNZeroPad * sg2;
    const bool* hs = s.bm.hassign;
    if (s.mdf[0] < s.rr[0] && (hs[2] || hs[3])) s.rr[0] = s.mdf[0];
    if (s.mdf[1] > s.rr[1] && (hs[0] || hs[1])) s.rr[1] = s.mdf[1];
    if (s.mdf[2] < s.rr[2] && (hs[1] || hs[3])) s.rr[2] = s.mdf[2];
    if (s.mdf[3] > s.rr[3] && (hs[0] || hs[2])) s.rr[3] = s.mdf[3];
    s.rr_set = true;
  }
  static_ok_ = false;
}

void Engine2::add_virtual_dataset(int bs, double sigma1, double sigma2) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  HostSet& s = sets_[bs];
  Data2 d;
  d.binned = true;
  s.data.push_back(std::move(d));
  s.sb1.push_back(sigma1);
  s.sb2.push_back(sigma2);
  s.lo.push_back(0.0);
  s.ln.push_back(1.0);
  s.maxsb1 = sigma1;
  s.maxsb2 = sigma2;
  static_ok_ = false;
}

void Engine2::set_virtual_sigma(int bs, double sigma1, double sigma2) {
  HostSet& s = sets_.at(bs);
  s.sb1.back() = sigma1;
  s.sb2.back() = sigma2;
  s.maxsb1 = sigma1;
  s.maxsb2 = sigma2;
  if (!static_ok_) return;
  const int d = h_bsets_[bs].ds_begin + h_bsets_[bs].nds - 1;
  h_dsets_[d].sb1 = sigma1;
  h_dsets_[d].sb2 = sigma2;
  h_bsets_[bs].maxsb1 = sigma1;
  h_bsets_[bs].maxsb2 = sigma2;
  ck(cudaMemcpy(d_dsets_ + d, &h_dsets_[d], sizeof(DSet2Dev), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(d_bsets_ + bs, &h_bsets_[bs], sizeof(BSet2Dev), cudaMemcpyHostToDevice), "upload");
}

void Engine2::set_rrange_explicit(int bs, double min1, double max1, double min2, double max2) {
  HostSet& s = sets_.at(bs);
  s.rr[0] = min1;
  s.rr[1] = max1;
  s.rr[2] = min2;
  s.rr[3] = max2;
  s.rr_set = true;
  static_ok_ = false;
}

void Engine2::rrange(int bs, double* r4) const {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  for (int k = 0; k < 4; ++k) r4[k] = sets_[bs].rr[k];
}

void Engine2::dataset_info(int bs, int ds, double* o, uint32_t* bins) const {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  const HostSet& s = sets_[bs];
  if (ds < 0 || ds >= static_cast<int>(s.data.size())) throw Error(POFD_E_ARG, "invalid dataset index");
  const Data2& d = s.data[ds];
  if (o) {
    o[0] = static_cast<double>(d.count()); o[1] = d.nbins1;
    o[2] = d.bc1; o[3] = d.bc2; o[4] = d.bd1; o[5] = d.bd2;
    o[6] = s.lo[ds]; o[7] = s.sb1[ds]; o[8] = s.sb2[ds]; o[9] = s.ln[ds];
  }
  if (bins) std::memcpy(bins, d.bins.data(), d.bins.size() * sizeof(uint32_t));
}

void Engine2::free_static() {
  for (void* q : static_allocs_) cudaFree(q);
  static_allocs_.clear();
  d_bsets_ = nullptr;
  d_dsets_ = nullptr;
  d_cwh_ = nullptr;
  d_cwl_ = nullptr;
  colspec_ = false;
  static_ok_ = false;
}

void Engine2::drop_graphs() {
  for (auto& kv : plans_) {
    for (auto& g : kv.second.graphs) cudaGraphExecDestroy(g.second);
    kv.second.graphs.clear();
  }
}

void Engine2::build_static() {
  if (device_ < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  free_static();
  if (sets_.empty()) throw Error(POFD_E_ARG, "no beam sets");
  auto up = [&](const std::vector<double>& v) -> const double* {
    double* q = dal<double>(v.size() ? v.size() : 1);
    static_allocs_.push_back(q);
    if (!v.empty()) ck(cudaMemcpy(q, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
    return q;
  };
  auto upi = [&](const std::vector<int>& v) -> const int* {
    int* q = dal<int>(v.size() ? v.size() : 1);
    static_allocs_.push_back(q);
    if (!v.empty()) ck(cudaMemcpy(q, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice), "upload");
    return q;
  };
  std::vector<double> lk(knots_.size());
  for (size_t i = 0; i < knots_.size(); ++i) lk[i] = std::log2(knots_[i]);
  model_.K = static_cast<int>(knots_.size());
  model_.ns = static_cast<int>(sigk_.size());
  model_.no = static_cast<int>(offk_.size());
  model_.logknots = up(lk);
  model_.sk = up(sigk_);
  model_.ok = up(offk_);
  model_.minknot = knots_.front();
  model_.maxknot = knots_.back();
  model_.min_sigma = 0.0;
  {
    // bonus integrals: 32 panels of 20 points per interval between the
    // knots and the colour-curve knots inside the knot range
    std::vector<double> extra;
    for (double v : sigk_) extra.push_back(std::log2(v));
    for (double v : offk_) extra.push_back(std::log2(v));
    KnotQuadrature kq;
    kq.build_breaks(lk.data(), static_cast<int>(knots_.size()), extra, 32, 20);
    d_qu_ = up(kq.u);
    d_qs_ = up(kq.s);
    d_qw_ = up(kq.w);
    int* qk = nullptr;
    ck(cudaMalloc(&qk, (kq.kidx.size() + 1) * sizeof(int)), "cudaMalloc");
    static_allocs_.push_back(qk);
    if (!kq.kidx.empty())
      ck(cudaMemcpy(qk, kq.kidx.data(), kq.kidx.size() * sizeof(int), cudaMemcpyHostToDevice),
         "upload");
    d_qk_ = qk;
    nq_ = static_cast<int>(kq.u.size());
  }

  const unsigned n = n_;
  B_ = static_cast<unsigned>(sets_.size());
  h_bsets_.assign(B_, BSet2Dev{});
  h_dsets_.clear();
  Tmax_ = 1;
  unsigned maxnnz = 1;
  const double normfac = 1.0 / std::sqrt(2 * kPi);
  for (unsigned b = 0; b < B_; ++b) {
    HostSet& s = sets_[b];
    if (!s.rr_set) throw Error(POFD_E_ARG, "R range not set");
    double mn1 = s.rr[0], mx1 = s.rr[1], mn2 = s.rr[2], mx2 = s.rr[3];
    if (mx1 <= 0.0) throw Error(POFD_E_ARG, "Invalid (non-positive) maxflux1");
    if (mx2 <= 0.0) throw Error(POFD_E_ARG, "Invalid (non-positive) maxflux2");
    if (mx1 == mn1) throw Error(POFD_E_ARG, "Invalid range (0) between min/max flux in band 1");
    if (mx2 == mn2) throw Error(POFD_E_ARG, "Invalid range (0) between min/max flux in band 2");
    if (mx1 < mn1) std::swap(mn1, mx1);
    if (mx2 < mn2) std::swap(mn2, mx2);
    RGrid2Axis a1, a2;
    a1.init(n, mn1, mx1);
    a2.init(n, mn2, mx2);
    BSet2Dev& bd = h_bsets_[b];
    bd.dflux1 = a1.dflux;
    bd.dflux2 = a2.dflux;
    bd.wrap1 = static_cast<int>(a1.wrapidx);
    bd.wrap2 = static_cast<int>(a2.wrapidx);
    const double pixdeg = s.bm.pixsize / 3600.0;
    bd.prefac = pixdeg * pixdeg * normfac;
    std::vector<double> E1, E2;
    if (edge_) {
      const double lowm = 1e-9;  // PDFactoryDouble.h:33
      const double me1 = a1.dflux * lowm, me2 = a2.dflux * lowm;
      const double ine = 1.0 / static_cast<double>(nedge_ - 1);
      const double di1 = -std::log(lowm) * ine;
      E1.resize(nedge_);
      for (unsigned i = 0; i < nedge_; ++i) E1[i] = me1 * std::exp(static_cast<double>(i) * di1);
      const double di2 = (a2.dflux - me2) * ine;
      E2.resize(nedge_);
      for (unsigned i = 0; i < nedge_; ++i) E2[i] = me2 + static_cast<double>(i) * di2;
      bd.iRxnorm = di1 / (a1.dflux - me1);
      bd.iRynorm = di2 / (a2.dflux - me2);
      bd.iR00norm = di1 * di2 / ((a1.dflux - me1) * (a2.dflux - me2));
    }
    const bool hasNegX1 = s.bm.hassign[2] || s.bm.hassign[3];
    std::vector<double> rowf(a1.flux), rowl, colinv, coll;
    rowf.insert(rowf.end(), E1.begin(), E1.end());
    std::vector<int> rows, cols;
    for (double f : rowf) {
      if (f == 0 || (f < 0 && !hasNegX1)) { rows.push_back(-1); rowl.push_back(0.0); }
      else { rows.push_back(f > 0 ? 0 : 2); rowl.push_back(std::log(std::fabs(f))); }
    }
    std::vector<double> colf(a2.flux);
    colf.insert(colf.end(), E2.begin(), E2.end());
    for (double f : colf) {
      if (f == 0) { colinv.push_back(0.0); coll.push_back(0.0); cols.push_back(0); continue; }
      cols.push_back(f > 0 ? 0 : 1);
      colinv.push_back(1.0 / std::fabs(f));
      coll.push_back(std::log(std::fabs(f)));
    }
    bd.nrows = static_cast<int>(rowf.size());
    bd.rowflux = up(rowf);
    bd.rowlog = up(rowl);
    bd.rowsgn = upi(rows);
    bd.colinv = up(colinv);
    bd.collog = up(coll);
    bd.colsgn = upi(cols);
    bd.rflux2 = up(a2.flux);
    bd.e1 = up(E1);
    int nt[4];
    for (int g = 0; g < 4; ++g) {
      Sign2Dev& sg = bd.sg[g];
      bd.hassign[g] = s.bm.hassign[g] ? 1 : 0;
      nt[g] = static_cast<int>(s.bm.nterms(g));
      sg.nt = nt[g];
      sg.ishist = s.bm.ishist[g] ? 1 : 0;
      if (s.bm.ishist[g]) {
        sg.w = up(s.bm.binwt[g]);
        sg.ieta1 = up(s.bm.binv1[g]);
        sg.logratio = up(s.bm.binlogratio[g]);
      } else {
        sg.w = up(std::vector<double>(s.bm.pix1[g].size(), 1.0));
        sg.ieta1 = up(s.bm.inv1[g]);
        sg.logratio = up(s.bm.logratio[g]);
      }
      sg.maxf1 = s.bm.hassign[g] ? knots_.back() * s.bm.maxbm1[g] : 0.0;
    }
    bd.T = std::max(nt[0] * bd.hassign[0] + nt[1] * bd.hassign[1],
                    nt[2] * bd.hassign[2] + nt[3] * bd.hassign[3]);
    if (bd.T < 1) bd.T = 1;
    if (bd.T > MAXT) throw Error(POFD_E_ARG, "beam has too many terms; histogram it");
    if (bd.T > Tmax_) Tmax_ = bd.T;
    bd.maxsb1 = s.maxsb1;
    bd.maxsb2 = s.maxsb2;
    bd.ds_begin = static_cast<int>(h_dsets_.size());
    bd.nds = static_cast<int>(s.data.size());
    for (size_t i = 0; i < s.data.size(); ++i) {
      const Data2& d = s.data[i];
      DSet2Dev dd{};
      dd.bs = static_cast<int>(b);
      dd.sb1 = s.sb1[i];
      dd.sb2 = s.sb2[i];
      dd.like_offset = s.lo[i];
      dd.like_norm = s.ln[i];
      std::vector<int> i1, i2;
      std::vector<double> c;
      dd.binned = d.binned ? 1 : 0;
      if (d.binned) {
        for (unsigned a = 0; a < d.nbins1; ++a)
          for (unsigned bb = 0; bb < d.nbins2; ++bb) {
            const uint32_t v = d.bins[static_cast<size_t>(a) * d.nbins2 + bb];
            if (v) { i1.push_back(static_cast<int>(a)); i2.push_back(static_cast<int>(bb)); c.push_back(v); }
          }
        dd.nnz = static_cast<int>(c.size());
        dd.f1 = dd.f2 = nullptr;
      } else {
        dd.nnz = static_cast<int>(d.d1.size());
        dd.f1 = up(d.d1);
        dd.f2 = up(d.d2);
      }
      dd.nzi1 = upi(i1);
      dd.nzi2 = upi(i2);
      dd.nzcnt = up(c);
      dd.bc1 = d.bc1; dd.bc2 = d.bc2; dd.bd1 = d.bd1; dd.bd2 = d.bd2;
      if (static_cast<unsigned>(dd.nnz) > maxnnz) maxnnz = static_cast<unsigned>(dd.nnz);
      h_dsets_.push_back(dd);
    }
  }
  D_ = static_cast<unsigned>(h_dsets_.size());
  for (auto& bd : h_bsets_) bd.Ts = Tmax_;  // common row stride of rw
  d_bsets_ = dal<BSet2Dev>(B_);
  static_allocs_.push_back(d_bsets_);
  ck(cudaMemcpy(d_bsets_, h_bsets_.data(), B_ * sizeof(BSet2Dev), cudaMemcpyHostToDevice), "upload");
  d_dsets_ = dal<DSet2Dev>(D_);
  static_allocs_.push_back(d_dsets_);
  ck(cudaMemcpy(d_dsets_, h_dsets_.data(), D_ * sizeof(DSet2Dev), cudaMemcpyHostToDevice), "upload");
  gx_ = (n + NT - 1) / NT;
  gy_ = (n - 1 + RB_MIN - 1) / RB_MIN;  // the most row groups any tuning uses
  nrt_ = (n + RTILE - 1) / RTILE;
  nct_ = (n + NT - 1) / NT;
  gchunks_ = (maxnnz + GCH - 1) / GCH;
  static_ok_ = true;
  drop_plans();
  setup_colspec();
  const unsigned P = ws_.P;
  free_work();
  if (P) reserve(P);
}

void Engine2::free_work() {
  void* ptrs[] = {ws_.cnt, ws_.mstatus, ws_.sigmult, ws_.rw, ws_.rcnt, ws_.rbuf,
                  ws_.rpart, ws_.redge, ws_.epart, ws_.fpart, ws_.mom, ws_.pbuf, ws_.rowpart,
                  ws_.colpart, ws_.pinfo, ws_.gpart, ws_.pdout,
                  ws_.theta_in, ws_.logl, ws_.status, ws_.bonus, ws_.bcnt,
                  ws_.bstatus, ws_.bsig, ws_.r0};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (ws_.h_theta) cudaFreeHost(ws_.h_theta);
  if (ws_.h_logl) cudaFreeHost(ws_.h_logl);
  if (ws_.h_status) cudaFreeHost(ws_.h_status);
  ws_ = Work{};
}

void Engine2::reserve(unsigned P) {
  if (P == 0) throw Error(POFD_E_ARG, "max_batch must be > 0");
  if (!static_ok_) {
    ws_.P = std::max(ws_.P, P);
    build_static();
    return;
  }
  if (ws_.P >= P && ws_.rbuf) return;
  // (proposal, beam set) and (proposal, dataset) pairs index grid y / z
  if (static_cast<size_t>(P) * std::max(B_, D_) > 65535u)
    throw Error(POFD_E_ARG, "batch x (beam sets or datasets) exceeds 65535");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  drop_graphs();
  free_work();
  const size_t n = n_, nc2 = 2 * (n / 2 + 1);
  size_t nrows = n + (edge_ ? nedge_ : 0);
  ws_.P = P;
  ws_.cnt = dal<double>(static_cast<size_t>(P) * 12 * KMAX);
  ws_.mstatus = dal<int>(P);
  ws_.sigmult = dal<double>(2 * static_cast<size_t>(P));
  ws_.bonus = dal<double>(8 * static_cast<size_t>(P));
  ws_.bcnt = dal<double>(static_cast<size_t>(P) * 12 * KMAX);
  ws_.bstatus = dal<int>(P);
  ws_.bsig = dal<double>(2 * static_cast<size_t>(P));
  ws_.rw = dal<double>(static_cast<size_t>(P) * B_ * nrows * Tmax_ * 3);
  ws_.rcnt = dal<int2>(static_cast<size_t>(P) * B_ * nrows);
  ws_.rbuf = dal<double>(static_cast<size_t>(P) * B_ * n * nc2);
  ws_.rpart = dal<double>(static_cast<size_t>(P) * B_ * gx_ * gy_ * 4);
  ws_.redge = dal<double>(static_cast<size_t>(P) * B_ * (2 * n + 1));
  const size_t ngr = edge_ ? (nedge_ + ER_MIN - 1) / ER_MIN : 0;
  ws_.epart = dal<double>(static_cast<size_t>(P) * B_ * (ngr ? ngr * (n + nedge_) : 1));
  ws_.mom = dal<double>(static_cast<size_t>(P) * B_ * 8);
  ws_.r0 = dal<double>(static_cast<size_t>(P) * B_);
  ws_.fpart = dal<double>(static_cast<size_t>(P) * B_ * ((n + NT - 1) / NT) * 4);
  ws_.pbuf = dal<double>(static_cast<size_t>(P) * D_ * n * nc2);
  ws_.rowpart = dal<double>(static_cast<size_t>(P) * D_ * n * nct_);
  ws_.colpart = dal<double>(static_cast<size_t>(P) * D_ * nrt_ * n);
  ws_.pinfo = dal<PDInfo2>(static_cast<size_t>(P) * D_);
  ws_.gpart = dal<double>(static_cast<size_t>(P) * D_ * gchunks_);
  ws_.pdout = dal<double>(n * n);
  ws_.logl = dal<double>(P);
  ws_.status = dal<int>(P);
  ck(cudaMemset(ws_.redge, 0, static_cast<size_t>(P) * B_ * (2 * n + 1) * sizeof(double)), "memset");
  ck(cudaFuncSetAttribute(k_psplit2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          static_cast<int>(3 * 8192 * sizeof(double))), "attr");
}

// Twiddle tables and kernel attributes of FFT mode 1 where the size allows.
void Engine2::setup_colspec() {
  const unsigned n = n_;
  colspec_ = fft_mode_ == 1 && (n == 512 || n == 1024 || n == 2048 || n == 4096);
  if (!colspec_) return;
  if (!d_cwh_) {
    std::vector<double2> wh(n / 32), wl(32);
    const long double tau = 6.283185307179586476925286766559005768L;
    for (unsigned h = 0; h < n / 32; ++h) {
      const long double a = -tau * static_cast<long double>(32 * h) / static_cast<long double>(n);
      wh[h] = make_double2(static_cast<double>(cosl(a)), static_cast<double>(sinl(a)));
    }
    for (unsigned l = 0; l < 32; ++l) {
      const long double a = -tau * static_cast<long double>(l) / static_cast<long double>(n);
      wl[l] = make_double2(static_cast<double>(cosl(a)), static_cast<double>(sinl(a)));
    }
    d_cwh_ = dal<double2>(wh.size());
    d_cwl_ = dal<double2>(wl.size());
    static_allocs_.push_back(d_cwh_);
    static_allocs_.push_back(d_cwl_);
    ck(cudaMemcpy(d_cwh_, wh.data(), wh.size() * sizeof(double2), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(d_cwl_, wl.data(), wl.size() * sizeof(double2), cudaMemcpyHostToDevice), "upload");
  }
  const int sm = static_cast<int>(colspec_smem(static_cast<int>(n)));
  switch (n) {
    case 512: ck(cudaFuncSetAttribute(k_colspec2<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr"); break;
    case 1024: ck(cudaFuncSetAttribute(k_colspec2<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr"); break;
    case 2048: ck(cudaFuncSetAttribute(k_colspec2<2048>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr"); break;
    default: ck(cudaFuncSetAttribute(k_colspec2<4096>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm), "attr"); break;
  }
}

void Engine2::drop_plans() {
  drop_graphs();
  for (auto& kv : plans_) {
    if (kv.second.fwd) { fftwork_.forget(kv.second.fwd); cufftDestroy(kv.second.fwd); }
    if (kv.second.inv) { fftwork_.forget(kv.second.inv); cufftDestroy(kv.second.inv); }
  }
  plans_.clear();
}

void Engine2::set_fft_mode(int mode) {
  if (mode != 0 && mode != 1) throw Error(POFD_E_ARG, "2D FFT mode must be 0 or 1");
  if (mode == fft_mode_) return;
  fft_mode_ = mode;
  if (device_ >= 0) ck(cudaSetDevice(device_), "cudaSetDevice");
  drop_plans();
  if (static_ok_) setup_colspec();
  else colspec_ = false;
}

double Engine2::time_sequence(unsigned nprop, const float* theta, unsigned npar, int reps) {
  std::vector<double> ll(nprop);
  std::vector<int> st(nprop);
  eval_host(nprop, theta, npar, ll.data(), st.data());
  enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);  // capture or warm
  enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);
  cudaEvent_t e0, e1;
  ck(cudaEventCreate(&e0), "event create");
  ck(cudaEventCreate(&e1), "event create");
  ck(cudaEventRecord(e0, stream_), "event record");
  for (int r = 0; r < reps; ++r) enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);
  ck(cudaEventRecord(e1, stream_), "event record");
  ck(cudaEventSynchronize(e1), "event sync");
  float ms = 0.f;
  ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return static_cast<double>(ms) / reps;
}

void Engine2::set_tuning(const Tune2& t) {
  if (t.fft_mode != 0 && t.fft_mode != 1) throw Error(POFD_E_ARG, "fft_mode must be 0 or 1");
  if (t.rgrid_rows != 2 && t.rgrid_rows != 4 && t.rgrid_rows != 8)
    throw Error(POFD_E_ARG, "rgrid_rows must be 2, 4 or 8");
  if (t.edge_rows != 4 && t.edge_rows != 8 && t.edge_rows != 16)
    throw Error(POFD_E_ARG, "edge_rows must be 4, 8 or 16");
  set_fft_mode(t.fft_mode);
  tune_ = t;
  drop_graphs();
}

// Coordinate descent over the knobs, one pass, each candidate timed on the
// captured graph of the whole sequence.
void Engine2::autotune(unsigned nprop, const float* theta, unsigned npar, int reps,
                       double* out5) {
  NvtxRange nvtx_range("pofd like2 autotune");
  if (nprop == 0 || reps < 1) throw Error(POFD_E_ARG, "autotune needs rows and reps >= 1");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  const double t_untuned = time_sequence(nprop, theta, npar, reps);
  Tune2 best = tuning();
  double best_ms = t_untuned;
  auto trial = [&](const Tune2& t) {
    set_tuning(t);
    const double ms = time_sequence(nprop, theta, npar, reps);
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  };
  {
    Tune2 t = best;
    t.fft_mode = best.fft_mode ? 0 : 1;
    trial(t);
  }
  for (int rb : {2, 4, 8}) {
    if (rb == best.rgrid_rows) continue;
    Tune2 t = best;
    t.rgrid_rows = rb;
    trial(t);
  }
  if (edge_) {
    for (int er : {4, 8, 16}) {
      if (er == best.edge_rows) continue;
      Tune2 t = best;
      t.edge_rows = er;
      trial(t);
    }
  }
  set_tuning(best);
  if (out5) {
    out5[0] = best.fft_mode;
    out5[1] = best.rgrid_rows;
    out5[2] = best.edge_rows;
    out5[3] = best_ms;
    out5[4] = t_untuned;
  }
}

void Engine2::set_reference_sums(bool on) {
  if (on == refsum_) return;
  refsum_ = on;
  drop_graphs();
}

void Engine2::ensure_plans(unsigned nprop) {
  auto it = plans_.find(nprop);
  if (it != plans_.end() && it->second.fwd) return;
  Plans pl;
  int nn[2] = {static_cast<int>(n_), static_cast<int>(n_)};
  const int nc = static_cast<int>(n_) / 2 + 1;
  if (colspec_) {
    // 1D row transforms of every (proposal, beam set) or (proposal, dataset)
    // grid: n rows each, padded real rows of 2 nc doubles / nc complex
    int n1[1] = {nn[0]};
    int ie[1] = {2 * nc}, oe[1] = {nc};
    bool grew = fftwork_.make(&pl.fwd, 1, n1, ie, 2 * nc, oe, nc, CUFFT_D2Z,
                              static_cast<int>(nprop * B_ * n_));
    int ie2[1] = {nc}, oe2[1] = {2 * nc};
    grew |= fftwork_.make(&pl.inv, 1, n1, ie2, nc, oe2, 2 * nc, CUFFT_Z2D,
                          static_cast<int>(nprop * D_ * n_));
    if (grew) drop_graphs();
    plans_[nprop] = pl;
    return;
  }
  int inemb[2] = {nn[0], 2 * nc}, onemb[2] = {nn[0], nc};
  bool grew = fftwork_.make(&pl.fwd, 2, nn, inemb, nn[0] * 2 * nc, onemb, nn[0] * nc,
                            CUFFT_D2Z, static_cast<int>(nprop * B_));
  int inemb2[2] = {nn[0], nc}, onemb2[2] = {nn[0], 2 * nc};
  grew |= fftwork_.make(&pl.inv, 2, nn, inemb2, nn[0] * nc, onemb2, nn[0] * 2 * nc, CUFFT_Z2D,
                        static_cast<int>(nprop * D_));
  if (grew) drop_graphs();  // captured transforms used the old work area
  plans_[nprop] = pl;
}

void Engine2::launch_all(unsigned nprop, const float* theta, unsigned npar,
                         double* logl, int* status, cudaStream_t st,
                         cudaEvent_t* ev, bool r_only) {
  auto mark = [&](int i) {
    if (ev) ck(cudaEventRecord(ev[i], st), "event record");
  };
  const int n = static_cast<int>(n_), nc = n / 2 + 1, nc2 = 2 * nc;
  const int P = static_cast<int>(nprop), B = static_cast<int>(B_), D = static_cast<int>(D_);
  const int ne = edge_ ? static_cast<int>(nedge_) : 0;
  Plans& pl = plans_.at(nprop);
  mark(0);
  k_model2<<<P, 32, 0, st>>>(model_, theta, static_cast<int>(npar), std::log2(10.0),
                             ws_.cnt, ws_.mstatus, ws_.sigmult);
  if (prior_.needs_bonus())
    k_bonus2<<<P, kBonus2Threads, 0, st>>>(model_, const_cast<float*>(theta), static_cast<int>(npar),
                                           std::log2(10.0), ws_.cnt, ws_.mstatus, d_qu_, d_qs_,
                                           d_qw_, d_qk_, nq_, ws_.bonus, -1);
  mark(1);
  {
    const unsigned nrows = static_cast<unsigned>(n + ne);
    const unsigned gxr = (nrows + ROWS_PER_BLOCK - 1) / ROWS_PER_BLOCK;
    k_rows2<<<dim3(gxr, P * B), NT, 0, st>>>(d_bsets_, model_, B, 1.0 / std::log(2.),
                                             ws_.mstatus, ws_.cnt, ws_.rw, ws_.rcnt);
  }
  mark(2);
  const int rb = tune_.rgrid_rows;
  const unsigned gy = static_cast<unsigned>((n - 1 + rb - 1) / rb);
  const unsigned gxg = static_cast<unsigned>((n + RG_COLS - 1) / RG_COLS);
  switch (rb) {
    case 2:
      k_rgrid2<2><<<dim3(gxg, gy, P * B), NT, 0, st>>>(d_bsets_, B, n, nc2, ws_.mstatus, ws_.rw,
                                                       ws_.rcnt, ws_.rbuf, ws_.rpart);
      break;
    case 8:
      k_rgrid2<8><<<dim3(gxg, gy, P * B), NT, 0, st>>>(d_bsets_, B, n, nc2, ws_.mstatus, ws_.rw,
                                                       ws_.rcnt, ws_.rbuf, ws_.rpart);
      break;
    default:
      k_rgrid2<4><<<dim3(gxg, gy, P * B), NT, 0, st>>>(d_bsets_, B, n, nc2, ws_.mstatus, ws_.rw,
                                                       ws_.rcnt, ws_.rbuf, ws_.rpart);
  }
  mark(3);
  const int er = tune_.edge_rows;
  const int ngr = (ne + er - 1) / er;
  if (edge_) {
    const unsigned gxe = static_cast<unsigned>((n + ne + RG_COLS - 1) / RG_COLS);
    switch (er) {
      case 4:
        k_redge2<4><<<dim3(gxe, ngr, P * B), NT, 0, st>>>(d_bsets_, B, n, ne, ws_.mstatus, ws_.rw,
                                                          ws_.rcnt, ws_.epart);
        break;
      case 16:
        k_redge2<16><<<dim3(gxe, ngr, P * B), NT, 0, st>>>(d_bsets_, B, n, ne, ws_.mstatus, ws_.rw,
                                                           ws_.rcnt, ws_.epart);
        break;
      default:
        k_redge2<8><<<dim3(gxe, ngr, P * B), NT, 0, st>>>(d_bsets_, B, n, ne, ws_.mstatus, ws_.rw,
                                                          ws_.rcnt, ws_.epart);
    }
    k_ry2<<<dim3((n - 1 + RY_ROWS - 1) / RY_ROWS, P * B), NT, 0, st>>>(
        d_bsets_, B, n, ne, ws_.mstatus, ws_.rw, ws_.rcnt, ws_.redge);
  }
  mark(4);
  {
    const int nfp = (n + NT - 1) / NT;
    k_rfinish2<<<dim3(nfp, P * B), NT, 0, st>>>(d_bsets_, B, n, nc2, edge_ ? 1 : 0, ne, ngr,
                                                static_cast<int>(gxg * gy), ws_.mstatus,
                                                ws_.redge, ws_.epart, ws_.rpart, ws_.rbuf,
                                                ws_.fpart);
    k_rfinal2<<<P * B, NT, 0, st>>>(d_bsets_, B, n, nc2, edge_ ? 1 : 0, ne, ngr, nfp,
                                    ws_.mstatus, ws_.epart, ws_.fpart, ws_.rbuf, ws_.mom);
  }
  mark(5);
  if (r_only) {
    ck(cudaGetLastError(), "kernel launch");
    return;
  }
  fk(cufftSetStream(pl.fwd, st), "cufftSetStream");
  fk(cufftExecD2Z(pl.fwd, ws_.rbuf, reinterpret_cast<cufftDoubleComplex*>(ws_.rbuf)),
     colspec_ ? "cufftExecD2Z rows" : "cufftExecD2Z 2D");
  mark(6);
  if (colspec_) {
    k_r0sum2<<<P * B, NT, 0, st>>>(n, nc, ws_.mstatus, B, ws_.rbuf, ws_.r0);
    const int C = CS_THREADS / (n / 16);
    const dim3 g((nc + C - 1) / C, P * B);
    const size_t sm = colspec_smem(n);
#define POFD_CS(NN)                                                                        \
  k_colspec2<NN><<<g, CS_THREADS, sm, st>>>(d_bsets_, d_dsets_, B, D, ws_.mstatus,          \
                                             ws_.sigmult, ws_.mom, ws_.r0, ws_.rbuf, ws_.pbuf, \
                                             d_cwh_, d_cwl_)
    switch (n) {
      case 512: POFD_CS(512); break;
      case 1024: POFD_CS(1024); break;
      case 2048: POFD_CS(2048); break;
      case 4096: POFD_CS(4096); break;
      default: throw Error(POFD_E_ARG, "column transform: unsupported size");
    }
#undef POFD_CS
  } else {
    const unsigned gs = static_cast<unsigned>((static_cast<size_t>(n) * nc + NT - 1) / NT);
    k_spectrum2<<<dim3(gs, P * B), NT, 0, st>>>(d_bsets_, d_dsets_, B, D, n, nc, ws_.mstatus,
                                                ws_.sigmult, ws_.mom, ws_.rbuf, ws_.pbuf);
  }
  mark(7);
  fk(cufftSetStream(pl.inv, st), "cufftSetStream");
  fk(cufftExecZ2D(pl.inv, reinterpret_cast<cufftDoubleComplex*>(ws_.pbuf), ws_.pbuf),
     colspec_ ? "cufftExecZ2D rows" : "cufftExecZ2D 2D");
  mark(8);
  k_pscan2<<<dim3(nct_, nrt_, P * D), NT, 0, st>>>(D, n, nc2, ws_.mstatus, ws_.pbuf,
                                                    ws_.rowpart, ws_.colpart);
  mark(9);
  k_psplit2<<<P * D, SNT, 3 * static_cast<size_t>(n) * sizeof(double), st>>>(
      d_bsets_, d_dsets_, B, D, n, nc2, static_cast<int>(nct_), static_cast<int>(nrt_),
      ws_.mstatus, ws_.sigmult, ws_.mom, ws_.pbuf, ws_.rowpart, ws_.colpart, ws_.pinfo);
  if (refsum_)
    k_pseq2<<<P * D, NT, static_cast<size_t>(n) * sizeof(double), st>>>(
        d_bsets_, d_dsets_, D, n, nc2, ws_.mstatus, ws_.pbuf, ws_.pinfo);
  mark(10);
  k_pgather2<<<dim3(gchunks_, P * D), NT, 0, st>>>(d_bsets_, d_dsets_, D, n, nc2,
                                                    static_cast<int>(gchunks_), ws_.mstatus,
                                                    ws_.pbuf, ws_.pinfo, ws_.gpart);
  mark(11);
  k_reduce2<<<(P + 127) / 128, 128, 0, st>>>(d_bsets_, d_dsets_, B, D, P,
                                            static_cast<int>(gchunks_), std::log(2.0),
                                            ws_.mstatus, ws_.sigmult, ws_.pinfo,
                                            ws_.gpart, prior_, ws_.bonus, logl, status);
  mark(12);
  ck(cudaGetLastError(), "kernel launch");
}

cudaGraphExec_t Engine2::graph_for(unsigned nprop, const float* theta,
                                   unsigned npar, double* logl, int* status) {
  Plans& pl = plans_.at(nprop);
  if (pl.no_graph) return nullptr;
  const GraphKey key{theta, npar, logl, status};
  for (auto& kv : pl.graphs)
    if (kv.first == key) return kv.second;
  if (!pl.warmed) {
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
    pl.no_graph = true;
    return nullptr;
  }
  if (pl.graphs.size() >= 8) {
    cudaGraphExecDestroy(pl.graphs.front().second);
    pl.graphs.erase(pl.graphs.begin());
  }
  pl.graphs.push_back({key, ge});
  return ge;
}

void Engine2::enqueue(unsigned nprop, const float* theta_dev, unsigned npar,
                      double* logl_dev, int* status_dev, cudaStream_t st) {
  NvtxRange nvtx_range("pofd like2 enqueue");
  if (nprop == 0) return;
  if (npar < nparams() + 2) throw Error(POFD_E_ARG, "Not enough elements in params");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ensure_plans(nprop);
  if (!st) st = stream_;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ck(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing");
  if (cs != cudaStreamCaptureStatusNone) {
    launch_all(nprop, theta_dev, npar, logl_dev, status_dev, st, nullptr);
    return;
  }
  cudaGraphExec_t g = graph_for(nprop, theta_dev, npar, logl_dev, status_dev);
  if (g) ck(cudaGraphLaunch(g, st), "graph launch");
  else launch_all(nprop, theta_dev, npar, logl_dev, status_dev, st, nullptr);
}

void Engine2::eval_host(unsigned nprop, const float* theta, unsigned npar,
                        double* logl, int* status) {
  NvtxRange nvtx_range("pofd like2 eval_batch");
  if (nprop == 0) return;
  if (npar < nparams() + 2) throw Error(POFD_E_ARG, "Not enough elements in params");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (!ws_.theta_in || ws_.h_npar < npar) {
    if (ws_.theta_in) cudaFree(ws_.theta_in);
    if (ws_.h_theta) cudaFreeHost(ws_.h_theta);
    ws_.theta_in = dal<float>(static_cast<size_t>(ws_.P) * npar);
    ck(cudaMallocHost(&ws_.h_theta, static_cast<size_t>(ws_.P) * npar * sizeof(float)), "cudaMallocHost");
    ws_.h_npar = npar;
    drop_graphs();
  }
  if (!ws_.h_logl) {
    ck(cudaMallocHost(&ws_.h_logl, ws_.P * sizeof(double)), "cudaMallocHost");
    ck(cudaMallocHost(&ws_.h_status, ws_.P * sizeof(int)), "cudaMallocHost");
  }
  std::memcpy(ws_.h_theta, theta, static_cast<size_t>(nprop) * npar * sizeof(float));
  ck(cudaMemcpyAsync(ws_.theta_in, ws_.h_theta, static_cast<size_t>(nprop) * npar * sizeof(float),
                     cudaMemcpyHostToDevice, stream_), "H2D theta");
  enqueue(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_);
  ck(cudaMemcpyAsync(ws_.h_logl, ws_.logl, nprop * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H");
  ck(cudaMemcpyAsync(ws_.h_status, ws_.status, nprop * sizeof(int), cudaMemcpyDeviceToHost, stream_), "D2H");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  std::memcpy(logl, ws_.h_logl, nprop * sizeof(double));
  std::memcpy(status, ws_.h_status, nprop * sizeof(int));
}

// Prior setters (calcLikeDouble.h:310-341); prior values are launch
// arguments of the reduction kernel, so captured graphs are dropped.
void Engine2::set_sigma_prior(int band, bool on, double width) {
  if (band != 0 && band != 1) throw Error(POFD_E_ARG, "band must be 0 or 1");
  if (on && !(width > 0.0)) throw Error(POFD_E_ARG, "Invalid (non-positive) sigma prior width");
  prior_.has_sigma[band] = on ? 1 : 0;
  if (on) {
    prior_.sigma_width[band] = width;
    prior_.log_sigma_width[band] = std::log(width);
  }
  drop_graphs();
}

void Engine2::set_cfirb_prior(int band, bool on, double mean, double sigma) {
  if (band != 0 && band != 1) throw Error(POFD_E_ARG, "band must be 0 or 1");
  if (on) {
    if (mean < 0.0) throw Error(POFD_E_ARG, "Invalid (negative) CFIRB mean");
    if (!(sigma > 0.0)) throw Error(POFD_E_ARG, "Invalid (non-positive) CFIRB sigma");
    prior_.cfirb_mean[band] = mean;
    prior_.cfirb_sigma[band] = sigma;
    prior_.log_cfirb_sigma[band] = std::log(sigma);
  }
  prior_.has_cfirb[band] = on ? 1 : 0;
  drop_graphs();
}

void Engine2::set_poisson_prior(int band, bool on, double mean, double sigma) {
  if (band != 0 && band != 1) throw Error(POFD_E_ARG, "band must be 0 or 1");
  if (on) {
    if (mean < 0.0) throw Error(POFD_E_ARG, "Invalid (negative) Poisson prior mean");
    if (!(sigma > 0.0)) throw Error(POFD_E_ARG, "Invalid (non-positive) Poisson prior sigma");
    prior_.poisson_mean[band] = mean;
    prior_.poisson_sigma[band] = sigma;
    prior_.log_poisson_sigma[band] = std::log(sigma);
  }
  prior_.has_poisson[band] = on ? 1 : 0;
  drop_graphs();
}

void Engine2::set_regularization(double alpha) {
  if (!(alpha >= 0.0)) throw Error(POFD_E_ARG, "Invalid (negative) regularization alpha");
  prior_.alpha = alpha;
  drop_graphs();
}

// Model set-up into the bonus scratch, then the integrals (fill_at < 0:
// into ws_.bonus).
void Engine2::bonus_launch(unsigned nprop, float* theta_dev, unsigned npar, int fill_at,
                           cudaStream_t st) {
  const int P = static_cast<int>(nprop);
  k_model2<<<P, 32, 0, st>>>(model_, theta_dev, static_cast<int>(npar), std::log2(10.0),
                             ws_.bcnt, ws_.bstatus, ws_.bsig);
  k_bonus2<<<P, kBonus2Threads, 0, st>>>(model_, theta_dev, static_cast<int>(npar),
                                         std::log2(10.0), ws_.bcnt, ws_.bstatus, d_qu_, d_qs_,
                                         d_qw_, d_qk_, nq_, fill_at < 0 ? ws_.bonus : nullptr,
                                         fill_at);
  ck(cudaGetLastError(), "k_bonus2");
}

void Engine2::bonus_host(unsigned nprop, const float* theta, unsigned npar, double* out) {
  if (nprop == 0) return;
  if (npar < nparams() + 2) throw Error(POFD_E_ARG, "Not enough elements in params");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  ck(cudaSetDevice(device_), "cudaSetDevice");
  const size_t nb = static_cast<size_t>(nprop) * npar * sizeof(float);
  float* d = nullptr;
  ck(cudaMalloc(&d, nb), "cudaMalloc");
  std::vector<double> o(static_cast<size_t>(nprop) * 8);
  cudaError_t e = cudaMemcpyAsync(d, theta, nb, cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) {
    try {
      bonus_launch(nprop, d, npar, -1, stream_);
    } catch (...) {
      cudaFree(d);
      throw;
    }
    e = cudaMemcpyAsync(o.data(), ws_.bonus, o.size() * sizeof(double), cudaMemcpyDeviceToHost,
                        stream_);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  cudaFree(d);
  ck(e, "bonus evaluation");
  for (unsigned i = 0; i < nprop; ++i)
    for (int c = 0; c < 4; ++c) out[4 * i + c] = o[8 * i + c];
}

void Engine2::fill_bonus(unsigned nprop, float* theta_dev, unsigned npar, cudaStream_t st) {
  if (nprop == 0) return;
  const unsigned nm = nparams();
  if (npar < nm + 6) throw Error(POFD_E_ARG, "Not enough room to fill");
  if (!static_ok_ || ws_.P < nprop) reserve(std::max(nprop, ws_.P));
  ck(cudaSetDevice(device_), "cudaSetDevice");
  bonus_launch(nprop, theta_dev, npar, static_cast<int>(nm + 2), st ? st : stream_);
}

int Engine2::pd_host(int bs, int ds, const float* theta, unsigned npar,
                     bool setlog, double* pd_out, double* info16) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  if (ds < 0 || ds >= static_cast<int>(sets_[bs].data.size())) throw Error(POFD_E_ARG, "invalid dataset index");
  double ll;
  int st;
  eval_host(1, theta, npar, &ll, &st);
  const int d = h_bsets_[bs].ds_begin + ds;
  PDInfo2 info;
  ck(cudaMemcpy(&info, ws_.pinfo + d, sizeof(PDInfo2), cudaMemcpyDeviceToHost), "D2H info");
  double mom[8];
  ck(cudaMemcpy(mom, ws_.mom + static_cast<size_t>(bs) * 8, sizeof(mom), cudaMemcpyDeviceToHost), "D2H mom");
  if (info16) {
    const BSet2Dev& b = h_bsets_[bs];
    info16[0] = b.dflux1; info16[1] = b.dflux2; info16[2] = mom[0]; info16[3] = mom[1];
    info16[4] = mom[2]; info16[5] = mom[3]; info16[6] = mom[4]; info16[7] = mom[5];
    info16[8] = info.s1; info16[9] = info.s2; info16[10] = info.minflux1; info16[11] = info.minflux2;
    info16[12] = info.sg1pos; info16[13] = info.sg1neg; info16[14] = info.sg2pos; info16[15] = info.sg2neg;
  }
  if (info.status != 0) return info.status;
  const size_t n = n_, nc2 = 2 * (n / 2 + 1);
  const unsigned blocks = static_cast<unsigned>((n * n + 255) / 256);
  k_pdwrite2<<<blocks, 256, 0, stream_>>>(ws_.pbuf + static_cast<size_t>(d) * n * nc2,
                                          static_cast<int>(n), static_cast<int>(nc2), info.s1,
                                          info.s2, info.itot, setlog ? 1 : 0, ws_.pdout);
  ck(cudaGetLastError(), "pdwrite2");
  ck(cudaMemcpyAsync(pd_out, ws_.pdout, n * n * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H pd");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  return 0;
}

void Engine2::active_terms(const float* theta, unsigned npar, long long* out2) {
  double ll;
  int st;
  eval_host(1, theta, npar, &ll, &st);
  out2[0] = out2[1] = 0;
  for (unsigned b = 0; b < B_; ++b) {
    const BSet2Dev& bs = h_bsets_[b];
    std::vector<int2> rc(bs.nrows);
    ck(cudaMemcpy(rc.data(), ws_.rcnt + static_cast<size_t>(b) * bs.nrows,
                  rc.size() * sizeof(int2), cudaMemcpyDeviceToHost), "D2H row counts");
    for (int r = 1; r < bs.nrows; ++r)
      out2[r < static_cast<int>(n_) ? 0 : 1] += rc[r].x + rc[r].y;
  }
}

void Engine2::rgrid_host(int bs, const float* theta, unsigned npar, double* out) {
  if (bs < 0 || bs >= static_cast<int>(sets_.size())) throw Error(POFD_E_ARG, "invalid beam set index");
  double ll;
  int st;
  eval_host(1, theta, npar, &ll, &st);  // staging, plans
  ck(cudaMemcpy(ws_.theta_in, theta, npar * sizeof(float), cudaMemcpyHostToDevice), "H2D");
  launch_all(1, ws_.theta_in, npar, ws_.logl, ws_.status, stream_, nullptr, true);
  const size_t n = n_, nc2 = 2 * (n / 2 + 1);
  ck(cudaMemcpy2DAsync(out, n * sizeof(double), ws_.rbuf + static_cast<size_t>(bs) * n * nc2,
                       nc2 * sizeof(double), n * sizeof(double), n, cudaMemcpyDeviceToHost, stream_),
     "D2H R grid");
  ck(cudaStreamSynchronize(stream_), "synchronize");
}

void Engine2::profile_stages(unsigned nprop, const float* theta, unsigned npar,
                             int reps, double* stage_ms) {
  std::vector<double> lls(nprop);
  std::vector<int> sts(nprop);
  eval_host(nprop, theta, npar, lls.data(), sts.data());
  cudaEvent_t ev[kNumStages + 1];
  for (auto& e : ev) ck(cudaEventCreate(&e), "event create");
  for (int k = 0; k < kNumStages; ++k) stage_ms[k] = 0.0;
  for (int r = 0; r < reps; ++r) {
    launch_all(nprop, ws_.theta_in, npar, ws_.logl, ws_.status, stream_, ev);
    ck(cudaStreamSynchronize(stream_), "synchronize");
    for (int k = 0; k < kNumStages; ++k) {
      float ms = 0.f;
      ck(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]), "elapsed");
      stage_ms[k] += ms / reps;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
}

const char* Engine2::stage_name(int i) {
  static const char* names[kNumStages] = {
      "k_model2", "k_rows2", "k_rgrid2", "k_redge2+k_ry2", "k_rfinish2+k_rfinal2",
      "cufft_d2z_2d", "k_spectrum2", "cufft_z2d_2d", "k_pscan2", "k_psplit2",
      "k_pgather2", "k_reduce2"};
  return (i >= 0 && i < kNumStages) ? names[i] : "";
}

const char* Engine2::stage_name_now(int i) const {
  static const char* names[kNumStages] = {
      "k_model2", "k_rows2", "k_rgrid2", "k_redge2+k_ry2", "k_rfinish2+k_rfinal2",
      "cufft_d2z_rows", "k_r0sum2+k_colspec2", "cufft_z2d_rows", "k_pscan2", "k_psplit2",
      "k_pgather2", "k_reduce2"};
  if (!colspec_) return stage_name(i);
  return (i >= 0 && i < kNumStages) ? names[i] : "";
}

}  // namespace pofd
