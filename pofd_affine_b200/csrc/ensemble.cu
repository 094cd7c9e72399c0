// ensemble.cu -- batched stretch-move ensemble and acor.
#include "ensemble.cuh"

#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>

#include "common.cuh"
#include "setup.hh"
#include "surrogate.cuh"

namespace pofd {

namespace {

constexpr int ENT = 128;
constexpr unsigned kMaxIters = 40;  // affineEnsemble.cc:1150

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
  return static_cast<T*>(p);
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds of the two 32x32->64 multiplies with
// the published multipliers and Weyl key increments.
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

__device__ __forceinline__ uint4 draw(unsigned long long seed,
                                      unsigned long long step, unsigned walker,
                                      unsigned tag) {
  return philox(make_uint4(static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32),
                           walker, tag),
                make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)));
}

// uniform float in [0, 1) with 24 random bits (ran::flt)
__device__ __forceinline__ float u01f(uint32_t x) {
  return static_cast<float>(x >> 8) * (1.0f / 16777216.0f);
}
// uniform double in [0, 1) with 53 random bits (ran::doub)
__device__ __forceinline__ double u01d(uint32_t a, uint32_t b) {
  const unsigned long long v =
      (static_cast<unsigned long long>(a >> 5) << 26) | static_cast<unsigned long long>(b >> 6);
  return static_cast<double>(v) * (1.0 / 9007199254740992.0);
}

// generateZ (affineEnsemble.cc:116-126): z = ((a-1) u + 1)^2 / a, u ~ U[0,1)
__device__ __forceinline__ float gen_z(double a, uint32_t x) {
  const double val = __dadd_rn(__dmul_rn(a - 1.0, static_cast<double>(u01f(x))), 1.0);
  return static_cast<float>(__ddiv_rn(__dmul_rn(val, val), a));
}

__device__ __forceinline__ bool valid_param(float v, float lo, float hi) {
  return v >= lo && v <= hi;  // NaN fails
}

// generateNewStep (affineEnsemble.cc:1144-1228) for one half of the
// ensemble: walker i combines with a uniformly drawn partner of the other
// half, retrying z up to 40 more times while the step is invalid.  With
// reject_outside the first z is kept and a step outside the limits is
// rejected (the limits act as a prior that is zero outside them): no
// retries, no error.  Redrawing z until the step is inside makes the
// proposal's normalisation depend on the walker's distance to a limit, which
// breaks detailed balance for walkers near one; rejecting keeps the move
// exact for the posterior truncated to the limits.
__global__ void k_propose(int half, unsigned nw, unsigned np, double scalefac,
                          int reject_outside, unsigned long long seed,
                          const int* __restrict__ pstate,
                          const float* __restrict__ plo,
                          const float* __restrict__ phi,
                          const float* __restrict__ theta,
                          float* __restrict__ prop, float* __restrict__ zout,
                          const unsigned long long* __restrict__ ctr,
                          int* __restrict__ err) {
  const unsigned nh0 = nw / 2;
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned nh = half ? nw - nh0 : nh0;
  if (t >= nh) return;
  const unsigned i = half ? nh0 + t : t;
  const unsigned pmin = half ? 0u : nh0, prange = half ? nh0 : nw - nh0;
  const unsigned long long step = ctr[0];
  const uint4 r0 = draw(seed, step, i, static_cast<unsigned>(half) << 16);
  const unsigned j = pmin + static_cast<unsigned>((static_cast<unsigned long long>(r0.x) * prange) >> 32);
  const float* xo = theta + static_cast<size_t>(i) * np;
  const float* xj = theta + static_cast<size_t>(j) * np;
  float* y = prop + static_cast<size_t>(t) * np;
  const float qnan = __int_as_float(0x7fc00000);
  float z = gen_z(scalefac, r0.y);
  bool ok = false;
  for (unsigned iter = 0;; ++iter) {
    const float omz = 1.0f - z;
    ok = true;
    for (unsigned p = 0; p < np; ++p) {
      const int s = pstate[p];
      float v;
      if (s & POFD_PARAM_FIXED) {
        v = xo[p];
      } else if (s & POFD_PARAM_BONUS) {
        v = qnan;
      } else {
        v = __fadd_rn(__fmul_rn(z, xo[p]), __fmul_rn(omz, xj[p]));
        if (!valid_param(v, plo[p], phi[p])) ok = false;
      }
      y[p] = v;
    }
    if (ok || reject_outside || iter > kMaxIters) break;
    const uint4 rr = draw(seed, step, i, (static_cast<unsigned>(half) << 16) | (iter + 1));
    z = gen_z(scalefac, rr.x);
  }
  if (!ok) {
    // "Unable to generate new step after 40 tries" (or a step outside the
    // limits under reject_outside): evaluate the old position and reject it
    for (unsigned p = 0; p < np; ++p) y[p] = xo[p];
    z = qnan;
    if (!reject_outside && atomicCAS(err, 0, 1) == 0) err[1] = static_cast<int>(i);
  }
  zout[t] = z;
}

// Acceptance (affineEnsemble.cc:1360-1433): rejected parameters keep the
// old step; otherwise accept with min(1, z^(nparams-nfixed-1) e^{dL/T}).
// The second half also writes the step into the chain.
__global__ void k_accept(int half, unsigned nw, unsigned np, double zexp,
                         double invtemp, unsigned long long seed, int reject_fail,
                         unsigned long long* __restrict__ nfail,
                         const float* __restrict__ prop,
                         const float* __restrict__ zin,
                         const double* __restrict__ lnew,
                         const int* __restrict__ snew, float* __restrict__ theta,
                         double* __restrict__ logl, unsigned* __restrict__ nacc,
                         const unsigned long long* __restrict__ ctr,
                         int* __restrict__ err, float* __restrict__ ch_theta,
                         double* __restrict__ ch_logl, unsigned cap) {
  const unsigned nh0 = nw / 2;
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned nh = half ? nw - nh0 : nh0;
  if (t < nh) {
    const unsigned i = half ? nh0 + t : t;
    const float z = zin[t];
    const int s = snew[t];
    const double ln = lnew[t];
    bool take = false;
    if (isnan(z) || s == POFD_REJECTED) {
      take = false;
    } else if (s != POFD_OK || isinf(ln) || isnan(ln)) {
      if (reject_fail) {
        atomicAdd(nfail, 1ull);
      } else if (s != POFD_OK) {
        if (atomicCAS(err, 0, 2) == 0) { err[1] = static_cast<int>(i); err[2] = s; }
      } else {
        if (atomicCAS(err, 0, 3) == 0) err[1] = static_cast<int>(i);
      }
    } else {
      const double prob = exp(zexp * log(static_cast<double>(z)) + invtemp * (ln - logl[i]));
      if (prob >= 1.0) {
        take = true;
      } else {
        const uint4 r = draw(seed, ctr[0], i, (static_cast<unsigned>(half) << 16) | 0x8000u);
        take = u01d(r.x, r.y) < prob;
      }
    }
    if (take) {
      const float* y = prop + static_cast<size_t>(t) * np;
      float* x = theta + static_cast<size_t>(i) * np;
      for (unsigned p = 0; p < np; ++p) x[p] = y[p];
      logl[i] = ln;
      nacc[i] += 1;
    }
  }
  if (half == 1 && t < nh && ctr[2] != 0ull && ctr[1] < cap) {
    // after the second half every walker is final: thread t records its own
    // second-half walker and, for t < nw/2, first-half walker t
    const size_t rec = static_cast<size_t>(ctr[1]);
    const unsigned ws[2] = {t, nh0 + t};
    for (int q = (t < nh0) ? 0 : 1; q < 2; ++q) {
      const unsigned w = ws[q];
      const float* x = theta + static_cast<size_t>(w) * np;
      float* o = ch_theta + (rec * nw + w) * np;
      for (unsigned p = 0; p < np; ++p) o[p] = x[p];
      ch_logl[rec * nw + w] = logl[w];
    }
  }
}

// Delayed acceptance, stage one (Christen & Fox 2005): accept with
// min(1, z^zexp e^{(S' - S)/T}) on the first-stage values; survivors are
// compacted in walker order into exprop / exidx.  One block.
__global__ void k_stage1(int half, unsigned nw, unsigned np, double zexp, double invtemp,
                         unsigned long long seed, const float* __restrict__ prop,
                         const float* __restrict__ zin, const double* __restrict__ spred,
                         const int* __restrict__ sst, const double* __restrict__ scur,
                         const unsigned long long* __restrict__ ctr,
                         float* __restrict__ exprop, int* __restrict__ exidx,
                         int* __restrict__ count) {
  __shared__ int wsum[32];
  __shared__ int base;
  const unsigned nh0 = nw / 2;
  const unsigned nh = half ? nw - nh0 : nh0;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (unsigned b0 = 0; b0 < nh; b0 += blockDim.x) {
    const unsigned t = b0 + threadIdx.x;
    bool pass = false;
    if (t < nh) {
      const unsigned i = half ? nh0 + t : t;
      const float z = zin[t];
      if (!isnan(z) && sst[t] == POFD_OK) {
        const double a = exp(zexp * log(static_cast<double>(z)) + invtemp * (spred[t] - scur[i]));
        if (a >= 1.0) {
          pass = true;
        } else {
          const uint4 r = draw(seed, ctr[0], i, (static_cast<unsigned>(half) << 16) | 0x4000u);
          pass = u01d(r.x, r.y) < a;
        }
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, pass);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int k = 0; k < w; ++k) off += wsum[k];
    const int pos = off + __popc(bal & ((1u << lane) - 1u));
    if (pass) {
      exidx[pos] = static_cast<int>(t);
      for (unsigned p = 0; p < np; ++p)
        exprop[static_cast<size_t>(pos) * np + p] = prop[static_cast<size_t>(t) * np + p];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) tot += wsum[k];
      base += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = base;
}

// Pads the survivor batch to its bucket size with copies of survivor 0.
__global__ void k_pad(int count, int b, unsigned np, float* __restrict__ exprop) {
  const int r = count + blockIdx.x;
  if (r >= b) return;
  for (unsigned p = threadIdx.x; p < np; p += blockDim.x)
    exprop[static_cast<size_t>(r) * np + p] = exprop[p];
}

// Stage two: min(1, e^{((L' - L) - (S' - S))/T}) on the exact values.
__global__ void k_stage2(int half, unsigned nw, unsigned np, double invtemp,
                         unsigned long long seed, int reject_fail,
                         unsigned long long* __restrict__ nfail, int count, const int* __restrict__ exidx,
                         const float* __restrict__ exprop, const double* __restrict__ exl,
                         const int* __restrict__ exs, const double* __restrict__ spred,
                         float* __restrict__ theta, double* __restrict__ logl,
                         double* __restrict__ scur, unsigned* __restrict__ nacc,
                         const unsigned long long* __restrict__ ctr, int* __restrict__ err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const unsigned nh0 = nw / 2;
  const int t = exidx[q];
  const unsigned i = half ? nh0 + t : t;
  const int s = exs[q];
  const double ln = exl[q];
  if (s == POFD_REJECTED) return;
  if (s != POFD_OK || isinf(ln) || isnan(ln)) {
    if (reject_fail) {
      atomicAdd(nfail, 1ull);
    } else if (s != POFD_OK) {
      if (atomicCAS(err, 0, 2) == 0) { err[1] = static_cast<int>(i); err[2] = s; }
    } else {
      if (atomicCAS(err, 0, 3) == 0) err[1] = static_cast<int>(i);
    }
    return;
  }
  const double a = exp(invtemp * ((ln - logl[i]) - (spred[t] - scur[i])));
  bool take;
  if (a >= 1.0) {
    take = true;
  } else {
    const uint4 r = draw(seed, ctr[0], i, (static_cast<unsigned>(half) << 16) | 0x8000u);
    take = u01d(r.x, r.y) < a;
  }
  if (take) {
    const float* y = exprop + static_cast<size_t>(q) * np;
    float* x = theta + static_cast<size_t>(i) * np;
    for (unsigned p = 0; p < np; ++p) x[p] = y[p];
    logl[i] = ln;
    scur[i] = spred[t];
    nacc[i] += 1;
  }
}

__global__ void k_record(unsigned nw, unsigned np, const float* __restrict__ theta,
                         const double* __restrict__ logl,
                         const unsigned long long* __restrict__ ctr,
                         float* __restrict__ ch_theta, double* __restrict__ ch_logl,
                         unsigned cap) {
  const unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw || ctr[2] == 0ull || ctr[1] >= cap) return;
  const size_t rec = static_cast<size_t>(ctr[1]);
  for (unsigned p = 0; p < np; ++p)
    ch_theta[(rec * nw + w) * np + p] = theta[static_cast<size_t>(w) * np + p];
  ch_logl[rec * nw + w] = logl[w];
}

__global__ void k_advance(unsigned long long* ctr, unsigned cap) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (ctr[2] != 0ull && ctr[1] < cap) ctr[1] += 1;
    ctr[0] += 1;
  }
}

}  // namespace

Ensemble::Ensemble(int device, cudaStream_t stream, unsigned nwalkers,
                   unsigned npar, double scalefac, uint64_t seed)
    : device_(device), stream_(stream), nw_(nwalkers), np_(npar),
      scalefac_(scalefac), seed_(seed) {
  if (device < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  if (nwalkers < 2) throw Error(POFD_E_ARG, "Need at least 2 walkers");
  if (npar == 0 || npar > kMaxParams) throw Error(POFD_E_ARG, "nparams must be in [1, 64]");
  if (!(scalefac > 1.0)) throw Error(POFD_E_ARG, "scalefac must be > 1");
  state_.assign(np_, 0);
  lo_.assign(np_, -std::numeric_limits<float>::infinity());
  hi_.assign(np_, std::numeric_limits<float>::infinity());
  ck(cudaSetDevice(device_), "cudaSetDevice");
  const unsigned nh = nw_ - nw_ / 2;
  theta_ = dal<float>(static_cast<size_t>(nw_) * np_);
  logl_ = dal<double>(nw_);
  prop_ = dal<float>(static_cast<size_t>(nh) * np_);
  z_ = dal<float>(nh);
  lnew_ = dal<double>(nh);
  snew_ = dal<int>(nh);
  nacc_ = dal<unsigned>(nw_);
  pstate_ = dal<int>(np_);
  plo_ = dal<float>(np_);
  phi_ = dal<float>(np_);
  ctr_ = dal<unsigned long long>(3);
  err_ = dal<int>(4);
  spred_ = dal<double>(nh);
  sst_ = dal<int>(nw_);
  scur_ = dal<double>(nw_);
  exprop_ = dal<float>(static_cast<size_t>(nh) * np_);
  exl_ = dal<double>(nh);
  exs_ = dal<int>(nh);
  exidx_ = dal<int>(nh);
  dcount_ = dal<int>(1);
  nfail_ = dal<unsigned long long>(1);
  ck(cudaMemset(nfail_, 0, sizeof(unsigned long long)), "memset");
  ck(cudaMallocHost(&hcount_, sizeof(int)), "cudaMallocHost");
  ck(cudaMemset(ctr_, 0, 3 * sizeof(unsigned long long)), "memset");
  ck(cudaMemset(err_, 0, 4 * sizeof(int)), "memset");
  ck(cudaMemset(nacc_, 0, nw_ * sizeof(unsigned)), "memset");
}

Ensemble::~Ensemble() {
  cudaSetDevice(device_);
  if (graph_) cudaGraphExecDestroy(graph_);
  void* ptrs[] = {theta_, logl_, prop_, z_, lnew_, snew_, nacc_, pstate_, plo_,
                  phi_, ch_theta_, ch_logl_, ctr_, err_, spred_, sst_, scur_,
                  exprop_, exl_, exs_, exidx_, dcount_, nfail_};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (hcount_) cudaFreeHost(hcount_);
}

void Ensemble::set_like(pofd_batch_loglike_fn fn, void* like) {
  if (!fn) throw Error(POFD_E_ARG, "null likelihood");
  fn_ = fn;
  like_ = like;
  params_dirty_ = true;
}

void Ensemble::set_param_state(unsigned i, int state) {
  if (i >= np_) throw Error(POFD_E_ARG, "parameter index out of range");
  state_[i] = state;
  params_dirty_ = true;
}

void Ensemble::set_limits(unsigned i, float lo, float hi) {
  if (i >= np_) throw Error(POFD_E_ARG, "parameter index out of range");
  if (!(lo <= hi)) throw Error(POFD_E_ARG, "lower limit above upper limit");
  lo_[i] = lo;
  hi_[i] = hi;
  params_dirty_ = true;
}

void Ensemble::set_temperature(double t) {
  if (!(t > 0)) throw Error(POFD_E_ARG, "Invalid temperature");
  temp_ = t;
  params_dirty_ = true;
}

void Ensemble::upload_params() {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemcpy(pstate_, state_.data(), np_ * sizeof(int), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(plo_, lo_.data(), np_ * sizeof(float), cudaMemcpyHostToDevice), "upload");
  ck(cudaMemcpy(phi_, hi_.data(), np_ * sizeof(float), cudaMemcpyHostToDevice), "upload");
  drop_graph();
  params_dirty_ = false;
}

void Ensemble::init(const float* walkers, const double* logl) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemcpy(theta_, walkers, static_cast<size_t>(nw_) * np_ * sizeof(float),
                cudaMemcpyHostToDevice), "upload walkers");
  std::vector<double> l(nw_, -std::numeric_limits<double>::infinity());
  if (logl) std::memcpy(l.data(), logl, nw_ * sizeof(double));
  ck(cudaMemcpy(logl_, l.data(), nw_ * sizeof(double), cudaMemcpyHostToDevice), "upload logl");
  ck(cudaMemset(nacc_, 0, nw_ * sizeof(unsigned)), "memset");
  ck(cudaMemset(err_, 0, 4 * sizeof(int)), "memset");
  for (auto& v : stats_) v = 0;
  ck(cudaMemset(nfail_, 0, sizeof(unsigned long long)), "memset");
  init_ = true;
}

void Ensemble::reserve_chain(unsigned nsteps) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (nsteps <= cap_) return;
  float* nt = dal<float>(static_cast<size_t>(nsteps) * nw_ * np_);
  double* nl = dal<double>(static_cast<size_t>(nsteps) * nw_);
  const unsigned n = nrecorded();
  if (n) {
    ck(cudaMemcpy(nt, ch_theta_, static_cast<size_t>(n) * nw_ * np_ * sizeof(float),
                  cudaMemcpyDeviceToDevice), "copy chain");
    ck(cudaMemcpy(nl, ch_logl_, static_cast<size_t>(n) * nw_ * sizeof(double),
                  cudaMemcpyDeviceToDevice), "copy chain");
  }
  if (ch_theta_) cudaFree(ch_theta_);
  if (ch_logl_) cudaFree(ch_logl_);
  ch_theta_ = nt;
  ch_logl_ = nl;
  cap_ = nsteps;
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
}

void Ensemble::clear_chain() {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemsetAsync(ctr_ + 1, 0, sizeof(unsigned long long), stream_), "memset");
  ck(cudaStreamSynchronize(stream_), "synchronize");
}

unsigned long long Ensemble::step_counter() const {
  unsigned long long c = 0;
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemcpyAsync(&c, ctr_, sizeof(c), cudaMemcpyDeviceToHost, stream_), "D2H");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  return c;
}

void Ensemble::set_step_counter(unsigned long long step) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemcpyAsync(ctr_, &step, sizeof(step), cudaMemcpyHostToDevice, stream_), "H2D");
  ck(cudaStreamSynchronize(stream_), "synchronize");
}

void Ensemble::set_naccept(const unsigned* in) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemcpyAsync(nacc_, in, nw_ * sizeof(unsigned), cudaMemcpyHostToDevice, stream_), "H2D");
  ck(cudaStreamSynchronize(stream_), "synchronize");
}

unsigned Ensemble::nrecorded() const {
  unsigned long long c[3];
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaMemcpyAsync(c, ctr_, sizeof(c), cudaMemcpyDeviceToHost, stream_), "D2H");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  return static_cast<unsigned>(c[1]);
}

void Ensemble::launch_step(cudaStream_t st) {
  const unsigned nh0 = nw_ / 2, nh1 = nw_ - nh0;
  unsigned nfixed = 0;
  for (int s : state_)
    if (s & POFD_PARAM_FIXED) ++nfixed;
  // (nparams - nfixed - 1) with nparams counting bonus parameters, as the
  // reference does (affineEnsemble.cc:1398)
  const double zexp = static_cast<double>(np_) - static_cast<double>(nfixed) - 1.0;
  const double invt = 1.0 / temp_;
  for (int half = 0; half < 2; ++half) {
    const unsigned nh = half ? nh1 : nh0;
    const unsigned g = (nh + ENT - 1) / ENT;
    k_propose<<<g, ENT, 0, st>>>(half, nw_, np_, scalefac_, reject_outside_ ? 1 : 0, seed_,
                                 pstate_, plo_, phi_, theta_, prop_, z_, ctr_, err_);
    ck(cudaGetLastError(), "k_propose");
    const int rc = fn_(like_, nh, prop_, np_, lnew_, snew_, st);
    if (rc < 0) throw Error(rc, "batched likelihood enqueue failed");
    if (bfn_ && bfn_(blike_, nh, prop_, np_, st) < 0)
      throw Error(POFD_E_ARG, "bonus parameter fill failed");
    if (collect_) collect_->add_pairs(nh, prop_, np_, lnew_, snew_, st);
    k_accept<<<g, ENT, 0, st>>>(half, nw_, np_, zexp, invt, seed_, reject_fail_ ? 1 : 0,
                                nfail_, prop_, z_, lnew_, snew_,
                                theta_, logl_, nacc_, ctr_, err_, ch_theta_, ch_logl_, cap_);
    ck(cudaGetLastError(), "k_accept");
  }
  k_advance<<<1, 32, 0, st>>>(ctr_, cap_);
  ck(cudaGetLastError(), "k_advance");
}

void Ensemble::check_error() {
  ck(cudaStreamSynchronize(stream_), "synchronize");
  int e[4];
  ck(cudaMemcpy(e, err_, sizeof(e), cudaMemcpyDeviceToHost), "D2H err");
  if (e[0] == 0) return;
  ck(cudaMemset(err_, 0, sizeof(e)), "memset");
  std::ostringstream s;
  if (e[0] == 1) {
    s << "Unable to generate new step after " << kMaxIters << " tries (walker " << e[1] << ")";
    throw Error(POFD_E_ARG, s.str());
  }
  if (e[0] == 2) {
    s << "Problem encountered in likelihood (walker " << e[1] << ", status " << e[2] << ")";
    throw Error(e[2] < 0 ? e[2] : POFD_E_ARG, s.str());
  }
  s << "Invalid likelihood (walker " << e[1] << ")";
  throw Error(POFD_E_ARG, s.str());
}

void Ensemble::do_steps(unsigned nsteps, bool record) {
  NvtxRange nvtx_range("pofd ensemble do_steps");
  if (!init_) throw Error(POFD_E_ARG, "Chains not initialised");
  if (!fn_) throw Error(POFD_E_ARG, "No likelihood set");
  if (nsteps == 0) return;
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (params_dirty_) upload_params();
  if (record) {
    const unsigned have = nrecorded();
    if (have + nsteps > cap_) reserve_chain(have + nsteps);
  }
  const unsigned long long flag = record ? 1ull : 0ull;
  ck(cudaMemcpyAsync(ctr_ + 2, &flag, sizeof(flag), cudaMemcpyHostToDevice, stream_), "flag");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  unsigned done = 0;
  if (!warmed_ || !graph_) {
    // one eager step: sizes every buffer and plan of the likelihood
    launch_step(stream_);
    ck(cudaStreamSynchronize(stream_), "synchronize");
    check_error();
    warmed_ = true;
    ++done;
    if (done < nsteps) {
      cudaGraph_t g = nullptr;
      ck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
      bool threw = false;
      try {
        launch_step(stream_);
      } catch (...) {
        threw = true;
      }
      const cudaError_t ec = cudaStreamEndCapture(stream_, &g);
      if (!threw && ec == cudaSuccess && g &&
          cudaGraphInstantiate(&graph_, g, 0) != cudaSuccess)
        graph_ = nullptr;
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
    }
  }
  for (; done < nsteps; ++done) {
    if (graph_) ck(cudaGraphLaunch(graph_, stream_), "graph launch");
    else launch_step(stream_);
    if ((done & 255u) == 255u) {
      ck(cudaStreamSynchronize(stream_), "synchronize");
      check_error();
    }
  }
  ck(cudaStreamSynchronize(stream_), "synchronize");
  check_error();
  const unsigned long long ev = static_cast<unsigned long long>(nsteps) * nw_;
  stats_[0] += ev;  // every proposal is evaluated exactly
  stats_[1] += ev;
  stats_[2] += ev;
}

void Ensemble::drop_graph() {
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
}

void Ensemble::set_error_policy(bool reject_failures) {
  reject_fail_ = reject_failures;
  drop_graph();
}

void Ensemble::set_limit_policy(bool reject_outside) {
  reject_outside_ = reject_outside;
  drop_graph();
}

unsigned long long Ensemble::failures() const {
  unsigned long long v = 0;
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  ck(cudaMemcpy(&v, nfail_, sizeof(v), cudaMemcpyDeviceToHost), "D2H");
  return v;
}

void Ensemble::set_stage1(pofd_batch_loglike_fn fn, void* sur) {
  sfn_ = fn;
  sur_ = sur;
}

// A wider stretch than the plain steps' pays under delayed acceptance: a
// rejected proposal then costs one surrogate evaluation instead of an exact
// one, so larger moves with a lower pass rate give more effective samples
// per exact evaluation.  Any a > 1 leaves the target exact (the stretch
// move's z^(d-1) factor is in the first-stage ratio).
void Ensemble::set_da_scale(double a) {
  if (!(a > 1.0) && a != 0.0) throw Error(POFD_E_ARG, "stretch parameter must be > 1 (or 0)");
  da_scale_ = a;
}

// Survivor batches are rounded up so that the likelihood sees a bounded
// number of batch sizes (each has its own FFT plans and graphs; the plans
// share one work area): multiples of 2 up to 32, of 4 up to 64, of 8 up to
// 256, then of 32.
unsigned Ensemble::bucket(unsigned n) {
  if (n <= 32) return (n + 1) / 2 * 2;
  if (n <= 64) return (n + 3) / 4 * 4;
  if (n <= 256) return (n + 7) / 8 * 8;
  return (n + 31) / 32 * 32;
}

void Ensemble::da_half(int half, double zexp, double invt) {
  const unsigned nh0 = nw_ / 2, nh = half ? nw_ - nh0 : nh0;
  const unsigned g = (nh + ENT - 1) / ENT;
  const double a = (da_scale_ > 1.0) ? da_scale_ : scalefac_;
  k_propose<<<g, ENT, 0, stream_>>>(half, nw_, np_, a, reject_outside_ ? 1 : 0, seed_, pstate_,
                                    plo_, phi_, theta_, prop_, z_, ctr_, err_);
  ck(cudaGetLastError(), "k_propose");
  int rc = sfn_(sur_, nh, prop_, np_, spred_, sst_, stream_);
  if (rc < 0) throw Error(rc, "first-stage evaluation failed");
  const unsigned tb = std::min(1024u, (nh + 31) / 32 * 32);
  k_stage1<<<1, tb, 0, stream_>>>(half, nw_, np_, zexp, invt, seed_, prop_, z_, spred_, sst_,
                                  scur_, ctr_, exprop_, exidx_, dcount_);
  ck(cudaGetLastError(), "k_stage1");
  ck(cudaMemcpyAsync(hcount_, dcount_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "D2H count");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  const unsigned count = static_cast<unsigned>(*hcount_);
  stats_[0] += nh;
  stats_[1] += count;
  if (count == 0) return;
  const unsigned b = std::min(bucket(count), nh);
  if (b > count) k_pad<<<b - count, 32, 0, stream_>>>(static_cast<int>(count), static_cast<int>(b), np_, exprop_);
  rc = fn_(like_, b, exprop_, np_, exl_, exs_, stream_);
  if (rc < 0) throw Error(rc, "batched likelihood enqueue failed");
  if (bfn_ && bfn_(blike_, b, exprop_, np_, stream_) < 0)
    throw Error(POFD_E_ARG, "bonus parameter fill failed");
  stats_[2] += b;
  if (collect_) collect_->add_pairs(count, exprop_, np_, exl_, exs_, stream_);
  k_stage2<<<(count + ENT - 1) / ENT, ENT, 0, stream_>>>(
      half, nw_, np_, invt, seed_, reject_fail_ ? 1 : 0, nfail_, static_cast<int>(count), exidx_,
      exprop_, exl_, exs_, spred_,
      theta_, logl_, scur_, nacc_, ctr_, err_);
  ck(cudaGetLastError(), "k_stage2");
}

// Set-up for delayed acceptance: one exact evaluation of every batch size
// the survivor buckets can take, on the buffers the steps use, so that the
// likelihood's transform plans and captured graphs exist before sampling
// (the reference likewise plans its FFTs at set-up).
void Ensemble::prepare_da() {
  if (!init_) throw Error(POFD_E_ARG, "Chains not initialised");
  if (!fn_) throw Error(POFD_E_ARG, "No likelihood set");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  const unsigned nmax = nw_ - nw_ / 2;
  unsigned last = 0;
  for (unsigned c = 1; c <= nmax; ++c) {
    const unsigned b = std::min(bucket(c), nmax);
    if (b == last) continue;
    last = b;
    ck(cudaMemcpyAsync(exprop_, theta_, static_cast<size_t>(b) * np_ * sizeof(float),
                       cudaMemcpyDeviceToDevice, stream_), "copy walkers");
    const int rc = fn_(like_, b, exprop_, np_, exl_, exs_, stream_);
    if (rc < 0) throw Error(rc, "batched likelihood enqueue failed");
    ck(cudaStreamSynchronize(stream_), "synchronize");
  }
  if (nw_ / 2 != nmax) {
    // the first half's size, if it differs
    const unsigned b = std::min(bucket(nw_ / 2), nmax);
    ck(cudaMemcpyAsync(exprop_, theta_, static_cast<size_t>(b) * np_ * sizeof(float),
                       cudaMemcpyDeviceToDevice, stream_), "copy walkers");
    const int rc = fn_(like_, b, exprop_, np_, exl_, exs_, stream_);
    if (rc < 0) throw Error(rc, "batched likelihood enqueue failed");
    ck(cudaStreamSynchronize(stream_), "synchronize");
  }
}

void Ensemble::do_steps_da(unsigned nsteps, bool record) {
  NvtxRange nvtx_range("pofd ensemble do_steps_da");
  if (!init_) throw Error(POFD_E_ARG, "Chains not initialised");
  if (!fn_) throw Error(POFD_E_ARG, "No likelihood set");
  if (!sfn_) throw Error(POFD_E_ARG, "No first-stage evaluator set");
  if (nw_ - nw_ / 2 > 1024) throw Error(POFD_E_ARG, "delayed acceptance supports at most 2048 walkers");
  if (nsteps == 0) return;
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (params_dirty_) upload_params();
  if (record) {
    const unsigned have = nrecorded();
    if (have + nsteps > cap_) reserve_chain(have + nsteps);
  }
  const unsigned long long flag = record ? 1ull : 0ull;
  ck(cudaMemcpyAsync(ctr_ + 2, &flag, sizeof(flag), cudaMemcpyHostToDevice, stream_), "flag");
  // first-stage values of the current walkers (the evaluator may have been
  // retrained since the last call)
  int rc = sfn_(sur_, nw_, theta_, np_, scur_, sst_, stream_);
  if (rc < 0) throw Error(rc, "first-stage evaluation failed");
  unsigned nfixed = 0;
  for (int st : state_)
    if (st & POFD_PARAM_FIXED) ++nfixed;
  const double zexp = static_cast<double>(np_) - static_cast<double>(nfixed) - 1.0;
  const double invt = 1.0 / temp_;
  for (unsigned k = 0; k < nsteps; ++k) {
    da_half(0, zexp, invt);
    da_half(1, zexp, invt);
    k_record<<<(nw_ + ENT - 1) / ENT, ENT, 0, stream_>>>(nw_, np_, theta_, logl_, ctr_, ch_theta_,
                                                         ch_logl_, cap_);
    k_advance<<<1, 32, 0, stream_>>>(ctr_, cap_);
    ck(cudaGetLastError(), "k_record");
    if ((k & 63u) == 63u) check_error();
  }
  ck(cudaStreamSynchronize(stream_), "synchronize");
  check_error();
}

void Ensemble::da_stats(unsigned long long* out4) const {
  std::vector<unsigned> na(nw_);
  naccept(na.data());
  out4[0] = stats_[0];
  out4[1] = stats_[1];
  out4[2] = stats_[2];
  unsigned long long tot = 0;
  for (unsigned v : na) tot += v;
  out4[3] = tot;
}

void Ensemble::chain(float* theta, double* logl) const {
  const unsigned n = nrecorded();
  if (!n) return;
  if (theta)
    ck(cudaMemcpy(theta, ch_theta_, static_cast<size_t>(n) * nw_ * np_ * sizeof(float),
                  cudaMemcpyDeviceToHost), "D2H chain");
  if (logl)
    ck(cudaMemcpy(logl, ch_logl_, static_cast<size_t>(n) * nw_ * sizeof(double),
                  cudaMemcpyDeviceToHost), "D2H chain");
}

void Ensemble::last(float* theta, double* logl) const {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  if (theta)
    ck(cudaMemcpy(theta, theta_, static_cast<size_t>(nw_) * np_ * sizeof(float),
                  cudaMemcpyDeviceToHost), "D2H walkers");
  if (logl) ck(cudaMemcpy(logl, logl_, nw_ * sizeof(double), cudaMemcpyDeviceToHost), "D2H logl");
}

void Ensemble::naccept(unsigned* out) const {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaStreamSynchronize(stream_), "synchronize");
  ck(cudaMemcpy(out, nacc_, nw_ * sizeof(unsigned), cudaMemcpyDeviceToHost), "D2H naccept");
}

// Integrated autocorrelation time of one series by Goodman's acor method
// (affineChainSet::acor, affineChainSet.cc:884-951; Goodman's published
// acor: autocovariances to lag 10, tau = (C0 + 2 sum C_s) / C0, and while
// tau is long against that window the series is summed in adjacent pairs
// and the estimate repeated on the half-length series, the result scaled
// back up level by level).  Written as a descent through the levels
// followed by the scale-back, with the operation order of the recursive
// form so that tau is bitwise the same: the series is float (products of
// two elements rounded to float, then accumulated in double), the mean is
// a double sum in index order, and a level too short for the lag window
// leaves the previous level's sigma in place.  Returns 1 when the series
// is too short for the window at the top level.
int acor_series(double& mean, double& sigma, double& tau, std::vector<float>& X,
                unsigned L) {
  constexpr unsigned kWin = 5;              // window multiple of tau
  constexpr unsigned kLag = 2 * kWin;       // largest lag (tau up to 2)
  constexpr unsigned kMinLen = 5 * kLag;    // shortest series analysed
  struct Scale {
    double c0;
    unsigned len;
  };
  std::vector<Scale> descent;
  unsigned len = L;
  for (unsigned level = 0;; ++level) {
    double m = X[0];
    for (unsigned i = 1; i < len; ++i) m += X[i];
    m *= 1.0 / static_cast<double>(len);
    if (level == 0) mean = m;
    for (unsigned i = 0; i < len; ++i) X[i] -= m;
    if (len < kMinLen) {
      if (level == 0) return 1;
      break;  // the level above keeps its sigma
    }
    double cov[kLag + 1] = {};
    const unsigned span = len - kLag;
    for (unsigned i = 0; i < span; ++i)
      for (unsigned lag = 0; lag <= kLag; ++lag) cov[lag] += X[i] * X[i + lag];
    const double ispan = 1.0 / static_cast<double>(span);
    for (unsigned lag = 0; lag <= kLag; ++lag) cov[lag] *= ispan;
    double d = cov[0];
    for (unsigned lag = 1; lag <= kLag; ++lag) d += 2 * cov[lag];
    sigma = std::sqrt(d * (1.0 / static_cast<double>(len)));
    tau = d / cov[0];
    if (tau * kWin < kLag) break;
    descent.push_back({cov[0], len});
    const unsigned half = len / 2;
    for (unsigned i = 0; i < half; ++i) X[i] = X[2 * i] + X[2 * i + 1];
    len = half;
  }
  for (auto it = descent.rbegin(); it != descent.rend(); ++it) {
    const double d = 0.25 * sigma * sigma * static_cast<double>(it->len);
    tau = d / it->c0;
    sigma = std::sqrt(d * (1.0 / static_cast<double>(it->len)));
  }
  return 0;
}

// affineChainSet::getAcorVector / getAverageParamVector
// (affineChainSet.cc:824-867, 1010-1030).
int Ensemble::acor(double* tau) const {
  constexpr unsigned minlen = 5 * 10;
  const unsigned n = nrecorded();
  std::vector<float> th(static_cast<size_t>(n) * nw_ * np_);
  chain(th.data(), nullptr);
  int succ = 1;
  const double norm = 1.0 / static_cast<double>(nw_);
  for (unsigned p = 0; p < np_; ++p) {
    tau[p] = nan();
    if (state_[p] & POFD_PARAM_ACIGNORE) continue;
    std::vector<float> pv(n);
    for (unsigned s = 0; s < n; ++s) {
      const float* row = th.data() + static_cast<size_t>(s) * nw_ * np_;
      double cum = row[p];
      for (unsigned k = 1; k < nw_; ++k) cum += row[static_cast<size_t>(k) * np_ + p];
      pv[s] = static_cast<float>(norm * cum);
    }
    if (n < minlen) {
      succ = 0;
      continue;
    }
    double mn, sg, t;
    acor_series(mn, sg, t, pv, n);
    tau[p] = t;
  }
  return succ;
}

// ------------------------------------------------------------ LikeSum
namespace {
__global__ void k_lsum(unsigned nprop, unsigned k, unsigned cap, const double* __restrict__ l,
                       const int* __restrict__ s, double* __restrict__ logl,
                       int* __restrict__ status) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nprop) return;
  double acc = 0.0;
  int st = POFD_OK;
  for (unsigned m = 0; m < k; ++m) {
    const int sm = s[static_cast<size_t>(m) * cap + t];
    if (st == POFD_OK && sm != POFD_OK) st = sm;
    acc += l[static_cast<size_t>(m) * cap + t];
  }
  logl[t] = acc;
  status[t] = st;
}
}  // namespace

LikeSum::LikeSum(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  if (device < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ck(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "event");
}

LikeSum::~LikeSum() {
  cudaSetDevice(device_);
  for (auto e : done_) cudaEventDestroy(e);
  for (auto st : streams_) cudaStreamDestroy(st);
  if (fork_) cudaEventDestroy(fork_);
  if (l_) cudaFree(l_);
  if (s_) cudaFree(s_);
}

void LikeSum::add(pofd_batch_loglike_fn fn, void* like) {
  if (!fn) throw Error(POFD_E_ARG, "null likelihood");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  cudaStream_t st;
  ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  cudaEvent_t ev;
  ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
  fn_.push_back(fn);
  like_.push_back(like);
  streams_.push_back(st);
  done_.push_back(ev);
  if (l_) cudaFree(l_);
  if (s_) cudaFree(s_);
  l_ = nullptr;
  s_ = nullptr;
  cap_ = 0;
}

void LikeSum::ensure(unsigned nprop) {
  if (nprop <= cap_) return;
  if (l_) cudaFree(l_);
  if (s_) cudaFree(s_);
  const size_t k = fn_.size();
  l_ = dal<double>(k * nprop);
  s_ = dal<int>(k * nprop);
  cap_ = nprop;
}

void LikeSum::enqueue(unsigned nprop, const float* theta, unsigned npar, double* logl,
                      int* status, cudaStream_t st) {
  if (fn_.empty()) throw Error(POFD_E_ARG, "empty likelihood sum");
  if (nprop == 0) return;
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (!st) st = stream_;
  if (nprop > cap_) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    ck(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing");
    if (cs != cudaStreamCaptureStatusNone)
      throw Error(POFD_E_ARG, "likelihood sum must run once at this batch size before capture");
    ck(cudaStreamSynchronize(st), "synchronize");
    ensure(nprop);
  }
  ck(cudaEventRecord(fork_, st), "event record");
  for (size_t m = 0; m < fn_.size(); ++m) {
    ck(cudaStreamWaitEvent(streams_[m], fork_, 0), "stream wait");
    const int rc = fn_[m](like_[m], nprop, theta, npar, l_ + m * cap_, s_ + m * cap_, streams_[m]);
    if (rc < 0) throw Error(rc, "member likelihood failed");
    ck(cudaEventRecord(done_[m], streams_[m]), "event record");
    ck(cudaStreamWaitEvent(st, done_[m], 0), "stream wait");
  }
  k_lsum<<<(nprop + 127) / 128, 128, 0, st>>>(nprop, static_cast<unsigned>(fn_.size()), cap_, l_,
                                             s_, logl, status);
  ck(cudaGetLastError(), "k_lsum");
}

}  // namespace pofd
