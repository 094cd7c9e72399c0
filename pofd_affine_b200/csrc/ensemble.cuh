// ensemble.cuh -- single-process, batched affine-invariant stretch-move
// ensemble (Goodman & Weare 2010) over a batched likelihood.
//
// Restates affineEnsemble's sampling step (affineEnsemble.cc:116-126
// generateZ, 1144-1228 generateNewStep, 1233-1284 doMasterStep, 1398-1433
// acceptance) with the MPI master/worker farm replaced by one batched
// likelihood launch per half-ensemble: the first half of the walkers is
// updated from partners drawn in the second half, then the second half from
// the (updated) first half.  One full step -- two proposal kernels, two
// batched likelihood evaluations, two acceptance kernels and the chain
// record -- is captured into one CUDA graph and replayed.
//
// Random numbers come from a counter-based Philox4x32-10 generator keyed by
// the seed and indexed by (step, walker, draw), so a run is reproducible and
// independent of the launch shape.
//
// Acor (affineChainSet.cc:824-951) runs on the host over the walker-averaged
// parameter series.
#ifndef POFD_ENSEMBLE_CUH
#define POFD_ENSEMBLE_CUH

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/pofd_b200.h"

namespace pofd {

class Surrogate;

class Ensemble {
 public:
  static constexpr unsigned kMaxParams = 64;
  Ensemble(int device, cudaStream_t stream, unsigned nwalkers, unsigned npar,
           double scalefac, uint64_t seed);
  ~Ensemble();

  void set_like(pofd_batch_loglike_fn fn, void* like);
  void set_param_state(unsigned i, int state);
  void set_limits(unsigned i, float lo, float hi);
  void set_temperature(double t);
  void init(const float* walkers, const double* logl);
  void reserve_chain(unsigned nsteps);
  void clear_chain();
  // Runs nsteps full steps; records them into the chain if record.
  void do_steps(unsigned nsteps, bool record);
  // Delayed-acceptance steps with the first-stage evaluator set below.
  void set_stage1(pofd_batch_loglike_fn fn, void* sur);
  // stretch parameter of the delayed-acceptance steps (default: the plain
  // steps' scalefac)
  void set_da_scale(double a);
  void set_bonus(pofd_batch_bonus_fn fn, void* like) {
    bfn_ = fn;
    blike_ = like;
    drop_graph();
  }
  unsigned npar() const { return np_; }
  void collect_pairs(Surrogate* s) { collect_ = s; drop_graph(); }
  void do_steps_da(unsigned nsteps, bool record);
  void prepare_da();
  void da_stats(unsigned long long* out4) const;
  // false (default): a failed likelihood evaluation stops the run, as in the
  // reference; true: it rejects the step and is counted.
  void set_error_policy(bool reject_failures);
  // false (default): a step outside the parameter limits redraws z, up to
  // 40 times, as in the reference; true: it is rejected (exact for the
  // posterior truncated to the limits).
  void set_limit_policy(bool reject_outside);
  unsigned long long failures() const;
  unsigned nrecorded() const;
  void chain(float* theta, double* logl) const;
  void last(float* theta, double* logl) const;
  void naccept(unsigned* out) const;
  // checkpoint / resume: the generator's step counter (draws are keyed by
  // (seed; step, walker, draw)), the seed, and the accepted-step counts
  unsigned long long step_counter() const;
  void set_step_counter(unsigned long long step);
  void set_naccept(const unsigned* in);
  uint64_t seed() const { return seed_; }
  // Acor of every parameter over the recorded chain (NaN where ignored or
  // the chain is too short); returns 1 if every non-ignored parameter
  // succeeded.
  int acor(double* tau) const;
  unsigned nwalkers() const { return nw_; }
  unsigned nparams() const { return np_; }
  int kernels_per_step() const { return 5; }

 private:
  void check_error();
  void launch_step(cudaStream_t st);
  void upload_params();
  void drop_graph();
  void da_half(int half, double zexp, double invt);
  static unsigned bucket(unsigned n);

  int device_;
  cudaStream_t stream_;
  unsigned nw_, np_;
  double scalefac_, temp_ = 1.0;
  double da_scale_ = 0.0;  // 0: use scalefac_
  uint64_t seed_;
  pofd_batch_loglike_fn fn_ = nullptr;
  void* like_ = nullptr;
  pofd_batch_bonus_fn bfn_ = nullptr;
  void* blike_ = nullptr;
  std::vector<int> state_;
  std::vector<float> lo_, hi_;
  bool params_dirty_ = true, init_ = false;
  unsigned cap_ = 0;
  // device
  float* theta_ = nullptr;    // [nw][np] current walkers
  double* logl_ = nullptr;    // [nw]
  float* prop_ = nullptr;     // [nw - nw/2][np] proposals of one half
  float* z_ = nullptr;        // [nw - nw/2]
  double* lnew_ = nullptr;    // [nw - nw/2]
  int* snew_ = nullptr;       // [nw - nw/2]
  unsigned* nacc_ = nullptr;  // [nw]
  int* pstate_ = nullptr;     // [np]
  float* plo_ = nullptr;      // [np]
  float* phi_ = nullptr;      // [np]
  float* ch_theta_ = nullptr; // [cap][nw][np]
  double* ch_logl_ = nullptr; // [cap][nw]
  unsigned long long* ctr_ = nullptr;  // [0] step counter, [1] records, [2] record flag
  int* err_ = nullptr;        // [0] code, [1] walker
  cudaGraphExec_t graph_ = nullptr;
  bool warmed_ = false;
  // delayed acceptance
  pofd_batch_loglike_fn sfn_ = nullptr;
  void* sur_ = nullptr;
  Surrogate* collect_ = nullptr;
  double* spred_ = nullptr;   // [nh] first-stage values of the proposals
  int* sst_ = nullptr;        // [nw] first-stage status
  double* scur_ = nullptr;    // [nw] first-stage values of the walkers
  float* exprop_ = nullptr;   // [nh][np] stage-one survivors (padded)
  double* exl_ = nullptr;     // [nh]
  int* exs_ = nullptr;        // [nh]
  int* exidx_ = nullptr;      // [nh]
  int* dcount_ = nullptr;     // [1]
  int* hcount_ = nullptr;     // pinned
  unsigned long long stats_[4] = {0, 0, 0, 0};
  bool reject_fail_ = false;
  bool reject_outside_ = false;
  unsigned long long* nfail_ = nullptr;
};

// Sum of several batched likelihoods on the same proposals (fields of
// different FFT sizes fitted jointly): the members run concurrently on
// forked streams and join into one sum, so a captured step holds all of
// them in one graph.
class LikeSum {
 public:
  LikeSum(int device, cudaStream_t stream);
  ~LikeSum();
  void add(pofd_batch_loglike_fn fn, void* like);
  void enqueue(unsigned nprop, const float* theta, unsigned npar, double* logl, int* status,
               cudaStream_t st);
  size_t size() const { return fn_.size(); }

 private:
  void ensure(unsigned nprop);
  int device_;
  cudaStream_t stream_;
  std::vector<pofd_batch_loglike_fn> fn_;
  std::vector<void*> like_;
  std::vector<cudaStream_t> streams_;
  std::vector<cudaEvent_t> done_;
  cudaEvent_t fork_ = nullptr;
  unsigned cap_ = 0;
  double* l_ = nullptr;     // [members][cap]
  int* s_ = nullptr;        // [members][cap]
};

// Goodman's acor on a series (destroyed); returns 1 when the series is
// shorter than minfac * maxlag (no estimate), else 0.
int acor_series(double& mean, double& sigma, double& tau, std::vector<float>& x,
                unsigned L);

}  // namespace pofd
#endif
