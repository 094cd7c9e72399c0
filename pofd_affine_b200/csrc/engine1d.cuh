// engine1d.cuh -- batched 1D P(D) likelihood engine (host class).
//
// One Engine1 evaluates calcLike::getLogLike (calcLike.cc:884-955) for a
// batch of proposals in one stream-ordered sequence of launches: model set-up,
// R at the interpolation nodes, the node spline, the wrapped R grid with its
// moments, a batched D2Z, the spectrum (exp/shift/noise, one output per
// dataset), a batched Z2D, the P(D) reduction/split pass and the finishing
// kernel (split point, normalisation, mean, binned log-likelihood), then the
// per-proposal sum.  The sequence is captured once per batch size into a CUDA
// graph and replayed.
#ifndef POFD_ENGINE1D_CUH
#define POFD_ENGINE1D_CUH

#include <cuda_runtime.h>
#include <cufft.h>

#include <map>
#include <memory>
#include <vector>

#include "fftplan.hh"
#include "setup.hh"

namespace pofd {

// ---- device-side descriptors (plain structs, arrays live in device memory)
struct Side1Dev {
  int nodes;        // 1 if this side's R nodes are computed (beam has it)
  int nterms;       // beam terms summed by R
  const double* w;  // term weights
  const double* ieta;
  const double* x;      // ninterp node fluxes
  const double* ih;     // 1/(x[i+1]-x[i])
  const double* alpha;  // LDL^T diagonal (ninterp-2)
  const double* gamma;  // LDL^T sub-diagonal ratio (ninterp-2)
  const double* lxa;    // log2|x| of the nodes
  const double* lie;    // log2 of the inverse beam terms
  const unsigned char* kidx;  // [nterms][ninterp] knot interval of term j at
                              // node i (255: outside the knot range)
  const int2* jrange;         // [ninterp] first and one past the last term
                              // inside the knot range at node i
  int grid_lo, grid_hi; // inclusive grid index range filled from this side
  double grid_off;      // grid flux = i*dflux + grid_off
};

struct BSet1Dev {
  Side1Dev side[2];
  double prefac;        // (pixsize/3600)^2
  double rr_lo, rr_hi;  // R range of the model over this beam
  int haspos, hasneg;
  double dflux, minflux_R;
  int wrapRidx;
  double maxsb;         // max sigma_base of the set
  int ds_begin, nds;
  const int* gidx;      // node interval of each grid point, -1 if uncovered
  const int2* runs;     // the grid cut into runs of <= 16 points of one
                        // interval and side: x = first index, y = (q + 1) << 8
                        // | len << 2 | kind (0 uncovered, 1 point by point,
                        // 2 running products)
  int nruns;
  const int2* aruns;    // the same cut per block of the forward pass A
  const int* arun_off;  // (own FFT sizes), balanced over the block's 256
                        // threads: thread t of block bx takes aruns[
                        // arun_off[257 bx + t] .. arun_off[257 bx + t + 1])
};

struct DSet1Dev {
  int bs;
  double sigma_base, like_offset, like_norm;
  int binned;
  int nnz;               // nonzero bins (binned) or pixels (unbinned)
  const int* nzidx;      // bin indices of nonzero bins
  const double* nzcnt;   // their counts
  const double* flux;    // unbinned pixel values
  double bincent0, bindelta;
};

struct Model1Dev {
  int K;
  const double* logknots;  // log2 knot positions
  double minknot, maxknot;
};

// Priors and regularisation of calcLike (calcLike.h:184-195), applied after
// the beam-set sum in the reference's order (calcLike.cc:918-952).  The logs
// of the widths are taken on the host.
struct Prior1 {
  int has_sigma = 0, has_cfirb = 0, has_poisson = 0;
  double sigma_width = 0, log_sigma_width = 0;
  double cfirb_mean = 0, cfirb_sigma = 0, log_cfirb_sigma = 0;
  double poisson_mean = 0, poisson_sigma = 0, log_poisson_sigma = 0;
  double alpha = 0;  // regularisation multiplier, 0 = off
  bool needs_bonus() const { return has_cfirb || has_poisson || alpha > 0.0; }
};

// Per-(proposal, dataset) record written by the finishing kernel.
struct PDInfo1 {
  int status;
  int split;
  double itot;     // 1 / trapezoid integral of the unwrapped P(D)
  double minflux;  // flux of the first unwrapped element (-mean)
  double sgpos, sgneg;
  double ll;       // (logL - like_offset) / like_norm
  double pad;
};

struct Workspace1 {
  unsigned P = 0;  // capacity (proposals)
  double* theta = nullptr;   // unused: theta is read from the caller pointer
  double* cnt = nullptr;     // [P][4*KMAX] model spline: y, b, c, d per knot
  int* mstatus = nullptr;    // [P] model status
  double* sigmult = nullptr; // [P]
  double* nodes = nullptr;   // [P][B][2][NI] R at nodes -> log2 R
  double* spl = nullptr;     // [P][B][2][NI][4] spline (y,b,c,d) per interval
  double* rbuf = nullptr;    // [P][B][2*(n/2+1)] R grid / spectrum
  double* rpart = nullptr;   // [P][B][ntile][2]
  double* mom = nullptr;     // [P][B][4] mean, var, shift, doshift
  int* kcut_set = nullptr;   // [P][B] noise cut-off of the forward spectrum
  int* kcut_ds = nullptr;    // [P][D] noise cut-off of each dataset's spectrum
  double* pbuf = nullptr;    // [P][D][2*(n/2+1)] spectrum / P(D)
  double* tmp = nullptr;     // [P][max(B,D)][2*(n/2+1)] own-FFT pass-A rows
  double* ppart = nullptr;   // [P][D][nchunk][4] max, sum, wsum, minval
  int* pmidx = nullptr;      // [P][D][nchunk] argmin index
  PDInfo1* pinfo = nullptr;  // [P][D]
  double* pdout = nullptr;   // [n] one P(D) for the full-array path
  float* theta_in = nullptr; // [P][npar] staging for host calls
  double* logl = nullptr;    // [P]
  int* status = nullptr;     // [P]
  double* bonus = nullptr;   // [P][4] <S>, <S^2>, slope penalty, -
  // pinned host staging
  float* h_theta = nullptr;
  double* h_logl = nullptr;
  int* h_status = nullptr;
  unsigned h_npar = 0;
};

// Launch-shape knobs chosen by Engine1::autotune (none changes what is
// computed; the R-fill tile changes the grouping of the R moment partial sums
// and the FFT choice the rounding of the transform).
struct Tune1 {
  int own_fft = 1;          // own FP64 FFT where the size allows (else cuFFT)
  int rfill_per = 8;        // R grid points per thread of k_rfill1 (4, 8, 16)
  int rnodes_threads = 128; // threads per block of k_rnodes1 (64, 128, 256)
  int spec_blocks = 4;      // blocks per row of k_spectrum1f (2 ... 32)
  int rfill_mode = 3;       // R grid fill: 0 materialised, one exp2 per grid
                            // point; 1 the same inside the forward FFT pass
                            // A (own FFT), the grid never stored; 2
                            // materialised by running products over runs
                            // of <= 16 points in one node interval; 3 the
                            // runs inside the forward pass A (own FFT)
};

class Engine1 {
 public:
  static constexpr int KMAX = 64;
  Engine1(int device, cudaStream_t stream);
  ~Engine1();

  // configuration (host set-up)
  void configure(unsigned nknots, const double* knotpos, unsigned fftsize,
                 unsigned ninterp, bool bin_data, unsigned nbins);
  int add_beamset(const Beam1& bm, double exp_conf);
  void add_dataset(int bs, const double* data, size_t nd, bool meansub,
                   double sigma_base, double like_norm);
  // pixels in device memory (mean-subtracted in place when meansub)
  void add_dataset_device(int bs, double* data_dev, size_t nd, bool meansub,
                          double sigma_base, double like_norm);
  void set_rranges(const float* theta, unsigned npar);
  void set_rrange_explicit(int bs, double minR, double maxR);
  void add_virtual_dataset(int bs, double sigma_base);
  void set_virtual_sigma(int bs, double sigma);
  std::pair<double, double> rrange(int bs) const;
  void dataset_info(int bs, int ds, double* info9, uint32_t* bins) const;

  // device preparation
  void reserve(unsigned max_batch);
  // enqueue a batch (device pointers)
  void enqueue(unsigned nprop, const float* theta_dev, unsigned npar,
               double* logl_dev, int* status_dev, cudaStream_t st);
  // host convenience: H2D theta, graph launch, D2H results, synchronize
  void eval_host(unsigned nprop, const float* theta, unsigned npar,
                 double* logl, int* status);
  // P(D) of one dataset for one proposal
  int pd_host(int bs, int ds, const float* theta, unsigned npar, bool setlog,
              double* pd_out, double* info12);
  void rnodes_host(int bs, int side, const float* theta, unsigned npar,
                   double* x_out, double* r_out);
  void rgrid_host(int bs, const float* theta, unsigned npar, double* out);
  int kernels_per_eval() const {
    return (own_fft_ ? (fused_fill() ? 12 : 13) : 9) + (prior_.needs_bonus() ? 1 : 0);
  }
  // the R grid fill runs inside the forward FFT pass A (own FFT, plain passes)
  bool fused_fill() const {
    return own_fft_ && (tune_.rfill_mode == 1 || tune_.rfill_mode == 3);
  }
  // priors (calcLike::setSigmaPrior / setCFIRBPrior / setPoissonPrior /
  // setRegularizationAlpha and their unset forms, calcLike.h:251-269)
  void set_sigma_prior(bool on, double width);
  void set_cfirb_prior(bool on, double mean, double sigma);
  void set_poisson_prior(bool on, double mean, double sigma);
  void set_regularization(double alpha);
  const Prior1& priors() const { return prior_; }
  // Times the full launch sequence (graph replays, CUDA events) for the
  // candidate values of each knob in turn on nprop host rows and keeps the
  // fastest; out (optional) receives {own_fft, rfill_per, rnodes_threads,
  // spec_blocks, rfill_mode, best ms per launch, untuned ms per
  // launch}.
  void autotune(unsigned nprop, const float* theta, unsigned npar, int reps, double* out7);
  const Tune1& tuning() const { return tune_; }
  // grid points per thread of the materialised R fill
  // blocks per row of the materialised R fill: PER points per thread, or
  // (running products) NT runs per block
  unsigned fill_tiles() const;
  void set_tuning(const Tune1& t);
  // <S>, <S^2> of each proposal's model (calcLike::fillBonusParams,
  // calcLike.cc:958-980): host rows -> out[nprop][2]
  void bonus_host(unsigned nprop, const float* theta, unsigned npar, double* out);
  // the same written into theta_dev[i][nknots + 1], [nknots + 2] (device)
  void fill_bonus(unsigned nprop, float* theta_dev, unsigned npar, cudaStream_t st);
  static constexpr int kNumStages = 10;
  void profile_stages(unsigned nprop, const float* theta, unsigned npar,
                      int reps, double* stage_ms);
  const char* stage_name(int i) const;
  // 0: own FFT where n allows (power of two in [4096, 131072]), else cuFFT;
  // 1: cuFFT always.
  void set_fft_mode(int mode);
  bool own_fft() const { return own_fft_; }
  unsigned fftsize() const { return n_; }
  unsigned nknots() const { return static_cast<unsigned>(knots_.size()); }

 private:
  struct HostSet {
    Beam1 bm;
    double exp_conf = 0;
    std::vector<Data1> data;
    std::vector<double> sb, lo, ln;
    double maxsb = nan(), minDF = nan(), maxDF = nan();
    double minR = nan(), maxR = nan();
    bool rr_set = false;
  };
  void refresh_set(HostSet& s);
  void build_static();
  void free_static();
  void free_work();
  void ensure_plans(unsigned nprop);
  void launch_all(unsigned nprop, const float* theta, unsigned npar,
                  double* logl, int* status, cudaStream_t st, cudaEvent_t* ev);

  int device_;
  cudaStream_t stream_;
  // configuration
  std::vector<double> knots_;
  unsigned n_ = 0, ninterp_ = 2048, nbins_ = 1000;
  bool bin_data_ = true;
  std::vector<HostSet> sets_;
  bool static_ok_ = false;
  // static device data
  std::vector<void*> static_allocs_;
  BSet1Dev* d_bsets_ = nullptr;
  DSet1Dev* d_dsets_ = nullptr;
  Model1Dev model_{};
  std::vector<BSet1Dev> h_bsets_;
  std::vector<DSet1Dev> h_dsets_;
  unsigned B_ = 0, D_ = 0;
  unsigned ntile_ = 0, nchunk_ = 0;
  unsigned runblk_ = 0;  // most run blocks of any beam set's grid
  int maxterms_ = 1;
  // work space
  Workspace1 ws_;
  // cuFFT plans and graphs per batch size
  struct GraphKey {
    const float* theta;
    unsigned npar;
    double* logl;
    int* status;
    bool operator==(const GraphKey& o) const {
      return theta == o.theta && npar == o.npar && logl == o.logl &&
             status == o.status;
    }
  };
  struct Plans {
    cufftHandle fwd = 0, inv = 0;
    std::vector<std::pair<GraphKey, cudaGraphExec_t>> graphs;
    bool warmed = false;
    bool no_graph = false;
    // eval_host's graph: theta upload, the launch sequence and the result
    // download in one launch (for host_npar parameters per row)
    cudaGraphExec_t host_graph = nullptr;
    unsigned host_npar = 0;
  };
  cudaGraphExec_t graph_for(unsigned nprop, const float* theta, unsigned npar,
                            double* logl, int* status);
  cudaGraphExec_t host_graph_for(unsigned nprop, unsigned npar);
  void drop_graphs();
  std::map<unsigned, Plans> plans_;
  FftWorkArea fftwork_;
  int fft_mode_ = -1;  // -1 automatic (own FFT from n = 8192), 0 own, 1 cuFFT
  bool own_fft_ = false;
  int sm_count_ = 148;
  double2* d_wh_ = nullptr;  // e^{-2 pi i 128 j / m}, j < m / 128
  double2* d_wl_ = nullptr;  // e^{-2 pi i i / m}, i < 128
  double2* d_wn_ = nullptr;  // e^{-2 pi i k / n}, k <= m
  double time_sequence(unsigned nprop, const float* theta, unsigned npar, int reps);
  Tune1 tune_;
  // priors and the knot quadrature of the bonus integrals
  Prior1 prior_;
  const double* d_qu_ = nullptr;
  const double* d_qs_ = nullptr;
  const double* d_qw_ = nullptr;
  int qper_ = 0;
};

}  // namespace pofd
#endif
