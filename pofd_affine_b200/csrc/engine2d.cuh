// engine2d.cuh -- batched 2D (two-band) P(D) likelihood engine.
//
// One Engine2 evaluates calcLikeDouble::getLogLike (calcLikeDouble.cc:
// 1195-1277) for a batch of proposals: model set-up (knot counts, sigma and
// offset curves), per-row precompute of the log-normal colour terms,
// the direct n x n R grid with the edge integrals, R moments and shifts, a
// batched 2D D2Z, the spectrum (exp/shift, Hermitian projection of the
// self-conjugate columns, one noise product per dataset), a batched 2D Z2D,
// marginal sums, split points, normalisation and means, and the bilinear
// log-likelihood gather.  Captured into a CUDA graph per batch size and
// pointer set.
#ifndef POFD_ENGINE2D_CUH
#define POFD_ENGINE2D_CUH

#include <cuda_runtime.h>
#include <cufft.h>

#include <map>
#include <vector>

#include "fftplan.hh"
#include "setup.hh"

namespace pofd {

struct Sign2Dev {
  int nt;                 // terms (histogram bins or pixels)
  int ishist;             // weight/product order of the reference
  const double* w;        // weights (1 for raw)
  const double* ieta1;    // inverse band-1 beam
  const double* logratio; // log(beam1 / beam2)
  double maxf1;           // maxknot * max band-1 beam
};

struct BSet2Dev {
  Sign2Dev sg[4];
  int hassign[4];
  int T;                  // terms per row slot (max of np+nn over row signs)
  int Ts;                 // row stride of the term buffer (max T over sets)
  double prefac;          // (pixsize/3600)^2 / sqrt(2 pi)
  double dflux1, dflux2;
  int wrap1, wrap2;
  int nrows;              // n (+ nedge edge rows)
  const double* rowflux;  // [nrows] RFlux1 then edge band-1 fluxes
  const double* rowlog;   // log|f1|
  const int* rowsgn;      // 0 (f1 > 0), 2 (f1 < 0), -1 (R row is zero)
  const double* colinv;   // [n + nedge] 1/|f2| (0 where f2 == 0)
  const double* collog;   // log|f2|
  const int* colsgn;      // 0 (f2 > 0), 1 (f2 < 0)
  const double* rflux2;   // RFlux2 [n]
  const double* e1;       // edge band-1 fluxes [nedge]
  double iRxnorm, iRynorm, iR00norm;
  double maxsb1, maxsb2;
  int ds_begin, nds;
};

struct DSet2Dev {
  int bs;
  double sb1, sb2, like_offset, like_norm;
  int binned;
  int nnz;                // non-zero bins (binned) or pixels (unbinned)
  const int* nzi1;
  const int* nzi2;
  const double* nzcnt;
  const double* f1;       // unbinned pixel fluxes
  const double* f2;
  double bc1, bc2, bd1, bd2;
};

struct Model2Dev {
  int K, ns, no;
  const double* logknots;
  const double* sk;
  const double* ok;
  double minknot, maxknot, min_sigma;
};

// Priors and regularisation of calcLikeDouble (calcLikeDouble.h:213-232),
// per band, applied after the beam-set sum in the reference's order
// (calcLikeDouble.cc:1236-1276); logs of the widths taken on the host.
struct Prior2 {
  int has_sigma[2] = {0, 0}, has_cfirb[2] = {0, 0}, has_poisson[2] = {0, 0};
  double sigma_width[2] = {0, 0}, log_sigma_width[2] = {0, 0};
  double cfirb_mean[2] = {0, 0}, cfirb_sigma[2] = {0, 0}, log_cfirb_sigma[2] = {0, 0};
  double poisson_mean[2] = {0, 0}, poisson_sigma[2] = {0, 0}, log_poisson_sigma[2] = {0, 0};
  double alpha = 0;
  bool needs_bonus() const {
    return has_cfirb[0] || has_cfirb[1] || has_poisson[0] || has_poisson[1] || alpha > 0.0;
  }
};

struct PDInfo2 {
  int status, s1, s2, pad;
  double itot, minflux1, minflux2, sg1pos, sg1neg, sg2pos, sg2neg, pad2;
};

// Launch-shape knobs of the 2D sequence chosen by Engine2::autotune (none
// changes what is computed; the FFT mode changes the transform's rounding).
struct Tune2 {
  int fft_mode = 1;     // see set_fft_mode
  int rgrid_rows = 8;   // R-grid rows per block of k_rgrid2 (2, 4, 8)
  int edge_rows = 16;   // band-1 edge rows per group of k_redge2 (4, 8, 16)
};

class Engine2 {
 public:
  static constexpr int KMAX = 64;
  static constexpr int kNumStages = 12;
  Engine2(int device, cudaStream_t stream);
  ~Engine2();

  void configure(unsigned nknots, const double* knotpos, unsigned nsigma,
                 const double* sigmapos, unsigned noffset,
                 const double* offsetpos, unsigned fftsize, unsigned nedge,
                 bool edge_integ, bool bin_data, unsigned nbins);
  int add_beamset(const Beam2& bm, double exp_conf1, double exp_conf2);
  void add_dataset(int bs, const double* d1, const double* d2, size_t nd,
                   bool meansub, double sigma1, double sigma2,
                   double like_norm);
  // pixels in device memory (mean-subtracted in place when meansub)
  void add_dataset_device(int bs, double* d1_dev, double* d2_dev, size_t nd, bool meansub,
                          double sigma1, double sigma2, double like_norm);
  void set_rranges(const float* theta, unsigned npar);
  // P(D) factory use: a dataset without pixels whose noise is set per call,
  // and explicit R ranges (PDFactoryDouble::initPD / getPD).
  void add_virtual_dataset(int bs, double sigma1, double sigma2);
  void set_virtual_sigma(int bs, double sigma1, double sigma2);
  void set_rrange_explicit(int bs, double min1, double max1, double min2, double max2);
  void rrange(int bs, double* r4) const;
  void dataset_info(int bs, int ds, double* info10, uint32_t* bins) const;
  void reserve(unsigned max_batch);
  void enqueue(unsigned nprop, const float* theta_dev, unsigned npar,
               double* logl_dev, int* status_dev, cudaStream_t st);
  void eval_host(unsigned nprop, const float* theta, unsigned npar,
                 double* logl, int* status);
  int pd_host(int bs, int ds, const float* theta, unsigned npar, bool setlog,
              double* pd_out, double* info16);
  void rgrid_host(int bs, const float* theta, unsigned npar, double* out);
  // Active colour terms (c0 != 0) of one proposal's R grid rows, summed over
  // the main rows 1 .. n-1 (out[0]) and the edge rows (out[1]) of every beam
  // set: the R builders' algorithmic work is these times the columns.
  void active_terms(const float* theta, unsigned npar, long long* out2);
  void profile_stages(unsigned nprop, const float* theta, unsigned npar,
                      int reps, double* stage_ms);
  static const char* stage_name(int i);
  // the stage names of the FFT mode in use
  const char* stage_name_now(int i) const;
  int kernels_per_eval() const {
    return (edge_ ? 12 : 10) + (colspec_ ? 1 : 0) + (prior_.needs_bonus() ? 1 : 0) +
           (refsum_ ? 1 : 0);
  }
  // Reference-order normalisation and means (k_pseq2 after the split
  // search): the P(D) integral and the two means summed in one sequential
  // chain in the reference's order instead of the default tree sums.  For
  // parity checks only (a 2n^2-long dependent chain per dataset).
  void set_reference_sums(bool on);
  // Times the whole launch sequence (graph replays, CUDA events) for each
  // candidate of each knob in turn on nprop host rows and keeps the
  // fastest; out5 (optional) = {fft_mode, rgrid_rows, edge_rows, best ms per
  // launch, untuned ms per launch}.
  void autotune(unsigned nprop, const float* theta, unsigned npar, int reps, double* out5);
  Tune2 tuning() const {
    Tune2 t = tune_;
    t.fft_mode = fft_mode_;
    return t;
  }
  void set_tuning(const Tune2& t);
  bool reference_sums() const { return refsum_; }
  // 0: batched 2D cuFFT transforms with k_spectrum2 between them; 1: batched
  // 1D cuFFT row transforms around this library's fused column-transform +
  // spectrum kernel (k_colspec2), where n is a power of two in [512, 4096]
  // (mode 0 otherwise).
  void set_fft_mode(int mode);
  int fft_mode() const { return fft_mode_; }
  // the fused column path is (or, before the first evaluation, will be) used
  bool colspec() const {
    if (static_ok_) return colspec_;
    return fft_mode_ == 1 && (n_ == 512 || n_ == 1024 || n_ == 2048 || n_ == 4096);
  }
  // priors per band (calcLikeDouble::setSigmaPrior1/2, setCFIRBPrior1/2,
  // setPoissonPrior1/2 and unset forms, setRegularizationAlpha,
  // calcLikeDouble.h:310-341)
  void set_sigma_prior(int band, bool on, double width);
  void set_cfirb_prior(int band, bool on, double mean, double sigma);
  void set_poisson_prior(int band, bool on, double mean, double sigma);
  void set_regularization(double alpha);
  // <S1>, <S2>, <S1^2>, <S2^2> per host row -> out[nprop][4]
  void bonus_host(unsigned nprop, const float* theta, unsigned npar, double* out);
  // fillBonusParams (calcLikeDouble.cc:1283-1310) on device rows: the four
  // values at theta_dev[i][nparams() + 2 .. + 5]
  void fill_bonus(unsigned nprop, float* theta_dev, unsigned npar, cudaStream_t st);
  unsigned nparams() const {
    return static_cast<unsigned>(knots_.size() + sigk_.size() + offk_.size());
  }

 private:
  struct HostSet {
    Beam2 bm;
    double ec1 = 0, ec2 = 0;
    std::vector<Data2> data;
    std::vector<double> sb1, sb2, lo, ln;
    double maxsb1 = nan(), maxsb2 = nan();
    double mdf[4] = {nan(), nan(), nan(), nan()};
    double rr[4] = {nan(), nan(), nan(), nan()};
    bool rr_set = false;
  };
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
    bool warmed = false, no_graph = false;
  };
  void refresh_set(HostSet& s);
  void bonus_launch(unsigned nprop, float* theta_dev, unsigned npar, int fill_at,
                    cudaStream_t st);
  void build_static();
  void free_static();
  void free_work();
  void drop_graphs();
  void ensure_plans(unsigned nprop);
  cudaGraphExec_t graph_for(unsigned nprop, const float* theta, unsigned npar,
                            double* logl, int* status);
  void launch_all(unsigned nprop, const float* theta, unsigned npar,
                  double* logl, int* status, cudaStream_t st, cudaEvent_t* ev,
                  bool r_only = false);

  int device_;
  cudaStream_t stream_;
  std::vector<double> knots_, sigk_, offk_;
  unsigned n_ = 0, nedge_ = 256, nbins_ = 1000;
  bool edge_ = true, bin_data_ = true;
  std::vector<HostSet> sets_;
  bool static_ok_ = false;
  std::vector<void*> static_allocs_;
  BSet2Dev* d_bsets_ = nullptr;
  DSet2Dev* d_dsets_ = nullptr;
  Model2Dev model_{};
  std::vector<BSet2Dev> h_bsets_;
  std::vector<DSet2Dev> h_dsets_;
  unsigned B_ = 0, D_ = 0;
  int Tmax_ = 1;
  unsigned gx_ = 0, gy_ = 0;      // R grid blocks (columns, row groups)
  unsigned nrt_ = 0, nct_ = 0;    // P(D) row / column tiles
  unsigned gchunks_ = 1;          // gather chunks per dataset
  std::map<unsigned, Plans> plans_;
  FftWorkArea fftwork_;
  void setup_colspec();
  void drop_plans();
  int fft_mode_ = 1;
  bool colspec_ = false;
  bool refsum_ = false;
  Tune2 tune_;
  double time_sequence(unsigned nprop, const float* theta, unsigned npar, int reps);
  double2* d_cwh_ = nullptr;  // e^{-2 pi i 32 h / n}, h < n / 32
  double2* d_cwl_ = nullptr;  // e^{-2 pi i l / n}, l < 32
  Prior2 prior_;
  const double* d_qu_ = nullptr;
  const double* d_qs_ = nullptr;
  const double* d_qw_ = nullptr;
  const int* d_qk_ = nullptr;
  int nq_ = 0;
  struct Work {
    unsigned P = 0;
    double* cnt = nullptr;      // [P][12*KMAX]
    int* mstatus = nullptr;
    double* sigmult = nullptr;  // [P][2]
    double* rw = nullptr;       // [P][B][nrows][T][3] compacted row terms
    int2* rcnt = nullptr;       // [P][B][nrows] (positive, negative) term counts
    double* rbuf = nullptr;     // [P][B][n][2nc]
    double* rpart = nullptr;    // [P][B][gy][gx][4]
    double* redge = nullptr;    // [P][B][2n+1]: Ry at [n, 2n)
    double* epart = nullptr;    // [P][B][edge row groups][n + nedge]
    double* mom = nullptr;      // [P][B][8]
    double* r0 = nullptr;       // [P][B] R~00 (FFT mode 1)
    double* fpart = nullptr;    // [P][B][n/256][4] edge-cell moment partials
    double* pbuf = nullptr;     // [P][D][n][2nc]
    double* rowpart = nullptr;  // [P][D][n][nct]
    double* colpart = nullptr;  // [P][D][nrt][n]
    PDInfo2* pinfo = nullptr;   // [P][D]
    double* gpart = nullptr;    // [P][D][gchunks]
    double* pdout = nullptr;    // [n*n]
    double* bonus = nullptr;    // [P][8] <S1>, <S2>, <S1^2>, <S2^2>, penalty
    double* bcnt = nullptr;     // [P][12*KMAX] model scratch of fill_bonus
    int* bstatus = nullptr;     // [P]
    double* bsig = nullptr;     // [P][2]
    float* theta_in = nullptr;
    double* logl = nullptr;
    int* status = nullptr;
    float* h_theta = nullptr;
    double* h_logl = nullptr;
    int* h_status = nullptr;
    unsigned h_npar = 0;
  } ws_;
};

}  // namespace pofd
#endif
