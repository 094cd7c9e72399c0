// surrogate.cuh -- online-trained MLP surrogate of the log-likelihood on
// BF16 tensor cores (tcgen05), the first stage of a delayed-acceptance
// stretch move.  No counterpart in the reference.
#ifndef POFD_SURROGATE_CUH
#define POFD_SURROGATE_CUH

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace pofd {

class Surrogate {
 public:
  static constexpr int kInPad = 16;      // inputs padded to one MMA K step
  static constexpr int kNumTensors = 8;  // W1 b1 W2 b2 W3 b3 w4 b4
  Surrogate(int device, cudaStream_t stream, unsigned npar, const int* free_idx,
            unsigned nin, unsigned hidden, unsigned capacity, uint64_t seed);
  ~Surrogate();

  // Training pairs (device theta [n][npar], logl [n], optional status: only
  // POFD_OK pairs with finite logL are kept), appended to a ring buffer.
  void add_pairs(unsigned n, const float* theta, unsigned npar, const double* logl,
                 const int* status, cudaStream_t st);
  unsigned npairs() const;
  // The first n pairs held (buffer order) into host theta [n][npar], logl [n].
  void pairs_host(unsigned n, float* theta, double* logl) const;
  // iters Adam steps on random minibatches of the pairs held.
  void train(unsigned iters, unsigned batch, float lr, float* last_loss);
  // Predicted logL of n device rows (batched-likelihood signature).
  void predict(unsigned n, const float* theta, unsigned npar, double* out, int* status,
               cudaStream_t st);
  // Loss gradients over the first n pairs (no update): grads_dev[8] device
  // buffers of the tensor sizes.
  void gradients(unsigned n, float** grads_dev, float* loss);
  void get_params_host(std::vector<std::vector<float>>& host) const;
  void set_params_host(const std::vector<std::vector<float>>& host);
  size_t tensor_size(int t) const { return size_[t]; }
  // mu[16], W[16][16], ymax, ys, clip, whitened (276 values)
  void scaling(double* out) const;
  void refresh_scaling();
  unsigned hidden() const { return H_; }
  unsigned nin() const { return nin_; }
  unsigned npar() const { return npar_; }

 private:
  void init_weights();
  void refresh_bf16(const std::vector<std::vector<float>>& host);
  void ensure_work(int Mp);
  void forward(int M, const float* theta, int npar, const int* rows, bool train,
               cudaStream_t st);
  float iteration(int Mb, const int* rows, float lr, float** grads, cudaStream_t st);
  void check_err();

  int device_;
  cudaStream_t stream_;
  unsigned npar_, nin_, H_, cap_;
  uint64_t seed_;
  unsigned step_ = 0;
  bool scaled_ = false;
  double ymax_ = 0.0, ys_ = 1.0, clip_ = 1e300;
  int* idx_ = nullptr;
  float* mu_ = nullptr;
  float* wm_ = nullptr;    // input whitening W [16][16]
  bool whitened_ = false;
  float* p_[kNumTensors] = {};
  float* m_[kNumTensors] = {};
  float* v_[kNumTensors] = {};
  size_t size_[kNumTensors] = {};
  __nv_bfloat16 *w1b_ = nullptr, *w2b_ = nullptr, *w3b_ = nullptr;
  __nv_bfloat16 *w2t_ = nullptr, *w3t_ = nullptr;
  float* ptheta_ = nullptr;
  double* plogl_ = nullptr;
  unsigned* counters_ = nullptr;
  int* err_ = nullptr;
  struct Work {
    int Mp = 0;
    __nv_bfloat16 *x = nullptr, *xt = nullptr;
    __nv_bfloat16* h[3] = {};
    __nv_bfloat16* ht[3] = {};
    float* z[3] = {};
    __nv_bfloat16* dz[3] = {};
    __nv_bfloat16* dzt[3] = {};
    float *y = nullptr, *ypart = nullptr, *t = nullptr, *dy = nullptr, *loss = nullptr;
    int* rows = nullptr;
  } ws_;
};

// C[M][N] (fp32, ldc) = A[M][K] B[N][K]^T with A, B bf16 on the tensor cores.
void bf16_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C,
               int ldc, int* err, cudaStream_t st);

}  // namespace pofd
#endif
