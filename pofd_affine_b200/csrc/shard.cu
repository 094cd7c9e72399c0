// shard.cu -- a batched likelihood split over the GPUs of one node.
//
// The reference farms proposals out to MPI workers, one at a time
// (affineEnsemble.cc:1233-1521).  Here every rank (one process per GPU)
// runs the same ensemble -- same seed, counter-based draws, so the same
// proposals -- and its likelihood is a ShardLike: rank r evaluates rows
// [P r / W, P (r + 1) / W) of each batch of P proposals with its own
// replica of the likelihood (data, beams and plans on every GPU), then one
// NCCL all-gather on the caller's stream assembles (logL, status) of the
// whole batch on every rank.  The acceptance steps that follow therefore
// see identical inputs everywhere and the chains stay identical, draw for
// draw, to a single-GPU run's.  Each rank sends W x 2 ceil(P / W) doubles
// per batch; the collective is enqueued like any kernel, so a captured
// ensemble step includes it.  NCCL is opened at run time (libnccl.so.2: the
// copy already loaded into the process, e.g. by torch, or the system one).
#include <dlfcn.h>
#include <nccl.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>

#include "../../include/pofd_b200.h"
#include "common.cuh"
#include "setup.hh"

namespace pofd {

namespace {

struct NcclApi {
  void* h = nullptr;
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) comm_init_rank = nullptr;
  decltype(&ncclAllGather) all_gather = nullptr;
  decltype(&ncclCommDestroy) comm_destroy = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
};

const NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
    api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
    api.all_gather = reinterpret_cast<decltype(api.all_gather)>(dlsym(h, "ncclAllGather"));
    api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
    api.error_string = reinterpret_cast<decltype(api.error_string)>(dlsym(h, "ncclGetErrorString"));
    if (api.get_unique_id && api.comm_init_rank && api.all_gather && api.comm_destroy &&
        api.error_string)
      api.h = h;
  });
  if (!api.h) throw Error(POFD_E_CUDA, "libnccl.so.2 could not be opened");
  return api;
}

void nk(ncclResult_t r, const char* what) {
  if (r != ncclSuccess) {
    std::ostringstream s;
    s << what << ": " << nccl().error_string(r);
    throw Error(POFD_E_CUDA, s.str());
  }
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << what << ": " << cudaGetErrorString(e);
    throw Error(e == cudaErrorMemoryAllocation ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}

// This rank's rows of a batch of nprop proposals over world ranks.
__host__ __device__ inline void rows_of(unsigned nprop, int world, int rank, unsigned* lo,
                                        unsigned* hi) {
  *lo = static_cast<unsigned>(static_cast<unsigned long long>(nprop) * rank / world);
  *hi = static_cast<unsigned>(static_cast<unsigned long long>(nprop) * (rank + 1) / world);
}

// send = [logL of this rank's m rows, NaN padded to cap | their statuses as
// doubles, 0 padded]
__global__ void k_shard_pack(unsigned m, unsigned cap, const double* __restrict__ logl,
                             const int* __restrict__ status, double* __restrict__ send) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cap) return;
  send[i] = (i < m) ? logl[i] : __longlong_as_double(0x7ff8000000000000LL);
  send[cap + i] = (i < m) ? static_cast<double>(status[i]) : 0.0;
}

// recv = the world ranks' send buffers in rank order; row g of the batch
// is row g - lo(r) of its owner r
__global__ void k_shard_unpack(unsigned nprop, int world, unsigned cap,
                               const double* __restrict__ recv, double* __restrict__ logl,
                               int* __restrict__ status) {
  const unsigned g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nprop) return;
  for (int r = 0; r < world; ++r) {
    unsigned lo, hi;
    rows_of(nprop, world, r, &lo, &hi);
    if (g >= lo && g < hi) {
      const double* src = recv + static_cast<size_t>(r) * 2 * cap;
      logl[g] = src[g - lo];
      status[g] = static_cast<int>(src[cap + g - lo]);
      return;
    }
  }
}

}  // namespace

class ShardLike {
 public:
  ShardLike(int device, cudaStream_t stream, const unsigned char* id, int rank, int world,
            pofd_batch_loglike_fn inner, void* inner_like)
      : device_(device), stream_(stream), rank_(rank), world_(world), inner_(inner),
        inner_like_(inner_like) {
    if (device < 0) throw Error(POFD_E_CUDA, "host-only context has no GPU");
    if (world < 1 || rank < 0 || rank >= world) throw Error(POFD_E_ARG, "need 0 <= rank < world");
    if (!inner) throw Error(POFD_E_ARG, "no inner likelihood");
    ck(cudaSetDevice(device_), "cudaSetDevice");
    ncclUniqueId uid;
    static_assert(sizeof(uid.internal) == 128, "NCCL unique id is 128 bytes");
    std::memcpy(uid.internal, id, 128);
    nk(nccl().comm_init_rank(&comm_, world_, uid, rank_), "ncclCommInitRank");
  }
  ~ShardLike() {
    cudaSetDevice(device_);
    if (comm_) nccl().comm_destroy(comm_);
    free_buffers();
  }
  void eval(unsigned nprop, const float* theta, unsigned npar, double* logl, int* status,
            cudaStream_t st) {
    if (nprop == 0) return;
    ck(cudaSetDevice(device_), "cudaSetDevice");
    if (!st) st = stream_;  // as the inner likelihoods read a NULL stream
    const unsigned cap = (nprop + world_ - 1) / world_;
    if (cap > cap_) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      ck(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing");
      if (cs != cudaStreamCaptureStatusNone)
        throw Error(POFD_E_ARG, "sharded likelihood: first use of a batch size inside a capture");
      reserve((cap + 31) / 32 * 32);
    }
    unsigned lo, hi;
    rows_of(nprop, world_, rank_, &lo, &hi);
    if (hi > lo) {
      const int rc = inner_(inner_like_, hi - lo, theta + static_cast<size_t>(lo) * npar, npar,
                            sl_logl_, sl_status_, st);
      if (rc < 0) throw Error(rc, "sharded likelihood: the inner likelihood failed");
    }
    k_shard_pack<<<(cap + 127) / 128, 128, 0, st>>>(hi - lo, cap, sl_logl_, sl_status_, send_);
    ck(cudaGetLastError(), "k_shard_pack");
    nk(nccl().all_gather(send_, recv_, 2 * static_cast<size_t>(cap), ncclDouble, comm_, st),
       "ncclAllGather");
    k_shard_unpack<<<(nprop + 127) / 128, 128, 0, st>>>(nprop, world_, cap, recv_, logl, status);
    ck(cudaGetLastError(), "k_shard_unpack");
  }

 private:
  void free_buffers() {
    cudaFree(sl_logl_);
    cudaFree(sl_status_);
    cudaFree(send_);
    cudaFree(recv_);
    sl_logl_ = nullptr;
    sl_status_ = nullptr;
    send_ = recv_ = nullptr;
    cap_ = 0;
  }
  void reserve(unsigned cap) {
    free_buffers();
    ck(cudaMalloc(&sl_logl_, cap * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc(&sl_status_, cap * sizeof(int)), "cudaMalloc");
    ck(cudaMalloc(&send_, 2 * static_cast<size_t>(cap) * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc(&recv_, 2 * static_cast<size_t>(cap) * world_ * sizeof(double)), "cudaMalloc");
    cap_ = cap;
  }
  int device_;
  cudaStream_t stream_;
  int rank_, world_;
  pofd_batch_loglike_fn inner_;
  void* inner_like_;
  ncclComm_t comm_ = nullptr;
  unsigned cap_ = 0;
  double* sl_logl_ = nullptr;
  int* sl_status_ = nullptr;
  double* send_ = nullptr;
  double* recv_ = nullptr;
};

}  // namespace pofd

struct pofd_ctx;
struct pofd_shard {
  std::unique_ptr<pofd::ShardLike> s;
};

namespace pofd {
void set_last_error(const char* msg);  // capi.cu
int ctx_device(const pofd_ctx* ctx);   // capi.cu
cudaStream_t ctx_stream(const pofd_ctx* ctx);
}

namespace {
template <class F>
int shard_guard(F&& f) {
  try {
    return f();
  } catch (const pofd::Error& e) {
    pofd::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    pofd::set_last_error(e.what());
    return POFD_E_ARG;
  }
}
}  // namespace

extern "C" {

int pofd_shard_rows(unsigned nprop, int world, int rank, unsigned* lo, unsigned* hi) {
  if (!lo || !hi || world < 1 || rank < 0 || rank >= world) {
    pofd::set_last_error("pofd_shard_rows: need lo, hi and 0 <= rank < world");
    return POFD_E_ARG;
  }
  pofd::rows_of(nprop, world, rank, lo, hi);
  return POFD_OK;
}

int pofd_nccl_unique_id(unsigned char* id_out) {
  return shard_guard([&] {
    if (!id_out) throw pofd::Error(POFD_E_ARG, "null argument");
    ncclUniqueId uid;
    pofd::nk(pofd::nccl().get_unique_id(&uid), "ncclGetUniqueId");
    std::memcpy(id_out, uid.internal, 128);
    return POFD_OK;
  });
}

int pofd_shard_create(pofd_ctx* ctx, const unsigned char* id, int rank, int world,
                      pofd_batch_loglike_fn inner, void* inner_like, pofd_shard** out) {
  return shard_guard([&] {
    if (!ctx || !id || !inner || !out) throw pofd::Error(POFD_E_ARG, "null argument");
    std::unique_ptr<pofd_shard> s(new pofd_shard());
    s->s.reset(new pofd::ShardLike(pofd::ctx_device(ctx), pofd::ctx_stream(ctx), id, rank, world,
                                   inner, inner_like));
    *out = s.release();
    return POFD_OK;
  });
}

int pofd_shard_destroy(pofd_shard* s) {
  delete s;
  return POFD_OK;
}

int pofd_shard_eval_batch_device(void* sv, unsigned nprop, const float* theta_dev,
                                 unsigned npar, double* logl_dev, int* status_dev,
                                 void* stream) {
  return shard_guard([&] {
    pofd_shard* s = static_cast<pofd_shard*>(sv);
    if (!s || !theta_dev || !logl_dev || !status_dev) throw pofd::Error(POFD_E_ARG, "null argument");
    s->s->eval(nprop, theta_dev, npar, logl_dev, status_dev, static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

}  // extern "C"
