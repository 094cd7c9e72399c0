// fftplan.hh -- batched cuFFT plans of several batch sizes sharing one
// work area.
//
// The engines keep a plan pair per batch size (the delayed-acceptance
// sampler evaluates survivor batches of varying size); with cuFFT's own
// allocation every plan would hold a work area of its own.  Here plans are
// made without auto-allocation and all point at one area sized for the
// largest, which is safe because an engine runs its transforms one after
// another on one stream.
#ifndef POFD_FFTPLAN_HH
#define POFD_FFTPLAN_HH

#include <cuda_runtime.h>
#include <cufft.h>

#include <sstream>
#include <vector>

#include "setup.hh"

namespace pofd {

inline void fft_check(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) {
    std::ostringstream s;
    s << what << ": cuFFT error " << static_cast<int>(r);
    throw Error(r == CUFFT_ALLOC_FAILED ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}

class FftWorkArea {
 public:
  ~FftWorkArea() {
    if (ptr_) cudaFree(ptr_);
  }
  // Makes a plan (no auto-allocation) and attaches it to the shared area;
  // returns true when the area had to grow, in which case every plan made
  // earlier has been re-pointed and graphs captured before are stale.
  bool make(cufftHandle* h, int rank, int* n, int* inembed, int idist, int* onembed, int odist,
            cufftType type, int batch) {
    fft_check(cufftCreate(h), "cufftCreate");
    fft_check(cufftSetAutoAllocation(*h, 0), "cufftSetAutoAllocation");
    size_t ws = 0;
    fft_check(cufftMakePlanMany(*h, rank, n, inembed, 1, idist, onembed, 1, odist, type, batch,
                                &ws),
              "cufftMakePlanMany");
    bool grew = false;
    if (ws > bytes_) {
      void* p = nullptr;
      if (cudaMalloc(&p, ws) != cudaSuccess) throw Error(POFD_E_NOMEM, "cuFFT work area");
      if (ptr_) {
        cudaDeviceSynchronize();
        cudaFree(ptr_);
      }
      ptr_ = p;
      bytes_ = ws;
      for (cufftHandle o : plans_) fft_check(cufftSetWorkArea(o, ptr_), "cufftSetWorkArea");
      grew = true;
    }
    if (ptr_) fft_check(cufftSetWorkArea(*h, ptr_), "cufftSetWorkArea");
    plans_.push_back(*h);
    return grew;
  }
  void forget(cufftHandle h) {
    for (size_t i = 0; i < plans_.size(); ++i)
      if (plans_[i] == h) {
        plans_.erase(plans_.begin() + static_cast<long>(i));
        return;
      }
  }
  size_t bytes() const { return bytes_; }

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
  std::vector<cufftHandle> plans_;
};

}  // namespace pofd
#endif
