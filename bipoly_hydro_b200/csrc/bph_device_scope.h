// bph_device_scope.h -- the caller's current CUDA device, saved and restored.
//
// Every C-ABI entry point that works on a context makes the context's device
// current for the duration of the call and puts the caller's current device
// back before it returns, so a host program that drives other work on
// another GPU from the same thread never finds its device switched.  The
// Fortran host of the reference owns one GPU per rank; a library that left
// a different device current would redirect that rank's later CUDA calls.
//
// The guard is a template over the two runtime calls it needs so that its
// logic can be tested on a machine without a GPU (tests/test_device_scope.py
// compiles it against a fake runtime); DeviceScope below binds it to the
// CUDA runtime.
#pragma once

namespace bph {

// Rt provides: using err_t; static constexpr err_t ok; static err_t get(int*);
// static err_t set(int).
template <class Rt>
class DeviceScopeT {
  public:
    explicit DeviceScopeT(int device) {
        err_ = Rt::get(&prev_);
        if (err_ != Rt::ok) return;
        if (prev_ != device) {
            err_ = Rt::set(device);
            switched_ = (err_ == Rt::ok);
        }
    }
    ~DeviceScopeT() {
        if (switched_) Rt::set(prev_);
    }
    DeviceScopeT(const DeviceScopeT &) = delete;
    DeviceScopeT &operator=(const DeviceScopeT &) = delete;
    // Result of saving the caller's device and selecting the context's one.
    typename Rt::err_t status() const { return err_; }
    int previous() const { return prev_; }

  private:
    int prev_ = -1;
    bool switched_ = false;
    typename Rt::err_t err_ = Rt::ok;
};

}  // namespace bph

#ifdef __CUDACC__
#include <cuda_runtime.h>

namespace bph {
struct CudaDeviceRt {
    using err_t = cudaError_t;
    static constexpr cudaError_t ok = cudaSuccess;
    static cudaError_t get(int *d) { return cudaGetDevice(d); }
    static cudaError_t set(int d) { return cudaSetDevice(d); }
};
using DeviceScope = DeviceScopeT<CudaDeviceRt>;
}  // namespace bph

// Declares `scope_` making ctx->device current until the end of the
// enclosing block; returns BPH_ERR_CUDA from the enclosing function when the
// device cannot be selected.
#define BPH_DEVICE_SCOPE(ctx)                                               \
    ::bph::DeviceScope scope_((ctx)->device);                               \
    do {                                                                    \
        if (scope_.status() != cudaSuccess)                                 \
            return ::bph::cuda_fail(scope_.status(), "select the context's device"); \
    } while (0)
#endif
