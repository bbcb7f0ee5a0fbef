// Internal helpers shared by the libdec_b200 translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "dec_b200.h"

namespace decb {

// Error carried from the implementation to the C ABI, which turns it into a dec_status.
struct Error : std::runtime_error {
  dec_status status;
  Error(dec_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

#define DEC_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t err__ = (call);                                                            \
    if (err__ != cudaSuccess) {                                                            \
      if (err__ == cudaErrorMemoryAllocation) {                                            \
        cudaGetLastError();                                                                \
        throw ::decb::Error(DEC_ERR_OOM, std::string(#call) + ": " + cudaGetErrorString(err__)); \
      }                                                                                    \
      throw ::decb::Error(DEC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err__)); \
    }                                                                                      \
  } while (0)

#define DEC_CHECK_LAUNCH() DEC_CUDA(cudaGetLastError())

inline void require(bool ok, const std::string& msg) {
  if (!ok) throw Error(DEC_ERR_INVALID_ARG, msg);
}
// A literal message builds no string unless the check fails (checks inside per-element loops).
inline void require(bool ok, const char* msg) {
  if (!ok) throw Error(DEC_ERR_INVALID_ARG, msg);
}

// Owning device array.
template <class T>
struct DArr {
  T* p = nullptr;
  size_t n = 0;
  DArr() = default;
  explicit DArr(size_t count) { alloc(count); }
  DArr(const DArr&) = delete;
  DArr& operator=(const DArr&) = delete;
  DArr(DArr&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DArr& operator=(DArr&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DArr() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) DEC_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T* h, size_t count) {
    alloc(count);
    if (count) DEC_CUDA(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
  }
  void upload(const std::vector<T>& h) { upload(h.data(), h.size()); }
  std::vector<T> download() const {
    std::vector<T> h(n);
    if (n) DEC_CUDA(cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
  }
  size_t bytes() const { return n * sizeof(T); }
};

inline int num_sms() {
  static int sms = [] {
    int dev = 0, v = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
  }();
  return sms;
}

// Grid for a grid-stride loop over n items: at most `per_sm` resident CTAs per SM.
inline unsigned grid_for(long long n, int threads, int per_sm = 8) {
  long long want = (n + threads - 1) / threads;
  long long cap = (long long)num_sms() * per_sm;
  if (want < 1) want = 1;
  return (unsigned)(want < cap ? want : cap);
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace decb
