// Grow-only device arena owned by a tribit context.
//
// The reference allocates and frees every intermediate array from the
// default CUDA memory pool inside the timed region (tribit.cu:48-84, 825-838).
// Here a context plans all buffers of a call up front (a measuring pass of the
// same layout code), reserves one block, and hands out 256-byte-aligned
// slices; later calls of the same or smaller size allocate nothing, which also
// keeps every launch address stable for CUDA-graph replay.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tb {

class Arena {
 public:
  Arena() = default;
  Arena(const Arena&) = delete;
  Arena& operator=(const Arena&) = delete;
  ~Arena() { release(); }

  // Start a layout pass. With measure == true nothing is handed out and only
  // the total size is accumulated.
  void begin(bool measure) {
    measuring_ = measure;
    off_ = 0;
  }
  size_t used() const { return off_; }
  size_t capacity() const { return cap_; }

  // headroom: 1/16 more, so that slightly larger calls reuse the allocation
  // (taken only when it can be had; never under a device budget).
  void reserve(size_t bytes, bool headroom = true) {
    if (bytes <= cap_) return;
    if (base_ && !owned_)
      throw StatusError(TRIBIT_ERR_TOO_LARGE, "graph needs more scratch than the fixed device buffer holds");
    release();
    size_t want = headroom ? bytes + (bytes >> 4) : bytes;
    cudaError_t e = cudaMalloc(&base_, want);
    if (e != cudaSuccess && want != bytes) {
      (void)cudaGetLastError();
      want = bytes;
      e = cudaMalloc(&base_, want);
    }
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      base_ = nullptr;
      throw StatusError(TRIBIT_ERR_OUT_OF_MEMORY, "device arena allocation failed");
    }
    cap_ = want;
  }

  template <typename T>
  T* take(uint64_t count) {
    size_t bytes = (size_t)count * sizeof(T);
    size_t at = (off_ + 255) & ~(size_t)255;
    off_ = at + bytes;
    if (measuring_) return nullptr;
    if (off_ > cap_) throw StatusError(TRIBIT_ERR_INTERNAL, "arena layout exceeded its reservation");
    return reinterpret_cast<T*>(static_cast<char*>(base_) + at);
  }

  bool measuring() const { return measuring_; }

  // Moves the layout cursor back to `at` (a used() of this pass): later takes
  // reuse the space after it, which the caller no longer needs once the work
  // queued on it has run (stream order).
  void rewind(size_t at) {
    if (at > off_) throw StatusError(TRIBIT_ERR_INTERNAL, "arena rewound past its cursor");
    off_ = at;
  }

  void release() {
    if (base_ && owned_) cudaFree(base_);
    base_ = nullptr;
    cap_ = 0;
    owned_ = true;
  }

  // Hands out slices of caller-owned device memory instead of allocating:
  // reserve() then only checks that the layout fits in `bytes`.
  void attach(void* base, size_t bytes) {
    release();
    base_ = base;
    cap_ = bytes;
    owned_ = false;
  }
  bool attached() const { return !owned_; }

 private:
  void* base_ = nullptr;
  size_t cap_ = 0;
  size_t off_ = 0;
  bool measuring_ = false;
  bool owned_ = true;
};

}  // namespace tb
