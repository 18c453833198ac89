// devbuf.cuh -- owning device buffer that only grows (host-side helper).
// A buffer that has to grow takes at least 1.5x its old capacity and never
// less than 64 KiB, so sizes that creep up step by step from zero (contacts,
// pairs) reallocate rarely: cudaFree synchronises the whole device.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace ando {

template <class T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t reserve(size_t count) {
    if (count <= n && p) return cudaSuccess;
    constexpr size_t floor_elems = (size_t(64) << 10) / sizeof(T) > 0 ? (size_t(64) << 10) / sizeof(T) : 1;
    size_t c = count > floor_elems ? count : floor_elems;
    if (p) { c = c > n + n / 2 ? c : n + n / 2; cudaFree(p); p = nullptr; n = 0; }
    cudaError_t e = cudaMalloc(&p, c * sizeof(T));
    if (e == cudaSuccess) n = c;
    return e;
  }
  // exactly `count` elements (at least one), contents dropped
  cudaError_t resize_exact(size_t count) {
    if (p) { cudaFree(p); p = nullptr; n = 0; }
    cudaError_t e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
    if (e == cudaSuccess) n = count ? count : 1;
    return e;
  }
  cudaError_t upload(const T* h, size_t count, cudaStream_t s) {
    cudaError_t e = reserve(count);
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
  }
};

}  // namespace ando
