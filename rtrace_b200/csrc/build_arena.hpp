// Device scratch memory for the build steps that run on the device (k-d
// tree, mesh search data).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <utility>
#include <vector>

namespace rtb {

// Chunks kept from build to build, handed out by a bump pointer that each
// build resets.  A build no larger than an earlier one allocates and frees
// nothing (cudaMalloc and above all cudaFree, which waits for the device,
// cost more than the builds' kernels).  One build at a time per arena.
struct KdArena {
  std::vector<std::pair<char*, size_t>> chunks;
  size_t at = 0, used = 0;  // chunk in use, bytes used in it
  ~KdArena() {
    for (auto& c : chunks) cudaFree(c.first);
  }
  void reset() { at = used = 0; }
  template <class T>
  cudaError_t get(T** out, size_t count) {
    const size_t bytes = (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~(size_t)255;
    while (at < chunks.size()) {
      if (used + bytes <= chunks[at].second) {
        *out = reinterpret_cast<T*>(chunks[at].first + used);
        used += bytes;
        return cudaSuccess;
      }
      at++;
      used = 0;
    }
    size_t total = 0;
    for (auto& c : chunks) total += c.second;
    const size_t size = std::max(bytes, std::max(total, (size_t)64 << 20));
    char* c = nullptr;
    cudaError_t e = cudaMalloc((void**)&c, size);
    if (e != cudaSuccess) return e;
    chunks.push_back({c, size});
    at = chunks.size() - 1;
    used = bytes;
    *out = reinterpret_cast<T*>(c);
    return cudaSuccess;
  }
};

}  // namespace rtb
