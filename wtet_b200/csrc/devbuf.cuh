// Device-buffer and scan helpers shared by the engine's host code
// (engine.cu) and the verifier / canonicaliser (verify.cu).  Internal to
// libwtet.so.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "engine.cuh"

namespace wtet {
namespace dev {

// ----------------------------------------------------------- scan utils ----

static __global__ void k_scan_blocks(const uint32_t* in, uint32_t* out, uint32_t* sums, uint32_t n) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t per = 4;
  uint32_t base = blockIdx.x * blockDim.x * per;
  uint32_t v[per];
  uint32_t local = 0;
  for (uint32_t k = 0; k < per; ++k) {
    uint32_t i = base + threadIdx.x * per + k;
    v[k] = i < n ? in[i] : 0u;
    local += v[k];
  }
  uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = local;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= uint32_t(o)) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= uint32_t(o)) w += y;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  uint32_t excl = x - local + (warp ? warp_tot[warp - 1] : 0u);
  for (uint32_t k = 0; k < per; ++k) {
    uint32_t i = base + threadIdx.x * per + k;
    if (i < n) out[i] = excl;
    excl += v[k];
  }
  if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = excl;
}

static __global__ void k_scan_add(uint32_t* out, const uint32_t* sums, uint32_t n) {
  uint32_t base = blockIdx.x * blockDim.x * 4;
  uint32_t add = sums[blockIdx.x];
  for (uint32_t k = 0; k < 4; ++k) {
    uint32_t i = base + threadIdx.x * 4 + k;
    if (i < n) out[i] += add;
  }
}


inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{WTET_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void reserve(size_t want, const char* what) {
    if (want <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    ck(cudaMalloc(&p, std::max<size_t>(want, 1) * sizeof(T)), what);
    n = want;
  }
  void grow_keep(size_t want, size_t used, cudaStream_t s, const char* what) {
    if (want <= n) return;
    T* q = nullptr;
    ck(cudaMalloc(&q, want * sizeof(T)), what);
    if (p && used) ck(cudaMemcpyAsync(q, p, used * sizeof(T), cudaMemcpyDeviceToDevice, s), what);
    ck(cudaStreamSynchronize(s), what);
    if (p) cudaFree(p);
    p = q;
    n = want;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Exclusive scan in place over n u32 (recursive over block sums).
inline int scan_u32(uint32_t* d, uint32_t n, cudaStream_t s, std::vector<DBuf<uint32_t>>& tmp, int depth = 0) {
  if (n == 0) return 0;
  const uint32_t threads = 256, per_block = threads * 4;
  uint32_t blocks = (n + per_block - 1) / per_block;
  if (int(tmp.size()) <= depth) tmp.resize(depth + 1);
  tmp[depth].reserve(size_t(blocks) + 1, "scan sums");
  k_scan_blocks<<<blocks, threads, 0, s>>>(d, d, tmp[depth].p, n);
  int launches = 1;
  if (blocks > 1) {
    launches += scan_u32(tmp[depth].p, blocks, s, tmp, depth + 1);
    k_scan_add<<<blocks, threads, 0, s>>>(d, tmp[depth].p, n);
    ++launches;
  }
  return launches;
}

}  // namespace dev
}  // namespace wtet
