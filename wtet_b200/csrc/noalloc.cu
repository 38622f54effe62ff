// Allocation-free variant of the exact quality check (wtet_check_quality).
//
// Some callers cannot allocate GPU memory while they run this check: serving
// loops whose GPU memory belongs to an allocator that another framework owns
// (a cudaMalloc from the library would stall on, or fragment, that pool), and
// hosts whose memory budget is fixed up front so that no call may grow it.
// This entry point therefore keeps its scratch -- the normalised points, the
// bounding box and the counters -- in one file-scope device array of fixed
// size, which every GPU that loads libwtet.so holds until the process exits.
// It calls no cudaMalloc, cudaFree or allocating library routine.
//
// The array is shared by every call on a device and keeps the last call's
// contents; each call clears the parts that must start at zero.  Calls whose
// work overlaps on the GPU (two streams, or two host threads) race on the
// array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/wtet.h"
#include "engine.cuh"
#include "exact.cuh"

namespace wtet_noalloc {

constexpr uint64_t kMaxPoints = WTET_NOALLOC_MAX_POINTS;
constexpr uint32_t NONE = 0xFFFFFFFFu;

// Layout: kMaxPoints float4 normalised points | 3 u32 min | 3 u32 max |
// 2 u64 counters | u32 error flags (offsets below, all 16-byte aligned).
constexpr size_t kPtsBytes = kMaxPoints * 16;
constexpr size_t kBoxOff = kPtsBytes;
constexpr size_t kCntOff = kBoxOff + 32;
constexpr size_t kErrOff = kCntOff + 16;
constexpr size_t kScratchBytes = kErrOff + 16;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}
__device__ __forceinline__ uint32_t comp(const uint4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Bounding box of the points (src/lib.rs:315-323), NaN ignored.
__global__ void k_box(const float* xyz, uint64_t n, unsigned char* scratch) {
  uint32_t* mn = reinterpret_cast<uint32_t*>(scratch + kBoxOff);
  uint32_t* mx = mn + 3;
  __shared__ uint32_t smn[3], smx[3];
  if (threadIdx.x < 3) {
    smn[threadIdx.x] = 0xFFFFFFFFu;
    smx[threadIdx.x] = 0u;
  }
  __syncthreads();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      float v = xyz[3 * i + k];
      if (v != v) continue;
      atomicMin(&smn[k], f2o(v));
      atomicMax(&smx[k], f2o(v));
    }
  __syncthreads();
  if (threadIdx.x < 3) {
    atomicMin(&mn[threadIdx.x], smn[threadIdx.x]);
    atomicMax(&mx[threadIdx.x], smx[threadIdx.x]);
  }
}

// p' = (p - min) / max_extent in f32 (src/lib.rs:325-334).
__global__ void k_norm(const float* xyz, uint64_t n, unsigned char* scratch) {
  const uint32_t* mn = reinterpret_cast<const uint32_t*>(scratch + kBoxOff);
  const uint32_t* mx = mn + 3;
  float4* pts = reinterpret_cast<float4*>(scratch);
  float lo[3], ext[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = o2f(mn[k]);
    ext[k] = o2f(mx[k]) - lo[k];
  }
  float s = fmaxf(fmaxf(fmaxf(ext[0], ext[1]), ext[2]), 1e-10f);
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    pts[i] = make_float4(__fdiv_rn(__fsub_rn(xyz[3 * i], lo[0]), s), __fdiv_rn(__fsub_rn(xyz[3 * i + 1], lo[1]), s),
                         __fdiv_rn(__fsub_rn(xyz[3 * i + 2], lo[2]), s), 0.f);
}

// Exact local-Delaunay count over pairs of all-real tets (src/lib.rs:25-78).
__global__ void k_check(uint64_t n, const uint4* tets, const uint4* adj, uint64_t m, unsigned char* scratch) {
  const float4* pts = reinterpret_cast<const float4*>(scratch);
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(scratch + kCntOff);
  uint32_t* err = reinterpret_cast<uint32_t*>(scratch + kErrOff);
  unsigned long long viol = 0, interior = 0;
  for (uint64_t ti = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; ti < m; ti += uint64_t(gridDim.x) * blockDim.x) {
    uint4 t = tets[ti];
    if (t.x >= n || t.y >= n || t.z >= n || t.w >= n) continue;
    ++interior;
    uint4 a = adj[ti];
    for (int f = 0; f < 4; ++f) {
      uint32_t packed = comp(a, f);
      if (packed == NONE) continue;
      uint64_t oti = packed >> 5;
      if (ti >= oti) continue;
      if (oti >= m) {
        atomicOr(err, 1u);
        continue;
      }
      uint4 o = tets[oti];
      if (o.x >= n || o.y >= n || o.z >= n || o.w >= n) continue;
      uint32_t vb = comp(o, packed & 3);
      double P[5][3];
      const uint32_t ids[5] = {t.x, t.y, t.z, t.w, vb};
      for (int k = 0; k < 5; ++k) {
        float4 q = pts[ids[k]];
        P[k][0] = q.x;
        P[k][1] = q.y;
        P[k][2] = q.z;
      }
      int s = wtet::ex::insphere(P[0], P[1], P[2], P[3], P[4], err);
      if (s == 0) s = wtet::ex::orient4d_sos_degenerate(P[0], P[1], P[2], P[3], P[4], ids[0], ids[1], ids[2],
                                                         ids[3], ids[4], err);
      if (s < 0) ++viol;
    }
  }
  atomicAdd(&cnt[0], viol);
  atomicAdd(&cnt[1], interior);
}

// The device address of g_scratch belongs to the context the module was
// loaded into: after cudaDeviceReset the primary context is created anew and
// the array may move.  The cache is therefore keyed on the context's unique
// id (cuCtxGetId, reached through the runtime's driver entry points so that
// the library needs no link against libcuda).
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

struct ScratchEntry {
  unsigned long long ctx_id = 0;
  void* ptr = nullptr;
};

std::mutex g_mu;
ScratchEntry g_cache[64];

// Unique id of the current context (0 when it cannot be read).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    looked_up = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
  return 0;
}

// Device address of g_scratch in the current device's context, looked up once
// per context with that device current (host code must not use &g_scratch:
// in host code that name is a host-side stand-in, not a device address).
int scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    wtet::set_last_error("no usable CUDA device");
    return WTET_ERR_CUDA;
  }
  // cudaSetDevice creates the device's primary context (CUDA 12), so that its
  // id can be read before the first launch.
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    wtet::set_last_error(std::string("no usable CUDA context: ") + cudaGetErrorString(e));
    return WTET_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  const unsigned long long ctx = current_context_id();
  ScratchEntry& c = g_cache[dev];
  if (!c.ptr || ctx == 0 || c.ctx_id != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      wtet::set_last_error(std::string("cudaGetSymbolAddress(scratch) failed: ") + cudaGetErrorString(e));
      return WTET_ERR_CUDA;
    }
    c.ptr = p;
    c.ctx_id = ctx;
  }
  *out = static_cast<unsigned char*>(c.ptr);
  return WTET_OK;
}

}  // namespace wtet_noalloc

extern "C" {

int wtet_check_quality_noalloc(const float* d_xyz, uint64_t n, const uint32_t* d_tets,
                               const uint32_t* d_adjacency, uint64_t m, uint64_t* violations,
                               uint64_t* interior_tets, void* stream) {
  using namespace wtet_noalloc;
  if (!d_xyz || !violations || !interior_tets || (m && (!d_tets || !d_adjacency))) {
    wtet::set_last_error("null pointer argument");
    return WTET_ERR_ARG;
  }
  if (n > kMaxPoints) {
    wtet::set_last_error("wtet_check_quality_noalloc: " + std::to_string(n) + " points exceed its fixed scratch of " +
            std::to_string(kMaxPoints) + " points; use wtet_check_quality");
    return WTET_ERR_ARG;
  }
  unsigned char* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != WTET_OK) return rc;
  // An error left pending by the caller's own earlier work is neither taken
  // (cleared) nor reported as this call's: the call refuses to run instead.
  cudaError_t prior = cudaPeekAtLastError();
  if (prior != cudaSuccess) {
    wtet::set_last_error(std::string("a CUDA error from earlier work on this thread is pending: ") +
                         cudaGetErrorString(prior));
    return WTET_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Only the box, the counters and the error word must start cleared.
  cudaError_t e = cudaMemsetAsync(scratch + kBoxOff, 0xFF, 12, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch + kBoxOff + 12, 0x00, 12, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch + kCntOff, 0, kScratchBytes - kCntOff, s);
  if (e != cudaSuccess) {
    wtet::set_last_error(std::string("clearing scratch: ") + cudaGetErrorString(e));
    return WTET_ERR_CUDA;
  }
  if (n) {
    k_box<<<148, 256, 0, s>>>(d_xyz, n, scratch);
    k_norm<<<148 * 4, 256, 0, s>>>(d_xyz, n, scratch);
  }
  if (m)
    k_check<<<148 * 8, 128, 0, s>>>(n, reinterpret_cast<const uint4*>(d_tets),
                                    reinterpret_cast<const uint4*>(d_adjacency), m, scratch);
  unsigned long long cnt[2] = {0, 0};
  uint32_t err = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, scratch + kCntOff, 16, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, scratch + kErrOff, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    wtet::set_last_error(std::string("check kernels: ") + cudaGetErrorString(e));
    return WTET_ERR_CUDA;
  }
  if (err & 1u) {
    wtet::set_last_error("adjacency refers to a tet out of range");
    return WTET_ERR_ARG;
  }
  if (err) {
    wtet::set_last_error("exact arithmetic buffer overflow");
    return WTET_ERR_PRECISION;
  }
  *violations = cnt[0];
  *interior_tets = cnt[1];
  return WTET_OK;
}

}  // extern "C"
