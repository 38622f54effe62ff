// Host-side engine interface shared by the C ABI (capi.cu) and the kernels
// (engine.cu).  No CUDA or torch types cross the public C ABI; this header is
// internal to libwtet.so.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/wtet.h"

namespace wtet {

// Raised inside the engine; the C ABI turns it into a status + message.
struct Error {
  int status;
  std::string msg;
};

// Device buffers for one triangulation job; kept per thread and grown on
// demand so that repeated calls do not pay for cudaMalloc.
struct Workspace;

// One job: `num_clouds` clouds; cloud c has points offsets[c]..offsets[c+1]-1
// of the device array d_xyz (f32 triples).  Output rows for cloud c start at
// out_off[c] (host, filled by run()).  d_tets / d_adj receive cloud-local ids.
struct Job {
  const float* d_xyz = nullptr;
  std::vector<uint64_t> offsets;  // host, num_clouds + 1
  wtet_config cfg{};
  cudaStream_t stream = nullptr;
  uint32_t rounds_per_graph = 0;  // 0: default
};

struct JobResult {
  std::vector<uint64_t> tet_offsets;  // host, num_clouds + 1
  std::vector<uint64_t> failed;       // global input indices of exact duplicates, ascending
  wtet_stats stats{};
};

// Triangulates on the device; output written to d_tets / d_adj (device, row
// major u32x4) when they are non-null and capacity suffices, else only the
// counts are produced (status WTET_ERR_CAPACITY is raised by the caller).
JobResult run_job(const Job& job, uint32_t* d_tets, uint32_t* d_adj, uint64_t capacity);

// Exact local-Delaunay count of src/lib.rs:25-78 on the device.
void check_quality_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adj,
                          uint64_t m, uint64_t* violations, uint64_t* interior, cudaStream_t stream);

// Upper bound on output tets for a cloud of n points.
uint64_t max_tets_for(uint64_t n);

void release_thread_workspace();

// Message returned by wtet_last_error() on this thread.
void set_last_error(const std::string& msg);

// Per-thread device buffers reused across calls (grown on demand).
float* ws_input(size_t nfloats);
void ws_outputs(size_t rows, uint32_t** tets, uint32_t** adj);

}  // namespace wtet
