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
  // Training log of the learned scheduler (recorded when d_log_x is set):
  // features (log_cap x 12 f32) and labels (log_cap u8) of 1 in 2^log_shift
  // vote winners.
  float* d_log_x = nullptr;
  uint8_t* d_log_y = nullptr;
  uint64_t log_cap = 0;
  uint32_t log_shift = 0;
};

struct JobResult {
  std::vector<uint64_t> tet_offsets;  // host, num_clouds + 1
  std::vector<uint64_t> failed;       // global input indices of exact duplicates, ascending
  wtet_stats stats{};
  uint64_t logged = 0;  // training records written (<= log_cap)
};

// Triangulates on the device; output written to d_tets / d_adj (device, row
// major u32x4) when they are non-null and capacity suffices, else only the
// counts are produced (status WTET_ERR_CAPACITY is raised by the caller).
JobResult run_job(const Job& job, uint32_t* d_tets, uint32_t* d_adj, uint64_t capacity);

// Exact local-Delaunay count of src/lib.rs:25-78 on the device.
void check_quality_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adj,
                          uint64_t m, uint64_t* violations, uint64_t* interior, cudaStream_t stream);

// Normalised points (src/lib.rs:313-337) of one cloud into d_out (n float4,
// w = 0); box is scratch for 6 u32 (ordered min / max per axis).
void normalize_points_device(const float* d_xyz, uint64_t n, float4* d_out, uint32_t* box, cudaStream_t stream);

// Every-face exact verification of a triangulation (verify.cu).
void verify_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adj, uint64_t m,
                   wtet_verify_report* report, cudaStream_t stream);

// Canonical parity form on the device (verify.cu); returns the row count.
uint64_t canonicalize_device(const uint32_t* d_tets, const uint32_t* d_adj, uint64_t m, uint64_t n,
                             uint32_t* d_out_tets, uint32_t* d_out_adj, cudaStream_t stream);
void release_verify_workspace();

// Signs of the round kernels' predicates on records of five points (testing).
void predicate_signs_device(const float* d_pts, const uint32_t* d_keys, uint64_t m, int32_t* d_o3, int32_t* d_o4,
                            cudaStream_t stream);

// Upper bound on output tets for a cloud of n points.
uint64_t max_tets_for(uint64_t n);

void release_thread_workspace();

// Learned-vote weights: FP32 parameters in the flat layout of learned.cuh,
// converted to the BF16 device image and uploaded to each device on first use.
void set_mlp_params(const float* params);
bool has_mlp_params();
// Device image of the installed weights on the current device (uploads on
// `stream` when stale); throws when no weights are installed.
const void* mlp_image(cudaStream_t stream);

// Autotuner table (wtet_autotune_set_table) and the knob resolution it drives.
void set_tune_table(const wtet_tune_entry* entries, uint32_t count);
std::vector<wtet_tune_entry> get_tune_table();
wtet_config tuned_config(const wtet_config& cfg, uint64_t n, uint32_t num_clouds);

// Message returned by wtet_last_error() on this thread.
void set_last_error(const std::string& msg);

// Per-thread device buffers reused across calls (grown on demand).
float* ws_input(size_t nfloats);
void ws_outputs(size_t rows, uint32_t** tets, uint32_t** adj);

}  // namespace wtet
