// C ABI of libwtet.so (include/wtet.h).  Host orchestration lives in
// engine.cu; this file validates arguments, moves data between host and
// device, and turns engine errors into status codes and messages.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wtet.h"
#include "engine.cuh"
#include "order.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw wtet::Error{WTET_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

wtet_config resolve(const wtet_config* cfg) {
  wtet_config c;
  wtet_config_default(&c);
  if (cfg) c = *cfg;
  if (c.max_insert_iterations == 0) c.max_insert_iterations = 100;
  return c;
}

void require_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    throw wtet::Error{WTET_ERR_CUDA, "no CUDA device available: the wtet_b200 device path needs a GPU"};
}

void fill_stats(wtet_stats* dst, const wtet_stats& s) {
  if (dst) *dst = s;
}

// Runs one job whose input already sits in device memory; returns device
// output pointers owned by the per-thread workspace.
wtet::JobResult run_dev(const float* d_xyz, const std::vector<uint64_t>& offsets, const wtet_config& cfg,
                        cudaStream_t s, uint32_t** d_t, uint32_t** d_a) {
  wtet::Job job;
  job.d_xyz = d_xyz;
  job.offsets = offsets;
  job.cfg = cfg;
  job.stream = s;
  uint64_t guess = 0;
  for (size_t c = 0; c + 1 < offsets.size(); ++c) guess += wtet::max_tets_for(offsets[c + 1] - offsets[c]);
  wtet::ws_outputs(guess, d_t, d_a);
  wtet::JobResult r = wtet::run_job(job, *d_t, *d_a, guess);
  if (r.tet_offsets.back() > guess) {
    uint64_t need = r.tet_offsets.back();
    wtet::ws_outputs(need, d_t, d_a);
    r = wtet::run_job(job, *d_t, *d_a, need);
  }
  return r;
}

}  // namespace

namespace wtet {
// Lets other translation units of the library report through wtet_last_error().
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace wtet

extern "C" {

void wtet_config_default(wtet_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->insertion_rule = WTET_RULE_CIRCUMCENTER;
  cfg->enable_flipping = 1;
  cfg->enable_sorting = 0;
  cfg->enable_hilbert_sorting = 0;
  cfg->enable_splaying = 1;
  cfg->max_insert_iterations = 100;
  cfg->max_flip_iterations = 10;
  cfg->vote_mode = WTET_VOTE_PLAIN;
  cfg->block_size = 0;
}

uint64_t wtet_max_tets(uint64_t n) { return wtet::max_tets_for(n); }

const char* wtet_last_error(void) { return g_last_error.c_str(); }

const char* wtet_version(void) { return "0.1.0"; }

int wtet_delaunay_into(const float* xyz, uint64_t n, const wtet_config* cfg, uint32_t* tets, uint32_t* adjacency,
                       uint64_t capacity, uint64_t* num_tets, uint32_t* failed_verts, wtet_stats* stats) {
  if (!xyz || !num_tets) return fail(WTET_ERR_ARG, "null pointer argument");
  if (n < 4) return fail(WTET_ERR_ARG, "Need at least 4 points for 3D Delaunay, got " + std::to_string(n));
  try {
    require_device();
    wtet_config c = resolve(cfg);
    cudaStream_t s = nullptr;
    float* d_xyz = wtet::ws_input(3 * n);
    ck(cudaMemcpyAsync(d_xyz, xyz, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s), "copy points to device");
    uint32_t *d_t = nullptr, *d_a = nullptr;
    wtet::JobResult r = run_dev(d_xyz, {0, n}, c, s, &d_t, &d_a);
    uint64_t m = r.tet_offsets.back();
    *num_tets = m;
    r.stats.num_failed = r.failed.size();
    fill_stats(stats, r.stats);
    if (failed_verts)
      for (size_t k = 0; k < r.failed.size(); ++k) failed_verts[k] = uint32_t(r.failed[k]);
    if (m > capacity || !tets || !adjacency)
      return fail(WTET_ERR_CAPACITY, "output capacity " + std::to_string(capacity) + " < " + std::to_string(m) + " tets");
    ck(cudaMemcpyAsync(tets, d_t, m * 16, cudaMemcpyDeviceToHost, s), "copy tets to host");
    ck(cudaMemcpyAsync(adjacency, d_a, m * 16, cudaMemcpyDeviceToHost, s), "copy adjacency to host");
    ck(cudaStreamSynchronize(s), "synchronize");
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_delaunay(const float* xyz, uint64_t n, const wtet_config* cfg, wtet_result* out) {
  if (!xyz || !out) return fail(WTET_ERR_ARG, "null pointer argument");
  std::memset(out, 0, sizeof(*out));
  if (n < 4) return fail(WTET_ERR_ARG, "Need at least 4 points for 3D Delaunay, got " + std::to_string(n));
  try {
    require_device();
    wtet_config c = resolve(cfg);
    cudaStream_t s = nullptr;
    float* d_xyz = wtet::ws_input(3 * n);
    ck(cudaMemcpyAsync(d_xyz, xyz, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s), "copy points to device");
    uint32_t *d_t = nullptr, *d_a = nullptr;
    wtet::JobResult r = run_dev(d_xyz, {0, n}, c, s, &d_t, &d_a);
    uint64_t m = r.tet_offsets.back();
    out->tets = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(m, 1) * 16));
    out->adjacency = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(m, 1) * 16));
    out->failed_verts = static_cast<uint32_t*>(std::malloc(4 * (r.failed.size() + 1)));
    if (!out->tets || !out->adjacency || !out->failed_verts) {
      wtet_result_free(out);
      return fail(WTET_ERR_CAPACITY, "host allocation failed");
    }
    ck(cudaMemcpyAsync(out->tets, d_t, m * 16, cudaMemcpyDeviceToHost, s), "copy tets to host");
    ck(cudaMemcpyAsync(out->adjacency, d_a, m * 16, cudaMemcpyDeviceToHost, s), "copy adjacency to host");
    ck(cudaStreamSynchronize(s), "synchronize");
    out->num_tets = m;
    out->num_failed = r.failed.size();
    for (size_t k = 0; k < r.failed.size(); ++k) out->failed_verts[k] = uint32_t(r.failed[k]);
    r.stats.num_failed = r.failed.size();
    out->stats = r.stats;
    return WTET_OK;
  } catch (const wtet::Error& e) {
    wtet_result_free(out);
    return fail(e.status, e.msg);
  }
}

int wtet_delaunay_device(const float* d_xyz, uint64_t n, const wtet_config* cfg, uint32_t* d_tets,
                         uint32_t* d_adjacency, uint64_t capacity, uint64_t* num_tets, wtet_stats* stats,
                         void* stream) {
  if (!d_xyz || !num_tets) return fail(WTET_ERR_ARG, "null pointer argument");
  if (n < 4) return fail(WTET_ERR_ARG, "Need at least 4 points for 3D Delaunay, got " + std::to_string(n));
  try {
    require_device();
    wtet_config c = resolve(cfg);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    wtet::Job job;
    job.d_xyz = d_xyz;
    job.offsets = {0, n};
    job.cfg = c;
    job.stream = s;
    wtet::JobResult r = wtet::run_job(job, d_tets, d_adjacency, (d_tets && d_adjacency) ? capacity : 0);
    *num_tets = r.tet_offsets.back();
    r.stats.num_failed = r.failed.size();
    fill_stats(stats, r.stats);
    if (*num_tets > capacity || !d_tets || !d_adjacency)
      return fail(WTET_ERR_CAPACITY, "output capacity " + std::to_string(capacity) + " < " +
                                         std::to_string(*num_tets) + " tets");
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_delaunay_batched(const float* xyz, const uint64_t* offsets, uint32_t num_clouds, const wtet_config* cfg,
                          uint32_t* tets, uint32_t* adjacency, uint64_t capacity, uint64_t* tet_offsets,
                          wtet_stats* stats) {
  if (!xyz || !offsets || !tet_offsets || num_clouds == 0) return fail(WTET_ERR_ARG, "bad batched arguments");
  std::vector<uint64_t> off(offsets, offsets + num_clouds + 1);
  if (off[0] != 0) return fail(WTET_ERR_ARG, "offsets[0] must be 0");
  for (uint32_t c = 0; c < num_clouds; ++c) {
    if (off[c + 1] < off[c] + 4)
      return fail(WTET_ERR_ARG, "cloud " + std::to_string(c) + ": Need at least 4 points for 3D Delaunay");
  }
  try {
    require_device();
    wtet_config c = resolve(cfg);
    cudaStream_t s = nullptr;
    uint64_t n = off.back();
    float* d_xyz = wtet::ws_input(3 * n);
    ck(cudaMemcpyAsync(d_xyz, xyz, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s), "copy points to device");
    uint32_t *d_t = nullptr, *d_a = nullptr;
    wtet::JobResult r = run_dev(d_xyz, off, c, s, &d_t, &d_a);
    for (uint32_t k = 0; k <= num_clouds; ++k) tet_offsets[k] = r.tet_offsets[k];
    r.stats.num_failed = r.failed.size();
    fill_stats(stats, r.stats);
    uint64_t m = r.tet_offsets.back();
    if (m > capacity || !tets || !adjacency)
      return fail(WTET_ERR_CAPACITY, "output capacity " + std::to_string(capacity) + " < " + std::to_string(m) + " tets");
    ck(cudaMemcpyAsync(tets, d_t, m * 16, cudaMemcpyDeviceToHost, s), "copy tets to host");
    ck(cudaMemcpyAsync(adjacency, d_a, m * 16, cudaMemcpyDeviceToHost, s), "copy adjacency to host");
    ck(cudaStreamSynchronize(s), "synchronize");
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_check_quality(const float* xyz, uint64_t n, const uint32_t* tets, const uint32_t* adjacency, uint64_t m,
                       uint64_t* violations, uint64_t* interior_tets) {
  if (!xyz || !violations || !interior_tets || (m && (!tets || !adjacency)))
    return fail(WTET_ERR_ARG, "null pointer argument");
  try {
    require_device();
    cudaStream_t s = nullptr;
    float* d_xyz = wtet::ws_input(3 * n + 8 * m + 8);
    uint32_t* d_t = reinterpret_cast<uint32_t*>(d_xyz + 3 * n + ((4 - (3 * n) % 4) % 4));
    uint32_t* d_a = d_t + 4 * m;
    ck(cudaMemcpyAsync(d_xyz, xyz, 3 * n * 4, cudaMemcpyHostToDevice, s), "copy points");
    if (m) {
      ck(cudaMemcpyAsync(d_t, tets, m * 16, cudaMemcpyHostToDevice, s), "copy tets");
      ck(cudaMemcpyAsync(d_a, adjacency, m * 16, cudaMemcpyHostToDevice, s), "copy adjacency");
    }
    wtet::check_quality_device(d_xyz, n, d_t, d_a, m, violations, interior_tets, s);
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_verify_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adjacency,
                       uint64_t m, wtet_verify_report* report, void* stream) {
  if (!d_xyz || !report || (m && (!d_tets || !d_adjacency))) return fail(WTET_ERR_ARG, "null pointer argument");
  try {
    require_device();
    wtet::verify_device(d_xyz, n, d_tets, d_adjacency, m, report, static_cast<cudaStream_t>(stream));
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_verify(const float* xyz, uint64_t n, const uint32_t* tets, const uint32_t* adjacency, uint64_t m,
                wtet_verify_report* report) {
  if (!xyz || !report || (m && (!tets || !adjacency))) return fail(WTET_ERR_ARG, "null pointer argument");
  try {
    require_device();
    cudaStream_t s = nullptr;
    float* d_xyz = wtet::ws_input(3 * n + 8 * m + 8);
    uint32_t* d_t = reinterpret_cast<uint32_t*>(d_xyz + 3 * n + ((4 - (3 * n) % 4) % 4));
    uint32_t* d_a = d_t + 4 * m;
    ck(cudaMemcpyAsync(d_xyz, xyz, 3 * n * 4, cudaMemcpyHostToDevice, s), "copy points");
    if (m) {
      ck(cudaMemcpyAsync(d_t, tets, m * 16, cudaMemcpyHostToDevice, s), "copy tets");
      ck(cudaMemcpyAsync(d_a, adjacency, m * 16, cudaMemcpyHostToDevice, s), "copy adjacency");
    }
    wtet::verify_device(d_xyz, n, d_t, d_a, m, report, s);
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_canonicalize_device(const uint32_t* d_tets, const uint32_t* d_adjacency, uint64_t m, uint64_t n,
                             uint32_t* d_out_tets, uint32_t* d_out_adjacency, uint64_t* num_rows, void* stream) {
  if (!num_rows || (m && (!d_tets || !d_adjacency || !d_out_tets || !d_out_adjacency)))
    return fail(WTET_ERR_ARG, "null pointer argument");
  try {
    require_device();
    *num_rows = wtet::canonicalize_device(d_tets, d_adjacency, m, n, d_out_tets, d_out_adjacency,
                                          static_cast<cudaStream_t>(stream));
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_canonicalize(const uint32_t* tets, const uint32_t* adjacency, uint64_t m, uint64_t n, uint32_t* out_tets,
                      uint32_t* out_adjacency, uint64_t* num_rows) {
  if (!num_rows || (m && (!tets || !adjacency || !out_tets || !out_adjacency)))
    return fail(WTET_ERR_ARG, "null pointer argument");
  try {
    require_device();
    cudaStream_t s = nullptr;
    // inputs in the per-thread input buffer, outputs in the output buffers
    uint32_t* d_in = reinterpret_cast<uint32_t*>(wtet::ws_input(8 * m + 4));
    uint32_t *d_ot = nullptr, *d_oa = nullptr;
    wtet::ws_outputs(std::max<uint64_t>(m, 1), &d_ot, &d_oa);
    if (m) {
      ck(cudaMemcpyAsync(d_in, tets, m * 16, cudaMemcpyHostToDevice, s), "copy tets");
      ck(cudaMemcpyAsync(d_in + 4 * m, adjacency, m * 16, cudaMemcpyHostToDevice, s), "copy adjacency");
    }
    const uint64_t k = wtet::canonicalize_device(d_in, d_in + 4 * m, m, n, d_ot, d_oa, s);
    *num_rows = k;
    if (k) {
      ck(cudaMemcpyAsync(out_tets, d_ot, k * 16, cudaMemcpyDeviceToHost, s), "copy canonical tets");
      ck(cudaMemcpyAsync(out_adjacency, d_oa, k * 16, cudaMemcpyDeviceToHost, s), "copy canonical adjacency");
    }
    ck(cudaStreamSynchronize(s), "synchronize");
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_predicate_signs(const float* pts, const uint32_t* keys, uint64_t m, int32_t* out3, int32_t* out4) {
  if (m && (!pts || !keys || !out3 || !out4)) return fail(WTET_ERR_ARG, "null pointer argument");
  try {
    require_device();
    cudaStream_t s = nullptr;
    // records, keys and both outputs in the per-thread input buffer
    float* d = wtet::ws_input(15 * m + 5 * m + 2 * m + 16);
    uint32_t* d_keys = reinterpret_cast<uint32_t*>(d + 15 * m);
    int32_t* d_o3 = reinterpret_cast<int32_t*>(d + 20 * m);
    int32_t* d_o4 = d_o3 + m;
    if (m) {
      ck(cudaMemcpyAsync(d, pts, 15 * m * 4, cudaMemcpyHostToDevice, s), "copy points");
      ck(cudaMemcpyAsync(d_keys, keys, 5 * m * 4, cudaMemcpyHostToDevice, s), "copy keys");
    }
    wtet::predicate_signs_device(d, d_keys, m, d_o3, d_o4, s);
    if (m) {
      ck(cudaMemcpyAsync(out3, d_o3, m * 4, cudaMemcpyDeviceToHost, s), "copy signs");
      ck(cudaMemcpyAsync(out4, d_o4, m * 4, cudaMemcpyDeviceToHost, s), "copy signs");
    }
    ck(cudaStreamSynchronize(s), "synchronize");
    return WTET_OK;
  } catch (const wtet::Error& e) {
    return fail(e.status, e.msg);
  }
}

void wtet_result_free(wtet_result* r) {
  if (!r) return;
  std::free(r->tets);
  std::free(r->adjacency);
  std::free(r->failed_verts);
  r->tets = r->adjacency = r->failed_verts = nullptr;
  r->num_tets = r->num_failed = 0;
}

static int device_string(char* buf, size_t len, bool init) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  std::string s;
  if (e != cudaSuccess || n == 0) {
    s = "No CUDA device available";
    if (buf && len) std::snprintf(buf, len, "%s", s.c_str());
    return fail(WTET_ERR_CUDA, s);
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp p{};
  cudaGetDeviceProperties(&p, dev);
  if (init) cudaFree(nullptr);
  char tmp[512];
  std::snprintf(tmp, sizeof tmp,
                "%sGPU Device: %s (sm_%d%d), %d SMs, %.1f GiB\nLimits: max_threads_per_block=%d, "
                "shared_mem_per_block_optin=%zu",
                init ? "GPU initialized: " : "", p.name, p.major, p.minor, p.multiProcessorCount,
                double(p.totalGlobalMem) / (1024.0 * 1024.0 * 1024.0), p.maxThreadsPerBlock,
                size_t(p.sharedMemPerBlockOptin));
  if (buf && len) std::snprintf(buf, len, "%s", tmp);
  return WTET_OK;
}

int wtet_autotune_set_table(const wtet_tune_entry* entries, uint32_t count) {
  if (count && !entries) return fail(WTET_ERR_ARG, "null pointer argument");
  for (uint32_t i = 0; i < count; ++i) {
    const wtet_tune_entry& e = entries[i];
    if (e.batched > 1 || (e.block_size && e.block_size != 128 && e.block_size != 256 && e.block_size != 512) ||
        e.rounds_per_graph > 64 || e.overlap_shift > 16 || e.candidate_filter > 2 || e.pool_factor > 64)
      return fail(WTET_ERR_ARG, "autotune entry " + std::to_string(i) + " holds an out-of-range knob");
  }
  wtet::set_tune_table(entries, count);
  return WTET_OK;
}

int wtet_autotune_get_table(wtet_tune_entry* entries, uint32_t capacity, uint32_t* count) {
  if (!count || (capacity && !entries)) return fail(WTET_ERR_ARG, "null pointer argument");
  std::vector<wtet_tune_entry> t = wtet::get_tune_table();
  *count = uint32_t(t.size());
  for (uint32_t i = 0; i < capacity && i < t.size(); ++i) entries[i] = t[i];
  return WTET_OK;
}

int wtet_autotune_resolve(const wtet_config* cfg, uint64_t n, uint32_t num_clouds, wtet_config* out) {
  if (!out) return fail(WTET_ERR_ARG, "null pointer argument");
  *out = wtet::tuned_config(resolve(cfg), n, num_clouds ? num_clouds : 1u);
  return WTET_OK;
}

uint32_t wtet_morton_index(uint32_t x, uint32_t y, uint32_t z) {
  return wtet::morton3(x & 1023u, y & 1023u, z & 1023u);
}

uint32_t wtet_hilbert_index(uint32_t x, uint32_t y, uint32_t z, uint32_t bits) {
  if (bits < 1 || bits > 10) return 0xFFFFFFFFu;
  const uint32_t m = (1u << bits) - 1u;
  return wtet::hilbert3(x & m, y & m, z & m, bits);
}

int wtet_initialize_gpu(char* buf, size_t len) { return device_string(buf, len, true); }
int wtet_gpu_info(char* buf, size_t len) { return device_string(buf, len, false); }

}  // extern "C"
