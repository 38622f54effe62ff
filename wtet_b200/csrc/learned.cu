// Learned insertion scheduler: training kernels and the C ABI around them.
//
// The network (learned.cuh) is trained on the device by the kernels below:
// a fused forward + backward pass over a tile of 32 samples per block (FP32,
// activations in shared memory), per-block parameter gradients reduced in a
// fixed order (so a training run is deterministic), and Adam (Kingma & Ba,
// "Adam: A Method for Stochastic Optimization", 2015, Algorithm 1).  The loss
// is the mean binary cross-entropy of the logit against the label "this vote
// winner's cavity is large (more tets than a two-ring pre-claim covers)",
// computed in the numerically stable form
// max(l, 0) - l*y + log(1 + exp(-|l|)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wtet.h"
#include "engine.cuh"
#include "learned.cuh"

namespace wtet {
namespace {

using namespace mlp;

constexpr int TS = 32;          // samples per block of the training step
constexpr int TT = 256;         // threads per block of the training step
constexpr uint32_t kMaxStepBlocks = 1024;

struct TrainSmem {
  float x[TS][kIn];
  float h1[TS][kHidden];
  float h2[TS][kHidden];
  float h3[TS][kHidden];
  float da[TS][kHidden];
  float db[TS][kHidden];
  float dl[TS];
  float loss[TS];
};

// One dense ReLU layer on the tile: out[r][o] = relu(b[o] + sum_k in[r][k] W[o][k]).
template <int K>
__device__ __forceinline__ void dense_relu(const float (*in)[K], float (*out)[kHidden], const float* W, const float* b) {
  for (int e = threadIdx.x; e < TS * kHidden; e += TT) {
    const int r = e / kHidden, o = e % kHidden;
    float a = b[o];
#pragma unroll 4
    for (int k = 0; k < K; ++k) a += in[r][k] * W[o * K + k];
    out[r][o] = fmaxf(a, 0.f);
  }
}

// Forward + backward of samples [s0, s0 + TS) of this block (sample s is row
// idx[s] of X when idx is given).  Writes this block's gradient of the mean
// loss (scaled by inv_n) to part[blockIdx.x] and its loss share to part_loss.
__global__ void __launch_bounds__(TT) k_train_step(const float* __restrict__ X, const float* __restrict__ Y,
                                                   const uint32_t* __restrict__ idx, uint32_t n, uint32_t first,
                                                   float inv_n, const float* __restrict__ P, float* part,
                                                   float* part_loss) {
  __shared__ TrainSmem S;
  const int tid = threadIdx.x;
  const uint32_t s0 = first + blockIdx.x * TS;
  for (int e = tid; e < TS * kIn; e += TT) {
    const int r = e / kIn, k = e % kIn;
    const uint32_t s = s0 + r;
    float v = 0.f;
    if (s < n) v = X[size_t(idx ? idx[s] : s) * kIn + k];
    S.x[r][k] = v;
  }
  __syncthreads();
  dense_relu<kIn>(S.x, S.h1, P + kOffW1, P + kOffB1);
  __syncthreads();
  dense_relu<kHidden>(S.h1, S.h2, P + kOffW2, P + kOffB2);
  __syncthreads();
  dense_relu<kHidden>(S.h2, S.h3, P + kOffW3, P + kOffB3);
  __syncthreads();
  if (tid < TS) {
    const uint32_t s = s0 + tid;
    const bool valid = s < n;
    float l = P[kOffB4];
    for (int k = 0; k < kHidden; ++k) l += S.h3[tid][k] * P[kOffW4 + k];
    const float y = valid ? Y[idx ? idx[s] : s] : 0.f;
    const float sp = fmaxf(l, 0.f) - l * y + log1pf(expf(-fabsf(l)));
    const float sig = 1.f / (1.f + expf(-l));
    S.dl[tid] = valid ? (sig - y) * inv_n : 0.f;
    S.loss[tid] = valid ? sp * inv_n : 0.f;
  }
  __syncthreads();
  float* G = part + size_t(blockIdx.x) * kParams;
  // output layer
  if (tid < kHidden) {
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.dl[r] * S.h3[r][tid];
    G[kOffW4 + tid] = g;
  } else if (tid == kHidden) {
    float g = 0.f, L = 0.f;
    for (int r = 0; r < TS; ++r) {
      g += S.dl[r];
      L += S.loss[r];
    }
    G[kOffB4] = g;
    part_loss[blockIdx.x] = L;
  }
  for (int e = tid; e < TS * kHidden; e += TT) {
    const int r = e / kHidden, k = e % kHidden;
    S.da[r][k] = S.h3[r][k] > 0.f ? S.dl[r] * P[kOffW4 + k] : 0.f;
  }
  __syncthreads();
  // layer 3: dW3 = da^T h2, db3 = sum da, dh2 = (da W3) * [h2 > 0]
  for (int e = tid; e < kHidden * kHidden; e += TT) {
    const int o = e / kHidden, k = e % kHidden;
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.da[r][o] * S.h2[r][k];
    G[kOffW3 + e] = g;
  }
  if (tid < kHidden) {
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.da[r][tid];
    G[kOffB3 + tid] = g;
  }
  for (int e = tid; e < TS * kHidden; e += TT) {
    const int r = e / kHidden, k = e % kHidden;
    float g = 0.f;
    for (int o = 0; o < kHidden; ++o) g += S.da[r][o] * P[kOffW3 + o * kHidden + k];
    S.db[r][k] = S.h2[r][k] > 0.f ? g : 0.f;
  }
  __syncthreads();
  // layer 2
  for (int e = tid; e < kHidden * kHidden; e += TT) {
    const int o = e / kHidden, k = e % kHidden;
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.db[r][o] * S.h1[r][k];
    G[kOffW2 + e] = g;
  }
  if (tid < kHidden) {
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.db[r][tid];
    G[kOffB2 + tid] = g;
  }
  for (int e = tid; e < TS * kHidden; e += TT) {
    const int r = e / kHidden, k = e % kHidden;
    float g = 0.f;
    for (int o = 0; o < kHidden; ++o) g += S.db[r][o] * P[kOffW2 + o * kHidden + k];
    S.da[r][k] = S.h1[r][k] > 0.f ? g : 0.f;
  }
  __syncthreads();
  // layer 1
  for (int e = tid; e < kHidden * kIn; e += TT) {
    const int o = e / kIn, k = e % kIn;
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.da[r][o] * S.x[r][k];
    G[kOffW1 + e] = g;
  }
  if (tid < kHidden) {
    float g = 0.f;
    for (int r = 0; r < TS; ++r) g += S.da[r][tid];
    G[kOffB1 + tid] = g;
  }
}

// grads (+)= sum over blocks of the per-block gradients, in block order.
__global__ void k_reduce_grads(const float* part, uint32_t blocks, float* grads, int accumulate,
                               const float* part_loss, float* loss_acc) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < uint32_t(kParams)) {
    float g = accumulate ? grads[j] : 0.f;
    for (uint32_t b = 0; b < blocks; ++b) g += part[size_t(b) * kParams + j];
    grads[j] = g;
  }
  if (j == 0) {
    float L = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) L += part_loss[b];
    *loss_acc += L;
  }
}

// Adam with bias correction folded into the step size lr_t.
__global__ void k_adam(float* P, const float* G, float* M, float* V, float lr_t, float b1, float b2, float eps) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= uint32_t(kParams)) return;
  const float g = G[j];
  const float m = b1 * M[j] + (1.f - b1) * g;
  const float v = b2 * V[j] + (1.f - b2) * g * g;
  M[j] = m;
  V[j] = v;
  P[j] -= lr_t * m / (sqrtf(v) + eps);
}

// Scores feature rows through the fused inference routine of the vote.
__global__ void __launch_bounds__(128) k_score(const Image* img, const float* X, uint32_t n, float* out) {
  __shared__ __align__(16) Smem S;
  __shared__ __align__(16) uint32_t rows[4][32 * kRowStride];
  __shared__ float outs[4][32];
  load_image(S, img);
  __syncthreads();
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * 4;
  for (uint32_t base = (blockIdx.x * 4 + w) * 32; base < n; base += warps * 32) {
    const uint32_t i = base + lane;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) f[k] = i < n ? X[size_t(i) * kIn + k] : 0.f;
    stage_row(rows[w] + lane * kRowStride, f);
    __syncwarp();
    score32(S, rows[w], outs[w]);
    if (i < n) out[i] = outs[w][lane];
    __syncwarp();
  }
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{WTET_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class T>
struct Buf {
  T* p = nullptr;
  explicit Buf(size_t n, const char* what) { ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), what); }
  ~Buf() {
    if (p) cudaFree(p);
  }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
};

void require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    throw Error{WTET_ERR_CUDA, "no CUDA device available: the wtet_b200 device path needs a GPU"};
}

// splitmix64 (Steele, Lea & Flood 2014): the shuffling generator.
uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Forward + backward over samples [0, n) (or idx[0..n) when idx is set) in
// chunks of kMaxStepBlocks tiles; gradient of loss * scale summed into d_grads.
void loss_grad_device(const float* d_x, const float* d_y, const uint32_t* d_idx, uint32_t n, float inv_n,
                      const float* d_p, float* d_grads, float* d_part, float* d_part_loss, float* d_loss,
                      cudaStream_t s) {
  const uint32_t tiles = (n + TS - 1) / TS;
  for (uint32_t t0 = 0; t0 < tiles; t0 += kMaxStepBlocks) {
    const uint32_t blocks = std::min(kMaxStepBlocks, tiles - t0);
    k_train_step<<<blocks, TT, 0, s>>>(d_x, d_y, d_idx, n, t0 * TS, inv_n, d_p, d_part, d_part_loss);
    k_reduce_grads<<<(kParams + 255) / 256, 256, 0, s>>>(d_part, blocks, d_grads, t0 > 0 ? 1 : 0, d_part_loss,
                                                         d_loss);
  }
  ck(cudaGetLastError(), "training kernels");
}

}  // namespace
}  // namespace wtet

using wtet::Error;

namespace {
int fail(int status, const std::string& msg) {
  wtet::set_last_error(msg);
  return status;
}
}  // namespace

extern "C" {

int wtet_learned_set_weights(const float* params, uint64_t count) {
  if (!params) return fail(WTET_ERR_ARG, "null pointer argument");
  if (count != uint64_t(wtet::mlp::kParams))
    return fail(WTET_ERR_ARG, "expected " + std::to_string(wtet::mlp::kParams) + " parameters, got " +
                                  std::to_string(count));
  for (uint64_t i = 0; i < count; ++i)
    if (!std::isfinite(params[i])) return fail(WTET_ERR_ARG, "non-finite parameter at index " + std::to_string(i));
  wtet::set_mlp_params(params);
  return WTET_OK;
}

int wtet_learned_has_weights(void) { return wtet::has_mlp_params() ? 1 : 0; }

int wtet_learned_collect(const float* xyz, const uint64_t* offsets, uint32_t num_clouds, const wtet_config* cfg,
                         uint32_t sample_shift, float* features, uint8_t* labels, uint64_t capacity,
                         uint64_t* count, wtet_stats* stats) {
  if (!xyz || !offsets || !count || num_clouds == 0 || (capacity && (!features || !labels)))
    return fail(WTET_ERR_ARG, "bad collect arguments");
  if (capacity > 0xFFFFFFF0ull) return fail(WTET_ERR_ARG, "capacity too large");
  std::vector<uint64_t> off(offsets, offsets + num_clouds + 1);
  if (off[0] != 0) return fail(WTET_ERR_ARG, "offsets[0] must be 0");
  for (uint32_t c = 0; c < num_clouds; ++c)
    if (off[c + 1] < off[c] + 4)
      return fail(WTET_ERR_ARG, "cloud " + std::to_string(c) + ": Need at least 4 points for 3D Delaunay");
  try {
    wtet::require_device();
    wtet_config c;
    wtet_config_default(&c);
    if (cfg) c = *cfg;
    if (c.max_insert_iterations == 0) c.max_insert_iterations = 100;
    const uint64_t n = off.back();
    cudaStream_t s = nullptr;
    float* d_xyz = wtet::ws_input(3 * n);
    wtet::ck(cudaMemcpyAsync(d_xyz, xyz, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s), "copy points");
    wtet::Buf<float> lx(std::max<uint64_t>(capacity, 1) * wtet::mlp::kIn, "log features");
    wtet::Buf<uint8_t> ly(std::max<uint64_t>(capacity, 1), "log labels");
    wtet::Job job;
    job.d_xyz = d_xyz;
    job.offsets = off;
    job.cfg = c;
    job.stream = s;
    job.d_log_x = lx.p;
    job.d_log_y = ly.p;
    job.log_cap = capacity;
    job.log_shift = sample_shift;
    wtet::JobResult r = wtet::run_job(job, nullptr, nullptr, 0);
    *count = r.logged;
    if (r.logged) {
      wtet::ck(cudaMemcpy(features, lx.p, r.logged * wtet::mlp::kIn * sizeof(float), cudaMemcpyDeviceToHost),
               "copy features");
      wtet::ck(cudaMemcpy(labels, ly.p, r.logged, cudaMemcpyDeviceToHost), "copy labels");
    }
    r.stats.num_failed = r.failed.size();
    if (stats) *stats = r.stats;
    return WTET_OK;
  } catch (const Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_mlp_loss_grad(const float* x, const float* y, uint64_t n, const float* params, float* loss,
                       float* grads) {
  using namespace wtet;
  if (!x || !y || !params || !loss || !grads || n == 0) return fail(WTET_ERR_ARG, "bad loss_grad arguments");
  if (n > 0x7FFFFFFFull) return fail(WTET_ERR_ARG, "too many samples");
  try {
    require_device();
    cudaStream_t s = nullptr;
    Buf<float> dx(n * mlp::kIn, "samples"), dy(n, "labels"), dp(mlp::kParams, "params"), dg(mlp::kParams, "grads");
    Buf<float> part(size_t(kMaxStepBlocks) * mlp::kParams, "partial grads"), pl(kMaxStepBlocks, "partial loss");
    Buf<float> dl(1, "loss");
    ck(cudaMemcpy(dx.p, x, n * mlp::kIn * 4, cudaMemcpyHostToDevice), "copy samples");
    ck(cudaMemcpy(dy.p, y, n * 4, cudaMemcpyHostToDevice), "copy labels");
    ck(cudaMemcpy(dp.p, params, mlp::kParams * 4, cudaMemcpyHostToDevice), "copy params");
    ck(cudaMemset(dl.p, 0, 4), "memset");
    loss_grad_device(dx.p, dy.p, nullptr, uint32_t(n), float(1.0 / double(n)), dp.p, dg.p, part.p, pl.p, dl.p, s);
    ck(cudaMemcpy(grads, dg.p, mlp::kParams * 4, cudaMemcpyDeviceToHost), "copy grads");
    ck(cudaMemcpy(loss, dl.p, 4, cudaMemcpyDeviceToHost), "copy loss");
    return WTET_OK;
  } catch (const Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_mlp_train(const float* x, const float* y, uint64_t n, const wtet_train_config* tc, float* params,
                   float* epoch_loss) {
  using namespace wtet;
  if (!x || !y || !tc || !params || n == 0) return fail(WTET_ERR_ARG, "bad train arguments");
  if (n > 0x7FFFFFFFull) return fail(WTET_ERR_ARG, "too many samples");
  if (tc->batch == 0 || tc->batch > kMaxStepBlocks * TS)
    return fail(WTET_ERR_ARG, "batch must be in 1.." + std::to_string(kMaxStepBlocks * TS));
  if (!(tc->lr > 0.f) || !(tc->beta1 >= 0.f && tc->beta1 < 1.f) || !(tc->beta2 >= 0.f && tc->beta2 < 1.f) ||
      !(tc->eps > 0.f))
    return fail(WTET_ERR_ARG, "bad Adam hyper-parameters");
  try {
    require_device();
    cudaStream_t s = nullptr;
    Buf<float> dx(n * mlp::kIn, "samples"), dy(n, "labels"), dp(mlp::kParams, "params"), dg(mlp::kParams, "grads");
    Buf<float> dm(mlp::kParams, "adam m"), dv(mlp::kParams, "adam v");
    Buf<float> part(size_t(kMaxStepBlocks) * mlp::kParams, "partial grads"), pl(kMaxStepBlocks, "partial loss");
    Buf<float> dl(1, "loss");
    Buf<uint32_t> didx(n, "permutation");
    ck(cudaMemcpy(dx.p, x, n * mlp::kIn * 4, cudaMemcpyHostToDevice), "copy samples");
    ck(cudaMemcpy(dy.p, y, n * 4, cudaMemcpyHostToDevice), "copy labels");
    ck(cudaMemcpy(dp.p, params, mlp::kParams * 4, cudaMemcpyHostToDevice), "copy params");
    ck(cudaMemset(dm.p, 0, mlp::kParams * 4), "memset");
    ck(cudaMemset(dv.p, 0, mlp::kParams * 4), "memset");
    std::vector<uint32_t> perm(n);
    uint64_t rng = tc->seed;
    uint64_t step = 0;
    for (uint32_t ep = 0; ep < tc->epochs; ++ep) {
      for (uint64_t i = 0; i < n; ++i) perm[i] = uint32_t(i);
      for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix(rng) % (i + 1)]);  // Fisher-Yates
      ck(cudaMemcpy(didx.p, perm.data(), n * 4, cudaMemcpyHostToDevice), "copy permutation");
      ck(cudaMemset(dl.p, 0, 4), "memset");
      uint64_t batches = 0;
      for (uint64_t b = 0; b < n; b += tc->batch) {
        const uint32_t nb = uint32_t(std::min<uint64_t>(tc->batch, n - b));
        loss_grad_device(dx.p, dy.p, didx.p + b, nb, 1.f / float(nb), dp.p, dg.p, part.p, pl.p, dl.p, s);
        ++step;
        const double c1 = 1.0 - std::pow(double(tc->beta1), double(step));
        const double c2 = 1.0 - std::pow(double(tc->beta2), double(step));
        const float lr_t = float(double(tc->lr) * std::sqrt(c2) / c1);
        k_adam<<<(mlp::kParams + 255) / 256, 256, 0, s>>>(dp.p, dg.p, dm.p, dv.p, lr_t, tc->beta1, tc->beta2,
                                                           tc->eps * float(std::sqrt(c2)));
        ++batches;
      }
      ck(cudaGetLastError(), "adam");
      float L = 0.f;
      ck(cudaMemcpy(&L, dl.p, 4, cudaMemcpyDeviceToHost), "copy loss");
      if (epoch_loss) epoch_loss[ep] = L / float(batches);
    }
    ck(cudaMemcpy(params, dp.p, mlp::kParams * 4, cudaMemcpyDeviceToHost), "copy params");
    return WTET_OK;
  } catch (const Error& e) {
    return fail(e.status, e.msg);
  }
}

int wtet_mlp_score(const float* x, uint64_t n, float* scores) {
  using namespace wtet;
  if (!x || !scores || n == 0) return fail(WTET_ERR_ARG, "bad score arguments");
  if (n > 0x7FFFFFFFull) return fail(WTET_ERR_ARG, "too many samples");
  try {
    require_device();
    cudaStream_t s = nullptr;
    const mlp::Image* img = static_cast<const mlp::Image*>(mlp_image(s));
    Buf<float> dx(n * mlp::kIn, "samples"), dout(n, "scores");
    ck(cudaMemcpy(dx.p, x, n * mlp::kIn * 4, cudaMemcpyHostToDevice), "copy samples");
    const uint32_t blocks = uint32_t(std::min<uint64_t>((n + 127) / 128, 148 * 8));
    k_score<<<blocks, 128, 0, s>>>(img, dx.p, uint32_t(n), dout.p);
    ck(cudaGetLastError(), "score kernel");
    ck(cudaMemcpy(scores, dout.p, n * 4, cudaMemcpyDeviceToHost), "copy scores");
    return WTET_OK;
  } catch (const Error& e) {
    return fail(e.status, e.msg);
  }
}

}  // extern "C"
