// Learned insertion scheduler: per vote-winner features and the fused BF16
// MLP that sets the claim priority of the vote winners.
//
// The reference orders insertions by the circumsphere determinant alone
// (src/shaders/vote.wgsl:401-494); it has no learned scheduler.  Here every
// tet still votes for the point deepest in its circumsphere; the vote winners
// then compete for their cavities by claim keys, and the one with the smaller
// key wins a contested tet.  With hashed keys (the plain method) the winners
// of a crowded neighbourhood lose to each other round after round, and those
// neighbourhoods set the number of rounds.  The network (12 -> 64 -> 64 -> 64
// -> 1, ReLU, BF16 weights and activations, FP32 accumulate; trained on the
// plain method's own logs) predicts each winner's probability of inserting in
// this round under hashed keys; winners predicted least likely to insert --
// the crowded ones -- claim first.  It is used in the rounds of the first
// strata, which cost a fixed overhead per round whatever their size; the
// bulk rounds, where the work per round dominates, keep hashed keys.  Only
// the order changes: every round still inserts an exactly
// Delaunay-compatible set of points, so the final tet set is the same unique
// SoS triangulation.
//
// Inference runs on the tensor cores with warp-level mma.m16n8k16 (BF16 in,
// FP32 accumulate), fused into the kernel that turns votes into winners: each
// warp scores its 32 points at once, the activations stay in registers
// between layers (an accumulator fragment of one layer is the A fragment of
// the next), and the weights sit in shared memory with padded rows so that
// every fragment load is bank-conflict free.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wtet {
namespace mlp {

constexpr int kIn = 12;      // features
constexpr int kHidden = 64;  // width of the three hidden layers
// Flat FP32 parameter layout shared by training, the C ABI and Python:
// W1[64][12] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kIn;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kHidden * kHidden;
constexpr int kOffW4 = kOffB3 + kHidden;
constexpr int kOffB4 = kOffW4 + kHidden;
constexpr int kParams = kOffB4 + 1;  // 9217

// Shared-memory copy of the inference weights.  BF16 pairs are stored as
// 32-bit words; rows are padded (24 and 72 BF16) so that the 8 row groups x
// 4 column pairs of an mma fragment hit 32 distinct banks.
constexpr int kW1Stride = 12;  // words per row of W1 (16 BF16 inputs + 8 pad)
constexpr int kWStride = 36;   // words per row of W2 / W3 (64 BF16 + 8 pad)
constexpr int kRowStride = 12; // words per staged feature row
struct Smem {
  uint32_t w1[kHidden * kW1Stride];
  uint32_t w2[kHidden * kWStride];
  uint32_t w3[kHidden * kWStride];
  float w4[kHidden];
  float b1[kHidden], b2[kHidden], b3[kHidden];
  float b4;
};

// Device image of the inference weights, produced once from the FP32
// parameters (BF16 round-to-nearest-even) and copied into Smem per block.
struct Image {
  uint32_t w1[kHidden * kW1Stride];
  uint32_t w2[kHidden * kWStride];
  uint32_t w3[kHidden * kWStride];
  float w4[kHidden];  // BF16-rounded values held as FP32
  float b1[kHidden], b2[kHidden], b3[kHidden];
  float b4;
  float pad[3];
};
static_assert(sizeof(Image) % 16 == 0, "image copied in 16-byte words");
static_assert(sizeof(Smem) <= sizeof(Image), "smem image fits");

__device__ __forceinline__ void load_image(Smem& S, const Image* __restrict__ img) {
  const uint4* src = reinterpret_cast<const uint4*>(img);
  uint4* dst = reinterpret_cast<uint4*>(&S);
  constexpr int words = int(sizeof(Smem) / 16);
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  if (threadIdx.x == 0) S.b4 = img->b4;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ReLU, BF16 rounding and the accumulator -> A-fragment hand-over: n-tiles
// 2kk and 2kk+1 of this layer's output are k-step kk of the next layer.
__device__ __forceinline__ void relu_pack(const float (*acc)[4], uint32_t (*a)[4]) {
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    a[kk][0] = pack_bf16(fmaxf(acc[2 * kk][0], 0.f), fmaxf(acc[2 * kk][1], 0.f));
    a[kk][1] = pack_bf16(fmaxf(acc[2 * kk][2], 0.f), fmaxf(acc[2 * kk][3], 0.f));
    a[kk][2] = pack_bf16(fmaxf(acc[2 * kk + 1][0], 0.f), fmaxf(acc[2 * kk + 1][1], 0.f));
    a[kk][3] = pack_bf16(fmaxf(acc[2 * kk + 1][2], 0.f), fmaxf(acc[2 * kk + 1][3], 0.f));
  }
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Scores the 32 staged rows of one warp (features as BF16 pairs, row stride
// kRowStride words) into out[0..31].  All 32 lanes must call it.
__device__ __forceinline__ void score32(const Smem& S, const uint32_t* rows, float* out) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const uint32_t* r0 = rows + (16 * mt + g) * kRowStride;
    const uint32_t* r1 = r0 + 8 * kRowStride;
    float acc[8][4];
    uint32_t a[4][4];
    // layer 1: K = 16 (12 features, 4 zero columns)
    {
      const uint32_t x[4] = {r0[t], r1[t], r0[t + 4], r1[t + 4]};
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float c0 = S.b1[8 * j + 2 * t], c1 = S.b1[8 * j + 2 * t + 1];
        acc[j][0] = c0, acc[j][1] = c1, acc[j][2] = c0, acc[j][3] = c1;
        const uint32_t* w = S.w1 + (8 * j + g) * kW1Stride;
        mma_bf16(acc[j], x, w[t], w[t + 4]);
      }
    }
    relu_pack(acc, a);
    // layers 2 and 3: K = 64
#pragma unroll
    for (int layer = 0; layer < 2; ++layer) {
      const uint32_t* W = layer == 0 ? S.w2 : S.w3;
      const float* B = layer == 0 ? S.b2 : S.b3;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float c0 = B[8 * j + 2 * t], c1 = B[8 * j + 2 * t + 1];
        acc[j][0] = c0, acc[j][1] = c1, acc[j][2] = c0, acc[j][3] = c1;
        const uint32_t* w = W + (8 * j + g) * kWStride;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) mma_bf16(acc[j], a[kk], w[8 * kk + t], w[8 * kk + t + 4]);
      }
      if (layer == 0) relu_pack(acc, a);
    }
    // layer 4: 64 -> 1 on the FP32 pipes, reduced over the 4 lanes of a row group
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float w0 = S.w4[8 * j + 2 * t], w1 = S.w4[8 * j + 2 * t + 1];
      s0 += bf16r(fmaxf(acc[j][0], 0.f)) * w0 + bf16r(fmaxf(acc[j][1], 0.f)) * w1;
      s1 += bf16r(fmaxf(acc[j][2], 0.f)) * w0 + bf16r(fmaxf(acc[j][3], 0.f)) * w1;
    }
    s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, 1);
    s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, 2);
    s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, 1);
    s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, 2);
    if (t == 0) {
      out[16 * mt + g] = s0 + S.b4;
      out[16 * mt + g + 8] = s1 + S.b4;
    }
  }
  __syncwarp();
}

// Stores 12 features as one staged BF16 row (columns 12..15 zero).
__device__ __forceinline__ void stage_row(uint32_t* row, const float* f) {
#pragma unroll
  for (int k = 0; k < 6; ++k) row[k] = pack_bf16(f[2 * k], f[2 * k + 1]);
  row[6] = 0u;
  row[7] = 0u;
}

__device__ __forceinline__ float finite_or(float x, float dflt) { return isfinite(x) ? x : dflt; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// The 12 features of vote winner q in tet (a, b, c, d), all O(1) by construction:
//  0 |q - circumcenter|^2 / R^2            6 log2(1 + round) / 8
//  1 log2(vote score) / 64                 7 log2(1 + earlier wins of q that did not insert) / 4
//  2 6*sqrt(2)*V / emax^3 (1 = regular)    8 uninserted points / points of the last stratum, / 2
//  3 log2(R / emax) / 4                    9 log2(1 + uninserted points) / 24
//  4 face-neighbour tets holding a winner / 4          10 -log2(emax) / 16 (tet size)
//  5 of those, winners with a larger vote score / 4    11 the tet has a super vertex
__device__ __forceinline__ void features(float4 a, float4 b, float4 c, float4 d, float4 q, float score,
                                         uint32_t rivals1, uint32_t rivals2, uint32_t round, uint32_t losses,
                                         uint32_t n_active, uint32_t stratum, float* f) {
  const float abx = b.x - a.x, aby = b.y - a.y, abz = b.z - a.z;
  const float acx = c.x - a.x, acy = c.y - a.y, acz = c.z - a.z;
  const float adx = d.x - a.x, ady = d.y - a.y, adz = d.z - a.z;
  const float bcx = c.x - b.x, bcy = c.y - b.y, bcz = c.z - b.z;
  const float bdx = d.x - b.x, bdy = d.y - b.y, bdz = d.z - b.z;
  const float cdx = d.x - c.x, cdy = d.y - c.y, cdz = d.z - c.z;
  const float lab = abx * abx + aby * aby + abz * abz, lac = acx * acx + acy * acy + acz * acz;
  const float lad = adx * adx + ady * ady + adz * adz, lbc = bcx * bcx + bcy * bcy + bcz * bcz;
  const float lbd = bdx * bdx + bdy * bdy + bdz * bdz, lcd = cdx * cdx + cdy * cdy + cdz * cdz;
  const float emax2 = fmaxf(fmaxf(fmaxf(lab, lac), fmaxf(lad, lbc)), fmaxf(lbd, lcd));
  const float emax = sqrtf(emax2);
  // cross products for the circumcenter (relative to a)
  const float x1 = acy * adz - acz * ady, y1 = acz * adx - acx * adz, z1 = acx * ady - acy * adx;  // ac x ad
  const float x2 = ady * abz - adz * aby, y2 = adz * abx - adx * abz, z2 = adx * aby - ady * abx;  // ad x ab
  const float x3 = aby * acz - abz * acy, y3 = abz * acx - abx * acz, z3 = abx * acy - aby * acx;  // ab x ac
  const float vol6 = abx * x1 + aby * y1 + abz * z1;
  const float inv = 0.5f / vol6;
  const float ox = (lab * x1 + lac * x2 + lad * x3) * inv;
  const float oy = (lab * y1 + lac * y2 + lad * y3) * inv;
  const float oz = (lab * z1 + lac * z2 + lad * z3) * inv;
  const float R2 = ox * ox + oy * oy + oz * oz;
  const float qx = q.x - (a.x + ox), qy = q.y - (a.y + oy), qz = q.z - (a.z + oz);
  const float av6 = fabsf(vol6);
  const bool sup = a.x < -50.f || a.x > 200.f || b.x < -50.f || b.x > 200.f || c.x < -50.f || c.x > 200.f ||
                   d.x < -50.f || d.x > 200.f;
  f[0] = clampf(finite_or((qx * qx + qy * qy + qz * qz) / R2, 1.f), 0.f, 1.f);
  f[1] = clampf(finite_or(__log2f(score + 1e-37f), -128.f) * (1.f / 64.f), -2.f, 2.f);
  f[2] = clampf(finite_or(av6 * 1.41421356f / (emax2 * emax), 0.f), 0.f, 1.f);
  f[3] = clampf(finite_or(0.5f * __log2f(R2 / emax2), 8.f), -8.f, 8.f) * 0.25f;
  f[4] = float(rivals1) * 0.25f;
  f[5] = float(rivals2) * 0.25f;
  f[6] = __log2f(1.f + float(round)) * 0.125f;
  f[7] = __log2f(1.f + float(losses)) * 0.25f;
  f[8] = clampf(float(n_active) / float(max(stratum, 1u)), 0.f, 2.f) * 0.5f;
  f[9] = __log2f(1.f + float(n_active)) * (1.f / 24.f);
  f[10] = clampf(finite_or(-__log2f(emax), 0.f) * (1.f / 16.f), -1.f, 2.f);
  f[11] = sup ? 1.f : 0.f;
}

}  // namespace mlp
}  // namespace wtet
