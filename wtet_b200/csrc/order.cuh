// Space-filling-curve cell indices used to order points before insertion
// (host and device): Morton (bit interleave) and Hilbert.  Only the order in
// which points are inserted depends on them, never the triangulation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace wtet {

__host__ __device__ __forceinline__ uint32_t expand10(uint32_t v) {
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Morton index of cell (x, y, z): bits interleaved z, y, x from the top.
__host__ __device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return (expand10(z) << 2) | (expand10(y) << 1) | expand10(x);
}

// Hilbert index of cell (x, y, z) on a 2^bits grid (bits <= 10), by
// Skilling's transpose method ("Programming the Hilbert curve", AIP Conf.
// Proc. 707, 2004): undo the rotations/reflections level by level, Gray-code,
// then interleave the transposed coordinates.  Consecutive indices are
// face-adjacent cells.  The reference reaches a Hilbert order through the
// hilbert_index crate (src/hilbert.rs:20-38); only the order of insertion
// depends on it, never the result.
__host__ __device__ __forceinline__ uint32_t hilbert3(uint32_t x, uint32_t y, uint32_t z, uint32_t bits) {
  uint32_t X[3] = {x, y, z};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  return (expand10(X[0]) << 2) | (expand10(X[1]) << 1) | expand10(X[2]);
}

}  // namespace wtet
