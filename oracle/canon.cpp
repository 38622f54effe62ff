// Oracle (test infrastructure only): the canonical parity form of a
// triangulation, used to compare two outputs byte for byte.
//
// Canonical tets: every tet that does not use the infinity vertex n+4, its
// vertex ids sorted ascending, the rows sorted lexicographically.  Canonical
// adjacency: for canonical tet i and the face opposite its sorted slot s,
// (canonical index of the neighbour << 5) | (slot of the neighbour's opposite
// vertex in the neighbour's sorted row), or 0xFFFFFFFF where the neighbour is
// missing or is an infinity tet.  The adjacency is derived from the given
// links (src/types.rs:165-174 encoding), so comparing it also checks them.
#include <algorithm>
#include <array>
#include <cstdint>
#include <vector>

#include "oracle.h"

namespace {
constexpr uint32_t NONE = 0xFFFFFFFFu;

// Sorted slot of row slot j (rank of v[j] among the row's four ids).
inline uint32_t rank_in_row(const uint32_t* v, int j) {
  uint32_t r = 0;
  for (int k = 0; k < 4; ++k) r += v[k] < v[j] ? 1u : 0u;
  return r;
}

struct Row {
  uint64_t hi, lo;  // (a << 32 | b), (c << 32 | d): sorted vertex ids
  uint64_t src;     // input row
};
}  // namespace

extern "C" uint64_t oracle_canonical(const uint32_t* tets, const uint32_t* adj, uint64_t m, uint32_t n,
                                     uint32_t* out_tets, uint32_t* out_adj) {
  const uint32_t inf = n + 4;
  std::vector<Row> rows;
  rows.reserve(m);
  for (uint64_t r = 0; r < m; ++r) {
    const uint32_t* v = tets + 4 * r;
    if (v[0] == inf || v[1] == inf || v[2] == inf || v[3] == inf) continue;
    std::array<uint32_t, 4> s = {v[0], v[1], v[2], v[3]};
    std::sort(s.begin(), s.end());
    rows.push_back(Row{(uint64_t(s[0]) << 32) | s[1], (uint64_t(s[2]) << 32) | s[3], r});
  }
  std::sort(rows.begin(), rows.end(),
            [](const Row& a, const Row& b) { return a.hi != b.hi ? a.hi < b.hi : a.lo < b.lo; });
  std::vector<int64_t> pos(m, -1);
  for (uint64_t i = 0; i < rows.size(); ++i) pos[rows[i].src] = int64_t(i);
  for (uint64_t i = 0; i < rows.size(); ++i) {
    const Row& R = rows[i];
    out_tets[4 * i + 0] = uint32_t(R.hi >> 32);
    out_tets[4 * i + 1] = uint32_t(R.hi);
    out_tets[4 * i + 2] = uint32_t(R.lo >> 32);
    out_tets[4 * i + 3] = uint32_t(R.lo);
    const uint32_t* v = tets + 4 * R.src;
    for (int j = 0; j < 4; ++j) {
      const uint32_t a = adj[4 * R.src + j];
      uint32_t val = NONE;
      if (a != NONE) {
        const uint64_t nb = a >> 5;
        const int nf = int(a & 3u);
        if (nb < m && pos[nb] >= 0) val = uint32_t((uint64_t(pos[nb]) << 5) | rank_in_row(tets + 4 * nb, nf));
      }
      out_adj[4 * i + rank_in_row(v, j)] = val;
    }
  }
  return rows.size();
}
