// Device verifier and canonicaliser of a triangulation in the reference's
// output format (src/types.rs:165-174: rows of 4 vertex ids, adjacency
// (tet << 5) | face, super vertices n..n+3, infinity vertex n+4).
//
// wtet_verify extends check_delaunay_quality (src/lib.rs:25-78), which only
// tests faces between two all-real tets, to the whole finite triangulation:
// every face between two tets without the infinity vertex -- faces with super
// vertices included, at the reference's super coordinates
// (src/gpu/mod.rs:151-158), which are exact in f32 -- gets the exact
// orient4d + SoS test; every finite tet gets the exact orient3d + SoS
// orientation test; every link is checked for symmetry and for sharing its
// face; faces with no finite neighbour are counted (the super tetrahedron's
// four faces in a complete output).  Locally Delaunay faces everywhere in a
// consistently oriented, face-to-face triangulation whose boundary is the
// super tetrahedron make it the Delaunay triangulation of the points plus the
// super vertices.
//
// wtet_canonicalize produces the canonical parity form used to compare two
// outputs byte for byte: tets without the infinity vertex, ids sorted in each
// row, rows sorted lexicographically, adjacency re-indexed to that order
// ((neighbour << 5) | sorted slot of the neighbour's opposite vertex, INVALID
// towards a missing or infinity neighbour).  Rows are counting-sorted by their
// smallest vertex, then ranked inside each bucket (one thread per row,
// comparing with the bucket's other rows: a bucket holds the tets whose
// smallest vertex is the same, ~7 on average).
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "devbuf.cuh"
#include "engine.cuh"
#include "exact.cuh"

namespace wtet {

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t cmp4(const uint4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

__device__ __forceinline__ void ld_pt(const float4* pts, uint32_t v, double* o) {
  const float4 q = pts[v];
  o[0] = q.x;
  o[1] = q.y;
  o[2] = q.z;
}

// Sorted copy of a row (5-comparator network).
__device__ __forceinline__ uint4 sorted4(uint4 v) {
  uint32_t a = v.x, b = v.y, c = v.z, d = v.w, t;
#define WTET_CS(x, y) \
  if (x > y) {        \
    t = x;            \
    x = y;            \
    y = t;            \
  }
  WTET_CS(a, b) WTET_CS(c, d) WTET_CS(a, c) WTET_CS(b, d) WTET_CS(b, c)
#undef WTET_CS
  return make_uint4(a, b, c, d);
}

// Slot of row slot j in the sorted row (rank of v[j] among the four ids).
__device__ __forceinline__ uint32_t rank_in_row(const uint4& v, int j) {
  const uint32_t x = cmp4(v, j);
  return uint32_t(v.x < x) + uint32_t(v.y < x) + uint32_t(v.z < x) + uint32_t(v.w < x);
}

__device__ __forceinline__ bool has(const uint4& v, uint32_t x) {
  return v.x == x || v.y == x || v.z == x || v.w == x;
}

struct VerifyCounts {
  unsigned long long finite, faces, violations, misoriented, broken, hull, bad_ids;
  uint32_t err;  // exact-arithmetic overflow
  uint32_t pad;
};

// Points 0..n-1 normalised, super vertices n..n+3 at the reference's
// coordinates (src/gpu/mod.rs:151-158).
__global__ void k_super_points(float4* pts, uint32_t n) {
  const float S[4][3] = {{-100.f, -100.f, -100.f}, {400.f, -100.f, -100.f}, {-100.f, 400.f, -100.f},
                         {-100.f, -100.f, 400.f}};
  const uint32_t k = threadIdx.x;
  if (k < 4) pts[n + k] = make_float4(S[k][0], S[k][1], S[k][2], 0.f);
}

__global__ void __launch_bounds__(128) k_verify(const float4* pts, uint32_t n, const uint4* tets, const uint4* adj,
                                                uint64_t m, VerifyCounts* out) {
  const uint32_t inf = n + 4;
  unsigned long long finite = 0, faces = 0, viol = 0, mis = 0, broken = 0, hull = 0, bad = 0;
  for (uint64_t ti = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; ti < m; ti += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 t = tets[ti];
    if (t.x > inf || t.y > inf || t.z > inf || t.w > inf) {
      ++bad;
      continue;
    }
    if (has(t, inf)) continue;
    ++finite;
    double P[4][3];
    ld_pt(pts, t.x, P[0]);
    ld_pt(pts, t.y, P[1]);
    ld_pt(pts, t.z, P[2]);
    ld_pt(pts, t.w, P[3]);
    // orient3d_sos == +1 (Shewchuk determinant < 0, src/phase2.rs:404-410)
    int o = ex::orient3d(P[0], P[1], P[2], P[3], &out->err);
    o = o != 0 ? (o < 0 ? 1 : -1)
               : ex::orient3d_sos_degenerate(P[0], P[1], P[2], P[3], t.x, t.y, t.z, t.w);
    if (o != 1) ++mis;
    const uint4 a = adj[ti];
    const uint4 ts = sorted4(t);
    for (int f = 0; f < 4; ++f) {
      const uint32_t packed = cmp4(a, f);
      if (packed == NONE) {
        ++hull;
        continue;
      }
      const uint64_t oti = packed >> 5;
      const int of = int(packed & 3u);
      if (oti >= m) {
        ++broken;
        continue;
      }
      const uint4 ot = tets[oti];
      if (cmp4(adj[oti], of) != ((uint32_t(ti) << 5) | uint32_t(f))) {
        ++broken;
        continue;
      }
      // the two tets share the face: same ids once the opposite vertices are
      // removed (compare the sorted rows with the opposite slot dropped)
      const uint32_t xa = cmp4(t, f), xb = cmp4(ot, of);
      const uint4 os = sorted4(ot);
      uint32_t fa[3], fb[3];
      int ka = 0, kb = 0;
      for (int k = 0; k < 4; ++k) {
        if (cmp4(ts, k) != xa && ka < 3) fa[ka++] = cmp4(ts, k);
        if (cmp4(os, k) != xb && kb < 3) fb[kb++] = cmp4(os, k);
      }
      if (ka != 3 || kb != 3 || fa[0] != fb[0] || fa[1] != fb[1] || fa[2] != fb[2] || xa == xb) {
        ++broken;
        continue;
      }
      if (has(ot, inf)) {
        ++hull;
        continue;
      }
      if (ti > oti) continue;  // each face once
      ++faces;
      double E[3];
      ld_pt(pts, xb, E);
      int s = ex::insphere(P[0], P[1], P[2], P[3], E, &out->err);
      if (s == 0)
        s = ex::orient4d_sos_degenerate(P[0], P[1], P[2], P[3], E, t.x, t.y, t.z, t.w, xb, &out->err);
      if (s < 0) ++viol;
    }
  }
  atomicAdd(&out->finite, finite);
  atomicAdd(&out->faces, faces);
  atomicAdd(&out->violations, viol);
  atomicAdd(&out->misoriented, mis);
  atomicAdd(&out->broken, broken);
  atomicAdd(&out->hull, hull);
  atomicAdd(&out->bad_ids, bad);
}

// ---- canonical form ----

// Finite rows: counted by their smallest vertex; infinity rows get perm NONE.
__global__ void k_canon_count(const uint4* tets, uint64_t m, uint32_t n, uint32_t* hist, uint32_t* perm,
                              uint32_t* bad) {
  const uint32_t inf = n + 4;
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < m; r += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 v = tets[r];
    perm[r] = NONE;
    if (v.x > inf || v.y > inf || v.z > inf || v.w > inf) {
      atomicOr(bad, 1u);
      continue;
    }
    if (has(v, inf)) continue;
    atomicAdd(&hist[sorted4(v).x], 1u);
  }
}

// Scatter into buckets (order inside a bucket is arbitrary; ranked next).
__global__ void k_canon_scatter(const uint4* tets, uint64_t m, uint32_t n, uint32_t* cursor, uint4* rows,
                                uint32_t* lead) {
  const uint32_t inf = n + 4;
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < m; r += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 v = tets[r];
    if (v.x > inf || v.y > inf || v.z > inf || v.w > inf || has(v, inf)) continue;
    const uint4 s = sorted4(v);
    const uint32_t i = atomicAdd(&cursor[s.x], 1u);
    rows[i] = make_uint4(s.y, s.z, s.w, uint32_t(r));
    lead[i] = s.x;
  }
}

__device__ __forceinline__ bool row_less(const uint4& a, const uint4& b) {
  if (a.x != b.x) return a.x < b.x;
  if (a.y != b.y) return a.y < b.y;
  if (a.z != b.z) return a.z < b.z;
  return a.w < b.w;  // duplicate rows (invalid input) keep a strict order by source row
}

// Final position of each row: bucket start + rank inside the bucket.
__global__ void k_canon_place(const uint4* rows, const uint32_t* lead, const uint32_t* bstart, uint64_t k,
                              uint4* out_t, uint32_t* perm, uint32_t* srcof) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < k; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 me = rows[i];
    const uint32_t a = lead[i];
    const uint32_t b0 = bstart[a], b1 = bstart[a + 1];
    uint32_t rank = 0;
    for (uint32_t j = b0; j < b1; ++j) rank += row_less(rows[j], me) ? 1u : 0u;
    const uint32_t dst = b0 + rank;
    out_t[dst] = make_uint4(a, me.x, me.y, me.z);
    perm[me.w] = dst;
    srcof[dst] = me.w;
  }
}

__global__ void k_canon_adj(const uint4* tets, const uint4* adj, uint64_t m, uint64_t k, const uint32_t* perm,
                            const uint32_t* srcof, uint4* out_a) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < k; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t r = srcof[i];
    const uint4 v = tets[r];
    const uint4 a = adj[r];
    uint4 o = make_uint4(NONE, NONE, NONE, NONE);
    for (int j = 0; j < 4; ++j) {
      const uint32_t x = cmp4(a, j);
      uint32_t val = NONE;
      if (x != NONE) {
        const uint64_t nb = x >> 5;
        if (nb < m && perm[nb] != NONE) val = (perm[nb] << 5) | rank_in_row(tets[nb], int(x & 3u));
      }
      const uint32_t s = rank_in_row(v, j);
      if (s == 0) o.x = val;
      else if (s == 1) o.y = val;
      else if (s == 2) o.z = val;
      else o.w = val;
    }
    out_a[i] = o;
  }
}

struct VerifyWorkspace {
  dev::DBuf<float4> pts;
  dev::DBuf<uint32_t> box, hist, cursor, lead, perm, srcof, bad;
  dev::DBuf<uint4> rows;
  dev::DBuf<VerifyCounts> cnt;
  std::vector<dev::DBuf<uint32_t>> scan_tmp;
};
thread_local VerifyWorkspace* tl_vws = nullptr;

VerifyWorkspace& vws() {
  if (!tl_vws) tl_vws = new VerifyWorkspace;
  return *tl_vws;
}

inline uint32_t grid_for(uint64_t n, uint32_t threads, uint32_t cap) {
  uint64_t b = (n + threads - 1) / threads;
  return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(b, cap)));
}

}  // namespace

void verify_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adj, uint64_t m,
                   wtet_verify_report* rep, cudaStream_t s) {
  using dev::ck;
  if (m >= (1ull << 27)) throw Error{WTET_ERR_ARG, "more tets than the (tet << 5) | face encoding can address"};
  if (n + 5 >= 0xFFFFFFFFull) throw Error{WTET_ERR_ARG, "too many points"};
  VerifyWorkspace& W = vws();
  W.pts.reserve(n + 4, "verify points");
  W.box.reserve(6, "verify box");
  W.cnt.reserve(1, "verify counters");
  normalize_points_device(d_xyz, n, W.pts.p, W.box.p, s);
  k_super_points<<<1, 32, 0, s>>>(W.pts.p, uint32_t(n));
  ck(cudaMemsetAsync(W.cnt.p, 0, sizeof(VerifyCounts), s), "memset");
  if (m)
    k_verify<<<grid_for(m, 128, 148 * 16), 128, 0, s>>>(W.pts.p, uint32_t(n), reinterpret_cast<const uint4*>(d_tets),
                                                       reinterpret_cast<const uint4*>(d_adj), m, W.cnt.p);
  ck(cudaGetLastError(), "verify kernels");
  VerifyCounts h{};
  ck(cudaMemcpyAsync(&h, W.cnt.p, sizeof h, cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "verify");
  if (h.err) throw Error{WTET_ERR_PRECISION, "exact arithmetic buffer overflow"};
  rep->finite_tets = h.finite;
  rep->faces_checked = h.faces;
  rep->violations = h.violations;
  rep->misoriented = h.misoriented;
  rep->broken_links = h.broken;
  rep->hull_faces = h.hull;
  rep->bad_vertex_ids = h.bad_ids;
}

uint64_t canonicalize_device(const uint32_t* d_tets, const uint32_t* d_adj, uint64_t m, uint64_t n,
                             uint32_t* d_out_t, uint32_t* d_out_a, cudaStream_t s) {
  using dev::ck;
  if (m >= (1ull << 27)) throw Error{WTET_ERR_ARG, "more tets than the (tet << 5) | face encoding can address"};
  if (n + 5 >= 0xFFFFFFFFull) throw Error{WTET_ERR_ARG, "too many points"};
  VerifyWorkspace& W = vws();
  const uint32_t nb = uint32_t(n + 5);  // buckets: every possible smallest vertex, + 1 for the scan's total
  W.hist.reserve(nb + 1, "canon hist");
  W.perm.reserve(std::max<uint64_t>(m, 1), "canon perm");
  W.rows.reserve(std::max<uint64_t>(m, 1), "canon rows");
  W.lead.reserve(std::max<uint64_t>(m, 1), "canon rows");
  W.srcof.reserve(std::max<uint64_t>(m, 1), "canon rows");
  W.bad.reserve(1, "canon flags");
  ck(cudaMemsetAsync(W.hist.p, 0, (nb + 1) * 4ull, s), "memset");
  ck(cudaMemsetAsync(W.bad.p, 0, 4, s), "memset");
  const uint4* T = reinterpret_cast<const uint4*>(d_tets);
  const uint4* A = reinterpret_cast<const uint4*>(d_adj);
  const uint32_t g = grid_for(m, 256, 148 * 32);
  if (m) k_canon_count<<<g, 256, 0, s>>>(T, m, uint32_t(n), W.hist.p, W.perm.p, W.bad.p);
  dev::scan_u32(W.hist.p, nb + 1, s, W.scan_tmp);  // exclusive: bucket starts, total at [nb]
  uint32_t k32 = 0, bad = 0;
  ck(cudaMemcpyAsync(&k32, W.hist.p + nb, 4, cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaMemcpyAsync(&bad, W.bad.p, 4, cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "canon count");
  if (bad) throw Error{WTET_ERR_ARG, "a tet refers to a vertex beyond the infinity vertex n+4"};
  const uint64_t k = k32;
  // each bucket's fill cursor starts at the bucket's start
  W.cursor.reserve(nb + 1, "canon cursor");
  ck(cudaMemcpyAsync(W.cursor.p, W.hist.p, (nb + 1) * 4ull, cudaMemcpyDeviceToDevice, s), "d2d");
  if (m) k_canon_scatter<<<g, 256, 0, s>>>(T, m, uint32_t(n), W.cursor.p, W.rows.p, W.lead.p);
  if (k) {
    const uint32_t gk = grid_for(k, 256, 148 * 32);
    k_canon_place<<<gk, 256, 0, s>>>(W.rows.p, W.lead.p, W.hist.p, k, reinterpret_cast<uint4*>(d_out_t), W.perm.p,
                                     W.srcof.p);
    k_canon_adj<<<gk, 256, 0, s>>>(T, A, m, k, W.perm.p, W.srcof.p, reinterpret_cast<uint4*>(d_out_a));
  }
  ck(cudaGetLastError(), "canonical kernels");
  ck(cudaStreamSynchronize(s), "canonical");
  return k;
}

void release_verify_workspace() {
  if (!tl_vws) return;
  VerifyWorkspace& w = *tl_vws;
  w.pts.release();
  w.box.release();
  w.hist.release();
  w.cursor.release();
  w.lead.release();
  w.perm.release();
  w.srcof.release();
  w.bad.release();
  w.rows.release();
  w.cnt.release();
  for (auto& b : w.scan_tmp) b.release();
  delete tl_vws;
  tl_vws = nullptr;
}

}  // namespace wtet
