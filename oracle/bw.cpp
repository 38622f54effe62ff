// Oracle (test infrastructure only): sequential Bowyer-Watson Delaunay
// triangulation with exact predicates and SoS, plus the reference's small
// deterministic helpers (normalisation, Morton codes, stratified order) and
// validators.  Restates:
//   src/lib.rs:313-337            normalize_points
//   src/lib.rs:25-78              check_delaunay_quality
//   src/gpu/mod.rs:147-158        vertex numbering and super-tet coordinates
//   src/phase2.rs:383-606         full_bw_reconstruction (cavity = tets with
//                                 orient4d < 0, new tets joined to the point)
//   src/morton.rs:22-80           Morton codes
//   src/gpu/mod.rs:422-460,533-600 Morton order, initial stride, stratified order
// The reference seeds each cavity with a linear scan over all tets
// (src/phase2.rs:424-440); this restatement locates the point with a visibility
// walk instead.  The SoS Delaunay triangulation is unique, so the output is the
// same tet set.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "oracle.h"
#include "predicates.hpp"

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;
thread_local std::string g_err;

struct Bnd {
  uint32_t c;      // cavity tet
  int f;           // its face on the cavity boundary
  uint32_t outer;  // encoded neighbour across that face, or NONE
};
struct Half {
  uint32_t a, b;   // boundary edge (sorted)
  uint32_t j;      // new tet
  int k;           // its face through p and the edge
};

struct Mesh {
  std::vector<double> P;  // xyz of n + 4 vertices
  uint32_t n = 0;         // real points
  std::vector<std::array<uint32_t, 4>> V;
  std::vector<std::array<uint32_t, 4>> A;  // (t << 2) | f, or NONE
  std::vector<uint32_t> freelist;
  std::vector<uint32_t> mark;  // stamp: s = in cavity, s + 1 = tested outside
  uint32_t stamp = 0;
  oracle_stats st{};
  std::vector<uint32_t> cav, slot;
  std::vector<Bnd> bnd;
  std::vector<Half> pend;
  std::vector<std::array<uint32_t, 4>> nv;

  const double* pt(uint32_t v) const { return &P[3 * size_t(v)]; }

  // p is beyond face f of t: replacing vertex f by p flips the orientation.
  bool beyond(uint32_t t, int f, uint32_t p) const {
    std::array<uint32_t, 4> w = V[t];
    w[f] = p;
    return oracle::orient3d_sos(pt(w[0]), pt(w[1]), pt(w[2]), pt(w[3]), w[0], w[1], w[2], w[3]) == -1;
  }
  bool in_sphere(uint32_t t, uint32_t p) const {
    const auto& w = V[t];
    return oracle::orient4d_sos(pt(w[0]), pt(w[1]), pt(w[2]), pt(w[3]), pt(p), w[0], w[1], w[2], w[3],
                                p) == -1;
  }

  bool locate(uint32_t p, uint32_t& t) {
    int entry = -1;
    for (uint64_t step = 0; step < 100000000ull; ++step) {
      ++st.walk_steps;
      int moved = -1;
      for (int i = 0; i < 4; ++i) {
        int f = (i + int(step)) & 3;
        if (f == entry) continue;
        if (beyond(t, f, p)) { moved = f; break; }
      }
      if (moved < 0) return true;
      uint32_t nb = A[t][moved];
      if (nb == NONE) { g_err = "walk left the super tetrahedron"; return false; }
      t = nb >> 2;
      entry = int(nb & 3);
    }
    g_err = "walk did not terminate";
    return false;
  }

  uint32_t alloc_slot() {
    if (!freelist.empty()) { uint32_t s = freelist.back(); freelist.pop_back(); return s; }
    V.push_back({NONE, NONE, NONE, NONE});
    A.push_back({NONE, NONE, NONE, NONE});
    mark.push_back(0);
    return uint32_t(V.size() - 1);
  }

  // Inserts p; t is the located tet on entry and a new tet of p on return.
  bool insert(uint32_t p, uint32_t& t) {
    stamp += 2;
    if (stamp < 2) { std::fill(mark.begin(), mark.end(), 0u); stamp = 2; }
    const uint32_t in_mark = stamp, out_mark = stamp + 1;
    if (!in_sphere(t, p)) { g_err = "containing tet does not hold the point in its circumsphere"; return false; }
    cav.clear();
    cav.push_back(t);
    mark[t] = in_mark;
    bnd.clear();
    for (size_t i = 0; i < cav.size(); ++i) {
      uint32_t c = cav[i];
      for (int f = 0; f < 4; ++f) {
        uint32_t nb = A[c][f];
        if (nb == NONE) { bnd.push_back({c, f, NONE}); continue; }
        uint32_t nt = nb >> 2;
        if (mark[nt] == in_mark) continue;
        if (mark[nt] != out_mark) {
          if (in_sphere(nt, p)) { mark[nt] = in_mark; cav.push_back(nt); continue; }
          mark[nt] = out_mark;
        }
        bnd.push_back({c, f, nb});
      }
    }
    const size_t K = cav.size(), F = bnd.size();
    st.cavity_tets += K;
    st.boundary_faces += F;
    st.max_cavity = std::max<uint32_t>(st.max_cavity, uint32_t(K));
    st.max_boundary = std::max<uint32_t>(st.max_boundary, uint32_t(F));
    {
      int b = 0;
      while (b < 15 && (size_t(2) << b) <= K) ++b;
      ++st.cavity_hist[b];
    }
    // New tets: the cavity tet with the boundary face's opposite vertex replaced by p.
    nv.resize(F);
    for (size_t j = 0; j < F; ++j) { nv[j] = V[bnd[j].c]; nv[j][bnd[j].f] = p; }
    slot.resize(F);
    for (size_t j = 0; j < F; ++j) slot[j] = (j < K) ? cav[j] : alloc_slot();
    for (size_t j = F; j < K; ++j) {
      V[cav[j]] = {NONE, NONE, NONE, NONE};
      A[cav[j]] = {NONE, NONE, NONE, NONE};
      freelist.push_back(cav[j]);
    }
    for (size_t j = 0; j < F; ++j) {
      uint32_t s = slot[j];
      V[s] = nv[j];
      A[s] = {NONE, NONE, NONE, NONE};
      mark[s] = 0;
      A[s][bnd[j].f] = bnd[j].outer;
      if (bnd[j].outer != NONE) A[bnd[j].outer >> 2][bnd[j].outer & 3] = (s << 2) | uint32_t(bnd[j].f);
    }
    // Faces through p pair up across the boundary edges.
    pend.clear();
    for (size_t j = 0; j < F; ++j) {
      int fp = bnd[j].f;
      for (int k = 0; k < 4; ++k) {
        if (k == fp) continue;
        uint32_t e[2];
        int ne = 0;
        for (int q = 0; q < 4; ++q)
          if (q != k && q != fp) e[ne++] = nv[j][q];
        uint32_t a = std::min(e[0], e[1]), b = std::max(e[0], e[1]);
        bool found = false;
        for (size_t q = 0; q < pend.size(); ++q) {
          if (pend[q].a == a && pend[q].b == b) {
            uint32_t s0 = slot[j], s1 = slot[pend[q].j];
            A[s0][k] = (s1 << 2) | uint32_t(pend[q].k);
            A[s1][pend[q].k] = (s0 << 2) | uint32_t(k);
            pend[q] = pend.back();
            pend.pop_back();
            found = true;
            break;
          }
        }
        if (!found) pend.push_back({a, b, uint32_t(j), k});
      }
    }
    if (!pend.empty()) { g_err = "cavity boundary is not a closed surface"; return false; }
    t = slot[0];
    return true;
  }
};

// Super-tet vertex coordinates, src/gpu/mod.rs:151-158 (f32 values).
const float kSuper[4][3] = {{-100.f, -100.f, -100.f}, {400.f, -100.f, -100.f},
                            {-100.f, 400.f, -100.f}, {-100.f, -100.f, 400.f}};

void build_points(const float* norm, uint32_t n, std::vector<double>& P) {
  P.resize(3 * size_t(n + 4));
  for (size_t i = 0; i < 3 * size_t(n); ++i) P[i] = double(norm[i]);
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) P[3 * size_t(n + k) + c] = double(kSuper[k][c]);
}

struct DTHandle {
  std::vector<uint32_t> tets, adj, failed;
};

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

void oracle_normalize(const float* xyz, uint64_t n, float* out, float* min3, float* scale) {
  float mn[3] = {3.40282347e38f, 3.40282347e38f, 3.40282347e38f};
  float mx[3] = {-3.40282347e38f, -3.40282347e38f, -3.40282347e38f};
  for (uint64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      float v = xyz[3 * i + c];
      // Rust f32::min/max ignore NaN the same way: keep the non-NaN operand.
      if (v < mn[c] || std::isnan(mn[c])) mn[c] = std::isnan(v) ? mn[c] : v;
      if (v > mx[c] || std::isnan(mx[c])) mx[c] = std::isnan(v) ? mx[c] : v;
    }
  float ext[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
  float s = std::max(std::max(std::max(ext[0], ext[1]), ext[2]), 1e-10f);
  for (uint64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) out[3 * i + c] = (xyz[3 * i + c] - mn[c]) / s;
  if (min3) for (int c = 0; c < 3; ++c) min3[c] = mn[c];
  if (scale) *scale = s;
}

uint32_t oracle_expand_bits(uint32_t v) {
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

uint32_t oracle_interleave_bits(uint32_t x, uint32_t y, uint32_t z) {
  return (oracle_expand_bits(z) << 2) | (oracle_expand_bits(y) << 1) | oracle_expand_bits(x);
}

static inline float clamp01(float v) { return v < 0.f ? 0.f : (v > 1.f ? 1.f : v); }

uint32_t oracle_morton_code(const float* p, const float* mn, const float* mx) {
  uint32_t q[3];
  for (int c = 0; c < 3; ++c) {
    float nrm = clamp01((p[c] - mn[c]) / (mx[c] - mn[c]));
    float s = nrm * 1023.0f;
    q[c] = s >= 4294967295.0f ? 0xFFFFFFFFu : (s > 0.f ? uint32_t(s) : 0u);  // Rust `as u32` saturates
  }
  return oracle_interleave_bits(q[0], q[1], q[2]);
}

void oracle_morton_order(const float* xyz, uint64_t n, uint32_t* mapping) {
  float mn[3] = {3.40282347e38f, 3.40282347e38f, 3.40282347e38f};
  float mx[3] = {-3.40282347e38f, -3.40282347e38f, -3.40282347e38f};
  for (uint64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      mn[c] = std::min(mn[c], xyz[3 * i + c]);
      mx[c] = std::max(mx[c], xyz[3 * i + c]);
    }
  std::vector<uint32_t> key(n);
  for (uint64_t i = 0; i < n; ++i) key[i] = oracle_morton_code(&xyz[3 * i], mn, mx);
  std::vector<uint32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
  std::memcpy(mapping, idx.data(), n * sizeof(uint32_t));
}

uint64_t oracle_initial_stride(uint64_t n) {
  double sq = std::sqrt(double(n));
  double scaled = n > 100000 ? sq * 2.0 : sq;
  double stride = std::min(std::max(scaled, 64.0), 16384.0);
  double lg = std::ceil(std::log2(stride));
  return uint64_t(std::pow(2.0, lg));
}

void oracle_strided_order(uint64_t n, uint64_t stride, uint32_t* order) {
  std::vector<char> done(n, 0);
  uint64_t k = 0;
  for (uint64_t s = stride; s >= 1; s /= 2) {
    for (uint64_t i = 0; i < n; i += s)
      if (!done[i]) { order[k++] = uint32_t(i); done[i] = 1; }
  }
}

int oracle_orient3d(const double* a, const double* b, const double* c, const double* d) {
  return oracle::orient3d_sign(a, b, c, d);
}
int oracle_insphere(const double* a, const double* b, const double* c, const double* d, const double* e) {
  return oracle::insphere_sign(a, b, c, d, e);
}
int oracle_orient3d_sos(const double* a, const double* b, const double* c, const double* d, uint32_t ia,
                        uint32_t ib, uint32_t ic, uint32_t id) {
  return oracle::orient3d_sos(a, b, c, d, ia, ib, ic, id);
}
int oracle_orient4d(const double* a, const double* b, const double* c, const double* d, const double* e,
                    uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id, uint32_t ie) {
  return oracle::orient4d_sos(a, b, c, d, e, ia, ib, ic, id, ie);
}
int oracle_orient3d_lifted(const double* a, const double* b, const double* c, const double* d, int p0,
                           int p1, int p2) {
  return oracle::orient3d_lifted_sign(a, b, c, d, p0, p1, p2);
}
int oracle_orient2d_lifted(const double* a, const double* b, const double* c, int p0) {
  return oracle::orient2d_lifted_sign(a, b, c, p0);
}
int oracle_orient1d_lifted(const double* a, const double* b) { return oracle::orient1d_lifted_sign(a, b); }

void* oracle_dt_run(const float* xyz, uint64_t n64, int order_mode, oracle_stats* stats) {
  g_err.clear();
  if (n64 < 4 || n64 > 0x7FFFFFF0ull) { g_err = "need 4 <= n < 2^31 points"; return nullptr; }
  const uint32_t n = uint32_t(n64);
  std::vector<float> norm(3 * size_t(n));
  oracle_normalize(xyz, n, norm.data(), nullptr, nullptr);
  oracle::pred_stats_reset();
  Mesh m;
  m.n = n;
  build_points(norm.data(), n, m.P);
  // Initial super tet oriented with orient3d_sos > 0 (src/phase2.rs:404-410).
  uint32_t s0 = n, s1 = n + 1, s2 = n + 2, s3 = n + 3;
  int o = oracle::orient3d_sos(m.pt(s0), m.pt(s1), m.pt(s2), m.pt(s3), s0, s1, s2, s3);
  m.V.push_back(o > 0 ? std::array<uint32_t, 4>{s0, s1, s2, s3} : std::array<uint32_t, 4>{s1, s0, s2, s3});
  m.A.push_back({NONE, NONE, NONE, NONE});
  m.mark.push_back(0);
  std::vector<uint32_t> order(n);
  if (order_mode == 1) {
    std::vector<uint32_t> mort(n), strided(n);
    oracle_morton_order(norm.data(), n, mort.data());
    oracle_strided_order(n, oracle_initial_stride(n), strided.data());
    for (uint32_t i = 0; i < n; ++i) order[i] = mort[strided[i]];
  } else {
    std::iota(order.begin(), order.end(), 0u);
  }
  // Exact duplicates of the normalised coordinates: the lowest index is
  // triangulated, later copies are reported as failed vertices.
  std::vector<char> dup(n, 0);
  {
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    auto key = [&](uint32_t i) {
      uint32_t b[3];
      std::memcpy(b, &norm[3 * size_t(i)], 12);
      return std::array<uint32_t, 3>{b[0], b[1], b[2]};
    };
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return key(a) < key(b); });
    for (uint32_t k = 1; k < n; ++k)
      if (key(idx[k]) == key(idx[k - 1])) dup[idx[k]] = 1;  // stable: earlier index kept
  }
  uint32_t t = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t p = order[i];
    if (dup[p]) continue;
    if (!m.locate(p, t)) return nullptr;
    if (!m.insert(p, t)) return nullptr;
  }
  auto* h = new DTHandle;
  for (uint32_t i = 0; i < n; ++i)
    if (dup[i]) h->failed.push_back(i);
  std::vector<uint32_t> remap(m.V.size(), NONE);
  uint32_t cnt = 0;
  for (size_t i = 0; i < m.V.size(); ++i)
    if (m.V[i][0] != NONE) remap[i] = cnt++;
  h->tets.resize(4 * size_t(cnt));
  h->adj.resize(4 * size_t(cnt));
  for (size_t i = 0; i < m.V.size(); ++i) {
    if (remap[i] == NONE) continue;
    size_t o4 = 4 * size_t(remap[i]);
    for (int k = 0; k < 4; ++k) {
      h->tets[o4 + k] = m.V[i][k];
      uint32_t a = m.A[i][k];
      h->adj[o4 + k] = (a == NONE) ? NONE : ((remap[a >> 2] << 5) | (a & 3));
    }
  }
  if (stats) {
    *stats = m.st;
    stats->num_tets = cnt;
    auto ps = oracle::pred_stats();
    stats->o3d_exact = ps.o3d_exact;
    stats->o3d_sos = ps.o3d_sos;
    stats->isp_exact = ps.isp_exact;
    stats->isp_sos = ps.isp_sos;
  }
  return h;
}

uint64_t oracle_dt_num_tets(void* h) { return static_cast<DTHandle*>(h)->tets.size() / 4; }
uint64_t oracle_dt_num_failed(void* h) { return static_cast<DTHandle*>(h)->failed.size(); }
void oracle_dt_copy_failed(void* h, uint32_t* out) {
  auto* d = static_cast<DTHandle*>(h);
  if (out) std::memcpy(out, d->failed.data(), d->failed.size() * 4);
}
void oracle_dt_copy(void* h, uint32_t* tets, uint32_t* adj) {
  auto* d = static_cast<DTHandle*>(h);
  if (tets) std::memcpy(tets, d->tets.data(), d->tets.size() * 4);
  if (adj) std::memcpy(adj, d->adj.data(), d->adj.size() * 4);
}
void oracle_dt_free(void* h) { delete static_cast<DTHandle*>(h); }

int64_t oracle_check_delaunay_quality(const float* xyz, uint64_t n, const uint32_t* tets, const uint32_t* adj,
                                      uint64_t m) {
  std::vector<float> norm(3 * n);
  oracle_normalize(xyz, n, norm.data(), nullptr, nullptr);
  std::vector<double> P(3 * n);
  for (size_t i = 0; i < 3 * n; ++i) P[i] = norm[i];
  int64_t viol = 0;
  for (uint64_t ti = 0; ti < m; ++ti) {
    const uint32_t* t = &tets[4 * ti];
    if (t[0] >= n || t[1] >= n || t[2] >= n || t[3] >= n) continue;
    for (int f = 0; f < 4; ++f) {
      uint32_t packed = adj[4 * ti + f];
      if (packed == NONE) continue;
      uint64_t oti = packed >> 5, of = packed & 3;
      if (ti >= oti) continue;
      if (oti >= m) return -1;
      const uint32_t* o = &tets[4 * oti];
      if (o[0] >= n || o[1] >= n || o[2] >= n || o[3] >= n) continue;
      uint32_t vb = o[of];
      if (oracle::orient4d_sos(&P[3 * t[0]], &P[3 * t[1]], &P[3 * t[2]], &P[3 * t[3]], &P[3 * vb], t[0], t[1],
                               t[2], t[3], vb) < 0)
        ++viol;
    }
  }
  return viol;
}

int64_t oracle_check_local_delaunay(const float* xyz, uint64_t n, const uint32_t* tets, const uint32_t* adj,
                                    uint64_t m) {
  std::vector<float> norm(3 * n);
  oracle_normalize(xyz, n, norm.data(), nullptr, nullptr);
  std::vector<double> P;
  build_points(norm.data(), uint32_t(n), P);
  const uint64_t inf = n + 4;
  int64_t viol = 0;
  for (uint64_t ti = 0; ti < m; ++ti) {
    const uint32_t* t = &tets[4 * ti];
    bool has_inf = false;
    for (int k = 0; k < 4; ++k) {
      if (t[k] == inf) has_inf = true;
      else if (t[k] > inf) return -1;
    }
    if (has_inf) continue;
    for (int f = 0; f < 4; ++f) {
      uint32_t packed = adj[4 * ti + f];
      if (packed == NONE) continue;
      uint64_t oti = packed >> 5, of = packed & 3;
      if (oti >= m) return -1;
      const uint32_t* o = &tets[4 * oti];
      uint32_t vb = o[of];
      if (vb == inf) continue;
      if (ti >= oti) continue;
      if (oracle::orient4d_sos(&P[3 * t[0]], &P[3 * t[1]], &P[3 * t[2]], &P[3 * t[3]], &P[3 * vb], t[0], t[1],
                               t[2], t[3], vb) < 0)
        ++viol;
    }
  }
  return viol;
}

int64_t oracle_check_orientation(const float* xyz, uint64_t n, const uint32_t* tets, uint64_t m) {
  std::vector<float> norm(3 * n);
  oracle_normalize(xyz, n, norm.data(), nullptr, nullptr);
  std::vector<double> P;
  build_points(norm.data(), uint32_t(n), P);
  const uint64_t inf = n + 4;
  int64_t bad = 0;
  for (uint64_t ti = 0; ti < m; ++ti) {
    const uint32_t* t = &tets[4 * ti];
    if (t[0] == inf || t[1] == inf || t[2] == inf || t[3] == inf) continue;
    if (t[0] > inf || t[1] > inf || t[2] > inf || t[3] > inf) return -1;
    if (oracle::orient3d_sos(&P[3 * t[0]], &P[3 * t[1]], &P[3 * t[2]], &P[3 * t[3]], t[0], t[1], t[2], t[3]) != 1)
      ++bad;
  }
  return bad;
}

}  // extern "C"
