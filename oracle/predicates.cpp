// Oracle (test infrastructure only): exact predicates and the reference's SoS
// cascades, restated in C++ from src/predicates.rs.
//
// Exact signs use an FP64 stage-A filter (Shewchuk 1997, error bounds
// (7+56e)e for orient3d and (16+224e)e for insphere, e = 2^-53) and otherwise
// evaluate the determinant exactly from the raw coordinates with expansion
// arithmetic (expansion.hpp), expanding the 4x4 / 5x5 determinants with a
// column of ones by cofactors.  The SoS cascades follow src/predicates.rs
// verbatim in their arithmetic, including the places where the reference uses
// plain double arithmetic (orient2d at :73-75, coordinate differences) and the
// lifted orient3d fast path with its own error bound (:390-435), so that the
// oracle reproduces the reference's decisions bit for bit.
#include "predicates.hpp"

#include <algorithm>
#include <cmath>
#include <vector>

#include "expansion.hpp"

namespace oracle {
namespace {

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
constexpr double kO3dBoundA = (7.0 + 56.0 * kEps) * kEps;
constexpr double kIspBoundA = (16.0 + 224.0 * kEps) * kEps;
// src/predicates.rs:426-427
constexpr double kO3dBoundLifted = (11.0 + 112.0 * kEps) * kEps;

// per thread: concurrent triangulations (the CPU reference arm) share nothing
thread_local PredStats g_stats{};

// 2-component expansion of a*b (increasing magnitude).
inline int prod2(double a, double b, double* h) {
  double x, y;
  two_product(a, b, x, y);
  h[0] = y;
  h[1] = x;
  return 2;
}

// p[u]*q[v] - q[u]*p[v]
inline int minor2(const double* p, const double* q, int u, int v, double* h) {
  double a[2], b[2];
  prod2(p[u], q[v], a);
  prod2(q[u], p[v], b);
  b[0] = -b[0];
  b[1] = -b[1];
  return exp_sum(2, a, 2, b, h);
}

// det[[p_u, p_v, 1], [q_u, q_v, 1], [r_u, r_v, 1]] = m(p,q) + m(q,r) + m(r,p)
inline int minor3(const double* p, const double* q, const double* r, int u, int v, double* h) {
  double m1[4], m2[4], m3[4], t[8];
  int l1 = minor2(p, q, u, v, m1);
  int l2 = minor2(q, r, u, v, m2);
  int l3 = minor2(r, p, u, v, m3);
  int lt = exp_sum(l1, m1, l2, m2, t);
  return exp_sum(lt, t, l3, m3, h);
}

// |p|^2 as an exact expansion (<= 6 components).
inline int lift(const double* p, double* h) {
  double a[2], b[2], c[2], t[4];
  prod2(p[0], p[0], a);
  prod2(p[1], p[1], b);
  prod2(p[2], p[2], c);
  int lt = exp_sum(2, a, 2, b, t);
  return exp_sum(lt, t, 2, c, h);
}

// det4 with columns (u, v, K, 1), K given per row as an expansion:
//   K_a M(b,c,d) - K_b M(a,c,d) + K_c M(a,b,d) - K_d M(a,b,c).
// Result compressed into h (capacity >= 1200).
int det4_k(const double* a, const double* b, const double* c, const double* d, int u, int v,
           const int* klen, const double (*K)[8], double* h) {
  const double* P[4] = {a, b, c, d};
  static const int others[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  double acc[1200], tmp[1200], m[16], pr[400], t1[400], t2[400];
  int alen = 0;
  for (int i = 0; i < 4; ++i) {
    int ml = minor3(P[others[i][0]], P[others[i][1]], P[others[i][2]], u, v, m);
    ml = exp_compress(ml, m, m);
    int pl = exp_mul(ml, m, klen[i], K[i], pr, t1, t2);
    if (i & 1) exp_negate(pl, pr);
    if (alen == 0) {
      for (int k = 0; k < pl; ++k) acc[k] = pr[k];
      alen = pl;
    } else {
      int nl = exp_sum(alen, acc, pl, pr, tmp);
      for (int k = 0; k < nl; ++k) acc[k] = tmp[k];
      alen = nl;
    }
  }
  return exp_compress(alen, acc, h);
}

// Exact D4 = det[[x,y,z,1]] rows a..d = Shewchuk orient3d(a,b,c,d).
int orient3d_exact(const double* a, const double* b, const double* c, const double* d, double* h) {
  int kl[4] = {1, 1, 1, 1};
  double K[4][8] = {{a[2]}, {b[2]}, {c[2]}, {d[2]}};
  return det4_k(a, b, c, d, 0, 1, kl, K, h);
}

}  // namespace

PredStats pred_stats() { return g_stats; }
void pred_stats_reset() { g_stats = PredStats{}; }

int orient3d_sign(const double* pa, const double* pb, const double* pc, const double* pd) {
  ++g_stats.o3d_calls;
  double adx = pa[0] - pd[0], bdx = pb[0] - pd[0], cdx = pc[0] - pd[0];
  double ady = pa[1] - pd[1], bdy = pb[1] - pd[1], cdy = pc[1] - pd[1];
  double adz = pa[2] - pd[2], bdz = pb[2] - pd[2], cdz = pc[2] - pd[2];
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
  double cdxady = cdx * ady, adxcdy = adx * cdy;
  double adxbdy = adx * bdy, bdxady = bdx * ady;
  double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
  double perm = (std::fabs(bdxcdy) + std::fabs(cdxbdy)) * std::fabs(adz) +
                (std::fabs(cdxady) + std::fabs(adxcdy)) * std::fabs(bdz) +
                (std::fabs(adxbdy) + std::fabs(bdxady)) * std::fabs(cdz);
  double err = kO3dBoundA * perm;
  if (det > err) return 1;
  if (-det > err) return -1;
  ++g_stats.o3d_exact;
  double h[1200];
  int n = orient3d_exact(pa, pb, pc, pd, h);
  return exp_sign(n, h);
}

int insphere_sign(const double* pa, const double* pb, const double* pc, const double* pd,
                  const double* pe) {
  ++g_stats.isp_calls;
  double aex = pa[0] - pe[0], bex = pb[0] - pe[0], cex = pc[0] - pe[0], dex = pd[0] - pe[0];
  double aey = pa[1] - pe[1], bey = pb[1] - pe[1], cey = pc[1] - pe[1], dey = pd[1] - pe[1];
  double aez = pa[2] - pe[2], bez = pb[2] - pe[2], cez = pc[2] - pe[2], dez = pd[2] - pe[2];
  double aexbey = aex * bey, bexaey = bex * aey, ab = aexbey - bexaey;
  double bexcey = bex * cey, cexbey = cex * bey, bc = bexcey - cexbey;
  double cexdey = cex * dey, dexcey = dex * cey, cd = cexdey - dexcey;
  double dexaey = dex * aey, aexdey = aex * dey, da = dexaey - aexdey;
  double aexcey = aex * cey, cexaey = cex * aey, ac = aexcey - cexaey;
  double bexdey = bex * dey, dexbey = dex * bey, bd = bexdey - dexbey;
  double abc = aez * bc - bez * ac + cez * ab;
  double bcd = bez * cd - cez * bd + dez * bc;
  double cda = cez * da + dez * ac + aez * cd;
  double dab = dez * ab + aez * bd + bez * da;
  double alift = aex * aex + aey * aey + aez * aez;
  double blift = bex * bex + bey * bey + bez * bez;
  double clift = cex * cex + cey * cey + cez * cez;
  double dlift = dex * dex + dey * dey + dez * dez;
  double det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd);
  double az = std::fabs(aez), bz = std::fabs(bez), cz = std::fabs(cez), dz = std::fabs(dez);
  double p_ab = std::fabs(aexbey) + std::fabs(bexaey);
  double p_bc = std::fabs(bexcey) + std::fabs(cexbey);
  double p_cd = std::fabs(cexdey) + std::fabs(dexcey);
  double p_da = std::fabs(dexaey) + std::fabs(aexdey);
  double p_ac = std::fabs(aexcey) + std::fabs(cexaey);
  double p_bd = std::fabs(bexdey) + std::fabs(dexbey);
  double perm = (p_cd * bz + p_bd * cz + p_bc * dz) * alift +
                (p_da * cz + p_ac * dz + p_cd * az) * blift +
                (p_ab * dz + p_bd * az + p_da * bz) * clift +
                (p_bc * az + p_ac * bz + p_ab * cz) * dlift;
  double err = kIspBoundA * perm;
  if (det > err) return 1;
  if (-det > err) return -1;
  ++g_stats.isp_exact;
  // Exact: D5 = -w_a D4(b,c,d,e) + w_b D4(a,c,d,e) - w_c D4(a,b,d,e) + w_d D4(a,b,c,e) - w_e D4(a,b,c,d)
  const double* P[5] = {pa, pb, pc, pd, pe};
  static const int others[5][4] = {{1, 2, 3, 4}, {0, 2, 3, 4}, {0, 1, 3, 4}, {0, 1, 2, 4}, {0, 1, 2, 3}};
  std::vector<double> acc, tmp, pr, t1, t2;
  double d4[1200], w[8];
  int alen = 0;
  for (int i = 0; i < 5; ++i) {
    int dl = orient3d_exact(P[others[i][0]], P[others[i][1]], P[others[i][2]], P[others[i][3]], d4);
    if (dl == 1 && d4[0] == 0.0) continue;
    int wl = lift(P[i], w);
    wl = exp_compress(wl, w, w);
    size_t cap = 2 * size_t(dl) * size_t(wl) + 8;
    pr.resize(cap);
    t1.resize(cap);
    t2.resize(cap);
    int pl = exp_mul(dl, d4, wl, w, pr.data(), t1.data(), t2.data());
    if ((i & 1) == 0) exp_negate(pl, pr.data());
    if (alen == 0) {
      acc.assign(pr.begin(), pr.begin() + pl);
      alen = pl;
    } else {
      tmp.resize(size_t(alen) + size_t(pl) + 8);
      int nl = exp_sum(alen, acc.data(), pl, pr.data(), tmp.data());
      acc.resize(size_t(nl) + 8);
      nl = exp_compress(nl, tmp.data(), acc.data());
      alen = nl;
    }
  }
  if (alen == 0) return 0;
  return exp_sign(alen, acc.data());
}

// ---- lifted sub-predicates used by the orient4d SoS cascade ----

int orient3d_lifted_sign(const double* a0, const double* b0, const double* c0, const double* d0,
                         int q0, int q1, int q2) {
  // Fast path, src/predicates.rs:395-432, on the permuted coordinates.
  double pa[3] = {a0[q0], a0[q1], a0[q2]};
  double pb[3] = {b0[q0], b0[q1], b0[q2]};
  double pc[3] = {c0[q0], c0[q1], c0[q2]};
  double pd[3] = {d0[q0], d0[q1], d0[q2]};
  double adx = pa[0] - pd[0], bdx = pb[0] - pd[0], cdx = pc[0] - pd[0];
  double ady = pa[1] - pd[1], bdy = pb[1] - pd[1], cdy = pc[1] - pd[1];
  double adzr = pa[2] - pd[2], bdzr = pb[2] - pd[2], cdzr = pc[2] - pd[2];
  double adz = adx * adx + ady * ady + adzr * adzr;
  double bdz = bdx * bdx + bdy * bdy + bdzr * bdzr;
  double cdz = cdx * cdx + cdy * cdy + cdzr * cdzr;
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy, cdxady = cdx * ady;
  double adxcdy = adx * cdy, adxbdy = adx * bdy, bdxady = bdx * ady;
  double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
  double perm = (std::fabs(bdxcdy) + std::fabs(cdxbdy)) * std::fabs(adz) +
                (std::fabs(cdxady) + std::fabs(adxcdy)) * std::fabs(bdz) +
                (std::fabs(adxbdy) + std::fabs(bdxady)) * std::fabs(cdz);
  double err = kO3dBoundLifted * perm;
  if (det > err || -det > err) return (det > 0.0) - (det < 0.0);
  // Exact: det[[u, v, |p|^2, 1]] rows a..d.
  int kl[4];
  double K[4][8];
  kl[0] = lift(pa, K[0]);
  kl[1] = lift(pb, K[1]);
  kl[2] = lift(pc, K[2]);
  kl[3] = lift(pd, K[3]);
  double h[1200];
  int n = det4_k(pa, pb, pc, pd, 0, 1, kl, K, h);
  return exp_sign(n, h);
}

int orient2d_lifted_sign(const double* a0, const double* b0, const double* c0, int q0) {
  // a_u (w_b - w_c) + b_u (w_c - w_a) + c_u (w_a - w_b), src/predicates.rs:260-290.
  double wa[8], wb[8], wc[8];
  int la = lift(a0, wa), lb = lift(b0, wb), lc = lift(c0, wc);
  const double* W[3] = {wa, wb, wc};
  const int L[3] = {la, lb, lc};
  const double U[3] = {a0[q0], b0[q0], c0[q0]};
  double acc[200], tmp[200], t[20];
  int alen = 0;
  // terms: U[i] * W[(i+1)%3] - U[i] * W[(i+2)%3]
  for (int i = 0; i < 3; ++i) {
    for (int s = 0; s < 2; ++s) {
      int j = (i + 1 + s) % 3;
      int tl = exp_scale(L[j], W[j], s == 0 ? U[i] : -U[i], t);
      if (alen == 0) {
        for (int k = 0; k < tl; ++k) acc[k] = t[k];
        alen = tl;
      } else {
        int nl = exp_sum(alen, acc, tl, t, tmp);
        for (int k = 0; k < nl; ++k) acc[k] = tmp[k];
        alen = nl;
      }
    }
  }
  return exp_sign(alen, acc);
}

int orient1d_lifted_sign(const double* a, const double* b) {
  double wa[8], wb[8], h[16];
  int la = lift(a, wa), lb = lift(b, wb);
  exp_negate(lb, wb);
  int n = exp_sum(la, wa, lb, wb, h);
  return exp_sign(n, h);
}

namespace {

// Plain double orient2d of src/predicates.rs:73-75 on coordinates (u, v).
inline double orient2d_plain(const double* a, const double* b, const double* c, int u, int v) {
  return (a[u] - c[u]) * (b[v] - c[v]) - (a[v] - c[v]) * (b[u] - c[u]);
}

// Sort up to 5 (index, point) pairs by index; returns the permutation parity.
inline int sort_by_index(int n, uint32_t* idx, const double** pts) {
  int parity = 0;
  for (int i = 1; i < n; ++i) {
    for (int j = i; j > 0 && idx[j] < idx[j - 1]; --j) {
      std::swap(idx[j], idx[j - 1]);
      std::swap(pts[j], pts[j - 1]);
      parity ^= 1;
    }
  }
  return parity;
}

// One level of the orient4d SoS cascade: the term's kind, the sorted points it
// uses, the coordinate permutation and whether its sign is flipped.
enum Kind : uint8_t { kO3, kO3L, kO2, kO2L, kO1, kO1L, kConst };
struct Level {
  Kind kind;
  uint8_t p[4];
  uint8_t perm[3];
  bool flip;
};

// The 49 levels of src/predicates.rs:513-651 with the flips of :662-667.
constexpr Level kCascade4[49] = {
    {kO3, {1, 2, 3, 4}, {0, 1, 2}, true},     // 1
    {kO3L, {1, 2, 3, 4}, {0, 1, 2}, false},   // 2
    {kO3L, {1, 2, 3, 4}, {0, 2, 1}, true},    // 3
    {kO3L, {1, 2, 3, 4}, {1, 2, 0}, false},   // 4
    {kO3, {0, 2, 3, 4}, {0, 1, 2}, false},    // 5
    {kO2, {2, 3, 4}, {0, 1, 2}, false},       // 6
    {kO2, {2, 3, 4}, {0, 2, 1}, true},        // 7
    {kO2, {2, 3, 4}, {1, 2, 0}, false},       // 8
    {kO3L, {0, 2, 3, 4}, {0, 1, 2}, true},    // 9
    {kO2L, {2, 3, 4}, {0, 1, 2}, false},      // 10
    {kO2L, {2, 3, 4}, {1, 0, 2}, true},       // 11
    {kO3L, {0, 2, 3, 4}, {0, 2, 1}, false},   // 12
    {kO2L, {2, 3, 4}, {2, 0, 1}, false},      // 13
    {kO3L, {0, 2, 3, 4}, {1, 2, 0}, true},    // 14
    {kO3, {0, 1, 3, 4}, {0, 1, 2}, true},     // 15
    {kO2, {1, 3, 4}, {0, 1, 2}, true},        // 16
    {kO2, {1, 3, 4}, {0, 2, 1}, false},       // 17
    {kO2, {1, 3, 4}, {1, 2, 0}, true},        // 18
    {kO2, {0, 3, 4}, {0, 1, 2}, false},       // 19
    {kO1, {3, 4}, {0, 1, 2}, true},           // 20
    {kO1, {3, 4}, {1, 0, 2}, false},          // 21
    {kO2, {0, 3, 4}, {0, 2, 1}, true},        // 22
    {kO1, {3, 4}, {2, 0, 1}, true},           // 23
    {kO2, {0, 3, 4}, {1, 2, 0}, false},       // 24
    {kO3L, {0, 1, 3, 4}, {0, 1, 2}, false},   // 25
    {kO2L, {1, 3, 4}, {0, 1, 2}, true},       // 26
    {kO2L, {1, 3, 4}, {1, 0, 2}, false},      // 27
    {kO2L, {0, 3, 4}, {0, 1, 2}, false},      // 28
    {kO1L, {3, 4}, {0, 1, 2}, false},         // 29
    {kO2L, {0, 3, 4}, {1, 0, 2}, true},       // 30
    {kO3L, {0, 1, 3, 4}, {0, 2, 1}, true},    // 31
    {kO2L, {1, 3, 4}, {2, 0, 1}, true},       // 32
    {kO2L, {0, 3, 4}, {2, 0, 1}, false},      // 33
    {kO3L, {0, 1, 3, 4}, {1, 2, 0}, false},   // 34
    {kO3, {0, 1, 2, 4}, {0, 1, 2}, false},    // 35
    {kO2, {1, 2, 4}, {0, 1, 2}, false},       // 36
    {kO2, {1, 2, 4}, {0, 2, 1}, true},        // 37
    {kO2, {1, 2, 4}, {1, 2, 0}, false},       // 38
    {kO2, {0, 2, 4}, {0, 1, 2}, true},        // 39
    {kO1, {2, 4}, {0, 1, 2}, false},          // 40
    {kO1, {2, 4}, {1, 0, 2}, true},           // 41
    {kO2, {0, 2, 4}, {0, 2, 1}, false},       // 42
    {kO1, {2, 4}, {2, 0, 1}, false},          // 43
    {kO2, {0, 2, 4}, {1, 2, 0}, true},        // 44
    {kO2, {0, 1, 4}, {0, 1, 2}, false},       // 45
    {kO1, {1, 4}, {0, 1, 2}, true},           // 46
    {kO1, {1, 4}, {1, 0, 2}, false},          // 47
    {kO1, {0, 4}, {0, 1, 2}, false},          // 48
    {kConst, {0, 0, 0, 0}, {0, 1, 2}, false}, // 49
};

int eval_level(const Level& L, const double* const* ip) {
  const double* a = ip[L.p[0]];
  const double* b = ip[L.p[1]];
  const double* c = ip[L.p[2]];
  const double* d = ip[L.p[3]];
  switch (L.kind) {
    case kO3: return orient3d_sign(a, b, c, d);
    case kO3L: return orient3d_lifted_sign(a, b, c, d, L.perm[0], L.perm[1], L.perm[2]);
    case kO2: {
      double v = orient2d_plain(a, b, c, L.perm[0], L.perm[1]);
      return (v > 0.0) - (v < 0.0);
    }
    case kO2L: return orient2d_lifted_sign(a, b, c, L.perm[0]);
    case kO1: {
      double v = a[L.perm[0]] - b[L.perm[0]];
      return (v > 0.0) - (v < 0.0);
    }
    case kO1L: return orient1d_lifted_sign(a, b);
    default: return 1;
  }
}

}  // namespace

int orient3d_sos(const double* a, const double* b, const double* c, const double* d, uint32_t ia,
                 uint32_t ib, uint32_t ic, uint32_t id) {
  int s = orient3d_sign(a, b, c, d);
  if (s != 0) return s < 0 ? 1 : -1;
  ++g_stats.o3d_sos;
  uint32_t v[4] = {ia, ib, ic, id};
  const double* p[4] = {a, b, c, d};
  int parity = sort_by_index(4, v, p);
  // src/predicates.rs:140-204
  double r = 0.0;
  int depth = 0;
  for (; depth < 14; ++depth) {
    switch (depth) {
      case 0: r = orient2d_plain(p[1], p[2], p[3], 0, 1); break;
      case 1: r = orient2d_plain(p[1], p[2], p[3], 0, 2); break;
      case 2: r = orient2d_plain(p[1], p[2], p[3], 1, 2); break;
      case 3: r = orient2d_plain(p[0], p[2], p[3], 0, 1); break;
      case 4: r = p[2][0] - p[3][0]; break;
      case 5: r = p[2][1] - p[3][1]; break;
      case 6: r = orient2d_plain(p[0], p[2], p[3], 0, 2); break;
      case 7: r = p[2][2] - p[3][2]; break;
      case 8: r = orient2d_plain(p[0], p[2], p[3], 1, 2); break;
      case 9: r = orient2d_plain(p[0], p[1], p[3], 0, 1); break;
      case 10: r = p[1][0] - p[3][0]; break;
      case 11: r = p[1][1] - p[3][1]; break;
      case 12: r = p[0][0] - p[3][0]; break;
      default: r = 1.0; break;
    }
    if (r != 0.0) break;
  }
  int sg = (r > 0.0) - (r < 0.0);
  if (depth == 1 || depth == 3 || depth == 5 || depth == 8 || depth == 10) sg = -sg;
  if (parity) sg = -sg;
  return sg < 0 ? 1 : -1;
}

int orient4d_sos(const double* a, const double* b, const double* c, const double* d,
                 const double* e, uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id,
                 uint32_t ie) {
  int s = insphere_sign(a, b, c, d, e);
  if (s != 0) return s;
  ++g_stats.isp_sos;
  uint32_t v[5] = {ia, ib, ic, id, ie};
  const double* p[5] = {a, b, c, d, e};
  int parity = sort_by_index(5, v, p);
  int sg = 0;
  for (int k = 0; k < 49; ++k) {
    sg = eval_level(kCascade4[k], p);
    if (sg != 0) {
      if (kCascade4[k].flip) sg = -sg;
      break;
    }
  }
  if (parity) sg = -sg;
  return sg;
}

}  // namespace oracle
