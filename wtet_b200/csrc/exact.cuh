// Exact geometric predicates on the device: an FP64 static filter, an FP64
// expansion-arithmetic exact stage built from two-sum / two-product, then
// Simulation of Simplicity with the reference's cascades.
//
//   orient3d / insphere signs   src/predicates.rs:14-21 (Shewchuk semantics)
//   orient3d_sos                src/predicates.rs:106-208
//   orient4d (insphere + SoS)   src/predicates.rs:450-675
//
// An FP32 stage may run ahead of the FP64 filter (insphere_f32 /
// orient3d_f32): the same determinant and permanent in single precision with
// Shewchuk's stage-A bound for unit roundoff 2^-24.  Those bounds hold for any
// IEEE precision as long as nothing underflows, so the stage answers only when
// the permanent is far above the smallest normal float (and the values are
// finite); it returns 0 -- "not certain" -- otherwise, and the FP64 filter,
// the exact stage and SoS decide as before.  It never changes a sign.
//
// Coordinates are f32 values widened to f64.  The exact stage evaluates the
// determinants from raw coordinates (4x4 / 5x5 with a column of ones, expanded
// by cofactors), so it needs no exact coordinate differences.  The SoS
// cascades reproduce the reference's arithmetic operation by operation,
// including its plain-double orient2d and coordinate differences and its own
// filtered lifted orient3d; every product and sum is a separately rounded
// intrinsic, as in the reference, whatever the translation unit's
// contraction setting.
#pragma once
#include <cstdint>

namespace wtet {
namespace ex {
// Internal linkage: every translation unit of the library gets its own copy.
namespace {

// Error flag bit raised when an expansion would outgrow its fixed buffer.
constexpr uint32_t kErrPrecision = 1u << 4;

struct ErrSink {
  uint32_t* flags;
};

__device__ __forceinline__ void raise_precision(uint32_t* flags) {
  if (flags) atomicOr(flags, kErrPrecision);
}

// Every FP64 operation of this file is a separately rounded intrinsic
// (__dadd_rn, __dsub_rn, __dmul_rn), which the compiler never contracts into
// a fused multiply-add: the filters' error bounds, the expansion arithmetic
// and the reference's plain-double SoS arithmetic all assume one rounding per
// operation.  Only two_prod uses a fused multiply-add, for the exact error of
// a product.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

__device__ __forceinline__ void two_sum(double a, double b, double& x, double& y) {
  x = dadd(a, b);
  double bv = dsub(x, a);
  double av = dsub(x, bv);
  y = dadd(dsub(a, av), dsub(b, bv));
}
__device__ __forceinline__ void fast_two_sum(double a, double b, double& x, double& y) {
  x = dadd(a, b);
  y = dsub(b, dsub(x, a));
}
// Exact product with one fused multiply-add for the rounding error.
__device__ __forceinline__ void two_prod(double a, double b, double& x, double& y) {
  x = dmul(a, b);
  y = __fma_rn(a, b, -x);
}

// h = e + f with zero elimination.  Components are stored with increasing
// magnitude; the result has at least one component.
__device__ __noinline__ int esum(int el, const double* e, int fl, const double* f, double* h) {
  double Q, Qn, hh;
  double en = e[0], fn = f[0];
  int ei = 0, fi = 0, hi = 0;
  if ((fn > en) == (fn > -en)) {
    Q = en;
    en = (++ei < el) ? e[ei] : 0.0;
  } else {
    Q = fn;
    fn = (++fi < fl) ? f[fi] : 0.0;
  }
  if (ei < el && fi < fl) {
    if ((fn > en) == (fn > -en)) {
      fast_two_sum(en, Q, Qn, hh);
      en = (++ei < el) ? e[ei] : 0.0;
    } else {
      fast_two_sum(fn, Q, Qn, hh);
      fn = (++fi < fl) ? f[fi] : 0.0;
    }
    Q = Qn;
    if (hh != 0.0) h[hi++] = hh;
    while (ei < el && fi < fl) {
      if ((fn > en) == (fn > -en)) {
        two_sum(Q, en, Qn, hh);
        en = (++ei < el) ? e[ei] : 0.0;
      } else {
        two_sum(Q, fn, Qn, hh);
        fn = (++fi < fl) ? f[fi] : 0.0;
      }
      Q = Qn;
      if (hh != 0.0) h[hi++] = hh;
    }
  }
  while (ei < el) {
    two_sum(Q, en, Qn, hh);
    en = (++ei < el) ? e[ei] : 0.0;
    Q = Qn;
    if (hh != 0.0) h[hi++] = hh;
  }
  while (fi < fl) {
    two_sum(Q, fn, Qn, hh);
    fn = (++fi < fl) ? f[fi] : 0.0;
    Q = Qn;
    if (hh != 0.0) h[hi++] = hh;
  }
  if (Q != 0.0 || hi == 0) h[hi++] = Q;
  return hi;
}

// h = b * e with zero elimination.
__device__ __noinline__ int escale(int el, const double* e, double b, double* h) {
  double Q, s, hh, p1, p0;
  int hi = 0;
  two_prod(e[0], b, Q, hh);
  if (hh != 0.0) h[hi++] = hh;
  for (int i = 1; i < el; ++i) {
    two_prod(e[i], b, p1, p0);
    two_sum(Q, p0, s, hh);
    if (hh != 0.0) h[hi++] = hh;
    fast_two_sum(p1, s, Q, hh);
    if (hh != 0.0) h[hi++] = hh;
  }
  if (Q != 0.0 || hi == 0) h[hi++] = Q;
  return hi;
}

// In-place compression (most significant component last).
__device__ __noinline__ int ecompress(int el, double* e) {
  double Q = e[el - 1], q, Qn;
  int bottom = el - 1;
  for (int i = el - 2; i >= 0; --i) {
    fast_two_sum(Q, e[i], Qn, q);
    if (q != 0.0) {
      e[bottom--] = Qn;
      Q = q;
    } else {
      Q = Qn;
    }
  }
  int top = 0;
  for (int i = bottom + 1; i < el; ++i) {
    fast_two_sum(e[i], Q, Qn, q);
    if (q != 0.0) e[top++] = q;
    Q = Qn;
  }
  e[top++] = Q;
  return top;
}

__device__ __forceinline__ int esign(int n, const double* e) {
  double v = e[n - 1];
  return (v > 0.0) - (v < 0.0);
}

// p_u q_v - q_u p_v as a 4-component expansion.
__device__ __forceinline__ int minor2(const double* p, const double* q, int u, int v, double* h) {
  double a[2], b[2];
  two_prod(p[u], q[v], a[1], a[0]);
  two_prod(q[u], p[v], b[1], b[0]);
  b[0] = -b[0];
  b[1] = -b[1];
  return esum(2, a, 2, b, h);
}

// det[[p_u,p_v,1],[q_u,q_v,1],[r_u,r_v,1]] (<= 12 components).
__device__ __forceinline__ int minor3(const double* p, const double* q, const double* r, int u, int v,
                                      double* h) {
  double m1[4], m2[4], m3[4], t[8];
  int l1 = minor2(p, q, u, v, m1);
  int l2 = minor2(q, r, u, v, m2);
  int l3 = minor2(r, p, u, v, m3);
  int lt = esum(l1, m1, l2, m2, t);
  return esum(lt, t, l3, m3, h);
}

// |p|^2 exactly (<= 6 components, compressed).
__device__ __forceinline__ int lift(const double* p, double* h) {
  double a[2], b[2], c[2], t[4];
  two_prod(p[0], p[0], a[1], a[0]);
  two_prod(p[1], p[1], b[1], b[0]);
  two_prod(p[2], p[2], c[1], c[0]);
  int lt = esum(2, a, 2, b, t);
  int n = esum(lt, t, 2, c, h);
  return ecompress(n, h);
}

// det4 with columns (u, v, K, 1) over rows a..d where K is an expansion per
// row of at most 6 components.  Returns the compressed length in h (<= 32),
// or -1 if a buffer would overflow.
__device__ __noinline__ int det4k(const double* a, const double* b, const double* c, const double* d, int u,
                                  int v, const int* kl, const double (*K)[6], double* h) {
  const double* P[4] = {a, b, c, d};
  double acc[64], tmp[64], m[12], sc[24];
  int alen = 0;
#pragma unroll 1
  for (int i = 0; i < 4; ++i) {
    const double* x = P[i == 0 ? 1 : 0];
    const double* y = P[i <= 1 ? 2 : 1];
    const double* z = P[i <= 2 ? 3 : 2];
    int ml = minor3(x, y, z, u, v, m);
    ml = ecompress(ml, m);
#pragma unroll 1
    for (int j = 0; j < kl[i]; ++j) {
      double kv = (i & 1) ? -K[i][j] : K[i][j];
      int sl = escale(ml, m, kv, sc);
      if (alen == 0) {
        for (int q = 0; q < sl; ++q) acc[q] = sc[q];
        alen = sl;
      } else {
        if (alen + sl > 64) return -1;
        int nl = esum(alen, acc, sl, sc, tmp);
        nl = ecompress(nl, tmp);
        for (int q = 0; q < nl; ++q) acc[q] = tmp[q];
        alen = nl;
      }
    }
  }
  alen = ecompress(alen, acc);
  if (alen > 32) return -1;
  for (int q = 0; q < alen; ++q) h[q] = acc[q];
  return alen;
}

// Exact Shewchuk orient3d value = det[[x,y,z,1]] rows a..d.
__device__ __forceinline__ int orient3d_expansion(const double* a, const double* b, const double* c,
                                                  const double* d, double* h) {
  const int kl[4] = {1, 1, 1, 1};
  const double K[4][6] = {{a[2]}, {b[2]}, {c[2]}, {d[2]}};
  return det4k(a, b, c, d, 0, 1, kl, K, h);
}

__device__ __noinline__ int orient3d_exact_sign(const double* a, const double* b, const double* c,
                                                const double* d, uint32_t* flags) {
  double h[32];
  int n = orient3d_expansion(a, b, c, d, h);
  if (n < 0) {
    raise_precision(flags);
    return 0;
  }
  return esign(n, h);
}

// Exact insphere: D5 = -w_a D4(bcde) + w_b D4(acde) - w_c D4(abde) + w_d D4(abce) - w_e D4(abcd).
__device__ __noinline__ int insphere_exact_sign(const double* a, const double* b, const double* c,
                                                const double* d, const double* e, uint32_t* flags) {
  const double* P[5] = {a, b, c, d, e};
  double acc[96], tmp[96], d4[32], w[6], sc[64];
  int alen = 0;
#pragma unroll 1
  for (int i = 0; i < 5; ++i) {
    const double* q[4];
    int k = 0;
    for (int j = 0; j < 5; ++j)
      if (j != i) q[k++] = P[j];
    int dl = orient3d_expansion(q[0], q[1], q[2], q[3], d4);
    if (dl < 0) {
      raise_precision(flags);
      return 0;
    }
    if (dl == 1 && d4[0] == 0.0) continue;
    int wl = lift(P[i], w);
#pragma unroll 1
    for (int j = 0; j < wl; ++j) {
      double wv = (i & 1) ? w[j] : -w[j];
      int sl = escale(dl, d4, wv, sc);
      if (alen == 0) {
        for (int t = 0; t < sl; ++t) acc[t] = sc[t];
        alen = sl;
      } else {
        if (alen + sl > 96) {
          raise_precision(flags);
          return 0;
        }
        int nl = esum(alen, acc, sl, sc, tmp);
        nl = ecompress(nl, tmp);
        for (int t = 0; t < nl; ++t) acc[t] = tmp[t];
        alen = nl;
      }
    }
  }
  if (alen == 0) return 0;
  return esign(alen, acc);
}

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
constexpr double kO3dBoundA = (7.0 + 56.0 * kEps) * kEps;
constexpr double kIspBoundA = (16.0 + 224.0 * kEps) * kEps;
constexpr double kO3dBoundLifted = (11.0 + 112.0 * kEps) * kEps;  // src/predicates.rs:426-427

// ---- Exact stage by modular arithmetic ----
//
// Every finite double is a dyadic rational m * 2^e (m odd).  With S the
// smallest e among the coordinates of a predicate's points, every coordinate
// is an integer multiple of 2^S, and orient3d / insphere -- homogeneous
// polynomials of degree 3 / 5 in the coordinate differences with integer
// coefficients -- equal det_int * 2^(3S) / det_int * 2^(5S) for the same
// polynomial evaluated on the integers X = x / 2^S.  The stage evaluates that
// polynomial in the residue rings Z / 2^64 and Z / P (P = 2^61 - 1, a Mersenne
// prime) and reconstructs det_int by the Chinese remainder theorem, which is
// exact for |det_int| < 2^64 P / 2 (about 2^124).  The bound comes from the
// FP64 filter that ran first: when it cannot decide, |det_fp| <= err, so the
// exact determinant is at most 2 err and |det_int| <= 2 err 2^(-dS).  The
// stage answers only when that bound is below 2^122 and S >= -160 (points of
// f32 origin, where the filter's bound is valid: no product of differences
// reaches the FP64 underflow range); otherwise the expansion stage decides.
// On exactly degenerate inputs -- cospherical corners of lattice boxes,
// coplanar lattice faces -- it replaces hundreds of expansion operations by
// about forty residue products.
constexpr uint64_t kP61 = (1ull << 61) - 1ull;

struct Res {  // a value mod 2^64 and mod P
  uint64_t a, b;
};
__device__ __forceinline__ uint64_t mod_p(uint64_t x) {
  x = (x & kP61) + (x >> 61);
  return x >= kP61 ? x - kP61 : x;
}
__device__ __forceinline__ uint64_t mulmod_p(uint64_t x, uint64_t y) {
  const uint64_t lo = x * y, hi = __umul64hi(x, y);  // x, y < 2^61: the product has < 122 bits
  const uint64_t r = (lo & kP61) + ((hi << 3) | (lo >> 61));
  return mod_p(r);
}
__device__ __forceinline__ Res radd(Res x, Res y) { return {x.a + y.a, mod_p(x.b + y.b)}; }
__device__ __forceinline__ Res rsub(Res x, Res y) { return {x.a - y.a, mod_p(x.b + (kP61 - y.b))}; }
__device__ __forceinline__ Res rmul(Res x, Res y) { return {x.a * y.a, mulmod_p(x.b, y.b)}; }

// x = (-1)^neg m 2^e with m odd (m = 0 for zero).  Finite inputs only.
__device__ __forceinline__ void dyadic(double x, uint64_t& m, int& e, bool& neg) {
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
  neg = (bits >> 63) != 0;
  const int be = int((bits >> 52) & 0x7FF);
  m = bits & ((1ull << 52) - 1ull);
  if (be != 0) m |= 1ull << 52;
  e = (be != 0 ? be : 1) - 1075;
  if (m == 0) {
    e = 1 << 20;  // never the minimum
    return;
  }
  const int tz = __ffsll(static_cast<long long>(m)) - 1;
  m >>= tz;
  e += tz;
}

// Residues of x / 2^S (an integer: e >= S).
__device__ __forceinline__ Res residue(uint64_t m, int e, bool neg, int S) {
  if (m == 0) return {0ull, 0ull};
  const int k = e - S;
  const uint64_t a = k < 64 ? (m << k) : 0ull;
  const uint64_t b = mulmod_p(mod_p(m), 1ull << (k % 61));
  return neg ? Res{0ull - a, b ? kP61 - b : 0ull} : Res{a, b};
}

// Sign of the integer with residues r, known to satisfy |x| < 2^123.
__device__ __forceinline__ int crt_sign(Res r) {
  // x = r.a + 2^64 k with k = (r.b - r.a) / 2^64 mod P; 2^64 = 8 mod P and
  // 1/8 = 2^58 mod P.
  const uint64_t k = mulmod_p(mod_p(r.b + (kP61 - mod_p(r.a))), 1ull << 58);
  if (k == 0) return r.a == 0 ? 0 : 1;
  // x in [0, 2^64 P): negative when at least half the modulus
  const unsigned __int128 x = (static_cast<unsigned __int128>(k) << 64) | r.a;
  const unsigned __int128 half = static_cast<unsigned __int128>(kP61) << 63;
  return x >= half ? -1 : 1;
}

// Exact sign of Shewchuk's orient3d / insphere on the points' integer
// multiples of 2^S, or 2 when the stage does not apply.  `err` is the FP64
// filter's bound for the same points (the filter could not decide).
__device__ __noinline__ int orient3d_modular(const double* pa, const double* pb, const double* pc,
                                             const double* pd, double err) {
  const double* P[4] = {pa, pb, pc, pd};
  uint64_t m[12];
  int e[12];
  bool ng[12];
  int S = 1 << 20;
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    dyadic(P[i / 3][i % 3], m[i], e[i], ng[i]);
    S = min(S, e[i]);
  }
  if (S == (1 << 20)) return 0;  // all coordinates zero
  if (S < -160 || !(ldexp(dmul(err, 2.0 + 0x1p-39), -3 * S) < 0x1p122)) return 2;
  Res X[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) X[i] = residue(m[i], e[i], ng[i], S);
  const Res adx = rsub(X[0], X[9]), ady = rsub(X[1], X[10]), adz = rsub(X[2], X[11]);
  const Res bdx = rsub(X[3], X[9]), bdy = rsub(X[4], X[10]), bdz = rsub(X[5], X[11]);
  const Res cdx = rsub(X[6], X[9]), cdy = rsub(X[7], X[10]), cdz = rsub(X[8], X[11]);
  const Res det = radd(radd(rmul(adz, rsub(rmul(bdx, cdy), rmul(cdx, bdy))),
                            rmul(bdz, rsub(rmul(cdx, ady), rmul(adx, cdy)))),
                       rmul(cdz, rsub(rmul(adx, bdy), rmul(bdx, ady))));
  return crt_sign(det);
}

__device__ __noinline__ int insphere_modular(const double* pa, const double* pb, const double* pc,
                                             const double* pd, const double* pe, double err) {
  const double* P[5] = {pa, pb, pc, pd, pe};
  uint64_t m[15];
  int e[15];
  bool ng[15];
  int S = 1 << 20;
#pragma unroll
  for (int i = 0; i < 15; ++i) {
    dyadic(P[i / 3][i % 3], m[i], e[i], ng[i]);
    S = min(S, e[i]);
  }
  if (S == (1 << 20)) return 0;
  if (S < -160 || !(ldexp(dmul(err, 2.0 + 0x1p-39), -5 * S) < 0x1p122)) return 2;
  Res X[15];
#pragma unroll
  for (int i = 0; i < 15; ++i) X[i] = residue(m[i], e[i], ng[i], S);
  const Res aex = rsub(X[0], X[12]), aey = rsub(X[1], X[13]), aez = rsub(X[2], X[14]);
  const Res bex = rsub(X[3], X[12]), bey = rsub(X[4], X[13]), bez = rsub(X[5], X[14]);
  const Res cex = rsub(X[6], X[12]), cey = rsub(X[7], X[13]), cez = rsub(X[8], X[14]);
  const Res dex = rsub(X[9], X[12]), dey = rsub(X[10], X[13]), dez = rsub(X[11], X[14]);
  const Res ab = rsub(rmul(aex, bey), rmul(bex, aey)), bc = rsub(rmul(bex, cey), rmul(cex, bey));
  const Res cd = rsub(rmul(cex, dey), rmul(dex, cey)), da = rsub(rmul(dex, aey), rmul(aex, dey));
  const Res ac = rsub(rmul(aex, cey), rmul(cex, aey)), bd = rsub(rmul(bex, dey), rmul(dex, bey));
  const Res abc = radd(rsub(rmul(aez, bc), rmul(bez, ac)), rmul(cez, ab));
  const Res bcd = radd(rsub(rmul(bez, cd), rmul(cez, bd)), rmul(dez, bc));
  const Res cda = radd(radd(rmul(cez, da), rmul(dez, ac)), rmul(aez, cd));
  const Res dab = radd(radd(rmul(dez, ab), rmul(aez, bd)), rmul(bez, da));
  const Res al = radd(radd(rmul(aex, aex), rmul(aey, aey)), rmul(aez, aez));
  const Res bl = radd(radd(rmul(bex, bex), rmul(bey, bey)), rmul(bez, bez));
  const Res cl = radd(radd(rmul(cex, cex), rmul(cey, cey)), rmul(cez, cez));
  const Res dl = radd(radd(rmul(dex, dex), rmul(dey, dey)), rmul(dez, dez));
  const Res det = radd(rsub(rmul(dl, abc), rmul(cl, dab)), rsub(rmul(bl, cda), rmul(al, bcd)));
  return crt_sign(det);
}

// Exact sign of det[[p_0, p_1, |p|^2, 1]] over rows a..d (the lifted
// orient3d's exact stage), or 2 when the stage does not apply.  Subtracting
// row d gives the 3x3 determinant of (du, dv, |p|^2 - |d|^2) over rows a..c,
// which is evaluated on the residues.  Its magnitude is bounded from the
// coordinates: the permanent of (|du|, |dv|, sum_j |p_j - d_j| |p_j + d_j|)
// in FP64, with a margin for its own rounding.
__device__ __noinline__ int lifted_modular(const double* pa, const double* pb, const double* pc,
                                           const double* pd) {
  const double* P[4] = {pa, pb, pc, pd};
  uint64_t m[12];
  int e[12];
  bool ng[12];
  int S = 1 << 20;
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    dyadic(P[i / 3][i % 3], m[i], e[i], ng[i]);
    S = min(S, e[i]);
  }
  if (S == (1 << 20)) return 0;
  if (S < -160) return 2;
  double du[3], dv[3], dl[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    du[r] = fabs(dsub(P[r][0], pd[0]));
    dv[r] = fabs(dsub(P[r][1], pd[1]));
    dl[r] = dadd(dadd(dmul(du[r], fabs(dadd(P[r][0], pd[0]))), dmul(dv[r], fabs(dadd(P[r][1], pd[1])))),
                 dmul(fabs(dsub(P[r][2], pd[2])), fabs(dadd(P[r][2], pd[2]))));
  }
  const double perm = dadd(dadd(dmul(du[0], dadd(dmul(dv[1], dl[2]), dmul(dv[2], dl[1]))),
                                dmul(du[1], dadd(dmul(dv[0], dl[2]), dmul(dv[2], dl[0])))),
                           dmul(du[2], dadd(dmul(dv[0], dl[1]), dmul(dv[1], dl[0]))));
  if (!(ldexp(dmul(perm, 1.0 + 0x1p-30), -4 * S) < 0x1p122)) return 2;
  Res X[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) X[i] = residue(m[i], e[i], ng[i], S);
  Res L[4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
    L[r] = radd(radd(rmul(X[3 * r], X[3 * r]), rmul(X[3 * r + 1], X[3 * r + 1])), rmul(X[3 * r + 2], X[3 * r + 2]));
  Res U[3], V[3], W[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    U[r] = rsub(X[3 * r], X[9]);
    V[r] = rsub(X[3 * r + 1], X[10]);
    W[r] = rsub(L[r], L[3]);
  }
  const Res det = radd(rsub(rmul(U[0], rsub(rmul(V[1], W[2]), rmul(V[2], W[1]))),
                            rmul(U[1], rsub(rmul(V[0], W[2]), rmul(V[2], W[0])))),
                       rmul(U[2], rsub(rmul(V[0], W[1]), rmul(V[1], W[0]))));
  return crt_sign(det);
}

// Sign of Shewchuk orient3d(a,b,c,d): FP64 filter, then exact.
__device__ __forceinline__ int orient3d(const double* pa, const double* pb, const double* pc, const double* pd,
                                        uint32_t* flags) {
  double adx = dsub(pa[0], pd[0]), bdx = dsub(pb[0], pd[0]), cdx = dsub(pc[0], pd[0]);
  double ady = dsub(pa[1], pd[1]), bdy = dsub(pb[1], pd[1]), cdy = dsub(pc[1], pd[1]);
  double adz = dsub(pa[2], pd[2]), bdz = dsub(pb[2], pd[2]), cdz = dsub(pc[2], pd[2]);
  double bdxcdy = dmul(bdx, cdy), cdxbdy = dmul(cdx, bdy);
  double cdxady = dmul(cdx, ady), adxcdy = dmul(adx, cdy);
  double adxbdy = dmul(adx, bdy), bdxady = dmul(bdx, ady);
  double det = dadd(dadd(dmul(adz, dsub(bdxcdy, cdxbdy)), dmul(bdz, dsub(cdxady, adxcdy))),
                    dmul(cdz, dsub(adxbdy, bdxady)));
  double perm = dadd(dadd(dmul(dadd(fabs(bdxcdy), fabs(cdxbdy)), fabs(adz)),
                          dmul(dadd(fabs(cdxady), fabs(adxcdy)), fabs(bdz))),
                     dmul(dadd(fabs(adxbdy), fabs(bdxady)), fabs(cdz)));
  double err = dmul(kO3dBoundA, perm);
  if (det > err) return 1;
  if (-det > err) return -1;
  // Fresh copies for the out-of-line exact stages: the caller's coordinate
  // arrays never have their address taken, so they stay in registers.
  double a[3] = {pa[0], pa[1], pa[2]}, b[3] = {pb[0], pb[1], pb[2]};
  double c[3] = {pc[0], pc[1], pc[2]}, d[3] = {pd[0], pd[1], pd[2]};
  const int sm = orient3d_modular(a, b, c, d, err);
  if (sm != 2) return sm;
  return orient3d_exact_sign(a, b, c, d, flags);
}

// Sign of Shewchuk insphere(a,b,c,d,e): FP64 filter, then exact.
__device__ __forceinline__ int insphere(const double* pa, const double* pb, const double* pc, const double* pd,
                                        const double* pe, uint32_t* flags) {
  double aex = dsub(pa[0], pe[0]), bex = dsub(pb[0], pe[0]), cex = dsub(pc[0], pe[0]), dex = dsub(pd[0], pe[0]);
  double aey = dsub(pa[1], pe[1]), bey = dsub(pb[1], pe[1]), cey = dsub(pc[1], pe[1]), dey = dsub(pd[1], pe[1]);
  double aez = dsub(pa[2], pe[2]), bez = dsub(pb[2], pe[2]), cez = dsub(pc[2], pe[2]), dez = dsub(pd[2], pe[2]);
  double aexbey = dmul(aex, bey), bexaey = dmul(bex, aey), ab = dsub(aexbey, bexaey);
  double bexcey = dmul(bex, cey), cexbey = dmul(cex, bey), bc = dsub(bexcey, cexbey);
  double cexdey = dmul(cex, dey), dexcey = dmul(dex, cey), cd = dsub(cexdey, dexcey);
  double dexaey = dmul(dex, aey), aexdey = dmul(aex, dey), da = dsub(dexaey, aexdey);
  double aexcey = dmul(aex, cey), cexaey = dmul(cex, aey), ac = dsub(aexcey, cexaey);
  double bexdey = dmul(bex, dey), dexbey = dmul(dex, bey), bd = dsub(bexdey, dexbey);
  double abc = dadd(dsub(dmul(aez, bc), dmul(bez, ac)), dmul(cez, ab));
  double bcd = dadd(dsub(dmul(bez, cd), dmul(cez, bd)), dmul(dez, bc));
  double cda = dadd(dadd(dmul(cez, da), dmul(dez, ac)), dmul(aez, cd));
  double dab = dadd(dadd(dmul(dez, ab), dmul(aez, bd)), dmul(bez, da));
  double alift = dadd(dadd(dmul(aex, aex), dmul(aey, aey)), dmul(aez, aez));
  double blift = dadd(dadd(dmul(bex, bex), dmul(bey, bey)), dmul(bez, bez));
  double clift = dadd(dadd(dmul(cex, cex), dmul(cey, cey)), dmul(cez, cez));
  double dlift = dadd(dadd(dmul(dex, dex), dmul(dey, dey)), dmul(dez, dez));
  double det = dadd(dsub(dmul(dlift, abc), dmul(clift, dab)), dsub(dmul(blift, cda), dmul(alift, bcd)));
  double az = fabs(aez), bz = fabs(bez), cz = fabs(cez), dz = fabs(dez);
  double p_ab = dadd(fabs(aexbey), fabs(bexaey)), p_bc = dadd(fabs(bexcey), fabs(cexbey));
  double p_cd = dadd(fabs(cexdey), fabs(dexcey)), p_da = dadd(fabs(dexaey), fabs(aexdey));
  double p_ac = dadd(fabs(aexcey), fabs(cexaey)), p_bd = dadd(fabs(bexdey), fabs(dexbey));
  double perm = dadd(dadd(dadd(dmul(dadd(dadd(dmul(p_cd, bz), dmul(p_bd, cz)), dmul(p_bc, dz)), alift),
                               dmul(dadd(dadd(dmul(p_da, cz), dmul(p_ac, dz)), dmul(p_cd, az)), blift)),
                          dmul(dadd(dadd(dmul(p_ab, dz), dmul(p_bd, az)), dmul(p_da, bz)), clift)),
                     dmul(dadd(dadd(dmul(p_bc, az), dmul(p_ac, bz)), dmul(p_ab, cz)), dlift));
  double err = dmul(kIspBoundA, perm);
  if (det > err) return 1;
  if (-det > err) return -1;
  double a[3] = {pa[0], pa[1], pa[2]}, b[3] = {pb[0], pb[1], pb[2]};
  double c[3] = {pc[0], pc[1], pc[2]}, d[3] = {pd[0], pd[1], pd[2]};
  double e[3] = {pe[0], pe[1], pe[2]};
  const int sm = insphere_modular(a, b, c, d, e, err);
  if (sm != 2) return sm;
  return insphere_exact_sign(a, b, c, d, e, flags);
}

// ---- FP32 stage ----

constexpr float kEpsF = 5.9604644775390625e-08f;  // 2^-24
constexpr float kO3dBoundF = (7.0f + 56.0f * kEpsF) * kEpsF;
constexpr float kIspBoundF = (16.0f + 224.0f * kEpsF) * kEpsF;
// Permanents below this get no answer (typical permanents of the benchmark
// clouds are above 1e-16).
constexpr float kPermMinF = 1.0e-26f;
// Absolute slack added to the bound for gradual underflow: each of the ~60
// operations may lose at most 2^-150 to a subnormal result, which reaches the
// determinant multiplied by at most 500 * 7.5e5 (coordinate differences within
// the super tetrahedron's extent of 500, lifted terms below 7.5e5): < 2e-35 in
// all.  At the smallest permanent answered the bound itself is ~1e-32.
constexpr float kUnderflowSlackF = 1.0e-33f;

// Sign of Shewchuk orient3d(a,b,c,d) when certain from f32 arithmetic, else 0.
__device__ __forceinline__ int orient3d_f32(const float4& pa, const float4& pb, const float4& pc,
                                            const float4& pd) {
  const float adx = __fsub_rn(pa.x, pd.x), bdx = __fsub_rn(pb.x, pd.x), cdx = __fsub_rn(pc.x, pd.x);
  const float ady = __fsub_rn(pa.y, pd.y), bdy = __fsub_rn(pb.y, pd.y), cdy = __fsub_rn(pc.y, pd.y);
  const float adz = __fsub_rn(pa.z, pd.z), bdz = __fsub_rn(pb.z, pd.z), cdz = __fsub_rn(pc.z, pd.z);
  const float bdxcdy = __fmul_rn(bdx, cdy), cdxbdy = __fmul_rn(cdx, bdy);
  const float cdxady = __fmul_rn(cdx, ady), adxcdy = __fmul_rn(adx, cdy);
  const float adxbdy = __fmul_rn(adx, bdy), bdxady = __fmul_rn(bdx, ady);
  const float det = __fadd_rn(__fadd_rn(__fmul_rn(adz, __fsub_rn(bdxcdy, cdxbdy)),
                                        __fmul_rn(bdz, __fsub_rn(cdxady, adxcdy))),
                              __fmul_rn(cdz, __fsub_rn(adxbdy, bdxady)));
  const float perm = __fadd_rn(__fadd_rn(__fmul_rn(__fadd_rn(fabsf(bdxcdy), fabsf(cdxbdy)), fabsf(adz)),
                                         __fmul_rn(__fadd_rn(fabsf(cdxady), fabsf(adxcdy)), fabsf(bdz))),
                               __fmul_rn(__fadd_rn(fabsf(adxbdy), fabsf(bdxady)), fabsf(cdz)));
  if (!(perm >= kPermMinF && perm < 1.0e30f)) return 0;
  const float err = __fadd_rn(__fmul_rn(kO3dBoundF, perm), kUnderflowSlackF);
  if (det > err) return 1;
  if (-det > err) return -1;
  return 0;
}

// Sign of Shewchuk insphere(a,b,c,d,e) when certain from f32 arithmetic, else 0.
__device__ __forceinline__ int insphere_f32(const float4& pa, const float4& pb, const float4& pc, const float4& pd,
                                            const float4& pe) {
  const float aex = __fsub_rn(pa.x, pe.x), bex = __fsub_rn(pb.x, pe.x);
  const float cex = __fsub_rn(pc.x, pe.x), dex = __fsub_rn(pd.x, pe.x);
  const float aey = __fsub_rn(pa.y, pe.y), bey = __fsub_rn(pb.y, pe.y);
  const float cey = __fsub_rn(pc.y, pe.y), dey = __fsub_rn(pd.y, pe.y);
  const float aez = __fsub_rn(pa.z, pe.z), bez = __fsub_rn(pb.z, pe.z);
  const float cez = __fsub_rn(pc.z, pe.z), dez = __fsub_rn(pd.z, pe.z);
  const float aexbey = __fmul_rn(aex, bey), bexaey = __fmul_rn(bex, aey), ab = __fsub_rn(aexbey, bexaey);
  const float bexcey = __fmul_rn(bex, cey), cexbey = __fmul_rn(cex, bey), bc = __fsub_rn(bexcey, cexbey);
  const float cexdey = __fmul_rn(cex, dey), dexcey = __fmul_rn(dex, cey), cd = __fsub_rn(cexdey, dexcey);
  const float dexaey = __fmul_rn(dex, aey), aexdey = __fmul_rn(aex, dey), da = __fsub_rn(dexaey, aexdey);
  const float aexcey = __fmul_rn(aex, cey), cexaey = __fmul_rn(cex, aey), ac = __fsub_rn(aexcey, cexaey);
  const float bexdey = __fmul_rn(bex, dey), dexbey = __fmul_rn(dex, bey), bd = __fsub_rn(bexdey, dexbey);
  const float abc = __fadd_rn(__fsub_rn(__fmul_rn(aez, bc), __fmul_rn(bez, ac)), __fmul_rn(cez, ab));
  const float bcd = __fadd_rn(__fsub_rn(__fmul_rn(bez, cd), __fmul_rn(cez, bd)), __fmul_rn(dez, bc));
  const float cda = __fadd_rn(__fadd_rn(__fmul_rn(cez, da), __fmul_rn(dez, ac)), __fmul_rn(aez, cd));
  const float dab = __fadd_rn(__fadd_rn(__fmul_rn(dez, ab), __fmul_rn(aez, bd)), __fmul_rn(bez, da));
  const float alift = __fadd_rn(__fadd_rn(__fmul_rn(aex, aex), __fmul_rn(aey, aey)), __fmul_rn(aez, aez));
  const float blift = __fadd_rn(__fadd_rn(__fmul_rn(bex, bex), __fmul_rn(bey, bey)), __fmul_rn(bez, bez));
  const float clift = __fadd_rn(__fadd_rn(__fmul_rn(cex, cex), __fmul_rn(cey, cey)), __fmul_rn(cez, cez));
  const float dlift = __fadd_rn(__fadd_rn(__fmul_rn(dex, dex), __fmul_rn(dey, dey)), __fmul_rn(dez, dez));
  const float det = __fadd_rn(__fsub_rn(__fmul_rn(dlift, abc), __fmul_rn(clift, dab)),
                              __fsub_rn(__fmul_rn(blift, cda), __fmul_rn(alift, bcd)));
  const float az = fabsf(aez), bz = fabsf(bez), cz = fabsf(cez), dz = fabsf(dez);
  const float p_ab = __fadd_rn(fabsf(aexbey), fabsf(bexaey)), p_bc = __fadd_rn(fabsf(bexcey), fabsf(cexbey));
  const float p_cd = __fadd_rn(fabsf(cexdey), fabsf(dexcey)), p_da = __fadd_rn(fabsf(dexaey), fabsf(aexdey));
  const float p_ac = __fadd_rn(fabsf(aexcey), fabsf(cexaey)), p_bd = __fadd_rn(fabsf(bexdey), fabsf(dexbey));
  const float t_a = __fadd_rn(__fadd_rn(__fmul_rn(p_cd, bz), __fmul_rn(p_bd, cz)), __fmul_rn(p_bc, dz));
  const float t_b = __fadd_rn(__fadd_rn(__fmul_rn(p_da, cz), __fmul_rn(p_ac, dz)), __fmul_rn(p_cd, az));
  const float t_c = __fadd_rn(__fadd_rn(__fmul_rn(p_ab, dz), __fmul_rn(p_bd, az)), __fmul_rn(p_da, bz));
  const float t_d = __fadd_rn(__fadd_rn(__fmul_rn(p_bc, az), __fmul_rn(p_ac, bz)), __fmul_rn(p_ab, cz));
  // summed in Shewchuk's order: ((a + b) + c) + d
  const float perm = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(t_a, alift), __fmul_rn(t_b, blift)),
                                         __fmul_rn(t_c, clift)),
                               __fmul_rn(t_d, dlift));
  if (!(perm >= kPermMinF && perm < 1.0e30f)) return 0;
  const float err = __fadd_rn(__fmul_rn(kIspBoundF, perm), kUnderflowSlackF);
  if (det > err) return 1;
  if (-det > err) return -1;
  return 0;
}

// ---- SoS cascade pieces (src/predicates.rs) ----

// Plain double orient2d on coordinates (u, v): src/predicates.rs:73-75.
__device__ __forceinline__ double orient2d_plain(const double* a, const double* b, const double* c, int u,
                                                 int v) {
  return dsub(dmul(dsub(a[u], c[u]), dsub(b[v], c[v])), dmul(dsub(a[v], c[v]), dsub(b[u], c[u])));
}

// Lifted orient3d on permuted coordinates: the reference's filter and error
// bound (src/predicates.rs:390-435), then the exact sign of det[[u,v,|p|^2,1]].
__device__ __noinline__ int orient3d_lifted(const double* a0, const double* b0, const double* c0,
                                            const double* d0, int q0, int q1, int q2, uint32_t* flags) {
  double pa[3] = {a0[q0], a0[q1], a0[q2]};
  double pb[3] = {b0[q0], b0[q1], b0[q2]};
  double pc[3] = {c0[q0], c0[q1], c0[q2]};
  double pd[3] = {d0[q0], d0[q1], d0[q2]};
  double adx = dsub(pa[0], pd[0]), bdx = dsub(pb[0], pd[0]), cdx = dsub(pc[0], pd[0]);
  double ady = dsub(pa[1], pd[1]), bdy = dsub(pb[1], pd[1]), cdy = dsub(pc[1], pd[1]);
  double adzr = dsub(pa[2], pd[2]), bdzr = dsub(pb[2], pd[2]), cdzr = dsub(pc[2], pd[2]);
  double adz = dadd(dadd(dmul(adx, adx), dmul(ady, ady)), dmul(adzr, adzr));
  double bdz = dadd(dadd(dmul(bdx, bdx), dmul(bdy, bdy)), dmul(bdzr, bdzr));
  double cdz = dadd(dadd(dmul(cdx, cdx), dmul(cdy, cdy)), dmul(cdzr, cdzr));
  double bdxcdy = dmul(bdx, cdy), cdxbdy = dmul(cdx, bdy), cdxady = dmul(cdx, ady);
  double adxcdy = dmul(adx, cdy), adxbdy = dmul(adx, bdy), bdxady = dmul(bdx, ady);
  double det = dadd(dadd(dmul(adz, dsub(bdxcdy, cdxbdy)), dmul(bdz, dsub(cdxady, adxcdy))),
                    dmul(cdz, dsub(adxbdy, bdxady)));
  double perm = dadd(dadd(dmul(dadd(fabs(bdxcdy), fabs(cdxbdy)), fabs(adz)),
                          dmul(dadd(fabs(cdxady), fabs(adxcdy)), fabs(bdz))),
                     dmul(dadd(fabs(adxbdy), fabs(bdxady)), fabs(cdz)));
  double err = dmul(kO3dBoundLifted, perm);
  if (det > err || -det > err) return (det > 0.0) - (det < 0.0);
  const int sm = lifted_modular(pa, pb, pc, pd);
  if (sm != 2) return sm;
  int kl[4];
  double K[4][6];
  kl[0] = lift(pa, K[0]);
  kl[1] = lift(pb, K[1]);
  kl[2] = lift(pc, K[2]);
  kl[3] = lift(pd, K[3]);
  double h[32];
  int n = det4k(pa, pb, pc, pd, 0, 1, kl, K, h);
  if (n < 0) {
    raise_precision(flags);
    return 0;
  }
  return esign(n, h);
}

// Exact sign of a_u (w_b - w_c) + b_u (w_c - w_a) + c_u (w_a - w_b): src/predicates.rs:255-291.
__device__ __noinline__ int orient2d_lifted(const double* a, const double* b, const double* c, int q0) {
  double W[3][6];
  int L[3];
  L[0] = lift(a, W[0]);
  L[1] = lift(b, W[1]);
  L[2] = lift(c, W[2]);
  const double U[3] = {a[q0], b[q0], c[q0]};
  double acc[80], tmp[80], sc[12];
  int alen = 0;
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      int j = (i + 1 + s) % 3;
      int sl = escale(L[j], W[j], s == 0 ? U[i] : -U[i], sc);
      if (alen == 0) {
        for (int t = 0; t < sl; ++t) acc[t] = sc[t];
        alen = sl;
      } else {
        int nl = esum(alen, acc, sl, sc, tmp);
        nl = ecompress(nl, tmp);
        for (int t = 0; t < nl; ++t) acc[t] = tmp[t];
        alen = nl;
      }
    }
  }
  return esign(alen, acc);
}

// Exact sign of |a|^2 - |b|^2: src/predicates.rs:229-252.
__device__ __noinline__ int orient1d_lifted(const double* a, const double* b) {
  double wa[6], wb[6], h[12];
  int la = lift(a, wa), lb = lift(b, wb);
  for (int i = 0; i < lb; ++i) wb[i] = -wb[i];
  int n = esum(la, wa, lb, wb, h);
  return esign(n, h);
}

// One level of the orient4d SoS cascade (src/predicates.rs:513-667): term
// kind, the sorted points used, coordinate permutation, sign flip.
enum : uint8_t { kO3 = 0, kO3L, kO2, kO2L, kO1, kO1L, kConst };
struct SosLevel {
  uint8_t kind, p0, p1, p2, p3, q0, q1, q2, flip;
};

__constant__ SosLevel kSos4[49] = {
    {kO3, 1, 2, 3, 4, 0, 1, 2, 1},  {kO3L, 1, 2, 3, 4, 0, 1, 2, 0}, {kO3L, 1, 2, 3, 4, 0, 2, 1, 1},
    {kO3L, 1, 2, 3, 4, 1, 2, 0, 0}, {kO3, 0, 2, 3, 4, 0, 1, 2, 0},  {kO2, 2, 3, 4, 0, 0, 1, 2, 0},
    {kO2, 2, 3, 4, 0, 0, 2, 1, 1},  {kO2, 2, 3, 4, 0, 1, 2, 0, 0},  {kO3L, 0, 2, 3, 4, 0, 1, 2, 1},
    {kO2L, 2, 3, 4, 0, 0, 1, 2, 0}, {kO2L, 2, 3, 4, 0, 1, 0, 2, 1}, {kO3L, 0, 2, 3, 4, 0, 2, 1, 0},
    {kO2L, 2, 3, 4, 0, 2, 0, 1, 0}, {kO3L, 0, 2, 3, 4, 1, 2, 0, 1}, {kO3, 0, 1, 3, 4, 0, 1, 2, 1},
    {kO2, 1, 3, 4, 0, 0, 1, 2, 1},  {kO2, 1, 3, 4, 0, 0, 2, 1, 0},  {kO2, 1, 3, 4, 0, 1, 2, 0, 1},
    {kO2, 0, 3, 4, 0, 0, 1, 2, 0},  {kO1, 3, 4, 0, 0, 0, 1, 2, 1},  {kO1, 3, 4, 0, 0, 1, 0, 2, 0},
    {kO2, 0, 3, 4, 0, 0, 2, 1, 1},  {kO1, 3, 4, 0, 0, 2, 0, 1, 1},  {kO2, 0, 3, 4, 0, 1, 2, 0, 0},
    {kO3L, 0, 1, 3, 4, 0, 1, 2, 0}, {kO2L, 1, 3, 4, 0, 0, 1, 2, 1}, {kO2L, 1, 3, 4, 0, 1, 0, 2, 0},
    {kO2L, 0, 3, 4, 0, 0, 1, 2, 0}, {kO1L, 3, 4, 0, 0, 0, 1, 2, 0}, {kO2L, 0, 3, 4, 0, 1, 0, 2, 1},
    {kO3L, 0, 1, 3, 4, 0, 2, 1, 1}, {kO2L, 1, 3, 4, 0, 2, 0, 1, 1}, {kO2L, 0, 3, 4, 0, 2, 0, 1, 0},
    {kO3L, 0, 1, 3, 4, 1, 2, 0, 0}, {kO3, 0, 1, 2, 4, 0, 1, 2, 0},  {kO2, 1, 2, 4, 0, 0, 1, 2, 0},
    {kO2, 1, 2, 4, 0, 0, 2, 1, 1},  {kO2, 1, 2, 4, 0, 1, 2, 0, 0},  {kO2, 0, 2, 4, 0, 0, 1, 2, 1},
    {kO1, 2, 4, 0, 0, 0, 1, 2, 0},  {kO1, 2, 4, 0, 0, 1, 0, 2, 1},  {kO2, 0, 2, 4, 0, 0, 2, 1, 0},
    {kO1, 2, 4, 0, 0, 2, 0, 1, 0},  {kO2, 0, 2, 4, 0, 1, 2, 0, 1},  {kO2, 0, 1, 4, 0, 0, 1, 2, 0},
    {kO1, 1, 4, 0, 0, 0, 1, 2, 1},  {kO1, 1, 4, 0, 0, 1, 0, 2, 0},  {kO1, 0, 4, 0, 0, 0, 1, 2, 0},
    {kConst, 0, 0, 0, 0, 0, 1, 2, 0},
};

// Sorts (key, point) pairs by key with insertion sort; returns parity.
template <int N>
__device__ __forceinline__ int sort_keys(uint32_t* k, const double** p) {
  int parity = 0;
#pragma unroll
  for (int i = 1; i < N; ++i) {
#pragma unroll
    for (int j = i; j > 0; --j) {
      if (k[j] < k[j - 1]) {
        uint32_t tk = k[j];
        k[j] = k[j - 1];
        k[j - 1] = tk;
        const double* tp = p[j];
        p[j] = p[j - 1];
        p[j - 1] = tp;
        parity ^= 1;
      }
    }
  }
  return parity;
}

// gDel3D orientation with SoS: +1 iff the exact det < 0; never 0.
__device__ __noinline__ int orient3d_sos_degenerate(const double* a, const double* b, const double* c,
                                                    const double* d, uint32_t ia, uint32_t ib, uint32_t ic,
                                                    uint32_t id) {
  uint32_t k[4] = {ia, ib, ic, id};
  const double* p[4] = {a, b, c, d};
  int parity = sort_keys<4>(k, p);
  double r = 1.0;
  int depth = 13;
#pragma unroll 1
  for (int dd = 0; dd < 13; ++dd) {
    double v;
    switch (dd) {
      case 0: v = orient2d_plain(p[1], p[2], p[3], 0, 1); break;
      case 1: v = orient2d_plain(p[1], p[2], p[3], 0, 2); break;
      case 2: v = orient2d_plain(p[1], p[2], p[3], 1, 2); break;
      case 3: v = orient2d_plain(p[0], p[2], p[3], 0, 1); break;
      case 4: v = dsub(p[2][0], p[3][0]); break;
      case 5: v = dsub(p[2][1], p[3][1]); break;
      case 6: v = orient2d_plain(p[0], p[2], p[3], 0, 2); break;
      case 7: v = dsub(p[2][2], p[3][2]); break;
      case 8: v = orient2d_plain(p[0], p[2], p[3], 1, 2); break;
      case 9: v = orient2d_plain(p[0], p[1], p[3], 0, 1); break;
      case 10: v = dsub(p[1][0], p[3][0]); break;
      case 11: v = dsub(p[1][1], p[3][1]); break;
      default: v = dsub(p[0][0], p[3][0]); break;
    }
    if (v != 0.0) {
      r = v;
      depth = dd;
      break;
    }
  }
  int sg = (r > 0.0) - (r < 0.0);
  if (depth == 1 || depth == 3 || depth == 5 || depth == 8 || depth == 10) sg = -sg;
  if (parity) sg = -sg;
  return sg < 0 ? 1 : -1;
}

__device__ __forceinline__ int orient3d_sos(const double* a, const double* b, const double* c, const double* d,
                                            uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id,
                                            uint32_t* flags) {
  int s = orient3d(a, b, c, d, flags);
  if (s != 0) return s < 0 ? 1 : -1;
  return orient3d_sos_degenerate(a, b, c, d, ia, ib, ic, id);
}

__device__ __noinline__ int orient4d_sos_degenerate(const double* a, const double* b, const double* c,
                                                    const double* d, const double* e, uint32_t ia, uint32_t ib,
                                                    uint32_t ic, uint32_t id, uint32_t ie, uint32_t* flags) {
  uint32_t k[5] = {ia, ib, ic, id, ie};
  const double* p[5] = {a, b, c, d, e};
  int parity = sort_keys<5>(k, p);
  int sg = 1;
#pragma unroll 1
  for (int lv = 0; lv < 49; ++lv) {
    const SosLevel L = kSos4[lv];
    const double* x = p[L.p0];
    const double* y = p[L.p1];
    const double* z = p[L.p2];
    const double* w = p[L.p3];
    int s;
    switch (L.kind) {
      case kO3: s = orient3d(x, y, z, w, flags); break;
      case kO3L: s = orient3d_lifted(x, y, z, w, L.q0, L.q1, L.q2, flags); break;
      case kO2: {
        double v = orient2d_plain(x, y, z, L.q0, L.q1);
        s = (v > 0.0) - (v < 0.0);
        break;
      }
      case kO2L: s = orient2d_lifted(x, y, z, L.q0); break;
      case kO1: {
        double v = dsub(x[L.q0], y[L.q0]);
        s = (v > 0.0) - (v < 0.0);
        break;
      }
      case kO1L: s = orient1d_lifted(x, y); break;
      default: s = 1; break;
    }
    if (s != 0) {
      sg = L.flip ? -s : s;
      break;
    }
  }
  return parity ? -sg : sg;
}

// gDel3D sphere orientation with SoS: -1 = e inside the circumsphere of the
// (orient3d_sos = +1 oriented) tet a,b,c,d; never 0.
__device__ __forceinline__ int orient4d_sos(const double* a, const double* b, const double* c, const double* d,
                                            const double* e, uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id,
                                            uint32_t ie, uint32_t* flags) {
  int s = insphere(a, b, c, d, e, flags);
  if (s != 0) return s;
  return orient4d_sos_degenerate(a, b, c, d, e, ia, ib, ic, id, ie, flags);
}

}  // namespace
}  // namespace ex
}  // namespace wtet
