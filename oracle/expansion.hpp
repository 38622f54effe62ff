// Oracle (test infrastructure only): floating-point expansion arithmetic.
//
// Restates the error-free transformations and expansion algorithms published in
// J. R. Shewchuk, "Adaptive Precision Floating-Point Arithmetic and Fast Robust
// Geometric Predicates", Discrete & Computational Geometry 18:305-363, 1997
// (Two-Sum, Fast-Two-Sum, Split, Two-Product, Fast-Expansion-Sum with zero
// elimination, Scale-Expansion with zero elimination, Compress).  The reference
// (src/predicates.rs:9-21) reaches the same algorithms through the third-party
// crate geometry-predicates 0.3.0, which is not vendored; only signs of exact
// values are ever consumed, so any exact implementation agrees with it.
//
// Must be compiled with -ffp-contract=off: the transformations rely on every
// product and sum being rounded separately.
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

inline void two_sum(double a, double b, double& x, double& y) {
  x = a + b;
  double bv = x - a;
  double av = x - bv;
  y = (a - av) + (b - bv);
}

inline void fast_two_sum(double a, double b, double& x, double& y) {
  x = a + b;
  y = b - (x - a);
}

inline void two_diff(double a, double b, double& x, double& y) {
  x = a - b;
  double bv = a - x;
  double av = x + bv;
  y = (a - av) + (bv - b);
}

// Veltkamp/Dekker split into two 26-bit halves.
inline void split(double a, double& hi, double& lo) {
  double c = 134217729.0 * a;  // 2^27 + 1
  double big = c - a;
  hi = c - big;
  lo = a - hi;
}

inline void two_product(double a, double b, double& x, double& y) {
  x = a * b;
  double ahi, alo, bhi, blo;
  split(a, ahi, alo);
  split(b, bhi, blo);
  double e1 = x - ahi * bhi;
  double e2 = e1 - alo * bhi;
  double e3 = e2 - ahi * blo;
  y = alo * blo - e3;
}

// h = e + f ; inputs nonoverlapping, increasing magnitude; output with zeros removed.
// Returns the length of h (at least 1; a zero value is the one-component {0}).
inline int exp_sum(int elen, const double* e, int flen, const double* f, double* h) {
  double Q, Qnew, hh, enow = e[0], fnow = f[0];
  int ei = 0, fi = 0, hi = 0;
  if ((fnow > enow) == (fnow > -enow)) { Q = enow; enow = (++ei < elen) ? e[ei] : 0.0; }
  else { Q = fnow; fnow = (++fi < flen) ? f[fi] : 0.0; }
  if (ei < elen && fi < flen) {
    if ((fnow > enow) == (fnow > -enow)) { fast_two_sum(enow, Q, Qnew, hh); enow = (++ei < elen) ? e[ei] : 0.0; }
    else { fast_two_sum(fnow, Q, Qnew, hh); fnow = (++fi < flen) ? f[fi] : 0.0; }
    Q = Qnew;
    if (hh != 0.0) h[hi++] = hh;
    while (ei < elen && fi < flen) {
      if ((fnow > enow) == (fnow > -enow)) { two_sum(Q, enow, Qnew, hh); enow = (++ei < elen) ? e[ei] : 0.0; }
      else { two_sum(Q, fnow, Qnew, hh); fnow = (++fi < flen) ? f[fi] : 0.0; }
      Q = Qnew;
      if (hh != 0.0) h[hi++] = hh;
    }
  }
  while (ei < elen) { two_sum(Q, enow, Qnew, hh); enow = (++ei < elen) ? e[ei] : 0.0; Q = Qnew; if (hh != 0.0) h[hi++] = hh; }
  while (fi < flen) { two_sum(Q, fnow, Qnew, hh); fnow = (++fi < flen) ? f[fi] : 0.0; Q = Qnew; if (hh != 0.0) h[hi++] = hh; }
  if (Q != 0.0 || hi == 0) h[hi++] = Q;
  return hi;
}

// h = b * e ; zeros removed (at least one component).
inline int exp_scale(int elen, const double* e, double b, double* h) {
  double Q, sum, hh, p1, p0;
  int hi = 0;
  two_product(e[0], b, Q, hh);
  if (hh != 0.0) h[hi++] = hh;
  for (int i = 1; i < elen; ++i) {
    two_product(e[i], b, p1, p0);
    two_sum(Q, p0, sum, hh);
    if (hh != 0.0) h[hi++] = hh;
    fast_two_sum(p1, sum, Q, hh);
    if (hh != 0.0) h[hi++] = hh;
  }
  if (Q != 0.0 || hi == 0) h[hi++] = Q;
  return hi;
}

// Compress: the result is nonoverlapping with the most significant component last.
// h may alias e (the paper's in-place form: the first sweep writes h from the top
// down, the second from the bottom up, never overtaking the reads).
inline int exp_compress(int elen, const double* e, double* h) {
  double Q, q, Qnew;
  int bottom = elen - 1;
  Q = e[bottom];
  for (int i = elen - 2; i >= 0; --i) {
    fast_two_sum(Q, e[i], Qnew, q);
    if (q != 0.0) { h[bottom--] = Qnew; Q = q; } else { Q = Qnew; }
  }
  int top = 0;
  for (int i = bottom + 1; i < elen; ++i) {
    fast_two_sum(h[i], Q, Qnew, q);
    if (q != 0.0) h[top++] = q;
    Q = Qnew;
  }
  h[top++] = Q;
  return top;
}

inline void exp_negate(int n, double* e) { for (int i = 0; i < n; ++i) e[i] = -e[i]; }

inline int exp_sign(int n, const double* e) {
  double v = e[n - 1];
  return (v > 0.0) - (v < 0.0);
}

// h = e * f (product of two expansions) by repeated scaling and summing.
// h must hold 2*elen*flen doubles; tmp1/tmp2 likewise.
inline int exp_mul(int elen, const double* e, int flen, const double* f, double* h, double* t1, double* t2) {
  int hlen = exp_scale(elen, e, f[0], h);
  for (int i = 1; i < flen; ++i) {
    int tl = exp_scale(elen, e, f[i], t1);
    int nl = exp_sum(hlen, h, tl, t1, t2);
    for (int k = 0; k < nl; ++k) h[k] = t2[k];
    hlen = nl;
  }
  return hlen;
}

}  // namespace oracle
