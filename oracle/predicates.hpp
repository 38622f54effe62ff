// Oracle (test infrastructure only): exact geometric predicates with the
// reference's Simulation-of-Simplicity conventions.  Used by tests/, by the
// smoke check and by the CPU-baseline leg of bench.py -- never by the product.
#pragma once
#include <cstdint>

namespace oracle {

// Sign of Shewchuk's orient3d(a,b,c,d) = det[a-d; b-d; c-d], computed exactly.
// Positive when d lies below the plane of a,b,c (a,b,c counter-clockwise seen
// from above).  Reference: src/predicates.rs:14-16.
int orient3d_sign(const double* a, const double* b, const double* c, const double* d);

// Sign of Shewchuk's insphere(a,b,c,d,e), computed exactly.  Positive when e is
// inside the sphere through a,b,c,d and orient3d(a,b,c,d) > 0.
// Reference: src/predicates.rs:19-21.
int insphere_sign(const double* a, const double* b, const double* c, const double* d, const double* e);

// gDel3D orientation with SoS: +1 iff the exact det < 0 (ortToOrient), never 0.
// Reference: src/predicates.rs:77-86 and 106-208.
int orient3d_sos(const double* a, const double* b, const double* c, const double* d,
                 uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id);

// gDel3D sphere orientation with SoS: sign(insphere), -1 = e inside the
// circumsphere (a violation), never 0.  Reference: src/predicates.rs:450-675.
int orient4d_sos(const double* a, const double* b, const double* c, const double* d, const double* e,
                 uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id, uint32_t ie);

// Plain (non-SoS) sign of insphere: src/predicates.rs:679-688.
inline int orient4d_no_sos(const double* a, const double* b, const double* c, const double* d,
                           const double* e) {
  return insphere_sign(a, b, c, d, e);
}

// Sub-predicates of the SoS cascade, exposed for tests.
// orient3d_lifted with lifted=true: sign of det[[u, v, |p|^2, 1]] (rows a..d)
// where (u,v,t) = (p[perm0], p[perm1], p[perm2]); src/predicates.rs:390-435.
int orient3d_lifted_sign(const double* a, const double* b, const double* c, const double* d,
                         int perm0, int perm1, int perm2);
// orient2d_lifted with lifted=true: sign of det[[u, |p|^2, 1]] (rows a..c),
// u = p[perm0]; src/predicates.rs:255-291.
int orient2d_lifted_sign(const double* a, const double* b, const double* c, int perm0);
// orient1d_lifted with lifted=true: sign of |a|^2 - |b|^2; src/predicates.rs:229-252.
int orient1d_lifted_sign(const double* a, const double* b);

// Counters of how often each stage ran (process-wide, for diagnostics).
struct PredStats {
  uint64_t o3d_calls, o3d_exact, o3d_sos;
  uint64_t isp_calls, isp_exact, isp_sos;
};
PredStats pred_stats();
void pred_stats_reset();

}  // namespace oracle
