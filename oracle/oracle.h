/* Oracle (test infrastructure only) -- C interface loaded through ctypes by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.  It is the
 * checker, never the product: the wtet_b200 library does not link or call it.
 *
 * Parity pin: the predicates are pinned against exact rational arithmetic and the
 * reference's own predicate known-answer tests (src/predicates.rs:690-820,
 * src/tests.rs:12-80,1212-1281); Morton codes, the stride table and the
 * stratified order against src/morton.rs:88-151 and src/gpu/mod.rs:607-696;
 * the triangulation itself against the structural and exact local-Delaunay
 * validators of src/tests.rs:425-1090 (no reference test pins an exact tet set).
 */
#ifndef WTET_ORACLE_H
#define WTET_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_stats {
  uint64_t num_tets;         /* alive tets of DT(P + 4 super vertices) */
  uint64_t cavity_tets;      /* total tets deleted over all insertions */
  uint64_t boundary_faces;   /* total tets created over all insertions */
  uint32_t max_cavity;       /* largest single cavity (tets) */
  uint32_t max_boundary;     /* largest single cavity boundary (faces) */
  uint64_t walk_steps;       /* total point-location steps */
  uint64_t o3d_exact, o3d_sos, isp_exact, isp_sos; /* predicate stage counters */
  uint64_t cavity_hist[16];  /* insertions by cavity size: bucket k holds sizes in [2^k, 2^(k+1)) */
} oracle_stats;

/* src/lib.rs:313-337, bit-exact f32 arithmetic. */
void oracle_normalize(const float* xyz, uint64_t n, float* out, float* min3, float* scale);

/* src/morton.rs:22-80 */
uint32_t oracle_expand_bits(uint32_t v);
uint32_t oracle_interleave_bits(uint32_t x, uint32_t y, uint32_t z);
uint32_t oracle_morton_code(const float* p, const float* min3, const float* max3);
/* src/gpu/mod.rs:422-460: stable Morton order; mapping[i] = original index. */
void oracle_morton_order(const float* xyz, uint64_t n, uint32_t* mapping);
/* src/gpu/mod.rs:533-600 */
uint64_t oracle_initial_stride(uint64_t n);
void oracle_strided_order(uint64_t n, uint64_t initial_stride, uint32_t* order);

/* src/predicates.rs */
int oracle_orient3d(const double* a, const double* b, const double* c, const double* d);
int oracle_insphere(const double* a, const double* b, const double* c, const double* d, const double* e);
int oracle_orient3d_sos(const double* a, const double* b, const double* c, const double* d,
                        uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id);
int oracle_orient4d(const double* a, const double* b, const double* c, const double* d, const double* e,
                    uint32_t ia, uint32_t ib, uint32_t ic, uint32_t id, uint32_t ie);
int oracle_orient3d_lifted(const double* a, const double* b, const double* c, const double* d,
                           int p0, int p1, int p2);
int oracle_orient2d_lifted(const double* a, const double* b, const double* c, int p0);
int oracle_orient1d_lifted(const double* a, const double* b);

/* Bowyer-Watson Delaunay triangulation of the normalised points plus the four
 * super-tet vertices (src/phase2.rs:383-606 with walk-based point location).
 * order_mode: 0 = insert in index order (as the reference), 1 = stratified
 * Morton order (same output, faster).  Returns a handle, or NULL on failure
 * (oracle_last_error() says why). */
void* oracle_dt_run(const float* xyz, uint64_t n, int order_mode, oracle_stats* stats);
uint64_t oracle_dt_num_tets(void* h);
/* tets: (m,4) original vertex ids (super vertices n..n+3); adj: (m,4) encoded
 * (tet << 5) | face, 0xFFFFFFFF on the hull of the super tetrahedron. */
void oracle_dt_copy(void* h, uint32_t* tets, uint32_t* adj);
/* Input indices left out as exact duplicates (normalised coordinates equal to
 * an earlier point's), ascending. */
uint64_t oracle_dt_num_failed(void* h);
void oracle_dt_copy_failed(void* h, uint32_t* out);
void oracle_dt_free(void* h);
const char* oracle_last_error(void);

/* src/lib.rs:25-78 restated: violations among pairs of all-real tets. */
int64_t oracle_check_delaunay_quality(const float* xyz, uint64_t n, const uint32_t* tets,
                                      const uint32_t* adj, uint64_t m);
/* Exact local-Delaunay check of every face between two tets that do not use the
 * infinity vertex n+4, super vertices included (their coordinates are the
 * reference's, src/gpu/mod.rs:151-158).  Tets must be oriented with
 * orient3d_sos == +1.  Returns the violation count, or -1 on a structural error. */
int64_t oracle_check_local_delaunay(const float* xyz, uint64_t n, const uint32_t* tets,
                                    const uint32_t* adj, uint64_t m);
/* Canonical parity form (canon.cpp): tets without the infinity vertex n+4,
 * ids sorted in each row, rows sorted; adjacency re-indexed to that order
 * (neighbour << 5 | sorted slot of its opposite vertex), INVALID towards a
 * missing or infinity neighbour.  out_tets / out_adj need room for m rows;
 * returns the number of canonical rows. */
uint64_t oracle_canonical(const uint32_t* tets, const uint32_t* adj, uint64_t m, uint32_t n,
                          uint32_t* out_tets, uint32_t* out_adj);
/* Count of tets (without the infinity vertex) whose orient3d_sos != +1. */
int64_t oracle_check_orientation(const float* xyz, uint64_t n, const uint32_t* tets, uint64_t m);

#ifdef __cplusplus
}
#endif
#endif
