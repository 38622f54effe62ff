/* wtet_b200 -- C ABI of the B200-native 3D Delaunay tetrahedralizer.
 *
 * This is the drop-in boundary for half-potato/wtet's hot path: each entry
 * point replaces the reference interface named beside it (paths are inside the
 * reference project).  Plain pointers and sizes only; no CUDA or torch types.
 *
 * Semantics shared by all entry points
 *   - Input points are f32 xyz triples (AoS, n x 3).  They are normalised to
 *     [0,1]^3 exactly as src/lib.rs:313-337 does; triangulation runs on the
 *     normalised values.
 *   - Vertex ids of the output: 0..n-1 are the input points in input order,
 *     n..n+3 the super-tet vertices at (-100,-100,-100), (400,-100,-100),
 *     (-100,400,-100), (-100,-100,400) and n+4 the infinity vertex
 *     (src/gpu/mod.rs:147-162).
 *   - The tet set is the Delaunay triangulation of the points plus the four
 *     super vertices under the reference's Simulation of Simplicity
 *     (src/predicates.rs:106-675, tie-breaking by input index), plus the four
 *     infinity tets on the super tetrahedron's faces.  Every tet is oriented
 *     with orient3d_sos == +1 (Shewchuk det < 0, src/phase2.rs:404-410,490-498).
 *   - adjacency[4*t+f] = (neighbour << 5) | face_in_neighbour for the tet
 *     across the face opposite vertex f (src/types.rs:165-174), or
 *     WTET_INVALID where there is none.
 *   - Errors: every function returns WTET_OK (0) or a negative status;
 *     wtet_last_error() gives a per-thread message.
 */
#ifndef WTET_B200_H
#define WTET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WTET_INVALID 0xFFFFFFFFu

enum wtet_status {
  WTET_OK = 0,
  WTET_ERR_ARG = -1,         /* bad shape / size / pointer (Python: ValueError) */
  WTET_ERR_CAPACITY = -2,    /* caller-provided output buffer too small */
  WTET_ERR_NO_CONVERGE = -3, /* insertion rounds exceeded max_insert_iterations */
  WTET_ERR_CUDA = -4,        /* CUDA runtime failure or no usable device */
  WTET_ERR_INTERNAL = -5,    /* a device-side consistency check failed */
  WTET_ERR_PRECISION = -6    /* an exact-arithmetic buffer would overflow */
};

/* Insertion rule of the vote (src/types.rs:17-29).  Both rules give the same
 * triangulation; they change only which point a tet inserts first. */
enum wtet_insertion_rule { WTET_RULE_CIRCUMCENTER = 0, WTET_RULE_CENTROID = 1 };
/* Vote priority: the plain geometric vote or the learned scheduler. */
enum wtet_vote_mode { WTET_VOTE_PLAIN = 0, WTET_VOTE_LEARNED = 1 };

/* Mirrors GDelConfig (src/types.rs:32-61) plus the B200 additions. */
typedef struct wtet_config {
  uint32_t insertion_rule;         /* wtet_insertion_rule, default circumcenter */
  uint32_t enable_flipping;        /* accepted for compatibility; default 1 */
  uint32_t enable_sorting;         /* accepted; spatial order never changes SoS */
  uint32_t enable_hilbert_sorting; /* accepted; spatial order never changes SoS */
  uint32_t enable_splaying;        /* accepted; the device path needs no repair */
  uint32_t max_insert_iterations;  /* cap on insertion rounds per stratum, default 100 */
  uint32_t max_flip_iterations;    /* accepted for compatibility; default 10 */
  uint32_t vote_mode;              /* wtet_vote_mode, default plain */
  uint32_t block_size;             /* 0 = autotuned / default */
  uint32_t reserved[7];
} wtet_config;

/* Per-call statistics (the reference prints these as [DEBUG]/[TIMING] lines,
 * src/phase1.rs passim). */
typedef struct wtet_stats {
  uint32_t rounds;            /* insertion rounds over all strata */
  uint32_t strata;            /* BRIO strata (passes) */
  uint64_t inserted;          /* points inserted */
  uint64_t candidates;        /* cavity expansions attempted (incl. losers) */
  uint64_t big_cavities;      /* insertions that used the large-cavity path */
  uint64_t tets_created;      /* tets written over the whole run */
  uint64_t num_tets;          /* output tets (incl. super and infinity tets) */
  uint64_t walk_steps;        /* point-location steps */
  uint64_t num_failed;        /* points left out as exact duplicates */
  uint64_t kernel_launches;   /* CUDA kernels executed by the call (graph nodes included) */
  double device_ms;           /* device time of the call, CUDA events */
} wtet_stats;

/* Host-memory result owned by the library; release with wtet_result_free. */
typedef struct wtet_result {
  uint32_t* tets;          /* num_tets x 4 */
  uint32_t* adjacency;     /* num_tets x 4 */
  uint32_t* failed_verts;  /* num_failed (always 0 on the exact device path) */
  uint64_t num_tets;
  uint64_t num_failed;
  wtet_stats stats;
} wtet_result;

/* Defaults of GDelConfig::default() (src/types.rs:49-61). */
void wtet_config_default(wtet_config* cfg);

/* delaunay_3d (src/lib.rs:160-310) / wtet._core.delaunay (src/python.rs:166-257):
 * triangulate n >= 4 host points; the library allocates the result. */
int wtet_delaunay(const float* xyz, uint64_t n, const wtet_config* cfg, wtet_result* out);

/* Same, into caller-owned host buffers of `capacity` tets each (tets and
 * adjacency, capacity x 4 u32).  *num_tets receives the count; returns
 * WTET_ERR_CAPACITY (with *num_tets set) when capacity is too small.  Pinned
 * buffers make the copies fast.  failed_verts (optional, room for n) receives
 * the input indices left out as exact duplicates of an earlier point, count in
 * stats->num_failed (the reference leaves duplicate handling undefined,
 * src/tests.rs:1769-1781). */
int wtet_delaunay_into(const float* xyz, uint64_t n, const wtet_config* cfg, uint32_t* tets,
                       uint32_t* adjacency, uint64_t capacity, uint64_t* num_tets, uint32_t* failed_verts,
                       wtet_stats* stats);

/* Device-resident variant (zero-copy for torch / cupy buffers): d_xyz, d_tets
 * and d_adjacency are device pointers on the current device; the work runs on
 * `stream` (a cudaStream_t passed as void*, NULL = default stream) and the call
 * returns once the result is complete. */
int wtet_delaunay_device(const float* d_xyz, uint64_t n, const wtet_config* cfg, uint32_t* d_tets,
                         uint32_t* d_adjacency, uint64_t capacity, uint64_t* num_tets, wtet_stats* stats,
                         void* stream);

/* Batched triangulation (no reference counterpart; the reference runs one
 * cloud per delaunay_3d call, src/lib.rs:160-167): cloud c holds points
 * offsets[c]..offsets[c+1]-1 of xyz (offsets has num_clouds+1 entries).  All
 * clouds are triangulated together on the device.  Cloud c's tets are rows
 * tet_offsets[c]..tet_offsets[c+1]-1 of the output, with cloud-local vertex ids
 * and cloud-local adjacency, exactly as wtet_delaunay would give for that cloud
 * alone.  tet_offsets has num_clouds+1 entries. */
int wtet_delaunay_batched(const float* xyz, const uint64_t* offsets, uint32_t num_clouds,
                          const wtet_config* cfg, uint32_t* tets, uint32_t* adjacency, uint64_t capacity,
                          uint64_t* tet_offsets, wtet_stats* stats);

/* check_delaunay_quality (src/lib.rs:25-78) / wtet._core.check_quality
 * (src/python.rs:282-341), evaluated on the device with exact predicates:
 * counts faces between two all-real tets whose opposite vertex lies inside the
 * circumsphere (orient4d < 0), and the tets with only real vertices. */
int wtet_check_quality(const float* xyz, uint64_t n, const uint32_t* tets, const uint32_t* adjacency,
                       uint64_t m, uint64_t* violations, uint64_t* interior_tets);

/* Allocation-free exact quality check.  No counterpart in the reference.
 * For callers that must not allocate GPU memory during the call -- code that is
 * recording a CUDA stream capture, serving loops that cannot stall on or
 * fragment an allocator another framework owns, fixed memory budgets.  Same
 * result as wtet_check_quality, but d_xyz (n x 3 f32), d_tets and d_adjacency
 * (m x 4 u32) are device pointers and the scratch (normalised points, box,
 * counters) is a fixed 16 MiB array in device memory that each GPU holds while
 * the library is loaded.  n may not exceed WTET_NOALLOC_MAX_POINTS (larger n
 * returns WTET_ERR_ARG).  The first call on a device looks up that array's
 * address, so make it before any stream capture.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * Runs on `stream` (cudaStream_t as void*, NULL = default) and returns when the
 * counts are ready. */
#define WTET_NOALLOC_MAX_POINTS 1048576ull
int wtet_check_quality_noalloc(const float* d_xyz, uint64_t n, const uint32_t* d_tets,
                               const uint32_t* d_adjacency, uint64_t m, uint64_t* violations,
                               uint64_t* interior_tets, void* stream);

/* Upper bound on the output tet count for n points (for sizing buffers). */
uint64_t wtet_max_tets(uint64_t n);

void wtet_result_free(wtet_result* r);
const char* wtet_last_error(void);
/* initialize_gpu / gpu_info (src/python.rs:344-376). */
int wtet_initialize_gpu(char* buf, size_t len);
int wtet_gpu_info(char* buf, size_t len);
const char* wtet_version(void);

#ifdef __cplusplus
}
#endif
#endif /* WTET_B200_H */
