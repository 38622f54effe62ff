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
  uint32_t enable_sorting;         /* accepted: the device always inserts along a space-filling curve */
  uint32_t enable_hilbert_sorting; /* 1: insert in Hilbert instead of Morton order (never changes the result) */
  uint32_t enable_splaying;        /* accepted; the device path needs no repair */
  uint32_t max_insert_iterations;  /* cap on insertion rounds per stratum, default 100 */
  uint32_t max_flip_iterations;    /* accepted for compatibility; default 10 */
  uint32_t vote_mode;              /* wtet_vote_mode, default plain */
  /* Performance knobs.  0 = autotuned: the installed autotuner table's value
   * for the job's size bucket (wtet_autotune_set_table), else the default.
   * None of them changes the triangulation. */
  uint32_t block_size;             /* threads per block of the per-point kernels: 128, 256 (default), 512 */
  uint32_t rounds_per_graph;       /* insertion rounds replayed per CUDA-graph launch (default 8, max 64) */
  uint32_t overlap_shift;          /* next stratum starts when the current one has thinned to
                                      1/2^overlap_shift of its size (default 3) */
  uint32_t candidate_filter;       /* neighbourhood pre-claim before cavity growth: 1 = on (default),
                                      2 = off */
  uint32_t pool_factor;            /* cavity-pool entries per point (default 24, 4..64) */
  uint32_t learned_gate;           /* learned scheduler: rounds whose graph may see at most
                                      learned_gate x 1024 uninserted points take the network's claim
                                      priority, larger rounds the hashed one; 0 = default (2048) */
  uint32_t initial_capacity;       /* initial tet slots per point, in eighths; 0 = default (72, i.e. 9
                                      per point).  When a round runs out of slots the tet arrays grow
                                      in place by half (stats.capacity_grows counts it); small values
                                      force that path.  Never changes the result. */
  uint32_t reserved[1];
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
  uint64_t vote_winners;      /* points that won their tet's vote (insertion attempts) */
  uint64_t capacity_grows;    /* times the tet arrays grew during the run */
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

/* Every-face exact verification (extends check_delaunay_quality,
 * src/lib.rs:25-78, which tests only faces between two all-real tets): every
 * face between two tets that do not use the infinity vertex n+4 -- faces with
 * super vertices included, at the reference's super coordinates
 * (src/gpu/mod.rs:151-158) -- is tested with exact orient4d + SoS; every such
 * tet with exact orient3d + SoS (it must be +1, src/phase2.rs:404-410); every
 * adjacency link for symmetry and for sharing its face.  A complete output
 * passes with violations = misoriented = broken_links = bad_vertex_ids = 0 and
 * hull_faces = 4 (the super tetrahedron's faces, which border infinity tets):
 * it is then the Delaunay triangulation of the points plus the super vertices. */
typedef struct wtet_verify_report {
  uint64_t finite_tets;     /* tets without the infinity vertex */
  uint64_t faces_checked;   /* faces between two finite tets, each counted once */
  uint64_t violations;      /* of those: opposite vertex inside the circumsphere (orient4d < 0) */
  uint64_t misoriented;     /* finite tets with orient3d_sos != +1 */
  uint64_t broken_links;    /* links out of range, not symmetric, or not sharing the face */
  uint64_t hull_faces;      /* faces of finite tets with no finite neighbour */
  uint64_t bad_vertex_ids;  /* tets naming a vertex beyond n+4 */
} wtet_verify_report;

/* Host buffers (xyz n x 3 f32; tets, adjacency m x 4 u32). */
int wtet_verify(const float* xyz, uint64_t n, const uint32_t* tets, const uint32_t* adjacency, uint64_t m,
                wtet_verify_report* report);
/* Device pointers on the current device; runs on `stream` (cudaStream_t as
 * void*, NULL = default) and returns when the report is ready. */
int wtet_verify_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adjacency,
                       uint64_t m, wtet_verify_report* report, void* stream);

/* Canonical parity form (the sorted-vertex form in which two outputs compare
 * byte for byte; python.rs:282-341 / lib.rs:25-78 consume the reference's
 * unsorted rows): the tets without the infinity vertex n+4, vertex ids sorted
 * ascending in each row, rows sorted lexicographically; out_adjacency[4*i+s] =
 * (canonical index of the neighbour across the face opposite sorted slot s << 5)
 * | (sorted slot of the neighbour's opposite vertex), or WTET_INVALID towards a
 * missing or infinity neighbour.  out_tets / out_adjacency need room for m rows;
 * *num_rows receives the canonical row count. */
int wtet_canonicalize(const uint32_t* tets, const uint32_t* adjacency, uint64_t m, uint64_t n, uint32_t* out_tets,
                      uint32_t* out_adjacency, uint64_t* num_rows);
/* Same on device pointers of the current device, on `stream`. */
int wtet_canonicalize_device(const uint32_t* d_tets, const uint32_t* d_adjacency, uint64_t m, uint64_t n,
                             uint32_t* d_out_tets, uint32_t* d_out_adjacency, uint64_t* num_rows, void* stream);

/* Allocation-free exact quality check.  No counterpart in the reference.
 * For callers that cannot allocate GPU memory during the call: serving loops
 * whose GPU memory belongs to an allocator another framework owns (a
 * cudaMalloc from here would stall on, or fragment, that pool) and hosts whose
 * memory budget is fixed up front.  Same result as wtet_check_quality, but
 * d_xyz (n x 3 f32), d_tets and d_adjacency (m x 4 u32) are device pointers
 * and the scratch (normalised points, box, counters) is a fixed 16 MiB array
 * in device memory that each GPU holds while the library is loaded.  n may not
 * exceed WTET_NOALLOC_MAX_POINTS (larger n returns WTET_ERR_ARG).  The first
 * call on a device (and the first after that device's context was reset)
 * looks up that array's address, so make it before any stream capture.  Calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller.  Runs on `stream` (cudaStream_t as void*, NULL = default) and
 * returns when the counts are ready. */
#define WTET_NOALLOC_MAX_POINTS 1048576ull
int wtet_check_quality_noalloc(const float* d_xyz, uint64_t n, const uint32_t* d_tets,
                               const uint32_t* d_adjacency, uint64_t m, uint64_t* violations,
                               uint64_t* interior_tets, void* stream);

/* Signs of the device predicates as the insertion rounds evaluate them (FP32
 * stage, FP64 filter, exact expansion stage, SoS), for testing them against
 * other implementations of src/predicates.rs: for record i (points
 * pts[15i..15i+14] as five xyz triples a..e, used as given, and SoS keys
 * keys[5i..5i+4]) out3[i] = orient3d_sos(a,b,c,d) (+1 iff Shewchuk's
 * orient3d < 0, src/predicates.rs:106-217) and out4[i] = orient4d(a,b,c,d,e)
 * (sign of Shewchuk's insphere, SoS when 0: -1 = e inside,
 * src/predicates.rs:450-675).  Host buffers. */
int wtet_predicate_signs(const float* pts, const uint32_t* keys, uint64_t m, int32_t* out3, int32_t* out4);

/* ---- Learned insertion scheduler (no counterpart in the reference, which
 * orders insertions by the circumsphere determinant alone,
 * src/shaders/vote.wgsl:401-494).  Every tet votes for its point deepest in
 * its circumsphere; the vote winners then compete for their cavities by claim
 * keys (the smaller key wins a contested tet), hashed in the plain method.
 * With vote_mode = WTET_VOTE_LEARNED a 12 -> 64 -> 64 -> 64 -> 1 ReLU MLP,
 * fused into the kernel that turns votes into winners, predicts each winner's
 * probability of inserting in this round under hashed keys, and the winners
 * least likely to insert (crowded neighbourhoods, which set the number of
 * rounds) get the smallest keys.  It serves the rounds of the first strata
 * (learned_gate); the bulk rounds keep hashed keys.  Only the order of
 * insertions changes: the output is the same tet set.
 *
 * Parameters are FP32 in one flat array of WTET_MLP_PARAMS values:
 * W1[64][12] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4 (row =
 * output unit).  Inference rounds weights and activations to BF16 and
 * accumulates in FP32 on the tensor cores. */
#define WTET_MLP_FEATURES 12
#define WTET_MLP_HIDDEN 64
#define WTET_MLP_PARAMS 9217

/* Installs the weights used by WTET_VOTE_LEARNED (process-wide; uploaded to
 * each device on its next learned run).  count must be WTET_MLP_PARAMS. */
int wtet_learned_set_weights(const float* params, uint64_t count);
/* 1 when weights are installed, else 0. */
int wtet_learned_has_weights(void);

/* Training data from the plain method's own runs: triangulates the clouds
 * (layout of wtet_delaunay_batched) with the plain scheduler and records, for
 * 1 in 2^sample_shift of the vote winners in the rounds the learned scheduler
 * serves (cfg->learned_gate), the 12 features (features, capacity x 12) and
 * the label (labels, capacity): 1 if the winner inserted in its round, 0 if
 * not.
 * *count receives the records written (at most capacity).  The triangulation
 * itself is computed and discarded. */
int wtet_learned_collect(const float* xyz, const uint64_t* offsets, uint32_t num_clouds,
                         const wtet_config* cfg, uint32_t sample_shift, float* features, uint8_t* labels,
                         uint64_t capacity, uint64_t* count, wtet_stats* stats);

/* Mean binary cross-entropy (logits vs labels in {0,1}) of the FP32 network on
 * n samples and its gradient with respect to all parameters, computed by the
 * training kernels (forward + backward on the device, FP32). */
int wtet_mlp_loss_grad(const float* x, const float* y, uint64_t n, const float* params, float* loss,
                       float* grads);

typedef struct wtet_train_config {
  uint32_t epochs;    /* passes over the samples */
  uint32_t batch;     /* samples per Adam step */
  float lr;           /* Adam step size */
  float beta1, beta2; /* Adam moment decays */
  float eps;          /* Adam epsilon */
  uint64_t seed;      /* shuffling seed */
} wtet_train_config;

/* Trains the network on the device (forward and backward kernels, Adam):
 * params is read as the initial weights and receives the trained ones;
 * epoch_loss (optional, room for epochs) receives the mean loss per epoch. */
int wtet_mlp_train(const float* x, const float* y, uint64_t n, const wtet_train_config* tc, float* params,
                   float* epoch_loss);

/* Scores n feature rows with the installed weights through the same fused
 * BF16 tensor-core routine the learned vote runs (for testing it). */
int wtet_mlp_score(const float* x, uint64_t n, float* scores);

/* ---- Autotuner (no reference counterpart).  A table of size buckets, each
 * with the performance knobs measured fastest for it (wtet_b200.autotune
 * measures and persists it; the Python package installs its packaged table
 * on load).  A job uses the first entry of its kind (one cloud, or several)
 * whose max_points covers its total point count. */
typedef struct wtet_tune_entry {
  uint64_t max_points;       /* bucket: jobs with at most this many points in total */
  uint32_t batched;          /* 0: jobs of one cloud, 1: jobs of several clouds */
  uint32_t block_size;       /* knob values as in wtet_config (0 = default) */
  uint32_t rounds_per_graph;
  uint32_t overlap_shift;
  uint32_t candidate_filter;
  uint32_t pool_factor;
} wtet_tune_entry;

/* Installs the table (process-wide; replaces the previous one; count 0 clears). */
int wtet_autotune_set_table(const wtet_tune_entry* entries, uint32_t count);
/* Copies up to capacity entries of the installed table; *count = its size. */
int wtet_autotune_get_table(wtet_tune_entry* entries, uint32_t capacity, uint32_t* count);
/* The knobs a job of n points in num_clouds clouds would run with. */
int wtet_autotune_resolve(const wtet_config* cfg, uint64_t n, uint32_t num_clouds, wtet_config* out);

/* Cell indices of the point order (host functions, no GPU needed).  Points
 * are bucketed on a per-cloud grid of up to 2^10 cells per axis and inserted
 * in Morton order (default) or, with enable_hilbert_sorting, Hilbert order --
 * the reference's two sorts (src/morton.rs:22-80, src/hilbert.rs:20-38).
 * Neither changes the triangulation.  wtet_hilbert_index returns 0xFFFFFFFF
 * for bits outside 1..10. */
uint32_t wtet_morton_index(uint32_t x, uint32_t y, uint32_t z);
uint32_t wtet_hilbert_index(uint32_t x, uint32_t y, uint32_t z, uint32_t bits);

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
