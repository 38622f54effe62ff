// B200 Delaunay engine: parallel Bowyer-Watson cavity insertion with exact
// FP64 predicates and Simulation of Simplicity.
//
// What it replaces in half-potato/wtet: the phase-1 GPU loop (src/phase1.rs,
// src/gpu/*.rs, src/shaders/*.wgsl: vote, split, flip, relocate, compact) and
// the phase-2 host repair (src/phase2.rs, src/cpu/*).  Each insertion round
// keeps the triangulation exactly Delaunay: a point replaces the cavity of
// tets whose circumsphere contains it (the reference's own exact criterion,
// src/phase2.rs:428-470) by the star of the cavity boundary; concurrent
// insertions are admitted only when their cavities are disjoint and no cavity
// touches another's ring of neighbouring tets, which makes every round
// equivalent to some sequential order.  The result is therefore the unique
// SoS Delaunay triangulation, with no flip failures and nothing left to repair.
//
// Round structure (one insertion round over all clouds of a job; 9 kernels
// replayed from a CUDA graph):
//   k_activate    locate the new stratum's points (walk from the curve
//                 predecessor's tet)
//   (votes)       each uninserted point votes for its tet (64-bit atomicMax
//                 of score | ~point, src/shaders/vote.wgsl semantics) when it
//                 is located (k_activate) or relocated (k_relocate); a tet's
//                 vote stays valid until the tet is retired
//   k_cands       the winner of each tet becomes a candidate and pre-claims
//                 its tet's neighbourhood with its claim key (with the
//                 learned scheduler, k_cands_learned: the fused BF16 MLP sets
//                 the winners' claim priority in the rounds of the first
//                 strata)
//   k_bfs         candidates whose pre-claims all hold grow their cavities by
//                 breadth-first search with exact insphere (16 lanes per
//                 candidate), claiming cavity tets by 64-bit atomicMin of a
//                 round-stamped key; k_expand_big grows the huge ones, one
//                 block each
//   k_resolve     a candidate wins when it holds the minimum claim on all its
//                 cavity tets
//   k_shared      two winners whose cavities share a face both stay only if
//                 that face remains Delaunay (exact insphere); else the worse
//                 one steps back -- this exact test replaces a blanket
//                 exclusion of neighbouring cavities; the winners that stay
//                 get recycled / fresh slots for their new tets
//   k_write       new tets written, adjacency stitched through an edge table
//                 (rotation around boundary edges for the very largest
//                 cavities), cavity retired
//   k_relocate    points whose tet was retired walk (exact orient3d) from a
//                 tet of the inserting point; the rest keep their tet; the
//                 uninserted list is compacted with warp-aggregated appends;
//                 unused recycled slots carry over
//   k_end         list swap, stop conditions, and the next round's start:
//                 the next stratum once the current one has thinned
// The cavity search, shared-face test and tet writing take their work items
// dynamically (atomic cursors): cavity sizes vary by orders of magnitude.
// Strata: points are bucketed per cloud along a Morton (or Hilbert) curve
// (counting sort) and inserted in the reference's stratified stride order
// (src/gpu/mod.rs:533-600), each new stratum located by a walk from its
// predecessor on the curve.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "engine.cuh"
#include "exact.cuh"
#include "learned.cuh"
#include "order.cuh"
#include "devbuf.cuh"

// Resident blocks per SM the round kernels are compiled for (register caps):
// more resident warps hide more of the dependent-load latency, fewer
// registers spill more.
#ifndef WTET_BFS_MINB
#define WTET_BFS_MINB 8
#endif
#ifndef WTET_SHARED_MINB
#define WTET_SHARED_MINB 8
#endif
#ifndef WTET_WRITE_MINB
#define WTET_WRITE_MINB 8
#endif
// Rounds whose graph may see at most this many uninserted points run with one
// block per SM per kernel (a full wave of blocks costs more than their work).
#ifndef WTET_SMALL_ROUND_POINTS
#define WTET_SMALL_ROUND_POINTS 32768
#endif
#ifndef WTET_RELOC_MINB
#define WTET_RELOC_MINB 1
#endif

namespace wtet {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t DEAD = 0xFFFFFFFFu;  // tv.x of a retired tet; tv.y then forwards to a live tet
constexpr uint32_t INS_BIT = 0x80000000u;
// Cavity tiers: a lane group of k_bfs grows cavities of up to BIG_CAP tets;
// larger ones are re-grown the next round by a whole block (k_expand_big) in
// one of HUGE_SLOTS global slots of up to HUGE_CAP tets, with claim priority 0.
constexpr uint32_t BIG_CAP = 512;
constexpr uint32_t HUGE_CAP = 1u << 18;
constexpr uint32_t HUGE_SLOTS = 64;
// bigflag: tier (0 warp scratch, 2 huge slot) | kPending while the tier applies
// only from the next round (this round's partial claims carry its key).
constexpr uint8_t kPending = 0x80;
constexpr uint8_t kDup = 0x40;  // exact duplicate of an earlier point: never inserted
constexpr uint32_t WALK_LIMIT = 1u << 22;
// The start list is bucketed by the top bits of each winner's claim hash, so
// that the cavity search takes better-keyed winners first: a winner that
// meets a better one's claims then stops at its first contested tet instead
// of completing a cavity it loses later.
constexpr uint32_t kOrderBuckets = 16;
constexpr int ROT_LIMIT = 1 << 16;
constexpr int kMaxLevels = 15;

enum : uint32_t {
  kErrWalk = 1u << 0,
  kErrCapacity = 1u << 1,
  kErrRotate = 1u << 2,
  kErrSeed = 1u << 3,
  kErrPrec = ex::kErrPrecision,  // 1 << 4
  kErrHull = 1u << 5,
  kErrGuard = 1u << 6,  // an index failed a range guard (never expected)
  kErrBig = 1u << 7,    // a cavity outgrew the large-cavity slot
};

struct Counters {
  uint32_t n_next;        // uninserted points carried to the next round
  uint32_t n_cand;        // candidates that completed a cavity
  uint32_t pool_used;     // cavity-list pool entries
  uint32_t alloc_used;    // tet slots handed out this round (virtual index)
  uint32_t n_freed_next;  // tets retired this round
  uint32_t big_used;      // large-cavity slots used
  uint32_t n_inserted;    // winners this round
  uint32_t huge_used;     // huge-cavity slots used
  uint32_t btab_used;     // k_write's large edge tables handed out this round
  uint32_t bface_used;    // boundary-face list entries this round
  uint32_t work[4];       // dynamic work cursors of k_bfs, k_shared, k_write (one spare)
  uint32_t sbc[kOrderBuckets + 1];  // starts per order bucket (the last: overflow region)
  uint32_t err;           // error flags
  unsigned long long walk_steps;
  unsigned long long n_expanded;
  unsigned long long n_big;
  unsigned long long created;
};

// Round-loop state kept on the device, so that a round is a fixed kernel
// sequence that can be replayed from a CUDA graph without host round trips.
struct alignas(16) State {
  // read by every round kernel: the first 32 bytes, two vector loads
  uint32_t round;         // rounds executed
  uint32_t n_active;      // uninserted points in the current list
  uint32_t par;           // buffer parity: act[par] / freed[par] are current
  uint32_t n_freed_prev;  // recyclable slots in freed[par]
  uint32_t tet_top;       // first never-used tet slot
  uint32_t done;          // all points inserted
  uint32_t stop;          // 1 device error, 2 capacity exhausted, 3 no convergence
  uint32_t pad0;
  int32_t next_level;     // next stratum to locate (-1: none left)
  uint32_t stratum_size;  // size of the last located stratum
  uint32_t strata;
  uint32_t act_level, act_total, act_base;  // stratum located this round
  uint32_t max_rounds;
  uint32_t overlap_shift;
  uint32_t carry_used, carry_left;
  uint32_t log_used;      // scheduler training records reserved
  unsigned long long inserted;
  unsigned long long starts;  // vote winners that attempted an insertion
  // the last finished round's counts (the counters are reset when the next
  // round starts)
  uint32_t last_starts, last_cand, last_inserted, last_alloc;
};

// One tet slot: its vertex ids (retired: {DEAD, forward}) and its links,
// (neighbour << 2) | face, NONE on the super tetrahedron's hull -- one 32-byte
// sector, so that a visit reads both with one memory transaction.
struct __align__(32) Tet {
  uint4 v;
  uint4 n;
};
// The per-round words of one tet slot, likewise one sector: the cavity claim
// (64-bit key, smallest wins), the "tested outside" memo of the cavity search,
// the neighbourhood pre-claim and the vote (score | ~point).
struct __align__(32) Claim {
  unsigned long long cav;
  unsigned long long ring;
  unsigned long long pre;
  unsigned long long vote;
};

// Everything a kernel needs, passed by value.
struct Dev {
  State* st;
  uint32_t* act[2];
  uint32_t* freed[2];
  const struct CloudInfo* ci;
  const uint64_t* lvl_off;    // (maxtop+1) x (nc+1) first index of each cloud per stratum
  const uint32_t* lvl_total;  // points per stratum
  uint32_t nc;
  // vertices (internal ids)
  float4* pts;
  uint32_t* sos;     // SoS key = cloud-local input index (super vertices n_c..n_c+3)
  uint32_t* vcloud;  // cloud of each vertex
  uint32_t* vtet;    // a tet incident to each inserted vertex (hint, may be stale)
  uint32_t* loc;     // containing tet of uninserted points; INS_BIT once inserted
  uint8_t* bigflag;  // point needs the large-cavity path
  // tets
  Tet* T;
  Claim* C;
  uint4* nslot;
  uint32_t* bface;  // boundary faces of this round's winners, (tet << 2) | face, per winner contiguous
  uint32_t cap;
  uint32_t nv;  // vertices (range guard)
  // clouds
  uint32_t* centry;  // a live tet of each cloud
  // lists (act / freed above are the double-buffered ones)
  uint32_t* cand;
  uint32_t* cand_off;  // pool offset, or BIG flag | big slot
  uint32_t* cand_len;
  uint32_t* cand_base;
  uint32_t* cand_nf;   // boundary faces of each winning candidate (k_shared)
  uint8_t* st1;  // candidate owns its whole cavity
  uint8_t* st2;  // ... and no shared face with a better winner is violated
  uint32_t* bigcand;  // points taking the huge-cavity path this round
  uint32_t* starts;   // vote winners expanding their cavity this round, in order-bucket regions
  uint32_t start_rc;  // capacity of one order bucket's region
  uint32_t start_ovf; // offset of the overflow region
  uint32_t prefilter;
  uint32_t* wscratch; // one BIG_CAP cavity queue per lane group of k_bfs
  unsigned long long* etab_key;  // k_write's global edge tables, kEdgeSlotsG per warp
  uint32_t* etab_val;            // two values per slot
  uint32_t etab_warps;
  unsigned long long* btab_key;  // kBigTables tables of kBigTableSlots for larger cavities
  uint32_t* btab_val;
  uint32_t* pool;
  uint32_t pool_cap;
  uint32_t* big;
  Counters* ctr;
  int rule;
  // learned scheduler (vote_mode 1) and its training log (vote_mode 2)
  uint32_t vote_mode;
  uint8_t* losses;          // vote wins of each point that did not insert
  const mlp::Image* mlp;    // inference weights
  uint16_t* prio;           // learned scheduler: claim priority of this round's winners
  uint32_t learned_points;  // rounds with at most this many uninserted points use the network
  float* log_x;             // logged features (log_cap x 12)
  uint8_t* log_y;           // logged labels: the winner inserted this round (1) or not (0)
  uint32_t* log_pslot;      // log record of each winner this round, NONE if not recorded
  uint32_t log_cap;
  uint32_t log_shift;       // keep 1 in 2^log_shift winners
};

struct RoundArgs {
  // the current lists (the State's parity picks which buffer is which)
  uint32_t* active;
  uint32_t* active_next;
  uint32_t* freed_prev;
  uint32_t* freed_next;
  unsigned long long stamp;  // (~round mod 2^16) << 48
  uint32_t round;
  uint32_t n_active;
  uint32_t n_freed_prev;
  uint32_t tet_top;
  bool live;
};

// Reads this round's arguments from the device state, with the current list
// buffers.  D is not modified and its address never escapes into an
// out-of-line call, so the kernel parameter block is read in place rather
// than copied into each thread's local memory.
__device__ __forceinline__ RoundArgs load_round(const Dev& D) {
  // The state was written by earlier kernels of the sequence; kernel
  // boundaries make it visible, and no round kernel modifies these fields.
  const uint4 h0 = __ldcg(reinterpret_cast<const uint4*>(D.st));
  const uint4 h1 = __ldcg(reinterpret_cast<const uint4*>(D.st) + 1);
  RoundArgs R;
  R.live = !h1.y && !h1.z;  // !done && !stop
  R.round = h0.x;
  R.stamp = (unsigned long long)((~R.round) & 0xFFFFu) << 48;
  R.n_active = R.live ? h0.y : 0u;
  R.n_freed_prev = h0.w;
  R.tet_top = h1.x;
  const uint32_t par = h0.z & 1u;
  R.active = par ? D.act[1] : D.act[0];
  R.active_next = par ? D.act[0] : D.act[1];
  R.freed_prev = par ? D.freed[1] : D.freed[0];
  R.freed_next = par ? D.freed[0] : D.freed[1];
  return R;
}

__device__ __forceinline__ uint32_t comp(const uint4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(uint4& v, int i, uint32_t x) {
  if (i == 0) v.x = x;
  else if (i == 1) v.y = x;
  else if (i == 2) v.z = x;
  else v.w = x;
}
__device__ __forceinline__ void load_pt(const float4* pts, uint32_t v, double* o) {
  float4 q = pts[v];
  o[0] = q.x;
  o[1] = q.y;
  o[2] = q.z;
}

// Bijective 32-bit mixer (murmur3 finaliser) -> distinct priorities per round.
__device__ __forceinline__ uint32_t mix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}
// Claim key of candidate p: round stamp (16 bits, decreasing so that a new
// round's keys beat every stale one), priority (16 bits, smaller first) and a
// bijective hash of p that breaks ties and identifies the owner.  Smaller
// keys win.  Huge-cavity candidates (bigflag 2, at most HUGE_SLOTS a round)
// take priority 0: their cavities overlap many others, and at equal priority
// they would wait until their whole neighbourhood is quiet.  Every other
// candidate has priority 1, or with the learned scheduler the priority its
// network gave it this round (1..1023).
__device__ __forceinline__ unsigned long long make_key(const Dev& D, const RoundArgs& R, uint32_t p) {
  const unsigned long long prio = D.bigflag[p] == 2 ? 0u : (D.prio ? D.prio[p] : 1u);
  return R.stamp | (prio << 32) | mix32(p ^ (R.round * 0x9E3779B9u));
}

// Next work item of a warp-per-item kernel (dynamic: items differ widely in
// cost, so warps that finish early take more).
__device__ __forceinline__ uint32_t warp_next(uint32_t* cursor, uint32_t chunk) {
  uint32_t v = 0;
  if ((threadIdx.x & 31) == 0) v = atomicAdd(cursor, chunk);
  return __shfl_sync(0xFFFFFFFFu, v, 0);
}
// Items are taken kChunk at a time: one shared cursor serves every warp of
// the grid, and same-address atomics serialise in their L2 slice.  A round
// with fewer than kChunk items per warp takes them one at a time instead
// (there, a chunk would make a few warps do all the work in sequence).
constexpr uint32_t kChunk = 4;
__device__ __forceinline__ uint32_t chunk_for(uint32_t items) {
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  return items >= kChunk * warps ? kChunk : 1u;
}
// Stars of at most this many tets are written into their own cavity's slots
// (k_write holds one new tet per lane in registers until the warp has read
// the whole cavity).
constexpr uint32_t kInPlaceFaces = 32;

// Appends `pred` lanes to a list through one atomic per warp.
__device__ __forceinline__ uint32_t warp_append(uint32_t* ctr, bool pred) {
  unsigned mask = __activemask();
  unsigned ball = __ballot_sync(mask, pred);
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader && ball) base = atomicAdd(ctr, __popc(ball));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(ball & ((1u << lane) - 1u));
}

__device__ __forceinline__ int o3d_sos(const double* a, const double* b, const double* c, const double* d,
                                       uint32_t va, uint32_t vb, uint32_t vc, uint32_t vd, const uint32_t* sos,
                                       uint32_t* err) {
  int s = ex::orient3d(a, b, c, d, err);
  if (s != 0) return s < 0 ? 1 : -1;
  double A[3] = {a[0], a[1], a[2]}, B[3] = {b[0], b[1], b[2]}, C[3] = {c[0], c[1], c[2]}, Dd[3] = {d[0], d[1], d[2]};
  return ex::orient3d_sos_degenerate(A, B, C, Dd, sos[va], sos[vb], sos[vc], sos[vd]);
}

__device__ __forceinline__ int o4d_sos(const double* a, const double* b, const double* c, const double* d,
                                       const double* e, uint32_t va, uint32_t vb, uint32_t vc, uint32_t vd,
                                       uint32_t ve, const uint32_t* sos, uint32_t* err) {
  int s = ex::insphere(a, b, c, d, e, err);
  if (s != 0) return s;
  double A[3] = {a[0], a[1], a[2]}, B[3] = {b[0], b[1], b[2]}, C[3] = {c[0], c[1], c[2]}, Dd[3] = {d[0], d[1], d[2]};
  double E[3] = {e[0], e[1], e[2]};
  return ex::orient4d_sos_degenerate(A, B, C, Dd, E, sos[va], sos[vb], sos[vc], sos[vd], sos[ve], err);
}

// The same predicates on f32 points: the FP32 stage inline (it answers all
// but a tiny fraction of tests), the FP64 filter, exact stage and SoS out of
// line, so that the round kernels keep few registers live.
__device__ __noinline__ int o3d_sos_slow(float4 a, float4 b, float4 c, float4 d, uint32_t va, uint32_t vb,
                                         uint32_t vc, uint32_t vd, const uint32_t* sos, uint32_t* err) {
  const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z}, Dd[3] = {d.x, d.y, d.z};
  return o3d_sos(A, B, C, Dd, va, vb, vc, vd, sos, err);
}
__device__ __forceinline__ int o3d_sos_f(const float4& a, const float4& b, const float4& c, const float4& d,
                                         uint32_t va, uint32_t vb, uint32_t vc, uint32_t vd, const uint32_t* sos,
                                         uint32_t* err) {
  const int s = ex::orient3d_f32(a, b, c, d);
  if (s != 0) return s < 0 ? 1 : -1;
  return o3d_sos_slow(a, b, c, d, va, vb, vc, vd, sos, err);
}
__device__ __noinline__ int o4d_sos_slow(float4 a, float4 b, float4 c, float4 d, float4 e, uint32_t va,
                                         uint32_t vb, uint32_t vc, uint32_t vd, uint32_t ve, const uint32_t* sos,
                                         uint32_t* err) {
  const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z}, Dd[3] = {d.x, d.y, d.z};
  const double E[3] = {e.x, e.y, e.z};
  return o4d_sos(A, B, C, Dd, E, va, vb, vc, vd, ve, sos, err);
}
__device__ __forceinline__ int o4d_sos_f(const float4& a, const float4& b, const float4& c, const float4& d,
                                         const float4& e, uint32_t va, uint32_t vb, uint32_t vc, uint32_t vd,
                                         uint32_t ve, const uint32_t* sos, uint32_t* err) {
  const int s = ex::insphere_f32(a, b, c, d, e);
  if (s != 0) return s;
  return o4d_sos_slow(a, b, c, d, e, va, vb, vc, vd, ve, sos, err);
}

// The same insphere test out of line (FP32 stage included), for kernels that
// test a face only now and then: their main path then keeps fewer registers.
__device__ __noinline__ int o4d_sos_call(float4 a, float4 b, float4 c, float4 d, float4 e, uint32_t va, uint32_t vb,
                                         uint32_t vc, uint32_t vd, uint32_t ve, const uint32_t* sos,
                                         uint32_t* err) {
  return o4d_sos_f(a, b, c, d, e, va, vb, vc, vd, ve, sos, err);
}

// Visibility walk with exact orient3d + SoS from tet t to the tet containing p.
__device__ __forceinline__ uint32_t walk_to(const Dev& D, uint32_t t, uint32_t p, const float4& pq, uint32_t& steps) {
  int entry = -1;
  for (uint32_t s = 0; s < WALK_LIMIT; ++s) {
    if (t >= D.cap) {
      atomicOr(&D.ctr->err, kErrGuard);
      return 0;
    }
    const uint4 V = D.T[t].v;
    if (V.x >= D.nv || V.y >= D.nv || V.z >= D.nv || V.w >= D.nv) {
      atomicOr(&D.ctr->err, kErrGuard);
      return t;
    }
    const float4 P0 = D.pts[V.x], P1 = D.pts[V.y], P2 = D.pts[V.z], P3 = D.pts[V.w];
    int moved = -1;
    for (int i = 0; i < 4; ++i) {
      const int f = (i + int(s)) & 3;
      if (f == entry) continue;
      // the tet with vertex f replaced by p
      if (o3d_sos_f(f == 0 ? pq : P0, f == 1 ? pq : P1, f == 2 ? pq : P2, f == 3 ? pq : P3, f == 0 ? p : V.x,
                    f == 1 ? p : V.y, f == 2 ? p : V.z, f == 3 ? p : V.w, D.sos, &D.ctr->err) == -1) {
        moved = f;
        break;
      }
    }
    if (moved < 0) {
      steps += s + 1;
      return t;
    }
    const uint32_t n = comp(D.T[t].n, moved);
    if (n == NONE) {
      atomicOr(&D.ctr->err, kErrWalk);
      return t;
    }
    t = n >> 2;
    entry = int(n & 3);
  }
  atomicOr(&D.ctr->err, kErrWalk);
  return t;
}

// ---------------------------------------------------------------- setup ----

// Ordered-uint encoding of floats for atomic min / max.
__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

__device__ __forceinline__ uint32_t cloud_of(const uint64_t* off, uint32_t nc, uint64_t i) {
  uint32_t lo = 0, hi = nc;  // off[lo] <= i < off[hi]
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-cloud bounding box (src/lib.rs:315-323): block-reduce, then atomics.
__global__ void k_bbox(const float* xyz, const uint64_t* off, uint32_t nc, uint64_t n, uint32_t* mn, uint32_t* mx) {
  __shared__ uint32_t smn[3], smx[3];
  __shared__ uint32_t scloud_first, scloud_last;
  uint64_t base = uint64_t(blockIdx.x) * blockDim.x;
  uint64_t i = base + threadIdx.x;
  if (threadIdx.x == 0) {
    smn[0] = smn[1] = smn[2] = 0xFFFFFFFFu;
    smx[0] = smx[1] = smx[2] = 0u;
    scloud_first = cloud_of(off, nc, base);
    uint64_t last = min(base + blockDim.x, n) - 1;
    scloud_last = cloud_of(off, nc, last);
  }
  __syncthreads();
  bool uniform = scloud_first == scloud_last;
  if (i < n) {
    uint32_t c = uniform ? scloud_first : cloud_of(off, nc, i);
    for (int k = 0; k < 3; ++k) {
      float v = xyz[3 * i + k];
      if (v != v) continue;  // NaN is ignored, as f32::min / f32::max do
      uint32_t o = f2o(v);
      if (uniform) {
        atomicMin(&smn[k], o);
        atomicMax(&smx[k], o);
      } else {
        atomicMin(&mn[3 * c + k], o);
        atomicMax(&mx[3 * c + k], o);
      }
    }
  }
  __syncthreads();
  if (uniform && threadIdx.x < 3) {
    atomicMin(&mn[3 * scloud_first + threadIdx.x], smn[threadIdx.x]);
    atomicMax(&mx[3 * scloud_first + threadIdx.x], smx[threadIdx.x]);
  }
}

struct CloudInfo {
  uint64_t off;      // first input point
  uint32_t n;        // points
  uint32_t vbase;    // internal id of its first point (super vertices follow the points)
  uint32_t bbase;    // first Morton bucket
  uint32_t bbits;    // bits per axis of its buckets
  uint32_t top;      // top stratum level (log2 of the initial stride)
  uint32_t pad;
};



// Normalises (src/lib.rs:325-334, f32 arithmetic) and buckets each point by a
// per-cloud Morton code; counts bucket sizes.
__global__ void k_normalize(const float* xyz, const uint64_t* off, const CloudInfo* ci, uint32_t nc, uint64_t n,
                            const uint32_t* mn, const uint32_t* mx, float4* tmp, uint32_t* bucket,
                            uint32_t* hist, int hilbert) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = cloud_of(off, nc, i);
  float lo[3], ext[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = o2f(mn[3 * c + k]);
    ext[k] = o2f(mx[3 * c + k]) - lo[k];
  }
  float s = fmaxf(fmaxf(fmaxf(ext[0], ext[1]), ext[2]), 1e-10f);
  float q[3];
  for (int k = 0; k < 3; ++k) q[k] = __fdiv_rn(__fsub_rn(xyz[3 * i + k], lo[k]), s);
  tmp[i] = make_float4(q[0], q[1], q[2], 0.f);
  CloudInfo C = ci[c];
  uint32_t res = 1u << C.bbits;
  uint32_t code[3];
  for (int k = 0; k < 3; ++k) {
    float v = q[k] * float(res);
    uint32_t u = (v > 0.f) ? (v >= float(res) ? res - 1 : uint32_t(v)) : 0u;
    code[k] = u;
  }
  uint32_t b = C.bbase + (hilbert ? hilbert3(code[0], code[1], code[2], C.bbits) : morton3(code[0], code[1], code[2]));
  bucket[i] = b;
  atomicAdd(&hist[b], 1u);
}

// Exact duplicates (equal normalised coordinates within a cloud): an open
// addressing table keeps the lowest input index per coordinate triple.
__device__ __forceinline__ uint32_t coord_hash(float4 q, uint32_t c) {
  uint32_t h = mix32(__float_as_uint(q.x) ^ 0x9E3779B9u);
  h = mix32(h ^ __float_as_uint(q.y));
  h = mix32(h ^ __float_as_uint(q.z));
  return mix32(h ^ c);
}
__device__ __forceinline__ bool same_point(float4 a, float4 b) {
  return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
         __float_as_uint(a.z) == __float_as_uint(b.z);
}

__global__ void k_dedup_insert(const uint64_t* off, uint32_t nc, uint64_t n, const float4* tmp, uint32_t* table,
                               uint32_t mask) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 q = tmp[i];
  uint32_t c = cloud_of(off, nc, i);
  uint32_t slot = coord_hash(q, c) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    uint32_t cur = atomicCAS(&table[slot], NONE, uint32_t(i));
    if (cur == NONE) return;
    if (same_point(tmp[cur], q) && cloud_of(off, nc, cur) == c) {
      atomicMin(&table[slot], uint32_t(i));
      return;
    }
    slot = (slot + 1) & mask;
  }
}

__global__ void k_dedup_mark(const uint64_t* off, uint32_t nc, uint64_t n, const float4* tmp,
                             const uint32_t* table, uint32_t mask, uint8_t* dup, uint32_t* ndup) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 q = tmp[i];
  uint32_t c = cloud_of(off, nc, i);
  uint32_t slot = coord_hash(q, c) & mask;
  uint8_t d = 0;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    uint32_t cur = table[slot];
    if (cur == NONE) break;
    if (same_point(tmp[cur], q) && cloud_of(off, nc, cur) == c) {
      d = cur != uint32_t(i);
      break;
    }
    slot = (slot + 1) & mask;
  }
  dup[i] = d;
  if (d) atomicAdd(ndup, 1u);
}

// Scatters points into Morton order inside their cloud.
__global__ void k_scatter_points(const uint64_t* off, const CloudInfo* ci, uint32_t nc, uint64_t n,
                                 const float4* tmp, const uint32_t* bucket, uint32_t* cursor, const uint8_t* dup,
                                 Dev D) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = cloud_of(off, nc, i);
  uint32_t pos = atomicAdd(&cursor[bucket[i]], 1u);  // global Morton position
  uint32_t v = pos + 4u * c;                          // skip the super vertices of earlier clouds
  D.pts[v] = tmp[i];
  D.sos[v] = uint32_t(i - ci[c].off);
  D.vcloud[v] = c;
  D.loc[v] = 0;
  D.bigflag[v] = dup[i] ? kDup : 0;
  D.vtet[v] = NONE;
}

// Unused tet slots: dead, no links; claims and pre-claims at the largest key
// (any claim beats them), no vote.
__global__ void k_init_slots(Tet* T, Claim* C, uint64_t from, uint64_t to) {
  for (uint64_t i = from + uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < to;
       i += uint64_t(gridDim.x) * blockDim.x) {
    T[i].v = make_uint4(DEAD, DEAD, DEAD, DEAD);
    T[i].n = make_uint4(NONE, NONE, NONE, NONE);
    C[i] = Claim{~0ull, ~0ull, ~0ull, 0ull};
  }
}

// Super vertices (src/gpu/mod.rs:151-158) and the initial super tet of every
// cloud, oriented with orient3d_sos > 0 (src/phase2.rs:404-410).
__global__ void k_init_clouds(const CloudInfo* ci, uint32_t nc, Dev D) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  CloudInfo C = ci[c];
  const float S[4][3] = {{-100.f, -100.f, -100.f}, {400.f, -100.f, -100.f}, {-100.f, 400.f, -100.f},
                         {-100.f, -100.f, 400.f}};
  uint32_t s0 = C.vbase + C.n;
  for (int k = 0; k < 4; ++k) {
    D.pts[s0 + k] = make_float4(S[k][0], S[k][1], S[k][2], 0.f);
    D.sos[s0 + k] = C.n + k;
    D.vcloud[s0 + k] = c;
    D.vtet[s0 + k] = c;
    D.loc[s0 + k] = INS_BIT;
  }
  double P[4][3];
  for (int k = 0; k < 4; ++k) load_pt(D.pts, s0 + k, P[k]);
  int o = o3d_sos(P[0], P[1], P[2], P[3], s0, s0 + 1, s0 + 2, s0 + 3, D.sos, &D.ctr->err);
  D.T[c].v = (o > 0) ? make_uint4(s0, s0 + 1, s0 + 2, s0 + 3) : make_uint4(s0 + 1, s0, s0 + 2, s0 + 3);
  D.T[c].n = make_uint4(NONE, NONE, NONE, NONE);
  D.centry[c] = c;
}

// ---------------------------------------------------------------- rounds ----

// Vote score: larger = inserted first.  Circumcenter rule: depth of p inside
// the circumsphere (f32 insphere, src/shaders/vote.wgsl:401-494 semantics);
// centroid rule: inverse squared distance to the centroid.
__device__ __forceinline__ float vote_score(const float4* pts, uint4 V, float4 q, int rule) {
  float4 a = pts[V.x], b = pts[V.y], c = pts[V.z], d = pts[V.w];
  if (rule == 1) {
    float cx = 0.25f * (a.x + b.x + c.x + d.x) - q.x;
    float cy = 0.25f * (a.y + b.y + c.y + d.y) - q.y;
    float cz = 0.25f * (a.z + b.z + c.z + d.z) - q.z;
    return 1.0f / (1e-30f + cx * cx + cy * cy + cz * cz);
  }
  float aex = a.x - q.x, aey = a.y - q.y, aez = a.z - q.z;
  float bex = b.x - q.x, bey = b.y - q.y, bez = b.z - q.z;
  float cex = c.x - q.x, cey = c.y - q.y, cez = c.z - q.z;
  float dex = d.x - q.x, dey = d.y - q.y, dez = d.z - q.z;
  float ab = aex * bey - bex * aey, bc = bex * cey - cex * bey, cd = cex * dey - dex * cey;
  float da = dex * aey - aex * dey, ac = aex * cey - cex * aey, bd = bex * dey - dex * bey;
  float abc = aez * bc - bez * ac + cez * ab, bcd = bez * cd - cez * bd + dez * bc;
  float cda = cez * da + dez * ac + aez * cd, dab = dez * ab + aez * bd + bez * da;
  float al = aex * aex + aey * aey + aez * aez, bl = bex * bex + bey * bey + bez * bez;
  float cl = cex * cex + cey * cey + cez * cez, dl = dex * dex + dey * dey + dez * dez;
  float det = (dl * abc - cl * dab) + (bl * cda - al * bcd);
  float depth = -det;  // tets have Shewchuk orient3d < 0, so inside means det < 0
  return (depth > 0.f && depth < 3.0e38f) ? depth : 0.f;
}

// The vote of uninserted point p for tet t: 64-bit atomicMax of (score, ~p),
// so each tet's vote word names its point with the largest score (ties: the
// smallest index).  A tet's points change only when it is retired, so its
// vote word stays valid until then: points vote when they are located
// (k_activate) or relocated (k_relocate), and k_write clears the word of
// every slot it writes a new tet into.
__device__ __forceinline__ void cast_vote(const Dev& D, uint32_t p, uint32_t t) {
  if (t >= D.cap) {
    atomicOr(&D.ctr->err, kErrGuard);
    return;
  }
  const uint4 V = D.T[t].v;
  if (V.x >= D.nv || V.y >= D.nv || V.z >= D.nv || V.w >= D.nv) {
    atomicOr(&D.ctr->err, kErrGuard);
    return;
  }
  const float sc = vote_score(D.pts, V, D.pts[p], D.rule);
  atomicMax(&D.C[t].vote, ((unsigned long long)__float_as_uint(sc) << 32) | (unsigned long long)(~p));
}

// Locates the points of one stratum: walk from the tet of the point one
// stride earlier on the Morton curve (a point of an earlier stratum: its tet
// once inserted, else the tet that still contains it).  The located points are
// appended to the uninserted list at position `base`.
__global__ void __launch_bounds__(512, WTET_RELOC_MINB) k_activate(Dev D) {
  RoundArgs R = load_round(D);
  if (!R.live) return;
  volatile State* S = D.st;
  const uint32_t total = S->act_total;
  if (total == 0) return;
  const uint32_t level = S->act_level, base = S->act_base, nc = D.nc;
  const uint64_t* lvl_off = D.lvl_off + size_t(level) * (nc + 1);
  const CloudInfo* ci = D.ci;
  uint32_t steps = 0;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nc;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (lvl_off[mid] <= idx) lo = mid;
      else hi = mid;
    }
    uint32_t c = lo;
    CloudInfo C = ci[c];
    uint32_t k = idx - uint32_t(lvl_off[c]);
    uint32_t stride = 1u << level;
    uint32_t pos = (level == C.top) ? k * stride : (2u * k + 1u) * stride;
    uint32_t p = C.vbase + pos;
    R.active[base + idx] = p;
    if (D.bigflag[p] & kDup) continue;  // never located, dropped by k_relocate
    uint32_t t = NONE;
    if (level < C.top) {
      uint32_t hv = p - stride;
      uint32_t hl = D.loc[hv];
      uint32_t h = (hl & INS_BIT) ? D.vtet[hv] : hl;
      if (h != NONE && h < D.cap) {
        uint4 V = D.T[h].v;
        if (V.x < D.nv && D.vcloud[V.x] == c) t = h;
      }
    }
    if (t == NONE) t = D.centry[c];
    const uint32_t lt = walk_to(D, t, p, D.pts[p], steps);
    D.loc[p] = lt;
    D.bigflag[p] = 0;
    cast_vote(D, p, lt);
  }
  if (steps) atomicAdd(&D.ctr->walk_steps, (unsigned long long)steps);
}

// Prefix of the order buckets' start counts, in shared memory (sp has
// kOrderBuckets + 2 entries; sp[kOrderBuckets + 1] is the total).  Called by
// every thread of the block.
__device__ __forceinline__ void load_start_prefix(const Dev& D, uint32_t* sp) {
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t b = 0; b <= kOrderBuckets; ++b) {
      sp[b] = acc;
      const uint32_t c = __ldcg(&D.ctr->sbc[b]);
      acc += b < kOrderBuckets ? min(c, D.start_rc) : c;
    }
    sp[kOrderBuckets + 1] = acc;
  }
  __syncthreads();
}

// Start i of the round in bucket order.
__device__ __forceinline__ uint32_t start_at(const Dev& D, const uint32_t* sp, uint32_t i) {
  uint32_t b = 0;
#pragma unroll
  for (uint32_t k = 1; k <= kOrderBuckets; ++k) b += i >= sp[k] ? 1u : 0u;
  const uint32_t region = b < kOrderBuckets ? b * D.start_rc : D.start_ovf;
  return D.starts[region + (i - sp[b])];
}


// Inverse of mix32: recovers the point that owns a claim key.
__device__ __forceinline__ uint32_t unmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x7ed1b41du;
  h ^= (h >> 13) ^ (h >> 26);
  h *= 0xa5cb9243u;
  h ^= h >> 16;
  return h;
}
__device__ __forceinline__ uint32_t key_owner(const RoundArgs& R, unsigned long long key) {
  return unmix32(uint32_t(key)) ^ (R.round * 0x9E3779B9u);
}
__device__ __forceinline__ bool this_round(const RoundArgs& R, unsigned long long key) {
  return (key >> 48) == (R.stamp >> 48);
}

// Pre-claims of vote winner p in tet t with its key: t and its face
// neighbours, and with `two` also the other neighbours of those (up to 17
// tets).  A candidate whose pre-claimed tets are not all its own would lose its
// cavity to a better one, so it skips cavity growth (k_bfs checks them).
__device__ __forceinline__ void pre_claim(const Dev& D, uint32_t t, unsigned long long key, bool two) {
  atomicMin(&D.C[t].pre, key);
  const uint4 N = D.T[t].n;
  for (int f = 0; f < 4; ++f) {
    const uint32_t nb = comp(N, f);
    if (nb == NONE || (nb >> 2) >= D.cap) continue;
    atomicMin(&D.C[nb >> 2].pre, key);
    if (!two) continue;
    const uint4 N2 = D.T[nb >> 2].n;
    for (int g = 1; g < 4; ++g) {  // the three faces other than the one back to t
      const uint32_t nb2 = comp(N2, (int(nb & 3) + g) & 3);
      if (nb2 != NONE && (nb2 >> 2) < D.cap) atomicMin(&D.C[nb2 >> 2].pre, key);
    }
  }
}

// Tet k of p's pre-claim set (k = 0: t; k = 1 + 4i: face neighbour i;
// k = 1 + 4i + j, j = 1..3: the j-th other neighbour of face neighbour i), or
// NONE.
__device__ __forceinline__ uint32_t pre_claim_tet(const Dev& D, uint32_t t, uint32_t k) {
  if (k == 0) return t;
  const uint32_t i = (k - 1) / 4, j = (k - 1) % 4;
  const uint32_t nb = comp(D.T[t].n, int(i));
  if (nb == NONE || (nb >> 2) >= D.cap) return NONE;
  if (j == 0) return nb >> 2;
  const uint32_t nb2 = comp(D.T[nb >> 2].n, (int(nb & 3) + int(j)) & 3);
  return (nb2 == NONE || (nb2 >> 2) >= D.cap) ? NONE : nb2 >> 2;
}

// Features of vote winner p in its tet t (vote = the tet's vote word): the
// tet's shape and the winner's place in it, how many face neighbours hold a
// vote winner this round (a vote word is cleared when its tet's points move
// on, so a non-zero word is this round's) and how many of those winners have
// a larger vote score, the winner's earlier failed wins and the round's
// scale.  k_cands has already counted this win in losses[p].
__device__ __forceinline__ void winner_features(const Dev& D, const RoundArgs& R, uint32_t p, uint32_t t,
                                                unsigned long long vote, float* f) {
  const uint4 V = D.T[t].v;
  const uint4 N = D.T[t].n;
  uint32_t r1 = 0, r2 = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t nb = comp(N, i);
    if (nb == NONE || (nb >> 2) >= D.cap) continue;
    const unsigned long long nv = __ldcg(&D.C[nb >> 2].vote);
    if (nv != 0ull) ++r1;
    if ((nv >> 32) > (vote >> 32)) ++r2;  // a rival with a larger vote score
  }
  const uint32_t lost = D.losses[p] ? D.losses[p] - 1u : 0u;
  const uint32_t stratum = __ldcg(&D.st->stratum_size);
  mlp::features(D.pts[V.x], D.pts[V.y], D.pts[V.z], D.pts[V.w], D.pts[p], __uint_as_float(uint32_t(vote >> 32)),
                r1, r2, R.round, lost, R.n_active, stratum, f);
}

// Scheduler log (training data), after k_cands: in the rounds the learned
// scheduler serves (at most learned_points uninserted points), the features
// of 1 in 2^log_shift of the vote winners; label 0 here, set to 1 by k_write
// when the winner inserts in this round.
__global__ void k_log_features(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live || R.n_active > D.learned_points) return;
  __shared__ uint32_t sp[kOrderBuckets + 2];
  load_start_prefix(D, sp);
  const uint32_t nstart = sp[kOrderBuckets + 1];
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nstart; s += gridDim.x * blockDim.x) {
    const uint32_t p = start_at(D, sp, s);
    D.log_pslot[p] = NONE;
    if ((mix32(p ^ (R.round * 0x27D4EB2Fu)) & ((1u << D.log_shift) - 1u)) != 0u) continue;
    const uint32_t slot = atomicAdd(&D.st->log_used, 1u);
    if (slot >= D.log_cap) continue;
    D.log_pslot[p] = slot;
    D.log_y[slot] = 0;
    const uint32_t t = D.loc[p];
    float f[mlp::kIn];
    winner_features(D, R, p, t, __ldcg(&D.C[t].vote), f);
#pragma unroll
    for (int k = 0; k < mlp::kIn; ++k) D.log_x[size_t(slot) * mlp::kIn + k] = f[k];
  }
}

// Shared memory of the learned candidate kernel: the network's weights and
// one staged feature row per lane.
constexpr uint32_t kCandWarps = 8;  // k_cands_learned runs 256-thread blocks
struct CandSmem {
  mlp::Smem S;
  uint32_t rows[kCandWarps][32 * mlp::kRowStride];
  float outs[kCandWarps][32];
};

// Candidates: the vote winner of each tet (the reference's pick_winner_point
// and build_insert_list, src/shaders/vote.wgsl:508-616).  Points whose cavity
// outgrew the warp scratch in an earlier round go to the huge-cavity path.
// With kLearned, the fused network scores the warp's winners and sets their
// claim priority; the start list is bucketed by that priority (better first)
// instead of by the claim hash.
template <bool kLearned>
__device__ __forceinline__ void cands_body(const Dev& D, const RoundArgs& R, CandSmem* sm) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < R.n_active; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    bool start = false;
    uint32_t p = 0, t = 0;
    unsigned long long vote = 0;
    if (i < R.n_active) {
      p = R.active[i];
      const uint8_t tier = D.bigflag[p];
      t = D.loc[p];
      if (!(tier & kDup) && t < D.cap) vote = D.C[t].vote;
      if (!(tier & kDup) && t < D.cap && uint32_t(vote) == ~p) {
        if (D.losses && D.losses[p] < 255u) D.losses[p] += 1u;
        if (tier == 2) {
          uint32_t b = atomicAdd(&D.ctr->huge_used, 1u);
          if (b < HUGE_SLOTS) D.bigcand[b] = p;
        } else if (!tier) {
          start = true;
          D.st1[p] = 0;
          D.st2[p] = 0;
        }
      }
    }
    uint32_t b = 0;
    if constexpr (kLearned) {
      // the warp scores only if one of its points is a winner (warp-uniform)
      if (__any_sync(0xFFFFFFFFu, start)) {
        const uint32_t w = threadIdx.x >> 5;
        float f[mlp::kIn];
#pragma unroll
        for (int k = 0; k < mlp::kIn; ++k) f[k] = 0.f;
        if (start) winner_features(D, R, p, t, vote, f);
        mlp::stage_row(sm->rows[w] + lane * mlp::kRowStride, f);
        __syncwarp();
        mlp::score32(sm->S, sm->rows[w], sm->outs[w]);
        if (start) {
          float sc = sm->outs[w][lane];
          sc = (sc == sc) ? fminf(fmaxf(sc, -20.f), 20.f) : 0.f;
          // predicted probability of inserting under hashed keys: the least
          // likely (crowded neighbourhoods) claim first
          const float pr = 1.f / (1.f + __expf(-sc));
          const uint32_t prio = 1u + uint32_t(fminf(pr * 1022.f + 0.5f, 1022.f));
          D.prio[p] = uint16_t(prio);
          b = prio >> 6;  // 16 order buckets
        }
        __syncwarp();
      }
    } else {
      if (start && D.prio) D.prio[p] = 1;
      b = start ? (mix32(p ^ (R.round * 0x9E3779B9u)) >> 28) : 0u;
    }
    if (start && D.prefilter) pre_claim(D, t, make_key(D, R, p), false);
    warp_append(&D.ctr->big_used, start);  // total count
    const unsigned grp = __match_any_sync(0xFFFFFFFFu, start ? b : 0xFFFFFFFFu);
    const uint32_t leader = uint32_t(__ffs(grp) - 1);
    uint32_t base = 0;
    if (start && lane == leader) base = atomicAdd(&D.ctr->sbc[b], uint32_t(__popc(grp)));
    base = __shfl_sync(0xFFFFFFFFu, base, int(leader));
    if (start) {
      const uint32_t slot = base + uint32_t(__popc(grp & ((1u << lane) - 1u)));
      if (slot < D.start_rc) {
        D.starts[b * D.start_rc + slot] = p;
      } else {  // a bucket beyond its region (never expected): the overflow region
        D.starts[D.start_ovf + atomicAdd(&D.ctr->sbc[kOrderBuckets], 1u)] = p;
      }
    }
  }
}

__global__ void k_cands(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  cands_body<false>(D, R, nullptr);
}

// The learned scheduler's candidate kernel (256-thread blocks).
__global__ void __launch_bounds__(256) k_cands_learned(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  __shared__ __align__(16) CandSmem sm;
  mlp::load_image(sm.S, D.mlp);
  __syncthreads();
  cands_body<true>(D, R, &sm);
}

// Cavity growth by groups of kBfsLanes lanes, kWarpGroups candidates per
// warp: a group tests kBfsLanes (queued tet, face) pairs per pass, so a small
// cavity costs one dependent load chain (tet -> neighbour -> claim ->
// vertices -> coordinates -> insphere -> claim) per pass, and a warp keeps
// several such chains in flight.  The queue starts in shared memory and
// continues in the group's global region; cavities beyond BIG_CAP move to the
// huge path next round.
#ifndef WTET_BFS_LANES
#define WTET_BFS_LANES 16
#endif
constexpr uint32_t kBfsLanes = WTET_BFS_LANES;
constexpr uint32_t kWarpGroups = 32 / kBfsLanes;
constexpr uint32_t kBfsShared = 4 * kBfsLanes;  // queue entries (tet + neighbour words) per group in shared memory

// Loads issued as written (volatile asm is neither sunk into the branch that
// uses the value nor merged with later loads), so that a pass of the cavity
// search issues its claim, memo, vertex and neighbour loads together.
__device__ __forceinline__ uint4 ld_nc_u4(const uint4* p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned long long ld_cg_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

__global__ void __launch_bounds__(128, WTET_BFS_MINB) k_bfs(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  constexpr uint32_t FULL = 0xFFFFFFFFu, GM = (kBfsLanes == 32) ? 0xFFFFFFFFu : ((1u << kBfsLanes) - 1u);
  // queue of each lane group: cavity tets and their four neighbour words
  __shared__ uint32_t sq_all[4 * kWarpGroups][kBfsShared];
  __shared__ uint4 sn_all[4 * kWarpGroups][kBfsShared];
  const uint32_t lane = threadIdx.x & 31, gl = lane % kBfsLanes, shift = lane - gl;
  const uint32_t lt = (1u << gl) - 1u;
  const uint32_t gid = (blockIdx.x * blockDim.x + threadIdx.x) / kBfsLanes;  // global group index
  uint32_t* sq = sq_all[threadIdx.x / kBfsLanes];
  uint4* sn = sn_all[threadIdx.x / kBfsLanes];
  uint32_t* cav = D.wscratch + size_t(gid) * BIG_CAP;
  __shared__ uint32_t sp[kOrderBuckets + 2];
  __shared__ unsigned long long block_searches;
  if (threadIdx.x == 0) block_searches = 0;
  load_start_prefix(D, sp);
  const uint32_t nstart = sp[kOrderBuckets + 1];
  unsigned long long searches = 0;
  // Work is taken dynamically, one start per lane group (kWarpGroups per
  // warp) per fetch: cavities differ in size by orders of magnitude, and a
  // static grid-stride split leaves warps idle behind the slowest ones.
  const uint32_t bchunk = kWarpGroups;
  for (uint32_t chunk0 = warp_next(&D.ctr->work[0], bchunk); chunk0 < nstart;
       chunk0 = warp_next(&D.ctr->work[0], bchunk))
  for (uint32_t base = chunk0; base < min(chunk0 + bchunk, nstart); base += kWarpGroups) {
    const uint32_t si = base + lane / kBfsLanes;
    bool active = si < nstart;
    uint32_t p = 0, t0 = 0;
    if (active) {
      p = start_at(D, sp, si);
      t0 = D.loc[p];
    }
    unsigned long long key = 0;
    float4 pq = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
      key = make_key(D, R, p);
      pq = D.pts[p];
    }
    int pre_lost = 0;
    if (active && D.prefilter) {
      // the winner's own pre-claims (t0 and its face neighbours) must all hold
      for (uint32_t k = gl; k < 5; k += kBfsLanes) {
        const uint32_t t = pre_claim_tet(D, t0, k == 0 ? 0u : 4u * (k - 1u) + 1u);
        if (t != NONE && __ldcg(&D.C[t].pre) != key) pre_lost = 1;
      }
    }
    // warp collectives first, outside any short-circuit: every lane must reach them
    const uint32_t g_pre = (__ballot_sync(FULL, pre_lost) >> shift) & GM;
    const bool searched = active && !g_pre;
    int claim_lost = 0;
    if (searched && gl == 0) {
      const unsigned long long old = atomicMin(&D.C[t0].cav, key);
      claim_lost = old < key;
      sq[0] = t0;
      sn[0] = D.T[t0].n;
    }
    const int g_claim = __shfl_sync(FULL, claim_lost, shift);
    bool lost = !searched || g_claim;
    uint32_t K = 1, head = 0;
    bool overflow = false;
    bool running = !lost;
    __syncwarp();
    while (__any_sync(FULL, running)) {
      bool add = false, my_lost = false, my_guard = false;
      uint32_t nt = 0;
      uint4 nn = make_uint4(NONE, NONE, NONE, NONE);
      const uint32_t idx = head + gl / 4u;
      const uint32_t f = gl & 3u;
      if (running && idx < K) {
        // the neighbour word comes from the queue (loaded when the tet was
        // added), or from global memory for entries beyond the shared part
        const uint32_t nb = idx < kBfsShared ? comp(sn[idx], int(f))
                                             : reinterpret_cast<const uint32_t*>(&D.T[cav[idx]].n)[f];
        if (nb != NONE) {
          nt = nb >> 2;
          if (nt >= D.cap) {
            my_guard = true;
          } else {
            // one round trip: claim, memo, vertices and neighbours together
            const unsigned long long cc = ld_cg_u64(&D.C[nt].cav);
            const unsigned long long cr = ld_cg_u64(&D.C[nt].ring);
            const uint4 W = ld_nc_u4(&D.T[nt].v);
            nn = ld_nc_u4(&D.T[nt].n);
            if (cc != key && cr != key) {
              if (W.x >= D.nv || W.y >= D.nv || W.z >= D.nv || W.w >= D.nv) {
                my_guard = true;
              } else {
                const int sg = o4d_sos_f(D.pts[W.x], D.pts[W.y], D.pts[W.z], D.pts[W.w], pq, W.x, W.y, W.z, W.w, p,
                                         D.sos, &D.ctr->err);
                if (sg < 0) {
                  const unsigned long long old = atomicMin(&D.C[nt].cav, key);
                  if (old < key) my_lost = true;
                  else if (old != key) add = true;
                } else {
                  D.C[nt].ring = key;  // memo for this candidate only
                }
              }
            }
          }
        }
      }
      const uint32_t gball = (__ballot_sync(FULL, add) >> shift) & GM;
      const uint32_t pos = K + __popc(gball & lt);
      bool my_over = false;
      if (add) {
        if (pos < kBfsShared) {
          sq[pos] = nt;
          sn[pos] = nn;
        } else if (pos < BIG_CAP) {
          cav[pos] = nt;
        } else {
          my_over = true;
        }
      }
      const bool g_guard = (__ballot_sync(FULL, my_guard) >> shift) & GM;
      const bool g_lost = (__ballot_sync(FULL, my_lost) >> shift) & GM;
      const bool g_over = (__ballot_sync(FULL, my_over) >> shift) & GM;
      if (running) {
        if (g_guard) {
          if (gl == 0) atomicOr(&D.ctr->err, kErrGuard);
          lost = true;
        }
        lost = lost || g_lost;
        overflow = overflow || g_over;
        head = min(head + kBfsLanes / 4u, K);
        K += __popc(gball);
        running = !lost && !overflow && head < K;
      }
      __syncwarp();
    }
    if (searched && gl == 0) ++searches;
    // Partial claims carry this round's key: the huge path takes it next round.
    if (searched && overflow && gl == 0) D.bigflag[p] = kPending | 2;
    bool ok = searched && !lost && !overflow;
    // One reservation for the warp's completed cavities (pool entries and
    // candidate slots are shared counters of the whole grid).
    const uint32_t kk = ok ? K : 0u;
    uint32_t tot = 0, n_ok = 0, my_off = 0, my_ci = 0;  // each group follows the earlier groups' entries
#pragma unroll
    for (uint32_t g = 0; g < kWarpGroups; ++g) {
      const uint32_t kg = __shfl_sync(FULL, kk, int(g * kBfsLanes));
      if (g * kBfsLanes == shift) {
        my_off = tot;
        my_ci = n_ok;
      }
      tot += kg;
      n_ok += kg ? 1u : 0u;
    }
    uint32_t off = 0, ci = 0;
    if (lane == 0 && n_ok) {
      off = atomicAdd(&D.ctr->pool_used, tot);
      ci = atomicAdd(&D.ctr->n_cand, n_ok);
    }
    off = __shfl_sync(FULL, off, 0) + my_off;
    ci = __shfl_sync(FULL, ci, 0) + my_ci;
    ok = ok && off + K <= D.pool_cap;  // pool full: retry next round
    if (ok) {
      for (uint32_t k = gl; k < K; k += kBfsLanes) D.pool[off + k] = k < kBfsShared ? sq[k] : cav[k];
      if (gl == 0) {
        D.cand[ci] = p;
        D.cand_off[ci] = off;
        D.cand_len[ci] = K;
      }
    } else if (kk && gl == 0) {
      // a reserved candidate slot whose cavity did not fit the pool: it holds
      // no cavity, and k_resolve rejects it
      D.cand[ci] = p;
      D.cand_off[ci] = 0;
      D.cand_len[ci] = 0;
    }
    __syncwarp();
  }
  // per-block statistics, one atomic per block
  if (searches) atomicAdd(&block_searches, searches);
  __syncthreads();
  if (threadIdx.x == 0 && block_searches) atomicAdd(&D.ctr->n_expanded, block_searches);
}

// Global cavity slot bi of the huge path (HUGE_CAP tets each).
__device__ __forceinline__ uint32_t* big_slot(const Dev& D, uint32_t bi) {
  return D.big + size_t(bi) * HUGE_CAP;
}

__device__ __forceinline__ const uint32_t* cand_cavity(const Dev& D, uint32_t off) {
  return (off & 0x80000000u) ? big_slot(D, off & 0x7FFFFFFFu) : D.pool + off;
}


// Huge cavities: one block per candidate; each pass tests blockDim/4 queued
// tets x 4 faces, appending to the slot's list through a shared counter.
__global__ void __launch_bounds__(256) k_expand_big(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  const uint32_t nhuge = min(__ldcg(&D.ctr->huge_used), HUGE_SLOTS);
  const uint32_t bi = blockIdx.x;
  if (bi >= nhuge) return;  // block-uniform
  __shared__ uint32_t sK, sNew, sHead, sLost, sOver, sGuard;
  const uint32_t tid = threadIdx.x;
  const uint32_t p = D.bigcand[bi];
  const uint32_t t0 = D.loc[p];
  uint32_t* cav = big_slot(D, bi);
  const unsigned long long key = make_key(D, R, p);
  const float4 pq = D.pts[p];
  if (tid == 0) {
    D.st1[p] = 0;
    D.st2[p] = 0;
    const unsigned long long old = t0 < D.cap ? atomicMin(&D.C[t0].cav, key) : 0ull;
    sLost = old < key ? 1u : 0u;
    sOver = 0u;
    sGuard = t0 < D.cap ? 0u : 1u;
    cav[0] = t0;
    sK = 1u;
    sNew = 1u;
    sHead = 0u;
  }
  __syncthreads();
  for (;;) {
    const uint32_t K = sK, head = sHead;
    const bool stop = sLost || sOver || sGuard || head >= K;
    __syncthreads();  // every thread has read the pass state
    if (stop) break;   // block-uniform
    const uint32_t idx = head + tid / 4u, f = tid & 3u;
    if (idx < K) {
      const uint32_t c = cav[idx];
      const uint32_t nb = reinterpret_cast<const uint32_t*>(&D.T[c].n)[f];
      if (nb != NONE) {
        const uint32_t nt = nb >> 2;
        if (nt >= D.cap) {
          sGuard = 1u;
        } else if (__ldcg(&D.C[nt].cav) != key && __ldcg(&D.C[nt].ring) != key) {
          const uint4 W = D.T[nt].v;
          if (W.x >= D.nv || W.y >= D.nv || W.z >= D.nv || W.w >= D.nv) {
            sGuard = 1u;
          } else {
            const int sg = o4d_sos_f(D.pts[W.x], D.pts[W.y], D.pts[W.z], D.pts[W.w], pq, W.x, W.y, W.z, W.w, p,
                                     D.sos, &D.ctr->err);
            if (sg < 0) {
              const unsigned long long old = atomicMin(&D.C[nt].cav, key);
              if (old < key) {
                sLost = 1u;
              } else if (old != key) {
                const uint32_t pos = atomicAdd(&sNew, 1u);
                if (pos < HUGE_CAP) cav[pos] = nt;
                else sOver = 1u;
              }
            } else {
              D.C[nt].ring = key;
            }
          }
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      sHead = min(head + blockDim.x / 4u, K);
      sK = min(sNew, HUGE_CAP);
    }
    __syncthreads();
  }
  if (tid == 0) {
    atomicAdd(&D.ctr->n_big, 1ull);
    if (sGuard) atomicOr(&D.ctr->err, kErrGuard);
    if (sOver) atomicOr(&D.ctr->err, kErrBig);
    if (!sLost && !sOver && !sGuard) {
      const uint32_t ci = atomicAdd(&D.ctr->n_cand, 1u);
      D.cand[ci] = p;
      D.cand_off[ci] = 0x80000000u | bi;
      D.cand_len[ci] = sK;
    }
  }
}

// A candidate wins its cavity when it holds the minimum claim on every tet.
__global__ void k_resolve(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ncand = __ldcg(&D.ctr->n_cand);
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < ncand; ci += nwarps) {
    uint32_t p = D.cand[ci];
    uint32_t K = D.cand_len[ci];
    const uint32_t* cav = cand_cavity(D, D.cand_off[ci]);
    unsigned long long key = make_key(D, R, p);
    bool ok = K > 0;  // a slot whose cavity did not fit the pool holds none
    for (uint32_t i = lane; i < K; i += 32)
      if (__ldcg(&D.C[cav[i]].cav) != key) ok = false;
    bool win = __all_sync(0xFFFFFFFFu, ok);
    if (lane == 0) D.st1[p] = win ? 1 : 0;
  }
}

__device__ __forceinline__ uint32_t slot_of(const Dev& D, const RoundArgs& R, uint32_t v) {
  return v < R.n_freed_prev ? R.freed_prev[v] : R.tet_top + (v - R.n_freed_prev);
}

__device__ __forceinline__ bool boundary_face(const Dev& D, uint32_t nb, unsigned long long key) {
  return nb == NONE || __ldcg(&D.C[nb >> 2].cav) != key;
}

// The edge of face f of tet V opposite corner k (k != f): its two vertex ids,
// smaller and larger (register selects, no indexed local array).
__device__ __forceinline__ uint32_t edge_lo(const uint4& V, int f, int k) {
  const int q0 = (f != 0 && k != 0) ? 0 : (f != 1 && k != 1) ? 1 : 2;
  const int q1 = (f != 3 && k != 3) ? 3 : (f != 2 && k != 2) ? 2 : 1;
  return min(comp(V, q0), comp(V, q1));
}
__device__ __forceinline__ uint32_t edge_hi(const uint4& V, int f, int k) {
  const int q0 = (f != 0 && k != 0) ? 0 : (f != 1 && k != 1) ? 1 : 2;
  const int q1 = (f != 3 && k != 3) ? 3 : (f != 2 && k != 2) ? 2 : 1;
  return max(comp(V, q0), comp(V, q1));
}

// Two winners whose cavities share a face f may both insert iff f stays
// Delaunay: the better winner q must lie outside the circumsphere of the
// worse winner p's new tet on f (then either insertion order gives the same
// tets).  The worse one of a violating pair steps back.  A winner that stays
// is handed one slot per boundary face (recycled slots first, then fresh
// ones) in the same pass over its cavity.
__global__ void __launch_bounds__(128, WTET_SHARED_MINB) k_shared(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ncand = __ldcg(&D.ctr->n_cand);
  const uint32_t ch = chunk_for(ncand);
  for (uint32_t c0 = warp_next(&D.ctr->work[1], ch); c0 < ncand; c0 = warp_next(&D.ctr->work[1], ch)) {
    // Phase 1, per winner of the chunk: the shared-face test and the count of
    // boundary faces.  Phase 2: one allocation for the whole chunk (the slot
    // and list counters are shared by every warp of the grid).  Phase 3: the
    // slots of each winner's boundary faces.
    uint32_t need_fresh[kChunk], need_total[kChunk], bmask[kChunk];
    bool keep[kChunk], inpl[kChunk];
#pragma unroll
    for (uint32_t j = 0; j < kChunk; ++j) {
      const uint32_t ci = c0 + j;
      keep[j] = false;
      inpl[j] = false;
      need_fresh[j] = need_total[j] = bmask[j] = 0;
      if (j >= ch || ci >= ncand) continue;
      const uint32_t p = D.cand[ci];
      if (!D.st1[p]) {
        if (lane == 0) D.st2[p] = 0;
        continue;
      }
      const uint32_t K = D.cand_len[ci];
      const uint32_t* cav = cand_cavity(D, D.cand_off[ci]);
      const unsigned long long key = make_key(D, R, p);
      // one lane per (cavity tet, face): boundary faces are counted (their
      // flags kept in a register for cavities of up to 64 tets), faces shared
      // with a better winner are tested
      bool bad = false;
      uint32_t total = 0, bm = 0;
      for (uint32_t e0 = 0; e0 < 4 * K; e0 += 32) {
        const uint32_t e = e0 + lane;
        bool bnd = false;
        if (e < 4 * K) {
          const uint32_t c = cav[e >> 2];
          const int f = int(e & 3u);
          const uint32_t nb = reinterpret_cast<const uint32_t*>(&D.T[c].n)[f];
          const unsigned long long cc = nb == NONE ? 0ull : __ldcg(&D.C[nb >> 2].cav);
          bnd = nb == NONE || cc != key;
          if (bnd && nb != NONE && !bad && cc < key && this_round(R, cc)) {
            const uint32_t q = key_owner(R, cc);
            if (q < D.nv && D.st1[q]) {
              // the new tet on face f: p replaces vertex f
              const uint4 V = D.T[c].v;
              const uint32_t w0 = f == 0 ? p : V.x, w1 = f == 1 ? p : V.y, w2 = f == 2 ? p : V.z,
                             w3 = f == 3 ? p : V.w;
              if (o4d_sos_call(D.pts[w0], D.pts[w1], D.pts[w2], D.pts[w3], D.pts[q], w0, w1, w2, w3, q, D.sos,
                            &D.ctr->err) < 0)
                bad = true;
            }
          }
        }
        const uint32_t ball = __ballot_sync(FULL, bnd);
        total += __popc(ball);
        if (e0 < 256 && bnd) bm |= 1u << (e0 >> 5);
      }
      if (__any_sync(FULL, bad)) {
        if (lane == 0) D.st2[p] = 0;
        continue;
      }
      // A small star goes into the cavity's own slots (boundary face r < K
      // takes the slot of cavity tet r), plus fresh slots for the faces
      // beyond K: tets that are neighbours in space stay neighbours in memory.
      // Larger stars take recycled / fresh slots for every face.
      inpl[j] = total <= kInPlaceFaces && !(D.cand_off[ci] & 0x80000000u);
      keep[j] = true;
      need_total[j] = total;
      need_fresh[j] = total - (inpl[j] ? min(K, total) : 0u);
      bmask[j] = bm;
    }
    uint32_t sum_fresh = 0, sum_total = 0;
#pragma unroll
    for (uint32_t j = 0; j < kChunk; ++j) {
      sum_fresh += need_fresh[j];
      sum_total += need_total[j];
    }
    if (sum_total == 0) continue;  // warp-uniform
    uint32_t base = 0, bfo = 0;
    if (lane == 0) {
      base = atomicAdd(&D.ctr->alloc_used, sum_fresh);
      bfo = atomicAdd(&D.ctr->bface_used, sum_total);
    }
    base = __shfl_sync(FULL, base, 0);
    bfo = __shfl_sync(FULL, bfo, 0);
#pragma unroll
    for (uint32_t j = 0; j < kChunk; ++j) {
      const uint32_t mybase = base, mybfo = bfo;
      base += need_fresh[j];
      bfo += need_total[j];
      if (!keep[j]) continue;
      const uint32_t ci = c0 + j;
      const uint32_t p = D.cand[ci];
      const uint32_t K = D.cand_len[ci];
      const uint32_t* cav = cand_cavity(D, D.cand_off[ci]);
      const unsigned long long key = make_key(D, R, p);
      const uint32_t total = need_total[j], fresh = need_fresh[j];
      const uint32_t reuse = total - fresh;
      const uint32_t last = mybase + fresh;
      if ((last > R.n_freed_prev && R.tet_top + (last - R.n_freed_prev) > D.cap) || mybfo + total > D.cap) {
        if (lane == 0) {
          atomicOr(&D.ctr->err, kErrCapacity);
          D.st2[p] = 0;
        }
        continue;
      }
      // slots in (tet, face) order; inner faces get NONE
      uint32_t run = 0;
      for (uint32_t e0 = 0; e0 < 4 * K; e0 += 32) {
        const uint32_t e = e0 + lane;
        bool bnd = false;
        uint32_t c = 0;
        int f = 0;
        if (e < 4 * K) {
          c = cav[e >> 2];
          f = int(e & 3u);
          if (4 * K <= 256) {
            bnd = (bmask[j] >> (e0 >> 5)) & 1u;
          } else {
            const uint32_t nb = reinterpret_cast<const uint32_t*>(&D.T[c].n)[f];
            bnd = boundary_face(D, nb, key);
          }
        }
        const uint32_t ball = __ballot_sync(FULL, bnd);
        const uint32_t r = run + __popc(ball & ((1u << lane) - 1u));  // rank of this boundary face
        if (e < 4 * K)
          reinterpret_cast<uint32_t*>(D.nslot + c)[f] =
              !bnd ? NONE : (r < reuse ? cav[r] : slot_of(D, R, mybase + (r - reuse)));
        if (bnd) D.bface[mybfo + r] = (c << 2) | uint32_t(f);
        run += __popc(ball);
      }
      if (lane == 0) {
        D.cand_base[ci] = mybfo;
        D.cand_nf[ci] = total | (inpl[j] ? 0x80000000u : 0u);
        D.st2[p] = 1;
      }
    }
  }
}

// Writes the new tets of every winner.  The three faces through p of a new
// tet pair up across the boundary edges of the cavity (each boundary edge is
// shared by exactly two new tets): the pairs are matched in an open-addressing
// edge table of at least 3 slots per boundary face (load <= 1/2) -- in shared
// memory for up to kEdgeFaces faces, in the warp's region of a global table
// for up to kEdgeFacesG faces, in one of kBigTables large tables (taken per
// round, first come) for up to kBigTableFaces -- and the rest rotate around
// each edge inside the cavity.  A boundary face shared with another winner's cavity
// links to that winner's new tet.
constexpr uint32_t kEdgeSlots = 256;    // shared-memory slots per warp
constexpr uint32_t kEdgeFaces = 80;
constexpr uint32_t kEdgeSlotsG = 1024;  // global slots per warp
constexpr uint32_t kEdgeFacesG = 340;
constexpr uint32_t kBigTables = 16;         // large tables per round, taken first come
constexpr uint32_t kBigTableSlots = 1u << 14;
constexpr uint32_t kBigTableFaces = kBigTableSlots / 3;

__device__ __forceinline__ uint32_t edge_hash(uint32_t a, uint32_t b, uint32_t mask) {
  return mix32(a * 0x9E3779B9u ^ b) & mask;
}

__global__ void __launch_bounds__(128, WTET_WRITE_MINB) k_write(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  __shared__ unsigned long long ekey[4][kEdgeSlots];
  __shared__ uint32_t ev0[4][kEdgeSlots], ev1[4][kEdgeSlots];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t w = threadIdx.x >> 5;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t ncand = __ldcg(&D.ctr->n_cand);
  __shared__ uint32_t block_inserted;
  __shared__ unsigned long long block_created;
  if (threadIdx.x == 0) {
    block_inserted = 0;
    block_created = 0;
  }
  __syncthreads();
  uint32_t inserted = 0;
  unsigned long long created = 0;
  const uint32_t ch = chunk_for(ncand);
  for (uint32_t c0 = warp_next(&D.ctr->work[2], ch); c0 < ncand; c0 = warp_next(&D.ctr->work[2], ch))
  for (uint32_t ci = c0; ci < min(c0 + ch, ncand); ++ci) {
    uint32_t p = D.cand[ci];
    if (!D.st2[p]) continue;
    uint32_t K = D.cand_len[ci];
    const uint32_t* cav = cand_cavity(D, D.cand_off[ci]);
    unsigned long long key = make_key(D, R, p);
    const uint32_t nfw = D.cand_nf[ci];
    const uint32_t F = nfw & 0x7FFFFFFFu;    // boundary faces, counted by k_shared
    const bool inplace = (nfw >> 31) != 0u;  // the star takes the cavity's own slots
    const uint32_t bfo = D.cand_base[ci];    // first entry of its boundary-face list
    unsigned long long* tk = nullptr;
    uint32_t *t0 = nullptr, *t1 = nullptr;
    uint32_t mask = 31;
    while (mask + 1 < 3 * F) mask = 2 * mask + 1;
    if (F <= kEdgeFaces) {
      tk = ekey[w];
      t0 = ev0[w];
      t1 = ev1[w];
    } else if (F <= kEdgeFacesG && gwarp < D.etab_warps) {
      tk = D.etab_key + size_t(gwarp) * kEdgeSlotsG;
      t0 = D.etab_val + size_t(gwarp) * 2 * kEdgeSlotsG;
      t1 = t0 + kEdgeSlotsG;
    } else if (F <= kBigTableFaces) {
      uint32_t bt = 0;
      if (lane == 0) bt = atomicAdd(&D.ctr->btab_used, 1u);
      bt = __shfl_sync(0xFFFFFFFFu, bt, 0);
      if (bt < kBigTables) {
        tk = D.btab_key + size_t(bt) * kBigTableSlots;
        t0 = D.btab_val + size_t(bt) * 2 * kBigTableSlots;
        t1 = t0 + kBigTableSlots;
      }
    }
    const bool use_table = tk != nullptr;
    if (use_table) {
      for (uint32_t j = lane; j <= mask; j += 32) {
        tk[j] = ~0ull;
        t0[j] = NONE;
        t1[j] = NONE;
      }
      __syncwarp();
      for (uint32_t j = lane; j < F; j += 32) {
        const uint32_t bf = D.bface[bfo + j];
        const uint32_t c = bf >> 2;
        const int f = int(bf & 3u);
        const uint32_t sl = reinterpret_cast<const uint32_t*>(D.nslot + c)[f];
        const uint4 V = D.T[c].v;
        {
          for (int k = 0; k < 4; ++k) {
            if (k == f) continue;
            const uint32_t a = edge_lo(V, f, k), b = edge_hi(V, f, k);
            const unsigned long long ek = (static_cast<unsigned long long>(a) << 32) | b;
            const uint32_t val = (sl << 2) | uint32_t(k);
            uint32_t h = edge_hash(a, b, mask);
            for (uint32_t probe = 0; probe <= mask; ++probe) {
              const unsigned long long old = atomicCAS(&tk[h], ~0ull, ek);
              if (old == ~0ull || old == ek) {
                if (atomicCAS(&t0[h], NONE, val) != NONE) t1[h] = val;
                break;
              }
              h = (h + 1) & mask;
            }
          }
        }
      }
      __syncwarp();
    }
    bool bad = false;
    // The new tet of boundary face j (the compact list k_shared wrote): the
    // cavity tet with the face's opposite vertex replaced by p, linked to the
    // outer tet (or to another winner's new tet on a shared face) and, across
    // its three faces through p, to its neighbours in the star.
    auto build = [&](uint32_t j, uint4& nv, uint4& nn, uint32_t& sl, uint32_t& outer, bool& shared) {
      const uint32_t bf = D.bface[bfo + j];
      const uint32_t c = bf >> 2;
      const int f = int(bf & 3u);
      sl = reinterpret_cast<const uint32_t*>(D.nslot + c)[f];
      const uint4 V = D.T[c].v;
      outer = reinterpret_cast<const uint32_t*>(&D.T[c].n)[f];
      shared = false;
      uint32_t link_out = outer;
      if (outer != NONE) {
        const uint32_t o = outer >> 2;
        const unsigned long long cc = __ldcg(&D.C[o].cav);
        if (cc != key && this_round(R, cc)) {
          const uint32_t q = key_owner(R, cc);
          if (q < D.nv && D.st2[q]) {
            shared = true;
            link_out = (comp(D.nslot[o], outer & 3) << 2) | (outer & 3);
          }
        }
      }
      nv = V;
      set_comp(nv, f, p);
      nn = make_uint4(NONE, NONE, NONE, NONE);
      set_comp(nn, f, link_out);
      for (int k = 0; k < 4; ++k) {
        if (k == f) continue;
        uint32_t link = NONE;
        if (use_table) {
          const uint32_t a = edge_lo(V, f, k), b = edge_hi(V, f, k);
          const unsigned long long ek = (static_cast<unsigned long long>(a) << 32) | b;
          const uint32_t mine = (sl << 2) | uint32_t(k);
          uint32_t h = edge_hash(a, b, mask);
          for (uint32_t probe = 0; probe <= mask; ++probe) {
            const unsigned long long kk = tk[h];
            if (kk == ek) {
              link = t0[h] == mine ? t1[h] : t0[h];
              break;
            }
            if (kk == ~0ull) break;
            h = (h + 1) & mask;
          }
        } else {
          uint32_t cur = c;
          uint4 Vc = V;
          int kc = k, ms = f;
          for (int it = 0; it < ROT_LIMIT; ++it) {
            const uint32_t nb = comp(D.T[cur].n, kc);
            if (boundary_face(D, nb, key)) {
              link = (comp(D.nslot[cur], kc) << 2) | uint32_t(ms);
              break;
            }
            const uint32_t nt = nb >> 2;
            if (nt >= D.cap) break;
            const int entry = int(nb & 3);
            const uint32_t x = comp(Vc, ms);
            const uint4 Wt = D.T[nt].v;
            int kx = -1;
            for (int q = 0; q < 4; ++q)
              if (comp(Wt, q) == x) kx = q;
            if (kx < 0) break;
            cur = nt;
            Vc = Wt;
            kc = kx;
            ms = entry;
          }
        }
        if (link == NONE) bad = true;
        set_comp(nn, k, link);
      }
    };
    auto commit = [&](const uint4& nv, const uint4& nn, uint32_t sl, uint32_t outer, bool shared) {
      D.T[sl].v = nv;
      D.T[sl].n = nn;
      D.C[sl].vote = 0ull;  // the new tet's points vote in k_relocate
      // Every vertex on the cavity boundary gets a live incident tet, so a
      // vertex's hint tet is alive whenever it is read (strata activation).
      for (int q = 0; q < 4; ++q)
        if (comp(nv, q) != p) D.vtet[comp(nv, q)] = sl;
      if (outer != NONE && !shared && (outer >> 2) < D.cap) {
        uint32_t* wp = reinterpret_cast<uint32_t*>(&D.T[outer >> 2].n) + (outer & 3);
        const int f = comp(nv, 0) == p ? 0 : comp(nv, 1) == p ? 1 : comp(nv, 2) == p ? 2 : 3;
        *wp = (sl << 2) | uint32_t(f);
      }
    };
    if (inplace) {
      // The star overwrites the cavity's own slots: every lane reads first,
      // the warp synchronises, then every lane writes (F <= 32: one face each).
      uint4 nv = make_uint4(0, 0, 0, 0), nn = make_uint4(0, 0, 0, 0);
      uint32_t sl = 0, outer = NONE;
      bool shared = false;
      if (lane < F) build(lane, nv, nn, sl, outer, shared);
      __syncwarp();
      if (lane < F) commit(nv, nn, sl, outer, shared);
    } else {
      for (uint32_t j = lane; j < F; j += 32) {
        uint4 nv, nn;
        uint32_t sl, outer;
        bool shared;
        build(j, nv, nn, sl, outer, shared);
        commit(nv, nn, sl, outer, shared);
      }
    }
    if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(&D.ctr->err, kErrRotate);
    __syncwarp();  // every lane is done reading the cavity before it is retired
    uint32_t s0 = 0;
    if (lane == 0) {
      const uint32_t bf0 = D.bface[bfo];
      s0 = reinterpret_cast<const uint32_t*>(D.nslot + (bf0 >> 2))[bf0 & 3u];
    }
    s0 = __shfl_sync(0xFFFFFFFFu, s0, 0);
    // cavity tets whose slots the star did not take are retired
    const uint32_t reused = inplace ? min(K, F) : 0u;
    uint32_t fbase = 0;
    if (lane == 0 && K > reused) fbase = atomicAdd(&D.ctr->n_freed_next, K - reused);
    fbase = __shfl_sync(0xFFFFFFFFu, fbase, 0);
    for (uint32_t i = reused + lane; i < K; i += 32) {
      const uint32_t c = cav[i];
      // Points inside c relocate from a new tet on one of c's own faces.
      const uint4 S = D.nslot[c];
      const uint32_t fwd = S.x != NONE ? S.x : S.y != NONE ? S.y : S.z != NONE ? S.z : S.w != NONE ? S.w : s0;
      D.T[c].v = make_uint4(DEAD, fwd, 0u, 0u);
      R.freed_next[fbase + (i - reused)] = c;
    }
    if (lane == 0) {
      if (D.log_pslot && D.log_pslot[p] != NONE) D.log_y[D.log_pslot[p]] = 1;  // scheduler log: inserted
      D.vtet[p] = s0;
      D.loc[p] |= INS_BIT;
      D.centry[D.vcloud[p]] = s0;
      D.bigflag[p] = 0;
      ++inserted;
      created += F;
    }
    __syncwarp();
  }
  // per-block statistics, one atomic each per block
  if (inserted) {
    atomicAdd(&block_inserted, inserted);
    atomicAdd(&block_created, created);
  }
  __syncthreads();
  if (threadIdx.x == 0 && block_inserted) {
    atomicAdd(&D.ctr->n_inserted, block_inserted);
    atomicAdd(&D.ctr->created, block_created);
  }
}

// Clears the votes, relocates points whose tet was retired, compacts the
// uninserted list, and carries the recycled slots that were not handed out
// this round over to the next round's list.
__global__ void __launch_bounds__(512, WTET_RELOC_MINB) k_relocate(Dev D) {
  const RoundArgs R = load_round(D);
  if (!R.live) return;
  uint32_t steps = 0;
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < R.n_active; i0 += gridDim.x * blockDim.x) {
    uint32_t i = i0 + threadIdx.x;
    bool keep = false;
    uint32_t p = 0;
    if (i < R.n_active && (D.bigflag[R.active[i]] & kDup)) {
      // exact duplicate: leaves the list without being inserted
    } else if (i < R.n_active) {
      p = R.active[i];
      uint32_t L = D.loc[p];
      uint32_t t = L & ~INS_BIT;
      if (t >= D.cap) {
        atomicOr(&D.ctr->err, kErrGuard);
        t = 0;
        L |= INS_BIT;
      }
      if (!(L & INS_BIT)) {
        keep = true;
        if (D.bigflag[p] & kPending) D.bigflag[p] &= uint8_t(~kPending);
        const uint4 V = D.T[t].v;
        uint32_t from = NONE;
        if (V.x == DEAD) {
          from = V.y;  // retired: walk from a new tet on one of its faces
        } else {
          // retired and overwritten by a star in place: t held a cavity tet
          // of a winner that inserted (its claim is this round's), and now
          // holds a tet of that winner's star, which covers the point
          const unsigned long long cc = __ldcg(&D.C[t].cav);
          if (this_round(R, cc)) {
            const uint32_t q = key_owner(R, cc);
            if (q < D.nv && D.st2[q]) from = t;
          }
        }
        if (from != NONE) {
          const uint32_t lt = walk_to(D, from, p, D.pts[p], steps);
          D.loc[p] = lt;
          cast_vote(D, p, lt);
        }
      }
    }
    uint32_t slot = warp_append(&D.ctr->n_next, keep);
    if (keep) R.active_next[slot] = p;
  }
  if (steps) atomicAdd(&D.ctr->walk_steps, (unsigned long long)steps);
  // recycled slots not handed out this round (k_write has appended this
  // round's retired tets in front of them)
  const uint32_t used = __ldcg(&D.ctr->alloc_used);
  if (R.n_freed_prev > used) {
    const uint32_t nfn = __ldcg(&D.ctr->n_freed_next);
    const uint32_t left = R.n_freed_prev - used;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < left; i += gridDim.x * blockDim.x)
      R.freed_next[nfn + i] = R.freed_prev[used + i];
  }
}

// Start of a round (device side, one thread): locate the next stratum once
// the current one has thinned to 1/2^overlap_shift of its size, stop when
// nothing is left, reset the per-round counters.
__device__ void begin_round(const Dev& D) {
  State* S = D.st;
  if (S->done || S->stop) return;
  S->act_total = 0;
  while (S->next_level >= 0 &&
         (S->n_active == 0 || (uint64_t(S->n_active) << S->overlap_shift) <= S->stratum_size)) {
    const int L = S->next_level--;
    const uint32_t total = D.lvl_total[L];
    if (total == 0) continue;
    S->act_level = uint32_t(L);
    S->act_total = total;
    S->act_base = S->n_active;
    S->n_active += total;
    S->stratum_size = total;
    S->strata += 1;
    break;
  }
  if (S->n_active == 0) {
    S->done = 1;
    return;
  }
  S->round += 1;
  if (S->round > S->max_rounds) {
    S->stop = 3;
    return;
  }
  Counters* C = D.ctr;
  C->n_next = 0;
  C->n_cand = 0;
  C->pool_used = 0;
  C->alloc_used = 0;
  C->n_freed_next = 0;
  C->big_used = 0;
  C->n_inserted = 0;
  C->huge_used = 0;
  C->btab_used = 0;
  C->bface_used = 0;
  C->work[0] = C->work[1] = C->work[2] = C->work[3] = 0;
  for (uint32_t b = 0; b <= kOrderBuckets; ++b) C->sbc[b] = 0;
}

// The first round's start (later rounds are started by k_end).
__global__ void k_begin(Dev D) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  begin_round(D);
}

// End of a round: advance the slot top, swap the lists, stop on errors; then
// start the next round, so that a round is one kernel shorter.
__global__ void k_end(Dev D) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  State* S = D.st;
  if (S->done || S->stop) return;
  Counters* C = D.ctr;
  if (C->err & ~uint32_t(kErrCapacity)) {
    S->stop = 1;
    return;
  }
  const uint32_t used = C->alloc_used;
  const uint32_t fresh = used > S->n_freed_prev ? used - S->n_freed_prev : 0u;
  const uint32_t left = S->n_freed_prev > used ? S->n_freed_prev - used : 0u;
  // Winners that ran out of capacity reserved slot ranges they never wrote;
  // every written slot lies below the capacity, so the top never passes it
  // (the slots between are left dead).
  S->tet_top = uint32_t(min(uint64_t(S->tet_top) + fresh, uint64_t(D.cap)));
  S->n_freed_prev = C->n_freed_next + left;
  S->par ^= 1u;
  S->n_active = C->n_next;
  S->inserted += C->n_inserted;
  S->starts += C->big_used + min(C->huge_used, HUGE_SLOTS);
  S->last_starts = C->big_used;
  S->last_cand = C->n_cand;
  S->last_inserted = C->n_inserted;
  S->last_alloc = C->alloc_used;
  if (C->err & kErrCapacity) {
    S->stop = 2;
    return;
  }
  begin_round(D);
}

// ------------------------------------------------------ predicate check ----

// Signs of the round kernels' predicates on given records of five points and
// five SoS keys (testing only): orient3d_sos of the first four, orient4d of all
// five, through the same FP32 stage / FP64 filter / exact / SoS chain.
__global__ void k_predicate_signs(const float* pts, const uint32_t* keys, uint64_t m, int32_t* o3, int32_t* o4,
                                  uint32_t* err) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const float* q = pts + 15 * i;
    const float4 a = make_float4(q[0], q[1], q[2], 0.f), b = make_float4(q[3], q[4], q[5], 0.f);
    const float4 c = make_float4(q[6], q[7], q[8], 0.f), d = make_float4(q[9], q[10], q[11], 0.f);
    const float4 e = make_float4(q[12], q[13], q[14], 0.f);
    const uint32_t* k = keys + 5 * i;
    o3[i] = o3d_sos_f(a, b, c, d, 0, 1, 2, 3, k, err);
    o4[i] = o4d_sos_f(a, b, c, d, e, 0, 1, 2, 3, 4, k, err);
  }
}

// --------------------------------------------------------------- output ----

// Counts live tets per cloud and records the hull faces (no neighbour).
__global__ void k_count(Dev D, uint32_t tet_top, uint32_t* ccount, uint32_t* hullcnt, uint2* hull) {
  for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < tet_top; t0 += gridDim.x * blockDim.x) {
    const uint32_t t = t0 + threadIdx.x;
    uint4 V = t < tet_top ? D.T[t].v : make_uint4(DEAD, 0, 0, 0);
    const bool live = V.x != DEAD;
    const uint32_t c = live ? D.vcloud[V.x] : 0xFFFFFFFFu;
    // one atomic per (warp, cloud) group
    const unsigned grp = __match_any_sync(0xFFFFFFFFu, c);
    const int lane = threadIdx.x & 31;
    if (live && lane == __ffs(grp) - 1) atomicAdd(&ccount[c], __popc(grp));
    if (!live) continue;
    uint4 N = D.T[t].n;
    for (int f = 0; f < 4; ++f) {
      if (comp(N, f) == NONE) {
        uint32_t h = atomicAdd(&hullcnt[c], 1u);
        if (h < 4) hull[4 * c + h] = make_uint2(t, uint32_t(f));
        else atomicOr(&D.ctr->err, kErrHull);
      }
    }
  }
}

__global__ void k_number(Dev D, uint32_t tet_top, uint32_t* cfill, uint32_t* newid) {
  for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < tet_top; t0 += gridDim.x * blockDim.x) {
    const uint32_t t = t0 + threadIdx.x;
    uint4 V = t < tet_top ? D.T[t].v : make_uint4(DEAD, 0, 0, 0);
    const bool live = V.x != DEAD;
    const uint32_t c = live ? D.vcloud[V.x] : 0xFFFFFFFFu;
    const unsigned grp = __match_any_sync(0xFFFFFFFFu, c);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(grp) - 1;
    uint32_t base = 0;
    if (live && lane == leader) base = atomicAdd(&cfill[c], __popc(grp));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (live) newid[t] = base + __popc(grp & ((1u << lane) - 1u));
  }
}

__global__ void k_emit(Dev D, uint32_t tet_top, const uint32_t* newid, const uint64_t* coff, uint32_t* out_t,
                       uint32_t* out_a) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < tet_top; t += gridDim.x * blockDim.x) {
    uint4 V = D.T[t].v;
    if (V.x == DEAD) continue;
    uint32_t c = D.vcloud[V.x];
    uint64_t row = coff[c] + newid[t];
    uint4 N = D.T[t].n;
    uint4 ov = make_uint4(D.sos[V.x], D.sos[V.y], D.sos[V.z], D.sos[V.w]);
    uint4 oa;
    for (int f = 0; f < 4; ++f) {
      uint32_t nb = comp(N, f);
      if (nb != NONE && (nb >> 2) >= tet_top) {
        atomicOr(&D.ctr->err, kErrGuard);
        nb = NONE;
      }
      set_comp(oa, f, nb == NONE ? NONE : ((newid[nb >> 2] << 5) | (nb & 3)));
    }
    reinterpret_cast<uint4*>(out_t)[row] = ov;
    reinterpret_cast<uint4*>(out_a)[row] = oa;
  }
}

// Four infinity tets per cloud on the super tetrahedron's hull faces.
__global__ void k_infinity(Dev D, const CloudInfo* ci, uint32_t nc, const uint32_t* ccount,
                           const uint32_t* hullcnt, const uint2* hull, const uint32_t* newid, const uint64_t* coff,
                           uint32_t* out_t, uint32_t* out_a) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  if (hullcnt[c] != 4) {
    atomicOr(&D.ctr->err, kErrHull);
    return;
  }
  const uint32_t inf = ci[c].n + 4;
  uint32_t fv[4][3];  // the non-infinity vertices of each infinity tet (output ids)
  uint4 rows[4];
  uint32_t base = ccount[c];
  for (int j = 0; j < 4; ++j) {
    uint2 h = hull[4 * c + j];
    uint4 V = D.T[h.x].v;
    uint32_t w[4] = {D.sos[V.x], D.sos[V.y], D.sos[V.z], D.sos[V.w]};
    w[h.y] = inf;
    int a = -1, b = -1;
    for (int q = 0; q < 4; ++q)
      if (q != int(h.y)) {
        if (a < 0) a = q;
        else if (b < 0) b = q;
      }
    uint32_t tmp = w[a];
    w[a] = w[b];
    w[b] = tmp;
    rows[j] = make_uint4(w[0], w[1], w[2], w[3]);
    int k = 0;
    for (int q = 0; q < 4; ++q)
      if (q != int(h.y)) fv[j][k++] = w[q];
  }
  for (int j = 0; j < 4; ++j) {
    uint2 h = hull[4 * c + j];
    uint64_t row = coff[c] + base + j;
    uint32_t w[4] = {rows[j].x, rows[j].y, rows[j].z, rows[j].w};
    uint32_t adj[4];
    for (int q = 0; q < 4; ++q) {
      if (q == int(h.y)) {
        adj[q] = (newid[h.x] << 5) | h.y;
        continue;
      }
      // Face opposite slot q holds inf and the two other face vertices.
      uint32_t e[2];
      int ne = 0;
      for (int r = 0; r < 4; ++r)
        if (r != q && r != int(h.y)) e[ne++] = w[r];
      adj[q] = NONE;
      for (int o = 0; o < 4; ++o) {
        if (o == j) continue;
        bool ha = false, hb = false;
        for (int r = 0; r < 3; ++r) {
          ha |= fv[o][r] == e[0];
          hb |= fv[o][r] == e[1];
        }
        if (ha && hb) {
          uint32_t ow[4] = {rows[o].x, rows[o].y, rows[o].z, rows[o].w};
          int os = -1;
          for (int r = 0; r < 4; ++r)
            if (ow[r] != inf && ow[r] != e[0] && ow[r] != e[1]) os = r;
          adj[q] = ((base + o) << 5) | uint32_t(os);
        }
      }
    }
    reinterpret_cast<uint4*>(out_t)[row] = rows[j];
    reinterpret_cast<uint4*>(out_a)[row] = make_uint4(adj[0], adj[1], adj[2], adj[3]);
    // The regular tet's hull face points at this infinity tet.
    uint64_t rrow = coff[c] + newid[h.x];
    out_a[4 * rrow + h.y] = ((base + j) << 5) | h.y;
  }
}

// ------------------------------------------------------------- host side ----

using dev::ck;
using dev::DBuf;
using dev::scan_u32;

namespace {

uint32_t initial_stride_log2(uint64_t n) {
  // src/gpu/mod.rs:533-548
  double sq = std::sqrt(double(n));
  double scaled = n > 100000 ? sq * 2.0 : sq;
  double stride = std::min(std::max(scaled, 64.0), 16384.0);
  return uint32_t(std::ceil(std::log2(stride)));
}

uint64_t level_count(uint64_t n, uint32_t level, uint32_t top) {
  if (level > top) return 0;
  uint64_t s = 1ull << level;
  if (level == top) return (n + s - 1) / s;
  if (n <= s) return 0;
  return (n - s - 1) / (2 * s) + 1;
}

}  // namespace

struct Workspace {
  DBuf<float> xyz;
  DBuf<uint64_t> off;
  DBuf<CloudInfo> ci;
  DBuf<uint32_t> mn, mx, bucket, hist;
  DBuf<float4> tmp;
  DBuf<float4> pts;
  DBuf<uint32_t> sos, vcloud, vtet, loc;
  DBuf<uint8_t> bigflag;
  DBuf<Tet> T;
  DBuf<Claim> C;
  DBuf<uint4> nslot;
  DBuf<uint32_t> bface;
  DBuf<uint32_t> centry, active, active_next, cand, cand_off, cand_len, cand_base, cand_nf, pool, big, freed_a, freed_b;
  DBuf<uint8_t> st1, st2;
  DBuf<uint32_t> bigcand, starts, wscratch, etab_val;
  DBuf<unsigned long long> etab_key, btab_key;
  DBuf<uint32_t> btab_val;
  DBuf<uint64_t> lvl_off;
  DBuf<uint32_t> lvl_total;
  DBuf<State> state;
  DBuf<Counters> ctr;
  DBuf<uint32_t> ccount, hullcnt, cfill, newid;
  DBuf<uint2> hull;
  DBuf<uint64_t> coff;
  DBuf<uint32_t> out_t, out_a, dtab;
  DBuf<uint8_t> dup;
  DBuf<uint32_t> log_pslot;
  DBuf<uint8_t> losses;
  DBuf<uint16_t> prio;
  std::vector<DBuf<uint32_t>> scan_tmp;
  Counters* h_ctr = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t stream = nullptr;
  int device = -1;

  ~Workspace() {
    // Released explicitly by release_thread_workspace(); CUDA may already be
    // torn down at thread exit, so nothing is freed here.
  }
};

namespace {
thread_local Workspace* tl_ws = nullptr;

Workspace& ws() {
  if (!tl_ws) tl_ws = new Workspace;
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  if (tl_ws->device != dev) {
    tl_ws->device = dev;
  }
  if (!tl_ws->h_ctr) ck(cudaMallocHost(&tl_ws->h_ctr, sizeof(Counters)), "cudaMallocHost counters");
  if (!tl_ws->ev0) {
    ck(cudaEventCreate(&tl_ws->ev0), "event");
    ck(cudaEventCreate(&tl_ws->ev1), "event");
  }
  if (!tl_ws->stream) ck(cudaStreamCreate(&tl_ws->stream), "stream");
  return *tl_ws;
}

// One full wave of resident blocks of kernel k on the current device.
template <class K>
uint32_t wave(K* k, uint32_t threads) {
  int dev = 0, sms = 0, per = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device attribute");
  ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, int(threads), 0), "occupancy");
  return uint32_t(std::max(1, per) * std::max(1, sms));
}

inline uint32_t blocks_for(uint64_t n, uint32_t threads, uint32_t cap = 148 * 16) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return uint32_t(std::min<uint64_t>(b, cap));
}

}  // namespace

uint64_t max_tets_for(uint64_t n) { return 8 * n + 64; }

float* ws_input(size_t nfloats) {
  Workspace& W = ws();
  W.xyz.reserve(nfloats, "input");
  return W.xyz.p;
}

void ws_outputs(size_t rows, uint32_t** t, uint32_t** a) {
  Workspace& W = ws();
  W.out_t.reserve(4 * rows, "output tets");
  W.out_a.reserve(4 * rows, "output adjacency");
  *t = W.out_t.p;
  *a = W.out_a.p;
}

void release_thread_workspace() {
  if (!tl_ws) return;
  Workspace& w = *tl_ws;
  w.xyz.release(); w.off.release(); w.ci.release(); w.mn.release(); w.mx.release();
  w.bucket.release(); w.hist.release(); w.tmp.release(); w.pts.release(); w.sos.release();
  w.vcloud.release(); w.vtet.release(); w.loc.release(); w.bigflag.release(); w.T.release(); w.C.release();
  w.nslot.release(); w.bface.release();
  w.centry.release(); w.active.release(); w.active_next.release(); w.cand.release();
  w.cand_off.release(); w.cand_len.release(); w.cand_base.release(); w.cand_nf.release(); w.st1.release(); w.st2.release(); w.bigcand.release(); w.starts.release(); w.wscratch.release(); w.pool.release(); w.big.release();
  w.freed_a.release(); w.freed_b.release(); w.lvl_off.release(); w.lvl_total.release(); w.state.release(); w.ctr.release();
  w.ccount.release(); w.hullcnt.release(); w.cfill.release(); w.newid.release();
  w.hull.release(); w.coff.release(); w.out_t.release(); w.out_a.release(); w.dtab.release(); w.dup.release();
  w.etab_key.release(); w.etab_val.release(); w.btab_key.release(); w.btab_val.release();
  w.log_pslot.release(); w.losses.release(); w.prio.release();
  for (auto& b : w.scan_tmp) b.release();
  if (w.h_ctr) cudaFreeHost(w.h_ctr);
  if (w.ev0) cudaEventDestroy(w.ev0);
  if (w.ev1) cudaEventDestroy(w.ev1);
  if (w.stream) cudaStreamDestroy(w.stream);
  delete tl_ws;
  tl_ws = nullptr;
}

// ------------------------------------------------- learned-vote weights ----

namespace {
std::mutex g_mlp_mu;
std::vector<float> g_mlp_host;  // installed FP32 parameters (empty: none)
uint64_t g_mlp_version = 0;
struct MlpDevCopy {
  int dev;
  mlp::Image* p;
  uint64_t version;
};
std::vector<MlpDevCopy> g_mlp_dev;

// FP32 -> BF16, round to nearest even (NaN kept quiet).
uint16_t f2bf(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return uint16_t((u >> 16) | 0x40u);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return uint16_t(u >> 16);
}
float bf2f(uint16_t h) {
  uint32_t u = uint32_t(h) << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}
uint32_t bf_pair(float lo, float hi) { return uint32_t(f2bf(lo)) | (uint32_t(f2bf(hi)) << 16); }

void build_image(const float* P, mlp::Image& I) {
  using namespace mlp;
  memset(&I, 0, sizeof I);
  for (int o = 0; o < kHidden; ++o) {
    for (int k = 0; k < kIn / 2; ++k)
      I.w1[o * kW1Stride + k] = bf_pair(P[kOffW1 + o * kIn + 2 * k], P[kOffW1 + o * kIn + 2 * k + 1]);
    for (int k = 0; k < kHidden / 2; ++k) {
      I.w2[o * kWStride + k] = bf_pair(P[kOffW2 + o * kHidden + 2 * k], P[kOffW2 + o * kHidden + 2 * k + 1]);
      I.w3[o * kWStride + k] = bf_pair(P[kOffW3 + o * kHidden + 2 * k], P[kOffW3 + o * kHidden + 2 * k + 1]);
    }
    I.w4[o] = bf2f(f2bf(P[kOffW4 + o]));
    I.b1[o] = P[kOffB1 + o];
    I.b2[o] = P[kOffB2 + o];
    I.b3[o] = P[kOffB3 + o];
  }
  I.b4 = P[kOffB4];
}
}  // namespace

void set_mlp_params(const float* params) {
  std::lock_guard<std::mutex> g(g_mlp_mu);
  g_mlp_host.assign(params, params + mlp::kParams);
  ++g_mlp_version;
}

bool has_mlp_params() {
  std::lock_guard<std::mutex> g(g_mlp_mu);
  return !g_mlp_host.empty();
}

const void* mlp_image(cudaStream_t s) {
  std::lock_guard<std::mutex> g(g_mlp_mu);
  if (g_mlp_host.empty())
    throw Error{WTET_ERR_ARG, "the learned vote has no weights installed (wtet_learned_set_weights)"};
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  MlpDevCopy* e = nullptr;
  for (auto& c : g_mlp_dev)
    if (c.dev == dev) e = &c;
  if (!e) {
    mlp::Image* p = nullptr;
    ck(cudaMalloc(&p, sizeof(mlp::Image)), "learned weights");
    g_mlp_dev.push_back(MlpDevCopy{dev, p, 0});
    e = &g_mlp_dev.back();
  }
  if (e->version != g_mlp_version) {
    mlp::Image img;
    build_image(g_mlp_host.data(), img);
    ck(cudaMemcpyAsync(e->p, &img, sizeof img, cudaMemcpyHostToDevice, s), "learned weights upload");
    ck(cudaStreamSynchronize(s), "learned weights upload");
    e->version = g_mlp_version;
  }
  return e->p;
}

// ------------------------------------------------------------ autotuner ----

namespace {
std::mutex g_tune_mu;
std::vector<wtet_tune_entry> g_tune;  // sorted by (batched, max_points)
}  // namespace

void set_tune_table(const wtet_tune_entry* e, uint32_t count) {
  std::vector<wtet_tune_entry> t(e, e + count);
  std::stable_sort(t.begin(), t.end(), [](const wtet_tune_entry& a, const wtet_tune_entry& b) {
    return a.batched != b.batched ? a.batched < b.batched : a.max_points < b.max_points;
  });
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune = std::move(t);
}

std::vector<wtet_tune_entry> get_tune_table() {
  std::lock_guard<std::mutex> g(g_tune_mu);
  return g_tune;
}

// Knobs left at 0 in cfg take the installed table's entry for the job's size
// bucket (the first entry of its kind whose max_points covers n), then the
// built-in defaults.  No knob changes the triangulation.
wtet_config tuned_config(const wtet_config& cfg, uint64_t n, uint32_t nc) {
  wtet_config c = cfg;
  const uint32_t batched = nc > 1 ? 1u : 0u;
  wtet_tune_entry hit{};
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (const auto& e : g_tune)
      if (e.batched == batched && n <= e.max_points) {
        hit = e;
        break;
      }
  }
  auto pick = [](uint32_t user, uint32_t table, uint32_t dflt) { return user ? user : (table ? table : dflt); };
  c.block_size = pick(c.block_size, hit.block_size, 256u);
  c.rounds_per_graph = pick(c.rounds_per_graph, hit.rounds_per_graph, 8u);
  c.overlap_shift = pick(c.overlap_shift, hit.overlap_shift, 3u);
  c.candidate_filter = pick(c.candidate_filter, hit.candidate_filter, 1u);
  c.pool_factor = pick(c.pool_factor, hit.pool_factor, 24u);
  return c;
}

// Kernels with deep exact-arithmetic call chains need a few KB of stack per
// thread.  Reserving it once keeps the driver from re-growing local memory on
// every launch.
void reserve_stack_once() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> g(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  size_t need = 0;
  const void* ks[] = {(const void*)k_bfs, (const void*)k_expand_big, (const void*)k_shared,
                      (const void*)k_relocate, (const void*)k_activate, (const void*)k_init_clouds};
  for (const void* k : ks) {
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, k) == cudaSuccess) need = std::max<size_t>(need, a.localSizeBytes);
  }
  size_t cur = 0;
  cudaDeviceGetLimit(&cur, cudaLimitStackSize);
  size_t want = std::max<size_t>(need + 256, 4096);
  if (cur < want) ck(cudaDeviceSetLimit(cudaLimitStackSize, want), "cudaDeviceSetLimit(stack)");
  done[dev] = true;
}

JobResult run_job(const Job& job, uint32_t* d_out_t, uint32_t* d_out_a, uint64_t capacity) {
  reserve_stack_once();
  Workspace& W = ws();
  // The legacy default stream cannot be captured into a graph; the workspace's
  // own (blocking) stream orders with it implicitly.
  cudaStream_t s = job.stream ? job.stream : W.stream;
  const uint32_t nc = uint32_t(job.offsets.size() - 1);
  const uint64_t n = job.offsets.back();
  const wtet_config cfg = tuned_config(job.cfg, n, nc);
  if (n + 5ull * nc >= 0x7FFFFFF0ull) throw Error{WTET_ERR_ARG, "too many points for 31-bit vertex ids"};
  JobResult res;
  // scheduler: 0 plain (random claim priority), 1 learned priority, 2 plain + training log
  const uint32_t vmode = job.d_log_x ? 2u : (job.cfg.vote_mode == WTET_VOTE_LEARNED ? 1u : 0u);
  const mlp::Image* mlp_w = vmode == 1 ? static_cast<const mlp::Image*>(mlp_image(s)) : nullptr;
  ck(cudaEventRecord(W.ev0, s), "event record");

  // ---- per-cloud layout (host) ----
  std::vector<CloudInfo> ci(nc);
  uint64_t buckets = 0;
  uint32_t maxtop = 0;
  for (uint32_t c = 0; c < nc; ++c) {
    uint64_t nn = job.offsets[c + 1] - job.offsets[c];
    if (nn < 4) throw Error{WTET_ERR_ARG, "Need at least 4 points for 3D Delaunay"};
    CloudInfo& C = ci[c];
    C.off = job.offsets[c];
    C.n = uint32_t(nn);
    C.vbase = uint32_t(job.offsets[c] + 4ull * c);
    uint32_t lg = 0;
    while ((2ull << lg) <= nn) ++lg;  // floor(log2 n)
    C.bbits = std::max<uint32_t>(1, std::min<uint32_t>(10, lg / 3));
    C.bbase = uint32_t(buckets);
    buckets += 1ull << (3 * C.bbits);
    C.top = initial_stride_log2(nn);
    maxtop = std::max(maxtop, C.top);
  }
  const uint64_t nv = n + 4ull * nc;
  uint64_t cap0 = 0;
  const uint64_t slots_x8 = job.cfg.initial_capacity ? std::min<uint32_t>(job.cfg.initial_capacity, 1024u) : 72u;
  for (uint32_t c = 0; c < nc; ++c) cap0 += uint64_t(ci[c].n) * slots_x8 / 8 + 64;  // 9 n by default
  cap0 = std::min<uint64_t>(cap0, 0x7FFFFFF0ull);

  W.off.reserve(nc + 1, "offsets");
  W.ci.reserve(nc, "clouds");
  W.mn.reserve(3ull * nc, "bbox");
  W.mx.reserve(3ull * nc, "bbox");
  W.bucket.reserve(n, "bucket");
  W.hist.reserve(buckets + 1, "hist");
  W.tmp.reserve(n, "tmp");
  W.pts.reserve(nv, "pts");
  W.sos.reserve(nv, "sos");
  W.vcloud.reserve(nv, "vcloud");
  W.vtet.reserve(nv, "vtet");
  W.loc.reserve(nv, "loc");
  W.bigflag.reserve(nv, "bigflag");
  W.centry.reserve(nc, "centry");
  W.active.reserve(n, "active");
  W.active_next.reserve(n, "active");
  W.cand.reserve(n, "cand");
  W.cand_off.reserve(n, "cand");
  W.cand_len.reserve(n, "cand");
  W.cand_base.reserve(n, "cand");
  W.cand_nf.reserve(n, "cand");
  W.st1.reserve(nv, "status");
  W.bigcand.reserve(HUGE_SLOTS, "bigcand");
  // order-bucket regions: the expected n / kOrderBuckets starts per bucket
  // plus a 25% margin; anything beyond goes to the overflow region
  const uint64_t start_rc = n / kOrderBuckets + n / 64 + 1024;
  const uint64_t start_ovf = start_rc * kOrderBuckets;
  W.starts.reserve(start_ovf + n, "starts");
  // one overflow queue per lane group of a k_bfs wave
  W.wscratch.reserve(size_t(wave(k_bfs, 128)) * (128 / kBfsLanes) * BIG_CAP, "cavity queues");
  const uint32_t etab_warps = wave(k_write, 128) * 4;  // one edge table per warp of a k_write wave
  W.etab_key.reserve(size_t(etab_warps) * kEdgeSlotsG, "edge tables");
  W.etab_val.reserve(size_t(etab_warps) * 2 * kEdgeSlotsG, "edge tables");
  W.btab_key.reserve(size_t(kBigTables) * kBigTableSlots, "edge tables");
  W.btab_val.reserve(size_t(kBigTables) * 2 * kBigTableSlots, "edge tables");
  W.st2.reserve(nv, "status");
  const uint64_t pool_factor = std::min<uint32_t>(std::max<uint32_t>(cfg.pool_factor, 4u), 64u);
  const uint32_t pool_cap = uint32_t(std::min<uint64_t>(std::max<uint64_t>(n * pool_factor, 1 << 16), 1ull << 30));
  W.pool.reserve(pool_cap, "pool");
  W.big.reserve(size_t(HUGE_SLOTS) * HUGE_CAP, "big");
  W.ctr.reserve(1, "counters");
  W.lvl_off.reserve(size_t(maxtop + 1) * (nc + 1), "levels");
  W.lvl_total.reserve(maxtop + 1, "levels");
  W.state.reserve(1, "state");
  W.ccount.reserve(nc, "ccount");
  W.hullcnt.reserve(nc, "hull");
  W.cfill.reserve(nc, "cfill");
  W.hull.reserve(4ull * nc, "hull");
  W.coff.reserve(nc + 1, "coff");
  auto reserve_tets = [&](uint64_t cap) {
    W.T.reserve(cap, "tets");
    W.nslot.reserve(cap, "nslot");
    W.bface.reserve(cap, "boundary faces");
    W.C.reserve(cap, "claims");
    W.freed_a.reserve(cap, "freed");
    W.freed_b.reserve(cap, "freed");
    W.newid.reserve(cap, "newid");
  };
  reserve_tets(cap0);
  uint64_t cap = cap0;

  ck(cudaMemcpyAsync(W.off.p, job.offsets.data(), (nc + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s), "h2d");
  ck(cudaMemcpyAsync(W.ci.p, ci.data(), nc * sizeof(CloudInfo), cudaMemcpyHostToDevice, s), "h2d");
  ck(cudaMemsetAsync(W.mn.p, 0xFF, 3ull * nc * 4, s), "memset");
  ck(cudaMemsetAsync(W.mx.p, 0x00, 3ull * nc * 4, s), "memset");
  ck(cudaMemsetAsync(W.hist.p, 0, (buckets + 1) * 4, s), "memset");
  ck(cudaMemsetAsync(W.ctr.p, 0, sizeof(Counters), s), "memset");
  k_init_slots<<<blocks_for(cap, 256, 148 * 16), 256, 0, s>>>(W.T.p, W.C.p, 0, cap);
  if (vmode) {
    W.losses.reserve(nv, "losses");
    ck(cudaMemsetAsync(W.losses.p, 0, nv, s), "memset");
  }
  if (vmode == 2) {
    W.log_pslot.reserve(nv, "log slots");
    ck(cudaMemsetAsync(W.log_pslot.p, 0xFF, nv * 4, s), "memset");
  }
  if (vmode == 1) W.prio.reserve(nv, "claim priorities");
  // Rounds whose graph may see at most this many uninserted points use the
  // learned scheduler (its training log records the same rounds).
  const uint64_t learned_points = uint64_t(cfg.learned_gate ? cfg.learned_gate : 2048u) * 1024u;

  Dev D{};
  auto refresh = [&]() {
    D.pts = W.pts.p; D.sos = W.sos.p; D.vcloud = W.vcloud.p; D.vtet = W.vtet.p; D.loc = W.loc.p;
    D.bigflag = W.bigflag.p; D.T = W.T.p; D.C = W.C.p;
    D.nslot = W.nslot.p; D.bface = W.bface.p; D.cap = uint32_t(cap); D.nv = uint32_t(nv); D.centry = W.centry.p;
    D.cand = W.cand.p; D.cand_off = W.cand_off.p;
    D.cand_len = W.cand_len.p; D.cand_base = W.cand_base.p; D.cand_nf = W.cand_nf.p; D.st1 = W.st1.p; D.st2 = W.st2.p; D.bigcand = W.bigcand.p;
    D.starts = W.starts.p; D.wscratch = W.wscratch.p;
    D.start_rc = uint32_t(start_rc); D.start_ovf = uint32_t(start_ovf);
    D.etab_key = W.etab_key.p; D.etab_val = W.etab_val.p; D.etab_warps = etab_warps;
    D.btab_key = W.btab_key.p; D.btab_val = W.btab_val.p;
    D.prefilter = cfg.candidate_filter == 2 ? 0u : 1u; D.pool = W.pool.p; D.pool_cap = pool_cap; D.big = W.big.p;
    D.ctr = W.ctr.p;
    D.st = W.state.p; D.act[0] = W.active.p; D.act[1] = W.active_next.p;
    D.freed[0] = W.freed_a.p; D.freed[1] = W.freed_b.p; D.ci = W.ci.p; D.lvl_off = W.lvl_off.p;
    D.lvl_total = W.lvl_total.p; D.nc = nc;
    D.rule = int(job.cfg.insertion_rule == WTET_RULE_CENTROID ? 1 : 0);
    D.vote_mode = vmode;
    D.losses = vmode ? W.losses.p : nullptr;
    D.mlp = mlp_w;
    D.prio = vmode == 1 ? W.prio.p : nullptr;
    D.learned_points = uint32_t(std::min<uint64_t>(learned_points, 0xFFFFFFFFull));
    D.log_x = job.d_log_x;
    D.log_y = job.d_log_y;
    D.log_pslot = vmode == 2 ? W.log_pslot.p : nullptr;
    D.log_cap = uint32_t(std::min<uint64_t>(job.log_cap, 0xFFFFFFF0ull));
    D.log_shift = std::min<uint32_t>(job.log_shift, 31u);
  };
  refresh();

  // ---- normalise, Morton-bucket, scatter ----
  const uint32_t T = 256;
  uint32_t nb = uint32_t((n + T - 1) / T);
  k_bbox<<<nb, T, 0, s>>>(job.d_xyz, W.off.p, nc, n, W.mn.p, W.mx.p);
  k_normalize<<<nb, T, 0, s>>>(job.d_xyz, W.off.p, W.ci.p, nc, n, W.mn.p, W.mx.p, W.tmp.p, W.bucket.p, W.hist.p,
                               job.cfg.enable_hilbert_sorting ? 1 : 0);
  uint32_t hmask = 1;
  while (hmask < 2 * n) hmask <<= 1;
  W.dtab.reserve(hmask, "dedup table");
  W.dup.reserve(n, "dedup flags");
  hmask -= 1;
  ck(cudaMemsetAsync(W.dtab.p, 0xFF, size_t(hmask + 1) * 4, s), "memset");
  k_dedup_insert<<<nb, T, 0, s>>>(W.off.p, nc, n, W.tmp.p, W.dtab.p, hmask);
  k_dedup_mark<<<nb, T, 0, s>>>(W.off.p, nc, n, W.tmp.p, W.dtab.p, hmask, W.dup.p, &W.ctr.p->huge_used);
  uint64_t launches = 7;  // bbox, normalize, dedup x2, scatter, init, plus the scan below
  launches += scan_u32(W.hist.p, uint32_t(buckets + 1), s, W.scan_tmp);
  k_scatter_points<<<nb, T, 0, s>>>(W.off.p, W.ci.p, nc, n, W.tmp.p, W.bucket.p, W.hist.p, W.dup.p, D);
  k_init_clouds<<<(nc + 127) / 128, 128, 0, s>>>(W.ci.p, nc, D);
  ck(cudaGetLastError(), "setup kernels");
  uint32_t ndup = 0;
  ck(cudaMemcpyAsync(&ndup, &W.ctr.p->huge_used, 4, cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "dedup");
  if (ndup) {
    std::vector<uint8_t> flags(n);
    ck(cudaMemcpy(flags.data(), W.dup.p, n, cudaMemcpyDeviceToHost), "d2h");
    for (uint64_t i = 0; i < n; ++i)
      if (flags[i]) res.failed.push_back(i);
  }

  // ---- strata table: lvl_off[L][c] = first index of cloud c in stratum L ----
  std::vector<uint64_t> lvl(size_t(maxtop + 1) * (nc + 1));
  std::vector<uint32_t> lvl_total(maxtop + 1);
  for (uint32_t L = 0; L <= maxtop; ++L) {
    uint64_t acc = 0;
    for (uint32_t c = 0; c < nc; ++c) {
      lvl[size_t(L) * (nc + 1) + c] = acc;
      acc += level_count(ci[c].n, L, ci[c].top);
    }
    lvl[size_t(L) * (nc + 1) + nc] = acc;
    lvl_total[L] = uint32_t(acc);
  }
  ck(cudaMemcpyAsync(W.lvl_off.p, lvl.data(), lvl.size() * 8, cudaMemcpyHostToDevice, s), "h2d");

  wtet_stats st{};
  // max_insert_iterations bounds the rounds of each stratum (src/types.rs:44-46).
  // (the claim key holds a 16-bit round stamp)
  const uint32_t max_rounds = uint32_t(std::min<uint64_t>(
      uint64_t(std::max<uint32_t>(job.cfg.max_insert_iterations, 1u)) * (maxtop + 1), 65000ull));
  const char* tr = getenv("WTET_TRACE");
  const int trace = tr ? atoi(tr) : 0;
  const uint32_t TB = (cfg.block_size == 128 || cfg.block_size == 512) ? cfg.block_size : 256u;

  // ---- the round loop, driven from device state and replayed from a graph ----
  std::vector<uint32_t> lt(maxtop + 1);
  for (uint32_t L = 0; L <= maxtop; ++L) lt[L] = lvl_total[L];
  ck(cudaMemcpyAsync(W.lvl_total.p, lt.data(), (maxtop + 1) * 4, cudaMemcpyHostToDevice, s), "h2d");
  State S0{};
  S0.tet_top = nc;
  S0.next_level = int32_t(maxtop);
  S0.max_rounds = max_rounds;
  S0.overlap_shift = std::min<uint32_t>(cfg.overlap_shift, 16u);
  ck(cudaMemcpyAsync(W.state.p, &S0, sizeof(State), cudaMemcpyHostToDevice, s), "h2d");
  ck(cudaMemsetAsync(W.ctr.p, 0, sizeof(Counters), s), "memset");

  // Every round kernel loops grid-stride over its work, so each gets exactly
  // one full wave of resident blocks: an idle round then costs one short
  // wave per kernel.
  const uint32_t GB = HUGE_SLOTS;  // one block per huge-cavity slot
  struct Grids {
    uint32_t act, vote, cand, candl, logf, bfs, res, sh, wr, rel;
  };
  const Grids big{wave(k_activate, TB), 0u,      wave(k_cands, TB),
                  vmode == 1 ? wave(k_cands_learned, 256) : 0u,
                  wave(k_log_features, TB), wave(k_bfs, 128), wave(k_resolve, 128), wave(k_shared, 128),
                  wave(k_write, 128),  wave(k_relocate, TB)};
  // Rounds of the first strata have a few thousand points: a full wave of
  // blocks that exit at once costs more than their work, so those rounds
  // replay a graph with one block per SM.
  auto shrink = [](uint32_t g) { return std::min<uint32_t>(g, 148u); };
  const Grids small{shrink(big.act), 0u, shrink(big.cand), shrink(big.candl), shrink(big.logf),
                    shrink(big.bfs), shrink(big.res),  shrink(big.sh),   shrink(big.wr),    shrink(big.rel)};
  const uint64_t kernels_per_round = 9 + (vmode == 2 ? 1 : 0);

  // One round: k_end also starts the next round (k_begin starts the first).
  // `learned`: the learned scheduler's candidate kernel.
  auto enqueue_round = [&](const Grids& G, bool learned) {
    k_activate<<<G.act, TB, 0, s>>>(D);
    if (learned) k_cands_learned<<<G.candl, 256, 0, s>>>(D);
    else k_cands<<<G.cand, TB, 0, s>>>(D);
    if (vmode == 2) k_log_features<<<G.logf, TB, 0, s>>>(D);
    k_bfs<<<G.bfs, 128, 0, s>>>(D);
    k_expand_big<<<GB, 256, 0, s>>>(D);
    k_resolve<<<G.res, 128, 0, s>>>(D);
    k_shared<<<G.sh, 128, 0, s>>>(D);
    k_write<<<G.wr, 128, 0, s>>>(D);
    k_relocate<<<G.rel, TB, 0, s>>>(D);
    k_end<<<1, 32, 0, s>>>(D);
  };
  // Rounds per host check (the graph holds this many rounds).
  uint32_t rpg = std::min<uint32_t>(cfg.rounds_per_graph, 64u);
  if (trace) rpg = 1;
  // Three graphs: the first strata's rounds (one block per SM), the bulk
  // rounds (full waves), and with the learned scheduler the rounds in between
  // (full waves, learned candidate kernel).
  cudaGraphExec_t gexec = nullptr, gexec_small = nullptr, gexec_mid = nullptr;
  auto capture = [&](const Grids& G, bool learned) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    for (uint32_t r = 0; r < rpg; ++r) enqueue_round(G, learned);
    ck(cudaStreamEndCapture(s, &g), "end capture");
    ck(cudaGraphInstantiate(&e, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    return e;
  };
  auto destroy_graphs = [&]() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (gexec_small) cudaGraphExecDestroy(gexec_small);
    if (gexec_mid) cudaGraphExecDestroy(gexec_mid);
    gexec = gexec_small = gexec_mid = nullptr;
  };
  auto build_graph = [&]() {
    destroy_graphs();
    gexec = capture(big, false);
    gexec_small = capture(small, vmode == 1);
    if (vmode == 1) gexec_mid = capture(big, true);
  };
  // Points the next graph launch may see: the current list and the next two
  // strata (each stratum about doubles the previous one).
  auto upcoming = [&](const State& h) {
    uint64_t u = h.n_active;
    for (int L = h.next_level, k = 0; L >= 0 && k < 2; --L, ++k) u += lvl_total[L];
    return u;
  };
  constexpr uint64_t kSmallRoundPoints = WTET_SMALL_ROUND_POINTS;
  build_graph();
  k_begin<<<1, 32, 0, s>>>(D);
  launches += 1;
  State hs = S0;
  cudaEvent_t tr0 = nullptr, tr1 = nullptr;  // per-round device time when tracing
  if (trace) {
    ck(cudaEventCreate(&tr0), "event");
    ck(cudaEventCreate(&tr1), "event");
  }
  for (;;) {
    if (trace) ck(cudaEventRecord(tr0, s), "event record");
    const uint64_t u = upcoming(hs);
    ck(cudaGraphLaunch(u <= kSmallRoundPoints ? gexec_small : (gexec_mid && u <= learned_points) ? gexec_mid : gexec,
                       s),
       "graph launch");
    if (trace) ck(cudaEventRecord(tr1, s), "event record");
    launches += uint64_t(rpg) * kernels_per_round;
    ck(cudaMemcpyAsync(&hs, W.state.p, sizeof(State), cudaMemcpyDeviceToHost, s), "d2h");
    ck(cudaMemcpyAsync(W.h_ctr, W.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s), "d2h");
    ck(cudaStreamSynchronize(s), "rounds");
    const Counters& h = *W.h_ctr;
    if (trace) {
      float rms = 0.f;
      cudaEventElapsedTime(&rms, tr0, tr1);
      fprintf(stderr,
              "[wtet] round %u active %u winners %u expanded %llu cand %u inserted %u big %llu alloc %u top %u "
              "err %x ms %.3f\n",
              hs.round, hs.n_active, hs.last_starts, (unsigned long long)h.n_expanded, hs.last_cand,
              hs.last_inserted, (unsigned long long)h.n_big, hs.last_alloc, hs.tet_top, h.err, rms);
    }
    if (hs.stop == 1) {
      destroy_graphs();
      char buf[160];
      snprintf(buf, sizeof buf, "device consistency check failed (flags 0x%x) in round %u", h.err, hs.round);
      throw Error{(h.err & kErrPrec) ? WTET_ERR_PRECISION : WTET_ERR_INTERNAL, buf};
    }
    if (hs.stop == 3) {
      destroy_graphs();
      throw Error{WTET_ERR_NO_CONVERGE, "insertion did not converge within max_insert_iterations"};
    }
    if (hs.stop == 2) {
      // Grow the tet arrays (keeping contents); the displaced winners retry.
      uint64_t ncap = std::min<uint64_t>(cap * 3 / 2 + 1024, 0x7FFFFFF0ull);
      if (ncap <= cap) throw Error{WTET_ERR_CAPACITY, "tet capacity exhausted"};
      const uint32_t top = hs.tet_top;
      W.T.grow_keep(ncap, top, s, "grow tets");
      W.C.grow_keep(ncap, top, s, "grow claims");
      k_init_slots<<<blocks_for(ncap - top, 256, 148 * 16), 256, 0, s>>>(W.T.p, W.C.p, top, ncap);
      W.nslot.grow_keep(ncap, 0, s, "grow nslot");
      W.bface.grow_keep(ncap, 0, s, "grow boundary faces");
      W.freed_a.grow_keep(ncap, ncap > 0 ? W.freed_a.n : 0, s, "grow freed");
      W.freed_b.grow_keep(ncap, W.freed_b.n, s, "grow freed");
      W.newid.grow_keep(ncap, 0, s, "grow newid");
      cap = ncap;
      st.capacity_grows += 1;
      refresh();
      hs.stop = 0;
      ck(cudaMemcpyAsync(W.state.p, &hs, sizeof(State), cudaMemcpyHostToDevice, s), "h2d");
      uint32_t zero = 0;
      ck(cudaMemcpyAsync(&W.ctr.p->err, &zero, 4, cudaMemcpyHostToDevice, s), "clear err");
      ck(cudaStreamSynchronize(s), "grow");
      build_graph();
      k_begin<<<1, 32, 0, s>>>(D);  // the stopped round did not start its successor
      launches += 1;
      continue;
    }
    if (hs.done) break;
  }
  destroy_graphs();
  if (tr0) cudaEventDestroy(tr0);
  if (tr1) cudaEventDestroy(tr1);
  const uint32_t tet_top = hs.tet_top;
  const uint32_t round = hs.round;
  st.strata = hs.strata;
  st.inserted = hs.inserted;
  st.walk_steps = W.h_ctr->walk_steps;
  st.candidates = W.h_ctr->n_expanded;
  st.big_cavities = W.h_ctr->n_big;
  st.tets_created = W.h_ctr->created;
  st.rounds = round;
  st.vote_winners = hs.starts;
  res.logged = std::min<uint64_t>(hs.log_used, job.log_cap);

  // ---- output: per-cloud numbering, rows, infinity tets ----
  ck(cudaMemsetAsync(W.ccount.p, 0, nc * 4, s), "memset");
  ck(cudaMemsetAsync(W.hullcnt.p, 0, nc * 4, s), "memset");
  ck(cudaMemsetAsync(W.cfill.p, 0, nc * 4, s), "memset");
  uint32_t gt = blocks_for(tet_top, TB, 148 * 32);
  k_count<<<gt, TB, 0, s>>>(D, tet_top, W.ccount.p, W.hullcnt.p, W.hull.p);
  launches += 1;
  std::vector<uint32_t> ccount(nc);
  ck(cudaMemcpyAsync(ccount.data(), W.ccount.p, nc * 4, cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "count");
  res.tet_offsets.resize(nc + 1);
  uint64_t acc = 0;
  for (uint32_t c = 0; c < nc; ++c) {
    res.tet_offsets[c] = acc;
    acc += uint64_t(ccount[c]) + 4;
  }
  res.tet_offsets[nc] = acc;
  st.num_tets = acc;
  if (d_out_t && d_out_a && acc <= capacity) {
    ck(cudaMemcpyAsync(W.coff.p, res.tet_offsets.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, s), "h2d");
    k_number<<<gt, TB, 0, s>>>(D, tet_top, W.cfill.p, W.newid.p);
    k_emit<<<gt, TB, 0, s>>>(D, tet_top, W.newid.p, W.coff.p, d_out_t, d_out_a);
    k_infinity<<<(nc + 127) / 128, 128, 0, s>>>(D, W.ci.p, nc, W.ccount.p, W.hullcnt.p, W.hull.p, W.newid.p,
                                                W.coff.p, d_out_t, d_out_a);
    launches += 3;
    ck(cudaGetLastError(), "output kernels");
  }
  ck(cudaEventRecord(W.ev1, s), "event record");
  ck(cudaMemcpyAsync(W.h_ctr, W.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "output");
  if (W.h_ctr->err) {
    char buf[128];
    snprintf(buf, sizeof buf, "device consistency check failed in output (flags 0x%x)", W.h_ctr->err);
    throw Error{WTET_ERR_INTERNAL, buf};
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, W.ev0, W.ev1);
  st.device_ms = ms;
  st.kernel_launches = launches;
  res.stats = st;
  return res;
}

// ------------------------------------------------------- quality check ----

__global__ void k_check_quality(const float4* pts, uint32_t n, const uint4* tets, const uint4* adj, uint64_t m,
                                unsigned long long* out, uint32_t* err) {
  unsigned long long viol = 0, interior = 0;
  for (uint64_t ti = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; ti < m; ti += uint64_t(gridDim.x) * blockDim.x) {
    uint4 t = tets[ti];
    if (t.x >= n || t.y >= n || t.z >= n || t.w >= n) continue;
    ++interior;
    uint4 a = adj[ti];
    for (int f = 0; f < 4; ++f) {
      uint32_t packed = comp(a, f);
      if (packed == NONE) continue;
      uint64_t oti = packed >> 5;
      uint32_t of = packed & 3;
      if (ti >= oti) continue;
      if (oti >= m) {
        atomicOr(err, 1u);
        continue;
      }
      uint4 o = tets[oti];
      if (o.x >= n || o.y >= n || o.z >= n || o.w >= n) continue;
      uint32_t vb = comp(o, of);
      double P[5][3];
      load_pt(pts, t.x, P[0]);
      load_pt(pts, t.y, P[1]);
      load_pt(pts, t.z, P[2]);
      load_pt(pts, t.w, P[3]);
      load_pt(pts, vb, P[4]);
      int s = ex::insphere(P[0], P[1], P[2], P[3], P[4], err);
      if (s == 0) {
        // SoS keys are the input indices themselves.
        s = ex::orient4d_sos_degenerate(P[0], P[1], P[2], P[3], P[4], t.x, t.y, t.z, t.w, vb, err);
      }
      if (s < 0) ++viol;
    }
  }
  atomicAdd(&out[0], viol);
  atomicAdd(&out[1], interior);
}

__global__ void k_normalize_plain(const float* xyz, uint64_t n, const uint32_t* mn, const uint32_t* mx, float4* out) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float lo[3], ext[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = o2f(mn[k]);
    ext[k] = o2f(mx[k]) - lo[k];
  }
  float s = fmaxf(fmaxf(fmaxf(ext[0], ext[1]), ext[2]), 1e-10f);
  out[i] = make_float4(__fdiv_rn(__fsub_rn(xyz[3 * i], lo[0]), s), __fdiv_rn(__fsub_rn(xyz[3 * i + 1], lo[1]), s),
                       __fdiv_rn(__fsub_rn(xyz[3 * i + 2], lo[2]), s), 0.f);
}

// Single-cloud normalisation without the engine's workspace: the box is
// reduced with an offsets-free variant of k_bbox.
__global__ void k_bbox_one(const float* xyz, uint64_t n, uint32_t* mn, uint32_t* mx) {
  __shared__ uint32_t smn[3], smx[3];
  if (threadIdx.x < 3) {
    smn[threadIdx.x] = 0xFFFFFFFFu;
    smx[threadIdx.x] = 0u;
  }
  __syncthreads();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const float v = xyz[3 * i + k];
      if (v != v) continue;  // NaN is ignored, as f32::min / f32::max do
      atomicMin(&smn[k], f2o(v));
      atomicMax(&smx[k], f2o(v));
    }
  __syncthreads();
  if (threadIdx.x < 3) {
    atomicMin(&mn[threadIdx.x], smn[threadIdx.x]);
    atomicMax(&mx[threadIdx.x], smx[threadIdx.x]);
  }
}

void normalize_points_device(const float* d_xyz, uint64_t n, float4* d_out, uint32_t* box, cudaStream_t s) {
  ck(cudaMemsetAsync(box, 0xFF, 12, s), "memset");
  ck(cudaMemsetAsync(box + 3, 0x00, 12, s), "memset");
  if (n == 0) return;
  k_bbox_one<<<blocks_for(n, 256, 148 * 4), 256, 0, s>>>(d_xyz, n, box, box + 3);
  k_normalize_plain<<<uint32_t((n + 255) / 256), 256, 0, s>>>(d_xyz, n, box, box + 3, d_out);
  ck(cudaGetLastError(), "normalise kernels");
}

void check_quality_device(const float* d_xyz, uint64_t n, const uint32_t* d_tets, const uint32_t* d_adj, uint64_t m,
                          uint64_t* violations, uint64_t* interior, cudaStream_t s) {
  Workspace& W = ws();
  W.off.reserve(2, "off");
  W.mn.reserve(3, "bbox");
  W.mx.reserve(3, "bbox");
  W.tmp.reserve(n, "tmp");
  W.ctr.reserve(1, "ctr");
  uint64_t offs[2] = {0, n};
  ck(cudaMemcpyAsync(W.off.p, offs, 16, cudaMemcpyHostToDevice, s), "h2d");
  ck(cudaMemsetAsync(W.mn.p, 0xFF, 12, s), "memset");
  ck(cudaMemsetAsync(W.mx.p, 0, 12, s), "memset");
  ck(cudaMemsetAsync(W.ctr.p, 0, sizeof(Counters), s), "memset");
  uint32_t nb = uint32_t((n + 255) / 256);
  k_bbox<<<nb, 256, 0, s>>>(d_xyz, W.off.p, 1, n, W.mn.p, W.mx.p);
  k_normalize_plain<<<nb, 256, 0, s>>>(d_xyz, n, W.mn.p, W.mx.p, W.tmp.p);
  unsigned long long* out = reinterpret_cast<unsigned long long*>(&W.ctr.p->walk_steps);
  k_check_quality<<<blocks_for(m, 128, 148 * 16), 128, 0, s>>>(W.tmp.p, uint32_t(n), reinterpret_cast<const uint4*>(d_tets),
                                                                reinterpret_cast<const uint4*>(d_adj), m, out,
                                                                &W.ctr.p->err);
  ck(cudaMemcpyAsync(W.h_ctr, W.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "check");
  if (W.h_ctr->err & ~uint32_t(kErrPrec))
    throw Error{WTET_ERR_ARG, "adjacency refers to a tet out of range"};
  if (W.h_ctr->err & kErrPrec) throw Error{WTET_ERR_PRECISION, "exact arithmetic buffer overflow"};
  *violations = W.h_ctr->walk_steps;
  *interior = W.h_ctr->n_expanded;
}

void predicate_signs_device(const float* d_pts, const uint32_t* d_keys, uint64_t m, int32_t* d_o3, int32_t* d_o4,
                            cudaStream_t s) {
  Workspace& W = ws();
  W.ctr.reserve(1, "counters");
  ck(cudaMemsetAsync(W.ctr.p, 0, sizeof(Counters), s), "memset");
  if (m) k_predicate_signs<<<blocks_for(m, 128, 148 * 8), 128, 0, s>>>(d_pts, d_keys, m, d_o3, d_o4, &W.ctr.p->err);
  ck(cudaGetLastError(), "predicate kernel");
  uint32_t err = 0;
  ck(cudaMemcpyAsync(&err, &W.ctr.p->err, 4, cudaMemcpyDeviceToHost, s), "d2h");
  ck(cudaStreamSynchronize(s), "predicates");
  if (err) throw Error{WTET_ERR_PRECISION, "exact arithmetic buffer overflow"};
}

}  // namespace wtet
