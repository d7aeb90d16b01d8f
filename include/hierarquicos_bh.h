/*
 * hierarquicos_bh.h -- C ABI of the B200 Barnes-Hut force engine.
 *
 * Plain C types only: host or device pointers to float64 arrays, sizes as
 * int64_t, and an optional CUDA stream passed as void* (NULL = the legacy
 * default stream).  Every function returns a status code (BH_OK on success);
 * bh_last_error() gives the message of the last failure on the calling thread.
 *
 * Layout conventions, matching the reference's f2py module api_mod:
 *  - inputs are four separate float64 vectors m, x, y, z of length n;
 *  - results are written SoA, out[0..n) = fx, out[n..2n) = fy,
 *    out[2n..3n) = fz, which is the memory layout of the Fortran (N,3) array
 *    that api_mod.compute_forces returns;
 *  - theta and eps are passed unsquared and squared inside, as
 *    parareal/api3d.f90:30 does.
 */
#ifndef HIERARQUICOS_BH_H
#define HIERARQUICOS_BH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define BH_OK 0
#define BH_ERR_INVALID 1     /* bad argument (size, order, depth, pointer)          */
#define BH_ERR_CUDA 2        /* CUDA runtime error                                 */
#define BH_ERR_NOMEM 3       /* device allocation failed                           */
#define BH_ERR_NONFINITE 4   /* NaN/Inf input or zero total mass                   */
#define BH_ERR_CAPACITY 5    /* walk stack capacity exceeded (after retries)        */
#define BH_ERR_DUPLICATES 6  /* depth 0 asked but coincident bodies never separate  */
#define BH_ERR_INTERNAL 7    /* an internal consistency check failed               */
#define BH_ERR_NOT_BUILT 8   /* system queried before a successful build           */

/* ---- walk precision ---- */
#define BH_PREC_FP32 0       /* warp-cooperative group walk, FP32, Kahan-compensated */
#define BH_PREC_FP64 1       /* the same group walk in FP64                          */
#define BH_PREC_REFERENCE 2  /* per-target FP64 walk with the reference's MAC        */
#define BH_PREC_DEHNEN 3     /* Dehnen's dual-tree method in FP64 (octree_default.f90
                                :1095-1712, methods 20/21/22); the call synchronises
                                its stream once and cannot be captured in a graph    */

typedef struct bh_params {
    double theta;     /* opening angle, unsquared                                 */
    double G;         /* gravitational constant                                   */
    double eps;       /* softening length, unsquared                              */
    int order;        /* 1 monopole, 4 quadrupole, 8 octupole                     */
    int out_kind;     /* 0 forces G m_i a_i, 1 accelerations G a_i                */
    int depth;        /* Morton depth L in 1..21; 0 = smallest depth with unique keys */
    int precision;    /* BH_PREC_*                                                */
    double amp;       /* root cube side = amp * largest extent (reference: 1.2)   */
    int group_size;   /* targets per warp in the group walk: 32 or 64             */
    int leaf_cap;     /* nodes with <= leaf_cap bodies are opened into bodies (1..16) */
    int com_mode;     /* centre of mass for the keys: 0 separately rounded m*q,
                         1 fused multiply-add (what gfortran -O3 -march=native emits) */
    int strict_keys;  /* 1: keys provably equal the reference's: every body is checked
                         against the rounding margin of its cell edges, and only if one
                         lies inside it is the reference's sequential centre of mass
                         computed and the build redone when a key differs;
                         2: always run that sequential check; 0: no check          */
    int count_stats;  /* 1: the group walk counts its interactions (bh_system_get_stats) */
    int group_span;   /* target groups: consecutive subtrees of <= group_span bodies are
                         concatenated in key order and cut into groups of group_size;
                         0 = 2 * group_size                                         */
    int mac;          /* group walk acceptance of a node: 0 the group's box distance
                         (octree_default.f90:1927-1936); 1 also accept a node that
                         fails it when it holds none of the group's bodies and passes
                         every group member's own MAC (morton_octree.f90:701-706)   */
    int pipeline;     /* FP32 group walk: 0 one warp walks a group and evaluates it;
                         1 producer warps walk the tree and stage the batches into a
                         shared-memory ring, consumer warps evaluate them (the same
                         results bit for bit; no reference counterpart)            */
} bh_params;

/* Defaults: theta 0.5, G 1, eps 0, order 4, forces, depth 21, FP32, amp 1.2,
 * group 64, leaf_cap 8, com_mode 1, strict_keys 1, count_stats 0, group_span 0,
 * mac 1, pipeline 1. */
void bh_params_default(bh_params *p);

const char *bh_version(void);
int bh_last_error(char *buf, int len);

/* Drop-in for api_mod.compute_forces (fortran/api3d.f90:20-41; REAL(16) twin
 * parareal/api3d.f90:20-44): host arrays in, forces (N,3) out, every call a
 * fresh tree.  order: 1 monopole, 4 quadrupole (the f2py quad=.TRUE.), 8
 * octupole.  out_kind 0 forces, 1 accelerations.  Host arrays may be pinned
 * (copied straight by the copy engines, overlapped on several streams) or
 * ordinary pageable memory (staged through pinned chunks by a pool of host
 * threads while the copy engines move the neighbouring chunks); a device
 * pointer is refused (BH_ERR_INVALID).  Returns when out is written. */
int bh_compute_forces(const double *m, const double *x, const double *y, const double *z,
                      int64_t n, double theta, double G, double eps, int order, int out_kind,
                      double *out, void *stream);

/* bh_compute_forces with every parameter (host arrays). */
int bh_compute_forces_ex(const double *m, const double *x, const double *y, const double *z,
                         int64_t n, const bh_params *p, double *out, void *stream);

/* Drop-in for api_mod.compute_forces_direct (fortran/api3d.f90:43-72) and
 * direct_forces_mod.compute_forces_direct (fortran/direct_forces.f90:8-63):
 * FP64 O(N^2) sum on the device.  Host arrays. */
int bh_compute_forces_direct(const double *m, const double *x, const double *y,
                             const double *z, int64_t n, double G, double eps, int out_kind,
                             double *out, void *stream);

/* FP64 direct sum on a subset of targets, DEVICE arrays: out is SoA over the
 * ntargets targets (original indices in d_targets).  Used for error checks. */
int bh_direct_targets_device(const double *d_m, const double *d_x, const double *d_y,
                             const double *d_z, int64_t n, const int64_t *d_targets,
                             int64_t ntargets, double G, double eps, int out_kind, double *d_out,
                             void *stream);

/* ---- device-resident systems (replaces OctreeType / morton_tree_type:
 *      pre_init + init, octree_default.f90:178-387, morton_octree.f90:73-111) ---- */
typedef struct bh_system bh_system;

int bh_system_create(bh_system **sys, int device);
int bh_system_destroy(bh_system *sys);

/* Keys, sort, octree and multipoles for DEVICE arrays (morton_octree.f90:328-625,
 * octree_default.f90:744-882).  Asynchronous on `stream`. */
int bh_system_build(bh_system *sys, const double *d_m, const double *d_x, const double *d_y,
                    const double *d_z, int64_t n, const bh_params *p, void *stream);

/* Tree walk over the built tree (octree_default.f90:1811-2095 grouped walk;
 * morton_octree.f90:627-766 with BH_PREC_REFERENCE); d_out SoA n x 3 in the
 * ORIGINAL particle order.  Asynchronous. */
int bh_system_walk(bh_system *sys, const bh_params *p, double *d_out, void *stream);

/* The group walk over target groups [g_begin, g_end) only (groups are Morton-
 * contiguous runs of bodies; bh_system_info gives their number; g_end beyond
 * it is clamped): forces of those groups' bodies are written, all others are
 * left as they are.  For sharding one system's targets over GPUs: every rank
 * builds the whole tree, walks its range of groups into a zeroed d_out, and a
 * sum over the ranks (one all-reduce) gives the full result, bit for bit the
 * single-GPU walk's.  FP32 / FP64 group walk only.  Asynchronous. */
int bh_system_walk_groups(bh_system *sys, const bh_params *p, int64_t g_begin, int64_t g_end,
                          double *d_out, void *stream);

/* build + walk + bh_system_sync: the device-array form of bh_compute_forces. */
int bh_system_forces(bh_system *sys, const double *d_m, const double *d_x, const double *d_y,
                     const double *d_z, int64_t n, const bh_params *p, double *d_out,
                     void *stream);

/* Waits for the stream and turns device-side error flags into a status. */
int bh_system_sync(bh_system *sys, void *stream);

/* ---- batches of independent systems (no reference counterpart: the
 *      reference evaluates one system per api_mod.compute_forces call,
 *      fortran/api3d.f90:20-41, and callers loop over systems) ----
 * A batch is nsys systems stored back to back in DEVICE arrays: system s owns
 * entries [offsets[s], offsets[s+1]) of d_m, d_x, d_y, d_z (offsets is a HOST
 * array of nsys + 1 entries, offsets[0] = 0, strictly increasing).  Every
 * phase runs once for the whole batch; each system gets its own box, centre
 * of mass, keys, octree and groups, and its result is the one a build of that
 * system alone gives (bit for bit).  d_out holds one SoA block per system:
 * entries [3 offsets[s], 3 offsets[s+1]) are Fx, Fy, Fz of system s (the
 * (n_s, 3) Fortran array of that system).  depth 0 (automatic) needs nsys 1. */
int bh_system_build_batch(bh_system *sys, const double *d_m, const double *d_x,
                          const double *d_y, const double *d_z, const int64_t *offsets,
                          int nsys, const bh_params *p, void *stream);

/* build_batch + walk + sync. */
int bh_system_forces_batch(bh_system *sys, const double *d_m, const double *d_x,
                           const double *d_y, const double *d_z, const int64_t *offsets,
                           int nsys, const bh_params *p, double *d_out, void *stream);

/* Allocates the workspace for batches of up to n bodies in up to nsys
 * systems now, so that later builds within those bounds allocate nothing. */
int bh_system_reserve(bh_system *sys, int64_t n, int nsys);

/* Root node, centre of mass + mass (com4, 4 per system) and root cube side of
 * every system of the last build, copied to HOST arrays (any may be NULL). */
int bh_system_batch_info(bh_system *sys, int32_t *roots, double *com4, double *ssa);

/* Records the build and the walk of the current batch (the layout, device
 * input pointers and sizes of the last build, with the parameters p and
 * output d_out) into a CUDA graph owned by the handle.  A replay repeats that
 * work on whatever the input arrays hold then; follow it with bh_system_sync.
 * A build with another layout or size drops the graph. */
int bh_system_capture(bh_system *sys, const bh_params *p, double *d_out);
int bh_system_replay(bh_system *sys, void *stream);

/* After a build: particle count, depth L, compact node count, group count,
 * centre of mass + total mass (com4), root cube side. Synchronises. */
int bh_system_info(bh_system *sys, int64_t *n, int *depth, int64_t *n_nodes, int64_t *n_groups,
                   double *com4, double *ssa);

/* Sorted Morton keys and the permutation (sorted position -> original index),
 * copied to HOST buffers of n entries (morton_octree.f90:404-417). */
int bh_system_get_keys(bh_system *sys, uint64_t *keys, int32_t *perm);

/* Compact octree copied to HOST buffers (any pointer may be NULL), node count
 * from bh_system_info.  meta4: first, count, level, nchild per node; child8:
 * 8 per node, >= 0 a node, < 0 the particle ~c at sorted position; com4:
 * x, y, z, mass; quad6: xx yy zz xy xz yz; oct14: octree_default.f90 layout;
 * level_begin: L + 2 entries. */
int bh_system_get_nodes(bh_system *sys, int32_t *meta4, int32_t *child8, int32_t *parent,
                        double *com4, double *quad6, double *oct14, int32_t *level_begin);

/* Group ranges (first sorted particle of each group), n_groups + 1 entries. */
int bh_system_get_groups(bh_system *sys, int32_t *group_first);

/* Interaction counters of the last walk with counting enabled (count_stats = 1
 * in bh_params): [0] body-body, [1] body-cell, [2] groups, [3] node tests. */
int bh_system_get_stats(bh_system *sys, uint64_t *stats4);

/* Strict-key slow path of this handle since its creation (strict_keys 1/2 in
 * bh_params): checks2[0] = completed builds for which the reference's
 * sequential centre of mass (morton_octree.f90:364-370) was computed because
 * a body lay within the rounding margin of a cell edge (or strict_keys 2);
 * checks2[1] = builds redone because a key differed.  Host counters: no
 * device work, no synchronisation. */
int bh_system_get_key_checks(bh_system *sys, int64_t *checks2);

/* Per-target FP64 walk with the reference's semantics on a subset of targets
 * (DEVICE arrays, original indices); counts (optional, device, 2 per target):
 * body-body and cell interactions. */
int bh_system_reference_targets(bh_system *sys, const bh_params *p, const int64_t *d_targets,
                                int64_t ntargets, double *d_out, int64_t *d_counts,
                                void *stream);

/* Allocation-free force evaluation, for callers that may not allocate device
 * memory (their memory belongs to another allocator, a cudaMalloc would stall
 * their time-step loop, or their host forbids it).  No counterpart in the
 * reference.  Device inputs and output as bh_system_forces; everything else
 * comes from one fixed device array of about 7.9 MB inside the library, so n
 * is limited to BH_NOALLOC_MAX_N (larger n: BH_ERR_INVALID).  The first call on
 * a device looks that array up; all calls on a device share it, so calls that
 * overlap on the GPU race: run them one after another.  Synchronous: the call
 * synchronises its stream, so it cannot be captured into a CUDA graph (a call
 * on a capturing stream returns BH_ERR_INVALID and queues nothing). */
#define BH_NOALLOC_MAX_N 8192
int bh_compute_forces_noalloc(const double *d_m, const double *d_x, const double *d_y,
                              const double *d_z, int64_t n, const bh_params *p, double *d_out,
                              void *stream);

/* ---- time integration (momentum form, FP64 state; batch layout as above:
 *      positions, momenta and masses concatenated by system, d_offsets a
 *      DEVICE copy of the nsys + 1 offsets, forces in the walk's per-system
 *      (n_s, 3) blocks) ----
 * For every body: p += kick1 f (skipped when kick1 = 0), p += kick2 f (skipped
 * when kick2 = 0), then q += (drift p) / m (skipped when drift = 0), with the
 * reference's operation order and no contraction.  Velocity Verlet
 * (parareal/parareal.f90:55-63; benchmarks/integration_verlet/integration.f90:
 * 152-168) is kick_drift(0, dt/2, dt), forces, and at each later step
 * kick_drift(dt/2, dt/2, dt), with a closing kick_drift(dt/2, 0, 0); the
 * symplectic Euler coarse step (parareal/parareal.f90:20-35) is
 * kick_drift(dt, 0, dt) after the forces. */
int bh_kick_drift(const double *d_m, const double *d_f, double *d_x, double *d_y, double *d_z,
                  double *d_px, double *d_py, double *d_pz, const int64_t *d_offsets, int nsys,
                  int64_t n, double kick1, double kick2, double drift, void *stream);

/* bh_kick_drift with coefficients per system: d_coef (DEVICE) holds kick1,
 * kick2, drift for each of the nsys systems (all zero: the system is left as
 * it is).  One launch advances systems at different stages of their steps. */
int bh_kick_drift_systems(const double *d_m, const double *d_f, double *d_x, double *d_y,
                          double *d_z, double *d_px, double *d_py, double *d_pz,
                          const int64_t *d_offsets, int nsys, int64_t n, const double *d_coef,
                          void *stream);

/* Conserved quantities per system (parareal/api3d.f90:108-153, in FP64): d_out
 * gets 9 doubles per system: total energy, kinetic, potential (softened pair
 * sum, each pair once), linear momentum (3), angular momentum q x p (3).
 * d_scratch: 8 n doubles.  O(n_s^2) per system. */
int bh_diagnostics(const double *d_m, const double *d_x, const double *d_y, const double *d_z,
                   const double *d_px, const double *d_py, const double *d_pz,
                   const int64_t *d_offsets, int nsys, int64_t n, double G, double eps,
                   double *d_scratch, double *d_out, void *stream);

/* ---- initial conditions on the device (initial_values/initial_values.f90:
 *      51-381; plummer.f90, hernquist.f90, homogeneous.f90) ----
 * profile: 0 uniform cube, 1 uniform sphere, 2 Plummer, 3 homogeneous sphere,
 * 4 Hernquist; par: b, R or a; size_qs >= 0 truncates radii (rejection),
 * size_ps >= 0 bounds the speeds; nm 1 equal masses 1/n, 0 random masses
 * summing to 1; two_d zeroes z.  Writes d_m (n), d_q and d_p (SoA, 3 n:
 * x block, y block, z block; momenta p = m v) with the centre of mass and the
 * total momentum at zero.  Counter-based streams: the result depends only on
 * the seed and n.  d_scratch: 2400 doubles.  Synchronous. */
int bh_generate_ics(int profile, int64_t n, double size_qs, double size_ps, int two_d, int nm,
                    double G, double par, uint64_t seed, int velocities, double *d_m,
                    double *d_q, double *d_p, double *d_scratch, void *stream);

/* Fused-multiply-add throughput probe (independent chains, CUDA events):
 * writes GFLOP/s into gflops2[0] (FP32), gflops2[1] (FP64) and gflops2[2]
 * (FP32 issued as paired f32x2 instructions); gflops2 holds 3 doubles. */
int bh_probe_fma_peak(int device, double *gflops2);

/* Check of the bounded waits of the pipelined walk (no reference counterpart):
 * one block of two warps uses the walk's mbarrier wait.  Warp 0 waits
 * `cycles` clock cycles (1e3..1e9) on a barrier nothing arrives at, gives up
 * and raises the block's abort flag; warp 1, waiting on the same barrier with
 * the walk's own limit (about 2 s), must be released by that flag.  out5:
 * [0] warp 0's result (0 = gave up), [1] 1 when a barrier phase that does
 * complete was seen, [2] warp 1's result (0 = released), [3] the cycles warp 1
 * waited, [4] the abort flag (1).  Synchronous; allocates 40 bytes. */
int bh_probe_bounded_wait(int device, long long cycles, long long *out5);

#ifdef __cplusplus
}
#endif

#endif /* HIERARQUICOS_BH_H */
