// Internal declarations shared by the CUDA translation units of the
// Barnes-Hut force engine.  Nothing here is part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hierarquicos_bh.h"

namespace bh {

constexpr int kWarp = 32;

__host__ __device__ __forceinline__ int64_t bh_min64(int64_t a, int64_t b) { return a < b ? a : b; }
constexpr int kMaxDepth = 21;          // 3 * 21 = 63 key bits
constexpr int kNumLevels = kMaxDepth + 2;  // level_begin has L + 2 entries

// Error bits collected on the device and returned as status codes.
enum DeviceError : int {
  kErrNone = 0,
  kErrNonFinite = 1 << 0,      // NaN / Inf position or mass, or zero total mass
  kErrStackOverflow = 1 << 1,  // walk stack capacity exceeded
  kErrIndex = 1 << 2,          // internal index out of range (a bug)
  kErrDuplicates = 1 << 3,     // automatic depth impossible: coincident bodies
  kErrChildren = 1 << 4,       // more than 8 children (a bug)
  kErrTimeout = 1 << 5,        // a bounded wait inside a kernel gave up
};

// A batch is a set of independent systems stored back to back: system s owns
// bodies [off, off + n) of the concatenated arrays, in the caller's order, and
// after the sort the same range in key order.  Every kernel runs once for the
// whole batch; a lone system is a batch of one.

// Scalars of one system, computed on the device.  Plain doubles so that the
// host can read them back with one copy.
struct SysScalars {
  double bmin[3], bmax[3];      // bounding box of the positions
  double com[3], mass;          // centre of mass used for the keys
  double com_seq[3], mass_seq;  // centre of mass in the reference's sequential order
  double ssa;                   // side of the root cube, amp * largest extent
  double vcen[3];               // centre of the normalised box (keys)
  double key_margin;            // rounding margin of the keys, in finest cells
  int64_t off, n;               // the system's range of bodies
  int root;                     // compact node of the system's root, -1 if n < 2
  int key_ambiguous;            // a body lies within the rounding margin of a cell edge
  int key_mismatch;             // a key differs from the sequential-sum key
  int err;                      // DeviceError bits of this system
};

// Batch-wide scalars.
struct Scalars {
  int L;              // key depth actually used
  int n_compact;      // compact internal nodes of all systems
  int n_groups;       // target groups of all systems
  int err;            // DeviceError bits of any system
  int key_mismatch;   // any system
  int key_ambiguous;  // any system
  int max_lcp;        // deepest shared octal prefix (automatic depth, one system)
  int nsys;
};

// Work item of the per-system reductions: bodies [start, end) of system sys.
struct RedItem {
  int sys, pad;
  int64_t start, end;
};
constexpr int64_t kRedChunk = 8192;

// Device workspace of a batch.  Sized for `cap` bodies and `sys_cap` systems.
struct Buffers {
  int64_t cap = 0;
  int sys_cap = 0;
  // batch layout
  int nsys = 0;
  SysScalars *ss = nullptr;        // nsys entries
  SysScalars *ss_host = nullptr;   // host mirror
  int32_t *sys_of = nullptr;       // system of each body (same in input and key order)
  RedItem *items = nullptr;        // reduction work items
  int n_items = 0;
  int items_cap = 0;
  // inputs staged from the host (host-pointer API only)
  double *hm = nullptr, *hx = nullptr, *hy = nullptr, *hz = nullptr;
  double *hout = nullptr;
  // keys and sort
  uint64_t *k0 = nullptr, *k1 = nullptr;
  int32_t *v0 = nullptr, *v1 = nullptr;
  int32_t *hist = nullptr;
  int64_t hist_cap = 0;
  double *partials = nullptr;
  // sorted particles (x, y, z, m)
  double4 *spos = nullptr;
  // binary radix tree over the sorted keys (n - 1 internal nodes)
  int32_t *bn_left = nullptr, *bn_right = nullptr, *bn_parent = nullptr;
  int32_t *bn_first = nullptr, *bn_last = nullptr, *bn_level = nullptr;
  int32_t *bn_flag = nullptr, *bin2cn = nullptr;
  // compact octree, ordered by (level, first particle)
  int32_t *cn_bin = nullptr;
  int4 *cn_meta = nullptr;       // first, count, level, nchild
  int32_t *cn_child = nullptr;   // 8 per node; >= 0 node, < 0 particle ~p
  int32_t *cn_parent = nullptr;
  double4 *cn_com = nullptr;     // com x, y, z, mass
  double *cn_quad = nullptr;     // 6 per node: xx yy zz xy xz yz
  double *cn_oct = nullptr;      // 14 per node (octree_default.f90 layout)
  float4 *cn_fq = nullptr;       // 2 per node, normalised FP32 quadrupole + trace
  float4 *cn_fo = nullptr;       // 4 per node, normalised FP32 octupole
  int32_t *level_begin = nullptr;  // kNumLevels + 1 entries
  // target groups
  int32_t *gflag = nullptr, *gscan = nullptr, *g_first = nullptr;
  // scan scratch
  int32_t *scan_tmp = nullptr;
  int64_t scan_tmp_cap = 0;
  // walk
  int32_t *wstack = nullptr;
  int64_t wstack_cap = 0;   // entries per warp slot
  int64_t wstack_slots = 0; // stacks: the walk launches at most this many one-warp blocks
  int32_t *counters = nullptr;   // [0] group cursor
  unsigned long long *stats = nullptr;  // interaction counters
  Scalars *sc = nullptr;
  Scalars *sc_host = nullptr;    // pinned mirror
};

// ---- kernels / launchers (one translation unit each) ----

// batch layout: sys_of from the per-system offsets in `ss`
void launch_layout(Buffers &b, cudaStream_t s);
// keys: bbox + COM + keys of every system.  com_mode: 0 separate multiply and
// add, 1 fused.
void launch_keys(const double *m, const double *x, const double *y, const double *z, int64_t n,
                 int L, double amp, int com_mode, Buffers &b, cudaStream_t s);
void launch_seq_com(const double *m, const double *x, const double *y, const double *z,
                    int com_mode, int all, Buffers &b, cudaStream_t s);
void launch_verify_keys(const double *x, const double *y, const double *z, int64_t n, int all,
                        Buffers &b, cudaStream_t s);
void launch_auto_depth(int64_t n, Buffers &b, cudaStream_t s);
void launch_adopt_seq_com(Buffers &b, cudaStream_t s);
void launch_keys_only(const double *x, const double *y, const double *z, int64_t n, int L,
                      Buffers &b, cudaStream_t s);
void set_seq_com_smem_limit();
inline int grid_for(int64_t n, int threads, int cap) {
  int64_t g = (n + threads - 1) / threads;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Host-array transfers through a pool of host threads and pinned slots
// (bh_hostcopy.cu): pageable arrays are staged chunk by chunk while the copy
// engines move the neighbouring chunks.
enum class HostKind { kPageable, kPinned, kDevice };
HostKind host_kind(const void *p);
struct HostCopy;
HostCopy *hostcopy_create(int device);  // nullptr when a CUDA call failed
void hostcopy_destroy(HostCopy *h);
// count host arrays of n doubles into device arrays; st waits for them
cudaError_t hostcopy_upload(HostCopy *h, const double *const *src, double *const *dst, int count,
                            int64_t n, cudaStream_t st);
// n doubles of device memory into a host array after the work queued on st;
// returns when the host array is written
cudaError_t hostcopy_download(HostCopy *h, double *dst, const double *src, int64_t n,
                              cudaStream_t st);

// stable LSD radix sort of (key, value) pairs over bits [0, bits); the
// result ends in (k0, v0).  n_dev, when given, holds the element count on the
// device (n is then an upper bound).  A look-back wait that gives up sets
// kErrTimeout in *err (device).
void radix_sort_pairs(uint64_t *k0, int32_t *v0, uint64_t *k1, int32_t *v1, int64_t n,
                      const int32_t *n_dev, int bits, int32_t *hist, int *err, cudaStream_t s);
// the same for 32-bit keys when only the values are wanted: the last pass
// writes no keys and nothing is copied back; returns the buffer holding the
// sorted values (0: v0, 1: v1).  key_counts, if given, holds the number of keys
// of every key value 0..n_key_values-1 (the digit counts then come from it
// instead of from a pass over the keys).
int radix_sort_values32(uint32_t *k0, int32_t *v0, uint32_t *k1, int32_t *v1, int64_t n, int bits,
                        int32_t *hist, int *err, cudaStream_t s,
                        const int32_t *key_counts = nullptr, int64_t n_key_values = 0);
// scratch of the scan, in int32 entries: a ticket and a 64-bit word per
// 8192-value tile; scratch of the radix sort: digit counts of 8 passes x 256
// digits, 8 tile counters, and a 64-bit word per (pass, 4096-key tile, digit)
constexpr int64_t scan_tmp_entries(int64_t n) { return 2 * ((n + 8191) / 8192) + 4; }
// radix sort tiles: sorts of at most kSortSmallMax keys use small tiles (more
// blocks in flight: a 2^14-body build 0.380 -> 0.350 ms), larger ones large
// tiles (fewer look-back words and less scratch to clear: with small tiles
// the 2^20-body build took 0.873 instead of 0.821 ms)
constexpr int64_t kSortTileLarge = 4096, kSortTileSmall = 1024, kSortSmallMax = (int64_t)1 << 16;
constexpr int64_t sort_tile(int64_t n) { return n <= kSortSmallMax ? kSortTileSmall : kSortTileLarge; }
constexpr int64_t radix_hist_entries(int64_t n) {
  // the most tiles any sort of up to n keys uses
  return 8 * 256 + 8 +
         2 * 8 * 256 *
             ((((n < kSortSmallMax ? n : kSortSmallMax) + kSortTileSmall - 1) / kSortTileSmall >
                       (n + kSortTileLarge - 1) / kSortTileLarge
                   ? ((n < kSortSmallMax ? n : kSortSmallMax) + kSortTileSmall - 1) / kSortTileSmall
                   : (n + kSortTileLarge - 1) / kSortTileLarge) +
              1);
}

// exclusive scan of n int32 values in one launch; total written to *total
// and *total2 (device) when given; a look-back wait that gives up sets
// kErrTimeout in *err
void exclusive_scan(const int32_t *in, int32_t *out, int64_t n, const int32_t *n_dev,
                    int32_t *total, int32_t *tmp, int *err, cudaStream_t s,
                    int32_t *total2 = nullptr);

void launch_gather(const double *m, const double *x, const double *y, const double *z, int64_t n,
                   Buffers &b, cudaStream_t s);
// after the key sort of a batch: stable sort by system, so that every system's
// bodies are again contiguous, in key order
void launch_sort_by_system(int64_t n, Buffers &b, cudaStream_t s);
void launch_build_tree(int64_t n, int L, Buffers &b, cudaStream_t s);
void launch_upward(int64_t n, int L, int order, Buffers &b, cudaStream_t s);
void launch_groups(int64_t n, int group_size, int group_span, Buffers &b, cudaStream_t s);

// Runs the check of the pipelined walk's bounded mbarrier waits (one block
// of two warps; `cycles` is the short limit); out5 as in wait_probe_kernel.
int probe_bounded_wait(long long cycles, long long *out5);

struct WalkParams {
  double theta2, G, eps2;
  int order;       // 1, 4, 8
  int out_kind;    // 0 forces, 1 accelerations
  int precision;   // BH_PREC_*
  int group_size;  // 32 or 64
  int leaf_cap;
  int count_stats;
  int mac;         // 0 box distance, 1 box distance or every member's own MAC
  int pipeline = 0;  // FP32 walk: 0 one warp per group, 1 producer/consumer warps
  int g_begin = 0, g_end = -1;  // target groups walked: [g_begin, g_end), g_end < 0 = all
};
// Work buffers of Dehnen's dual-tree method (allocated on first use, grown on
// demand): entity arrays for nodes and bodies (2n entities), the pair
// frontier, the mutual pairs and their sorted one-sided terms.
struct DehnenBuffers {
  double *rmax = nullptr, *F = nullptr, *H = nullptr, *T = nullptr;
  int64_t rmax_cap = 0, F_cap = 0, H_cap = 0, T_cap = 0;
  double *squad = nullptr;                // every node's quadrupole over its mass
  int64_t squad_cap = 0;
  int2 *front = nullptr, *mut = nullptr;
  int64_t front_cap = 0, mut_cap = 0;
  int64_t want_front = 0, want_mut = 0;   // pairs per frontier buffer, mutual pairs
  uint32_t *keys = nullptr;               // one-sided terms: target (key), source (value)
  int32_t *vals = nullptr, *cnt = nullptr, *beg = nullptr, *hist = nullptr, *scan_tmp = nullptr;
  unsigned long long *counters = nullptr;
  int64_t keys_cap = 0, vals_cap = 0, cnt_cap = 0, beg_cap = 0, hist_cap = 0, scan_tmp_cap = 0,
          counters_cap = 0;
  uint64_t *gen_status = nullptr;         // chained-scan words of every traversal generation
  int64_t gen_status_cap = 0;
  int32_t *gen_tiles = nullptr;           // tile tickets, one counter per generation
  int64_t gen_tiles_cap = 0;
  int64_t pairs = 0;                      // mutual interactions of the last run
};
// Dehnen's method over the built batch into out (same layout as the walk).
// Synchronises the stream once (to size the pair lists).  Returns 0, 1 out of
// device memory, 2 CUDA error, 3 traversal did not close, 4 pair lists too
// large.
int run_dehnen(int64_t n, const WalkParams &p, Buffers &b, DehnenBuffers &d, double *out,
               cudaStream_t s);
void free_dehnen(DehnenBuffers &d);

// Returns the number of warp slots used (for stack sizing).
void launch_walk(int64_t n, const WalkParams &p, Buffers &b, double *out, cudaStream_t s);
void launch_reference_walk(int64_t n, const WalkParams &p, Buffers &b, double *out,
                           const int64_t *targets, int64_t ntargets, int64_t *counts,
                           cudaStream_t s);
int64_t walk_slots();
int probe_fma(double *gflops2);

void launch_direct(const double *m, const double *x, const double *y, const double *z, int64_t n,
                   const int64_t *targets, int64_t ntargets, double G, double eps2, int out_kind,
                   double *out, cudaStream_t s);

}  // namespace bh

struct bh_system;
// bh_abi.cu: records `msg` as the calling thread's last error, returns code
int bh_report_error(int code, const char *msg);
namespace bh {
// bh_abi.cu: a system whose workspace is `b` (caller-owned, never grown)
bh_system *fixed_system_create(int device, const Buffers &b, Scalars *host_sc,
                               SysScalars *host_ss);
}  // namespace bh
