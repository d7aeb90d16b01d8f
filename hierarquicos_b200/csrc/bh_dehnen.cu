// Dehnen's dual-tree method on the device, FP64: fortran/octree_default.f90
// :1095-1712 (methods 20/21/22; Dehnen 2000, with the octupole torque term of
// :1530-1557 for multipole 8).
//
// The tree is the compact octree of the build.  Entities are its nodes
// [0, M) and the bodies n + p (sorted position p); a body is a leaf with no
// extent (rmax 0), a node's children are its child nodes and lone bodies, or,
// for a node of identical keys, its bodies.
//
//  1. rmax (evaluate_rmax :1095-1131), from the leaves up in one launch: the
//     largest distance from a node's centre of mass to any child's centre of
//     mass plus that child's rmax (massless children skipped).
//  2. Dual traversal (mutual_interaction_walk_* :1133-1402) as a sequence of
//     generations of node pairs, starting from (root, root) of every system:
//     a pair with a massless member is dropped; (a, a) becomes the pairs of
//     a's children (i <= j; a body with itself is dropped); a pair with
//     (rmax_a + rmax_b)^2 <= theta^2 |z_a - z_b|^2 is a mutual interaction;
//     otherwise the member with the larger rmax (a on ties) is replaced by its
//     children.  Each generation is one launch over the previous one's pairs,
//     a deterministic compaction (a chained scan over tiles of input pairs):
//     the new frontier and the mutual pairs come out in input order, so both
//     lists have one order whatever the schedule, and a system's pairs keep
//     their relative order inside a batch.  The lists live in preallocated
//     buffers whose fill the host reads once at the end, growing them and
//     repeating when one overflowed.
//  3. Each mutual pair (a, b) becomes the two one-sided terms (a <- b) and
//     (b <- a) of :1200-1221, keyed by target and sorted stably (radix passes
//     over the target id only), so every target sums its terms in the mutual
//     list's fixed order (results do not depend on the schedule nor on the
//     other systems of a batch).  Term (t <- s), with
//     R = z_t - z_s (evaluate_mutual_interaction_* :1425-1558):
//       field  += M_s (D1 + Q_s : D3 / (2 M_s))      D1 = -G R r^-3
//       hess   += M_s D2,  third += M_s D3           (r^2 = R^2 + eps^2)
//       field  += (octupole) 0.5 (3 G r^-5 c - 15 G r^-7 C:RR) / M_t,
//                 C_jkl = M_s O_t,jkl - M_t O_s,jkl, c_j = C_jkk
//                 (summed over the target's terms, then halved and divided
//                 by M_t once)
//     which is the reference's update of both nodes written once per side.
//     Terms between coincident points without softening (r = 0) are skipped.
//  4. Downward pass (dehnen_forces :1560-1673): child field += parent field +
//     H d + d.T.d / 2, child hessian += H + T d, child third += T, d = child
//     centre of mass - parent's.  The translation of this cubic expansion is
//     exact, so one launch lets every body sum its ancestors' own expansions
//     translated straight to it (down_bodies_kernel) instead of pushing level
//     by level.  A body's force is m times its field.
#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int kGenerations = 2 * (kMaxDepth + 2) + 4;  // each generation deepens a pair

struct Ent {
  const int4 *meta;
  const int32_t *child;
  const double4 *com;
  const double4 *spos;
  const double *quad;
  const double *squad;  // quad / mass per node (order >= 4)
  const double *oct;
  const double *rmax;
  int64_t n;  // bodies: entity n + p is body p
};

__device__ __forceinline__ double4 ent_com(const Ent &e, int64_t i) {
  return i < e.n ? e.com[i] : e.spos[i - e.n];
}
__device__ __forceinline__ double ent_rmax(const Ent &e, int64_t i) {
  return i < e.n ? e.rmax[i] : 0.0;
}
__device__ __forceinline__ int node_nchild(int4 mt) { return mt.w > 0 ? mt.w : mt.y; }
__device__ __forceinline__ int64_t node_child(const Ent &e, int64_t j, int4 mt, int k) {
  if (mt.w > 0) {
    const int32_t c = e.child[8 * j + k];
    return c >= 0 ? (int64_t)c : e.n + (int64_t)(~c);
  }
  return e.n + mt.x + k;
}

// rmax of node j from its children (evaluate_rmax, octree_default.f90:1095-1131);
// the children's rmax is read through L2 (ld.cg) because another thread of
// the same launch may have written it.
__device__ __forceinline__ double node_rmax(const Ent &e, int j) {
  const int4 mt = e.meta[j];
  const double4 c = e.com[j];
  double r = 0.0;
  const int k = node_nchild(mt);
  for (int q = 0; q < k; ++q) {
    const int64_t ch = node_child(e, j, mt, q);
    const double4 cc = ent_com(e, ch);
    if (cc.w == 0.0) continue;
    const double dx = cc.x - c.x, dy = cc.y - c.y, dz = cc.z - c.z;
    const double v = sqrt(dx * dx + dy * dy + dz * dz) + (ch < e.n ? __ldcg(e.rmax + ch) : 0.0);
    if (v > r) r = v;
  }
  return r;
}

__device__ __forceinline__ int node_children_count(const Ent &e, int j) {
  const int4 mt = e.meta[j];
  if (mt.w == 0) return 0;
  int k = 0;
  for (int q = 0; q < mt.w; ++q) k += e.child[8 * (int64_t)j + q] >= 0 ? 1 : 0;
  return k;
}

// All of evaluate_rmax in one launch, bottom-up with an arrival counter per
// node (the scheme of the upward pass): a thread starts at every node without
// node children, and the last child to arrive at a parent goes on with it.
// Every node is computed once, after its children, with the same arithmetic
// as the level-by-level form.  A chain longer than the deepest tree raises
// kErrIndex instead of looping.
__global__ void __launch_bounds__(256)
rmax_fused_kernel(const Scalars *__restrict__ scr, Ent e, const int32_t *__restrict__ parent,
                  double *rmax, int32_t *arrive, int *err) {
  const int M = scr->n_compact;
  for (int j0 = blockIdx.x * blockDim.x + threadIdx.x; j0 < M; j0 += gridDim.x * blockDim.x) {
    if (node_children_count(e, j0) != 0) continue;
    int j = j0;
    for (int step = 0;; ++step) {
      if (step > kNumLevels + 1) { atomicOr(err, kErrIndex); break; }
      rmax[j] = node_rmax(e, j);
      const int p = parent[j];
      if (p < 0) break;
      const int need = node_children_count(e, p);
      __threadfence();
      if (atomicAdd(&arrive[p], 1) != need - 1) break;
      __threadfence();
      j = p;
    }
  }
}

// Every node's quadrupole divided by its mass, once, for the terms that use
// it as a source (the same correctly rounded quotients the terms would form).
__global__ void __launch_bounds__(256)
spec_quad_kernel(const Scalars *__restrict__ scr, const double4 *__restrict__ com,
                 const double *__restrict__ quad, double *__restrict__ squad) {
  const int M = scr->n_compact;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
    const double m = com[j].w;
#pragma unroll
    for (int q = 0; q < 6; ++q) squad[6 * (int64_t)j + q] = m != 0.0 ? quad[6 * (int64_t)j + q] / m : 0.0;
  }
}

// The first frontier: (root, root) of every system, in system order (a
// system without a tree contributes (-1, -1), which the traversal drops).
__global__ void roots_frontier_kernel(const SysScalars *__restrict__ ss, int nsys, int2 *fout,
                                      unsigned long long *nout) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys) fout[s] = make_int2(ss[s].root, ss[s].root);
  if (s == 0) *nout = (unsigned long long)nsys;
}

constexpr int kGenThreads = 256;            // threads of a block; one tile per block at a time
constexpr int kGenItems = 4;                // consecutive input pairs per thread
constexpr int kGenBlocksPerSm = 4;          // 64 registers a thread: 32 warps per SM hide the loads
constexpr int kGenTile = kGenThreads * kGenItems;
constexpr int kGenWarps = kGenThreads / kWarp;
constexpr int kGenMutBits = 11;  // packed block scan: mutual count in the low bits
constexpr int kGenMutMask = (1 << kGenMutBits) - 1;
static_assert(kGenTile < (1 << kGenMutBits), "a tile's mutual pairs fit the low bits");
static_assert((int64_t)kGenTile * 36 << kGenMutBits < (1ll << 31), "the packed count fits an int");
// tile words of the chained scan: top 2 bits the state, low 62 bits the count
constexpr uint64_t kGenAggregate = 1ull << 62;  // the tile's own count
constexpr uint64_t kGenInclusive = 2ull << 62;  // sum of the counts of tiles 0..t
constexpr uint64_t kGenValue = (1ull << 62) - 1;
constexpr int64_t kGenSpins = 1 << 22;          // polls of one look-back; about a second at most

__device__ __forceinline__ uint64_t gen_ld(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void gen_st(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive scan of one value per thread over the block; `ws` holds
// kGenWarps ints; ends with a barrier so `ws` may be reused.
__device__ __forceinline__ int gen_block_scan(int v, int *ws, int *total) {
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  int x = v;
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == kWarp - 1) ws[warp] = x;
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kGenWarps; ++w) {
    const int c = ws[w];
    if (w < warp) before += c;
    all += c;
  }
  *total = all;
  __syncthreads();
  return before + x - v;
}

// Prefix of the counts of the tiles before tile t in one status list, by one
// whole warp: publish the tile's own count, then read the words of the 32
// tiles before a window's end at once and add them up to the nearest
// inclusive word (tile -1 counts as inclusive 0); a window with a word not yet
// published is read again.  Only tiles claimed earlier -- by blocks that are
// running and publish before they wait -- are waited for, and every wait is
// bounded: a wait that gives up raises kErrTimeout.
__device__ __forceinline__ int64_t gen_lookback(uint64_t *status, int t, int64_t count,
                                                int *err) {
  const int lane = threadIdx.x & (kWarp - 1);
  uint64_t *word = status + t;
  if (t == 0) {
    if (lane == 0) gen_st(word, kGenInclusive | (uint64_t)count);
    return 0;
  }
  if (lane == 0) gen_st(word, kGenAggregate | (uint64_t)count);
  int64_t excl = 0;
  int j = t - 1;  // the window is tiles j - 31 .. j, lane k reading tile j - k
  int64_t spins = 0;
  for (;;) {
    const int idx = j - lane;
    const uint64_t w = idx >= 0 ? gen_ld(status + idx) : kGenInclusive;
    const unsigned incl = __ballot_sync(0xffffffffu, (w & ~kGenValue) == kGenInclusive);
    const unsigned unset = __ballot_sync(0xffffffffu, (w & ~kGenValue) == 0);
    const int stop = incl ? __ffs(incl) - 1 : kWarp - 1;  // the last lane that counts
    const unsigned counted = stop == kWarp - 1 ? 0xffffffffu : ((2u << stop) - 1u);
    if (unset & counted) {
      if (++spins > kGenSpins) {
        if (lane == 0) atomicOr(err, kErrTimeout);
        break;
      }
      continue;
    }
    int64_t v = lane <= stop ? (int64_t)(w & kGenValue) : 0;
#pragma unroll
    for (int o = kWarp / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    if (incl) break;
    j -= kWarp;
  }
  if (lane == 0) gen_st(word, kGenInclusive | (uint64_t)(excl + count));
  return excl;
}

// Classification of one input pair (a, b): kind 0 nothing, 1 the children
// pairs of a self pair, 2 a mutual interaction, 3 open member `o` against
// `other`; n_out new frontier pairs.
struct GenPair {
  int kind, k;
  int64_t a, b, o, other;
  bool open_a;
  int4 mt;
};

__device__ __forceinline__ GenPair classify_pair(const Ent &e, int2 ab, double theta2,
                                                 unsigned long long *flags) {
  GenPair g;
  g.kind = 0; g.k = 0; g.a = ab.x; g.b = ab.y; g.o = 0; g.other = 0; g.open_a = false;
  g.mt = make_int4(0, 0, 0, 0);
  if (g.a < 0 || g.b < 0) return g;
  const double4 ca = ent_com(e, g.a), cb = ent_com(e, g.b);
  if (ca.w == 0.0 || cb.w == 0.0) return g;
  if (g.a == g.b) {
    if (g.a < e.n) {  // a body with itself is dropped
      g.mt = e.meta[g.a];
      g.k = node_nchild(g.mt);
      g.kind = 1;
    }
    return g;
  }
  const double dx = ca.x - cb.x, dy = ca.y - cb.y, dz = ca.z - cb.z;
  const double dist2 = dx * dx + dy * dy + dz * dz;
  const double ra = ent_rmax(e, g.a), rb = ent_rmax(e, g.b);
  const double rs = ra + rb;
  if (rs * rs <= theta2 * dist2) {
    g.kind = 2;
    return g;
  }
  g.open_a = ra >= rb;
  g.o = g.open_a ? g.a : g.b;
  g.other = g.open_a ? g.b : g.a;
  if (g.o >= e.n) {
    atomicOr(flags, 4ull);  // cannot happen: bodies have rmax 0
    return g;
  }
  g.mt = e.meta[g.o];
  g.k = node_nchild(g.mt);
  g.kind = 3;
  return g;
}

// One generation of the dual traversal, as a deterministic compaction: block
// tiles of kGenTile input pairs (kGenItems consecutive pairs per thread) are
// claimed in order from `tile_ctr`; every thread classifies its pairs, the
// block scans the counts of new frontier pairs and of mutual pairs, and a
// chained scan over the tiles (separate status words for the two lists)
// places every pair's outputs right after those of the pairs before it.  So
// both lists come out in input order, whatever the schedule: the frontier of
// the next generation, and the mutual pairs appended after the `mut_base`
// written by earlier generations.  The block of the last tile writes the two
// new totals (the next generation's input count and the mutual count after
// this generation).
__global__ void __launch_bounds__(kGenThreads, kGenBlocksPerSm)
dual_gen_kernel(Ent e, const int2 *__restrict__ fin, const unsigned long long *__restrict__ nin,
                int64_t cap_in, int2 *__restrict__ fout, unsigned long long *nout, int64_t cap_out,
                int2 *__restrict__ mut, const unsigned long long *__restrict__ nmut_in,
                unsigned long long *nmut_out, int64_t cap_mut, double theta2,
                unsigned long long *flags, uint64_t *status_f, uint64_t *status_m,
                int *tile_ctr, int *err) {
  __shared__ int ws[kGenWarps];
  __shared__ int s_tile;
  __shared__ int64_t s_base[2];
  // after an overflow the count exceeds what was written: read only the buffer
  const int64_t n_in = bh_min64((int64_t)*nin, cap_in);
  const int64_t mut_base = (int64_t)*nmut_in;
  const int64_t ntiles = (n_in + kGenTile - 1) / kGenTile;
  if (ntiles == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { *nout = 0; *nmut_out = (unsigned long long)mut_base; }
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1);
    __syncthreads();
    const int t = s_tile;
    __syncthreads();
    if ((int64_t)t >= ntiles) break;  // uniform across the block
    const int64_t i0 = (int64_t)t * kGenTile + (int64_t)threadIdx.x * kGenItems;
    int2 ab[kGenItems];
#pragma unroll
    for (int q = 0; q < kGenItems; ++q) ab[q] = i0 + q < n_in ? fin[i0 + q] : make_int2(-1, -1);
    GenPair g[kGenItems];
#pragma unroll
    for (int q = 0; q < kGenItems; ++q) g[q] = classify_pair(e, ab[q], theta2, flags);
    // this thread's outputs, in input order
    int n_out = 0, n_mut = 0;
#pragma unroll
    for (int q = 0; q < kGenItems; ++q) {
      n_out += g[q].kind == 1 ? g[q].k * (g[q].k + 1) / 2 : (g[q].kind == 3 ? g[q].k : 0);
      n_mut += g[q].kind == 2 ? 1 : 0;
    }
    // one scan of both counts: a tile has at most kGenTile mutual pairs
    // (< 2^kGenMutBits) and kGenTile * 36 new pairs, so the packed sum fits
    int tot;
    const int off = gen_block_scan((n_out << kGenMutBits) | n_mut, ws, &tot);
    const int off_f = off >> kGenMutBits, off_m = off & kGenMutMask;
    const int tot_f = tot >> kGenMutBits, tot_m = tot & kGenMutMask;
    // the two chained scans, one warp each, at the same time
    const int warp = threadIdx.x / kWarp;
    if (warp == 0) {
      const int64_t ef = gen_lookback(status_f, t, tot_f, err);
      if (threadIdx.x == 0) {
        s_base[0] = ef;
        if ((int64_t)t == ntiles - 1) *nout = (unsigned long long)(ef + tot_f);
      }
    } else if (warp == 1) {
      const int64_t em = gen_lookback(status_m, t, tot_m, err);
      if (threadIdx.x == kWarp) {
        s_base[1] = mut_base + em;
        if ((int64_t)t == ntiles - 1) *nmut_out = (unsigned long long)(mut_base + em + tot_m);
      }
    }
    __syncthreads();
    int64_t fo = s_base[0] + off_f, mo = s_base[1] + off_m;
    if (n_out > 0 && fo + n_out > cap_out) atomicOr(flags, 1ull);
    if (n_mut > 0 && mo + n_mut > cap_mut) atomicOr(flags, 2ull);
    const bool fits_f = fo + n_out <= cap_out, fits_m = mo + n_mut <= cap_mut;
#pragma unroll
    for (int q = 0; q < kGenItems; ++q) {
      const GenPair &h = g[q];
      if (h.kind == 2) {
        if (fits_m) mut[mo] = make_int2((int)h.a, (int)h.b);
        ++mo;
      } else if (h.kind == 1) {
        if (fits_f) {
          int64_t w = fo;
          for (int p = 0; p < h.k; ++p) {
            const int64_t cp = node_child(e, h.a, h.mt, p);
            for (int r = p; r < h.k; ++r) fout[w++] = make_int2((int)cp, (int)node_child(e, h.a, h.mt, r));
          }
        }
        fo += h.k * (h.k + 1) / 2;
      } else if (h.kind == 3) {
        if (fits_f) {
          for (int r = 0; r < h.k; ++r) {
            const int64_t c = node_child(e, h.o, h.mt, r);
            fout[fo + r] = h.open_a ? make_int2((int)c, (int)h.other) : make_int2((int)h.other, (int)c);
          }
        }
        fo += h.k;
      }
    }
    __syncthreads();  // s_base is rewritten by the next tile
  }
}

// Both one-sided terms of every mutual pair: key = target, value = source.
// The mutual list is in a deterministic order, and the stable sort by target
// keeps that order among a target's terms.
__global__ void __launch_bounds__(256)
expand_kernel(const int2 *__restrict__ mut, int64_t np, uint2 *__restrict__ keys,
              int2 *__restrict__ vals, int32_t *cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = mut[i].x, b = mut[i].y;
    keys[i] = make_uint2((uint32_t)a, (uint32_t)b);  // terms 2i (a <- b) and 2i + 1 (b <- a)
    vals[i] = make_int2(b, a);
    // one add per distinct target in the warp (consecutive mutual pairs often
    // share a member): 13.9 -> 13.6-13.8 ms per call at 2^20
    const unsigned act = __activemask(), lt = (1u << (threadIdx.x & 31)) - 1u;
    const unsigned pa = __match_any_sync(act, a), pb = __match_any_sync(act, b);
    if ((pa & lt) == 0) atomicAdd(&cnt[a], __popc(pa));
    if ((pb & lt) == 0) atomicAdd(&cnt[b], __popc(pb));
  }
}

// One one-sided term (t <- s; cs the source's centre of mass and mass) added
// to f (3), h (6), tt (10); the octupole torque term (order 8) goes to tq (3)
// without its 0.5 / M_t factor, which the caller applies once to the
// target's sum.
template <int ORDER>
__device__ __forceinline__ void add_term(const Ent &e, int64_t t, const double4 &ct, bool tnode,
                                         int64_t s, double G, double eps2, double *f, double *h,
                                         double *tt, double *tq, const double4 cs) {
  const double Ms = cs.w, Mt = ct.w;
  const double dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
  const double r2 = dx * dx + dy * dy + dz * dz + eps2;
  if (r2 == 0.0) return;
  const double rinv = rsqrt(r2);
  const double rinv2 = rinv * rinv;
  const double rinv3 = rinv * rinv2;
  const double D1x = -G * dx * rinv3, D1y = -G * dy * rinv3, D1z = -G * dz * rinv3;
  if (ORDER < 4) {
    f[0] = f[0] + Ms * D1x; f[1] = f[1] + Ms * D1y; f[2] = f[2] + Ms * D1z;
    return;
  }
  const double rinv5 = rinv3 * rinv2, rinv7 = rinv5 * rinv2;
  double D2[6], D3[10];
  D2[0] = G * (3.0 * dx * dx * rinv5 - rinv3);
  D2[1] = G * (3.0 * dy * dy * rinv5 - rinv3);
  D2[2] = G * (3.0 * dz * dz * rinv5 - rinv3);
  D2[3] = G * 3.0 * dx * dy * rinv5;
  D2[4] = G * 3.0 * dx * dz * rinv5;
  D2[5] = G * 3.0 * dy * dz * rinv5;
  D3[0] = G * (-15.0 * dx * dx * dx * rinv7 + 9.0 * dx * rinv5);
  D3[1] = G * (-15.0 * dx * dx * dy * rinv7 + 3.0 * dy * rinv5);
  D3[2] = G * (-15.0 * dx * dx * dz * rinv7 + 3.0 * dz * rinv5);
  D3[3] = G * (-15.0 * dx * dy * dy * rinv7 + 3.0 * dx * rinv5);
  D3[4] = G * (-15.0 * dx * dy * dz * rinv7);
  D3[5] = G * (-15.0 * dx * dz * dz * rinv7 + 3.0 * dx * rinv5);
  D3[6] = G * (-15.0 * dy * dy * dy * rinv7 + 9.0 * dy * rinv5);
  D3[7] = G * (-15.0 * dy * dy * dz * rinv7 + 3.0 * dz * rinv5);
  D3[8] = G * (-15.0 * dy * dz * dz * rinv7 + 3.0 * dy * rinv5);
  D3[9] = G * (-15.0 * dz * dz * dz * rinv7 + 9.0 * dz * rinv5);
  double cq[3] = {0.0, 0.0, 0.0};
  if (s < e.n) {  // a node's specific quadrupole (divided once per node); a body has none
    const double *q = e.squad + 6 * s;
    const double Q0 = q[0], Q1 = q[1], Q2 = q[2], Q3 = q[3], Q4 = q[4], Q5 = q[5];
    cq[0] = Q0 * D3[0] + 2.0 * Q3 * D3[1] + 2.0 * Q4 * D3[2] + Q1 * D3[3] + 2.0 * Q5 * D3[4] +
            Q2 * D3[5];
    cq[1] = Q0 * D3[1] + 2.0 * Q3 * D3[3] + 2.0 * Q4 * D3[4] + Q1 * D3[6] + 2.0 * Q5 * D3[7] +
            Q2 * D3[8];
    cq[2] = Q0 * D3[2] + 2.0 * Q3 * D3[4] + 2.0 * Q4 * D3[5] + Q1 * D3[7] + 2.0 * Q5 * D3[8] +
            Q2 * D3[9];
  }
  f[0] = f[0] + Ms * (D1x + 0.5 * cq[0]);
  f[1] = f[1] + Ms * (D1y + 0.5 * cq[1]);
  f[2] = f[2] + Ms * (D1z + 0.5 * cq[2]);
#pragma unroll
  for (int q = 0; q < 6; ++q) h[q] = h[q] + Ms * D2[q];
#pragma unroll
  for (int q = 0; q < 10; ++q) tt[q] = tt[q] + Ms * D3[q];
  if (ORDER >= 8 && (tnode || s < e.n)) {
    // octupole torque term (:1530-1557); a body's octupole is zero.
    // C_jkl = Ms O_t - Mt O_s, components 0 xxx 1 xyy 2 xzz 3 yxx 4 yyy 5 yzz
    // 6 zxx 7 zyy 8 zzz 9 xyz (the index map of :233-241)
    const double *ot = tnode ? e.oct + 14 * t : nullptr;
    const double *os = s < e.n ? e.oct + 14 * s : nullptr;
    double C[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) C[q] = (ot ? Ms * ot[q] : 0.0) - (os ? Mt * os[q] : 0.0);
    const double cx = C[0] + C[1] + C[2], cy = C[3] + C[4] + C[5], cz = C[6] + C[7] + C[8];
    const double crx = C[0] * dx * dx + C[1] * dy * dy + C[2] * dz * dz +
                       2.0 * (C[3] * dx * dy + C[6] * dx * dz + C[9] * dy * dz);
    const double cry = C[3] * dx * dx + C[4] * dy * dy + C[5] * dz * dz +
                       2.0 * (C[1] * dx * dy + C[9] * dx * dz + C[7] * dy * dz);
    const double crz = C[6] * dx * dx + C[7] * dy * dy + C[8] * dz * dz +
                       2.0 * (C[9] * dx * dy + C[2] * dx * dz + C[5] * dy * dz);
    const double a3 = 3.0 * G * rinv5, a15 = 15.0 * G * rinv7;
    tq[0] = tq[0] + (a3 * cx - a15 * crx);
    tq[1] = tq[1] + (a3 * cy - a15 * cry);
    tq[2] = tq[2] + (a3 * cz - a15 * crz);
  }
}

// Sum of the one-sided terms of every target, kEvalLanes lanes per target
// (two targets per warp): lane l of a target's group adds terms l, l + 16, ...
// of the target's list (in the mutual list's deterministic order), then the
// group's sums are combined by a fixed butterfly, so the result depends only
// on the target's own list.  A target has about a hundred terms; at 2^20 the
// quadrupole call took 14.6 / 14.2 / 14.0 / 14.7 ms with 4 / 8 / 16 / 32 lanes
// per target (the octupole 17.1 ms with 8, 16.8 with 16, 17.7 with 32): fewer
// lanes leave each lane a longer chain of loads, more make the butterfly over
// the 19-22 sums a larger share.
constexpr int kEvalLanes = 16;

template <int ORDER>
__global__ void __launch_bounds__(128)
eval_kernel(Ent e, int64_t ne, const int32_t *__restrict__ beg, const int32_t *__restrict__ src,
            double G, double eps2, double *__restrict__ F, double *__restrict__ H,
            double *__restrict__ T) {
  constexpr int NV = ORDER >= 8 ? 22 : (ORDER >= 4 ? 19 : 3);  // f, h, tt[, torque]
  constexpr int kPerWarp = kWarp / kEvalLanes;
  const int lane = threadIdx.x & (kWarp - 1);
  const int sub = lane / kEvalLanes, sl = lane % kEvalLanes;
  const int64_t warp_id = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) / kWarp;
  for (int64_t t0 = warp_id * kPerWarp; t0 < ne; t0 += wstride * kPerWarp) {
    const int64_t t = t0 + sub;
    double v[22];
#pragma unroll
    for (int q = 0; q < 22; ++q) v[q] = 0.0;
    if (t < ne) {
      const int kb = beg[t], ke = beg[t + 1];
      if (kb < ke) {
        const double4 ct = ent_com(e, t);
        const bool tnode = t < e.n;
        if (ORDER < 8) {
          // the next term's source and centre of mass load while this one
          // is computed (the octupole term needs those registers itself)
          int k = kb + sl;
          int64_t sn = k < ke ? (int64_t)src[k] : 0;
          double4 cn = k < ke ? ent_com(e, sn) : make_double4(0.0, 0.0, 0.0, 0.0);
          while (k < ke) {
            const int64_t sc = sn;
            const double4 cc = cn;
            k += kEvalLanes;
            if (k < ke) { sn = (int64_t)src[k]; cn = ent_com(e, sn); }
            add_term<ORDER>(e, t, ct, tnode, sc, G, eps2, v, v + 3, v + 9, v + 19, cc);
          }
        } else {
          for (int k = kb + sl; k < ke; k += kEvalLanes) {
            const int64_t sc = (int64_t)src[k];
            add_term<ORDER>(e, t, ct, tnode, sc, G, eps2, v, v + 3, v + 9, v + 19, ent_com(e, sc));
          }
        }
      }
    }
    // every lane of the warp takes part (lanes past ne hold zeros)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
      for (int o = kEvalLanes / 2; o > 0; o >>= 1) v[q] = v[q] + __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    if (sl == 0 && t < ne) {
      if (ORDER >= 8 && (v[19] != 0.0 || v[20] != 0.0 || v[21] != 0.0)) {
        const double Mt = ent_com(e, t).w;  // > 0: terms with a massless member are dropped
#pragma unroll
        for (int q = 0; q < 3; ++q) v[q] = v[q] + 0.5 * v[19 + q] / Mt;
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) F[3 * t + q] = v[q];
      if (ORDER >= 4) {
#pragma unroll
        for (int q = 0; q < 6; ++q) H[6 * t + q] = v[3 + q];
#pragma unroll
        for (int q = 0; q < 10; ++q) T[10 * t + q] = v[9 + q];
      }
    }
  }
}

// The node whose child a body is (a lone-particle child, or a body of a
// node of identical keys), for every sorted position.
__global__ void __launch_bounds__(256)
body_parent_kernel(const Scalars *__restrict__ scr, Ent e, int32_t *__restrict__ bp) {
  const int M = scr->n_compact;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
    const int4 mt = e.meta[j];
    if (mt.w == 0) {
      for (int c = 0; c < mt.y; ++c) bp[mt.x + c] = j;
    } else {
      for (int c = 0; c < mt.w; ++c) {
        const int32_t ch = e.child[8 * (int64_t)j + c];
        if (ch < 0) bp[~ch] = j;
      }
    }
  }
}

// The downward pass (dehnen_forces, octree_default.f90:1560-1673) and the
// output in one launch, one thread per body.  The pass adds to every child
// the parent's field translated to the child's centre of mass (F + H d +
// d.T.d / 2, H + T d, T), so a body ends with the sum of every ancestor's own
// expansion translated to it; the translation of a cubic-potential expansion
// is exact, so the body sums its ancestors' translations directly, from the
// root down, instead of waiting for the levels above it.  A massless body
// receives nothing (the pass skips massless children).  The force is m times
// the field; forces go out in the original order, one (n_s, 3) Fortran block
// per system.  A parent chain longer than the deepest tree raises kErrIndex.
template <int ORDER>
__global__ void __launch_bounds__(128)
down_bodies_kernel(int64_t n, Ent e, const int32_t *__restrict__ bp,
                   const int32_t *__restrict__ parent, const double *__restrict__ F,
                   const double *__restrict__ H, const double *__restrict__ T,
                   const int32_t *__restrict__ perm, const int32_t *__restrict__ sys_of,
                   const SysScalars *__restrict__ ss, int out_kind, double *__restrict__ out,
                   int *err) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const double4 cb = e.spos[p];
    const double *fl = F + 3 * (n + p);
    double fx = fl[0], fy = fl[1], fz = fl[2];
    const SysScalars &s = ss[sys_of[p]];
    if (cb.w != 0.0 && s.root >= 0) {
      int chain[kNumLevels + 2];
      int depth = 0;
      bool ok = true;
      for (int j = bp[p]; j >= 0; j = parent[j]) {
        if (depth >= kNumLevels + 2) { ok = false; break; }
        chain[depth++] = j;
      }
      if (!ok) atomicOr(err, kErrIndex);
      for (int k = ok ? depth - 1 : -1; k >= 0; --k) {
        const int j = chain[k];
        fx += F[3 * (int64_t)j]; fy += F[3 * (int64_t)j + 1]; fz += F[3 * (int64_t)j + 2];
        if (ORDER >= 4) {
          const double4 cj = e.com[j];
          const double dx = cb.x - cj.x, dy = cb.y - cj.y, dz = cb.z - cj.z;
          const double *h = H + 6 * (int64_t)j, *t = T + 10 * (int64_t)j;
          const double hxx = h[0], hyy = h[1], hzz = h[2], hxy = h[3], hxz = h[4], hyz = h[5];
          const double txxx = t[0], txxy = t[1], txxz = t[2], txyy = t[3], txyz = t[4],
                       txzz = t[5], tyyy = t[6], tyyz = t[7], tyzz = t[8], tzzz = t[9];
          fx += hxx * dx + hxy * dy + hxz * dz + txxy * dx * dy + txxz * dx * dz + txyz * dy * dz +
                0.5 * (txxx * dx * dx + txyy * dy * dy + txzz * dz * dz);
          fy += hxy * dx + hyy * dy + hyz * dz + txyy * dx * dy + txyz * dx * dz + tyyz * dy * dz +
                0.5 * (txxy * dx * dx + tyyy * dy * dy + tyzz * dz * dz);
          fz += hxz * dx + hyz * dy + hzz * dz + txyz * dx * dy + txzz * dx * dz + tyzz * dy * dz +
                0.5 * (txxz * dx * dx + tyyz * dy * dy + tzzz * dz * dz);
        }
      }
    }
    const double sc = out_kind == 0 ? cb.w : 1.0;
    const int64_t o = perm[p] - s.off;
    double *base = out + 3 * s.off;
    base[o] = sc * fx;
    base[s.n + o] = sc * fy;
    base[2 * s.n + o] = sc * fz;
  }
}

template <typename T>
cudaError_t grow(T *&p, int64_t &cap, int64_t need) {
  if (p && cap >= need) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const cudaError_t e = cudaMalloc((void **)&p, (size_t)need * sizeof(T));
  if (e == cudaSuccess) cap = need;
  return e;
}

int bits_for64(int64_t v) {
  int b = 1;
  while (((int64_t)1 << b) <= v) ++b;
  return b;
}

}  // namespace

void free_dehnen(DehnenBuffers &d) {
  void *ptrs[] = {d.rmax, d.F, d.H, d.T, d.squad, d.front, d.mut, d.keys, d.vals, d.cnt, d.beg,
                  d.hist, d.scan_tmp, d.counters, d.gen_status, d.gen_tiles};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  d = DehnenBuffers();
}

int run_dehnen(int64_t n, const WalkParams &p, Buffers &b, DehnenBuffers &d, double *out,
               cudaStream_t s) {
  const int64_t ne = 2 * n;
  if (grow(d.rmax, d.rmax_cap, n) != cudaSuccess) return 1;
  if (grow(d.F, d.F_cap, 3 * ne) != cudaSuccess) return 1;
  if (p.order >= 4 && grow(d.H, d.H_cap, 6 * ne) != cudaSuccess) return 1;
  if (p.order >= 4 && grow(d.T, d.T_cap, 10 * ne) != cudaSuccess) return 1;
  if (p.order >= 4 && grow(d.squad, d.squad_cap, 6 * n) != cudaSuccess) return 1;
  if (grow(d.cnt, d.cnt_cap, ne + 1) != cudaSuccess) return 1;
  if (grow(d.beg, d.beg_cap, ne + 1) != cudaSuccess) return 1;
  if (grow(d.scan_tmp, d.scan_tmp_cap, scan_tmp_entries(ne + 1)) != cudaSuccess) return 1;
  if (grow(d.counters, d.counters_cap, 8) != cudaSuccess) return 1;
  if (d.front_cap < 2 * 16 * n) d.want_front = 16 * n;  // per generation, either buffer
  if (d.mut_cap < 32 * n) d.want_mut = 32 * n;

  Ent e;
  e.meta = b.cn_meta; e.child = b.cn_child; e.com = b.cn_com; e.spos = b.spos;
  e.quad = b.cn_quad; e.oct = b.cn_oct; e.rmax = d.rmax; e.n = n;
  e.squad = p.order >= 4 ? d.squad : nullptr;
  const int lgrid = grid_for(n / 2 + 1, 256, 148 * 8);
  cudaMemsetAsync(d.cnt, 0, (ne + 1) * sizeof(int32_t), s);  // arrival counters (M < ne)
  rmax_fused_kernel<<<lgrid, 256, 0, s>>>(b.sc, e, b.cn_parent, d.rmax, d.cnt, &b.sc->err);
  if (p.order >= 4)
    spec_quad_kernel<<<lgrid, 256, 0, s>>>(b.sc, b.cn_com, b.cn_quad, d.squad);

  // counters: [0], [1] frontier sizes and [2], [3] mutual totals, each
  // alternating between generations; [4] overflow flags
  unsigned long long *cnt = d.counters;
  unsigned long long h[5] = {0, 0, 0, 0, 0};
  if (b.nsys > 16 * n) return 4;
  for (int attempt = 0; attempt < 8; ++attempt) {
    if (grow(d.front, d.front_cap, 2 * d.want_front) != cudaSuccess) return 1;
    if (grow(d.mut, d.mut_cap, d.want_mut) != cudaSuccess) return 1;
    int2 *f0 = d.front, *f1 = d.front + d.front_cap / 2;
    const int64_t fcap = d.front_cap / 2;
    const int64_t max_tiles = fcap / kGenTile + 1;  // tiles of one generation's input
    if (grow(d.gen_status, d.gen_status_cap, (int64_t)kGenerations * 2 * max_tiles) != cudaSuccess)
      return 1;
    if (grow(d.gen_tiles, d.gen_tiles_cap, (int64_t)kGenerations) != cudaSuccess) return 1;
    cudaMemsetAsync(d.counters, 0, 8 * sizeof(unsigned long long), s);
    cudaMemsetAsync(d.gen_status, 0, (size_t)kGenerations * 2 * max_tiles * sizeof(uint64_t), s);
    cudaMemsetAsync(d.gen_tiles, 0, kGenerations * sizeof(int32_t), s);
    roots_frontier_kernel<<<(b.nsys + 127) / 128, 128, 0, s>>>(b.ss, b.nsys, f0, cnt);
    for (int g = 0; g < kGenerations; ++g) {
      int2 *fi = (g & 1) ? f1 : f0, *fo = (g & 1) ? f0 : f1;
      uint64_t *st = d.gen_status + (int64_t)g * 2 * max_tiles;
      dual_gen_kernel<<<148 * 8, kGenThreads, 0, s>>>(
          e, fi, cnt + (g & 1), fcap, fo, cnt + ((g + 1) & 1), fcap, d.mut, cnt + 2 + (g & 1),
          cnt + 2 + ((g + 1) & 1), d.mut_cap, p.theta2, cnt + 4, st, st + max_tiles,
          d.gen_tiles + g, &b.sc->err);
    }
    if (cudaMemcpyAsync(h, d.counters, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return 2;
    if (h[4] & 4) return 3;
    const bool more_front = (h[4] & 1) != 0, more_mut = (h[4] & 2) != 0;
    if (!more_front && !more_mut) {
      if (h[kGenerations & 1] != 0) return 3;  // the traversal did not close
      break;
    }
    if (attempt == 7) return 4;
    if (more_front) d.want_front *= 2;
    if (more_mut) d.want_mut *= 2;
    if (d.want_mut > ((int64_t)1 << 30) || d.want_front > ((int64_t)1 << 30)) return 4;
  }
  const int64_t np = (int64_t)h[2 + (kGenerations & 1)];
  const int64_t nh = 2 * np;
  if (grow(d.keys, d.keys_cap, 2 * (nh > 0 ? nh : 1)) != cudaSuccess) return 1;
  if (grow(d.vals, d.vals_cap, 2 * (nh > 0 ? nh : 1)) != cudaSuccess) return 1;
  if (grow(d.hist, d.hist_cap, radix_hist_entries(nh > 0 ? nh : 1)) != cudaSuccess) return 1;
  cudaMemsetAsync(d.cnt, 0, (ne + 1) * sizeof(int32_t), s);
  const int32_t *sources = d.vals;  // the terms' sources in target order
  if (np > 0) {
    const int g = grid_for(np, 256, 148 * 16);
    expand_kernel<<<g, 256, 0, s>>>(d.mut, np, reinterpret_cast<uint2 *>(d.keys),
                                    reinterpret_cast<int2 *>(d.vals), d.cnt);
    // stable by target: a target's terms keep the mutual list's order
    // the digit counts come from the terms per target that expand counted
    if (radix_sort_values32(d.keys, d.vals, d.keys + nh, d.vals + nh, nh, bits_for64(ne), d.hist,
                            &b.sc->err, s, d.cnt, ne) == 1)
      sources = d.vals + nh;
  }
  exclusive_scan(d.cnt, d.beg, ne + 1, nullptr, nullptr, d.scan_tmp, &b.sc->err, s);
  const int egrid = grid_for(ne * kEvalLanes, 128, 148 * 32);
  const double G = p.G, eps2 = p.eps2;
  if (p.order >= 8)
    eval_kernel<8><<<egrid, 128, 0, s>>>(e, ne, d.beg, sources, G, eps2, d.F, d.H, d.T);
  else if (p.order >= 4)
    eval_kernel<4><<<egrid, 128, 0, s>>>(e, ne, d.beg, sources, G, eps2, d.F, d.H, d.T);
  else
    eval_kernel<1><<<egrid, 128, 0, s>>>(e, ne, d.beg, sources, G, eps2, d.F, d.H, d.T);
  // downward pass and output: every body sums its ancestors' translated
  // expansions (cnt is free after the scan: it holds each body's parent node)
  int32_t *bp = d.cnt;
  body_parent_kernel<<<lgrid, 256, 0, s>>>(b.sc, e, bp);
  const int bgrid = grid_for(n, 128, 148 * 16);
  if (p.order >= 4)
    down_bodies_kernel<4><<<bgrid, 128, 0, s>>>(n, e, bp, b.cn_parent, d.F, d.H, d.T, b.v0,
                                                 b.sys_of, b.ss, p.out_kind, out, &b.sc->err);
  else
    down_bodies_kernel<1><<<bgrid, 128, 0, s>>>(n, e, bp, b.cn_parent, d.F, d.H, d.T, b.v0,
                                                 b.sys_of, b.ss, p.out_kind, out, &b.sc->err);
  d.pairs = np;
  return 0;
}

}  // namespace bh
