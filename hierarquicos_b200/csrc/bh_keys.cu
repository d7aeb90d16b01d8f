// Bounding box, centre of mass, normalisation and 63-bit Morton keys, for
// every system of a batch in one launch per step.
//
// Follows fortran/morton/morton_octree.f90:359-395 (generate_nodes steps 1-5)
// and :184-213 (morton_key).  All arithmetic that feeds a key uses explicitly
// rounded intrinsics so that no multiply-add is contracted.
//
// Keys and the centre of mass.  The reference sums the centre of mass c
// sequentially (:364-370) and normalises x_n = fl(fl(fl(q - c)/ssa) + 0.5) -
// vcen, vcen = 0.5 fl(vmin + vmax) with vmin/vmax the normalised extremes
// (:373-384).  In exact arithmetic c cancels: x_n = (q - (qmin+qmax)/2)/ssa +
// 1/2.  So two evaluations with different roundings of c differ only by their
// rounding errors, |x_n(c1) - x_n(c2)| <= 2 u (6.02 V + 1.5) with u = 2^-53 and
// V = max |v| <= 0.84 for non-negative masses (each of the five rounded
// operations contributes at most u times its operand).  A body whose
// 2^21 x_n lies farther than that (times a safety factor 1.5) from an integer
// on every axis therefore gets the reference's key whatever c is.  The keys
// kernel computes c with a deterministic parallel sum, checks that margin for
// every body and raises `key_ambiguous` for its system if any body is inside
// it; only then does the host run the reference's sequential sum
// (seq_com_kernel) for that system and compare the keys (verify_keys_kernel),
// rebuilding if one differs.
#include <math.h>

#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int kRedThreads = 256;

// 21-bit coordinate -> 63-bit interleave, x in the most significant slot of
// each octal digit (morton_octree.f90:205-212).
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ int64_t quantise(double xn, int L) {
  // FLOOR(x * 2^L) clamped to 2^L - 1; x * 2^L is exact.
  const double scale = (double)(1ll << L);
  double f = floor(__dmul_rn(xn, scale));
  int64_t i = (int64_t)f;
  int64_t top = (1ll << L) - 1;
  if (i > top) i = top;
  if (i < 0) i = 0;
  return i;
}

// fraction of the finest cell: ambiguous when within `margin` of an edge
__device__ __forceinline__ bool near_edge(double xn, double margin) {
  const double f = __dmul_rn(xn, 2097152.0);  // exact
  const double r = f - floor(f);               // exact
  return r < margin || r > 1.0 - margin;
}

__device__ __forceinline__ uint64_t key_of(double x, double y, double z, const double com[3],
                                           double ssa, const double vcen[3], int *bad,
                                           double margin = -1.0, int *amb = nullptr) {
  // positions_norm = (q - qcm) / ssa, then + 0.5 - ssi (morton_octree.f90:373-384)
  double vx = __ddiv_rn(__dsub_rn(x, com[0]), ssa);
  double vy = __ddiv_rn(__dsub_rn(y, com[1]), ssa);
  double vz = __ddiv_rn(__dsub_rn(z, com[2]), ssa);
  double xn = __dsub_rn(__dadd_rn(vx, 0.5), vcen[0]);
  double yn = __dsub_rn(__dadd_rn(vy, 0.5), vcen[1]);
  double zn = __dsub_rn(__dadd_rn(vz, 0.5), vcen[2]);
  if (!(xn >= 0.0 && xn < 1.0 && yn >= 0.0 && yn < 1.0 && zn >= 0.0 && zn < 1.0)) *bad = 1;
  if (amb && (near_edge(xn, margin) || near_edge(yn, margin) || near_edge(zn, margin))) *amb = 1;
  uint64_t ix = (uint64_t)quantise(xn, kMaxDepth), iy = (uint64_t)quantise(yn, kMaxDepth),
           iz = (uint64_t)quantise(zn, kMaxDepth);
  return (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
}

// Partial reductions over one work item (a slice of one system): min/max per
// axis, sum m, sum m x, sum m y, sum m z.  Fixed slices and a fixed tree
// order: the result is deterministic.
__global__ void __launch_bounds__(kRedThreads)
reduce_partials(const double *__restrict__ m, const double *__restrict__ x,
                const double *__restrict__ y, const double *__restrict__ z,
                const RedItem *__restrict__ items, int com_mode, double *__restrict__ partials) {
  __shared__ double s[10][kRedThreads];
  const RedItem it = items[blockIdx.x];
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  double sm = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  for (int64_t p = it.start + threadIdx.x; p < it.end; p += kRedThreads) {
    double a = x[p], b = y[p], c = z[p], w = m[p];
    mn[0] = fmin(mn[0], a); mx[0] = fmax(mx[0], a);
    mn[1] = fmin(mn[1], b); mx[1] = fmax(mx[1], b);
    mn[2] = fmin(mn[2], c); mx[2] = fmax(mx[2], c);
    sm = __dadd_rn(sm, w);
    if (com_mode) {
      sx = __fma_rn(w, a, sx); sy = __fma_rn(w, b, sy); sz = __fma_rn(w, c, sz);
    } else {
      sx = __dadd_rn(sx, __dmul_rn(w, a));
      sy = __dadd_rn(sy, __dmul_rn(w, b));
      sz = __dadd_rn(sz, __dmul_rn(w, c));
    }
  }
  int t = threadIdx.x;
  s[0][t] = mn[0]; s[1][t] = mn[1]; s[2][t] = mn[2];
  s[3][t] = mx[0]; s[4][t] = mx[1]; s[5][t] = mx[2];
  s[6][t] = sm; s[7][t] = sx; s[8][t] = sy; s[9][t] = sz;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (t < w) {
      for (int k = 0; k < 3; ++k) s[k][t] = fmin(s[k][t], s[k][t + w]);
      for (int k = 3; k < 6; ++k) s[k][t] = fmax(s[k][t], s[k][t + w]);
      for (int k = 6; k < 10; ++k) s[k][t] = __dadd_rn(s[k][t], s[k][t + w]);
    }
    __syncthreads();
  }
  if (t < 10) partials[blockIdx.x * 10 + t] = s[t][0];
}

__device__ void finalize_norm(SysScalars *ss, const double com[3], double vcen[3]) {
  // normalised box centre: min/max of fl(fl(q - com) / ssa) are the images of
  // the coordinate min/max because rounding is monotonic.
  for (int k = 0; k < 3; ++k) {
    double vmin = __ddiv_rn(__dsub_rn(ss->bmin[k], com[k]), ss->ssa);
    double vmax = __ddiv_rn(__dsub_rn(ss->bmax[k], com[k]), ss->ssa);
    vcen[k] = __dmul_rn(0.5, __dadd_rn(vmin, vmax));
  }
}

// One block per system: one warp per reduced quantity over the system's work
// items (items are ordered by system), fixed lane strides and a fixed
// butterfly (deterministic).  Thread 0 then derives ssa, the centre of mass,
// the normalised box centre and the key margin.
__global__ void __launch_bounds__(320)
finalize_kernel(const double *__restrict__ partials, const RedItem *__restrict__ items,
                int n_items, double amp, int L, SysScalars *__restrict__ sys, Scalars *sc) {
  __shared__ double red[10];
  __shared__ int range[2];
  const int s = blockIdx.x;
  if (threadIdx.x == 0) {
    int a = 0, b = n_items;
    while (a < b) { int mid = (a + b) / 2; if (items[mid].sys < s) a = mid + 1; else b = mid; }
    range[0] = a;
    b = n_items;
    while (a < b) { int mid = (a + b) / 2; if (items[mid].sys <= s) a = mid + 1; else b = mid; }
    range[1] = a;
  }
  __syncthreads();
  const int w = threadIdx.x / kWarp, lane = threadIdx.x & (kWarp - 1);
  if (w < 10) {
    double acc = w < 3 ? INFINITY : (w < 6 ? -INFINITY : 0.0);
    for (int b = range[0] + lane; b < range[1]; b += kWarp) {
      const double v = partials[10 * b + w];
      acc = w < 3 ? fmin(acc, v) : (w < 6 ? fmax(acc, v) : __dadd_rn(acc, v));
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double v = __shfl_xor_sync(0xffffffffu, acc, o);
      acc = w < 3 ? fmin(acc, v) : (w < 6 ? fmax(acc, v) : __dadd_rn(acc, v));
    }
    if (lane == 0) red[w] = acc;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  SysScalars *ss = sys + s;
  double mn[3] = {red[0], red[1], red[2]}, mx[3] = {red[3], red[4], red[5]};
  const double sm = red[6], sx = red[7], sy = red[8], sz = red[9];
  for (int k = 0; k < 3; ++k) { ss->bmin[k] = mn[k]; ss->bmax[k] = mx[k]; }
  double ext = __dsub_rn(mx[0], mn[0]);
  double ey = __dsub_rn(mx[1], mn[1]), ez = __dsub_rn(mx[2], mn[2]);
  if (ey > ext) ext = ey;
  if (ez > ext) ext = ez;
  ss->ssa = __dmul_rn(amp, ext);
  ss->mass = sm;
  ss->com[0] = __ddiv_rn(sx, sm);
  ss->com[1] = __ddiv_rn(sy, sm);
  ss->com[2] = __ddiv_rn(sz, sm);
  ss->err = 0;
  ss->key_mismatch = 0;
  ss->key_ambiguous = 0;
  // a lone body has no extent; it feels no force and gets no tree
  bool ok = isfinite(sm) && sm > 0.0 && isfinite(ss->com[0]) && isfinite(ss->com[1]) &&
            isfinite(ss->com[2]) && isfinite(ext) && (ext > 0.0 || ss->n < 2);
  if (!ok) {
    ss->err |= kErrNonFinite;
    atomicOr(&sc->err, kErrNonFinite);
  }
  if (!(ext > 0.0)) ss->ssa = 1.0;  // lone body: any positive side
  finalize_norm(ss, ss->com, ss->vcen);
  // V = largest |normalised coordinate| before the shift
  double V = 0.0;
  for (int k = 0; k < 3; ++k) {
    V = fmax(V, fabs((ss->bmin[k] - ss->com[k]) / ss->ssa));
    V = fmax(V, fabs((ss->bmax[k] - ss->com[k]) / ss->ssa));
  }
  // 2 evaluations x (6.02 V + 1.5) u, x 1.5 safety, in units of 2^-21
  ss->key_margin = 3.0 * (6.1 * V + 1.6) * ldexp(1.0, -32);
  if (s == 0) {
    sc->L = L;
    sc->nsys = gridDim.x;
  }
}

__global__ void __launch_bounds__(256)
keys_kernel(const double *__restrict__ x, const double *__restrict__ y,
            const double *__restrict__ z, int64_t n, int L, const int32_t *__restrict__ sys_of,
            SysScalars *sys, Scalars *sc, uint64_t *__restrict__ keys,
            int32_t *__restrict__ vals) {
  int bad = 0, amb_any = 0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    SysScalars *ss = sys + sys_of[p];
    const double com[3] = {ss->com[0], ss->com[1], ss->com[2]};
    const double vcen[3] = {ss->vcen[0], ss->vcen[1], ss->vcen[2]};
    int amb = 0;
    uint64_t k = key_of(x[p], y[p], z[p], com, ss->ssa, vcen, &bad, ss->key_margin, &amb);
    keys[p] = (L == kMaxDepth || L == 0) ? k : (k >> (3 * (kMaxDepth - L)));
    vals[p] = (int32_t)p;
    if (amb && ss->n > 1) {
      ss->key_ambiguous = 1;  // every writer stores the same value
      amb_any = 1;
    }
  }
  if (bad) atomicOr(&sc->err, kErrNonFinite);
  if (amb_any) atomicOr(&sc->key_ambiguous, 1);
}

// Sequential centre of mass in the reference's order (morton_octree.f90:364-370):
// qcm = qcm + m_p q_p, mass = mass + m_p for p = 1..N, one dependent chain per
// component.  One block per system (systems without ambiguous keys return
// unless `all` is set).  Warps 0..3 each fold one chain (x, y, z, mass) over
// the current shared-memory tile, all lanes of a warp running the same chain on
// broadcast reads, while warps 4..7 stage the next tile.
constexpr int kSeqTile = 1024;
constexpr int kSeqThreads = 256;

__global__ void __launch_bounds__(kSeqThreads)
seq_com_kernel(const double *__restrict__ m, const double *__restrict__ x,
               const double *__restrict__ y, const double *__restrict__ z, int com_mode,
               int all, SysScalars *sys) {
  extern __shared__ double4 tile[];  // 2 x kSeqTile entries: (m, x, y, z)
  __shared__ double res[4];
  SysScalars *ss = sys + blockIdx.x;
  if (!all && !ss->key_ambiguous) return;  // uniform across the block
  const int64_t off = ss->off, n = ss->n;
  const int warp = threadIdx.x / kWarp;
  const int64_t ntiles = (n + kSeqTile - 1) / kSeqTile;
  double acc = 0.0;
  auto stage = [&](int64_t t, int buf) {
    if (warp < 4) return;
    for (int i = threadIdx.x - 4 * kWarp; i < kSeqTile; i += kSeqThreads - 4 * kWarp) {
      int64_t p = t * kSeqTile + i;
      double4 v = make_double4(0.0, 0.0, 0.0, 0.0);
      if (p < n) v = make_double4(m[off + p], x[off + p], y[off + p], z[off + p]);
      tile[buf * kSeqTile + i] = v;
    }
  };
  stage(0, 0);
  __syncthreads();
  for (int64_t t = 0; t < ntiles; ++t) {
    const int buf = (int)(t & 1);
    if (t + 1 < ntiles) stage(t + 1, buf ^ 1);
    if (warp < 4) {
      const int cnt = (int)bh_min64(kSeqTile, n - t * kSeqTile);
      const double *q = reinterpret_cast<const double *>(tile + buf * kSeqTile);
      if (warp == 3) {
#pragma unroll 16
        for (int i = 0; i < cnt; ++i) acc = __dadd_rn(acc, q[4 * i]);
      } else if (com_mode) {
#pragma unroll 16
        for (int i = 0; i < cnt; ++i) acc = __fma_rn(q[4 * i], q[4 * i + 1 + warp], acc);
      } else {
#pragma unroll 16
        for (int i = 0; i < cnt; ++i) acc = __dadd_rn(acc, __dmul_rn(q[4 * i], q[4 * i + 1 + warp]));
      }
    }
    __syncthreads();
  }
  if (warp < 4 && (threadIdx.x & (kWarp - 1)) == 0) res[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    ss->mass_seq = res[3];
    ss->com_seq[0] = __ddiv_rn(res[0], res[3]);
    ss->com_seq[1] = __ddiv_rn(res[1], res[3]);
    ss->com_seq[2] = __ddiv_rn(res[2], res[3]);
  }
}

// Recomputes every key of a checked system with its sequential-order centre
// of mass and compares it with the key the tree was built from (sorted
// position i holds original body perm[i]).
__global__ void __launch_bounds__(256)
verify_keys_kernel(const double *__restrict__ x, const double *__restrict__ y,
                   const double *__restrict__ z, int64_t n, int all,
                   const int32_t *__restrict__ sys_of, SysScalars *sys, Scalars *sc,
                   const uint64_t *__restrict__ skeys, const int32_t *__restrict__ perm) {
  const int L = sc->L;
  int bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    SysScalars *ss = sys + sys_of[i];
    if (!all && !ss->key_ambiguous) continue;
    if (ss->com_seq[0] == ss->com[0] && ss->com_seq[1] == ss->com[1] &&
        ss->com_seq[2] == ss->com[2])
      continue;  // identical centre of mass: nothing can differ
    double vcen[3];
    for (int k = 0; k < 3; ++k) {
      double vmin = __ddiv_rn(__dsub_rn(ss->bmin[k], ss->com_seq[k]), ss->ssa);
      double vmax = __ddiv_rn(__dsub_rn(ss->bmax[k], ss->com_seq[k]), ss->ssa);
      vcen[k] = __dmul_rn(0.5, __dadd_rn(vmin, vmax));
    }
    const double com[3] = {ss->com_seq[0], ss->com_seq[1], ss->com_seq[2]};
    const int32_t p = perm[i];
    uint64_t k = key_of(x[p], y[p], z[p], com, ss->ssa, vcen, &bad);
    if (L != kMaxDepth) k >>= 3 * (kMaxDepth - L);
    if (k != skeys[i]) {
      ss->key_mismatch = 1;
      atomicExch(&sc->key_mismatch, 1);
    }
  }
}

// For systems whose keys differ: the sequential centre of mass replaces the
// parallel one (rebuild path).
__global__ void adopt_seq_com_kernel(SysScalars *sys, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  SysScalars *ss = sys + s;
  if (!ss->key_mismatch) return;
  ss->com[0] = ss->com_seq[0];
  ss->com[1] = ss->com_seq[1];
  ss->com[2] = ss->com_seq[2];
  ss->mass = ss->mass_seq;
  finalize_norm(ss, ss->com, ss->vcen);
}

// Keys from the centres of mass already in the scalars (rebuild path).
__global__ void __launch_bounds__(256)
rekey_kernel(const double *__restrict__ x, const double *__restrict__ y,
             const double *__restrict__ z, int64_t n, int L, const int32_t *__restrict__ sys_of,
             const SysScalars *__restrict__ sys, uint64_t *__restrict__ keys,
             int32_t *__restrict__ vals) {
  int bad = 0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const SysScalars *ss = sys + sys_of[p];
    const double com[3] = {ss->com[0], ss->com[1], ss->com[2]};
    const double vcen[3] = {ss->vcen[0], ss->vcen[1], ss->vcen[2]};
    uint64_t k = key_of(x[p], y[p], z[p], com, ss->ssa, vcen, &bad);
    keys[p] = (L == kMaxDepth || L == 0) ? k : (k >> (3 * (kMaxDepth - L)));
    vals[p] = (int32_t)p;
  }
}

// Smallest depth with unique keys (choose_depth, morton_octree.f90:217-244):
// keys at depth L are the 21-level keys shifted right, so depth L separates
// every pair iff L exceeds the deepest common octal prefix of sorted
// neighbours.  One system only.
__global__ void max_lcp_kernel(const uint64_t *__restrict__ k, int64_t n, Scalars *sc) {
  int best = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t d = k[i] ^ k[i - 1];
    int lcp = d ? (__clzll(d) - 1) / 3 : kMaxDepth;
    best = max(best, lcp);
  }
  atomicMax(&sc->max_lcp, best);
}

__global__ void apply_depth_kernel(uint64_t *__restrict__ k, int64_t n, Scalars *sc) {
  int L = sc->max_lcp + 1;
  if (sc->max_lcp >= kMaxDepth) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      sc->err |= kErrDuplicates;
      sc->L = kMaxDepth;
    }
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->L = L;
  int shift = 3 * (kMaxDepth - L);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    k[i] >>= shift;
}

// system of every body, from the offsets (one block per system)
__global__ void sys_of_kernel(const SysScalars *__restrict__ sys, int32_t *__restrict__ sys_of) {
  const int64_t off = sys[blockIdx.x].off, n = sys[blockIdx.x].n;
  for (int64_t p = threadIdx.x; p < n; p += blockDim.x) sys_of[off + p] = (int32_t)blockIdx.x;
}

}  // namespace

void launch_layout(Buffers &b, cudaStream_t s) {
  sys_of_kernel<<<b.nsys, 256, 0, s>>>(b.ss, b.sys_of);
}

void launch_keys(const double *m, const double *x, const double *y, const double *z, int64_t n,
                 int L, double amp, int com_mode, Buffers &b, cudaStream_t s) {
  cudaMemsetAsync(b.sc, 0, sizeof(Scalars), s);  // batch-wide flags start clear
  reduce_partials<<<b.n_items, kRedThreads, 0, s>>>(m, x, y, z, b.items, com_mode, b.partials);
  finalize_kernel<<<b.nsys, 320, 0, s>>>(b.partials, b.items, b.n_items, amp,
                                         L == 0 ? kMaxDepth : L, b.ss, b.sc);
  keys_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(x, y, z, n, L == 0 ? kMaxDepth : L,
                                                         b.sys_of, b.ss, b.sc, b.k0, b.v0);
}

// The reference's sequential centre of mass (slow path): the systems with
// ambiguous keys, or all systems when `all` is set.
void launch_seq_com(const double *m, const double *x, const double *y, const double *z,
                    int com_mode, int all, Buffers &b, cudaStream_t s) {
  seq_com_kernel<<<b.nsys, kSeqThreads, 2 * kSeqTile * sizeof(double4), s>>>(m, x, y, z, com_mode,
                                                                             all, b.ss);
}

void launch_verify_keys(const double *x, const double *y, const double *z, int64_t n, int all,
                        Buffers &b, cudaStream_t s) {
  verify_keys_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(x, y, z, n, all, b.sys_of, b.ss,
                                                                b.sc, b.k0, b.v0);
}

void launch_adopt_seq_com(Buffers &b, cudaStream_t s) {
  adopt_seq_com_kernel<<<(b.nsys + 127) / 128, 128, 0, s>>>(b.ss, b.nsys);
}

void launch_keys_only(const double *x, const double *y, const double *z, int64_t n, int L,
                      Buffers &b, cudaStream_t s) {
  rekey_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(x, y, z, n, L == 0 ? kMaxDepth : L,
                                                          b.sys_of, b.ss, b.k0, b.v0);
}

void launch_auto_depth(int64_t n, Buffers &b, cudaStream_t s) {
  cudaMemsetAsync(&b.sc->max_lcp, 0, sizeof(int), s);
  max_lcp_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(b.k0, n, b.sc);
  apply_depth_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(b.k0, n, b.sc);
}

void set_seq_com_smem_limit() {
  cudaFuncSetAttribute(seq_com_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(2 * kSeqTile * sizeof(double4)));
}

}  // namespace bh
