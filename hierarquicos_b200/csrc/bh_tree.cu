// Octree from the sorted Morton keys, and the target groups of the walk.
//
// The reference (fortran/morton/morton_octree.f90:420-493) materialises one
// node per distinct key prefix at every level 0..L, so a run of particles that
// does not split between two levels appears once per level (a chain), and
// every lone particle is followed down to level L.  The walk of :627-766
// visits such a chain top-down with the same centre of mass and mass at every
// link and opens the next link while the cell-size test fails; since the cell
// size shrinks with depth, the chain is accepted exactly when its deepest
// link passes.  The compact octree built here keeps one node per distinct
// particle range with >= 2 particles (at the deepest level of its chain), and
// lists lone particles as particle children.  It therefore has the
// reference's topology without the chains, and its node order is the
// reference's node order (level, then first particle) restricted to those
// nodes.
//
// Construction: a binary radix tree over the sorted keys (Karras 2012, with
// the index as tie-break for equal keys), whose nodes get the octal level
// floor(common prefix bits / 3); a binary node whose level is deeper than its
// parent's starts a new octree node.  Those nodes are sorted by (level, first
// particle) with the radix sort, and each one enumerates its octree children
// by descending at most three binary levels.
#include "bh_internal.cuh"

namespace bh {

namespace {

__device__ __forceinline__ int delta(const uint64_t *__restrict__ k, int64_t n, int64_t i,
                                     uint64_t ki, int64_t j) {
  if (j < 0 || j >= n) return -1;
  uint64_t kj = k[j];
  if (ki != kj) return __clzll((long long)(ki ^ kj));
  return 64 + __clz((int)(i ^ j));
}

__global__ void __launch_bounds__(256)
karras_kernel(const uint64_t *__restrict__ k, int64_t n, const Scalars *__restrict__ sc,
              int32_t *__restrict__ left, int32_t *__restrict__ right,
              int32_t *__restrict__ parent, int32_t *__restrict__ first,
              int32_t *__restrict__ last, int32_t *__restrict__ level) {
  const int L = sc->L;
  const int lead = 64 - 3 * L;  // leading zero bits of every key
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n - 1;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t ki = k[i];
    const int d = (delta(k, n, i, ki, i + 1) - delta(k, n, i, ki, i - 1)) > 0 ? 1 : -1;
    const int dmin = delta(k, n, i, ki, i - d);
    int64_t lmax = 2;
    while (delta(k, n, i, ki, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (delta(k, n, i, ki, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(k, n, i, ki, j);
    int64_t s = 0, t = l;
    do {
      t = (t + 1) >> 1;
      if (delta(k, n, i, ki, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
    const int64_t f = min(i, j), la = max(i, j);
    const int32_t lc = (f == gamma) ? ~(int32_t)gamma : (int32_t)gamma;
    const int32_t rc = (la == gamma + 1) ? ~(int32_t)(gamma + 1) : (int32_t)(gamma + 1);
    left[i] = lc;
    right[i] = rc;
    first[i] = (int32_t)f;
    last[i] = (int32_t)la;
    int v = (dnode - lead) / 3;
    level[i] = v > L ? L : v;
    if (lc >= 0) parent[lc] = (int32_t)i;
    if (rc >= 0) parent[rc] = (int32_t)i;
    if (i == 0) parent[0] = -1;
  }
}

__global__ void __launch_bounds__(256)
mark_kernel(int64_t n, const int32_t *__restrict__ parent, const int32_t *__restrict__ level,
            int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n - 1;
       i += (int64_t)gridDim.x * blockDim.x) {
    int p = parent[i];
    flag[i] = (i == 0 || level[i] > level[p]) ? 1 : 0;
  }
}

__global__ void __launch_bounds__(256)
compact_keys_kernel(int64_t n, const int32_t *__restrict__ flag, const int32_t *__restrict__ rank,
                    const int32_t *__restrict__ level, const int32_t *__restrict__ first,
                    int first_bits, uint64_t *__restrict__ ckey, int32_t *__restrict__ cval) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n - 1;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    int r = rank[i];
    ckey[r] = ((uint64_t)level[i] << first_bits) | (uint64_t)first[i];
    cval[r] = (int32_t)i;
  }
}

__global__ void __launch_bounds__(256)
bin2cn_kernel(const int32_t *__restrict__ order, const Scalars *__restrict__ sc,
              int32_t *__restrict__ bin2cn) {
  const int M = sc->n_compact;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x)
    bin2cn[order[j]] = j;
}

__global__ void __launch_bounds__(256)
records_kernel(const int32_t *__restrict__ order, Scalars *__restrict__ sc,
               const int32_t *__restrict__ left, const int32_t *__restrict__ right,
               const int32_t *__restrict__ first, const int32_t *__restrict__ last,
               const int32_t *__restrict__ level, const int32_t *__restrict__ flag,
               const int32_t *__restrict__ bin2cn, int4 *__restrict__ meta,
               int32_t *__restrict__ child, int32_t *__restrict__ cparent) {
  const int M = sc->n_compact;
  const int L = sc->L;
  int err = 0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
    const int b = order[j];
    const int f = first[b], la = last[b], v = level[b];
    int nc = 0;
    int32_t ch[8];
    if (v < L) {
      int32_t st[8];
      int top = 0;
      st[top++] = right[b];
      st[top++] = left[b];
      int guard = 0;
      while (top > 0) {
        if (++guard > 64) { err |= kErrChildren; break; }
        int32_t c = st[--top];
        if (c < 0) {
          if (nc < 8) ch[nc] = c;  // particle ~c, stored as ~c (< 0)
          ++nc;
        } else if (flag[c]) {
          if (nc < 8) ch[nc] = bin2cn[c];
          ++nc;
        } else {
          if (top + 2 > 8) { err |= kErrChildren; break; }
          st[top++] = right[c];
          st[top++] = left[c];
        }
      }
      if (nc > 8) { err |= kErrChildren; nc = 8; }
    }
    meta[j] = make_int4(f, la - f + 1, v, nc);
    for (int c = 0; c < 8; ++c) child[8 * j + c] = c < nc ? ch[c] : 0x7fffffff;
    for (int c = 0; c < nc; ++c)
      if (ch[c] >= 0) cparent[ch[c]] = j;
    if (j == 0) cparent[0] = -1;
  }
  if (err) atomicOr(&sc->err, err);
}

// level_begin[l] = first compact node of level >= l; entries up to kNumLevels.
__global__ void __launch_bounds__(256)
level_begin_kernel(const int4 *__restrict__ meta, const Scalars *__restrict__ sc,
                   int32_t *__restrict__ level_begin) {
  const int M = sc->n_compact;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= M; j += gridDim.x * blockDim.x) {
    int lo = (j == 0) ? 0 : meta[j - 1].z + 1;
    int hi = (j == M) ? kNumLevels : meta[j].z;
    for (int l = lo; l <= hi; ++l) level_begin[l] = j;
  }
}

__global__ void count_to_scalars(const int32_t *__restrict__ total, Scalars *sc, int which) {
  if (threadIdx.x == 0) {
    if (which == 0) sc->n_compact = *total;
    else sc->n_groups = *total;
  }
}

// ---- target groups ----
// Each node with more than G bodies packs its consecutive small children
// (lone particles and nodes with <= G bodies) greedily into groups of <= G
// bodies; a big child closes the open group.  A node of identical keys (no
// children) is cut into chunks of G.  gflag marks the first body of each group.
__global__ void __launch_bounds__(256)
group_flags_kernel(const int4 *__restrict__ meta, const int32_t *__restrict__ child,
                   const Scalars *__restrict__ sc, int G, int32_t *__restrict__ gflag) {
  const int M = sc->n_compact;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
    const int4 mt = meta[j];  // first, count, level, nchild
    if (mt.y <= G) {
      if (j == 0) gflag[mt.x] = 1;
      continue;
    }
    if (mt.w == 0) {
      for (int s = 0; s < mt.y; s += G) gflag[mt.x + s] = 1;
      continue;
    }
    int cur = 0;
    for (int c = 0; c < mt.w; ++c) {
      int32_t ch = child[8 * j + c];
      int cfirst, ccount;
      if (ch < 0) { cfirst = ~ch; ccount = 1; }
      else { int4 cm = meta[ch]; cfirst = cm.x; ccount = cm.y; }
      if (ccount > G) { cur = 0; continue; }
      if (cur == 0 || cur + ccount > G) { gflag[cfirst] = 1; cur = ccount; }
      else cur += ccount;
    }
  }
}

__global__ void __launch_bounds__(256)
group_first_kernel(int64_t n, const int32_t *__restrict__ gflag, const int32_t *__restrict__ gscan,
                   const Scalars *__restrict__ sc, int32_t *__restrict__ g_first) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (gflag[i]) g_first[gscan[i]] = (int32_t)i;
  if (blockIdx.x == 0 && threadIdx.x == 0) g_first[sc->n_groups] = (int32_t)n;
}

int bits_for(int64_t v) {
  int b = 1;
  while (((int64_t)1 << b) <= v) ++b;
  return b;
}

}  // namespace

void launch_build_tree(int64_t n, int L, Buffers &b, cudaStream_t s) {
  (void)L;
  const int grid = grid_for(n, 256, 148 * 16);
  karras_kernel<<<grid, 256, 0, s>>>(b.k0, n, b.sc, b.bn_left, b.bn_right, b.bn_parent,
                                     b.bn_first, b.bn_last, b.bn_level);
  mark_kernel<<<grid, 256, 0, s>>>(n, b.bn_parent, b.bn_level, b.bn_flag);
  // rank of each marked node in binary order, total -> n_compact
  int32_t *rank = b.gscan;          // free until the group pass
  int32_t *total = b.counters + 2;  // scratch counter
  exclusive_scan(b.bn_flag, rank, n - 1, nullptr, total, b.scan_tmp, s);
  count_to_scalars<<<1, 32, 0, s>>>(total, b.sc, 0);
  // sort the compact nodes by (level, first particle)
  const int first_bits = bits_for(n);
  uint64_t *ck0 = b.k1;
  int32_t *cv0 = b.v1;
  uint64_t *ck1 = reinterpret_cast<uint64_t *>(b.cn_quad);  // scratch: filled later
  int32_t *cv1 = b.cn_parent;                                // scratch: filled later
  compact_keys_kernel<<<grid, 256, 0, s>>>(n, b.bn_flag, rank, b.bn_level, b.bn_first, first_bits,
                                           ck0, cv0);
  radix_sort_pairs(ck0, cv0, ck1, cv1, n - 1, total, first_bits + 5, b.hist, s);
  cudaMemcpyAsync(b.cn_bin, cv0, (n - 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
  bin2cn_kernel<<<grid, 256, 0, s>>>(b.cn_bin, b.sc, b.bin2cn);
  records_kernel<<<grid, 256, 0, s>>>(b.cn_bin, b.sc, b.bn_left, b.bn_right, b.bn_first,
                                      b.bn_last, b.bn_level, b.bn_flag, b.bin2cn, b.cn_meta,
                                      b.cn_child, b.cn_parent);
  level_begin_kernel<<<grid, 256, 0, s>>>(b.cn_meta, b.sc, b.level_begin);
}

void launch_groups(int64_t n, int group_size, Buffers &b, cudaStream_t s) {
  const int grid = grid_for(n, 256, 148 * 16);
  cudaMemsetAsync(b.gflag, 0, n * sizeof(int32_t), s);
  group_flags_kernel<<<grid, 256, 0, s>>>(b.cn_meta, b.cn_child, b.sc, group_size, b.gflag);
  int32_t *total = b.counters + 3;
  exclusive_scan(b.gflag, b.gscan, n, nullptr, total, b.scan_tmp, s);
  count_to_scalars<<<1, 32, 0, s>>>(total, b.sc, 1);
  group_first_kernel<<<grid, 256, 0, s>>>(n, b.gflag, b.gscan, b.sc, b.g_first);
}

}  // namespace bh
