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
//
// In a batch every system is its own segment of the sorted arrays: the
// binary tree of a segment [s0, s1) uses internal nodes s0 .. s1 - 2 (the slot
// s1 - 1 stays unused) and treats bodies outside the segment as absent, so
// every system gets its own root; all later steps run over all systems at once.
#include "bh_internal.cuh"

namespace bh {

namespace {

__device__ __forceinline__ int delta(const uint64_t *__restrict__ k, int64_t s0, int64_t s1,
                                     int64_t i, uint64_t ki, int64_t j) {
  if (j < s0 || j >= s1) return -1;
  uint64_t kj = k[j];
  if (ki != kj) return __clzll((long long)(ki ^ kj));
  return 64 + __clz((int)(i ^ j));
}

__global__ void __launch_bounds__(256)
karras_kernel(const uint64_t *__restrict__ k, int64_t n, const int32_t *__restrict__ sys_of,
              const SysScalars *__restrict__ sys, const Scalars *__restrict__ sc,
              int32_t *__restrict__ left, int32_t *__restrict__ right,
              int32_t *__restrict__ parent, int32_t *__restrict__ first,
              int32_t *__restrict__ last, int32_t *__restrict__ level) {
  const int L = sc->L;
  const int lead = 64 - 3 * L;  // leading zero bits of every key
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const SysScalars &ss = sys[sys_of[i]];
    const int64_t s0 = ss.off, s1 = ss.off + ss.n;
    if (i == s1 - 1) continue;  // the segment's unused slot (marked by mark_kernel)
    const uint64_t ki = k[i];
    const int d = (delta(k, s0, s1, i, ki, i + 1) - delta(k, s0, s1, i, ki, i - 1)) > 0 ? 1 : -1;
    const int dmin = delta(k, s0, s1, i, ki, i - d);
    int64_t lmax = 2;
    while (delta(k, s0, s1, i, ki, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (delta(k, s0, s1, i, ki, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(k, s0, s1, i, ki, j);
    int64_t s = 0, t = l;
    do {
      t = (t + 1) >> 1;
      if (delta(k, s0, s1, i, ki, i + (s + t) * d) > dnode) s += t;
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
    if (i == s0) parent[i] = -1;  // the segment's root
  }
}

__global__ void __launch_bounds__(256)
mark_kernel(int64_t n, const int32_t *__restrict__ sys_of, const SysScalars *__restrict__ sys,
            const int32_t *__restrict__ parent, const int32_t *__restrict__ level,
            int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const SysScalars &ss = sys[sys_of[i]];
    if (i == ss.off + ss.n - 1) { flag[i] = 0; continue; }  // unused slot
    const int p = parent[i];
    flag[i] = (p < 0 || level[i] > level[p]) ? 1 : 0;
  }
}

__global__ void __launch_bounds__(256)
compact_keys_kernel(int64_t n, const int32_t *__restrict__ flag, const int32_t *__restrict__ rank,
                    const int32_t *__restrict__ level, const int32_t *__restrict__ first,
                    int first_bits, uint64_t *__restrict__ ckey, int32_t *__restrict__ cval) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
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
      if (ch[c] >= 0) cparent[ch[c]] = j;  // roots keep the -1 of the initial fill
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

// root node of every system (its segment's binary root), -1 for lone bodies
__global__ void roots_kernel(SysScalars *__restrict__ sys, int nsys,
                             const int32_t *__restrict__ bin2cn) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  sys[s].root = sys[s].n >= 2 ? bin2cn[sys[s].off] : -1;
}

// ---- target groups ----
// Units are the subtrees of <= U bodies whose parent holds more than U bodies
// (lone particles included).  Consecutive units under the same parent are
// concatenated in key order and cut into groups of G bodies (the last one of a
// run shorter); a child with more than U bodies ends the run and is cut by its
// own children.  A node of identical keys (no children) with more than U
// bodies, or a root of <= U bodies, is cut into groups of G directly.
// gflag marks the first body of each group.  With U = G this packs small
// siblings; a larger U fills more groups completely at the price of groups
// that span neighbouring subtrees.
__global__ void __launch_bounds__(256)
group_flags_kernel(const int4 *__restrict__ meta, const int32_t *__restrict__ child,
                   const int32_t *__restrict__ cparent, const Scalars *__restrict__ sc, int G,
                   int U, const SysScalars *__restrict__ sys, int nsys,
                   int32_t *__restrict__ gflag) {
  // every system starts a group (this also covers lone bodies, which have no node)
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nsys; q += gridDim.x * blockDim.x)
    if (sys[q].n > 0) gflag[sys[q].off] = 1;
  const int M = sc->n_compact;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
    const int4 mt = meta[j];  // first, count, level, nchild
    if (mt.y <= U) {
      if (cparent[j] < 0)  // a system's root
        for (int s = 0; s < mt.y; s += G) gflag[mt.x + s] = 1;
      continue;
    }
    if (mt.w == 0) {
      for (int s = 0; s < mt.y; s += G) gflag[mt.x + s] = 1;
      continue;
    }
    int run_first = -1, run_len = 0;
    for (int c = 0; c <= mt.w; ++c) {
      int cfirst = 0, ccount = U + 1;  // c == nchild: closes the last run
      if (c < mt.w) {
        const int32_t ch = child[8 * j + c];
        if (ch < 0) { cfirst = ~ch; ccount = 1; }
        else { const int4 cm = meta[ch]; cfirst = cm.x; ccount = cm.y; }
      }
      if (ccount > U) {
        for (int s = 0; s < run_len; s += G) gflag[run_first + s] = 1;
        run_first = -1;
        run_len = 0;
        continue;
      }
      if (run_first < 0) run_first = cfirst;
      run_len += ccount;
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
  karras_kernel<<<grid, 256, 0, s>>>(b.k0, n, b.sys_of, b.ss, b.sc, b.bn_left, b.bn_right,
                                     b.bn_parent, b.bn_first, b.bn_last, b.bn_level);
  mark_kernel<<<grid, 256, 0, s>>>(n, b.sys_of, b.ss, b.bn_parent, b.bn_level, b.bn_flag);
  // rank of each marked node in binary order, total -> n_compact
  int32_t *rank = b.gscan;          // free until the group pass
  int32_t *total = b.counters + 2;  // scratch counter
  exclusive_scan(b.bn_flag, rank, n, nullptr, total, b.scan_tmp, &b.sc->err, s, &b.sc->n_compact);
  // sort the compact nodes by (level, first particle)
  const int first_bits = bits_for(n);
  uint64_t *ck0 = b.k1;
  int32_t *cv0 = b.v1;
  uint64_t *ck1 = reinterpret_cast<uint64_t *>(b.cn_quad);  // scratch: filled later
  int32_t *cv1 = b.cn_parent;                                // scratch: filled later
  compact_keys_kernel<<<grid, 256, 0, s>>>(n, b.bn_flag, rank, b.bn_level, b.bn_first, first_bits,
                                           ck0, cv0);
  radix_sort_pairs(ck0, cv0, ck1, cv1, n, total, first_bits + 5, b.hist, &b.sc->err, s);
  cudaMemcpyAsync(b.cn_bin, cv0, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
  cudaMemsetAsync(b.cn_parent, 0xff, n * sizeof(int32_t), s);  // roots keep -1
  bin2cn_kernel<<<grid, 256, 0, s>>>(b.cn_bin, b.sc, b.bin2cn);
  records_kernel<<<grid, 256, 0, s>>>(b.cn_bin, b.sc, b.bn_left, b.bn_right, b.bn_first,
                                      b.bn_last, b.bn_level, b.bn_flag, b.bin2cn, b.cn_meta,
                                      b.cn_child, b.cn_parent);
  level_begin_kernel<<<grid, 256, 0, s>>>(b.cn_meta, b.sc, b.level_begin);
  roots_kernel<<<(b.nsys + 127) / 128, 128, 0, s>>>(b.ss, b.nsys, b.bin2cn);
}

void launch_groups(int64_t n, int group_size, int group_span, Buffers &b, cudaStream_t s) {
  const int grid = grid_for(n, 256, 148 * 16);
  cudaMemsetAsync(b.gflag, 0, n * sizeof(int32_t), s);
  group_flags_kernel<<<grid, 256, 0, s>>>(b.cn_meta, b.cn_child, b.cn_parent, b.sc, group_size,
                                          group_span, b.ss, b.nsys, b.gflag);
  int32_t *total = b.counters + 3;
  exclusive_scan(b.gflag, b.gscan, n, nullptr, total, b.scan_tmp, &b.sc->err, s, &b.sc->n_groups);
  group_first_kernel<<<grid, 256, 0, s>>>(n, b.gflag, b.gscan, b.sc, b.g_first);
}

}  // namespace bh
