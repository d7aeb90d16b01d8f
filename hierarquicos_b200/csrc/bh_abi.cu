// C ABI of the force engine: workspace management, the build/walk pipeline
// for batches of systems, CUDA-graph capture and status reporting.  See
// include/hierarquicos_bh.h for the contract.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "bh_internal.cuh"

using bh::Buffers;

struct bh_system {
  int device = 0;
  Buffers b;
  int64_t n = 0;                 // bodies of the current batch
  int nsys = 0;                  // systems of the current batch
  std::vector<int64_t> offsets;  // layout uploaded to the device (nsys + 1 entries)
  std::vector<bh::RedItem> items_host;
  int built = 0;
  int keys_checked = 0;   // strict-key check done for the current build
  // strict-key slow path since creation: sequential centre-of-mass checks run,
  // and builds redone because a key differed
  int64_t key_checks = 0, key_rebuilds = 0;
  int64_t walks_enqueued = 0;  // every walk put on a stream (a redone walk included)
  int order = 4;
  int64_t stack_cap = 4096;
  int fixed_buffers = 0;  // buffers provided by the caller: never reallocated
  const double *m = nullptr, *x = nullptr, *y = nullptr, *z = nullptr;
  bh_params p{};
  // the last walk of the current build, repeated if the build is redone
  int walked = 0;
  bh_params walk_p{};
  double *walk_out = nullptr;
  int walk_g0 = 0, walk_g1 = -1;  // its target groups (bh_system_walk_groups)
  // captured build + walk of the current layout
  cudaGraphExec_t graph = nullptr;
  // pinned staging of the layout's reduction items; the event marks the end
  // of the last layout upload, after which ss_host and items_pin may be reused
  bh::RedItem *items_pin = nullptr;
  int items_pin_cap = 0;
  cudaEvent_t layout_ev = nullptr;
  bool layout_pending = false;
  // Dehnen's method, allocated on first use
  bh::DehnenBuffers dehnen;
  // host-array entry points: the four input copies run on four streams at
  // once (one copy engine stream does not fill the host link), created on
  // first use
  cudaStream_t copy_st[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t copy_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // pageable host arrays: staged by host threads through pinned slots
  bh::HostCopy *hcopy = nullptr;
};

namespace {

thread_local char g_err[512] = "";

int set_err(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

#define BH_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return set_err(e_ == cudaErrorMemoryAllocation ? BH_ERR_NOMEM : BH_ERR_CUDA, "%s: %s", \
                     #call, cudaGetErrorString(e_));                                         \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, int64_t count) {
  if (count < 1) count = 1;
  return cudaMalloc((void **)p, (size_t)count * sizeof(T));
}

void drop_graph(bh_system *s) {
  if (s->graph) cudaGraphExecDestroy(s->graph);
  s->graph = nullptr;
}

void free_body_buffers(Buffers &b) {
  void *ptrs[] = {b.hm, b.hx, b.hy, b.hz, b.hout, b.k0, b.k1, b.v0, b.v1, b.hist, b.sys_of,
                  b.spos, b.bn_left, b.bn_right, b.bn_parent, b.bn_first, b.bn_last, b.bn_level,
                  b.bn_flag, b.bin2cn, b.cn_bin, b.cn_meta, b.cn_child, b.cn_parent, b.cn_com,
                  b.cn_quad, b.cn_oct, b.cn_fq, b.cn_fo, b.gflag, b.gscan, b.g_first, b.scan_tmp};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  b.hm = b.hx = b.hy = b.hz = b.hout = nullptr;
  b.k0 = b.k1 = nullptr;
  b.v0 = b.v1 = b.hist = b.sys_of = nullptr;
  b.spos = nullptr;
  b.bn_left = b.bn_right = b.bn_parent = b.bn_first = b.bn_last = b.bn_level = nullptr;
  b.bn_flag = b.bin2cn = b.cn_bin = b.cn_child = b.cn_parent = nullptr;
  b.cn_meta = nullptr;
  b.cn_com = nullptr;
  b.cn_quad = b.cn_oct = nullptr;
  b.cn_fq = b.cn_fo = nullptr;
  b.gflag = b.gscan = b.g_first = b.scan_tmp = nullptr;
  b.cap = 0;
}

void free_buffers(Buffers &b) {
  free_body_buffers(b);
  void *ptrs[] = {b.partials, b.items, b.ss, b.level_begin, b.wstack, b.counters, b.stats, b.sc};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (b.sc_host) cudaFreeHost(b.sc_host);
  if (b.ss_host) cudaFreeHost(b.ss_host);
  b = Buffers();
}

// Workspace for n bodies in nsys systems with n_items reduction items.  Each
// part grows on its own; growing the body arrays forces a new layout upload.
int ensure_capacity(bh_system *s, int64_t n, int nsys, int n_items) {
  Buffers &b = s->b;
  const bool body_ok = b.cap >= n;
  const bool sys_ok = b.sys_cap >= nsys && b.items_cap >= n_items;
  const bool stack_ok = b.wstack && b.wstack_cap >= s->stack_cap;
  if (body_ok && sys_ok && stack_ok && b.sc) return BH_OK;
  if (s->fixed_buffers)
    return set_err(BH_ERR_CAPACITY,
                   "fixed workspace too small (n=%lld in %d systems, capacity %lld bodies)",
                   (long long)n, nsys, (long long)b.cap);
  drop_graph(s);
  if (!b.sc) {
    BH_CUDA(dalloc(&b.level_begin, bh::kNumLevels + 2));
    BH_CUDA(dalloc(&b.counters, 8));
    BH_CUDA(dalloc(&b.stats, 4));
    BH_CUDA(dalloc(&b.sc, 1));
    BH_CUDA(cudaMallocHost((void **)&b.sc_host, sizeof(bh::Scalars)));
    BH_CUDA(cudaMemset(b.sc, 0, sizeof(bh::Scalars)));
    BH_CUDA(cudaMemset(b.stats, 0, 4 * sizeof(unsigned long long)));
  }
  if (!stack_ok) {
    if (b.wstack) cudaFree(b.wstack);
    b.wstack = nullptr;
    b.wstack_slots = bh::walk_slots();
    BH_CUDA(dalloc(&b.wstack, b.wstack_slots * s->stack_cap));
    b.wstack_cap = s->stack_cap;
  }
  if (!sys_ok) {
    if (s->layout_pending) cudaEventSynchronize(s->layout_ev);
    s->layout_pending = false;
    if (b.ss) cudaFree(b.ss);
    if (b.ss_host) cudaFreeHost(b.ss_host);
    if (b.items) cudaFree(b.items);
    if (b.partials) cudaFree(b.partials);
    b.ss = nullptr;
    b.ss_host = nullptr;
    b.items = nullptr;
    b.partials = nullptr;
    const int sc_ = nsys > b.sys_cap ? nsys : b.sys_cap;
    const int ic = n_items > b.items_cap ? n_items : b.items_cap;
    BH_CUDA(dalloc(&b.ss, sc_));
    BH_CUDA(cudaMallocHost((void **)&b.ss_host, (size_t)sc_ * sizeof(bh::SysScalars)));
    BH_CUDA(dalloc(&b.items, ic));
    BH_CUDA(dalloc(&b.partials, 10 * (int64_t)ic));
    if (s->layout_pending) cudaEventSynchronize(s->layout_ev);
    s->layout_pending = false;
    if (s->items_pin) cudaFreeHost(s->items_pin);
    s->items_pin = nullptr;
    BH_CUDA(cudaMallocHost((void **)&s->items_pin, (size_t)ic * sizeof(bh::RedItem)));
    s->items_pin_cap = ic;
    b.sys_cap = sc_;
    b.items_cap = ic;
    b.nsys = 0;
    s->offsets.clear();
  }
  if (!body_ok) {
    free_body_buffers(b);
    const int64_t c = n < 2 ? 2 : n;
    BH_CUDA(dalloc(&b.k0, c)); BH_CUDA(dalloc(&b.k1, c));
    BH_CUDA(dalloc(&b.v0, c)); BH_CUDA(dalloc(&b.v1, c));
    b.hist_cap = bh::radix_hist_entries(c);
    BH_CUDA(dalloc(&b.hist, b.hist_cap));
    BH_CUDA(dalloc(&b.sys_of, c));
    BH_CUDA(dalloc(&b.spos, c));
    BH_CUDA(dalloc(&b.bn_left, c)); BH_CUDA(dalloc(&b.bn_right, c)); BH_CUDA(dalloc(&b.bn_parent, c));
    BH_CUDA(dalloc(&b.bn_first, c)); BH_CUDA(dalloc(&b.bn_last, c)); BH_CUDA(dalloc(&b.bn_level, c));
    BH_CUDA(dalloc(&b.bn_flag, c)); BH_CUDA(dalloc(&b.bin2cn, c));
    BH_CUDA(dalloc(&b.cn_bin, c)); BH_CUDA(dalloc(&b.cn_meta, c)); BH_CUDA(dalloc(&b.cn_child, 8 * c));
    BH_CUDA(dalloc(&b.cn_parent, c)); BH_CUDA(dalloc(&b.cn_com, c));
    BH_CUDA(dalloc(&b.cn_quad, 6 * c)); BH_CUDA(dalloc(&b.cn_oct, 14 * c));
    BH_CUDA(dalloc(&b.cn_fq, 2 * c)); BH_CUDA(dalloc(&b.cn_fo, 4 * c));
    BH_CUDA(dalloc(&b.gflag, c + 1)); BH_CUDA(dalloc(&b.gscan, c + 1)); BH_CUDA(dalloc(&b.g_first, c + 1));
    b.scan_tmp_cap = bh::scan_tmp_entries(c + 1);
    BH_CUDA(dalloc(&b.scan_tmp, b.scan_tmp_cap));
    b.cap = c;
    b.nsys = 0;
    s->offsets.clear();
  }
  return BH_OK;
}

int ensure_host_staging(bh_system *s, int64_t n) {
  Buffers &b = s->b;
  if (b.hm && b.cap >= n) return BH_OK;
  if (b.hm) { cudaFree(b.hm); cudaFree(b.hx); cudaFree(b.hy); cudaFree(b.hz); cudaFree(b.hout); }
  const int64_t c = b.cap;
  BH_CUDA(dalloc(&b.hm, c)); BH_CUDA(dalloc(&b.hx, c)); BH_CUDA(dalloc(&b.hy, c));
  BH_CUDA(dalloc(&b.hz, c)); BH_CUDA(dalloc(&b.hout, 3 * c));
  return BH_OK;
}

// reduction work items: every system is cut into chunks of kRedChunk bodies
int count_items(const int64_t *off, int nsys) {
  int64_t k = 0;
  for (int q = 0; q < nsys; ++q) k += (off[q + 1] - off[q] + bh::kRedChunk - 1) / bh::kRedChunk;
  return (int)k;
}

// Uploads a batch layout (offsets, reduction items, system of every body)
// unless it is the one already on the device.
int set_layout(bh_system *s, const int64_t *off, int nsys, cudaStream_t st) {
  Buffers &b = s->b;
  if (b.nsys == nsys && (int)s->offsets.size() == nsys + 1 &&
      memcmp(s->offsets.data(), off, (size_t)(nsys + 1) * sizeof(int64_t)) == 0)
    return BH_OK;
  drop_graph(s);
  // pinned staging (pageable host memory for caller-provided workspaces)
  bh::RedItem *items = s->items_pin;
  if (s->fixed_buffers || !items) {
    s->items_host.resize((size_t)count_items(off, nsys));
    items = s->items_host.data();
  } else if (s->layout_pending) {
    BH_CUDA(cudaEventSynchronize(s->layout_ev));  // the previous upload has left the staging
  }
  int k = 0;
  for (int q = 0; q < nsys; ++q)
    for (int64_t a = off[q]; a < off[q + 1]; a += bh::kRedChunk)
      items[k++] = bh::RedItem{q, 0, a, a + bh::kRedChunk < off[q + 1] ? a + bh::kRedChunk : off[q + 1]};
  for (int q = 0; q < nsys; ++q) {
    memset(&b.ss_host[q], 0, sizeof(bh::SysScalars));
    b.ss_host[q].off = off[q];
    b.ss_host[q].n = off[q + 1] - off[q];
    b.ss_host[q].root = -1;
  }
  BH_CUDA(cudaMemcpyAsync(b.ss, b.ss_host, (size_t)nsys * sizeof(bh::SysScalars),
                          cudaMemcpyHostToDevice, st));
  BH_CUDA(cudaMemcpyAsync(b.items, items, (size_t)k * sizeof(bh::RedItem), cudaMemcpyHostToDevice, st));
  b.n_items = k;
  b.nsys = nsys;
  bh::launch_layout(b, st);
  if (items == s->items_pin) {
    if (!s->layout_ev) BH_CUDA(cudaEventCreateWithFlags(&s->layout_ev, cudaEventDisableTiming));
    BH_CUDA(cudaEventRecord(s->layout_ev, st));
    s->layout_pending = true;
  } else {
    BH_CUDA(cudaStreamSynchronize(st));  // pageable staging is reused by the next layout
  }
  s->offsets.assign(off, off + nsys + 1);
  return BH_OK;
}

int check_params(const bh_params *p, int64_t n) {
  if (!p) return set_err(BH_ERR_INVALID, "params is NULL");
  if (n < 1 || n > (int64_t)(1 << 30)) return set_err(BH_ERR_INVALID, "n=%lld out of range [1, 2^30]", (long long)n);
  if (p->order != 1 && p->order != 4 && p->order != 8)
    return set_err(BH_ERR_INVALID, "order must be 1, 4 or 8 (got %d)", p->order);
  if (p->depth < 0 || p->depth > bh::kMaxDepth)
    return set_err(BH_ERR_INVALID, "depth must be in 0..21 (got %d)", p->depth);
  if (!(p->theta >= 0.0) || !isfinite(p->theta)) return set_err(BH_ERR_INVALID, "theta must be finite and >= 0");
  if (!(p->eps >= 0.0) || !isfinite(p->eps)) return set_err(BH_ERR_INVALID, "eps must be finite and >= 0");
  if (!isfinite(p->G)) return set_err(BH_ERR_INVALID, "G must be finite");
  if (!(p->amp > 0.0) || !isfinite(p->amp)) return set_err(BH_ERR_INVALID, "amp must be > 0");
  if (p->precision < 0 || p->precision > 3) return set_err(BH_ERR_INVALID, "precision must be 0, 1, 2 or 3");
  if (p->group_size != 32 && p->group_size != 64) return set_err(BH_ERR_INVALID, "group_size must be 32 or 64");
  if (p->leaf_cap < 1 || p->leaf_cap > 64) return set_err(BH_ERR_INVALID, "leaf_cap must be in 1..64");
  if (p->out_kind != 0 && p->out_kind != 1) return set_err(BH_ERR_INVALID, "out_kind must be 0 or 1");
  if (p->com_mode != 0 && p->com_mode != 1) return set_err(BH_ERR_INVALID, "com_mode must be 0 or 1");
  if (p->strict_keys < 0 || p->strict_keys > 2) return set_err(BH_ERR_INVALID, "strict_keys must be 0, 1 or 2");
  if (p->group_span != 0 && (p->group_span < p->group_size || p->group_span > (1 << 20)))
    return set_err(BH_ERR_INVALID, "group_span must be 0 or in [group_size, 2^20]");
  if (p->mac != 0 && p->mac != 1) return set_err(BH_ERR_INVALID, "mac must be 0 or 1");
  if (p->pipeline != 0 && p->pipeline != 1) return set_err(BH_ERR_INVALID, "pipeline must be 0 or 1");
  return BH_OK;
}

int status_from_device(bh_system *s) {
  const bh::Scalars &h = *s->b.sc_host;
  const int e = h.err;
  if (e & bh::kErrNonFinite)
    return set_err(BH_ERR_NONFINITE, "non-finite position or mass, or total mass <= 0");
  if (e & bh::kErrDuplicates)
    return set_err(BH_ERR_DUPLICATES, "depth 0: coincident bodies never get distinct keys");
  if (e & bh::kErrTimeout)
    return set_err(BH_ERR_INTERNAL, "a bounded wait inside a kernel gave up (flags 0x%x)", e);
  if (e & (bh::kErrIndex | bh::kErrChildren))
    return set_err(BH_ERR_INTERNAL, "internal tree check failed (flags 0x%x)", e);
  if (e & bh::kErrStackOverflow)
    return set_err(BH_ERR_CAPACITY, "walk stack capacity %lld exceeded", (long long)s->stack_cap);
  return BH_OK;
}

int read_scalars(bh_system *s, cudaStream_t st) {
  BH_CUDA(cudaMemcpyAsync(s->b.sc_host, s->b.sc, sizeof(bh::Scalars), cudaMemcpyDeviceToHost, st));
  BH_CUDA(cudaStreamSynchronize(st));
  return BH_OK;
}

// keys (from scratch, or from the centres of mass already in the system
// scalars) -> sort -> octree -> multipoles -> groups, for the whole batch
void enqueue_build(bh_system *s, int keys_from_scalars, cudaStream_t st) {
  Buffers &b = s->b;
  const bh_params &p = s->p;
  const int64_t n = s->n;
  const int L = p.depth;
  if (keys_from_scalars)
    bh::launch_keys_only(s->x, s->y, s->z, n, L, b, st);
  else
    bh::launch_keys(s->m, s->x, s->y, s->z, n, L, p.amp, p.com_mode, b, st);
  const int bits = (L == 0) ? 3 * bh::kMaxDepth : 3 * L;
  bh::radix_sort_pairs(b.k0, b.v0, b.k1, b.v1, n, nullptr, bits, b.hist, &b.sc->err, st);
  bh::launch_sort_by_system(n, b, st);
  if (L == 0) bh::launch_auto_depth(n, b, st);
  bh::launch_gather(s->m, s->x, s->y, s->z, n, b, st);
  bh::launch_build_tree(n, L, b, st);
  bh::launch_upward(n, L, p.order, b, st);
  bh::launch_groups(n, p.group_size, p.group_span > 0 ? p.group_span : 2 * p.group_size, b, st);
}

bh::WalkParams walk_params(const bh_params *p, int order) {
  bh::WalkParams w;
  w.theta2 = p->theta * p->theta;
  w.G = p->G;
  w.eps2 = p->eps * p->eps;
  w.order = p->order < order ? p->order : order;
  w.out_kind = p->out_kind;
  w.precision = p->precision;
  w.group_size = p->group_size;
  w.leaf_cap = p->leaf_cap;
  w.count_stats = p->count_stats;
  w.mac = p->mac;
  w.pipeline = p->pipeline;
  return w;
}

// the walk of the whole batch, enqueued without host synchronisation
int enqueue_walk(bh_system *s, const bh_params *p, double *d_out, cudaStream_t st) {
  ++s->walks_enqueued;
  bh::WalkParams w = walk_params(p, s->order);
  w.g_begin = s->walk_g0;
  w.g_end = s->walk_g1;
  if (w.count_stats) cudaMemsetAsync(s->b.stats, 0, 4 * sizeof(unsigned long long), st);
  if (p->precision == BH_PREC_DEHNEN) {
    switch (bh::run_dehnen(s->n, w, s->b, s->dehnen, d_out, st)) {
      case 0: return BH_OK;
      case 1: return set_err(BH_ERR_NOMEM, "Dehnen: device allocation failed");
      case 2: return set_err(BH_ERR_CUDA, "Dehnen: %s", cudaGetErrorString(cudaGetLastError()));
      case 3: return set_err(BH_ERR_INTERNAL, "Dehnen: the dual traversal did not close");
      default: return set_err(BH_ERR_CAPACITY, "Dehnen: more than 2^30 mutual interactions");
    }
  }
  if (p->precision == BH_PREC_REFERENCE)
    bh::launch_reference_walk(s->n, w, s->b, d_out, nullptr, 0, nullptr, st);
  else
    bh::launch_walk(s->n, w, s->b, d_out, st);
  return BH_OK;
}

int validate_offsets(const int64_t *off, int nsys, int64_t *total) {
  if (!off || nsys < 1) return set_err(BH_ERR_INVALID, "a batch needs at least one system");
  if (nsys > (1 << 24)) return set_err(BH_ERR_INVALID, "more than 2^24 systems");
  if (off[0] != 0) return set_err(BH_ERR_INVALID, "offsets[0] must be 0");
  for (int q = 0; q < nsys; ++q)
    if (off[q + 1] <= off[q])
      return set_err(BH_ERR_INVALID, "system %d is empty (offsets must increase strictly)", q);
  *total = off[nsys];
  return BH_OK;
}

int build_common(bh_system *s, const double *d_m, const double *d_x, const double *d_y,
                 const double *d_z, const int64_t *off, int nsys, const bh_params *p,
                 cudaStream_t st) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  int64_t n = 0;
  int rc = validate_offsets(off, nsys, &n);
  if (rc) return rc;
  rc = check_params(p, n);
  if (rc) return rc;
  if (!d_m || !d_x || !d_y || !d_z) return set_err(BH_ERR_INVALID, "NULL input array");
  if (nsys > 1 && p->depth == 0)
    return set_err(BH_ERR_INVALID, "depth 0 (automatic) applies to a single system only");
  BH_CUDA(cudaSetDevice(s->device));
  rc = ensure_capacity(s, n, nsys, count_items(off, nsys));
  if (rc) return rc;
  rc = set_layout(s, off, nsys, st);
  if (rc) return rc;
  s->p = *p;
  s->m = d_m; s->x = d_x; s->y = d_y; s->z = d_z;
  s->n = n;
  s->nsys = nsys;
  s->order = p->order;
  s->walked = 0;
  enqueue_build(s, 0, st);
  BH_CUDA(cudaGetLastError());
  s->built = 1;
  s->keys_checked = p->strict_keys ? 0 : 1;
  return BH_OK;
}

// Completes a build + walk: strict-key check (slow path only when a body lies
// within the rounding margin of a cell edge), stack-capacity retries, status.
int finish(bh_system *s, cudaStream_t st) {
  int rc = read_scalars(s, st);
  if (rc) return rc;
  if (!s->keys_checked && (s->b.sc_host->key_ambiguous || s->p.strict_keys == 2) &&
      !(s->b.sc_host->err & bh::kErrNonFinite)) {
    // the reference's sequential centre of mass decides the ambiguous keys
    const int all = s->p.strict_keys == 2;
    bh::launch_seq_com(s->m, s->x, s->y, s->z, s->p.com_mode, all, s->b, st);
    bh::launch_verify_keys(s->x, s->y, s->z, s->n, all, s->b, st);
    rc = read_scalars(s, st);
    if (rc) return rc;
    ++s->key_checks;
    if (s->b.sc_host->key_mismatch) {
      ++s->key_rebuilds;
      bh::launch_adopt_seq_com(s->b, st);
      enqueue_build(s, 1, st);
      if (s->walked) {
        rc = enqueue_walk(s, &s->walk_p, s->walk_out, st);
        if (rc) return rc;
      }
      BH_CUDA(cudaGetLastError());
      rc = read_scalars(s, st);
      if (rc) return rc;
    }
  }
  s->keys_checked = 1;
  for (int attempt = 0;
       attempt < 4 && s->walked && !s->fixed_buffers && (s->b.sc_host->err & bh::kErrStackOverflow);
       ++attempt) {
    s->stack_cap *= 2;
    rc = ensure_capacity(s, s->n, s->nsys, s->b.n_items);
    if (rc) return rc;
    BH_CUDA(cudaMemsetAsync(&s->b.sc->err, 0, sizeof(int), st));
    rc = enqueue_walk(s, &s->walk_p, s->walk_out, st);
    if (rc) return rc;
    BH_CUDA(cudaGetLastError());
    rc = read_scalars(s, st);
    if (rc) return rc;
  }
  return status_from_device(s);
}

std::mutex g_default_mu;
bh_system *g_default[64] = {nullptr};

int default_system(bh_system **out) {
  int dev = 0;
  BH_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_err(BH_ERR_INVALID, "device %d out of range", dev);
  if (!g_default[dev]) {
    int rc = bh_system_create(&g_default[dev], dev);
    if (rc) return rc;
  }
  *out = g_default[dev];
  return BH_OK;
}

int ensure_hostcopy(bh_system *s) {
  if (!s->hcopy) s->hcopy = bh::hostcopy_create(s->device);
  if (!s->hcopy) return set_err(BH_ERR_CUDA, "host staging: %s", cudaGetErrorString(cudaGetLastError()));
  return BH_OK;
}

// copies host arrays into the default system's staging buffers: pinned
// arrays straight from the caller's memory, pageable ones through the host
// staging threads
int stage_inputs(bh_system *s, const double *m, const double *x, const double *y,
                 const double *z, int64_t n, cudaStream_t st) {
  const int64_t off[2] = {0, n};
  int rc = ensure_capacity(s, n, 1, count_items(off, 1));
  if (rc) return rc;
  rc = ensure_host_staging(s, n);
  if (rc) return rc;
  Buffers &b = s->b;
  const double *in[4] = {m, x, y, z};
  bool pinned = true;
  for (const double *a : in) {
    const bh::HostKind k = bh::host_kind(a);
    if (k == bh::HostKind::kDevice)
      return set_err(BH_ERR_INVALID, "a device pointer was passed where host arrays are expected");
    pinned = pinned && k == bh::HostKind::kPinned;
  }
  if (!pinned) {
    rc = ensure_hostcopy(s);
    if (rc) return rc;
    double *dst[4] = {b.hm, b.hx, b.hy, b.hz};
    BH_CUDA(bh::hostcopy_upload(s->hcopy, in, dst, 4, n, st));
    return BH_OK;
  }
  if (!s->copy_ev[0]) {
    for (int k = 0; k < 3; ++k)
      BH_CUDA(cudaStreamCreateWithFlags(&s->copy_st[k], cudaStreamNonBlocking));
    for (int k = 0; k < 4; ++k)
      BH_CUDA(cudaEventCreateWithFlags(&s->copy_ev[k], cudaEventDisableTiming));
  }
  // the copy streams start after the work already queued on st (the staging
  // buffers may still be read by it); st then waits for all four copies
  BH_CUDA(cudaEventRecord(s->copy_ev[3], st));
  const double *src[3] = {x, y, z};
  double *dst[3] = {b.hx, b.hy, b.hz};
  for (int k = 0; k < 3; ++k) {
    BH_CUDA(cudaStreamWaitEvent(s->copy_st[k], s->copy_ev[3], 0));
    BH_CUDA(cudaMemcpyAsync(dst[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice,
                            s->copy_st[k]));
    BH_CUDA(cudaEventRecord(s->copy_ev[k], s->copy_st[k]));
  }
  BH_CUDA(cudaMemcpyAsync(b.hm, m, n * sizeof(double), cudaMemcpyHostToDevice, st));
  for (int k = 0; k < 3; ++k) BH_CUDA(cudaStreamWaitEvent(st, s->copy_ev[k], 0));
  return BH_OK;
}

}  // namespace

int bh_report_error(int code, const char *msg) { return set_err(code, "%s", msg); }

// A system over caller-provided buffers (the allocation-free entry point):
// never reallocated; the host mirrors are the caller's.
bh_system *bh::fixed_system_create(int device, const Buffers &b, Scalars *host_sc,
                                   SysScalars *host_ss) {
  bh_system *s = new bh_system();
  s->device = device;
  bh_params_default(&s->p);
  s->b = b;
  s->b.sc_host = host_sc;
  s->b.ss_host = host_ss;
  s->stack_cap = b.wstack_cap;
  s->fixed_buffers = 1;
  s->items_host.reserve(1);
  bh::set_seq_com_smem_limit();
  return s;
}

extern "C" {

void bh_params_default(bh_params *p) {
  memset(p, 0, sizeof *p);
  p->theta = 0.5;
  p->G = 1.0;
  p->eps = 0.0;
  p->order = 4;
  p->out_kind = 0;
  p->depth = 21;
  p->precision = BH_PREC_FP32;
  p->amp = 1.2;
  p->group_size = 64;
  p->leaf_cap = 8;
  p->com_mode = 1;
  p->strict_keys = 1;
  p->mac = 1;
  p->pipeline = 1;
}

const char *bh_version(void) { return "hierarquicos-b200 0.2.0 (sm_100a)"; }

int bh_last_error(char *buf, int len) {
  if (buf && len > 0) {
    strncpy(buf, g_err, (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)strlen(g_err);
}

int bh_system_create(bh_system **sys, int device) {
  if (!sys) return set_err(BH_ERR_INVALID, "sys is NULL");
  *sys = nullptr;
  int ndev = 0;
  BH_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return set_err(BH_ERR_INVALID, "no CUDA device %d", device);
  BH_CUDA(cudaSetDevice(device));
  bh_system *s = new bh_system();
  s->device = device;
  bh_params_default(&s->p);
  bh::set_seq_com_smem_limit();
  *sys = s;
  return BH_OK;
}

int bh_system_destroy(bh_system *s) {
  if (!s) return BH_OK;
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  drop_graph(s);
  bh::free_dehnen(s->dehnen);
  if (!s->fixed_buffers) free_buffers(s->b);
  if (s->items_pin) cudaFreeHost(s->items_pin);
  if (s->layout_ev) cudaEventDestroy(s->layout_ev);
  for (int k = 0; k < 3; ++k)
    if (s->copy_st[k]) cudaStreamDestroy(s->copy_st[k]);
  for (int k = 0; k < 4; ++k)
    if (s->copy_ev[k]) cudaEventDestroy(s->copy_ev[k]);
  bh::hostcopy_destroy(s->hcopy);
  delete s;
  return BH_OK;
}

int bh_system_reserve(bh_system *s, int64_t n, int nsys) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (n < 1 || n > (int64_t)(1 << 30) || nsys < 1 || nsys > n)
    return set_err(BH_ERR_INVALID, "reserve: need 1 <= nsys <= n <= 2^30");
  BH_CUDA(cudaSetDevice(s->device));
  // every system adds at most one partial reduction chunk
  const int64_t items = (n + bh::kRedChunk - 1) / bh::kRedChunk + nsys;
  return ensure_capacity(s, n, nsys, (int)items);
}

int bh_system_build(bh_system *s, const double *d_m, const double *d_x, const double *d_y,
                    const double *d_z, int64_t n, const bh_params *p, void *stream) {
  if (n < 1 || n > (int64_t)(1 << 30))
    return set_err(BH_ERR_INVALID, "n=%lld out of range [1, 2^30]", (long long)n);
  const int64_t off[2] = {0, n};
  return build_common(s, d_m, d_x, d_y, d_z, off, 1, p, (cudaStream_t)stream);
}

int bh_system_build_batch(bh_system *s, const double *d_m, const double *d_x,
                          const double *d_y, const double *d_z, const int64_t *offsets,
                          int nsys, const bh_params *p, void *stream) {
  return build_common(s, d_m, d_x, d_y, d_z, offsets, nsys, p, (cudaStream_t)stream);
}

// The walk over target groups [g0, g1) (g1 < 0: all), remembered so that a
// repeated walk (strict-key rebuild, stack growth) covers the same groups.
static int walk_impl(bh_system *s, const bh_params *p, int g0, int g1, double *d_out,
                     void *stream) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (!s->built) return set_err(BH_ERR_NOT_BUILT, "walk before build");
  int rc = check_params(p, s->n);
  if (rc) return rc;
  if (p->order > s->order) return set_err(BH_ERR_INVALID, "order %d above the built order %d", p->order, s->order);
  if (!d_out) return set_err(BH_ERR_INVALID, "NULL output");
  BH_CUDA(cudaSetDevice(s->device));
  s->walk_g0 = g0;
  s->walk_g1 = g1;
  rc = enqueue_walk(s, p, d_out, (cudaStream_t)stream);
  if (rc) return rc;
  BH_CUDA(cudaGetLastError());
  s->walked = 1;
  s->walk_p = *p;
  s->walk_out = d_out;
  return BH_OK;
}

int bh_system_walk(bh_system *s, const bh_params *p, double *d_out, void *stream) {
  return walk_impl(s, p, 0, -1, d_out, stream);
}

int bh_system_walk_groups(bh_system *s, const bh_params *p, int64_t g_begin, int64_t g_end,
                          double *d_out, void *stream) {
  if (!p) return set_err(BH_ERR_INVALID, "params is NULL");
  if (p->precision != BH_PREC_FP32 && p->precision != BH_PREC_FP64)
    return set_err(BH_ERR_INVALID, "a range of target groups needs the group walk (FP32 or FP64)");
  if (g_begin < 0 || g_end < g_begin || g_end > ((int64_t)1 << 30))
    return set_err(BH_ERR_INVALID, "group range [%lld, %lld) invalid", (long long)g_begin,
                   (long long)g_end);
  return walk_impl(s, p, (int)g_begin, (int)g_end, d_out, stream);
}

int bh_system_sync(bh_system *s, void *stream) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (!s->built) return set_err(BH_ERR_NOT_BUILT, "sync before build");
  BH_CUDA(cudaSetDevice(s->device));
  return finish(s, (cudaStream_t)stream);
}

int bh_system_forces(bh_system *s, const double *d_m, const double *d_x, const double *d_y,
                     const double *d_z, int64_t n, const bh_params *p, double *d_out,
                     void *stream) {
  int rc = bh_system_build(s, d_m, d_x, d_y, d_z, n, p, stream);
  if (rc) return rc;
  rc = bh_system_walk(s, p, d_out, stream);
  if (rc) return rc;
  return finish(s, (cudaStream_t)stream);
}

int bh_system_forces_batch(bh_system *s, const double *d_m, const double *d_x,
                           const double *d_y, const double *d_z, const int64_t *offsets,
                           int nsys, const bh_params *p, double *d_out, void *stream) {
  int rc = bh_system_build_batch(s, d_m, d_x, d_y, d_z, offsets, nsys, p, stream);
  if (rc) return rc;
  rc = bh_system_walk(s, p, d_out, stream);
  if (rc) return rc;
  return finish(s, (cudaStream_t)stream);
}

int bh_system_capture(bh_system *s, const bh_params *p, double *d_out) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (!s->built) return set_err(BH_ERR_NOT_BUILT, "capture needs a build of the batch first");
  int rc = check_params(p, s->n);
  if (rc) return rc;
  if (!d_out) return set_err(BH_ERR_INVALID, "NULL output");
  if (p->precision == BH_PREC_DEHNEN)
    return set_err(BH_ERR_INVALID, "Dehnen's method sizes its lists on the host: no graph capture");
  BH_CUDA(cudaSetDevice(s->device));
  BH_CUDA(cudaDeviceSynchronize());
  drop_graph(s);
  cudaStream_t cap = nullptr;
  BH_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  const bh_params saved = s->p;
  const int saved_order = s->order;
  s->p = *p;
  s->order = p->order;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue_build(s, 0, cap);
    (void)enqueue_walk(s, p, d_out, cap);
    e = cudaStreamEndCapture(cap, &g);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s->graph, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cap);
  if (e != cudaSuccess) {
    s->graph = nullptr;
    s->p = saved;
    s->order = saved_order;
    cudaGetLastError();
    return set_err(BH_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  }
  s->walk_p = *p;
  s->walk_out = d_out;
  s->built = 0;  // nothing ran yet: the first replay builds
  return BH_OK;
}

int bh_system_replay(bh_system *s, void *stream) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (!s->graph) return set_err(BH_ERR_NOT_BUILT, "replay before capture");
  BH_CUDA(cudaSetDevice(s->device));
  BH_CUDA(cudaGraphLaunch(s->graph, (cudaStream_t)stream));
  s->built = 1;
  s->walked = 1;
  s->keys_checked = s->p.strict_keys ? 0 : 1;
  return BH_OK;
}

int bh_system_info(bh_system *s, int64_t *n, int *depth, int64_t *n_nodes, int64_t *n_groups,
                   double *com4, double *ssa) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (!s->built) return set_err(BH_ERR_NOT_BUILT, "info before build");
  BH_CUDA(cudaSetDevice(s->device));
  int rc = read_scalars(s, 0);
  if (rc) return rc;
  const bh::Scalars &h = *s->b.sc_host;
  bh::SysScalars s0;
  BH_CUDA(cudaMemcpy(&s0, s->b.ss, sizeof s0, cudaMemcpyDeviceToHost));
  if (n) *n = s->n;
  if (depth) *depth = h.L;
  if (n_nodes) *n_nodes = h.n_compact;
  if (n_groups) *n_groups = h.n_groups;
  if (com4) { com4[0] = s0.com[0]; com4[1] = s0.com[1]; com4[2] = s0.com[2]; com4[3] = s0.mass; }
  if (ssa) *ssa = s0.ssa;
  return BH_OK;
}

int bh_system_batch_info(bh_system *s, int32_t *roots, double *com4, double *ssa) {
  if (!s) return set_err(BH_ERR_INVALID, "sys is NULL");
  if (!s->built) return set_err(BH_ERR_NOT_BUILT, "info before build");
  BH_CUDA(cudaSetDevice(s->device));
  BH_CUDA(cudaDeviceSynchronize());
  std::vector<bh::SysScalars> h((size_t)s->nsys);
  BH_CUDA(cudaMemcpy(h.data(), s->b.ss, h.size() * sizeof(bh::SysScalars), cudaMemcpyDeviceToHost));
  for (int q = 0; q < s->nsys; ++q) {
    if (roots) roots[q] = h[q].root;
    if (com4)
      for (int k = 0; k < 3; ++k) com4[4 * q + k] = h[q].com[k];
    if (com4) com4[4 * q + 3] = h[q].mass;
    if (ssa) ssa[q] = h[q].ssa;
  }
  return BH_OK;
}

int bh_system_get_keys(bh_system *s, uint64_t *keys, int32_t *perm) {
  if (!s || !s->built) return set_err(BH_ERR_NOT_BUILT, "keys before build");
  BH_CUDA(cudaSetDevice(s->device));
  BH_CUDA(cudaDeviceSynchronize());
  if (keys) BH_CUDA(cudaMemcpy(keys, s->b.k0, s->n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (perm) BH_CUDA(cudaMemcpy(perm, s->b.v0, s->n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return BH_OK;
}

int bh_system_get_nodes(bh_system *s, int32_t *meta4, int32_t *child8, int32_t *parent,
                        double *com4, double *quad6, double *oct14, int32_t *level_begin) {
  if (!s || !s->built) return set_err(BH_ERR_NOT_BUILT, "nodes before build");
  BH_CUDA(cudaSetDevice(s->device));
  int rc = read_scalars(s, 0);
  if (rc) return rc;
  const int64_t M = s->b.sc_host->n_compact;
  const Buffers &b = s->b;
  if (M > 0) {
    if (meta4) BH_CUDA(cudaMemcpy(meta4, b.cn_meta, M * sizeof(int4), cudaMemcpyDeviceToHost));
    if (child8) BH_CUDA(cudaMemcpy(child8, b.cn_child, M * 8 * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (parent) BH_CUDA(cudaMemcpy(parent, b.cn_parent, M * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (com4) BH_CUDA(cudaMemcpy(com4, b.cn_com, M * sizeof(double4), cudaMemcpyDeviceToHost));
    if (quad6 && s->order >= 4) BH_CUDA(cudaMemcpy(quad6, b.cn_quad, M * 6 * sizeof(double), cudaMemcpyDeviceToHost));
    if (oct14 && s->order >= 8) BH_CUDA(cudaMemcpy(oct14, b.cn_oct, M * 14 * sizeof(double), cudaMemcpyDeviceToHost));
  }
  if (level_begin)
    BH_CUDA(cudaMemcpy(level_begin, b.level_begin, (s->b.sc_host->L + 2) * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return BH_OK;
}

int bh_system_get_groups(bh_system *s, int32_t *group_first) {
  if (!s || !s->built) return set_err(BH_ERR_NOT_BUILT, "groups before build");
  BH_CUDA(cudaSetDevice(s->device));
  int rc = read_scalars(s, 0);
  if (rc) return rc;
  if (group_first)
    BH_CUDA(cudaMemcpy(group_first, s->b.g_first, (s->b.sc_host->n_groups + 1) * sizeof(int32_t),
                       cudaMemcpyDeviceToHost));
  return BH_OK;
}

int bh_system_get_stats(bh_system *s, uint64_t *stats4) {
  if (!s || !stats4) return set_err(BH_ERR_INVALID, "NULL argument");
  BH_CUDA(cudaSetDevice(s->device));
  BH_CUDA(cudaDeviceSynchronize());
  BH_CUDA(cudaMemcpy(stats4, s->b.stats, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return BH_OK;
}

int bh_system_get_key_checks(bh_system *s, int64_t *checks2) {
  if (!s || !checks2) return set_err(BH_ERR_INVALID, "NULL argument");
  checks2[0] = s->key_checks;
  checks2[1] = s->key_rebuilds;
  return BH_OK;
}

int bh_system_reference_targets(bh_system *s, const bh_params *p, const int64_t *d_targets,
                                int64_t ntargets, double *d_out, int64_t *d_counts,
                                void *stream) {
  if (!s || !s->built) return set_err(BH_ERR_NOT_BUILT, "reference walk before build");
  int rc = check_params(p, s->n);
  if (rc) return rc;
  if (!d_targets || ntargets < 1 || !d_out) return set_err(BH_ERR_INVALID, "bad targets/output");
  if (p->order > s->order) return set_err(BH_ERR_INVALID, "order above the built order");
  BH_CUDA(cudaSetDevice(s->device));
  bh::WalkParams w = walk_params(p, s->order);
  bh::launch_reference_walk(s->n, w, s->b, d_out, d_targets, ntargets, d_counts,
                            (cudaStream_t)stream);
  BH_CUDA(cudaGetLastError());
  return BH_OK;
}

int bh_compute_forces_ex(const double *m, const double *x, const double *y, const double *z,
                         int64_t n, const bh_params *p, double *out, void *stream) {
  int rc = check_params(p, n);
  if (rc) return rc;
  if (!m || !x || !y || !z || !out) return set_err(BH_ERR_INVALID, "NULL array");
  std::lock_guard<std::mutex> lock(g_default_mu);
  bh_system *s = nullptr;
  rc = default_system(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const bh::HostKind ok = bh::host_kind(out);
  if (ok == bh::HostKind::kDevice)
    return set_err(BH_ERR_INVALID, "a device pointer was passed as the host result array");
  rc = stage_inputs(s, m, x, y, z, n, st);
  if (rc) return rc;
  Buffers &b = s->b;
  rc = bh_system_build(s, b.hm, b.hx, b.hy, b.hz, n, p, stream);
  if (rc) return rc;
  rc = bh_system_walk(s, p, b.hout, stream);
  if (rc) return rc;
  if (ok != bh::HostKind::kPinned) {
    // pageable result: the status first (it may redo the walk), then the
    // staged copy, which returns when the caller's array is written
    rc = finish(s, st);
    if (rc) return rc;
    rc = ensure_hostcopy(s);
    if (rc) return rc;
    BH_CUDA(bh::hostcopy_download(s->hcopy, out, b.hout, 3 * n, st));
    return BH_OK;
  }
  // the result's copy goes on the stream before the status is read, so it
  // follows the walk without a host round trip; if the status check redoes
  // the walk (strict-key rebuild, larger stack) the copy is made again
  const int64_t walks = s->walks_enqueued;
  BH_CUDA(cudaMemcpyAsync(out, b.hout, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
  rc = finish(s, st);
  if (rc) return rc;
  if (s->walks_enqueued != walks)
    BH_CUDA(cudaMemcpyAsync(out, b.hout, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
  BH_CUDA(cudaStreamSynchronize(st));
  return BH_OK;
}

int bh_compute_forces(const double *m, const double *x, const double *y, const double *z,
                      int64_t n, double theta, double G, double eps, int order, int out_kind,
                      double *out, void *stream) {
  bh_params p;
  bh_params_default(&p);
  p.theta = theta;
  p.G = G;
  p.eps = eps;
  p.order = order;
  p.out_kind = out_kind;
  return bh_compute_forces_ex(m, x, y, z, n, &p, out, stream);
}

int bh_compute_forces_direct(const double *m, const double *x, const double *y,
                             const double *z, int64_t n, double G, double eps, int out_kind,
                             double *out, void *stream) {
  if (n < 1 || n > (int64_t)(1 << 30)) return set_err(BH_ERR_INVALID, "n out of range");
  if (!m || !x || !y || !z || !out) return set_err(BH_ERR_INVALID, "NULL array");
  if (out_kind != 0 && out_kind != 1) return set_err(BH_ERR_INVALID, "out_kind must be 0 or 1");
  std::lock_guard<std::mutex> lock(g_default_mu);
  bh_system *s = nullptr;
  int rc = default_system(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const bh::HostKind ok = bh::host_kind(out);
  if (ok == bh::HostKind::kDevice)
    return set_err(BH_ERR_INVALID, "a device pointer was passed as the host result array");
  rc = stage_inputs(s, m, x, y, z, n, st);
  if (rc) return rc;
  Buffers &b = s->b;
  bh::launch_direct(b.hm, b.hx, b.hy, b.hz, n, nullptr, 0, G, eps * eps, out_kind, b.hout, st);
  BH_CUDA(cudaGetLastError());
  if (ok != bh::HostKind::kPinned) {
    rc = ensure_hostcopy(s);
    if (rc) return rc;
    BH_CUDA(bh::hostcopy_download(s->hcopy, out, b.hout, 3 * n, st));
    return BH_OK;
  }
  BH_CUDA(cudaMemcpyAsync(out, b.hout, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
  BH_CUDA(cudaStreamSynchronize(st));
  return BH_OK;
}

int bh_direct_targets_device(const double *d_m, const double *d_x, const double *d_y,
                             const double *d_z, int64_t n, const int64_t *d_targets,
                             int64_t ntargets, double G, double eps, int out_kind, double *d_out,
                             void *stream) {
  if (n < 1) return set_err(BH_ERR_INVALID, "n must be >= 1");
  if (!d_m || !d_x || !d_y || !d_z || !d_out) return set_err(BH_ERR_INVALID, "NULL array");
  if (d_targets && ntargets < 1) return set_err(BH_ERR_INVALID, "ntargets must be >= 1");
  if (out_kind != 0 && out_kind != 1) return set_err(BH_ERR_INVALID, "out_kind must be 0 or 1");
  bh::launch_direct(d_m, d_x, d_y, d_z, n, d_targets, ntargets, G, eps * eps, out_kind, d_out,
                    (cudaStream_t)stream);
  BH_CUDA(cudaGetLastError());
  return BH_OK;
}

int bh_probe_bounded_wait(int device, long long cycles, long long *out5) {
  if (!out5) return set_err(BH_ERR_INVALID, "NULL output");
  if (cycles < 1000 || cycles > 1000000000LL)
    return set_err(BH_ERR_INVALID, "cycles must be in [1e3, 1e9]");
  BH_CUDA(cudaSetDevice(device));
  if (bh::probe_bounded_wait(cycles, out5)) return set_err(BH_ERR_CUDA, "wait probe failed");
  return BH_OK;
}

int bh_probe_fma_peak(int device, double *gflops2) {
  if (!gflops2) return set_err(BH_ERR_INVALID, "NULL output");
  BH_CUDA(cudaSetDevice(device));
  if (bh::probe_fma(gflops2)) return set_err(BH_ERR_CUDA, "probe failed");
  return BH_OK;
}

}  // extern "C"
