// Stable LSD radix sort of (64-bit key, 32-bit value) pairs, a device-wide
// exclusive scan, and the gather of particles into key order.
//
// Replaces the stable recursive merge sort of fortran/morton/morton_octree.f90
// :501-560 (argsort).  An LSD radix sort whose every pass is stable produces
// exactly the stable sort's permutation: equal keys keep ascending original
// index, as the merge sort's "ties take the left element" rule (:537-538).
//
// Digit counts of every pass come from one histogram kernel over the keys;
// each pass (8-bit digit) is then ONE kernel with decoupled look-back: a block
// claims the next tile (4096 keys; 1024 for sorts of at most 65,536 keys, whose
// few large tiles would leave most SMs idle) from an atomic counter, ranks its keys inside
// the tile with warp __match_any_sync / popc ranking (element order = warp,
// iteration, lane, so ranks are stable), publishes its per-digit counts, adds
// up the counts of the tiles before it (each tile's word holds either its own
// count or, once known, the inclusive prefix of all tiles up to it), stages
// the tile in shared memory in digit order and writes it out so that runs of
// equal digits land on consecutive addresses.  A block only waits for tiles
// claimed before its own, by blocks that are already running; every wait is
// bounded and a wait that gives up raises an error flag instead of hanging.
#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;
constexpr int kItems = 16;       // keys per thread of a large sort's tile
constexpr int kSmallItems = kSortTileSmall / 256;  // and of a small sort's
constexpr int kTile = kSortThreads * kItems;  // 4096 keys per block (large sorts)
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;  // 64-bit keys

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & (kWarp - 1);
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Exclusive scan of one value per thread across the block; `ws` needs
// blockDim/32 ints.  Ends with a barrier so `ws` may be reused.
__device__ int block_excl_scan(int v, int *ws, int *total) {
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const int nwarps = blockDim.x / kWarp;
  int incl = warp_incl_scan(v);
  if (lane == kWarp - 1) ws[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int s = lane < nwarps ? ws[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < nwarps) ws[lane] = s;
  }
  __syncthreads();
  int off = warp > 0 ? ws[warp - 1] : 0;
  if (total) *total = ws[nwarps - 1];
  __syncthreads();
  return off + incl - v;
}

// Digit histograms of all passes: ghist[p][d] = number of keys whose digit p
// is d (warp-aggregated shared-memory counts, then one global add per bin).
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
digit_hist_kernel(const K *__restrict__ keys, int64_t n_max, const int32_t *n_dev,
                  int passes, uint32_t *__restrict__ ghist) {
  __shared__ uint32_t h[kMaxPasses][kRadix];
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const unsigned lt = lanemask_lt();
  const int64_t stride = (int64_t)gridDim.x * kSortThreads;
  for (int64_t base = (int64_t)blockIdx.x * kSortThreads; base < n; base += stride) {
    const int64_t idx = base + threadIdx.x;
    const bool valid = idx < n;
    const K k = valid ? keys[idx] : (K)0;
    for (int p = 0; p < passes; ++p) {
      const int d = valid ? (int)((k >> (8 * p)) & 0xff) : kRadix;
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      if (d < kRadix && (peers & lt) == 0) atomicAdd(&h[p][d], (uint32_t)__popc(peers));
    }
    (void)lane;
  }
  __syncthreads();
  for (int p = 0; p < passes; ++p) {
    const uint32_t c = h[p][threadIdx.x];  // kSortThreads == kRadix
    if (c) atomicAdd(&ghist[p * kRadix + threadIdx.x], c);
  }
}

// The same digit counts from the number of keys of every key value v (keys are
// the values 0..n_values-1): pass p's count of digit d sums count[v] over the
// values whose digit p is d -- one read of the counts instead of all keys.
__global__ void __launch_bounds__(kSortThreads)
count_hist_kernel(const int32_t *__restrict__ count, int64_t n_values, int passes,
                  uint32_t *__restrict__ ghist) {
  __shared__ uint32_t h[kMaxPasses][kRadix];
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t v = (int64_t)blockIdx.x * kSortThreads + threadIdx.x; v < n_values;
       v += (int64_t)gridDim.x * kSortThreads) {
    const uint32_t c = (uint32_t)count[v];
    if (c == 0) continue;
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(v >> (8 * p)) & 0xff], c);
  }
  __syncthreads();
  for (int p = 0; p < passes; ++p) {
    const uint32_t c = h[p][threadIdx.x];  // kSortThreads == kRadix
    if (c) atomicAdd(&ghist[p * kRadix + threadIdx.x], c);
  }
}

// Exclusive scan of each pass's 256 digit counts, in place.
__global__ void __launch_bounds__(kSortThreads) digit_scan_kernel(uint32_t *ghist, int passes) {
  __shared__ int ws[kSortWarps];
  for (int p = 0; p < passes; ++p) {
    const int v = (int)ghist[p * kRadix + threadIdx.x];
    const int ex = block_excl_scan(v, ws, nullptr);
    ghist[p * kRadix + threadIdx.x] = (uint32_t)ex;
  }
}

// tile words: top 2 bits the state, low 62 bits the count
constexpr uint64_t kTileAggregate = 1ull << 62;  // the tile's own count
constexpr uint64_t kTileInclusive = 2ull << 62;  // sum of the counts of tiles 0..t
constexpr uint64_t kTileValue = (1ull << 62) - 1;
constexpr int64_t kLookbackSpins = 1 << 22;     // per word; about a second at most

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

template <typename K, int ITEMS>
struct PassSmem {
  K sk[ITEMS * kSortThreads];
  int32_t sv[ITEMS * kSortThreads];
  int wh[kSortWarps][kRadix];
  int tile_start[kRadix];
  int gbase[kRadix];
  int ws[kSortWarps];
  int tile;
};

// kout may be null: the pass then writes only the values (a last pass whose
// keys nobody reads).
// 3 blocks per SM (80 registers, no spills; the compiler's own choice was 128
// and 2 blocks): the 181 M-term sort of Dehnen's method 1 ms faster.
template <typename K, int ITEMS>
__global__ void __launch_bounds__(kSortThreads, 3)
onesweep_kernel(const K *__restrict__ kin, const int32_t *__restrict__ vin,
                K *__restrict__ kout, int32_t *__restrict__ vout, int64_t n_max,
                const int32_t *n_dev, int shift, const uint32_t *__restrict__ gofs,
                uint64_t *__restrict__ tiles, int32_t *__restrict__ tile_ctr, int *err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PassSmem<K, ITEMS> &S = *reinterpret_cast<PassSmem<K, ITEMS> *>(smem_raw);
  constexpr int kItems = ITEMS;
  constexpr int kTile = ITEMS * kSortThreads;
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  if (threadIdx.x == 0) S.tile = atomicAdd(tile_ctr, 1);
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&S.wh[0][0])[i] = 0;
  __syncthreads();
  const int t = S.tile;
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  const int64_t tile_base = (int64_t)t * kTile;
  if (tile_base >= n) return;  // uniform across the block; later tiles return too
  const int tile_n = (int)bh_min64(kTile, n - tile_base);

  K k[kItems];
  int32_t v[kItems];
  int dig[kItems], rank[kItems];
  const int wbase = warp * kWarp * kItems;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    int li = wbase + i * kWarp + lane;
    bool valid = li < tile_n;
    k[i] = valid ? kin[tile_base + li] : (K)0;
    v[i] = valid ? vin[tile_base + li] : 0;
    dig[i] = valid ? (int)((k[i] >> shift) & 0xff) : kRadix;
  }
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const int d = dig[i];
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rin = __popc(peers & lt);
    const int pre = d < kRadix ? S.wh[warp][d] : 0;
    __syncwarp();
    if (d < kRadix && rin == 0) S.wh[warp][d] = pre + __popc(peers);
    __syncwarp();
    rank[i] = pre + rin;
  }
  __syncthreads();
  // per digit (thread d): exclusive offsets of the warps and the tile's count
  const int d = threadIdx.x;  // kSortThreads == kRadix
  int cnt = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const int c = S.wh[w][d];
    S.wh[w][d] = cnt;
    cnt += c;
  }
  // publish, then look back over the earlier tiles for this digit
  uint64_t *word = tiles + (int64_t)t * kRadix + d;
  int64_t excl = 0;
  if (t == 0) {
    st_relaxed(word, kTileInclusive | (uint64_t)cnt);
  } else {
    st_relaxed(word, kTileAggregate | (uint64_t)cnt);
    int j = t - 1;
    int64_t spins = 0;
    while (j >= 0) {
      const uint64_t w = ld_relaxed(tiles + (int64_t)j * kRadix + d);
      if ((w & ~kTileValue) == 0) {
        if (++spins > kLookbackSpins) { atomicOr(err, kErrTimeout); break; }
        continue;
      }
      excl += (int64_t)(w & kTileValue);
      if ((w & ~kTileValue) == kTileInclusive) break;
      --j;
    }
    st_relaxed(word, kTileInclusive | (uint64_t)(excl + cnt));
  }
  S.gbase[d] = (int)(gofs[d] + excl);
  int start = block_excl_scan(cnt, S.ws, nullptr);
  S.tile_start[d] = start;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const int dd = dig[i];
    if (dd < kRadix) {
      int pos = S.tile_start[dd] + S.wh[warp][dd] + rank[i];
      S.sk[pos] = k[i];
      S.sv[pos] = v[i];
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
    const K key = S.sk[j];
    const int dd = (int)((key >> shift) & 0xff);
    const int64_t o = (int64_t)S.gbase[dd] + (j - S.tile_start[dd]);
    if (kout) kout[o] = key;
    vout[o] = S.sv[j];
  }
}

// ---- exclusive scan ----

// Single-pass exclusive scan (chained scan with decoupled look-back): block b
// claims tile t (kScanChunk values) from a ticket, sums it, publishes the sum,
// adds up the earlier tiles' words (an inclusive word ends the walk), then
// writes its outputs.  A block only waits for tiles claimed before its own by
// blocks that are running and publish before they wait; every wait is
// bounded and one that gives up raises kErrTimeout in *err.
// tmp (int32 entries): [0] ticket, [1] unused, then one 64-bit word per tile.
__global__ void __launch_bounds__(kScanThreads)
scan_onepass_kernel(const int32_t *__restrict__ in, int32_t *__restrict__ out, int64_t n_max,
                    const int32_t *n_dev, int32_t *tmp, int32_t *total_out, int32_t *total_out2,
                    int *err) {
  __shared__ int ws[kScanThreads / kWarp];
  __shared__ int s_tile;
  __shared__ int64_t s_excl;
  if (threadIdx.x == 0) s_tile = atomicAdd(tmp, 1);
  __syncthreads();
  const int t = s_tile;
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  const int64_t ntiles = n > 0 ? (n + kScanChunk - 1) / kScanChunk : 1;
  if ((int64_t)t >= ntiles) return;  // uniform across the block
  uint64_t *words = reinterpret_cast<uint64_t *>(tmp + 2);
  const int64_t base = (int64_t)t * kScanChunk + (int64_t)threadIdx.x * kScanItems;
  int vals[kScanItems];
  int sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = (base + i < n) ? in[base + i] : 0;
    sum += vals[i];
  }
  int tile_total;
  int off = block_excl_scan(sum, ws, &tile_total);
  if (threadIdx.x == 0) {
    int64_t excl = 0;
    if (t == 0) {
      st_relaxed(words, kTileInclusive | (uint64_t)tile_total);
    } else {
      st_relaxed(words + t, kTileAggregate | (uint64_t)tile_total);
      int j = t - 1;
      int64_t spins = 0;
      while (j >= 0) {
        const uint64_t w = ld_relaxed(words + j);
        if ((w & ~kTileValue) == 0) {
          if (++spins > kLookbackSpins) { atomicOr(err, kErrTimeout); break; }
          continue;
        }
        excl += (int64_t)(w & kTileValue);
        if ((w & ~kTileValue) == kTileInclusive) break;
        --j;
      }
      st_relaxed(words + t, kTileInclusive | (uint64_t)(excl + tile_total));
    }
    s_excl = excl;
    if ((int64_t)t == ntiles - 1) {
      if (total_out) *total_out = (int32_t)(excl + tile_total);
      if (total_out2) *total_out2 = (int32_t)(excl + tile_total);
    }
  }
  __syncthreads();
  int64_t o = s_excl + off;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = (int32_t)o;
    o += vals[i];
  }
}

__global__ void __launch_bounds__(256)
gather_kernel(const double *__restrict__ m, const double *__restrict__ x,
              const double *__restrict__ y, const double *__restrict__ z,
              const int32_t *__restrict__ perm, int64_t n, double4 *__restrict__ spos) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int32_t p = perm[i];
    spos[i] = make_double4(x[p], y[p], z[p], m[p]);
  }
}

// stage 2 of a batch sort: key = system of the body at sorted position i
__global__ void __launch_bounds__(256)
sys_keys_kernel(const int32_t *__restrict__ perm, const int32_t *__restrict__ sys_of, int64_t n,
                uint64_t *__restrict__ ck, int32_t *__restrict__ cv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    ck[i] = (uint64_t)sys_of[perm[i]];
    cv[i] = (int32_t)i;
  }
}

__global__ void __launch_bounds__(256)
regather_kernel(const uint64_t *__restrict__ k0, const int32_t *__restrict__ v0,
                const int32_t *__restrict__ order, int64_t n, uint64_t *__restrict__ k1,
                int32_t *__restrict__ v1) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t j = order[i];
    k1[i] = k0[j];
    v1[i] = v0[j];
  }
}

template <typename K, int ITEMS>
void set_pass_smem() {
  static bool done = false;  // a function attribute: once per process
  if (!done) {
    cudaFuncSetAttribute(onesweep_kernel<K, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PassSmem<K, ITEMS>));
    done = true;
  }
}

template <typename K, int ITEMS>
void launch_pass(int64_t ntiles, const K *ki, const int32_t *vi, K *ko, int32_t *vo, int64_t n,
                 const int32_t *n_dev, int shift, const uint32_t *gofs, uint64_t *tiles,
                 int32_t *ctr, int *err, cudaStream_t s) {
  set_pass_smem<K, ITEMS>();
  onesweep_kernel<K, ITEMS><<<(unsigned)(ntiles > 0 ? ntiles : 1), kSortThreads,
                              sizeof(PassSmem<K, ITEMS>), s>>>(ki, vi, ko, vo, n, n_dev, shift,
                                                               gofs, tiles, ctr, err);
}

}  // namespace

static_assert(kScanChunk == 8192 && kTile == kSortTileLarge && kRadix == 256 && kMaxPasses == 8 &&
                  kSortThreads * kSmallItems == kSortTileSmall,
              "scan_tmp_entries / radix_hist_entries in bh_internal.cuh assume these sizes");

void exclusive_scan(const int32_t *in, int32_t *out, int64_t n, const int32_t *n_dev,
                    int32_t *total, int32_t *tmp, int *err, cudaStream_t s, int32_t *total2) {
  int nb = (int)((n + kScanChunk - 1) / kScanChunk);
  if (nb < 1) nb = 1;
  cudaMemsetAsync(tmp, 0, (2 + 2 * (int64_t)nb) * sizeof(int32_t), s);
  scan_onepass_kernel<<<nb, kScanThreads, 0, s>>>(in, out, n, n_dev, tmp, total, total2, err);
}

// The passes of one sort; returns the buffer (0: k0/v0, 1: k1/v1) that holds
// the result.  With keys_out false the last pass writes only the values.
template <typename K>
static int sort_passes(K *k0, int32_t *v0, K *k1, int32_t *v1, int64_t n, const int32_t *n_dev,
                       int bits, int32_t *hist, int *err, bool keys_out, cudaStream_t s,
                       const int32_t *key_counts = nullptr, int64_t n_key_values = 0) {
  // small sorts take small tiles: more blocks in flight for the same keys
  const int64_t tile = sort_tile(n);
  const int64_t ntiles = (n + tile - 1) / tile;
  int passes = (bits + 7) / 8;
  if (passes < 1) passes = 1;
  if (passes > (int)sizeof(K)) passes = (int)sizeof(K);
  // scratch layout (int32 entries): digit counts [8][256], tile counters [8],
  // then the tile words (uint64) [passes][ntiles][256]
  uint32_t *ghist = reinterpret_cast<uint32_t *>(hist);
  int32_t *ctr = hist + kMaxPasses * kRadix;
  uint64_t *tiles = reinterpret_cast<uint64_t *>(hist + kMaxPasses * kRadix + kMaxPasses);
  const int64_t used = kMaxPasses * kRadix + kMaxPasses + 2 * (int64_t)passes * ntiles * kRadix;
  cudaMemsetAsync(hist, 0, used * sizeof(int32_t), s);
  if (key_counts)
    count_hist_kernel<<<grid_for(n_key_values, kSortThreads, 148 * 8), kSortThreads, 0, s>>>(
        key_counts, n_key_values, passes, ghist);
  else
    digit_hist_kernel<K><<<grid_for(n, kSortThreads, 148 * 8), kSortThreads, 0, s>>>(k0, n, n_dev,
                                                                                     passes, ghist);
  digit_scan_kernel<<<1, kSortThreads, 0, s>>>(ghist, passes);
  K *ki = k0, *ko = k1;
  int32_t *vi = v0, *vo = v1;
  for (int p = 0; p < passes; ++p) {
    K *kw = (p == passes - 1 && !keys_out) ? nullptr : ko;
    if (tile == kSortTileSmall)
      launch_pass<K, kSmallItems>(ntiles, ki, vi, kw, vo, n, n_dev, 8 * p, ghist + p * kRadix,
                                  tiles + (int64_t)p * ntiles * kRadix, ctr + p, err, s);
    else
      launch_pass<K, kItems>(ntiles, ki, vi, kw, vo, n, n_dev, 8 * p, ghist + p * kRadix,
                             tiles + (int64_t)p * ntiles * kRadix, ctr + p, err, s);
    K *tk = ki; ki = ko; ko = tk;
    int32_t *tv = vi; vi = vo; vo = tv;
  }
  return ki == k0 ? 0 : 1;
}

void radix_sort_pairs(uint64_t *k0, int32_t *v0, uint64_t *k1, int32_t *v1, int64_t n,
                      const int32_t *n_dev, int bits, int32_t *hist, int *err, cudaStream_t s) {
  if (sort_passes<uint64_t>(k0, v0, k1, v1, n, n_dev, bits, hist, err, true, s) == 1) {
    // odd number of passes: the result sits in the second buffer
    cudaMemcpyAsync(k0, k1, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(v0, v1, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
  }
}

int radix_sort_values32(uint32_t *k0, int32_t *v0, uint32_t *k1, int32_t *v1, int64_t n, int bits,
                        int32_t *hist, int *err, cudaStream_t s, const int32_t *key_counts,
                        int64_t n_key_values) {
  return sort_passes<uint32_t>(k0, v0, k1, v1, n, nullptr, bits, hist, err, false, s, key_counts,
                               n_key_values);
}

// The key sort orders all bodies of a batch by key; a stable sort by system
// then restores the systems' ranges with each range in key order (LSD order:
// the system is the most significant part of the (system, key) pair).
void launch_sort_by_system(int64_t n, Buffers &b, cudaStream_t s) {
  if (b.nsys < 2) return;
  int bits = 1;
  while ((1 << bits) < b.nsys) ++bits;
  uint64_t *ck0 = reinterpret_cast<uint64_t *>(b.cn_quad);       // scratch until the upward pass
  uint64_t *ck1 = reinterpret_cast<uint64_t *>(b.cn_quad) + b.cap;
  int32_t *cv0 = b.cn_parent;                                    // scratch until the records
  int32_t *cv1 = b.bn_flag;                                      // scratch until the marks
  const int grid = grid_for(n, 256, 148 * 16);
  sys_keys_kernel<<<grid, 256, 0, s>>>(b.v0, b.sys_of, n, ck0, cv0);
  radix_sort_pairs(ck0, cv0, ck1, cv1, n, nullptr, bits, b.hist, &b.sc->err, s);
  regather_kernel<<<grid, 256, 0, s>>>(b.k0, b.v0, cv0, n, b.k1, b.v1);
  cudaMemcpyAsync(b.k0, b.k1, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(b.v0, b.v1, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
}

void launch_gather(const double *m, const double *x, const double *y, const double *z, int64_t n,
                   Buffers &b, cudaStream_t s) {
  gather_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(m, x, y, z, b.v0, n, b.spos);
}

}  // namespace bh
