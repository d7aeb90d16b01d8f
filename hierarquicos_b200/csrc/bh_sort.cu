// Stable LSD radix sort of (64-bit key, 32-bit value) pairs, a device-wide
// exclusive scan, and the gather of particles into key order.
//
// Replaces the stable recursive merge sort of fortran/morton/morton_octree.f90
// :501-560 (argsort).  An LSD radix sort whose every pass is stable produces
// exactly the stable sort's permutation: equal keys keep ascending original
// index, as the merge sort's "ties take the left element" rule (:537-538).
//
// Each pass (8-bit digit): an upsweep counts digits per 4096-key tile, one
// exclusive scan over the digit-major count table gives every (digit, tile)
// its output base, and a downsweep ranks keys inside the tile with warp
// __match_any_sync / popc ranking (element order = warp, iteration, lane, so
// ranks are stable), stages the tile in shared memory in digit order and
// writes it out so that runs of equal digits land on consecutive addresses.
// No pass waits on another block: there is no spin wait anywhere.
#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;
constexpr int kItems = 16;
constexpr int kTile = kSortThreads * kItems;  // 4096 keys per block
constexpr int kRadix = 256;

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

__global__ void __launch_bounds__(kSortThreads)
upsweep_kernel(const uint64_t *__restrict__ keys, int64_t n_max, const int32_t *n_dev, int shift,
               int32_t *__restrict__ hist, int nblocks) {
  __shared__ int wh[kSortWarps][kRadix];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&wh[0][0])[i] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile + warp * kWarp * kItems;
#pragma unroll 4
  for (int i = 0; i < kItems; ++i) {
    int64_t idx = base + i * kWarp + lane;
    if (idx < n) atomicAdd(&wh[warp][(int)((keys[idx] >> shift) & 0xff)], 1);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
    int s = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s += wh[w][d];
    hist[(int64_t)d * nblocks + blockIdx.x] = s;
  }
}

struct DownSmem {
  uint64_t sk[kTile];
  int32_t sv[kTile];
  int wh[kSortWarps][kRadix];
  int tile_start[kRadix];
  int gbase[kRadix];
  int ws[kSortWarps];
};

__global__ void __launch_bounds__(kSortThreads)
downsweep_kernel(const uint64_t *__restrict__ kin, const int32_t *__restrict__ vin,
                 uint64_t *__restrict__ kout, int32_t *__restrict__ vout, int64_t n_max,
                 const int32_t *n_dev, int shift, const int32_t *__restrict__ hist, int nblocks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DownSmem &S = *reinterpret_cast<DownSmem *>(smem_raw);
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  const int64_t tile_base = (int64_t)blockIdx.x * kTile;
  if (tile_base >= n) return;  // uniform across the block
  const int tile_n = (int)bh_min64(kTile, n - tile_base);

  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&S.wh[0][0])[i] = 0;
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
    S.gbase[d] = hist[(int64_t)d * nblocks + blockIdx.x];
  __syncthreads();

  uint64_t k[kItems];
  int32_t v[kItems];
  int dig[kItems], rank[kItems];
  const int wbase = warp * kWarp * kItems;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    int li = wbase + i * kWarp + lane;
    bool valid = li < tile_n;
    k[i] = valid ? kin[tile_base + li] : 0ull;
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
  // per digit: exclusive offsets of the warps, tile count
  int cnt = 0;
  {
    const int d = threadIdx.x;  // kSortThreads == kRadix
    int run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      int c = S.wh[w][d];
      S.wh[w][d] = run;
      run += c;
    }
    cnt = run;
  }
  int start = block_excl_scan(cnt, S.ws, nullptr);
  S.tile_start[threadIdx.x] = start;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const int d = dig[i];
    if (d < kRadix) {
      int pos = S.tile_start[d] + S.wh[warp][d] + rank[i];
      S.sk[pos] = k[i];
      S.sv[pos] = v[i];
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
    uint64_t key = S.sk[j];
    int d = (int)((key >> shift) & 0xff);
    int64_t o = (int64_t)S.gbase[d] + (j - S.tile_start[d]);
    kout[o] = key;
    vout[o] = S.sv[j];
  }
}

// ---- exclusive scan ----

__global__ void __launch_bounds__(kScanThreads)
scan_reduce_kernel(const int32_t *__restrict__ in, int64_t n_max, const int32_t *n_dev,
                   int32_t *__restrict__ block_sums) {
  __shared__ int ws[kScanThreads / kWarp];
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) s += in[base + i];
  int total;
  block_excl_scan(s, ws, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
scan_blocks_kernel(int32_t *block_sums, int nb, int32_t *total_out) {
  __shared__ int ws[kScanThreads / kWarp];
  int carry = 0;
  for (int base = 0; base < nb; base += kScanThreads) {
    int i = base + threadIdx.x;
    int v = i < nb ? block_sums[i] : 0;
    int tot;
    int ex = block_excl_scan(v, ws, &tot);
    if (i < nb) block_sums[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) {
    block_sums[nb] = carry;
    if (total_out) *total_out = carry;
  }
}

__global__ void __launch_bounds__(kScanThreads)
scan_apply_kernel(const int32_t *in, int32_t *out, int64_t n_max, const int32_t *n_dev,
                  const int32_t *__restrict__ block_sums) {
  __shared__ int ws[kScanThreads / kWarp];
  const int64_t n = n_dev ? bh_min64(n_max, (int64_t)*n_dev) : n_max;
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanItems;
  int vals[kScanItems];
  int s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = (base + i < n) ? in[base + i] : 0;
    s += vals[i];
  }
  int off = block_excl_scan(s, ws, nullptr) + block_sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = off;
    off += vals[i];
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

bool g_sort_attr_set = false;

}  // namespace

static_assert(kScanChunk == 8192 && kTile == 4096 && kRadix == 256,
              "scan_tmp_entries / radix_hist_entries in bh_internal.cuh assume these sizes");

void exclusive_scan(const int32_t *in, int32_t *out, int64_t n, const int32_t *n_dev,
                    int32_t *total, int32_t *tmp, cudaStream_t s) {
  int nb = (int)((n + kScanChunk - 1) / kScanChunk);
  if (nb < 1) nb = 1;
  scan_reduce_kernel<<<nb, kScanThreads, 0, s>>>(in, n, n_dev, tmp);
  scan_blocks_kernel<<<1, kScanThreads, 0, s>>>(tmp, nb, total);
  scan_apply_kernel<<<nb, kScanThreads, 0, s>>>(in, out, n, n_dev, tmp);
}

void radix_sort_pairs(uint64_t *k0, int32_t *v0, uint64_t *k1, int32_t *v1, int64_t n,
                      const int32_t *n_dev, int bits, int32_t *hist, cudaStream_t s) {
  if (!g_sort_attr_set) {
    cudaFuncSetAttribute(downsweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(DownSmem));
    g_sort_attr_set = true;
  }
  const int nblocks = (int)((n + kTile - 1) / kTile);
  const int64_t entries = (int64_t)kRadix * nblocks;
  // the scan's block sums live after the count table
  int32_t *scan_tmp = hist + entries + 1;
  int passes = (bits + 7) / 8;
  uint64_t *ki = k0, *ko = k1;
  int32_t *vi = v0, *vo = v1;
  for (int p = 0; p < passes; ++p) {
    int shift = 8 * p;
    upsweep_kernel<<<nblocks, kSortThreads, 0, s>>>(ki, n, n_dev, shift, hist, nblocks);
    exclusive_scan(hist, hist, entries, nullptr, nullptr, scan_tmp, s);
    downsweep_kernel<<<nblocks, kSortThreads, sizeof(DownSmem), s>>>(ki, vi, ko, vo, n, n_dev,
                                                                      shift, hist, nblocks);
    uint64_t *tk = ki; ki = ko; ko = tk;
    int32_t *tv = vi; vi = vo; vo = tv;
  }
  if (ki != k0) {
    // odd number of passes: the result sits in the second buffer
    cudaMemcpyAsync(k0, ki, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(v0, vi, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
  }
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
  radix_sort_pairs(ck0, cv0, ck1, cv1, n, nullptr, bits, b.hist, s);
  regather_kernel<<<grid, 256, 0, s>>>(b.k0, b.v0, cv0, n, b.k1, b.v1);
  cudaMemcpyAsync(b.k0, b.k1, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(b.v0, b.v1, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
}

void launch_gather(const double *m, const double *x, const double *y, const double *z, int64_t n,
                   Buffers &b, cudaStream_t s) {
  gather_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(m, x, y, z, b.v0, n, b.spos);
}

}  // namespace bh
