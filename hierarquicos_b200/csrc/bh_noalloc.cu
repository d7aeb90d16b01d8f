// bh_compute_forces_noalloc: the force pipeline without any device allocation.
//
// Who needs it: a caller whose device memory is not its own to allocate.  A
// host program whose framework keeps its own pool of device memory (and may
// already hold nearly all of it), a solver that calls the force routine from
// a time-step loop where a cudaMalloc -- which can synchronise the whole
// device -- would stall other work, or a plugin host that forbids its plugins
// to allocate.  Such a caller passes device inputs and a device output and
// gets forces back; every other byte the pipeline needs comes from one
// file-scope device array of fixed size defined here.
//
// Limits and behaviour:
//  * at most BH_NOALLOC_MAX_N bodies (8192); larger n is rejected with
//    BH_ERR_INVALID and a message;
//  * the array (about 7.9 MB) lives on every device on which this library's
//    module holding it is loaded, until the process exits;
//  * the first call on a device looks the array's device address up
//    (cudaGetSymbolAddress, with that device current) and keeps it; later
//    calls on that device reuse it;
//  * every call synchronises its stream (it reads the status back before
//    returning), so it cannot be part of a stream capture: a call on a
//    capturing stream is refused with BH_ERR_INVALID before anything is
//    queued;
//  * all calls on a device share the one array, which keeps the last call's
//    contents; every call initialises what it reads.  Calls that overlap on
//    the GPU (other streams, other host threads) race on that array: issue
//    them one after another.  Host threads are serialised by a lock, but work
//    already queued on the GPU is not.
//  * the walk stacks are fixed, with room for every node of the largest tree
//    (kMaxN entries per walking warp), so a walk never runs out of stack at
//    any theta; the stacks are about 4 MB of the array.
// The results are those of bh_system_forces on the same inputs and
// parameters, bit for bit: the same kernels run in the same order.
#include <stdio.h>

#include <mutex>
#include <type_traits>

#include "bh_internal.cuh"

namespace {

constexpr int64_t kMaxN = BH_NOALLOC_MAX_N;
constexpr int64_t kSlots = 128;       // walk stacks: at most 128 walking warps (128 one-warp
                                      // blocks, or 32 blocks of 4 producer warps), as many as
                                      // there are 64-body groups in kMaxN bodies
constexpr int64_t kStackCap = kMaxN;  // stack entries per warp: a group's walk pushes every
                                      // node at most once and a tree of n bodies has fewer
                                      // than n nodes, so the stack cannot overflow
constexpr int64_t kItems = (kMaxN + bh::kRedChunk - 1) / bh::kRedChunk;  // reduction items
constexpr int kNumBufs = 36;

constexpr int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

// Byte size of every workspace array, in carving order (see carve()).
struct Sizes {
  int64_t v[kNumBufs];
};
constexpr Sizes buffer_bytes(int64_t c) {
  Sizes z{};
  int i = 0;
  z.v[i++] = 8 * c;                                   // k0
  z.v[i++] = 8 * c;                                   // k1
  z.v[i++] = 4 * c;                                   // v0
  z.v[i++] = 4 * c;                                   // v1
  z.v[i++] = 4 * bh::radix_hist_entries(c);           // hist
  z.v[i++] = 8 * 10 * kItems;                         // partials
  z.v[i++] = (int64_t)sizeof(bh::SysScalars);          // ss (one system)
  z.v[i++] = 4 * c;                                   // sys_of
  z.v[i++] = (int64_t)sizeof(bh::RedItem) * kItems;    // items
  z.v[i++] = 32 * c;                                  // spos
  for (int k = 0; k < 8; ++k) z.v[i++] = 4 * c;       // bn_* and bin2cn
  z.v[i++] = 4 * c;                                   // cn_bin
  z.v[i++] = 16 * c;                                  // cn_meta
  z.v[i++] = 32 * c;                                  // cn_child
  z.v[i++] = 4 * c;                                   // cn_parent
  z.v[i++] = 32 * c;                                  // cn_com
  z.v[i++] = 48 * c;                                  // cn_quad
  z.v[i++] = 112 * c;                                 // cn_oct
  z.v[i++] = 32 * c;                                  // cn_fq
  z.v[i++] = 64 * c;                                  // cn_fo
  z.v[i++] = 4 * (bh::kNumLevels + 2);                // level_begin
  z.v[i++] = 4 * (c + 1);                             // gflag
  z.v[i++] = 4 * (c + 1);                             // gscan
  z.v[i++] = 4 * (c + 1);                             // g_first
  z.v[i++] = 4 * bh::scan_tmp_entries(c + 1);         // scan_tmp
  z.v[i++] = 4 * kSlots * kStackCap;                  // wstack
  z.v[i++] = 32;                                      // counters
  z.v[i++] = 32;                                      // stats
  z.v[i++] = (int64_t)sizeof(bh::Scalars);            // sc
  return z;
}
constexpr int64_t total_bytes(int64_t c) {
  const Sizes z = buffer_bytes(c);
  int64_t t = 0;
  for (int i = 0; i < kNumBufs; ++i) t += align256(z.v[i]);
  return t;
}
constexpr int64_t kScratchBytes = total_bytes(kMaxN);
static_assert(kScratchBytes < 8 * 1024 * 1024, "keep the static workspace modest");

// The workspace.  In host code this name is only a stand-in for the device
// array; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

bh::Buffers carve(unsigned char *base) {
  const Sizes z = buffer_bytes(kMaxN);
  int64_t off = 0;
  int i = 0;
  auto take = [&](auto *&ptr) {
    ptr = reinterpret_cast<std::remove_reference_t<decltype(ptr)>>(base + off);
    off += align256(z.v[i++]);
  };
  bh::Buffers b;
  take(b.k0); take(b.k1); take(b.v0); take(b.v1); take(b.hist); take(b.partials); take(b.ss);
  take(b.sys_of); take(b.items); take(b.spos);
  take(b.bn_left); take(b.bn_right); take(b.bn_parent); take(b.bn_first); take(b.bn_last);
  take(b.bn_level); take(b.bn_flag); take(b.bin2cn);
  take(b.cn_bin); take(b.cn_meta); take(b.cn_child); take(b.cn_parent); take(b.cn_com);
  take(b.cn_quad); take(b.cn_oct); take(b.cn_fq); take(b.cn_fo); take(b.level_begin);
  take(b.gflag); take(b.gscan); take(b.g_first); take(b.scan_tmp); take(b.wstack);
  take(b.counters); take(b.stats); take(b.sc);
  b.cap = kMaxN;
  b.sys_cap = 1;
  b.items_cap = (int)kItems;
  b.hist_cap = bh::radix_hist_entries(kMaxN);
  b.scan_tmp_cap = bh::scan_tmp_entries(kMaxN + 1);
  b.wstack_cap = kStackCap;
  b.wstack_slots = kSlots;
  return b;
}

struct DeviceWorkspace {
  bh_system *sys = nullptr;
  bh::Scalars host_sc{};
  bh::SysScalars host_ss{};
};

std::mutex g_mu;
DeviceWorkspace g_ws[64];

thread_local char g_msg[256];

}  // namespace

extern "C" int bh_compute_forces_noalloc(const double *d_m, const double *d_x, const double *d_y,
                                         const double *d_z, int64_t n, const bh_params *p,
                                         double *d_out, void *stream) {
  if (n < 1 || n > kMaxN) {
    snprintf(g_msg, sizeof g_msg,
             "bh_compute_forces_noalloc: n=%lld outside 1..%lld (the fixed workspace limit); use "
             "bh_compute_forces_ex or a bh_system for larger systems",
             (long long)n, (long long)kMaxN);
    return bh_report_error(BH_ERR_INVALID, g_msg);
  }
  if (!d_m || !d_x || !d_y || !d_z || !d_out || !p)
    return bh_report_error(BH_ERR_INVALID, "bh_compute_forces_noalloc: NULL argument");
  if (p->precision == BH_PREC_DEHNEN)
    return bh_report_error(BH_ERR_INVALID,
                           "bh_compute_forces_noalloc: Dehnen's method sizes its pair lists at run "
                           "time and needs allocated work buffers; use a bh_system");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing((cudaStream_t)stream, &cap) != cudaSuccess)
    return bh_report_error(BH_ERR_CUDA, "bh_compute_forces_noalloc: cudaStreamIsCapturing failed");
  if (cap != cudaStreamCaptureStatusNone)
    return bh_report_error(BH_ERR_INVALID,
                           "bh_compute_forces_noalloc: the stream is being captured; the call "
                           "synchronises its stream and cannot be captured");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return bh_report_error(BH_ERR_CUDA, "bh_compute_forces_noalloc: no current CUDA device");
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceWorkspace &w = g_ws[dev];
  if (!w.sys) {
    // once per device, with that device current: the array's device address
    void *base = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&base, g_scratch);
    if (e != cudaSuccess || base == nullptr) {
      snprintf(g_msg, sizeof g_msg, "cudaGetSymbolAddress of the workspace failed: %s",
               cudaGetErrorString(e));
      return bh_report_error(BH_ERR_CUDA, g_msg);
    }
    w.sys = bh::fixed_system_create(dev, carve(static_cast<unsigned char *>(base)), &w.host_sc,
                                      &w.host_ss);
  }
  return bh_system_forces(w.sys, d_m, d_x, d_y, d_z, n, p, d_out, stream);
}
