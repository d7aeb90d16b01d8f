// Host-array transfers of the host-array entry points (bh_compute_forces,
// bh_compute_forces_ex, bh_compute_forces_direct).
//
// A caller's pageable array (an ordinary numpy array from the f2py-style
// drop-in) cannot be read by the copy engines: cudaMemcpyAsync then stages it
// through the driver's own pinned buffers one piece after another at a
// fraction of the host link's bandwidth.  Here a process-wide pool of host
// threads does the staging instead, in parallel: worker w takes the chunks w,
// w + T, w + 2T, ... of the transfer and owns two pinned slots of kChunk
// bytes.  Inputs: the worker copies a chunk into a free slot and queues the
// slot's DMA to the device on its own stream, then fills its other slot while
// that DMA runs.  Results: the worker queues the DMA of its next chunk into
// one slot while it copies the previous chunk out of the other.  The T
// streams start after the work already queued on the caller's stream, and
// the caller's stream waits for all of them after an upload.  Pinned arrays
// keep the direct copy.
#include <string.h>

#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int64_t kChunk = 512 * 1024;  // bytes per slot
constexpr int kMaxWorkers = 8;

// Runs one job at a time on T threads (worker 0 is the calling thread).  The
// pool lives until the process exits; its threads wait on a condition
// variable between jobs.
class WorkerPool {
 public:
  static WorkerPool &get() {
    static WorkerPool *pool = new WorkerPool();  // never destroyed: threads outlive static teardown
    return *pool;
  }
  int size() const { return n_; }
  void run(const std::function<void(int)> &fn) {
    std::lock_guard<std::mutex> one(run_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &fn;
      pending_ = n_ - 1;
      ++gen_;
    }
    start_cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  WorkerPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    n_ = (int)(hw == 0 ? 1 : (hw < (unsigned)kMaxWorkers ? hw : (unsigned)kMaxWorkers));
    for (int w = 1; w < n_; ++w) std::thread([this, w] { loop(w); }).detach();
  }
  void loop(int w) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int)> *job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        start_cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        job = job_;
      }
      (*job)(w);
      {
        std::lock_guard<std::mutex> lk(mu_);
        --pending_;
      }
      done_cv_.notify_all();
    }
  }
  int n_ = 1;
  std::mutex run_mu_, mu_;
  std::condition_variable start_cv_, done_cv_;
  const std::function<void(int)> *job_ = nullptr;
  uint64_t gen_ = 0;
  int pending_ = 0;
};

// One piece of a transfer: `bytes` at host + off and device + off.
struct Piece {
  char *host;
  char *dev;
  int64_t bytes;
};

std::vector<Piece> cut(const double *const *host, double *const *dev, int count, int64_t n) {
  std::vector<Piece> v;
  const int64_t total = n * (int64_t)sizeof(double);
  for (int a = 0; a < count; ++a)
    for (int64_t o = 0; o < total; o += kChunk)
      v.push_back(Piece{(char *)host[a] + o, (char *)dev[a] + o, total - o < kChunk ? total - o : kChunk});
  return v;
}

}  // namespace

struct HostCopy {
  int device = 0;
  int workers = 0;
  char *slots = nullptr;  // 2 slots of kChunk bytes per worker, pinned
  std::vector<cudaStream_t> st;
  std::vector<cudaEvent_t> slot_ev;  // the last DMA through each slot
  std::vector<unsigned char> slot_used;  // one byte per slot: workers write their own slots
  cudaEvent_t start = nullptr;
  std::vector<cudaEvent_t> end;
};

HostKind host_kind(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // an unknown pointer is pageable host memory
    return HostKind::kPageable;
  }
  if (a.type == cudaMemoryTypeHost) return HostKind::kPinned;
  if (a.type == cudaMemoryTypeDevice) return HostKind::kDevice;
  return HostKind::kPageable;  // unregistered host memory, or managed memory
}

HostCopy *hostcopy_create(int device) {
  HostCopy *h = new HostCopy();
  h->device = device;
  h->workers = WorkerPool::get().size();
  const int W = h->workers;
  bool ok = cudaMallocHost((void **)&h->slots, (size_t)(2 * W) * kChunk) == cudaSuccess &&
            cudaEventCreateWithFlags(&h->start, cudaEventDisableTiming) == cudaSuccess;
  h->st.assign(W, nullptr);
  h->end.assign(W, nullptr);
  h->slot_ev.assign(2 * W, nullptr);
  h->slot_used.assign(2 * W, 0);
  for (int w = 0; ok && w < W; ++w)
    ok = cudaStreamCreateWithFlags(&h->st[w], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&h->end[w], cudaEventDisableTiming) == cudaSuccess;
  for (int k = 0; ok && k < 2 * W; ++k)
    ok = cudaEventCreateWithFlags(&h->slot_ev[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    hostcopy_destroy(h);
    return nullptr;
  }
  return h;
}

void hostcopy_destroy(HostCopy *h) {
  if (!h) return;
  for (cudaStream_t s : h->st)
    if (s) cudaStreamSynchronize(s);
  for (cudaStream_t s : h->st)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : h->end)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->slot_ev)
    if (e) cudaEventDestroy(e);
  if (h->start) cudaEventDestroy(h->start);
  if (h->slots) cudaFreeHost(h->slots);
  delete h;
}

cudaError_t hostcopy_upload(HostCopy *h, const double *const *src, double *const *dst, int count,
                            int64_t n, cudaStream_t st) {
  const std::vector<Piece> pieces = cut(src, dst, count, n);
  cudaError_t e = cudaEventRecord(h->start, st);  // the device arrays may still be read on st
  if (e != cudaSuccess) return e;
  std::atomic<int> first_err{(int)cudaSuccess};
  const int W = h->workers;
  WorkerPool::get().run([&](int w) {
    cudaError_t r = cudaSetDevice(h->device);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(h->st[w], h->start, 0);
    int it = 0;
    for (size_t k = (size_t)w; r == cudaSuccess && k < pieces.size(); k += (size_t)W, ++it) {
      const int slot = 2 * w + (it & 1);
      char *buf = h->slots + (int64_t)slot * kChunk;
      if (h->slot_used[slot]) r = cudaEventSynchronize(h->slot_ev[slot]);  // its last DMA is done
      if (r != cudaSuccess) break;
      memcpy(buf, pieces[k].host, (size_t)pieces[k].bytes);
      r = cudaMemcpyAsync(pieces[k].dev, buf, (size_t)pieces[k].bytes, cudaMemcpyHostToDevice,
                          h->st[w]);
      if (r == cudaSuccess) r = cudaEventRecord(h->slot_ev[slot], h->st[w]);
      h->slot_used[slot] = 1;
    }
    if (r == cudaSuccess) r = cudaEventRecord(h->end[w], h->st[w]);
    int ok = (int)cudaSuccess;
    if (r != cudaSuccess) first_err.compare_exchange_strong(ok, (int)r);
  });
  if (first_err.load() != (int)cudaSuccess) return (cudaError_t)first_err.load();
  for (int w = 0; w < W; ++w) {
    e = cudaStreamWaitEvent(st, h->end[w], 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t hostcopy_download(HostCopy *h, double *dst, const double *src, int64_t n,
                              cudaStream_t st) {
  const double *srcs[1] = {src};
  double *dsts[1] = {dst};
  // pieces with host = dst (written) and dev = src (read)
  const std::vector<Piece> pieces = cut(dsts, const_cast<double *const *>(srcs), 1, n);
  cudaError_t e = cudaEventRecord(h->start, st);  // the result is complete after st's work
  if (e != cudaSuccess) return e;
  std::atomic<int> first_err{(int)cudaSuccess};
  const int W = h->workers;
  WorkerPool::get().run([&](int w) {
    cudaError_t r = cudaSetDevice(h->device);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(h->st[w], h->start, 0);
    std::vector<size_t> mine;
    for (size_t k = (size_t)w; k < pieces.size(); k += (size_t)W) mine.push_back(k);
    auto issue = [&](size_t i) {
      const int slot = 2 * w + (int)(i & 1);
      char *buf = h->slots + (int64_t)slot * kChunk;
      cudaError_t q = cudaMemcpyAsync(buf, pieces[mine[i]].dev, (size_t)pieces[mine[i]].bytes,
                                      cudaMemcpyDeviceToHost, h->st[w]);
      if (q == cudaSuccess) q = cudaEventRecord(h->slot_ev[slot], h->st[w]);
      h->slot_used[slot] = 1;
      return q;
    };
    if (r == cudaSuccess && !mine.empty()) r = issue(0);
    for (size_t i = 0; r == cudaSuccess && i < mine.size(); ++i) {
      // the other slot was emptied in the previous round: its next DMA may start
      if (i + 1 < mine.size()) r = issue(i + 1);
      const int slot = 2 * w + (int)(i & 1);
      if (r == cudaSuccess) r = cudaEventSynchronize(h->slot_ev[slot]);
      if (r == cudaSuccess)
        memcpy(pieces[mine[i]].host, h->slots + (int64_t)slot * kChunk,
               (size_t)pieces[mine[i]].bytes);
    }
    int ok = (int)cudaSuccess;
    if (r != cudaSuccess) first_err.compare_exchange_strong(ok, (int)r);
  });
  return (cudaError_t)first_err.load();
}

}  // namespace bh
