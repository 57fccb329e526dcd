// fe_staging.cu -- host-buffer solves from pageable memory through a pinned
// staging ring owned by the plan.
//
// A cudaMemcpyAsync from pageable memory is staged by the driver at a
// fraction of the PCIe bandwidth and overlaps nothing.  Here every pageable
// column is cut into chunks that a pool of host threads copies into pinned
// ring slots, from which the DMA runs; the host copy of chunk k+1 overlaps
// the DMA of chunk k.  The uploads run on a helper thread (and an upload
// stream), so a tile's solve starts as soon as its own columns are on the
// device while the next tiles are still being staged; after each tile's solve
// a second helper thread brings its columns back through a second ring
// (device -> pinned slot -> the caller's column), overlapping the solves of
// the tiles that follow.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "fe_plan.h"
#include "fe_staging.h"

namespace fe {

namespace {

// A fixed pool of host threads splitting large memcpys.
class CopyPool {
 public:
  explicit CopyPool(int n) {
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // copies n bytes with every thread of the pool; returns when done
  void copy(char* d, const char* s, size_t n) {
    const size_t parts = std::max<size_t>(1, std::min<size_t>(th_.size(), n >> 20));
    const size_t piece = ((n + parts - 1) / parts + 63) & ~(size_t)63;
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t o = 0; o < n; o += piece) q_.push_back({d + o, s + o, std::min(piece, n - o)});
    }
    cv_.notify_all();
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [this] { return q_.empty() && busy_ == 0; });
  }

 private:
  struct Task {
    char* d;
    const char* s;
    size_t n;
  };
  void loop() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;  // stop_
        t = q_.front();
        q_.pop_front();
        ++busy_;
      }
      memcpy(t.d, t.s, t.n);
      {
        std::lock_guard<std::mutex> lk(mu_);
        --busy_;
        if (q_.empty() && busy_ == 0) done_.notify_all();
      }
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::deque<Task> q_;
  int busy_ = 0;
  bool stop_ = false;
};

int host_threads() {
  const unsigned h = std::thread::hardware_concurrency();
  return (int)std::max(2u, std::min(16u, h ? h : 4u));
}

}  // namespace

struct PageableStager {
  fe_plan* pl = nullptr;
  void* const* cols = nullptr;
  size_t col_bytes = 0;
  std::vector<int64_t> tile0;  // first column of each tile, then ncols
  char* dev = nullptr;         // device staging: column j at dev + j * col_bytes
  cudaStream_t up = nullptr, down = nullptr;
  std::vector<cudaEvent_t> up_ev, down_ev;      // per ring slot
  std::vector<cudaEvent_t> tile_up, tile_done;  // per tile
  std::thread up_thread, down_thread;
  std::mutex mu;
  std::condition_variable cv;
  size_t uploaded = 0;        // tiles whose uploads are enqueued (tile_up recorded)
  std::deque<size_t> solved;  // tiles whose solve is enqueued, to download
  bool finished = false;      // no more tiles to download
  int status = 0;             // first error of a helper thread
  std::string message;

  void fail(const std::string& what, cudaError_t e) {
    (void)cudaGetLastError();
    std::lock_guard<std::mutex> lk(mu);
    if (!status) {
      status = 2;  // FE_ERR_CUDA
      message = what + ": " + cudaGetErrorString(e);
    }
  }
};

namespace {

void upload_main(PageableStager* x) {
  cudaSetDevice(x->pl->device);
  CopyPool pool(std::max(1, host_threads() / 2));
  char* ring = static_cast<char*>(x->pl->ring_up);
  const size_t slot = x->pl->ring_slot_bytes;
  int64_t k = 0;
  cudaError_t e = cudaSuccess;
  for (size_t t = 0; t + 1 < x->tile0.size(); ++t) {
    for (int64_t j = x->tile0[t]; j < x->tile0[t + 1] && e == cudaSuccess; ++j) {
      const char* src = static_cast<const char*>(x->cols[j]);
      for (size_t o = 0; o < x->col_bytes && e == cudaSuccess; o += slot, ++k) {
        const int s = (int)(k % kRingSlots);
        if (k >= kRingSlots) e = cudaEventSynchronize(x->up_ev[s]);  // the slot's DMA is done
        if (e != cudaSuccess) break;
        const size_t n = std::min(slot, x->col_bytes - o);
        pool.copy(ring + (size_t)s * slot, src + o, n);
        e = cudaMemcpyAsync(x->dev + (size_t)j * x->col_bytes + o, ring + (size_t)s * slot, n,
                            cudaMemcpyHostToDevice, x->up);
        if (e == cudaSuccess) e = cudaEventRecord(x->up_ev[s], x->up);
      }
    }
    if (e == cudaSuccess) e = cudaEventRecord(x->tile_up[t], x->up);
    if (e != cudaSuccess) {
      x->fail("staged host to device copy failed", e);
      break;
    }
    {
      std::lock_guard<std::mutex> lk(x->mu);
      x->uploaded = t + 1;
    }
    x->cv.notify_all();
  }
  {
    std::lock_guard<std::mutex> lk(x->mu);
    x->uploaded = x->tile0.size();  // wakes a waiting solve after an error too
  }
  x->cv.notify_all();
}

void download_main(PageableStager* x) {
  cudaSetDevice(x->pl->device);
  CopyPool pool(std::max(1, host_threads() / 2));
  char* ring = static_cast<char*>(x->pl->ring_down);
  const size_t slot = x->pl->ring_slot_bytes;
  for (;;) {
    size_t t;
    {
      std::unique_lock<std::mutex> lk(x->mu);
      x->cv.wait(lk, [x] { return x->finished || !x->solved.empty(); });
      if (x->solved.empty()) return;
      t = x->solved.front();
      x->solved.pop_front();
    }
    cudaError_t e = cudaStreamWaitEvent(x->down, x->tile_done[t], 0);
    // chunk k is brought to its slot while chunk k-1 is copied out of its own
    struct Pending {
      char* dst;
      int slot;
      size_t n;
    };
    std::vector<Pending> chunks;
    for (int64_t j = x->tile0[t]; j < x->tile0[t + 1]; ++j)
      for (size_t o = 0; o < x->col_bytes; o += slot)
        chunks.push_back({static_cast<char*>(x->cols[j]) + o, 0,
                          std::min(slot, x->col_bytes - o)});
    int64_t k = 0;
    for (int64_t j = x->tile0[t]; j < x->tile0[t + 1] && e == cudaSuccess; ++j)
      for (size_t o = 0; o < x->col_bytes && e == cudaSuccess; o += slot, ++k) {
        const int s = (int)(k % kRingSlots);
        chunks[(size_t)k].slot = s;
        e = cudaMemcpyAsync(ring + (size_t)s * slot, x->dev + (size_t)j * x->col_bytes + o,
                            chunks[(size_t)k].n, cudaMemcpyDeviceToHost, x->down);
        if (e == cudaSuccess) e = cudaEventRecord(x->down_ev[s], x->down);
        if (e == cudaSuccess && k >= 1) {
          const Pending& p = chunks[(size_t)k - 1];
          e = cudaEventSynchronize(x->down_ev[p.slot]);
          if (e == cudaSuccess) pool.copy(p.dst, ring + (size_t)p.slot * slot, p.n);
        }
        // the slot of chunk k + 1 held chunk k + 1 - kRingSlots, already copied out
      }
    if (e == cudaSuccess && k >= 1) {
      const Pending& p = chunks[(size_t)k - 1];
      e = cudaEventSynchronize(x->down_ev[p.slot]);
      if (e == cudaSuccess) pool.copy(p.dst, ring + (size_t)p.slot * slot, p.n);
    }
    if (e != cudaSuccess) {
      x->fail("staged device to host copy failed", e);
      return;
    }
  }
}

}  // namespace

int stager_begin(fe_plan* pl, void* const* cols, size_t col_bytes, const std::vector<int64_t>& tile0,
                 char* dev, PageableStager** out) {
  *out = nullptr;
  if (!pl->ring_up) {
    const size_t bytes = (size_t)kRingSlots * kRingSlotBytes;
    FE_CK(cudaMallocHost(&pl->ring_up, bytes));
    FE_CK(cudaMallocHost(&pl->ring_down, bytes));
    pl->ring_slot_bytes = kRingSlotBytes;
  }
  PageableStager* x = new PageableStager();
  x->pl = pl;
  x->cols = cols;
  x->col_bytes = col_bytes;
  x->tile0 = tile0;
  x->dev = dev;
  auto cleanup = [x]() { stager_end(x); };
  cudaError_t e = cudaStreamCreateWithFlags(&x->up, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x->down, cudaStreamNonBlocking);
  // the uploads must not overtake work already queued on the plan's stream
  // that reads the staging buffer
  cudaEvent_t start = nullptr;
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&start, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(start, pl->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(x->up, start, 0);
  if (start) cudaEventDestroy(start);
  for (int s = 0; s < kRingSlots && e == cudaSuccess; ++s) {
    cudaEvent_t a = nullptr, b = nullptr;
    e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
    if (e == cudaSuccess) x->up_ev.push_back(a);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
    if (e == cudaSuccess) x->down_ev.push_back(b);
  }
  for (size_t t = 0; t + 1 < tile0.size() && e == cudaSuccess; ++t) {
    cudaEvent_t a = nullptr, b = nullptr;
    e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
    if (e == cudaSuccess) x->tile_up.push_back(a);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
    if (e == cudaSuccess) x->tile_done.push_back(b);
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_error(std::string("staging set-up failed: ") + cudaGetErrorString(e));
    cleanup();
    return 2;
  }
  x->up_thread = std::thread(upload_main, x);
  x->down_thread = std::thread(download_main, x);
  *out = x;
  return 0;
}

int stager_before_tile(PageableStager* x, size_t tile) {
  {
    std::unique_lock<std::mutex> lk(x->mu);
    x->cv.wait(lk, [x, tile] { return x->uploaded > tile; });
    if (x->status) {
      set_error(x->message);
      return x->status;
    }
  }
  FE_CK(cudaStreamWaitEvent(x->pl->stream, x->tile_up[tile], 0));
  return 0;
}

int stager_after_tile(PageableStager* x, size_t tile) {
  FE_CK(cudaEventRecord(x->tile_done[tile], x->pl->stream));
  {
    std::lock_guard<std::mutex> lk(x->mu);
    x->solved.push_back(tile);
  }
  x->cv.notify_all();
  return 0;
}

int stager_end(PageableStager* x) {
  if (!x) return 0;
  {
    std::lock_guard<std::mutex> lk(x->mu);
    x->finished = true;
  }
  x->cv.notify_all();
  if (x->up_thread.joinable()) x->up_thread.join();
  if (x->down_thread.joinable()) x->down_thread.join();
  if (x->up) cudaStreamSynchronize(x->up);
  if (x->down) cudaStreamSynchronize(x->down);
  for (cudaEvent_t ev : x->up_ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : x->down_ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : x->tile_up) cudaEventDestroy(ev);
  for (cudaEvent_t ev : x->tile_done) cudaEventDestroy(ev);
  if (x->up) cudaStreamDestroy(x->up);
  if (x->down) cudaStreamDestroy(x->down);
  const int st = x->status;
  if (st) set_error(x->message);
  delete x;
  return st;
}

}  // namespace fe
