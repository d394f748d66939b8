// Staged host-to-device upload of pageable caller buffers (see upload.cuh).
//
// An upload borrows one of a few process-wide sets of kSlots pinned staging
// slots of kChunk bytes (per device, allocated once). Chunk i is copied into
// slot i % kSlots by a process-wide pool of host threads (the caller takes
// one share), then its cudaMemcpyAsync is issued on the caller's stream and
// an event recorded; before a slot is refilled (by this or a later upload)
// the call waits for that event. So the host copies of chunk i + 1 overlap
// the DMA of chunk i.
#include "upload.cuh"
#include "common.cuh"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace fpls {

namespace {

constexpr size_t kChunk = size_t(16) << 20;
constexpr int kSlots = 3;

// A fixed pool of host threads running memcpy pieces.
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool pool;
    return pool;
  }
  int width() const { return (int)workers_.size() + 1; }

  // dst[0, bytes) = src[0, bytes), split over the pool and the caller.
  void copy(char* dst, const char* src, size_t bytes) {
    const int parts = std::max(1, std::min(width(), (int)(bytes >> 20)));
    if (parts == 1) {
      std::memcpy(dst, src, bytes);
      return;
    }
    const size_t piece = (bytes / parts + 63) & ~size_t(63);
    struct Done {
      std::mutex mu;
      std::condition_variable cv;
      int left = 0;
    } done;
    done.left = parts - 1;
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (int k = 1; k < parts; ++k) {
        const size_t off = std::min(bytes, piece * k);
        const size_t len = std::min(bytes - off, piece);
        tasks_.push_back([dst, src, off, len, &done] {
          if (len) std::memcpy(dst + off, src + off, len);
          std::lock_guard<std::mutex> l(done.mu);
          if (--done.left == 0) done.cv.notify_all();
        });
      }
    }
    cv_.notify_all();
    std::memcpy(dst, src, std::min(bytes, piece));
    std::unique_lock<std::mutex> lock(done.mu);
    done.cv.wait(lock, [&] { return done.left == 0; });
  }

  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }

 private:
  CopyPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const int n = (int)std::max(1u, std::min(8u, hw > 1 ? hw / 2 : 1u)) - 1;
    for (int k = 0; k < n; ++k) workers_.emplace_back([this] { run(); });
  }
  void run() {
    for (;;) {
      std::function<void()> task;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return stop_ || !tasks_.empty(); });
        if (stop_ && tasks_.empty()) return;
        task = std::move(tasks_.front());
        tasks_.pop_front();
      }
      task();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> tasks_;
  bool stop_ = false;
};

// A set of pinned slots with the events of their last DMAs.
struct Staging {
  int device = -1;
  char* slot[kSlots] = {};
  cudaEvent_t ev[kSlots] = {};
  bool pending[kSlots] = {};

  bool init(int dev) {
    device = dev;
    for (int k = 0; k < kSlots; ++k) {
      void* p = nullptr;
      if (cudaHostAlloc(&p, kChunk, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      slot[k] = static_cast<char*>(p);
      if (cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
    }
    return true;
  }
};

// Process-wide pool of staging sets per device, allocated on first use and
// kept for the life of the process (pinned allocations are slow, and the
// serving loop's worker threads come and go with each server). A caller
// borrows one set for its upload; at most kSets uploads stage at once, the
// others wait for a set.
constexpr int kSets = 4;
class StagingPool {
 public:
  static StagingPool& get() {
    static StagingPool* pool = new StagingPool();  // never destroyed: outlives CUDA teardown
    return *pool;
  }
  Staging* acquire(int dev) {
    std::unique_lock<std::mutex> lock(mu_);
    for (;;) {
      int made = 0;
      for (Staging* st : all_)
        if (st->device == dev) ++made;
      for (size_t k = 0; k < free_.size(); ++k)
        if (free_[k]->device == dev) {
          Staging* st = free_[k];
          free_.erase(free_.begin() + (long)k);
          return st;
        }
      if (made < kSets && !failed_) {
        Staging* st = new Staging();
        if (!st->init(dev)) {
          failed_ = true;  // pinned memory unavailable: fall back to direct copies
          return nullptr;
        }
        all_.push_back(st);
        return st;
      }
      if (failed_ && made == 0) return nullptr;
      cv_.wait(lock);
    }
  }
  void release(Staging* st) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      free_.push_back(st);
    }
    cv_.notify_one();
  }

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<Staging*> all_, free_;
  bool failed_ = false;
};

bool pinned(const void* p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

}  // namespace

void upload_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  Staging* st = nullptr;
  if (bytes >= kUploadStagedMin && !pinned(src)) {
    int dev = 0;
    FPLS_CHECK(cudaGetDevice(&dev));
    st = StagingPool::get().acquire(dev);
  }
  if (!st) {
    FPLS_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  struct Lend {
    Staging* st;
    ~Lend() { StagingPool::get().release(st); }
  } lend{st};
  char* d = static_cast<char*>(dst);
  const char* h = static_cast<const char*>(src);
  int k = 0;
  for (size_t off = 0; off < bytes; off += kChunk, k = (k + 1) % kSlots) {
    const size_t len = std::min(kChunk, bytes - off);
    if (st->pending[k]) {
      FPLS_CHECK(cudaEventSynchronize(st->ev[k]));
      st->pending[k] = false;
    }
    CopyPool::get().copy(st->slot[k], h + off, len);
    FPLS_CHECK(cudaMemcpyAsync(d + off, st->slot[k], len, cudaMemcpyHostToDevice, s));
    FPLS_CHECK(cudaEventRecord(st->ev[k], s));
    st->pending[k] = true;
  }
}

}  // namespace fpls
