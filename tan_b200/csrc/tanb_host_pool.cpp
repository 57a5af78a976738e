// Host worker pool (tanb_host_pool.h). A job is an index range handed out one
// index at a time through an atomic counter; workers sleep on a condition
// variable between jobs. Jobs are serialised by a mutex, so concurrent API
// calls from several threads take turns. In a process forked after the pool
// started, jobs run serially on the caller. copy_for_device streams large
// copies into pinned memory past the CPU caches.
#include "tanb_host_pool.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include <cstdint>
#include <cstring>

#include <unistd.h>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

namespace tanb {
namespace {

class Pool {
 public:
  explicit Pool(int nthreads) : pid_(getpid()) {
    for (int t = 0; t < nthreads; ++t) workers_.emplace_back([this] { loop(); });
  }

  // A process forked after the pool started has none of its threads.
  bool usable() const { return getpid() == pid_; }

  int threads() const { return (int)workers_.size(); }

  void run(int n, const std::function<void(int)>& fn) {
    std::lock_guard<std::mutex> job_lock(job_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      busy_ = (int)workers_.size();
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return busy_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (int i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) (*fn_)(i);
  }

  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      work();
      {
        std::lock_guard<std::mutex> lk(mu_);
        --busy_;
      }
      done_cv_.notify_one();
    }
  }

  const pid_t pid_;
  std::vector<std::thread> workers_;
  std::mutex job_mu_;  // one job at a time
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0;
  std::atomic<int> next_{0};
  int busy_ = 0;
  unsigned long long gen_ = 0;
};

Pool& pool() {
  // half of the host's hardware threads, at most 8: enough to saturate the
  // memory bandwidth of a copy without taking the whole host
  // Never destroyed: its idle workers end with the process (a destructor
  // would have to join them, also in a forked child that does not have them).
  static Pool* p = new Pool(std::max(1, std::min(8, (int)std::thread::hardware_concurrency() / 2) - 1));
  return *p;
}

}  // namespace

void host_parallel_for(int n, const std::function<void(int)>& fn) {
  if (n <= 0) return;
  Pool& p = pool();
  if (n == 1 || !p.usable()) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  p.run(n, fn);
}

int host_pool_threads() { return pool().threads(); }

namespace {

// Non-temporal copy without a fence (x86-64); false if not applicable.
bool stream_copy(void* dst, const void* src, size_t bytes, size_t min_bytes) {
#if defined(__x86_64__)
  if (bytes >= min_bytes) {
    auto* d = static_cast<uint8_t*>(dst);
    auto* s = static_cast<const uint8_t*>(src);
    const size_t lead = (16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15;
    std::memcpy(d, s, lead);
    d += lead;
    s += lead;
    bytes -= lead;
    const size_t body = bytes & ~size_t(63);
    for (size_t i = 0; i < body; i += 64) {
      const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i));
      const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 16));
      const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 32));
      const __m128i e = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 48));
      _mm_stream_si128(reinterpret_cast<__m128i*>(d + i), a);
      _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 16), b);
      _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 32), c);
      _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 48), e);
    }
    std::memcpy(d + body, s + body, bytes - body);
    return true;
  }
#endif
  (void)dst;
  (void)src;
  (void)bytes;
  (void)min_bytes;
  return false;
}

}  // namespace

void copy_for_device(void* dst, const void* src, size_t bytes) {
  if (stream_copy(dst, src, bytes, 4096))
    copy_for_device_fence();  // the stores are visible before anything this thread does next
  else
    std::memcpy(dst, src, bytes);
}

void copy_rows_for_device(void* dst, const void* src, size_t bytes) {
  if (!stream_copy(dst, src, bytes, 256)) std::memcpy(dst, src, bytes);
}

void copy_for_device_fence() {
#if defined(__x86_64__)
  _mm_sfence();
#endif
}

}  // namespace tanb
