// af_xfer.cu -- host<->device row-block copies at the link's rate from
// pinned or pageable host memory (see af_xfer.h).
#include "af_xfer.h"

#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace af {
namespace {

constexpr size_t kBufBytes = 16u << 20;  // each of the two pinned buffers
constexpr size_t kMinStaged = 1u << 20;  // smaller copies: the driver's own path is as quick

// Worker threads that run the pieces of one host-side copy; the calling
// thread takes pieces too.
class CopyPool {
 public:
  explicit CopyPool(int workers) {
    for (int k = 0; k < workers; k++) th_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  int threads() const { return (int)th_.size() + 1; }
  // fn(k) for k = 0 .. n-1; returns when every piece is done.
  void run(int n, const std::function<void(int)>& fn) {
    {
      std::lock_guard<std::mutex> g(mu_);
      fn_ = &fn;
      n_ = n;
      next_ = 0;
      busy_ = (int)th_.size();
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> l(mu_);
    done_.wait(l, [this] { return busy_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      const int k = next_.fetch_add(1);
      if (k >= n_) return;
      (*fn_)(k);
    }
  }
  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
      {
        std::lock_guard<std::mutex> g(mu_);
        busy_--;
      }
      done_.notify_all();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* fn_ = nullptr;  // set under mu_ before gen_ changes
  int n_ = 0;
  std::atomic<int> next_{0};
  int busy_ = 0;
  unsigned long long gen_ = 0;
  bool stop_ = false;
  std::vector<std::thread> th_;
};

// The process's two pinned buffers and copy threads, made on first use.
// Never freed: they live until the process exits (CUDA's own teardown at
// exit makes freeing pinned memory from a static destructor unsafe).
struct Staging {
  std::mutex mu;  // one staged copy at a time
  void* buf[2] = {nullptr, nullptr};
  CopyPool* pool = nullptr;
  bool tried = false;
  pid_t pid = 0;
};

Staging& staging() {
  static Staging* s = new Staging;
  return *s;
}

// Under s.mu.  A forked child starts over (its parent's threads are gone).
bool ready(Staging& s) {
  if (s.pid != getpid()) {
    s.pid = getpid();
    s.buf[0] = s.buf[1] = nullptr;
    s.pool = nullptr;
    s.tried = false;
  }
  if (!s.tried) {
    s.tried = true;
    for (int b = 0; b < 2; b++)
      if (cudaHostAlloc(&s.buf[b], kBufBytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        s.buf[b] = nullptr;
      }
    if (!s.buf[0] || !s.buf[1]) {
      for (int b = 0; b < 2; b++)
        if (s.buf[b]) cudaFreeHost(s.buf[b]);
      s.buf[0] = s.buf[1] = nullptr;
    }
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    s.pool = new CopyPool(std::max(0, std::min(7, hw - 1)));
  }
  return s.buf[0] != nullptr;
}

// Pageable host memory: the driver cannot DMA it directly.  A pointer CUDA
// cannot classify goes to cudaMemcpy2DAsync, which reports the error.
bool pageable(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// rows x width bytes from (src, spitch) to (dst, dpitch) on the pool's threads.
void host_rows(CopyPool& pool, char* dst, size_t dpitch, const char* src, size_t spitch,
               size_t width, size_t rows) {
  const int t = pool.threads();
  if (dpitch == width && spitch == width) {  // one contiguous block: split it by bytes
    const size_t total = width * rows;
    const size_t piece = (total + t - 1) / t;
    pool.run(t, [&](int k) {
      const size_t a = std::min(total, (size_t)k * piece), b = std::min(total, a + piece);
      if (b > a) std::memcpy(dst + a, src + a, b - a);
    });
    return;
  }
  const int n = (int)std::min<size_t>(rows, (size_t)t);
  pool.run(n, [&](int k) {
    const size_t r0 = rows * k / n, r1 = rows * (k + 1) / n;
    for (size_t r = r0; r < r1; r++) std::memcpy(dst + r * dpitch, src + r * spitch, width);
  });
}

}  // namespace

cudaError_t copy2d_h2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st) {
  if (rows == 0 || width == 0) return cudaSuccess;
  Staging& S = staging();
  if (width > kBufBytes || width * rows < kMinStaged || !pageable(src))
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyHostToDevice, st);
  std::lock_guard<std::mutex> g(S.mu);
  if (!ready(S))
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyHostToDevice, st);
  const size_t rpc = kBufBytes / width;  // rows per buffer
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t e = cudaSuccess;
  for (int b = 0; b < 2 && e == cudaSuccess; b++)
    e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
  size_t k = 0;
  for (size_t r = 0; r < rows && e == cudaSuccess; r += rpc, k++) {
    const int b = (int)(k & 1);
    const size_t n = std::min(rpc, rows - r);
    if (k >= 2) e = cudaEventSynchronize(ev[b]);  // the buffer's last copy has left it
    if (e != cudaSuccess) break;
    host_rows(*S.pool, static_cast<char*>(S.buf[b]), width,
              static_cast<const char*>(src) + r * spitch, spitch, width, n);
    e = cudaMemcpy2DAsync(static_cast<char*>(dst) + r * dpitch, dpitch, S.buf[b], width, width, n,
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[b], st);
  }
  // The buffers are free for the next copy once their last copies are done.
  for (int b = 0; b < 2; b++)
    if (ev[b]) {
      const cudaError_t e2 = cudaEventSynchronize(ev[b]);
      if (e == cudaSuccess) e = e2;
      cudaEventDestroy(ev[b]);
    }
  return e;
}

cudaError_t copy2d_d2h(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st) {
  if (rows == 0 || width == 0) return cudaSuccess;
  Staging& S = staging();
  if (width > kBufBytes || width * rows < kMinStaged || !pageable(dst))
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToHost, st);
  std::lock_guard<std::mutex> g(S.mu);
  if (!ready(S))
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToHost, st);
  const size_t rpc = kBufBytes / width;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t e = cudaSuccess;
  for (int b = 0; b < 2 && e == cudaSuccess; b++)
    e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
  // Chunk k is copied into buffer k & 1 while the host drains chunk k - 1.
  size_t prev_r = 0, prev_n = 0;
  int prev_b = -1;
  auto drain = [&]() {
    if (prev_b < 0) return;
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[prev_b]);
    if (e == cudaSuccess)
      host_rows(*S.pool, static_cast<char*>(dst) + prev_r * dpitch, dpitch,
                static_cast<const char*>(S.buf[prev_b]), width, width, prev_n);
    prev_b = -1;
  };
  size_t k = 0;
  for (size_t r = 0; r < rows && e == cudaSuccess; r += rpc, k++) {
    const int b = (int)(k & 1);
    const size_t n = std::min(rpc, rows - r);
    e = cudaMemcpy2DAsync(S.buf[b], width, static_cast<const char*>(src) + r * spitch, spitch,
                          width, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[b], st);
    drain();
    prev_r = r, prev_n = n, prev_b = b;
  }
  drain();
  for (int b = 0; b < 2; b++)
    if (ev[b]) {
      const cudaError_t e2 = cudaEventSynchronize(ev[b]);
      if (e == cudaSuccess) e = e2;
      cudaEventDestroy(ev[b]);
    }
  return e;
}

}  // namespace af
