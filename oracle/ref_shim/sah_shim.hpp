// sah_shim.hpp -- thread emulation for the reference's SAH build and raster
// kernels, whose 32 threads per block cooperate through __syncthreads and
// __shared__ data.
// Each emulated block runs on 32 host threads (a persistent pool) that meet at
// a barrier for every __syncthreads; blocks run one after another, which is
// the serial execution of the reference's launches (the block that pops the
// stack first finishes before the next pops). TEST INFRASTRUCTURE ONLY.
#pragma once
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#define __builtin_align__(a) __attribute__((aligned(a)))

// internal linkage: every checker TU that includes this file gets its own
// pool and barrier (inline members would otherwise merge across TUs)
namespace {

struct ShimBarrier {
  std::mutex m;
  std::condition_variable cv;
  int count, waiting = 0;
  unsigned gen = 0;
  explicit ShimBarrier(int n) : count(n) {}
  void wait() {
    std::unique_lock<std::mutex> lk(m);
    const unsigned g = gen;
    if (++waiting == count) {
      waiting = 0;
      ++gen;
      cv.notify_all();
    } else {
      cv.wait(lk, [&] { return gen != g; });
    }
  }
};

static ShimBarrier* g_block_sync = nullptr;
static inline void __syncthreads() { g_block_sync->wait(); }

static std::mutex g_atomic_mutex;
static inline int atomicAdd(int* p, int v) {
  std::lock_guard<std::mutex> l(g_atomic_mutex);
  const int o = *p;
  *p = o + v;
  return o;
}
static inline int atomicSub(int* p, int v) {
  std::lock_guard<std::mutex> l(g_atomic_mutex);
  const int o = *p;
  *p = o - v;
  return o;
}

// 32 persistent host threads that run one block of a kernel per round.
// Thread t gets threadIdx (t % block_x, t / block_x).
struct ShimBlockPool {
  static const int kThreads = 32;
  ShimBarrier start{kThreads + 1}, done{kThreads + 1}, sync{kThreads};
  std::function<void()> body;
  bool quit = false;
  std::vector<std::thread> workers;
  explicit ShimBlockPool(int block_x = kThreads) {
    g_block_sync = &sync;
    for (int t = 0; t < kThreads; ++t)
      workers.emplace_back([this, t, block_x] {
        threadIdx.x = (unsigned)(t % block_x); threadIdx.y = (unsigned)(t / block_x); threadIdx.z = 0;
        for (;;) {
          start.wait();
          if (quit) return;
          body();
          done.wait();
        }
      });
  }
  void run(const std::function<void()>& f) {
    body = f;
    start.wait();
    done.wait();
  }
  ~ShimBlockPool() {
    quit = true;
    start.wait();
    for (auto& w : workers) w.join();
    g_block_sync = nullptr;
  }
};
}  // namespace
