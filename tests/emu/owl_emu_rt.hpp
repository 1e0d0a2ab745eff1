// owl_emu_rt.hpp -- a CPU stand-in for the CUDA runtime features the libowl
// kernels use, so that the unchanged kernel source (gpuowl_b200/csrc/*.cuh)
// can run on the host under AddressSanitizer at small FFT sizes.
//
// TEST INFRASTRUCTURE ONLY: every CUDA thread becomes one host thread,
// __syncthreads is a std::barrier per block, warp shuffles exchange through a
// per-warp slot array, global-memory flags use std::atomic_ref with the same
// acquire/release order as the PTX in owl_compat.cuh.
#pragma once
#include <pthread.h>

#include <atomic>
#include <barrier>
#include <bit>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __grid_constant__

struct double2 {
  double x, y;
};
struct int2 {
  int x, y;
};
struct uint2 {
  unsigned x, y;
};
inline uint2 make_uint2(unsigned x, unsigned y) { return uint2{x, y}; }
inline double2 make_double2(double x, double y) { return double2{x, y}; }
inline int2 make_int2(int x, int y) { return int2{x, y}; }

struct emu_dim3 {
  unsigned x = 1, y = 1, z = 1;
};

struct EmuCta {
  int nthreads = 0;
  std::unique_ptr<std::barrier<>> bar;
  std::vector<std::unique_ptr<std::barrier<>>> warpBar;
  std::vector<uint64_t> slots;
  std::vector<char> dyn;
  std::mutex m;
  std::map<int, std::vector<char>> stat;
  std::vector<uint32_t> tmem;  // emulated tensor memory, 128 lanes x 512 columns
  uint32_t tmemUsed = 0;
};

struct EmuThread {
  emu_dim3 tid, bid, bdim, gdim;
  EmuCta* cta = nullptr;
};

inline thread_local EmuThread emu_t;

#define threadIdx (emu_t.tid)
#define blockIdx (emu_t.bid)
#define blockDim (emu_t.bdim)
#define gridDim (emu_t.gdim)

inline void __syncthreads() { emu_t.cta->bar->arrive_and_wait(); }
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }

inline void* emu_static_shared(int id, size_t bytes) {
  std::lock_guard<std::mutex> g(emu_t.cta->m);
  auto& v = emu_t.cta->stat[id];
  if (v.empty()) { v.assign(bytes + 16, 0); }
  return v.data();
}

#define OWL_DYN_SHARED(T, name) T* name = reinterpret_cast<T*>(emu_t.cta->dyn.data())
#define OWL_SHARED(T, name) T& name = *reinterpret_cast<T*>(emu_static_shared(__COUNTER__, sizeof(T)))
#define OWL_SHARED_ARR(T, name, n) T* name = reinterpret_cast<T*>(emu_static_shared(__COUNTER__, sizeof(T) * (n)))

template <typename T> inline T __ldg(const T* p) { return *p; }
template <typename T> inline T __ldcg(const T* p) { return *p; }

inline long long __double_as_longlong(double d) { return std::bit_cast<long long>(d); }
inline double __longlong_as_double(long long x) { return std::bit_cast<double>(x); }
inline unsigned __float_as_uint(float f) { return std::bit_cast<unsigned>(f); }
inline long long __double2ll_rn(double x) { return std::llrint(x); }
inline double __hiloint2double(int hi, int lo) {
  return std::bit_cast<double>(((uint64_t)(uint32_t)hi << 32) | (uint32_t)lo);
}
inline unsigned __byte_perm(unsigned x, unsigned y, unsigned s) {
  const uint64_t v = ((uint64_t)y << 32) | x;
  unsigned r = 0;
  for (int i = 0; i < 4; ++i) { r |= (unsigned)((v >> (8 * ((s >> (4 * i)) & 7))) & 0xff) << (8 * i); }
  return r;
}
struct uint4 {
  unsigned x, y, z, w;
};
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }

template <typename T> inline T emu_shfl_xor(T v, int o) {
  EmuCta* c = emu_t.cta;
  int t = (int)emu_t.tid.x;
  int w = t / 32;
  static_assert(sizeof(T) <= 8, "shfl size");
  uint64_t bits = 0;
  std::memcpy(&bits, &v, sizeof(T));
  c->slots[t] = bits;
  c->warpBar[w]->arrive_and_wait();
  int src = t ^ o;
  uint64_t got = (src < c->nthreads && src / 32 == w) ? c->slots[src] : bits;
  c->warpBar[w]->arrive_and_wait();
  T r;
  std::memcpy(&r, &got, sizeof(T));
  return r;
}
template <typename T> inline T __shfl_xor_sync(unsigned, T v, int o) { return emu_shfl_xor(v, o); }

inline bool __all_sync(unsigned, bool pred) {
  EmuCta* c = emu_t.cta;
  int t = (int)emu_t.tid.x;
  int w = t / 32;
  c->slots[t] = pred ? 1 : 0;
  c->warpBar[w]->arrive_and_wait();
  bool all = true;
  for (int i = w * 32; i < std::min(c->nthreads, w * 32 + 32); ++i) { all &= (c->slots[i] != 0); }
  c->warpBar[w]->arrive_and_wait();
  return all;
}

inline unsigned atomicAdd(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).fetch_add(v); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
  return std::atomic_ref<unsigned long long>(*p).fetch_add(v);
}
inline unsigned atomicExch(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).exchange(v); }
inline unsigned atomicOr(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).fetch_or(v); }
inline int atomicAnd(int* p, int v) { return std::atomic_ref<int>(*p).fetch_and(v); }
inline unsigned long long atomicMin(unsigned long long* p, unsigned long long v) {
  std::atomic_ref<unsigned long long> a(*p);
  unsigned long long cur = a.load();
  while (cur > v && !a.compare_exchange_weak(cur, v)) {
  }
  return cur;
}
inline unsigned long long atomicMax(unsigned long long* p, unsigned long long v) {
  std::atomic_ref<unsigned long long> a(*p);
  unsigned long long cur = a.load();
  while (cur < v && !a.compare_exchange_weak(cur, v)) {
  }
  return cur;
}
inline unsigned atomicMax(unsigned* p, unsigned v) {
  std::atomic_ref<unsigned> a(*p);
  unsigned cur = a.load();
  while (cur < v && !a.compare_exchange_weak(cur, v)) {
  }
  return cur;
}

namespace owl {
inline uint32_t ld_acquire(const uint32_t* p) {
  return std::atomic_ref<uint32_t>(*const_cast<uint32_t*>(p)).load(std::memory_order_acquire);
}
inline void st_release(uint32_t* p, uint32_t v) { std::atomic_ref<uint32_t>(*p).store(v, std::memory_order_release); }
inline long long ld_relaxed(const long long* p) {
  return std::atomic_ref<long long>(*const_cast<long long*>(p)).load(std::memory_order_relaxed);
}
inline void st_relaxed(long long* p, long long v) { std::atomic_ref<long long>(*p).store(v, std::memory_order_relaxed); }
inline unsigned long long gtimer() {
  return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
inline void spin_pause() { std::this_thread::yield(); }
inline void griddep_wait() {}
inline void griddep_launch() {}
inline unsigned long long l2_keep_policy() { return 0; }
inline double2 ld_state(const double2* p, unsigned long long) { return *p; }
inline void st_state(double2* p, double2 v, unsigned long long) { *p = v; }
}  // namespace owl

// Run `f` as a grid x block launch: every CUDA thread is a host thread with a
// small stack; all blocks run at once (the carry chain needs them live).
template <typename F> void emu_launch(unsigned grid, unsigned block, size_t dynSmem, F f) {
  std::vector<std::unique_ptr<EmuCta>> ctas;
  ctas.reserve(grid);
  for (unsigned g = 0; g < grid; ++g) {
    auto c = std::make_unique<EmuCta>();
    c->nthreads = (int)block;
    c->bar = std::make_unique<std::barrier<>>((std::ptrdiff_t)block);
    for (unsigned w = 0; w * 32 < block; ++w) {
      unsigned n = std::min(32u, block - w * 32);
      c->warpBar.push_back(std::make_unique<std::barrier<>>((std::ptrdiff_t)n));
    }
    c->slots.assign(block, 0);
    c->dyn.assign(dynSmem, 0);
    ctas.push_back(std::move(c));
  }
  struct Job {
    F* f;
    EmuThread t;
  };
  std::vector<Job> jobs(grid * (size_t)block);
  std::vector<pthread_t> th(jobs.size());
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, 1 << 20);
  for (unsigned g = 0; g < grid; ++g) {
    for (unsigned t = 0; t < block; ++t) {
      Job& j = jobs[(size_t)g * block + t];
      j.f = &f;
      j.t.tid.x = t;
      j.t.tid.y = j.t.tid.z = 0;
      j.t.bid.x = g;
      j.t.bid.y = j.t.bid.z = 0;  // one-dimensional grids (a grouped launch of one plan)
      j.t.bdim.x = block;
      j.t.gdim.x = grid;
      j.t.cta = ctas[g].get();
      int rc = pthread_create(
          &th[(size_t)g * block + t], &attr,
          [](void* arg) -> void* {
            Job* jj = static_cast<Job*>(arg);
            emu_t = jj->t;
            (*jj->f)();
            return nullptr;
          },
          &j);
      if (rc != 0) { throw std::runtime_error("pthread_create failed"); }
    }
  }
  for (auto& x : th) { pthread_join(x, nullptr); }
  pthread_attr_destroy(&attr);
}
