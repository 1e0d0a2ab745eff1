// owl_compat.cuh -- the few CUDA spellings the kernels use that differ when
// the same source is compiled as host C++ for the CPU kernel emulator
// (tests/emu, built with -DOWL_EMU). The product build never defines OWL_EMU.
#pragma once

#ifdef OWL_EMU
#include "owl_emu_rt.hpp"
#else
#include <cuda_runtime.h>
#include <cstdint>

#define OWL_DYN_SHARED(T, name) extern __shared__ T name[]
#define OWL_SHARED(T, name) __shared__ T name
#define OWL_SHARED_ARR(T, name, n) __shared__ T name[n]

namespace owl {
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// a carry word, read and written by single threads of different CTAs without further ordering: each
// word carries its own validity (nonzero), so no fence or flag orders it against other data
__device__ __forceinline__ long long ld_relaxed(const long long* p) {
  long long v;
  asm volatile("ld.relaxed.gpu.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(long long* p, long long v) {
  asm volatile("st.relaxed.gpu.global.s64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// the carry lookback polls without sleeping: each poll is already an L2 round trip, and a
// __nanosleep between polls measured 1.4 us slower per line pass at 8M
__device__ __forceinline__ void spin_pause() {}

// Programmatic dependent launch. A kernel launched with programmatic stream serialization may be
// scheduled while the previous kernel on its stream is still finishing: griddep_wait() returns once
// that kernel has completed and its memory operations are visible (at once for a normal launch).
// griddep_launch() allows the next such kernel to be scheduled once every CTA of this one has
// called it (or exited).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// The FFT state is streamed through L1 without allocating (so that the twiddle
// and weight tables stay resident) and kept in L2 with evict-last priority: at
// 8M words the 64 MiB state fits in the 126 MB L2 between the two passes.
__device__ __forceinline__ unsigned long long l2_keep_policy() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ double2 ld_state(const double2* ptr, unsigned long long pol) {
  double2 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
               : "=d"(v.x), "=d"(v.y)
               : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_state(double2* ptr, double2 v, unsigned long long pol) {
  asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(ptr), "d"(v.x), "d"(v.y),
               "l"(pol)
               : "memory");
}
}  // namespace owl
#endif
