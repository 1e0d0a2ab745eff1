// owl_tc.cuh -- the fifth-generation tensor-core primitives (tcgen05) the
// split-precision column pass uses: tensor-memory allocation, the INT8 MMA with
// both operands in shared memory, its completion barrier and the tensor-memory
// reads of the INT32 accumulators.
//
// Shared-memory operands are K-major; smem_desc describes either the no-swizzle canonical layout (a
// "core matrix" of 8 rows x 16 bytes stored as 128 contiguous bytes, core matrices SBO bytes apart
// along M/N and LBO bytes apart along K) or the 64-byte swizzled one (sw64_off).
//
// With -DOWL_EMU (the CPU kernel emulator in tests/emu) the same calls run on
// an emulated per-CTA tensor memory, and the MMA decodes its descriptors with
// the layout above, so the descriptor and digit-layout arithmetic of the
// kernels is exercised on the CPU as well.
#pragma once
#include <cstdint>

#include "owl_compat.cuh"

namespace owl {
namespace tc {

// instruction descriptor of tcgen05.mma kind::i8: signed A and B, INT32
// accumulator, both operands K-major, dense
constexpr uint32_t idesc_s8(int M, int N) {
  return (2u << 4)                      // D format: S32
         | (1u << 7)                    // A format: signed 8-bit
         | (1u << 10)                   // B format: signed 8-bit
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// shared-memory matrix descriptor, sm100 version field = 1; layout 0 = no swizzle, 4 = 64-byte swizzle
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout = 0) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
// 64-byte swizzle of a K-major operand with 64-byte rows in 512-byte atoms of 8 rows (the atom
// 1024-byte aligned): the 16-byte chunk c of row r is stored at chunk c ^ ((r % 8) / 2)
__host__ __device__ constexpr uint32_t sw64_off(int row, int kb) {
  return (uint32_t)((row / 8) * 512 + (row % 8) * 64 + (((kb / 16) ^ ((row % 8) >> 1)) * 16) + kb % 16);
}

__device__ __forceinline__ double exp2i(int k) { return __longlong_as_double((long long)(1023 + k) << 52); }
// exact int32 -> double without the conversion unit: 2^52 + 2^31 + v built from its bits, minus 2^52 + 2^31
__device__ __forceinline__ double i32_to_f64(int32_t v) {
  return __hiloint2double(0x43300000, (int)((uint32_t)v ^ 0x80000000u)) - 4503601774854144.0;
}

#ifndef OWL_EMU

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// warp-collective: allocate ncols tensor-memory columns, base address written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[taddr] = (acc ? D : 0) + A * B^T, M x N x 32 bytes of K, issued by one thread
__device__ __forceinline__ void mma_s8(uint32_t taddr, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)acc)
      : "memory");
}
// the barrier's pending arrival completes when every MMA this thread issued before has finished
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// waits for the phase of the given parity to complete; false after timeoutNs
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long timeoutNs) {
  const uint32_t a = smem_addr(bar);
  const unsigned long long t0 = gtimer();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) { return true; }
    if ((it & 63u) == 63u && gtimer() - t0 > timeoutNs) { return false; }
  }
  return false;
}
// warp-collective: 32 lanes x 16 consecutive 32-bit columns; this thread gets lane (taddr lane + laneid)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
// warp-collective: 32 lanes x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

#else  // OWL_EMU: emulated tensor memory and MMA (test infrastructure)

inline uint32_t smem_addr(const void* p) {
  return (uint32_t)(static_cast<const char*>(p) - emu_t.cta->dyn.data());
}
inline void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  if ((emu_t.tid.x & 31) != 0) { return; }
  EmuCta* c = emu_t.cta;
  std::lock_guard<std::mutex> g(c->m);
  if (c->tmem.empty()) { c->tmem.assign(128 * 512, 0xdeadbeefu); }
  if (c->tmemUsed + ncols > 512) { throw std::runtime_error("emu: tensor memory over-allocated"); }
  *slot = c->tmemUsed;
  c->tmemUsed += ncols;
}
inline void tmem_relinquish() {}
inline void tmem_dealloc(uint32_t, uint32_t ncols) {
  if ((emu_t.tid.x & 31) != 0) { return; }
  std::lock_guard<std::mutex> g(emu_t.cta->m);
  emu_t.cta->tmemUsed -= ncols;
}
inline void fence_before() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void fence_after() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void fence_proxy_async() { std::atomic_thread_fence(std::memory_order_seq_cst); }

inline void mma_s8(uint32_t taddr, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool acc) {
  EmuCta* c = emu_t.cta;
  if (idesc != idesc_s8((int)(((idesc >> 24) & 31u) << 4), (int)(((idesc >> 17) & 63u) << 3))) {
    throw std::runtime_error("emu: unexpected instruction descriptor");
  }
  const int M = (int)(((idesc >> 24) & 31u) << 4), N = (int)(((idesc >> 17) & 63u) << 3);
  auto decode = [&](uint64_t d, int rows, const char* what) {
    const uint32_t layout = (uint32_t)(d >> 61);
    if (((d >> 46) & 3u) != 1u || (layout != 0u && layout != 4u) || ((d >> 49) & 7u) != 0u) {
      throw std::runtime_error(std::string("emu: bad descriptor ") + what);
    }
    const uint32_t start = (uint32_t)(d & 0x3FFFu) << 4, lbo = (uint32_t)((d >> 16) & 0x3FFFu) << 4,
                   sbo = (uint32_t)((d >> 32) & 0x3FFFu) << 4;
    if (layout == 4u && (sbo != 512u || ((start & 1023u) & ~63u) != 0u)) {
      throw std::runtime_error(std::string("emu: 64-byte swizzle needs 512-byte atoms at an aligned base ") + what);
    }
    const size_t last = layout == 4u ? (size_t)start + (size_t)(rows / 8 - 1) * sbo + 511
                                     : (size_t)start + (size_t)(rows / 8 - 1) * sbo + lbo + 127;
    if (last >= c->dyn.size()) { throw std::runtime_error(std::string("emu: descriptor past smem ") + what); }
    return [=](int row, int k) -> int8_t {
      size_t off;
      if (layout == 4u) {
        // rows of 64 bytes; the start may point inside the row (a later k-step); the XOR of the
        // 16-byte chunk index with address bits 7-8 applies to the absolute address
        off = start + (size_t)(row / 8) * sbo + (size_t)(row % 8) * 64 + (size_t)k;
        off ^= ((off >> 7) & 3u) << 4;
      } else {
        off = start + (size_t)(row / 8) * sbo + (size_t)(row % 8) * 16 + (size_t)(k / 16) * lbo + (k % 16);
      }
      return static_cast<int8_t>(c->dyn[off]);
    };
  };
  auto A = decode(adesc, M, "A");
  auto B = decode(bdesc, N, "B");
  const uint32_t lane0 = taddr >> 16, col0 = taddr & 0xFFFFu;
  if (lane0 != 0 || col0 + N > 512) { throw std::runtime_error("emu: MMA accumulator out of range"); }
  for (int m = 0; m < M; ++m) {
    for (int n = 0; n < N; ++n) {
      int32_t s = 0;
      for (int k = 0; k < 32; ++k) { s += (int32_t)A(m, k) * (int32_t)B(n, k); }
      uint32_t& d = c->tmem[(size_t)m * 512 + col0 + n];
      d = (uint32_t)((acc ? (int32_t)d : 0) + s);
    }
  }
}
inline void commit(uint64_t* bar) { std::atomic_ref<uint64_t>(*bar).fetch_add(1); }
inline void mbar_init(uint64_t* bar, uint32_t) { std::atomic_ref<uint64_t>(*bar).store(0); }
// the emulated barrier counts completed phases; the phase of parity P is done once the count's parity differs
inline bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long timeoutNs) {
  const unsigned long long t0 = gtimer();
  while ((std::atomic_ref<uint64_t>(*bar).load() & 1u) == parity) {
    if (gtimer() - t0 > timeoutNs) { return false; }
    std::this_thread::yield();
  }
  return true;
}
inline void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  EmuCta* c = emu_t.cta;
  const uint32_t w = emu_t.tid.x / 32, lane = emu_t.tid.x % 32;
  const uint32_t lane0 = taddr >> 16, col0 = taddr & 0xFFFFu;
  if (lane0 != 32 * (w % 4) || col0 + 16 > 512) { throw std::runtime_error("emu: tensor-memory read out of range"); }
  for (int i = 0; i < 16; ++i) { r[i] = c->tmem[(size_t)(lane0 + lane) * 512 + col0 + i]; }
}
inline void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  EmuCta* c = emu_t.cta;
  const uint32_t w = emu_t.tid.x / 32, lane = emu_t.tid.x % 32;
  const uint32_t lane0 = taddr >> 16, col0 = taddr & 0xFFFFu;
  if (lane0 != 32 * (w % 4) || col0 + 8 > 512) { throw std::runtime_error("emu: tensor-memory read out of range"); }
  for (int i = 0; i < 8; ++i) { r[i] = c->tmem[(size_t)(lane0 + lane) * 512 + col0 + i]; }
}
inline void tmem_wait_ld() {}

#endif

}  // namespace tc
}  // namespace owl
