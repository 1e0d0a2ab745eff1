/*
 * owl.h -- C ABI of libowl, the B200 (sm_100a) engine for the PRP/LL iteration
 * x <- x^2 (or x^2 - 2) mod 2^E - 1 as an IBDWT squaring with fused carry.
 *
 * This boundary replaces the reference's OpenCL device layer (clwrap/Kernel/
 * KernelCompiler/Queue/Buffer, reference src/clwrap.h:54-68, src/Kernel.h:17-79,
 * src/Queue.h:41-53, src/Buffer.h:16-102) and the kernel-level methods of its
 * Gpu class (src/Gpu.h:213-300). Plain C types only; every call returns an int
 * status (OWL_OK or a negative OWL_ERR_*), where the reference threw strings
 * (src/clwrap.cpp:57-62) -- owl_error_string() and owl_last_error() give text.
 *
 * Data model. A "word buffer" is N int32 balanced digits in natural word order
 * on the plan's device (the reference's Buffer<int> bufData/bufCheck/bufAux,
 * src/Gpu.h:165-175; the reference keeps them in a transposed device layout and
 * converts in transposeIn/Out, src/cl/transpose.cl:31-40 -- here the natural
 * order is the device layout). Compact words are the E-bit little-endian u32
 * form of src/state.cpp:26-69 (nWords = (E-1)/32+1).
 *
 * Threading: a plan owns one CUDA stream and its FFT work buffers; calls on the
 * same plan must not run concurrently. Different plans (same or different
 * devices) are independent.
 */
#ifndef OWL_H
#define OWL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OWL_ABI_VERSION 1

enum {
  OWL_OK = 0,
  OWL_ERR_ARG = -1,      /* bad argument / shape not supported */
  OWL_ERR_NOMEM = -2,    /* device or host allocation failed (reference: bad_alloc, src/clwrap.cpp:286-293) */
  OWL_ERR_CUDA = -3,     /* CUDA runtime error */
  OWL_ERR_TIMEOUT = -4,  /* a device-side wait (carry lookback) gave up; results of that call are invalid */
  OWL_ERR_NODEV = -5,    /* no such device */
  OWL_ERR_READ = -6      /* checked read failed 3 times (reference "GPU persistent read errors", src/Gpu.cpp:677-705) */
};

/* flags for owl_square */
#define OWL_SQ_MUL3 1u /* multiply the result of the LAST squaring by 3 (src/Gpu.cpp:936-945 doTailMul3) */
#define OWL_SQ_LL 2u   /* LL step x^2 - 2 on every squaring (src/Gpu.cpp:1586-1663, src/cl/carryfused.cl:120-123) */
/* no round-off measurement in these squarings: the reference measures it on a sample of iterations
   only (wantROE: 2,000 after the first 30, then 400 per log step, src/Gpu.cpp:1026, 1459-1464; the
   kernel build without it, kCarryFused, src/Gpu.cpp:592-596); owl_read_roe gets no entries for them */
#define OWL_SQ_NO_ROE 4u

typedef struct owl_plan owl_plan;

int owl_abi_version(void);
const char* owl_error_string(int status);
/* text of the last error raised on this thread */
const char* owl_last_error(void);

/* Device enumeration -- reference getAllDeviceIDs/getDevice/Context (src/clwrap.h:54-68,
   src/clwrap.cpp:189-200). pci_bus_id replaces the AMD sysfs lookup in src/gpuid.cpp. */
int owl_device_count(int* count);
int owl_device_info(int ordinal, char* name, size_t name_len, size_t* total_mem, char* pci_bus_id, size_t pci_len);

/* FFT choice -- reference FFTConfig::bestFit (src/FFTConfig.cpp:235-263): the smallest
   supported N = 2*W*H (W, H powers of two in [64, 4096]) with E/N <= max_bpw
   (max_bpw <= 0 selects the default limit). */
int owl_fft_choose(uint32_t E, double max_bpw, uint32_t* N, uint32_t* W, uint32_t* H);

/* Plan = one exponent on one device with its tables and work buffers -- the reference's
   Gpu constructor (src/Gpu.cpp:394-564: clDefines, genWeights, trig tables, buffers).
   W = H = 0 picks the shape with owl_fft_choose(E, 0). */
int owl_plan_create(int device, uint32_t E, uint32_t W, uint32_t H, owl_plan** out);
int owl_plan_destroy(owl_plan* plan);
int owl_plan_shape(const owl_plan* plan, uint32_t* N, uint32_t* W, uint32_t* H);
/* limit of every device-side wait, in nanoseconds (default 2 s) */
int owl_plan_set_timeout(owl_plan* plan, uint64_t ns);
/* Split-precision form (the reference has only FP64 kernels; this selects between two
   implementations of its tailSquare / fftMiddleIn / fftMiddleOut step, src/cl/tailsquare.cl:225-313,
   and of the width FFT in carryFused, src/cl/carryfused.cl:21-231). flags:
     OWL_SPLIT_COLUMNS  the first forward and last inverse stages of every column FFT (32-point at
                        H = 2048, 40-point at H = 2560)
     OWL_SPLIT_LINES    the first inverse and last forward stages of every line FFT (16-point at
                        W = 2048)
   run as INT8 tensor-core GEMMs on 7 base-256 digit planes of the FP64 operands (Ozaki-style),
   recombined exactly in FP64; 0 returns to the FP64 form. Results stay bit-exact while the
   round-off stays below 0.5 (owl_read_roe reports it). A flag whose pass has no split form at the
   plan's shape fails with OWL_ERR_ARG. Drops the plan's cached squaring graphs; a batch keeps the
   form its plans had when it first ran a block of that size, so set the form before building
   batches. */
#define OWL_SPLIT_COLUMNS 1u
#define OWL_SPLIT_LINES 2u
int owl_plan_set_split(owl_plan* plan, int flags);

/* Column-pass tile variant -- the reference's tune.txt carries, besides the FFT shape, the build
   options measured fastest for it (src/tune.cpp:106-186, src/TuneEntry.cpp:94-105); here the choice
   is between kernels built for the same shape with another radix plan and tile:
     OWL_COL_V16       16 values a thread, H/8 threads a CTA (every H)
     OWL_COL_V8         8 values a thread, H/4 threads a CTA, radix plan 8 x ... x 4
                        (H a power of two up to 2048, 640 or 1280)
     OWL_COL_V16_OCC2  16 values a thread at two CTAs per SM instead of one (H = 2560)
   OWL_COL_AUTO selects the shape's default (measured on B200, gpuowl_b200.tune --variants). All
   variants give bit-identical results while the round-off stays below 0.5. A plan starts with its
   shape's default. Setting a variant that is not built for the plan's H fails with OWL_ERR_ARG.
   Drops the plan's cached squaring graphs; like the split form, set it before building batches
   (plans of one shape and variant share a grouped launch). */
#define OWL_COL_AUTO 0u
#define OWL_COL_V16 1u
#define OWL_COL_V8 2u
#define OWL_COL_V16_OCC2 3u
int owl_plan_set_column_variant(owl_plan* plan, uint32_t variant);
int owl_plan_column_variant(const owl_plan* plan, uint32_t* variant);
/* 1 if the variant (not OWL_COL_AUTO) is built for columns of H points, else 0 */
int owl_column_variant_supported(uint32_t H, uint32_t variant);

/* Word buffers -- Buffer<int> (src/Buffer.h:16-102), AllocTrac accounting aside. */
int owl_buf_alloc(owl_plan* plan, int32_t** buf);
int owl_buf_free(owl_plan* plan, int32_t* buf);
/* dst := src (operator<<, src/Buffer.h) */
int owl_buf_copy(owl_plan* plan, int32_t* dst, const int32_t* src);
/* buf := small integer value (Buffer::set, used by exponentiate for exp == 0) */
int owl_buf_set(owl_plan* plan, int32_t* buf, uint32_t value);

/* Raw digit transfer (N int32). */
int owl_write_digits(owl_plan* plan, int32_t* buf, const int32_t* host);
int owl_read_digits(owl_plan* plan, const int32_t* buf, int32_t* host);
/* Compact words: Gpu::writeIn (expandBits, src/Gpu.cpp:801-811, src/state.cpp:93-115) and
   Gpu::readAndCompress (readChecked + compactBits, src/Gpu.cpp:677-710). The read is
   verified with a device-side 64-bit sum and retried up to 3 times. */
int owl_write_words(owl_plan* plan, int32_t* buf, const uint32_t* words);
int owl_read_words(owl_plan* plan, const int32_t* buf, uint32_t* words);

/* Gpu::squareLoop(out, in, 0, n, flags & MUL3) (src/Gpu.cpp:936-945) with Gpu::square's
   kernel chain (src/Gpu.cpp:903-932): n squarings of `in` into `out` (out may equal in).
   OWL_SQ_LL makes every step x^2 - 2 (squareLL); OWL_SQ_NO_ROE skips the round-off measurement. */
int owl_square(owl_plan* plan, int32_t* out, const int32_t* in, uint32_t n, uint32_t flags);
/* Gpu::modMul(ioA, inB, mul3) (src/Gpu.cpp:712-736): ioA := ioA * inB (* 3). */
int owl_modmul(owl_plan* plan, int32_t* io_a, const int32_t* in_b, int mul3);
/* A := A^h * B (reference Gpu::expMul on buffers, src/Gpu.cpp:833-837, with exponentiate's
   left-to-right binary powering, 858-889): A's spectrum is kept while A is squared and multiplied
   per bit of h. h = 0 gives A := B. A and B must differ. Used by proof generation and verification. */
int owl_exp_mul(owl_plan* plan, int32_t* io_a, uint64_t h, const int32_t* in_b);
/* Gpu::isEqual (src/Gpu.cpp:947-953, src/cl/etc.cl:34-41): digit-wise equality. */
int owl_is_equal(owl_plan* plan, const int32_t* a, const int32_t* b, int* equal);
/* Gpu::bufResidue (src/Gpu.cpp:955-975): res64 from the words around the wrap; falls
   back to the full compact form when the top 32 words cannot decide the carry. */
int owl_res64(owl_plan* plan, const int32_t* buf, uint64_t* res64);
/* sum64 kernel (src/cl/etc.cl:19-29): the buffer as N/2 u64, summed mod 2^64. */
int owl_sum64(owl_plan* plan, const int32_t* buf, uint64_t* sum);
/* Gpu::readROE (src/Gpu.cpp:624-637): per-squaring max |x - rint(x)| recorded since the
   last call (at most cap values; *n gets the count), then cleared. */
int owl_read_roe(owl_plan* plan, float* out, uint32_t cap, uint32_t* n);
/* wait for the plan's stream; reports a device-side wait timeout as OWL_ERR_TIMEOUT */
int owl_sync(owl_plan* plan);

/* The plan's CUDA stream (a cudaStream_t), so that callers can order their own work and
   record CUDA events on the stream the engine's kernels run on. */
int owl_plan_stream(owl_plan* plan, void** stream);

/* n squarings of buf (in place, n <= 2047) with per-kernel device time, the counterpart of the
   reference's -time profile (src/Gpu.cpp:773-799, src/Queue.cpp:54-58). The block runs as the
   same CUDA graph as owl_square; each kernel launch stamps its first CTA start and last CTA end
   with the GPU's global timer. ms[0] = total pass-2 (column) time, ms[1] = total pass-1
   (line/carry) time, ms[2] = entry and exit passes; launches[0..2] the matching counts. flags as
   for owl_square. */
int owl_profile_square(owl_plan* plan, int32_t* buf, uint32_t n, uint32_t flags, float* ms, uint32_t* launches);

/* Failure-detection probe: one device wait on a flag nothing sets, with the plan's
   timeout. Returns OWL_ERR_TIMEOUT (the expected outcome) and leaves the plan usable. */
int owl_probe_wait_timeout(owl_plan* plan);
/* Test hook of the split-precision pass's completion wait: waits on an mbarrier that nothing
   arrives on, with the plan's timeout; returns OWL_ERR_TIMEOUT and leaves the plan usable. */
int owl_probe_tc_wait_timeout(owl_plan* plan);

/* Batches of exponents of uneven FFT lengths (the reference runs 1-4 independent
   workers, each with its own in-order queue, src/main.cpp:111-118). A batch groups plans of one
   device, each with its own exponent and FFT shape; owl_batch_square runs n squarings of every
   plan's buffer as ONE CUDA-graph launch (one fork-join graph, a branch per plan, captured on
   first use and cached), so that small FFTs of different exponents share the GPU. The call is
   asynchronous; later calls on any of the plans are ordered after it. */
typedef struct owl_batch owl_batch;
int owl_batch_create(int device, uint32_t count, owl_plan* const* plans, owl_batch** out);
int owl_batch_square(owl_batch* batch, int32_t* const* bufs, uint32_t n, uint32_t flags);
int owl_batch_sync(owl_batch* batch);
int owl_batch_destroy(owl_batch* batch);

/* No counterpart in the reference (its host allocates every device buffer up front).
   n squarings (flags as for owl_square) of `words`, a device buffer of N = 2*W*H balanced int32
   digits on `device`, in place, queued on `stream` (a cudaStream_t of that device; NULL is the
   legacy default stream) -- without allocating anything. It is meant for callers that cannot call
   cudaMalloc: hosts whose device memory all belongs to their own pool allocator, real-time loops
   that must not block in the allocator, and plug-ins whose host forbids allocation. All scratch
   (FFT state, carry rows, tables) lives in one fixed 1 MiB device array inside libowl, present on
   every GPU that loads the library until the process exits, so only small FFTs fit: W in {64, 128},
   H in {64, 128, 256}, N <= 65536, at most 19 bits per word (W = H = 0 picks the smallest shape
   that holds E); anything larger returns OWL_ERR_ARG. Every call shares that array and it keeps
   the last call's contents: calls that overlap on the GPU race and corrupt each other. The first
   call on a device looks up the array's address with that device current; make it before any
   stream capture. The call waits for its work; a device-side wait timeout returns
   OWL_ERR_TIMEOUT, a round-off above 0.4 OWL_ERR_ARG; the error text is in owl_last_error(). */
int owl_square_noalloc(int device, uint32_t E, uint32_t W, uint32_t H, int32_t* words, uint32_t n,
                       uint32_t flags, void* stream);

#ifdef __cplusplus
}
#endif
#endif
