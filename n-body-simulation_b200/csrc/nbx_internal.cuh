// nbx_internal.cuh -- device-side building blocks shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "nbx_math.h"

namespace nbx {

// Error bits collected in the device status word (Handle::status).
enum StatusBits : uint32_t {
  kStatusOk = 0,
  kStatusSpinLimit = 1u << 0,    // a bounded wait gave up
  kStatusTreeCapacity = 1u << 1, // node capacity would have been exceeded
  kStatusPairCapacity = 1u << 2, // collision partner capacity exceeded
  kStatusNonFinite = 1u << 3,    // a body position became NaN/inf
  kStatusLargeCapacity = 1u << 4,
  kStatusBadSegment = 1u << 5,
};

// Iteration cap of every spin-wait in this library: each round polls memory
// (an L2 round trip) and backs off, so a wait gives up after about a
// second; legitimate waits here last microseconds.
constexpr uint32_t kSpinLimit = 1u << 21;

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// 16-byte relaxed accesses: each 32-bit word is single-copy atomic, so a
// reader that sees no sentinel word sees the whole record as written.
__device__ __forceinline__ float4 ld_relaxed_f4(const float4 *p) {
  float4 v;
  asm volatile("ld.relaxed.gpu.global.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p)
               : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f4(float4 *p, float4 v) {
  asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p),
               "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// A second stream for a phase's independent branch: the branch waits on
// `fork` recorded on the main stream and records `join` for the main stream
// to wait on (in a captured step graph: two parallel branches).
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// Optional phase markers: when a profiling step is running on this thread
// (nbx_profile_step), launch sequences record an event after each stage.
struct PhaseMarks {
  static constexpr int kMax = 48;
  cudaEvent_t ev[kMax];
  const char *label[kMax];
  int count = 0;
};
extern thread_local PhaseMarks *g_marks;
inline void mark(cudaStream_t s, const char *label) {
  if (g_marks && g_marks->count < PhaseMarks::kMax) {
    cudaEventRecord(g_marks->ev[g_marks->count], s);
    g_marks->label[g_marks->count++] = label;
  }
}

// Grid-stride helpers sized from a device-side count.
__device__ __forceinline__ uint32_t load_count(const uint32_t *d_n, uint32_t n) {
  return d_n ? *d_n : n;
}

// ---------------------------------------------------------------------
// Device-wide primitives (scan_sort.cu).  All take a stream and never
// synchronise with the host, so they can be captured in a CUDA graph.
struct ScanScratch {
  uint64_t *status = nullptr; // per tile: its sum (low 32 bits used)
  uint32_t *tileCounter = nullptr; // [kScanSlots] tile claims of the slots
  uint64_t *slotStatus = nullptr;  // [kScanSlots][maxTiles] look-back words
  uint32_t maxTiles = 0;
};
// Scans with a slot of their own (a step's four scans): one launch each,
// over look-back words and a tile counter that the step prologue clears.
constexpr int kScanSlots = 4;

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

// out[i] = sum(in[0..i)) for i < n; if total != nullptr it receives the sum.
// n is *d_n when d_n != nullptr (n_max bounds the launch).  With owner,
// owner[out[i] + k] = i for k < in[i] (below owner_cap): the element that
// each unit of the scanned counts belongs to.
// With slot >= 0 the scan is one launch (decoupled look-back over that
// slot's words, which must be clear: the step prologue clears all slots);
// otherwise two (tile sums, then every tile's prefix), needing nothing
// cleared.
void exclusive_scan_u32(cudaStream_t s, const uint32_t *in, uint32_t *out,
                        uint32_t n_max, const uint32_t *d_n, uint32_t *total,
                        ScanScratch &sc, uint32_t *err, uint32_t *owner = nullptr,
                        uint32_t owner_cap = 0, int slot = -1);
size_t scan_scratch_tiles(uint32_t n_max);

constexpr int kSortThreads = 256;
constexpr int kSortItems = 12;
constexpr int kSortTile = kSortThreads * kSortItems; // 3072
constexpr int kSortWarps = kSortThreads / 32;

struct SortScratch {
  uint64_t *keys[2] = {nullptr, nullptr};
  uint32_t *vals[2] = {nullptr, nullptr};
  uint32_t *hist = nullptr;        // [8 passes][256] digit counts
  uint32_t *status = nullptr;      // [8 passes][maxTiles][256] look-back words
  uint32_t *tileCounter = nullptr; // [8]
  uint32_t maxTiles = 0;
  uint32_t capacity = 0;
};

size_t sort_tiles(uint32_t n_max);
// Look-back words of one pass over n_max keys (one slot of scratch.status).
size_t sort_pass_words(uint32_t n_max);
// Scratch slots of a step's two sorts: the Morton codes' passes use slots
// 0-3, the contact units' slots 4-6 (cleared together by the step prologue).
constexpr int kUnitSortSlot = 4;

// Stable LSD radix sort of (keys[0], vals[0]) on key bits [bit_lo, bit_hi)
// (multiples of 8).  If `have_hist` the caller already filled the digit
// counts for those passes (e.g. fused into the key-producing kernel).
// vals_identity: vals[0] is not read, value = original index.  The passes
// use the scratch's digit rows, look-back slots and tile counters from
// `slot` on (pass p of the key: row slot + bit_lo / 8 + p, slot and counter
// slot + p); with `zeroed` the caller has cleared those (the step
// prologue), else the sort does.  Returns the buffer index (0/1) holding
// the result.
int radix_sort_u64(cudaStream_t s, SortScratch &sc, uint32_t n_max,
                   const uint32_t *d_n, int bit_lo, int bit_hi,
                   bool vals_identity, bool have_hist, uint32_t *err,
                   int slot = 0, bool zeroed = false);

// The same sort with 32-bit keys, held in the key buffers' storage
// (keys32): two thirds of the bytes per pass of 64-bit keys.
inline uint32_t *keys32(SortScratch &sc, int buf) {
  return reinterpret_cast<uint32_t *>(sc.keys[buf]);
}
int radix_sort_u32(cudaStream_t s, SortScratch &sc, uint32_t n_max,
                   const uint32_t *d_n, int bit_lo, int bit_hi,
                   bool vals_identity, bool have_hist, uint32_t *err,
                   int slot = 0, bool zeroed = false);

// Completes a stable sort of 64-bit codes that ran its radix passes on the
// high 32 bits only (keys32(sc, buf) = codes[vals] >> 32, sorted): every run
// of equal keys is put in order of the low 32 bits of codes[vals], stably,
// in place.  longRuns holds cap run starts; *runCount is device scratch.
void sort_fix_low_bits32(cudaStream_t s, SortScratch &sc, int buf, uint32_t n,
                         const uint64_t *codes, uint32_t *longRuns, uint32_t *runCount,
                         uint32_t cap, uint32_t *err, bool zeroed = false);

// The same for the contact units, whose radix passes ran on a coarse,
// order-preserving key of the box's minX: every run of equal coarse keys
// (but the `skip` run of non-units) is put in order of the exact minX
// order key, stably (ties keep index order).
void sort_fix_units(cudaStream_t s, SortScratch &sc, int buf, uint32_t n, const float4 *box,
                    uint32_t skip, uint32_t *longRuns, uint32_t *runCount, uint32_t cap,
                    uint32_t *err, bool zeroed = false);

} // namespace nbx
