// scan_sort.cu -- exclusive scan and onesweep LSD radix sort.
//
// The scan reduces every tile first and then lets each tile add the sums
// of the tiles before it: two launches with no dependence between tiles.
// A step's own scans, whose look-back words the step prologue clears, run
// as one launch with decoupled look-back instead.
// The radix sort uses decoupled look-back (Merrill & Garland 2016; Adinets &
// Merrill 2022, "Onesweep"): tiles are claimed in order through an atomic
// counter, each tile publishes its digit counts, and looks back over its
// predecessors' published words until it finds an inclusive prefix.  Every
// wait is bounded (kSpinLimit); on expiry the kernel raises
// kStatusSpinLimit in the caller's status word and carries on with what it
// has, so a stuck predecessor can never hang the GPU.
//
// The radix sort is stable (ranks within a warp come from the lanes sharing
// a digit, found with one ballot per digit bit, over warp-striped items in
// input order), so equal keys keep their input order exactly as
// cub::DeviceRadixSort::SortPairs does (CudaQuadTree.cu:405-407), which the
// Morton permutation parity needs.
#include "nbx_internal.cuh"

namespace nbx {

// ------------------------------------------------------------------ scan
namespace {


// The tiles' items pass through shared memory between coalesced global
// accesses (item k * threads + t) and each thread's run of consecutive
// items (t * items + k); one padding word per 32 keeps both conflict-free
// (a run's start moves one bank per thread instead of 16).
constexpr int kScanPadded = kScanTile + kScanTile / 32;
__device__ __forceinline__ int scan_pad(int i) { return i + (i >> 5); }

// Reduce-then-apply scan: the tile sums first (no dependence between
// tiles), then every tile adds the sums of the tiles before it (read from
// L2, summed in shared memory) and scans its items.  Two launches and no
// look-back chain, whose length grows with the number of tiles.
__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, uint32_t *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  uint32_t t = 0;
  for (int w = 0; w < kScanThreads / 32; ++w) t += sh[w];
  return t;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_reduce(const uint32_t *__restrict__ in, uint32_t n_max, const uint32_t *d_n,
                  uint32_t *__restrict__ tileSum) {
  __shared__ uint32_t sh[kScanThreads / 32];
  const uint32_t n = load_count(d_n, n_max);
  const uint32_t base = blockIdx.x * kScanTile;
  if (base >= n) return;
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const uint32_t i = base + k * kScanThreads + threadIdx.x;
    if (i < n) v += in[i];
  }
  const uint32_t t = block_sum_u32(v, sh);
  if (threadIdx.x == 0) tileSum[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_apply(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                 uint32_t n_max, const uint32_t *d_n, uint32_t *total,
                 const uint32_t *__restrict__ tileSum, uint32_t *__restrict__ owner,
                 uint32_t ownerCap) {
  __shared__ uint32_t s_items[kScanPadded];
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t sh[kScanThreads / 32];
  const int tid = threadIdx.x;
  const uint32_t n = load_count(d_n, n_max);
  const uint32_t numTiles = (n + kScanTile - 1) / kScanTile;
  const uint32_t tile = blockIdx.x;
  if (n == 0) {
    if (tile == 0 && tid == 0 && total) *total = 0;
    return;
  }
  if (tile >= numTiles) return;
  uint32_t pre = 0;
  for (uint32_t t = tid; t < tile; t += kScanThreads) pre += tileSum[t];
  const uint32_t excl = block_sum_u32(pre, sh);
  const uint32_t base = tile * kScanTile;
  for (int k = 0; k < kScanItems; ++k) {
    const uint32_t i = base + k * kScanThreads + tid;
    s_items[scan_pad(k * kScanThreads + tid)] = i < n ? in[i] : 0u;
  }
  __syncthreads();
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = s_items[scan_pad(tid * kScanItems + k)];
    sum += v[k];
  }
  const int lane = tid & 31, warp = tid >> 5;
  uint32_t inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  uint32_t woff = 0, blockTotal = 0;
  for (int w = 0; w < kScanThreads / 32; ++w) {
    if (w < warp) woff += s_warp[w];
    blockTotal += s_warp[w];
  }
  if (total && tile == numTiles - 1 && tid == 0) *total = excl + blockTotal;
  uint32_t run = excl + woff + (inc - sum);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s_items[scan_pad(tid * kScanItems + k)] = run;
    run += v[k];
  }
  __syncthreads();
  for (int k = 0; k < kScanItems; ++k) {
    const uint32_t i = base + k * kScanThreads + tid;
    if (i < n) {
      const uint32_t o = s_items[scan_pad(k * kScanThreads + tid)];
      out[i] = o;
      if (owner) {
        const uint32_t c = in[i];
        for (uint32_t j = 0; j < c && o + j < ownerCap; ++j) owner[o + j] = i;
      }
    }
  }
}

// One-launch scan: tiles are claimed in launch order through the slot's
// counter; each publishes its sum at once, and warp 0 looks back over its
// predecessors' words (32 per round trip) until it meets an inclusive sum,
// then publishes its own inclusive sum.  Every wait is bounded.
constexpr uint64_t kScanAggregate = 1ull << 32, kScanInclusive = 2ull << 32;

__global__ void __launch_bounds__(kScanThreads)
    k_scan_onepass(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                   uint32_t n_max, const uint32_t *d_n, uint32_t *total, uint64_t *status,
                   uint32_t *tileCounter, uint32_t *__restrict__ owner, uint32_t ownerCap,
                   uint32_t *err) {
  __shared__ uint32_t s_items[kScanPadded];
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_tile, s_excl;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(tileCounter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t n = load_count(d_n, n_max);
  const uint32_t numTiles = (n + kScanTile - 1) / kScanTile;
  if (n == 0) {
    if (tile == 0 && tid == 0 && total) *total = 0;
    return;
  }
  if (tile >= numTiles) return;
  const uint32_t base = tile * kScanTile;
  for (int k = 0; k < kScanItems; ++k) {
    const uint32_t i = base + k * kScanThreads + tid;
    s_items[scan_pad(k * kScanThreads + tid)] = i < n ? in[i] : 0u;
  }
  __syncthreads();
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = s_items[scan_pad(tid * kScanItems + k)];
    sum += v[k];
  }
  uint32_t inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  uint32_t woff = 0, blockTotal = 0;
  for (int w = 0; w < kScanThreads / 32; ++w) {
    if (w < warp) woff += s_warp[w];
    blockTotal += s_warp[w];
  }
  if (warp == 0) {
    uint32_t excl = 0;
    if (tile == 0) {
      if (lane == 0) st_relaxed_u64(status, kScanInclusive | blockTotal);
    } else {
      if (lane == 0) st_relaxed_u64(status + tile, kScanAggregate | blockTotal);
      int pred = (int)tile - 1;
      uint32_t spins = 0;
      for (;;) {
        const int q = pred - lane;
        const uint64_t w = q >= 0 ? ld_relaxed_u64(status + q) : kScanInclusive;
        const uint32_t flag = (uint32_t)(w >> 32);
        const uint32_t ready = __ballot_sync(0xffffffffu, flag != 0u);
        const uint32_t incl = __ballot_sync(0xffffffffu, flag == 2u);
        // the lanes up to the nearest inclusive word, which must all be
        // published; all 32 when none is inclusive yet
        const uint32_t upto = incl ? (incl & (0u - incl)) * 2u - 1u : 0xffffffffu;
        if ((ready & upto) == upto) {
          uint32_t x = (upto >> lane) & 1u ? (uint32_t)w : 0u;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
          excl += x;
          if (incl) break;
          pred -= 32;
        } else if (++spins > kSpinLimit) {
          if (lane == 0) atomicOr(err, kStatusSpinLimit);
          break;
        } else {
          __nanosleep(32);
        }
      }
      if (lane == 0) st_relaxed_u64(status + tile, kScanInclusive | (uint32_t)(excl + blockTotal));
    }
    if (lane == 0) s_excl = excl;
  }
  __syncthreads();
  const uint32_t excl = s_excl;
  if (total && tile == numTiles - 1 && tid == 0) *total = excl + blockTotal;
  uint32_t run = excl + woff + (inc - sum);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s_items[scan_pad(tid * kScanItems + k)] = run;
    run += v[k];
  }
  __syncthreads();
  for (int k = 0; k < kScanItems; ++k) {
    const uint32_t i = base + k * kScanThreads + tid;
    if (i < n) {
      const uint32_t o = s_items[scan_pad(k * kScanThreads + tid)];
      out[i] = o;
      if (owner) {
        const uint32_t c = in[i];
        for (uint32_t j = 0; j < c && o + j < ownerCap; ++j) owner[o + j] = i;
      }
    }
  }
}

} // namespace

size_t scan_scratch_tiles(uint32_t n_max) {
  return (n_max + kScanTile - 1) / kScanTile + 1;
}

void exclusive_scan_u32(cudaStream_t s, const uint32_t *in, uint32_t *out,
                        uint32_t n_max, const uint32_t *d_n, uint32_t *total,
                        ScanScratch &sc, uint32_t *err, uint32_t *owner,
                        uint32_t owner_cap, int slot) {
  const uint32_t tiles = (n_max + kScanTile - 1) / kScanTile;
  if (slot >= 0) {
    k_scan_onepass<<<tiles > 0 ? tiles : 1, kScanThreads, 0, s>>>(
        in, out, n_max, d_n, total, sc.slotStatus + (size_t)slot * sc.maxTiles,
        sc.tileCounter + slot, owner, owner_cap, err);
    return;
  }
  uint32_t *tileSum = reinterpret_cast<uint32_t *>(sc.status);
  // a single tile adds no earlier tile sums: no reduce pass
  if (tiles > 1)
    k_scan_reduce<<<tiles, kScanThreads, 0, s>>>(in, n_max, d_n, tileSum);
  k_scan_apply<<<tiles > 0 ? tiles : 1, kScanThreads, 0, s>>>(in, out, n_max, d_n, total,
                                                               tileSum, owner, owner_cap);
}

// ------------------------------------------------------------ radix sort
namespace {

constexpr uint32_t kRFlagShift = 30;
constexpr uint32_t kRValueMask = (1u << 30) - 1;

template <typename K>
__global__ void k_radix_hist(const K *__restrict__ keys, uint32_t n_max,
                             const uint32_t *d_n, int pass_lo, int passes,
                             uint32_t *__restrict__ hist) {
  __shared__ uint32_t sh[8][256];
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
    sh[i / 256][i % 256] = 0;
  __syncthreads();
  const uint32_t n = load_count(d_n, n_max);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const K k = keys[i];
    for (int p = 0; p < passes; ++p)
      atomicAdd(&sh[p][(k >> (8 * (pass_lo + p))) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    const uint32_t v = sh[i / 256][i % 256];
    if (v) atomicAdd(&hist[(pass_lo + i / 256) * 256 + i % 256], v);
  }
}

// At least 3 blocks per SM (<= 85 registers): a 1M-key pass (342 tiles)
// is then resident in one wave on 148 SMs.
template <typename K, bool kIdentity>
__global__ void __launch_bounds__(kSortThreads, 3)
    k_onesweep(const K *__restrict__ keysIn,
               const uint32_t *__restrict__ valsIn,
               K *__restrict__ keysOut, uint32_t *__restrict__ valsOut,
               const uint32_t *__restrict__ digitCount, uint32_t *status,
               uint32_t *tileCounter, uint32_t n_max, const uint32_t *d_n,
               int shift, uint32_t *err) {
  __shared__ K s_keys[kSortTile];
  __shared__ uint32_t s_vals[kSortTile];
  __shared__ uint32_t s_whist[kSortWarps][256];
  __shared__ uint32_t s_local[256];  // local exclusive digit start in tile
  __shared__ uint32_t s_global[256]; // global start of digit for this tile
  __shared__ uint32_t s_tile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t n = load_count(d_n, n_max);
  const uint32_t numTiles = (n + kSortTile - 1) / kSortTile;
  if (tid == 0) s_tile = atomicAdd(tileCounter, 1u);
  for (int i = tid; i < kSortWarps * 256; i += kSortThreads)
    s_whist[i / 256][i % 256] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  if (tile >= numTiles) return;
  // the pass's count of digit tid over the whole array (kSortThreads == 256)
  const uint32_t digitTotal = digitCount[tid];
  const uint32_t base = tile * kSortTile;
  const uint32_t wbase = base + warp * (kSortItems * 32);

  K key[kSortItems];
  uint32_t val[kSortItems];
  uint32_t rank[kSortItems];
  uint32_t dig[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t i = wbase + k * 32 + lane;
    const bool ok = i < n;
    key[k] = ok ? keysIn[i] : (K)0;
    val[k] = ok ? (kIdentity ? i : valsIn[i]) : 0u;
    dig[k] = ok ? (uint32_t)((key[k] >> shift) & 255u) : 256u;
  }
  const uint32_t ltmask = lanemask_lt();
  // lanes holding the same digit, from one ballot per digit bit (plus one
  // for validity); all items' masks first, so the ballots overlap
  uint32_t peer[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t d = dig[k];
    uint32_t m = __ballot_sync(0xffffffffu, d < 256u);
#pragma unroll
    for (int bit = 0; bit < 8; ++bit) {
      const uint32_t bb = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
      m &= ((d >> bit) & 1u) ? bb : ~bb;
    }
    peer[k] = m;
  }
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t d = dig[k];
    const uint32_t peers = peer[k];
    const uint32_t before = __popc(peers & ltmask);
    uint32_t b = 0;
    if (d < 256u) b = s_whist[warp][d];
    __syncwarp();
    if (d < 256u && before == 0) s_whist[warp][d] = b + __popc(peers);
    __syncwarp();
    rank[k] = b + before;
  }
  __syncthreads();
  // per digit (one per thread): warp-exclusive prefixes and the tile count,
  // published at once so that successors can look past this tile while it
  // orders its items
  const int d = tid; // kSortThreads == 256
  uint32_t count = 0;
  {
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = s_whist[w][d];
      s_whist[w][d] = count;
      count += c;
    }
    st_relaxed_u32(status + (size_t)tile * 256 + d,
                   ((tile == 0 ? 2u : 1u) << kRFlagShift) | count);
  }
  // exclusive scans over digits (256 entries, one per thread) of the tile's
  // counts and of the pass's whole-array counts (the digit's global start)
  uint32_t digitStart;
  {
    uint32_t inc = count, incAll = digitTotal;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      const uint32_t tAll = __shfl_up_sync(0xffffffffu, incAll, o);
      if (lane >= o) {
        inc += t;
        incAll += tAll;
      }
    }
    __shared__ uint32_t s_wsum[kSortWarps], s_wsumAll[kSortWarps];
    if (lane == 31) {
      s_wsum[warp] = inc;
      s_wsumAll[warp] = incAll;
    }
    __syncthreads();
    uint32_t off = 0, offAll = 0;
    for (int w = 0; w < warp; ++w) {
      off += s_wsum[w];
      offAll += s_wsumAll[w];
    }
    s_local[tid] = off + inc - count;
    digitStart = offAll + incAll - digitTotal;
  }
  __syncthreads();
  // local reorder by digit (stable)
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t dk = dig[k];
    if (dk < 256u) {
      const uint32_t p = s_local[dk] + s_whist[warp][dk] + rank[k];
      s_keys[p] = key[k];
      s_vals[p] = val[k];
    }
  }
  // look-back for digit d, with the items already out of registers
  {
    uint32_t excl = 0;
    if (tile != 0) {
      // kLookBack predecessors per round trip (independent loads in
      // flight); tile 0 is always inclusive, so the walk ends before it
      // would read below tile 0
      constexpr int kLookBack = 16;
      int pred = (int)tile - 1;
      uint32_t spins = 0;
      for (;;) {
        uint32_t w[kLookBack];
#pragma unroll
        for (int j = 0; j < kLookBack; ++j)
          w[j] = pred - j >= 0 ? ld_relaxed_u32(status + (size_t)(pred - j) * 256 + d)
                               : (2u << kRFlagShift);
        int take = 0;
        bool done = false;
#pragma unroll
        for (int j = 0; j < kLookBack; ++j) {
          if (done || take < j) continue; // stopped at a gap or the prefix
          const uint32_t flag = w[j] >> kRFlagShift;
          if (flag == 0) continue;
          excl += w[j] & kRValueMask;
          ++take;
          done = flag == 2;
        }
        if (done) break;
        pred -= take;
        if (take == 0) {
          if (++spins > kSpinLimit) {
            atomicOr(err, kStatusSpinLimit);
            break;
          }
          __nanosleep(32);
        }
      }
      st_relaxed_u32(status + (size_t)tile * 256 + d,
                     (2u << kRFlagShift) | ((excl + count) & kRValueMask));
    }
    s_global[d] = digitStart + excl;
  }
  __syncthreads();
  const uint32_t valid = min((uint32_t)kSortTile, n - base);
  for (uint32_t p = tid; p < valid; p += kSortThreads) {
    const K k = s_keys[p];
    const uint32_t dk = (uint32_t)((k >> shift) & 255u);
    const uint32_t dest = s_global[dk] + (p - s_local[dk]);
    keysOut[dest] = k;
    valsOut[dest] = s_vals[p];
  }
}

constexpr uint32_t kShortRun = 16; // runs up to this length: one thread

// The key that orders the elements of a run of equal sort keys, from the
// element's value: the low half of its Morton code, or the order key of its
// box's minX.
struct CodeLow {
  const uint64_t *codes;
  __device__ uint32_t operator()(uint32_t v) const { return (uint32_t)codes[v]; }
};
struct BoxMinX {
  const float4 *box;
  __device__ uint32_t operator()(uint32_t v) const { return float_order_key(box[v].x); }
};

// Every run of equal keys is put in order of the elements' in-run keys
// (lk), stably, in place in vals; with hasSkip, a run of `skip` keys is
// left as it is.
// Runs of up to kShortRun are insertion-sorted by the thread at their
// start; longer ones are listed for k_long_runs32.
template <class LowKey>
__global__ void __launch_bounds__(256)
    k_fix_runs32(const uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                 uint32_t n, LowKey lowKey, bool hasSkip, uint32_t skip,
                 uint32_t *__restrict__ longRuns, uint32_t *longCount, uint32_t cap,
                 uint32_t *err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const uint32_t hi = keys[i];
    if (hasSkip && hi == skip) continue;
    if (i > 0 && keys[i - 1] == hi) continue;      // not a run start
    if (i + 1 >= n || keys[i + 1] != hi) continue; // single key
    uint32_t len = 2;
    while (i + len < n && len <= kShortRun && keys[i + len] == hi) ++len;
    if (len > kShortRun) {
      const uint32_t slot = atomicAdd(longCount, 1u);
      if (slot < cap) longRuns[slot] = i;
      else atomicOr(err, kStatusSpinLimit);
      continue;
    }
    uint32_t lk[kShortRun], v[kShortRun];
    for (uint32_t a = 0; a < len; ++a) {
      v[a] = vals[i + a];
      lk[a] = lowKey(v[a]);
    }
    for (uint32_t a = 1; a < len; ++a) { // stable: equal keys keep their order
      const uint32_t kk = lk[a], vv = v[a];
      uint32_t b = a;
      while (b > 0 && lk[b - 1] > kk) {
        lk[b] = lk[b - 1];
        v[b] = v[b - 1];
        --b;
      }
      lk[b] = kk;
      v[b] = vv;
    }
    for (uint32_t a = 0; a < len; ++a) vals[i + a] = v[a];
  }
}

// One block per long run: its keys are replaced by the in-run keys, a
// stable LSD radix sort (4 passes, through the other buffer over the same
// index range) orders the run, and the keys are restored.
template <class LowKey>
__global__ void __launch_bounds__(256)
    k_long_runs32(uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                  uint32_t *__restrict__ tmpK, uint32_t *__restrict__ tmpV, uint32_t n,
                  LowKey lowKey, const uint32_t *__restrict__ longRuns,
                  const uint32_t *longCount, uint32_t cap) {
  __shared__ uint32_t sHist[256], sOff[256], sWarp[8][256];
  __shared__ uint32_t sEnd;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t runs = min(*longCount, cap);
  const uint32_t ltmask = lanemask_lt();
  for (uint32_t r = blockIdx.x; r < runs; r += gridDim.x) {
    const uint32_t s0 = longRuns[r];
    const uint32_t hi = keys[s0];
    if (tid == 0) sEnd = n;
    __syncthreads();
    for (uint32_t base = s0; base < n; base += 256) {
      const uint32_t i = base + tid;
      if (i < n && keys[i] != hi) atomicMin(&sEnd, i);
      __syncthreads();
      const bool found = sEnd != n;
      __syncthreads(); // every thread has read sEnd before the next tile
      if (found) break;
    }
    const uint32_t e0 = sEnd;
    for (uint32_t i = s0 + tid; i < e0; i += 256) keys[i] = lowKey(vals[i]);
    __syncthreads();
    uint32_t *srcK = keys, *dstK = tmpK, *srcV = vals, *dstV = tmpV;
    for (int p = 0; p < 4; ++p) {
      const int sh = 8 * p;
      sHist[tid] = 0;
      __syncthreads();
      for (uint32_t i = s0 + tid; i < e0; i += 256) atomicAdd(&sHist[(srcK[i] >> sh) & 255u], 1u);
      __syncthreads();
      if (tid == 0) {
        uint32_t run = s0;
        for (int d = 0; d < 256; ++d) {
          sOff[d] = run;
          run += sHist[d];
        }
      }
      __syncthreads();
      for (uint32_t base = s0; base < e0; base += 256) {
        const uint32_t i = base + tid;
        const bool ok = i < e0;
        const uint32_t k = ok ? srcK[i] : 0u;
        const uint32_t v = ok ? srcV[i] : 0u;
        const uint32_t d = ok ? ((k >> sh) & 255u) : 256u;
        uint32_t peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
        for (int bit = 0; bit < 8; ++bit) {
          const uint32_t bb = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
          peers &= ((d >> bit) & 1u) ? bb : ~bb;
        }
        for (int w = 0; w < 8; ++w) sWarp[w][tid] = 0;
        __syncthreads();
        if (ok && __popc(peers & ltmask) == 0) sWarp[warp][d] = __popc(peers);
        __syncthreads();
        {
          uint32_t acc = 0;
          for (int w = 0; w < 8; ++w) {
            const uint32_t c = sWarp[w][tid];
            sWarp[w][tid] = acc;
            acc += c;
          }
          sHist[tid] = acc; // this tile's count of digit tid
        }
        __syncthreads();
        if (ok) {
          const uint32_t dst = sOff[d] + sWarp[warp][d] + __popc(peers & ltmask);
          dstK[dst] = k;
          dstV[dst] = v;
        }
        __syncthreads();
        sOff[tid] += sHist[tid];
        __syncthreads();
      }
      uint32_t *tk = srcK;
      srcK = dstK;
      dstK = tk;
      uint32_t *tv = srcV;
      srcV = dstV;
      dstV = tv;
    }
    // four passes: the result is back in keys/vals; restore the run's keys
    for (uint32_t i = s0 + tid; i < e0; i += 256) keys[i] = hi;
    __syncthreads();
  }
}

} // namespace

void sort_fix_low_bits32(cudaStream_t s, SortScratch &sc, int buf, uint32_t n,
                         const uint64_t *codes, uint32_t *longRuns, uint32_t *runCount,
                         uint32_t cap, uint32_t *err, bool zeroed) {
  if (n < 2) return;
  if (!zeroed) cudaMemsetAsync(runCount, 0, sizeof(uint32_t), s);
  uint32_t b = (n + 255) / 256;
  if (b > 148u * 16u) b = 148u * 16u;
  const CodeLow lk{codes};
  k_fix_runs32<<<b, 256, 0, s>>>(keys32(sc, buf), sc.vals[buf], n, lk, false, 0u, longRuns,
                                 runCount, cap, err);
  k_long_runs32<<<148, 256, 0, s>>>(keys32(sc, buf), sc.vals[buf], keys32(sc, buf ^ 1),
                                     sc.vals[buf ^ 1], n, lk, longRuns, runCount, cap);
}

void sort_fix_units(cudaStream_t s, SortScratch &sc, int buf, uint32_t n, const float4 *box,
                    uint32_t skip, uint32_t *longRuns, uint32_t *runCount, uint32_t cap,
                    uint32_t *err, bool zeroed) {
  if (n < 2) return;
  if (!zeroed) cudaMemsetAsync(runCount, 0, sizeof(uint32_t), s);
  uint32_t b = (n + 255) / 256;
  if (b > 148u * 16u) b = 148u * 16u;
  const BoxMinX lk{box};
  k_fix_runs32<<<b, 256, 0, s>>>(keys32(sc, buf), sc.vals[buf], n, lk, true, skip, longRuns,
                                 runCount, cap, err);
  k_long_runs32<<<148, 256, 0, s>>>(keys32(sc, buf), sc.vals[buf], keys32(sc, buf ^ 1),
                                     sc.vals[buf ^ 1], n, lk, longRuns, runCount, cap);
}

size_t sort_tiles(uint32_t n_max) {
  return (n_max + kSortTile - 1) / kSortTile + 1;
}

size_t sort_pass_words(uint32_t n_max) {
  return 256 * (size_t)((n_max + kSortTile - 1) / kSortTile + 1);
}

namespace {
template <typename K>
int radix_sort(cudaStream_t s, SortScratch &sc, K *const keys[2], uint32_t n_max,
               const uint32_t *d_n, int bit_lo, int bit_hi, bool vals_identity,
               bool have_hist, uint32_t *err, int slot, bool zeroed) {
  const int p0 = bit_lo / 8, np = (bit_hi - bit_lo) / 8;
  uint32_t *hist = sc.hist + (size_t)(slot + p0) * 256;
  if (!have_hist) {
    if (!zeroed) cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 256 * np, s);
    int blocks = (int)((n_max + 1023) / 1024);
    if (blocks > 1184) blocks = 1184;
    if (blocks < 1) blocks = 1;
    k_radix_hist<K><<<blocks, 256, 0, s>>>(keys[0], n_max, d_n, p0, np, sc.hist + slot * 256);
  }
  const uint32_t tiles = (n_max + kSortTile - 1) / kSortTile;
  // look-back words of every pass, cleared at once
  const size_t passWords = sort_pass_words(n_max);
  if (!zeroed) {
    cudaMemsetAsync(sc.tileCounter + slot, 0, sizeof(uint32_t) * np, s);
    cudaMemsetAsync(sc.status + passWords * slot, 0, sizeof(uint32_t) * passWords * np, s);
  }
  int cur = 0;
  for (int p = 0; p < np; ++p) {
    uint32_t *status = sc.status + passWords * (slot + p);
    const int shift = 8 * (p0 + p);
    if (p == 0 && vals_identity) {
      k_onesweep<K, true><<<tiles > 0 ? tiles : 1, kSortThreads, 0, s>>>(
          keys[cur], sc.vals[cur], keys[cur ^ 1], sc.vals[cur ^ 1], hist + p * 256, status,
          sc.tileCounter + slot + p, n_max, d_n, shift, err);
    } else {
      k_onesweep<K, false><<<tiles > 0 ? tiles : 1, kSortThreads, 0, s>>>(
          keys[cur], sc.vals[cur], keys[cur ^ 1], sc.vals[cur ^ 1], hist + p * 256, status,
          sc.tileCounter + slot + p, n_max, d_n, shift, err);
    }
    cur ^= 1;
  }
  return cur;
}
} // namespace

int radix_sort_u64(cudaStream_t s, SortScratch &sc, uint32_t n_max,
                   const uint32_t *d_n, int bit_lo, int bit_hi,
                   bool vals_identity, bool have_hist, uint32_t *err, int slot, bool zeroed) {
  return radix_sort<uint64_t>(s, sc, sc.keys, n_max, d_n, bit_lo, bit_hi, vals_identity,
                              have_hist, err, slot, zeroed);
}

int radix_sort_u32(cudaStream_t s, SortScratch &sc, uint32_t n_max,
                   const uint32_t *d_n, int bit_lo, int bit_hi,
                   bool vals_identity, bool have_hist, uint32_t *err, int slot, bool zeroed) {
  uint32_t *const keys[2] = {keys32(sc, 0), keys32(sc, 1)};
  return radix_sort<uint32_t>(s, sc, keys, n_max, d_n, bit_lo, bit_hi, vals_identity,
                              have_hist, err, slot, zeroed);
}

} // namespace nbx
