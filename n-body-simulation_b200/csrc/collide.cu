// collide.cu -- integrate, collision broadphase and ordered resolution.
//
// Semantics follow the reference's CPU collide() (src/Collision.cpp:135-349):
// the candidate set is every pair of boxes (pos -/+ radius) that overlaps
// under before()/overlaps() (Collision.cpp:88-98), and pairs are resolved
// one after another in pairLess order (Collision.cpp:333-348), each
// resolve() seeing the previous ones' results.
//
// GPU design:
//  * a hashed uniform grid (cell fixed per instance from the radii, as
//    CudaCollision.cu:201-232 does) finds each small box's overlaps in its
//    3x3 cell neighbourhood; boxes wider than ~a cell ("large", e.g. the
//    central body) are tested against every box of their instance;
//  * every body gets its partner list (CSR) sorted by the partners'
//    before() order.  A body's chain of pairs in the global pairLess order
//    is exactly that list: first the pairs where it is the later box
//    (partners before it), then those where it is the earlier box;
//  * resolution is a dataflow over "units" = bodies that are the later box
//    of at least one pair, claimed in before() order.  A unit resolves its
//    pairs in order; pair (L, E) waits until body E has completed the
//    entries of its chain that precede L.  Units only ever wait on
//    smaller units, so the smallest unfinished unit always progresses.
//    The result equals the sequential loop bit for bit (the resolve
//    arithmetic below is IEEE op for op, no contraction);
//  * a body's state after chain entry e is published once, into chain[e]
//    (16 bytes, preset to a sentinel in every word).  The pair that needs
//    it polls that record itself: the load that finds no sentinel word
//    already holds the state, so a dependency costs one L2 round trip and
//    the producer needs no fence.  A body's final state goes to pv.  A
//    sentinel word can only be a NaN with every payload bit set (0xffffffff),
//    which arithmetic never produces; a body carrying one in its input
//    state makes its consumer's wait run out (status: timeout).
#include "nbx_state.cuh"

#include <float.h>

namespace nbx {
namespace {

constexpr int kBlock = 256;

// Bucket of a grid cell: the Morton interleave of the cell coordinates
// (low 16 bits of each), so that cells close in space -- and bodies close in
// the current, Morton-sorted, array order -- share cache lines of the
// bucket table; instances are offset by a large odd stride.  Distinct cells
// may share a bucket; lookups filter on the exact cell.
__device__ __forceinline__ uint32_t cell_hash(uint32_t seg, int cx, int cy,
                                              uint32_t mask) {
  uint32_t x = (uint32_t)cx & 0xffffu, y = (uint32_t)cy & 0xffffu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  y = (y | (y << 8)) & 0x00FF00FFu;
  y = (y | (y << 4)) & 0x0F0F0F0Fu;
  y = (y | (y << 2)) & 0x33333333u;
  y = (y | (y << 1)) & 0x55555555u;
  const uint32_t hi = ((uint32_t)cx >> 16) * 0x9E3779B1u ^ ((uint32_t)cy >> 16) * 0x85EBCA77u;
  return ((x | (y << 1)) + hi + seg * 0x2545F491u) & mask;
}

// cell_hash of the 3x3 cells around (cx, cy), row by row from (cx-1, cy-1):
// the coordinates are interleaved once and their neighbours stepped in
// interleaved form (add or subtract 1 across the gaps of the spread bits),
// so h[k] == cell_hash(seg, cx + k % 3 - 1, cy + k / 3 - 1, mask).
__device__ __forceinline__ uint32_t spread16(uint32_t x) {
  x &= 0xffffu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  return (x | (x << 1)) & 0x55555555u;
}
__device__ __forceinline__ void cell_hash3x3(uint32_t seg, int cx, int cy, uint32_t mask,
                                             uint32_t h[9]) {
  const uint32_t dx = spread16((uint32_t)cx), dy = spread16((uint32_t)cy);
  const uint32_t xs[3] = {((dx & 0x55555555u) - 1u) & 0x55555555u, dx,
                          ((dx | 0xAAAAAAAAu) + 1u) & 0x55555555u};
  const uint32_t ys[3] = {((dy & 0x55555555u) - 1u) & 0x55555555u, dy,
                          ((dy | 0xAAAAAAAAu) + 1u) & 0x55555555u};
  const uint32_t so = seg * 0x2545F491u;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const uint32_t hy = ((uint32_t)(cy + b - 1) >> 16) * 0x85EBCA77u;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t hx = ((uint32_t)(cx + a - 1) >> 16) * 0x9E3779B1u;
      h[3 * b + a] = ((xs[a] | (ys[b] << 1)) + (hx ^ hy) + so) & mask;
    }
  }
}

// floor of the exact product v*inv (the reference takes the floor of the
// double product, Collision.cpp:100-104).
__device__ __forceinline__ int exact_floor_mul(float v, float inv) {
  const float p = __fmul_rn(v, inv);
  const float e = __fmaf_rn(v, inv, -p);
  float f = floorf(p);
  if (f == p && e < 0.0f) f -= 1.0f;
  return (int)f;
}

// before(): Collision.cpp:88-90.
__device__ __forceinline__ bool before_key(float aMinX, uint32_t a,
                                           float bMinX, uint32_t b) {
  return aMinX < bMinX || (aMinX == bMinX && a < b);
}

// overlaps(earlier, later): Collision.cpp:95-98.  box = {minX,maxX,minY,maxY}
__device__ __forceinline__ bool boxes_overlap(const float4 &a, uint32_t ia,
                                              const float4 &b, uint32_t ib) {
  const bool aFirst = before_key(a.x, ia, b.x, ib);
  const float4 &e = aFirst ? a : b;
  const float4 &l = aFirst ? b : a;
  return e.y >= l.x && l.z <= e.w && e.z <= l.w;
}

__device__ __forceinline__ bool is_small(const float4 &bx, float smallW) {
  const float w = __fsub_rn(bx.y, bx.x), h = __fsub_rn(bx.w, bx.z);
  return w <= smallW && h <= smallW;
}

// ---------------------------------------------------------------- kernels

// Body::update (Body.h:20-23) for every body, then the collision box, the
// grid cell and a slot in its bucket (or in its instance's large list).
__global__ void __launch_bounds__(kBlock)
    k_integrate_boxes(DevState S, int integrate, int collide) {
  const uint32_t n = S.n;
  const float dt = S.dt;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    float4 p = S.pv[i];
    if (integrate) {
      const float2 a = S.acc[i];
      p.z = __fadd_rn(p.z, __fmul_rn(a.x, dt));
      p.w = __fadd_rn(p.w, __fmul_rn(a.y, dt));
      p.x = __fadd_rn(p.x, __fmul_rn(p.z, dt));
      p.y = __fadd_rn(p.y, __fmul_rn(p.w, dt));
      S.pv[i] = p;
    }
    if (!collide) continue;
    const float r = S.mr[i].y;
    const float4 bx = make_float4(__fsub_rn(p.x, r), __fadd_rn(p.x, r),
                                  __fsub_rn(p.y, r), __fadd_rn(p.y, r));
    S.box[i] = bx;
    const uint32_t sg = S.segOf[i];
    const SegDev &G = S.seg[sg];
    bool small = is_small(bx, G.smallW);
    int cx = 0, cy = 0;
    if (small) {
      const float fx = __fmul_rn(bx.x, G.invCell);
      const float fy = __fmul_rn(bx.z, G.invCell);
      // far from the origin the float cell index loses integer precision:
      // such boxes are treated as large (compared against everything).
      if (!(fabsf(fx) < 8388608.0f && fabsf(fy) < 8388608.0f)) {
        small = false;
      } else {
        cx = exact_floor_mul(bx.x, G.invCell);
        cy = exact_floor_mul(bx.z, G.invCell);
      }
    }
    if (small) {
      const uint32_t h = cell_hash(sg, cx, cy, S.nBuckets - 1);
      S.slot[i] = atomicAdd(&S.bucketCount[h], 1u);
      S.cellXY[i] = make_int2(cx, cy);
    } else {
      S.slot[i] = atomicAdd(&S.largeCount[sg], 1u) | 0x80000000u;
      S.cellXY[i] = make_int2(0x7fffffff, 0x7fffffff);
      S.deg[i] = 0;       // accumulated by the partners' atomics
      S.fillLarge[i] = 0; // fill cursor of this large body's list
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_fill_grid(DevState S) {
  const uint32_t n = S.n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const uint32_t s = S.slot[i];
    const uint32_t sg = S.segOf[i];
    if (s & 0x80000000u) {
      S.largeList[S.largeStartA[sg] + (s & 0x7fffffffu)] = i;
    } else {
      const int2 c = S.cellXY[i];
      const uint32_t h = cell_hash(sg, c.x, c.y, S.nBuckets - 1);
      const uint32_t e = S.bucketStart[h] + s;
      S.grid[e] = i;
      S.gridBox[e] = S.box[i];
    }
  }
}

constexpr uint32_t kStash = 16; // partners remembered per body by the count pass

// Every small body of the same instance whose box overlaps small body i's,
// from the buckets of the 3x3 cells around i's cell: f(j) for each, in
// bucket order.  A bucket shared by two of the nine cells is read once.
// Bodies of other cells that share a bucket need no cell test: two small
// boxes that overlap lie in cells at most one apart on each axis (a box is
// at most 0.999 of a cell wide and the cell index is the exact floor), so a
// body from any other cell fails the overlap test by itself.  The boxes are
// read beside the indices (gridBox), so a candidate costs no dependent load.
template <class F>
__device__ __forceinline__ void for_each_cell_neighbour(const DevState &S, uint32_t i,
                                                        uint32_t sg, const float4 &bi,
                                                        uint32_t mask, F &&f) {
  const int2 c = S.cellXY[i];
  uint32_t hs[9];
  cell_hash3x3(sg, c.x, c.y, mask, hs);
  const bool oneInstance = S.nseg == 1;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    bool seen = false;
#pragma unroll
    for (int r = 0; r < q; ++r) seen |= hs[r] == hs[q];
    if (seen) continue;
    const uint32_t e0 = S.bucketStart[hs[q]], e1 = S.bucketStart[hs[q] + 1];
    for (uint32_t e = e0; e < e1; ++e) {
      const uint32_t j = S.grid[e];
      const float4 bj = S.gridBox[e];
      if (j == i) continue;
      if (!oneInstance && S.segOf[j] != sg) continue;
      if (boxes_overlap(bi, i, bj, j)) f(j);
    }
  }
}

// Partner discovery, count pass: every overlap of a small body's box in its
// 3x3 cell neighbourhood and with the large boxes of its instance.  The
// first kStash partners are stashed so that the fill pass need not search
// again; small-large pairs are appended for the large body's list.
__global__ void __launch_bounds__(kBlock) k_partners_count(DevState S) {
  const uint32_t n = S.n;
  const uint32_t mask = S.nBuckets - 1;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const uint32_t sg = S.segOf[i];
    const float4 bi = S.box[i];
    const uint32_t lStart = S.largeStartA[sg];
    const uint32_t lCount = S.largeCount[sg];
    uint32_t cnt = 0;
    uint32_t *stash = S.stash + (size_t)i * kStash;
    if (!(S.slot[i] & 0x80000000u)) {
      for_each_cell_neighbour(S, i, sg, bi, mask, [&](uint32_t j) {
        if (cnt < kStash) stash[cnt] = j;
        ++cnt;
      });
      for (uint32_t k = 0; k < lCount; ++k) {
        const uint32_t j = S.largeList[lStart + k];
        if (boxes_overlap(bi, i, S.box[j], j)) {
          if (cnt < kStash) stash[cnt] = j;
          ++cnt;
          atomicAdd(&S.deg[j], 1u);
          const uint32_t slot = atomicAdd(&S.counters[5], 1u);
          if (slot < S.n) S.largePairs[slot] = make_uint2(j, i);
          else atomicOr(S.status, kStatusPairCapacity);
        }
      }
      S.deg[i] = cnt;
    } else {
      // large vs large: each side counts its own half
      for (uint32_t k = 0; k < lCount; ++k) {
        const uint32_t j = S.largeList[lStart + k];
        if (j != i && boxes_overlap(bi, i, S.box[j], j)) ++cnt;
      }
      atomicAdd(&S.deg[i], cnt);
    }
  }
}

// Coarse sort key of a unit's minX: 24 bits over twice the instance's last
// root square, order-preserving (a float subtract, a multiply by a positive
// scale and floor are each monotone), clamped at the ends.  The sort on it
// is completed by ordering each run of equal keys by the exact minX
// (sort_fix_units), so only speed depends on how well it spreads.
constexpr uint32_t kUnitKeyMax = (1u << 24) - 2;  // largest unit key
constexpr uint32_t kNonUnitKey = (1u << 24) - 1;  // every non-unit, last
__device__ __forceinline__ uint32_t unit_coarse_key(const SegDev &G, float minX) {
  const float lo = G.cx - G.size;
  const float scale = G.size > 0.0f && G.size <= 1e30f ? (float)kUnitKeyMax / (2.0f * G.size)
                                                       : 0.0f;
  const float q = floorf((minX - lo) * scale);
  if (!(q > 0.0f)) return 0u;
  return q >= (float)kUnitKeyMax ? kUnitKeyMax : (uint32_t)q;
}

// Sort key of a body for the units' before()-order sort: its coarse minX
// key if it is a unit (the later box of >= 1 pair), kNonUnitKey otherwise
// (after every unit); the key's three digits go into the block's histogram.
__device__ __forceinline__ void unit_key(uint32_t i, bool unit, const SegDev &G, float minX,
                                         uint32_t *__restrict__ keys, uint32_t (*sh)[256],
                                         uint32_t &units) {
  const uint32_t k = unit ? unit_coarse_key(G, minX) : kNonUnitKey;
  keys[i] = k;
#pragma unroll
  for (int q = 0; q < 3; ++q) atomicAdd(&sh[q][(k >> (8 * q)) & 255u], 1u);
  units += unit ? 1u : 0u;
}

__device__ __forceinline__ void flush_unit_hist(uint32_t (*sh)[256], uint32_t units,
                                                uint32_t *sUnits, uint32_t *hist,
                                                uint32_t *unitCount) {
  atomicAdd(sUnits, units);
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) {
    const uint32_t v = sh[i >> 8][i & 255];
    if (v) atomicAdd(&hist[i], v);
  }
  if (threadIdx.x == 0 && *sUnits) atomicAdd(unitCount, *sUnits);
}

// Fill pass: small bodies copy their stash (or search again past kStash
// partners) into their CSR list and sort it by the partners' before()
// order; large bodies add their large-large partners, and the count pass's
// small-large pairs go into the large bodies' lists.  Every body's unit
// key and its digit counts come out too.
__global__ void __launch_bounds__(kBlock)
    k_partners_fill(DevState S, uint32_t *__restrict__ keys, uint32_t *hist) {
  __shared__ uint32_t sh[3][256];
  __shared__ uint32_t sUnits;
  for (int q = threadIdx.x; q < 3 * 256; q += blockDim.x) sh[q >> 8][q & 255] = 0;
  if (threadIdx.x == 0) sUnits = 0;
  __syncthreads();
  uint32_t units = 0;
  const uint32_t n = S.n;
  const uint32_t mask = S.nBuckets - 1;
  const bool overflow = S.counters[0] > S.pairCapacity;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const uint32_t sg = S.segOf[i];
    const float4 bi = S.box[i];
    const uint32_t lStart = S.largeStartA[sg];
    const uint32_t lCount = S.largeCount[sg];
    if (S.slot[i] & 0x80000000u) {
      if (!overflow) {
        for (uint32_t k = 0; k < lCount; ++k) {
          const uint32_t j = S.largeList[lStart + k];
          if (j != i && boxes_overlap(bi, i, S.box[j], j)) {
            const uint32_t slotI = atomicAdd(&S.fillLarge[i], 1u);
            S.plist[S.pstart[i] + slotI] = j;
          }
        }
      }
      continue;
    }
    if (overflow) {
      S.nLater[i] = 0;
      unit_key(i, false, S.seg[sg], bi.x, keys, sh, units);
      if (i == 0) atomicOr(S.status, kStatusPairCapacity);
      continue;
    }
    const uint32_t cnt = S.deg[i];
    const uint32_t base = S.pstart[i];
    if (cnt <= kStash) {
      const uint32_t *stash = S.stash + (size_t)i * kStash;
      for (uint32_t a = 0; a < cnt; ++a) S.plist[base + a] = stash[a];
    } else {
      uint32_t w = 0;
      for_each_cell_neighbour(S, i, sg, bi, mask,
                              [&](uint32_t j) { S.plist[base + w++] = j; });
      for (uint32_t k = 0; k < lCount; ++k) {
        const uint32_t j = S.largeList[lStart + k];
        if (boxes_overlap(bi, i, S.box[j], j)) S.plist[base + w++] = j;
      }
    }
    // insertion sort of the own list by the partners' before() order
    for (uint32_t a = 1; a < cnt; ++a) {
      const uint32_t v = S.plist[base + a];
      const float vk = S.box[v].x;
      uint32_t b = a;
      while (b > 0) {
        const uint32_t u = S.plist[base + b - 1];
        if (!before_key(vk, v, S.box[u].x, u)) break;
        S.plist[base + b] = u;
        --b;
      }
      S.plist[base + b] = v;
    }
    uint32_t nl = 0;
    for (uint32_t a = 0; a < cnt; ++a) {
      const uint32_t u = S.plist[base + a];
      if (before_key(S.box[u].x, u, bi.x, i)) ++nl;
    }
    S.nLater[i] = nl;
    unit_key(i, nl > 0, S.seg[sg], bi.x, keys, sh, units);
  }
  // the small-large pairs recorded by the count pass, into the large
  // bodies' lists (in any order: k_sort_large orders those lists)
  if (!overflow) {
    const uint32_t total = min(S.counters[5], S.n);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += gridDim.x * blockDim.x) {
      const uint2 pr = S.largePairs[q];
      const uint32_t slot = atomicAdd(&S.fillLarge[pr.x], 1u);
      S.plist[S.pstart[pr.x] + slot] = pr.y;
    }
  }
  flush_unit_hist(sh, units, &sUnits, hist, &S.counters[1]);
}

// Sorts each large body's partner list (filled by others through atomics)
// by before() order: one warp per large body, rank by counting.
__global__ void __launch_bounds__(kBlock)
    k_sort_large(DevState S, uint32_t *__restrict__ keys, uint32_t *hist) {
  const int lane = threadIdx.x & 31;
  const uint32_t warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nWarps = (gridDim.x * blockDim.x) >> 5;
  const bool overflow = S.counters[0] > S.pairCapacity;
  // large bodies of all instances, back to back in the large list
  const uint32_t totalLarge =
      S.largeStartA[S.nseg - 1] + S.largeCount[S.nseg - 1];
  for (uint32_t w = warpId; w < totalLarge; w += nWarps) {
    const uint32_t g = S.largeList[w];
    const uint32_t d = S.deg[g];
    const uint32_t base = S.pstart[g];
    const float gk = S.box[g].x;
    if (!overflow && d > 0) {
      // rank of each element, written to the scratch copy of the lists
      for (uint32_t a = lane; a < d; a += 32) {
        const uint32_t v = S.plist[base + a];
        const float vk = S.box[v].x;
        uint32_t rank = 0;
        for (uint32_t b = 0; b < d; ++b) {
          const uint32_t u = S.plist[base + b];
          rank += before_key(S.box[u].x, u, vk, v) ? 1u : 0u;
        }
        S.plistTmp[base + rank] = v;
      }
      __syncwarp();
      uint32_t nl = 0;
      for (uint32_t a = lane; a < d; a += 32) {
        const uint32_t u = S.plistTmp[base + a];
        S.plist[base + a] = u;
        nl += before_key(S.box[u].x, u, gk, g) ? 1u : 0u;
      }
      for (int o = 16; o > 0; o >>= 1) nl += __shfl_xor_sync(0xffffffffu, nl, o);
      if (lane == 0) S.nLater[g] = nl;
    } else if (lane == 0) {
      S.nLater[g] = 0;
    }
    if (lane == 0) {
      // the large body's sort key (few bodies: straight to the histogram)
      const bool unit = !overflow && d > 0 && S.nLater[g] > 0;
      const uint32_t k = unit ? unit_coarse_key(S.seg[S.segOf[g]], gk) : kNonUnitKey;
      keys[g] = k;
      for (int q = 0; q < 3; ++q) atomicAdd(&hist[q * 256 + ((k >> (8 * q)) & 255u)], 1u);
      if (unit) atomicAdd(&S.counters[1], 1u);
    }
  }
}


// resolve(bodies, i = later, j = earlier): Collision.cpp:16-84, IEEE op
// for op.  s = {x, y, vx, vy}.
__device__ void resolve_pair(float4 &s1, float m1, float r1, float4 &s2,
                             float m2, float r2) {
  float dx = __fsub_rn(s2.x, s1.x), dy = __fsub_rn(s2.y, s1.y);
  const float r = __fadd_rn(r1, r2);
  const float dd = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  if (dd > __fmul_rn(r, r)) return;
  const float v1x = s1.z, v1y = s1.w, v2x = s2.z, v2y = s2.w;
  const float vx = __fsub_rn(v2x, v1x), vy = __fsub_rn(v2y, v1y);
  float dDotV = __fadd_rn(__fmul_rn(dx, vx), __fmul_rn(dy, vy));
  const float msum = __fadd_rn(m1, m2);
  const float w1 = __fdiv_rn(m2, msum);
  const float w2 = __fdiv_rn(m1, msum);
  const bool dNonZero = !(dx == 0.0f && dy == 0.0f);
  if (dDotV >= 0.0f && dNonZero) {
    const float s = __fsub_rn(__fdiv_rn(r, __fsqrt_rn(dd)), 1.0f);
    const float tx = __fmul_rn(dx, s), ty = __fmul_rn(dy, s);
    s1.x = __fsub_rn(s1.x, __fmul_rn(w1, tx));
    s1.y = __fsub_rn(s1.y, __fmul_rn(w1, ty));
    s2.x = __fadd_rn(s2.x, __fmul_rn(w2, tx));
    s2.y = __fadd_rn(s2.y, __fmul_rn(w2, ty));
    return;
  }
  const float vSq = __fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy));
  if (vSq < 1e-12f) {
    float dirX = 1.0f, dirY = 0.0f;
    if (dNonZero) {
      const float inv = __fdiv_rn(1.0f, __fsqrt_rn(dd));
      dirX = __fmul_rn(dx, inv);
      dirY = __fmul_rn(dy, inv);
    }
    const float tx = __fmul_rn(dirX, r), ty = __fmul_rn(dirY, r);
    s1.x = __fsub_rn(s1.x, __fmul_rn(w1, tx));
    s1.y = __fsub_rn(s1.y, __fmul_rn(w1, ty));
    s2.x = __fadd_rn(s2.x, __fmul_rn(w2, tx));
    s2.y = __fadd_rn(s2.y, __fmul_rn(w2, ty));
    return;
  }
  const float rSq = __fmul_rn(r, r);
  const float disc = fmaxf(
      __fsub_rn(__fmul_rn(dDotV, dDotV), __fmul_rn(vSq, __fsub_rn(dd, rSq))),
      0.0f);
  const float t = __fdiv_rn(__fadd_rn(dDotV, __fsqrt_rn(disc)), vSq);
  s1.x = __fsub_rn(s1.x, __fmul_rn(v1x, t));
  s1.y = __fsub_rn(s1.y, __fmul_rn(v1y, t));
  s2.x = __fsub_rn(s2.x, __fmul_rn(v2x, t));
  s2.y = __fsub_rn(s2.y, __fmul_rn(v2y, t));
  dx = __fsub_rn(s2.x, s1.x);
  dy = __fsub_rn(s2.y, s1.y);
  dDotV = __fadd_rn(__fmul_rn(dx, vx), __fmul_rn(dy, vy));
  const float dSq2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float s = __fdiv_rn(__fmul_rn(1.5f, dDotV), dSq2);
  const float tx = __fmul_rn(dx, s), ty = __fmul_rn(dy, s);
  const float n1x = __fadd_rn(v1x, __fmul_rn(tx, w1));
  const float n1y = __fadd_rn(v1y, __fmul_rn(ty, w1));
  const float n2x = __fsub_rn(v2x, __fmul_rn(tx, w2));
  const float n2y = __fsub_rn(v2y, __fmul_rn(ty, w2));
  s1.z = n1x;
  s1.w = n1y;
  s2.z = n2x;
  s2.w = n2y;
  s1.x = __fadd_rn(s1.x, __fmul_rn(n1x, t));
  s1.y = __fadd_rn(s1.y, __fmul_rn(n1y, t));
  s2.x = __fadd_rn(s2.x, __fmul_rn(n2x, t));
  s2.y = __fadd_rn(s2.y, __fmul_rn(n2y, t));
}

// Position of body `who` in body e's sorted partner list.
__device__ __forceinline__ uint32_t chain_position(const DevState &S,
                                                   uint32_t e, uint32_t who,
                                                   float whoKey) {
  uint32_t lo = 0, hi = S.deg[e];
  const uint32_t base = S.pstart[e];
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    const uint32_t u = S.plist[base + mid];
    if (before_key(S.box[u].x, u, whoKey, who)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

constexpr uint32_t kUnpublished = 0xffffffffu; // sentinel word of chain[]
constexpr uint32_t kFirstEntry = 1u << 31;      // E's chain starts here
constexpr uint32_t kLastEntry = 1u << 30;       // E's chain ends here
constexpr uint32_t kEntryMask = kLastEntry - 1u;

__device__ __forceinline__ bool published(const float4 &v) {
  return (__float_as_uint(v.x) != kUnpublished) & (__float_as_uint(v.y) != kUnpublished) &
         (__float_as_uint(v.z) != kUnpublished) & (__float_as_uint(v.w) != kUnpublished);
}

// Per as-later pair (L, E): E's chain entry for it (where L sits in E's
// sorted partner list, offset by E's list start), flagged when it is E's
// first or last entry; computed in bulk so the resolution does not search.
// Also presets every chain record of the body to the sentinel.
__global__ void __launch_bounds__(kBlock) k_twins(DevState S) {
  if (S.counters[0] > S.pairCapacity) return;
  const float4 unset = make_float4(__uint_as_float(kUnpublished), __uint_as_float(kUnpublished),
                                   __uint_as_float(kUnpublished), __uint_as_float(kUnpublished));
  for (uint32_t L = blockIdx.x * blockDim.x + threadIdx.x; L < S.n;
       L += gridDim.x * blockDim.x) {
    const uint32_t pl = S.pstart[L], dl = S.deg[L];
    for (uint32_t k = 0; k < dl; ++k) __stcg(&S.chain[pl + k], unset);
    const uint32_t nl = S.nLater[L];
    const float key = S.box[L].x;
    for (uint32_t k = 0; k < nl; ++k) {
      const uint32_t E = S.plist[pl + k];
      const uint32_t m = chain_position(S, E, L, key);
      S.twin[pl + k] = (S.pstart[E] + m) | (m == 0 ? kFirstEntry : 0u) |
                       (m + 1 == S.deg[E] ? kLastEntry : 0u);
    }
  }
}

// Ordered resolution.  Lanes claim units in before() order through one
// atomic counter (warp-aggregated, so claims stay in order), and every
// round each lane whose next pair is ready (body E's state after the chain
// entries before this pair is published) resolves it; a lane whose unit is
// done claims the next one.  No lane ever spins alone, so a lane whose
// predecessor belongs to another lane of the same warp cannot starve it,
// and the smallest unfinished unit (all its predecessors done) always
// advances.  The next pair's partner is fetched while the current one waits.
__global__ void __launch_bounds__(kBlock)
    k_resolve(DevState S, const uint32_t *__restrict__ units) {
  const uint32_t numUnits = S.counters[1];
  const int lane = threadIdx.x & 31;
  if (S.counters[0] > S.pairCapacity) return;
  bool active = false, exhausted = false, lastL = false;
  uint32_t L = 0, nl = 0, pl = 0, k = 0;
  uint32_t E = 0, t = 0, nE = 0, nt = 0; // current and next pair
  float2 mrL = make_float2(0.0f, 0.0f), mrE = mrL, nmrE = mrL;
  bool nmrPending = false;
  float4 sL = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  uint32_t idle = 0;
  for (;;) {
    if (!exhausted) {
      const uint32_t need = __ballot_sync(0xffffffffu, !active);
      if (need) {
        const int leader = __ffs(need) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&S.counters[2], (uint32_t)__popc(need));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (!active) {
          const uint32_t u = base + __popc(need & lanemask_lt());
          if (u < numUnits) {
            L = units[u];
            S.unitOrder[u] = L; // kept for introspection of the pair order
            nl = S.nLater[L];
            pl = S.pstart[L];
            lastL = nl == S.deg[L];
            mrL = S.mr[L];
            sL = __ldcg(&S.pv[L]);
            k = 0;
            E = S.plist[pl];
            t = S.twin[pl];
            mrE = S.mr[E];
            if (nl > 1) {
              nE = S.plist[pl + 1];
              nt = S.twin[pl + 1];
              nmrPending = true;
            }
            active = true;
          }
        }
        if (base + (uint32_t)__popc(need) >= numUnits) exhausted = true;
      }
    }
    if (!__any_sync(0xffffffffu, active)) break; // nothing left to claim
    bool progressed = false;
    if (active) {
      if (nmrPending) { // nE has arrived by now
        nmrE = S.mr[nE];
        nmrPending = false;
      }
      const uint32_t e = t & kEntryMask;
      const bool first = (t & kFirstEntry) != 0;
      float4 sE = first ? __ldcg(&S.pv[E]) : ld_relaxed_f4(&S.chain[e - 1]);
      if (first || published(sE)) {
        resolve_pair(sL, mrL.x, mrL.y, sE, mrE.x, mrE.y);
        if (t & kLastEntry) __stcg(&S.pv[E], sE);
        else st_relaxed_f4(&S.chain[e], sE);
        progressed = true;
        if (++k == nl) {
          // L's own entries are the first of its chain: publish its state
          if (lastL) __stcg(&S.pv[L], sL);
          else st_relaxed_f4(&S.chain[pl + nl - 1], sL);
          active = false;
        } else {
          E = nE;
          t = nt;
          mrE = nmrE;
          if (k + 1 < nl) {
            nE = S.plist[pl + k + 1];
            nt = S.twin[pl + k + 1];
            nmrPending = true;
          }
        }
      }
    }
    if (__any_sync(0xffffffffu, progressed)) {
      idle = 0;
    } else {
      if (++idle > kSpinLimit) {
        if (lane == 0) atomicOr(S.status, kStatusSpinLimit);
        break;
      }
      __nanosleep(32);
    }
  }
}

// Bounding boxes per instance: each block takes a contiguous chunk;
// per-thread min/max keys, block-reduced when the whole block is in one
// instance, flushed with atomics otherwise.  The last block to finish sets
// every instance's root square and Morton frame (root_frame_seg).
__global__ void __launch_bounds__(kBlock) k_bounds(DevState S) {
  const uint32_t n = S.n;
  const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint32_t c0 = blockIdx.x * chunk;
  const uint32_t c1 = min(n, c0 + chunk);
  __shared__ uint32_t sb[4];
  __shared__ uint32_t sSeg;
  if (threadIdx.x == 0) {
    sb[0] = 0xffffffffu;
    sb[1] = 0u;
    sb[2] = 0xffffffffu;
    sb[3] = 0u;
    sSeg = c0 < c1 ? S.segOf[c1 - 1] : 0xffffffffu;
  }
  __syncthreads();
  uint32_t curSeg = 0xffffffffu;
  uint32_t k0 = 0xffffffffu, k1 = 0u, k2 = 0xffffffffu, k3 = 0u;
  bool any = false;
  for (uint32_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
    const uint32_t sg = S.segOf[i];
    if (sg != curSeg) {
      if (any) {
        uint32_t *b = S.bounds + 4 * curSeg;
        atomicMin(b + 0, k0);
        atomicMax(b + 1, k1);
        atomicMin(b + 2, k2);
        atomicMax(b + 3, k3);
      }
      curSeg = sg;
      k0 = 0xffffffffu;
      k1 = 0u;
      k2 = 0xffffffffu;
      k3 = 0u;
      any = false;
    }
    const float4 p = S.pv[i];
    if (!(fabsf(p.x) <= FLT_MAX && fabsf(p.y) <= FLT_MAX)) {
      if (p.x != p.x || p.y != p.y || fabsf(p.x) > FLT_MAX || fabsf(p.y) > FLT_MAX)
        atomicOr(S.status, kStatusNonFinite);
      if (p.x != p.x || p.y != p.y) continue; // NaN never wins a min/max
    }
    const uint32_t kx = float_order_key(p.x), ky = float_order_key(p.y);
    k0 = min(k0, kx);
    k1 = max(k1, kx);
    k2 = min(k2, ky);
    k3 = max(k3, ky);
    any = true;
  }
  if (any) {
    if (curSeg == sSeg) {
      atomicMin(&sb[0], k0);
      atomicMax(&sb[1], k1);
      atomicMin(&sb[2], k2);
      atomicMax(&sb[3], k3);
    } else {
      uint32_t *b = S.bounds + 4 * curSeg;
      atomicMin(b + 0, k0);
      atomicMax(b + 1, k1);
      atomicMin(b + 2, k2);
      atomicMax(b + 3, k3);
    }
  }
  __syncthreads();
  __shared__ bool sLast;
  if (threadIdx.x == 0) {
    if (sSeg != 0xffffffffu && sb[1] != 0u) {
      uint32_t *b = S.bounds + 4 * sSeg;
      atomicMin(b + 0, sb[0]);
      atomicMax(b + 1, sb[1]);
      atomicMin(b + 2, sb[2]);
      atomicMax(b + 3, sb[3]);
    }
    // this block's bounds before its arrival; the last block to arrive
    // sees every block's bounds
    __threadfence();
    sLast = atomicAdd(&S.counters[kCtrBoundsDone], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!sLast) return;
  __threadfence();
  for (uint32_t sg = threadIdx.x; sg < S.nseg; sg += blockDim.x) root_frame_seg(S, sg);
  if (threadIdx.x == 0) S.counters[kCtrBoundsDone] = 0u;
}

int grid_for(uint32_t n) {
  uint32_t b = (n + kBlock - 1) / kBlock;
  if (b > 148u * 16u) b = 148u * 16u;
  return b ? (int)b : 1;
}

struct ZeroRanges {
  uint32_t *p[12];
  uint32_t n[12];
  int count;
};

// Clears every range (16-byte aligned ranges with 16-byte stores).
__global__ void __launch_bounds__(kBlock) k_zero_ranges(ZeroRanges z) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int r = 0; r < z.count; ++r) {
    uint32_t *p = z.p[r];
    const uint32_t n = z.n[r];
    uint32_t head = 0;
    if ((reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
      uint4 *q = reinterpret_cast<uint4 *>(p);
      for (uint32_t i = t; i < n / 4; i += stride) q[i] = make_uint4(0u, 0u, 0u, 0u);
      head = n & ~3u;
    }
    for (uint32_t i = head + t; i < n; i += stride) p[i] = 0u;
  }
}

} // namespace

// What a step's phases expect cleared, in one launch: the collision
// counters (units, unit claims, small-large pairs, long runs of both
// sorts), both sorts' digit rows, tile counters and look-back words (the
// Morton sort in slots 0-3, the units' in 4-6) and the four scan slots
// (grid buckets, large lists, partner lists, traversal records); with
// grid, also the collision grid's bucket and large counts (a step or phase
// that collides).
void launch_step_zero(cudaStream_t s, const DevState &S, ScanScratch &scan, SortScratch &sort,
                      bool grid) {
  ZeroRanges z{};
  auto add = [&](uint32_t *p, size_t n) {
    z.p[z.count] = p;
    z.n[z.count] = (uint32_t)n;
    ++z.count;
  };
  if (grid) {
    add(S.bucketCount, S.nBuckets + 1);
    add(S.largeCount, S.nseg);
  }
  add(S.counters + 1, 2); // units, unit claims
  add(S.counters + 5, 1); // small-large pairs
  add(S.counters + 9, 2); // long runs of the Morton and the units' sorts
  add(sort.hist, 7 * 256);
  add(sort.tileCounter, 8);
  const uint32_t statusWords = 7 * (uint32_t)sort_pass_words(S.n);
  add(sort.status, statusWords);
  add(reinterpret_cast<uint32_t *>(scan.slotStatus), 2 * (size_t)kScanSlots * scan.maxTiles);
  add(scan.tileCounter, kScanSlots);
  const uint32_t big = grid && S.nBuckets + 1 > statusWords ? S.nBuckets + 1 : statusWords;
  k_zero_ranges<<<grid_for(big / 4 + 1), kBlock, 0, s>>>(z);
}

// Host-side sequencing of the collision phase (no host synchronisation).
void launch_integrate(cudaStream_t s, const DevState &S, bool integrate,
                      bool collide) {
  k_integrate_boxes<<<grid_for(S.n), kBlock, 0, s>>>(S, integrate ? 1 : 0,
                                                     collide ? 1 : 0);
}

void launch_collide(cudaStream_t s, DevState &S, ScanScratch &scan,
                    SortScratch &sort, const SideStream *side) {
  const uint32_t n = S.n;
  // grid buckets and large lists
  exclusive_scan_u32(s, S.bucketCount, S.bucketStart, S.nBuckets + 1, nullptr,
                     nullptr, scan, S.status, nullptr, 0, 0);
  exclusive_scan_u32(s, S.largeCount, S.largeStartA, S.nseg, nullptr, nullptr,
                     scan, S.status, nullptr, 0, 1);
  k_fill_grid<<<grid_for(n), kBlock, 0, s>>>(S);
  mark(s, "collide.grid");
  // partners: count (+ stash), scan, fill + sort
  k_partners_count<<<grid_for(n), kBlock, 0, s>>>(S);
  exclusive_scan_u32(s, S.deg, S.pstart, n, nullptr, &S.counters[0], scan,
                     S.status, nullptr, 0, 2);
  mark(s, "collide.count");
  // the fill kernels also write every body's key for the units' sort
  // (units first, in before() order) and its digit histograms
  uint32_t *unitHist = sort.hist + kUnitSortSlot * 256;
  k_partners_fill<<<grid_for(n), kBlock, 0, s>>>(S, keys32(sort, 0), unitHist);
  k_sort_large<<<64, kBlock, 0, s>>>(S, keys32(sort, 0), unitHist);
  mark(s, "collide.fill");
  // the pairs' chain entries (k_twins) need only the sorted lists: they
  // run beside the units' sort, on the side stream when there is one
  if (side) {
    cudaEventRecord(side->fork, s);
    cudaStreamWaitEvent(side->stream, side->fork, 0);
    k_twins<<<grid_for(n), kBlock, 0, side->stream>>>(S);
    cudaEventRecord(side->join, side->stream);
  }
  // units in before() order: a stable sort of all bodies' coarse keys
  // (value = index), then each run of equal coarse keys in exact minX order;
  // the first counters[1] entries are the units
  const int buf = radix_sort_u32(s, sort, n, nullptr, 0, 24, true, true, S.status,
                                 kUnitSortSlot, true);
  sort_fix_units(s, sort, buf, n, S.box, kNonUnitKey, S.longRuns, &S.counters[10],
                 n / 16 + 64, S.status, true);
  mark(s, "collide.units");
  // ordered resolution
  if (side) cudaStreamWaitEvent(s, side->join, 0);
  else k_twins<<<grid_for(n), kBlock, 0, s>>>(S);
  k_resolve<<<148 * 8, kBlock, 0, s>>>(S, sort.vals[buf]);
  mark(s, "collide.resolve");
}

void launch_bounds(cudaStream_t s, const DevState &S) {
  uint32_t blocks = (S.n + 1023) / 1024; // 4 bodies per thread
  if (blocks > 148u * 8u) blocks = 148u * 8u;
  if (blocks < 1) blocks = 1;
  k_bounds<<<blocks, kBlock, 0, s>>>(S);
}

} // namespace nbx
