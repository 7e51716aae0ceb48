// nbx_state.cuh -- device state of one simulation handle (one or many
// independent instances, "segments", laid out back to back).
#pragma once
#include "nbx_internal.cuh"

#include <float.h>

namespace nbx {

// Per-segment record in device memory.
struct SegDev {
  uint32_t start, count;       // body range [start, start+count)
  float cell, invCell, smallW; // collision grid cell; boxes wider than
                               // smallW go to the large list
  uint32_t wide;               // written every step: bodies reach beyond the
                               // clamp guard's coordinate limit
  // written every step
  float cx, cy, size; // root square (Quad::newContaining)
  uint32_t pad1;
  MortonFrame frame;  // quantisation constants (binary64 bit patterns)
  uint32_t nodeBase;  // first node of this segment's tree (breadth-first
                      // arrays, the reference's numbering)
  uint32_t nodeCount; // nodes in this segment's tree
  uint32_t levelCount;
  uint32_t largeStart, largeCount;
  uint32_t travCount; // nodes in the traversal layout (non-empty nodes)
  uint32_t travBase;  // first record of this segment's traversal layout
  uint32_t pad2;
};

// A node of the force traversal, in depth-first preorder: a = {comX, comY,
// mass, size*size}, b = {next, open, start, end}: next = the slot after the
// node's subtree (preorder, global; all ones past the instance's last node),
// open = where a walk that opens the node goes (next for a leaf, the next
// slot -- its first child -- for an interior node, so a node is a leaf iff
// open == next), [start, end) = its bodies.  32-byte aligned so that the
// traversal reads a record with one 256-bit load.
struct alignas(32) TravNode {
  float4 a;
  int4 b;
};
static_assert(sizeof(TravNode) == 32, "32-byte traversal records");

constexpr int kMaxDepth = 32;   // TreeKernels.cuh:29
constexpr int kLevelSlots = 34; // depths 0..32 plus an end slot

// counters[] slot of the force law's clamp guard.  The force pass may
// leave out the law's FLT_MAX clamp only while every distance it forms
// stays finite: the upload stores the largest coordinate allowed here
// (float bits), and each build marks the instances whose bodies reach
// beyond it (SegDev::wide), for the force pass to keep the clamp there.
constexpr int kCtrCoordLimit = 15;
constexpr int kCtrBoundsDone = 7; // blocks of the bounds pass done (self-resetting)

// Everything a step's kernels touch.  All pointers are device pointers.
struct DevState {
  uint32_t n;     // bodies over all segments
  uint32_t nseg;  // segments
  uint32_t nodeCapacity;
  uint32_t pairCapacity;
  float dt, tSq, eSq;
  int leafCapacity;
  int collisions;
  // force targets [forceBegin, forceEnd) of a force launch; forceEnd 0:
  // every body (the step graphs of nbx_step_io split the pass in ranges)
  uint32_t forceBegin, forceEnd;
  // with recOut, the force pass also writes each target's 9-word body
  // record (the nbx_body layout) there
  uint32_t *recOut;

  SegDev *seg;
  uint16_t *segOf; // segment of each body index (never permuted)

  // body state, current order (double-buffered across the Morton gather)
  float4 *pv;   // {x, y, vx, vy}
  float2 *mr;   // {mass, radius}
  uint32_t *id; // Body::id
  float4 *pv2;
  float2 *mr2;
  uint32_t *id2;
  float2 *acc;  // accelerations from the last force pass
  float4 *xym;  // {x, y, mass, 0} in Morton order (tree + forces)

  // bounds as float order keys: [seg][minX, maxX, minY, maxY]
  uint32_t *bounds;
  uint32_t *status; // error bits

  // collision scratch
  float4 *box;           // {minX, maxX, minY, maxY}
  int2 *cellXY;          // grid cell of small boxes
  uint32_t *slot;        // slot in bucket (small) or in large list (|bit31)
  uint32_t *bucketCount; // [buckets]
  uint32_t *bucketStart; // [buckets+1]
  uint32_t *grid;        // body index per bucket slot
  float4 *gridBox;       // the box of that body (read with the index)
  uint32_t nBuckets;     // power of two
  uint32_t *largeCount;  // [nseg]
  uint32_t *largeStartA; // [nseg]
  uint32_t *largeList;   // [n]
  uint32_t *deg;         // partners per body
  uint32_t *pstart;      // CSR start per body
  uint32_t *plist;       // partner indices
  uint32_t *plistTmp;    // scratch copy used to sort large bodies' lists
  uint32_t *twin;        // per as-later entry: the partner's chain entry
                         // (index | kFirstEntry | kLastEntry)
  float4 *chain;         // per chain entry: the body's state after it
                         // (published entries only; sentinel until then)
  uint32_t *stash;       // first partners of each body found by the count pass
  uint2 *largePairs;     // (large, small) pairs found by the count pass
  uint32_t *fillLarge;   // fill counters of large bodies
  uint32_t *nLater;      // partners that sort before the body
  uint32_t *unitOrder;   // units in before() order (last collide)
  uint32_t *longRuns;    // Morton sort: starts of runs of > 16 equal high keys
  uint32_t *counters;    // [0]=pairs*2 total [1]=units [2]=unit claim
                         // [3]=splitting entries [4]=total nodes
                         // [5]=small-large pairs [6]=traversal records
                         // [8]=id check
                         // [9]=long Morton runs [12]=upload mass bits
                         // [7]=bounds blocks done [10]=long unit runs
                         // [13]=expiry test flag [kCtrCoordLimit] (above)

  // Morton / sort
  uint64_t *codes; // unsorted codes (kept for the segment passes)
  uint32_t *perm;  // Morton permutation of the last build (sorted -> old)
  uint64_t *sortedCodes;

  // tree build
  uint32_t *splitCount; // per body
  uint32_t *splitStart;
  uint8_t *splitLo;
  uint32_t *groupStart; // [nseg][kLevelSlots]
  uint32_t *groupEnd;
  uint32_t *levelStart; // [nseg][kLevelSlots+1]
  // BFS-numbered node arrays (TreeKernels.cuh NodeArrays layout)
  float *comX, *comY, *mass, *centerX, *centerY, *size;
  int32_t *children, *next, *start, *end;
  int32_t *parent;
  float *sumX, *sumY;   // raw weighted sums (before the CoM divide)
  float4 *moments;      // {Ixx, Iyy, Ixy, spare}
  uint32_t *subtree;    // nodes in subtree
  uint32_t *arrive;     // bottom-up arrival counters
  // traversal layout (preorder)
  TravNode *tN; // preorder traversal records (32 bytes, one load each)
  float4 *tM; // {Ixx, Iyy, Ixy, size} for the learned correction
  float2 *tC; // square centre, for the learned correction

  // attractor: [0] = {x, y, mass, softening}, [1].x = active (0 or 1);
  // device-resident so it can move between steps of a captured graph
  float4 *attr;
};

// Camera and draw settings of the splat renderer (render.cu).
struct RenderParams {
  float camX, camY, scale, halfW, halfH;
  uint32_t width, height, tilesX, tilesY;
  int mode; // 0 speed ramp, over-composited; 1 glow, additive
  float pointScale, minPoint, brightness, speedMax;
};

// The viewer's attractor pull (attractorKernel, src/cuda/CudaSimulation.cu
// :14-31): acc += d * m / (sqrt(|d|^2 + 1e-12) (|d|^2 + soft^2)), d = a - p,
// added after the gravitational sum.  kExact: IEEE reciprocal square root
// and division, no contraction; otherwise the hardware rsqrt, an IEEE
// division and fused multiply-adds, as the reference's kernel compiles.
template <bool kExact>
__device__ __forceinline__ void add_attractor(const float4 *attr, float px, float py,
                                              float &ax, float &ay) {
  if (attr[1].x == 0.0f) return;
  const float4 a = attr[0];
  if (kExact) {
    const float dx = __fsub_rn(a.x, px), dy = __fsub_rn(a.y, py);
    const float dSq = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    const float f = __fdiv_rn(__fmul_rn(a.z, __frcp_rn(__fsqrt_rn(__fadd_rn(dSq, 1e-12f)))),
                              __fadd_rn(dSq, __fmul_rn(a.w, a.w)));
    ax = __fadd_rn(ax, __fmul_rn(dx, f));
    ay = __fadd_rn(ay, __fmul_rn(dy, f));
  } else {
    const float dx = a.x - px, dy = a.y - py;
    const float dSq = dx * dx + dy * dy;
    const float f = __fdiv_rn(a.z * rsqrtf(dSq + 1e-12f), dSq + a.w * a.w);
    ax = fmaf(dx, f, ax);
    ay = fmaf(dy, f, ay);
  }
}

__device__ __forceinline__ float key_to_float(uint32_t k) {
  return u2f((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Root square of instance sg (Quad::newContaining, QuadTree.cpp:30-51, and
// rootSquare, CudaQuadTree.cu:25-30) and its Morton frame, from the step's
// bound accumulators, which it resets for the next step.
__device__ __forceinline__ void root_frame_seg(const DevState &S, uint32_t sg) {
  uint32_t *b = S.bounds + 4 * sg;
  const uint32_t k0 = __ldcg(b), k1 = __ldcg(b + 1), k2 = __ldcg(b + 2), k3 = __ldcg(b + 3);
  const float minX = k0 == 0xffffffffu ? FLT_MAX : key_to_float(k0);
  const float maxX = k1 == 0u ? -FLT_MAX : key_to_float(k1);
  const float minY = k2 == 0xffffffffu ? FLT_MAX : key_to_float(k2);
  const float maxY = k3 == 0u ? -FLT_MAX : key_to_float(k3);
  const float cx = __fmul_rn(__fadd_rn(minX, maxX), 0.5f);
  const float cy = __fmul_rn(__fadd_rn(minY, maxY), 0.5f);
  const float w = __fsub_rn(maxX, minX), h = __fsub_rn(maxY, minY);
  const float size = (w < h) ? h : w;
  SegDev &G = S.seg[sg];
  G.cx = cx;
  G.cy = cy;
  G.size = size;
  // sd_morton_frame's binary64 steps in native FP64: the same IEEE
  // operations, each correctly rounded, give the same bits
  const double half = __dmul_rn(0.5, (double)size);
  G.frame.x0 = (uint64_t)__double_as_longlong(__dsub_rn((double)cx, half));
  G.frame.y0 = (uint64_t)__double_as_longlong(__dsub_rn((double)cy, half));
  G.frame.scale = size > 0.0f ? (uint64_t)__double_as_longlong(__ddiv_rn(4294967296.0, (double)size))
                              : 0ull;
  // clamp guard: bodies beyond the upload's coordinate limit (NaN-safe)
  const float lim = __uint_as_float(S.counters[kCtrCoordLimit]);
  const float reach = fmaxf(fmaxf(fabsf(minX), fabsf(maxX)), fmaxf(fabsf(minY), fabsf(maxY)));
  G.wide = (k0 != 0xffffffffu && !(reach < lim)) ? 1u : 0u;
  b[0] = 0xffffffffu;
  b[1] = 0u;
  b[2] = 0xffffffffu;
  b[3] = 0u;
}

} // namespace nbx
