// build.cu -- root square, Morton codes, Morton-order gather and the
// quadtree build, for every instance of a handle in one launch per phase.
//
// The tree is the reference's Morton tree (src/cuda/TreeKernels.cuh:68-177,
// driven as CudaQuadTree.cu:452-498): breadth-first node numbering, the 4
// children of a node consecutive at `children`, `next` skip pointers, body
// ranges [start, end), leaves of <= leafCapacity bodies (or at depth 32).
//
// The reference builds it level by level with grid-wide barriers.  Here
// every level is built at once, straight from the sorted codes:
//  * body i is the first body of the depth-d node containing it iff
//    d > lcp(code[i-1], code[i]); that node splits iff it holds more than
//    L bodies, i.e. code[i+L] shares its d-digit prefix, and d < 32.  So
//    body i starts the splitting nodes of depths [lo_i, hi_i] with
//    lo_i = lcp(i-1, i) + 1 and hi_i = min(lcp(i, i+L), 31);
//  * the (segment, depth, first body) entries are bucketed by depth with a
//    stable radix pass; a splitting node's rank among its level's
//    splitting nodes is its position in its bucket, which fixes the BFS
//    slot of its children (levelStart[d+1] + 4*rank), exactly the
//    numbering of the serial loop;
//  * centres are recomputed along the path from the root with the same
//    float operations as splitNode (bit-identical), and `next` is the slot
//    after the deepest ancestor that is not a last child;
//  * mass / centre-of-mass (and second moments) go up the tree with
//    arrival counters: the fourth child to finish sums its parent in the
//    fixed order c0+c1+c2+c3 of sumNode, so the sums are deterministic.
// A second pass lays the nodes out in depth-first preorder for the force
// traversal (force.cu).
#include "nbx_state.cuh"

#include <float.h>

namespace nbx {
namespace {

constexpr int kBlock = 256;

int grid_for(uint32_t n) {
  uint32_t b = (n + kBlock - 1) / kBlock;
  if (b > 148u * 16u) b = 148u * 16u;
  return b ? (int)b : 1;
}

// quantise() in native FP64 (TreeKernels.cuh:48-57): one IEEE subtract and
// one multiply, each rounded (no contraction), then floor -- the same
// doubles as the reference's, bit for bit, from the frame's binary64 bits.
__device__ __forceinline__ uint32_t quantise_fp64(float v, double lo, double scale) {
  const double q = floor(__dmul_rn(__dsub_rn((double)v, lo), scale));
  if (!(q > 0.0)) return 0u; // also NaN
  if (q >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)q;
}

// Morton code of every body; the sort key is its high half (depth-16
// cells), with the digit histograms of its four radix passes fused.
__global__ void __launch_bounds__(kBlock)
    k_morton(DevState S, uint32_t *__restrict__ keys, uint32_t *hist) {
  __shared__ uint32_t sh[4][256];
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) sh[i >> 8][i & 255] = 0;
  __syncthreads();
  const uint32_t n = S.n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const float4 p = S.pv[i];
    const MortonFrame f = S.seg[S.segOf[i]].frame;
    const double sc = __longlong_as_double((long long)f.scale);
    const uint64_t c =
        (spread_bits(quantise_fp64(p.y, __longlong_as_double((long long)f.y0), sc)) << 1) |
        spread_bits(quantise_fp64(p.x, __longlong_as_double((long long)f.x0), sc));
    const uint32_t k = (uint32_t)(c >> 32);
    keys[i] = k;
    S.codes[i] = c;
#pragma unroll
    for (int q = 0; q < 4; ++q) atomicAdd(&sh[q][(k >> (8 * q)) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
    const uint32_t v = sh[i >> 8][i & 255];
    if (v) atomicAdd(&hist[i], v);
  }
}

// Sort key for the instance passes: segment of the element's original index.
__global__ void k_seg_keys(DevState S, const uint32_t *__restrict__ vals,
                           uint32_t *__restrict__ keys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n;
       i += gridDim.x * blockDim.x)
    keys[i] = S.segOf[vals[i]];
}

// ------------------------------------------------------------ tree build

// Splitting nodes that start at body i: depths [lo, hi].
__global__ void __launch_bounds__(kBlock) k_split_counts(DevState S) {
  const uint64_t *c = S.sortedCodes;
  const int L = S.leafCapacity;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n;
       i += gridDim.x * blockDim.x) {
    const SegDev &G = S.seg[S.segOf[i]];
    const uint32_t s0 = G.start, s1 = G.start + G.count;
    const int lo = (i == s0) ? 0 : lcp_digits(c[i - 1], c[i]) + 1;
    int hi = -1;
    if ((uint64_t)i + (uint32_t)L < s1) {
      hi = lcp_digits(c[i], c[i + L]);
      if (hi > kMaxDepth - 1) hi = kMaxDepth - 1;
    }
    const int cnt = hi >= lo ? hi - lo + 1 : 0;
    S.splitCount[i] = (uint32_t)cnt;
    S.splitLo[i] = (uint8_t)(lo > 255 ? 255 : lo);
  }
}

__global__ void __launch_bounds__(kBlock)
    k_split_emit(DevState S, uint64_t *__restrict__ keys,
                 uint32_t *__restrict__ vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n;
       i += gridDim.x * blockDim.x) {
    const uint32_t cnt = S.splitCount[i];
    if (!cnt) continue;
    const uint32_t base = S.splitStart[i];
    const uint32_t lo = S.splitLo[i];
    const uint64_t sg = S.segOf[i];
    for (uint32_t k = 0; k < cnt; ++k) {
      keys[base + k] = (sg << 6) | (lo + k);
      vals[base + k] = i;
    }
  }
}

// Bucket boundaries of the depth-sorted entries.
__global__ void __launch_bounds__(kBlock)
    k_groups(DevState S, const uint64_t *__restrict__ keys) {
  const uint32_t total = S.counters[3];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += gridDim.x * blockDim.x) {
    const uint64_t key = keys[k];
    const uint32_t slot = (uint32_t)(key >> 6) * kLevelSlots + (uint32_t)(key & 63u);
    if (k == 0 || keys[k - 1] != key) S.groupStart[slot] = k;
    if (k + 1 == total || keys[k + 1] != key) S.groupEnd[slot] = k + 1;
  }
}

// Level starts, node counts and node bases per instance; root nodes.
__global__ void k_levels(DevState S) {
  __shared__ uint32_t sRun;
  if (threadIdx.x == 0) sRun = 0;
  __syncthreads();
  for (uint32_t base = 0; base < S.nseg; base += blockDim.x) {
    const uint32_t sg = base + threadIdx.x;
    uint32_t nodes = 0, levels = 0;
    if (sg < S.nseg) {
      SegDev &G = S.seg[sg];
      uint32_t *ls = S.levelStart + sg * (kLevelSlots + 1);
      const uint32_t *gs = S.groupStart + sg * kLevelSlots;
      const uint32_t *ge = S.groupEnd + sg * kLevelSlots;
      if (G.count > 0) {
        ls[0] = 0;
        ls[1] = 1;
        uint32_t maxLevel = 0; // deepest level with nodes
        for (int d = 1; d <= kMaxDepth; ++d) {
          const uint32_t split = ge[d - 1] - gs[d - 1];
          ls[d + 1] = ls[d] + 4u * split;
          if (split) maxLevel = d;
        }
        nodes = ls[maxLevel + 1];
        for (int d = maxLevel + 2; d <= kLevelSlots; ++d) ls[d] = nodes;
        levels = maxLevel + 1;
      } else {
        for (int d = 0; d <= kLevelSlots; ++d) ls[d] = 0;
      }
      G.nodeCount = nodes;
      G.levelCount = levels;
    }
    // block-wide exclusive scan of node counts -> node bases
    __shared__ uint32_t sScan[1024];
    sScan[threadIdx.x] = nodes;
    __syncthreads();
    for (uint32_t o = 1; o < blockDim.x; o <<= 1) {
      const uint32_t v = threadIdx.x >= o ? sScan[threadIdx.x - o] : 0u;
      __syncthreads();
      sScan[threadIdx.x] += v;
      __syncthreads();
    }
    const uint32_t excl = sRun + sScan[threadIdx.x] - nodes;
    if (sg < S.nseg) {
      SegDev &G = S.seg[sg];
      G.nodeBase = excl;
      if (excl + nodes <= S.nodeCapacity && nodes > 0) {
        const uint32_t r = excl;
        S.comX[r] = 0.0f;
        S.comY[r] = 0.0f;
        S.mass[r] = 0.0f;
        S.centerX[r] = G.cx;
        S.centerY[r] = G.cy;
        S.size[r] = G.size;
        S.children[r] = 0;
        S.next[r] = 0;
        S.start[r] = 0;
        S.end[r] = (int32_t)G.count;
        S.parent[r] = -1;
      }
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) sRun += sScan[blockDim.x - 1];
    __syncthreads();
  }
  __syncthreads();
  if (sRun > S.nodeCapacity) {
    // all-or-nothing: no instance gets a tree, the step reports the error
    for (uint32_t sg = threadIdx.x; sg < S.nseg; sg += blockDim.x)
      S.seg[sg].nodeCount = 0;
    if (threadIdx.x == 0) {
      atomicOr(S.status, kStatusTreeCapacity);
      S.counters[4] = 0;
    }
  } else if (threadIdx.x == 0) {
    S.counters[4] = sRun;
  }
}

// Index of the depth-t splitting node containing body i, by its rank.
__device__ __forceinline__ uint32_t split_rank(const DevState &S,
                                               const uint32_t *vals,
                                               uint32_t sg, int t, uint32_t i) {
  uint32_t lo = S.groupStart[sg * kLevelSlots + t];
  uint32_t hi = S.groupEnd[sg * kLevelSlots + t];
  const uint32_t g0 = lo;
  // last position with vals[pos] <= i
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (vals[mid] <= i) lo = mid + 1;
    else hi = mid;
  }
  return lo > g0 ? lo - 1 - g0 : 0u; // the parent always exists
}

// firstWithDigit (TreeKernels.cuh:72-85) over global body indices.
__device__ __forceinline__ uint32_t first_with_digit(const uint64_t *codes,
                                                     uint32_t lo, uint32_t hi,
                                                     int depth, int q) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (digit_at(codes[mid], depth) < q) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kBlock)
    k_split_nodes(DevState S, const uint64_t *__restrict__ keys,
                  const uint32_t *__restrict__ vals) {
  const uint32_t total = S.counters[3];
  const uint64_t *codes = S.sortedCodes;
  const uint32_t L = (uint32_t)S.leafCapacity;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += gridDim.x * blockDim.x) {
    const uint64_t key = keys[k];
    const uint32_t sg = (uint32_t)(key >> 6);
    const int d = (int)(key & 63u);
    const uint32_t i = vals[k];
    if (sg >= S.nseg || d >= kMaxDepth) continue;
    const SegDev &G = S.seg[sg];
    if (G.nodeCount == 0) continue; // capacity overflow: instance skipped
    const uint32_t nb = G.nodeBase;
    const uint32_t s0 = G.start, s1 = G.start + G.count;
    const uint32_t *ls = S.levelStart + sg * (kLevelSlots + 1);
    const uint32_t r = k - S.groupStart[sg * kLevelSlots + d];
    const uint64_t ci = codes[i];
    uint32_t own = 0;
    if (d > 0) own = ls[d] + 4u * split_rank(S, vals, sg, d - 1, i) +
                     (uint32_t)digit_at(ci, d - 1);
    const uint32_t childBase = ls[d + 1] + 4u * r;
    if (childBase + 4 > G.nodeCount || own >= G.nodeCount) {
      atomicOr(S.status, kStatusTreeCapacity);
      continue;
    }
    // end of this node's body range
    uint32_t end = s1;
    if (d > 0) {
      const uint64_t pre = ci >> (64 - 2 * d);
      uint32_t lo = i + 1, hi = s1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((codes[mid] >> (64 - 2 * d)) == pre) lo = mid + 1;
        else hi = mid;
      }
      end = lo;
    }
    uint32_t bound[5];
    bound[0] = i;
    bound[4] = end;
    for (int q = 1; q < 4; ++q)
      bound[q] = first_with_digit(codes, bound[q - 1], end, d, q);
    // centre and size along the path (splitNode's arithmetic)
    float cx = G.cx, cy = G.cy, size = G.size;
    for (int t = 0; t < d; ++t) {
      size = __fmul_rn(size, 0.5f);
      const int q = digit_at(ci, t);
      cx = __fadd_rn(cx, __fmul_rn((float)(q & 1) - 0.5f, size));
      cy = __fadd_rn(cy, __fmul_rn((float)(q >> 1) - 0.5f, size));
    }
    // own `next`: after the deepest ancestor-or-self that is not a last child
    uint32_t ownNext = 0;
    for (int t = d; t >= 1; --t) {
      const int q = digit_at(ci, t - 1);
      if (q < 3) {
        const uint32_t idx =
            (t == d) ? own
                     : ls[t] + 4u * split_rank(S, vals, sg, t - 1, i) + (uint32_t)q;
        ownNext = idx + 1;
        break;
      }
    }
    const float childSize = __fmul_rn(size, 0.5f);
    S.children[nb + own] = (int32_t)childBase;
    S.arrive[nb + own] = 0;
    for (int q = 0; q < 4; ++q) {
      const uint32_t ch = nb + childBase + q;
      S.comX[ch] = 0.0f;
      S.comY[ch] = 0.0f;
      S.mass[ch] = 0.0f;
      S.centerX[ch] = __fadd_rn(cx, __fmul_rn((float)(q & 1) - 0.5f, childSize));
      S.centerY[ch] = __fadd_rn(cy, __fmul_rn((float)(q >> 1) - 0.5f, childSize));
      S.size[ch] = childSize;
      S.next[ch] = (int32_t)(q < 3 ? childBase + q + 1 : ownNext);
      S.start[ch] = (int32_t)(bound[q] - s0);
      S.end[ch] = (int32_t)(bound[q + 1] - s0);
      S.parent[ch] = (int32_t)own;
      const bool splits = bound[q + 1] - bound[q] > L && d + 1 < kMaxDepth;
      if (!splits) S.children[ch] = 0;
    }
  }
}

__device__ __forceinline__ uint32_t seg_of_node(const DevState &S, uint32_t g) {
  uint32_t lo = 0, hi = S.nseg;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (S.seg[mid].nodeBase <= g) lo = mid;
    else hi = mid;
  }
  // skip empty instances sharing the same base
  while (lo + 1 < S.nseg && S.seg[lo].nodeCount == 0 && S.seg[lo + 1].nodeBase <= g)
    ++lo;
  return lo;
}

// Bottom-up pass: leaves sum their bodies (sumNode order), the last of
// four children to finish sums their parent, then finishNode's divide.
__global__ void __launch_bounds__(kBlock) k_upward(DevState S) {
  const uint32_t total = S.counters[4];
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += gridDim.x * blockDim.x) {
    if (S.children[g] != 0) continue;
    const uint32_t sg = seg_of_node(S, g);
    const SegDev &G = S.seg[sg];
    const uint32_t nb = G.nodeBase, s0 = G.start;
    const uint32_t b0 = s0 + (uint32_t)S.start[g], b1 = s0 + (uint32_t)S.end[g];
    float px = 0.0f, py = 0.0f, mm = 0.0f;
    for (uint32_t b = b0; b < b1; ++b) {
      const float4 q = S.xym[b];
      px = __fadd_rn(px, __fmul_rn(q.x, q.z));
      py = __fadd_rn(py, __fmul_rn(q.y, q.z));
      mm = __fadd_rn(mm, q.z);
    }
    const float div = fmaxf(mm, FLT_MIN);
    const float X = __fdiv_rn(px, div), Y = __fdiv_rn(py, div);
    float ixx = 0.0f, iyy = 0.0f, ixy = 0.0f;
    for (uint32_t b = b0; b < b1; ++b) {
      const float4 q = S.xym[b];
      const float dx = q.x - X, dy = q.y - Y;
      ixx += q.z * dx * dx;
      iyy += q.z * dy * dy;
      ixy += q.z * dx * dy;
    }
    S.sumX[g] = px;
    S.sumY[g] = py;
    S.mass[g] = mm;
    S.comX[g] = X;
    S.comY[g] = Y;
    S.moments[g] = make_float4(ixx, iyy, ixy, 0.0f);
    // empty leaves (no bodies) add nothing whether accepted or opened, so
    // the traversal layout leaves them out
    S.subtree[g] = b1 > b0 ? 1u : 0u;
    // climb (at most kMaxDepth levels; parent indices are range-checked)
    int32_t node = S.parent[g];
    for (int guard = 0; node >= 0 && guard <= kMaxDepth; ++guard) {
      if ((uint32_t)node >= G.nodeCount) {
        atomicOr(S.status, kStatusTreeCapacity);
        break;
      }
      const uint32_t pg = nb + (uint32_t)node;
      // release: this child's sums are visible to the last arriver; acquire:
      // the last arriver sees all four children's sums
      uint32_t old;
      asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                   : "=r"(old)
                   : "l"(&S.arrive[pg])
                   : "memory");
      if (old != 3u) break;
      const uint32_t c = nb + (uint32_t)S.children[pg];
      float sx = __ldcg(&S.sumX[c]), sy = __ldcg(&S.sumY[c]),
            sm = __ldcg(&S.mass[c]);
      uint32_t sub = 1 + __ldcg(&S.subtree[c]);
      for (int q = 1; q < 4; ++q) {
        sx = __fadd_rn(sx, __ldcg(&S.sumX[c + q]));
        sy = __fadd_rn(sy, __ldcg(&S.sumY[c + q]));
        sm = __fadd_rn(sm, __ldcg(&S.mass[c + q]));
        sub += __ldcg(&S.subtree[c + q]);
      }
      const float dv = fmaxf(sm, FLT_MIN);
      const float PX = __fdiv_rn(sx, dv), PY = __fdiv_rn(sy, dv);
      float jxx = 0.0f, jyy = 0.0f, jxy = 0.0f;
      for (int q = 0; q < 4; ++q) {
        const float4 mo = __ldcg(&S.moments[c + q]);
        const float cm = __ldcg(&S.mass[c + q]);
        const float dx = __ldcg(&S.comX[c + q]) - PX;
        const float dy = __ldcg(&S.comY[c + q]) - PY;
        jxx += mo.x + cm * dx * dx;
        jyy += mo.y + cm * dy * dy;
        jxy += mo.z + cm * dx * dy;
      }
      __stcg(&S.sumX[pg], sx);
      __stcg(&S.sumY[pg], sy);
      __stcg(&S.mass[pg], sm);
      __stcg(&S.comX[pg], PX);
      __stcg(&S.comY[pg], PY);
      __stcg(&S.moments[pg], make_float4(jxx, jyy, jxy, 0.0f));
      __stcg(&S.subtree[pg], sub);
      node = S.parent[pg];
    }
  }
}

// ------------------------------------------- traversal layout, built directly
//
// The force traversal needs only the non-empty nodes, in depth-first
// preorder, and those follow straight from the sorted codes:
//  * a node is (first body i, depth d).  The nodes starting at body i have
//    depths lo_i .. leaf_i: lo_i = lcp(i-1, i) + 1 (0 at an instance's
//    first body), and leaf_i is the depth of i's leaf.  A node containing
//    i splits iff it holds more than L bodies, i.e. iff some window
//    [j, j+L] of the instance around i shares its prefix, so
//    leaf_i = min(max over j in [i-L, i] of lcp(j, j+L), 31) + 1 (0 when no
//    window fits);
//  * in preorder, the nodes starting at i follow every node that starts
//    before i, shallowest first: with P = the exclusive scan of the counts,
//    node (i, d) is record P_i + d - lo_i;
//  * its subtree ends at the first body e past its prefix group, and the
//    record after the subtree is the first node starting at e, P_e;
//  * sums go up with arrival counters over the non-empty children in digit
//    order.  An empty child adds exactly +0 to sums that are never -0 (they
//    start at +0 and only add), so mass and centre of mass equal
//    sumNode/finishNode's over all four children (TreeKernels.cuh:150-177)
//    bit for bit.
// This replaces the breadth-first arrays on the step path; those are built
// only when asked for (launch_bfs_tree).

// Permute the state into Morton order (the 7 gathers of
// CudaQuadTree.cu:408-414, fused), write the {x, y, m} traversal array and,
// from the same sorted codes staged in shared memory, the traversal records
// that start at each body: their count (splitCount) and the depth of the
// first (splitLo).  hi_j = min(lcp(j, j+L), 31) (-1 when j+L leaves the
// instance) is formed once per body, then each body takes the maximum over
// its L+1 windows.  Each block takes 256 consecutive bodies and stages the
// codes of bodies [b0 - L, b0 + 256 + L) through the permutation, so the
// counts need no pass after the gather.
constexpr int kMaxLeafCap = 64; // nbx_params leaf_capacity bound
__global__ void __launch_bounds__(kBlock)
    k_gather_counts(DevState S, const uint32_t *__restrict__ perm) {
  __shared__ uint64_t sC[kBlock + 2 * kMaxLeafCap];
  __shared__ int8_t sHi[kBlock + kMaxLeafCap];
  const uint32_t n = S.n;
  const uint32_t L = (uint32_t)S.leafCapacity;
  for (uint32_t b0 = blockIdx.x * kBlock; b0 < n; b0 += gridDim.x * kBlock) {
    const uint32_t jBase = b0 >= L ? b0 - L : 0u;
    const uint32_t cEnd = min(n, b0 + kBlock + L); // codes [jBase, cEnd)
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < cEnd - jBase; t += kBlock)
      sC[t] = S.codes[perm[jBase + t]];
    const uint32_t i = b0 + threadIdx.x;
    if (i < n) {
      const uint32_t p = perm[i];
      const float4 v = S.pv[p];
      const float2 m = S.mr[p];
      S.pv2[i] = v;
      S.mr2[i] = m;
      S.id2[i] = S.id[p];
      S.xym[i] = make_float4(v.x, v.y, m.x, 0.0f);
      S.perm[i] = p;
    }
    __syncthreads();
    if (i < n) S.sortedCodes[i] = sC[i - jBase];
    // windows j in [jBase, b0 + kBlock)
    for (uint32_t t = threadIdx.x; t < b0 + kBlock - jBase; t += kBlock) {
      const uint32_t j = jBase + t;
      int hi = -1;
      if (j < n) {
        const SegDev &G = S.seg[S.segOf[j]];
        if ((uint64_t)j + L < (uint64_t)G.start + G.count)
          hi = min(lcp_digits(sC[t], sC[t + L]), kMaxDepth - 1);
      }
      sHi[t] = (int8_t)hi;
    }
    __syncthreads();
    if (i >= n) continue;
    const SegDev &G = S.seg[S.segOf[i]];
    const uint32_t s0 = G.start;
    const int lo = (i == s0) ? 0 : lcp_digits(sC[i - 1 - jBase], sC[i - jBase]) + 1;
    int w = -1;
    for (uint32_t j = i >= s0 + L ? i - L : s0; j <= i; ++j) w = max(w, (int)sHi[j - jBase]);
    const int leaf = w + 1;
    S.splitCount[i] = lo <= leaf ? (uint32_t)(leaf - lo + 1) : 0u;
    S.splitLo[i] = (uint8_t)lo; // <= 33
  }
}

// First index in (i, e] whose depth-d prefix differs from code[i]'s (pre),
// given that the codes from e on all differ (a gallop, then a binary
// search).  d >= 1.
__device__ __forceinline__ uint32_t prefix_end(const uint64_t *c, uint32_t i, uint32_t e,
                                               int d, uint64_t pre) {
  const int sh = 64 - 2 * d;
  uint32_t lo = i + 1, hi = e, step = 1;
  while (lo < hi) {
    const uint32_t probe = lo + step - 1;
    if (probe >= hi) break;
    if ((c[probe] >> sh) != pre) {
      hi = probe;
      break;
    }
    lo = probe + 1;
    step <<= 1;
  }
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((c[mid] >> sh) == pre) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// First index in [s0, i] with the depth-d prefix of code[i] (a gallop
// backwards, then a binary search).  d >= 1.
__device__ __forceinline__ uint32_t prefix_start(const uint64_t *c, uint32_t s0,
                                                 uint32_t i, int d) {
  const int sh = 64 - 2 * d;
  const uint64_t pre = c[i] >> sh;
  uint32_t lo = s0, hi = i, step = 1; // answer in [lo, hi]
  while (hi > lo) {
    const uint32_t probe = hi - lo >= step ? hi - step : lo;
    if ((c[probe] >> sh) != pre) {
      lo = probe + 1;
      break;
    }
    hi = probe;
    if (probe == lo) break;
    step <<= 1;
  }
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((c[mid] >> sh) == pre) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Record of the node at depth d starting at body b.
__device__ __forceinline__ uint32_t record_of(const DevState &S, uint32_t b, int d) {
  return S.splitStart[b] + (uint32_t)(d - (int)S.splitLo[b]);
}

// One thread per record: body range, next and open slots, size and centre
// (splitNode's arithmetic along the path), parent, the records of the
// non-empty children in digit order (all ones past the last); arrival
// counters cleared.  kFull: also the cell centres and sizes of tC/tM (read
// only by the corrected forms and the network's harvest).
template <bool kFull>
__global__ void __launch_bounds__(kBlock)
    k_trav_nodes(DevState S, const uint32_t *__restrict__ owner, uint4 *__restrict__ kids) {
  const uint64_t *c = S.sortedCodes;
  const uint32_t total = S.counters[6];
  const bool overflow = total > S.nodeCapacity;
  if (blockIdx.x == 0) {
    // instance bases: all-or-nothing on overflow (the step reports it)
    for (uint32_t sg = threadIdx.x; sg < S.nseg; sg += blockDim.x) {
      SegDev &G = S.seg[sg];
      if (G.count == 0) continue;
      const uint32_t s0 = G.start, s1 = G.start + G.count;
      const uint32_t P = S.splitStart[s0];
      G.travBase = overflow ? 0u : P;
      G.travCount = overflow ? 0u : (s1 < S.n ? S.splitStart[s1] : total) - P;
    }
    if (overflow && threadIdx.x == 0) atomicOr(S.status, kStatusTreeCapacity);
  }
  if (overflow) return;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total;
       p += gridDim.x * blockDim.x) {
    const uint32_t i = owner[p];
    const SegDev &G = S.seg[S.segOf[i]];
    const uint32_t s0 = G.start, s1 = G.start + G.count;
    const uint32_t P = S.splitStart[i];
    const uint32_t k = p - P;
    const int lo = S.splitLo[i];
    const int d = lo + (int)k;
    const bool leaf = k + 1 == S.splitCount[i];
    const uint64_t ci = c[i];
    float cx = G.cx, cy = G.cy, size = G.size;
    if (kFull || !(fabsf(G.size) >= 0x1p-90f && fabsf(G.size) <= 0x1p+120f)) {
      for (int t = 0; t < d; ++t) {
        size = __fmul_rn(size, 0.5f);
        const int q = digit_at(ci, t);
        cx = __fadd_rn(cx, __fmul_rn((float)(q & 1) - 0.5f, size));
        cy = __fadd_rn(cy, __fmul_rn((float)(q >> 1) - 0.5f, size));
      }
    } else {
      // d <= 32 halvings of a normal size stay normal: each is exact, so
      // the repeated halving is one exponent step
      size = ldexpf(size, -d);
    }
    const uint32_t e = d > 0 ? prefix_end(c, i, s1, d, ci >> (64 - 2 * d)) : s1;
    // the record after the subtree; all ones past the instance's last
    const uint32_t next = e < s1 ? S.splitStart[e] : 0xffffffffu;
    int32_t parent = -1;
    if (d > 0) {
      if (k > 0) {
        parent = (int32_t)(p - 1);
      } else {
        // the depth-(d-1) node around i starts before it (the root at s0)
        const uint32_t j = d == 1 ? s0 : prefix_start(c, s0, i, d - 1);
        parent = (int32_t)record_of(S, j, d - 1);
      }
    }
    uint4 ch = make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu);
    uint32_t children = 0;
    if (!leaf) {
      uint32_t bound[5];
      bound[0] = i;
      bound[4] = e;
      for (int q = 1; q < 4; ++q) bound[q] = first_with_digit(c, bound[q - 1], e, d, q);
      uint32_t r[4];
      for (int q = 0; q < 4; ++q)
        if (bound[q + 1] > bound[q]) r[children++] = record_of(S, bound[q], d + 1);
      for (uint32_t q = children; q < 4; ++q) r[q] = 0xffffffffu;
      ch = make_uint4(r[0], r[1], r[2], r[3]);
    }
    TravNode &T = S.tN[p];
    T.a = make_float4(0.0f, 0.0f, 0.0f, __fmul_rn(size, size));
    T.b = make_int4((int)next, (int)(leaf ? next : p + 1), (int)i, (int)e);
    if (kFull) {
      S.tM[p] = make_float4(0.0f, 0.0f, 0.0f, size);
      S.tC[p] = make_float2(cx, cy);
    }
    S.parent[p] = parent;
    S.subtree[p] = children;
    S.arrive[p] = 0u;
    kids[p] = ch;
  }
}

// Bottom-up sums over the traversal records: each leaf sums its bodies
// (sumNode's order) and climbs; the last non-empty child to arrive sums its
// parent's children in digit order, then finishNode's divide; second
// moments about each centre of mass for the corrected forms.
template <bool kMoments>
__global__ void __launch_bounds__(kBlock)
    k_trav_upward(DevState S, const uint4 *__restrict__ kids) {
  const uint32_t total = S.counters[6];
  if (total > S.nodeCapacity) return;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total;
       p += gridDim.x * blockDim.x) {
    if (S.subtree[p] != 0) continue; // interior: summed by its last child
    const int4 B = S.tN[p].b;
    const uint32_t b0 = (uint32_t)B.z, b1 = min((uint32_t)B.w, S.n);
    float px = 0.0f, py = 0.0f, mm = 0.0f;
    for (uint32_t b = b0; b < b1; ++b) {
      const float4 q = S.xym[b];
      px = __fadd_rn(px, __fmul_rn(q.x, q.z));
      py = __fadd_rn(py, __fmul_rn(q.y, q.z));
      mm = __fadd_rn(mm, q.z);
    }
    const float div = fmaxf(mm, FLT_MIN);
    const float X = __fdiv_rn(px, div), Y = __fdiv_rn(py, div);
    if (kMoments) {
      float ixx = 0.0f, iyy = 0.0f, ixy = 0.0f;
      for (uint32_t b = b0; b < b1; ++b) {
        const float4 q = S.xym[b];
        const float dx = q.x - X, dy = q.y - Y;
        ixx += q.z * dx * dx;
        iyy += q.z * dy * dy;
        ixy += q.z * dx * dy;
      }
      __stcg(&S.tM[p], make_float4(ixx, iyy, ixy, S.tM[p].w));
    }
    __stcg(&S.sumX[p], px);
    __stcg(&S.sumY[p], py);
    __stcg(&S.tN[p].a, make_float4(X, Y, mm, S.tN[p].a.w));
    int32_t node = S.parent[p];
    for (int guard = 0; node >= 0 && guard <= kMaxDepth; ++guard) {
      const uint32_t g = (uint32_t)node;
      if (g >= total) {
        atomicOr(S.status, kStatusTreeCapacity);
        break;
      }
      const uint32_t children = S.subtree[g];
      // release: this child's sums are visible to the last arriver;
      // acquire: the last arriver sees every child's sums
      uint32_t old;
      asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                   : "=r"(old)
                   : "l"(&S.arrive[g])
                   : "memory");
      if (old + 1 != children) break;
      const uint4 kv = kids[g];
      const uint32_t r[4] = {kv.x, kv.y, kv.z, kv.w};
      float cxs[4], cys[4];
      float4 ca[4], mo[4];
      for (uint32_t q = 0; q < 4; ++q) {
        if (q >= children || r[q] >= total) continue;
        cxs[q] = __ldcg(&S.sumX[r[q]]);
        cys[q] = __ldcg(&S.sumY[r[q]]);
        ca[q] = __ldcg(&S.tN[r[q]].a);
        if (kMoments) mo[q] = __ldcg(&S.tM[r[q]]);
      }
      float sx = 0.0f, sy = 0.0f, sm = 0.0f;
      for (uint32_t q = 0; q < children && q < 4; ++q) {
        if (r[q] >= total) break;
        sx = q == 0 ? cxs[q] : __fadd_rn(sx, cxs[q]);
        sy = q == 0 ? cys[q] : __fadd_rn(sy, cys[q]);
        sm = q == 0 ? ca[q].z : __fadd_rn(sm, ca[q].z);
      }
      const float dv = fmaxf(sm, FLT_MIN);
      const float PX = __fdiv_rn(sx, dv), PY = __fdiv_rn(sy, dv);
      if (kMoments) {
        float jxx = 0.0f, jyy = 0.0f, jxy = 0.0f;
        for (uint32_t q = 0; q < children && q < 4; ++q) {
          if (r[q] >= total) break;
          const float dx = ca[q].x - PX, dy = ca[q].y - PY;
          jxx += mo[q].x + ca[q].z * dx * dx;
          jyy += mo[q].y + ca[q].z * dy * dy;
          jxy += mo[q].z + ca[q].z * dx * dy;
        }
        __stcg(&S.tM[g], make_float4(jxx, jyy, jxy, S.tM[g].w));
      }
      __stcg(&S.sumX[g], sx);
      __stcg(&S.sumY[g], sy);
      __stcg(&S.tN[g].a, make_float4(PX, PY, sm, S.tN[g].a.w));
      node = S.parent[g];
    }
  }
}

} // namespace

void launch_bounds(cudaStream_t s, const DevState &S);
void launch_trav_tree(cudaStream_t s, const DevState &S, ScanScratch &scan, bool moments);

void launch_build(cudaStream_t s, DevState &S, ScanScratch &scan,
                  SortScratch &sort, bool moments) {
  const uint32_t n = S.n;
  launch_bounds(s, S); // and the root frames (its last block)
  mark(s, "build.bounds");
  // digit rows, tile counters, look-back words and the long-run count were
  // cleared by the step prologue (launch_step_zero)
  k_morton<<<grid_for(n), kBlock, 0, s>>>(S, keys32(sort, 0), sort.hist);
  mark(s, "build.morton");
  // radix passes over the codes' high 32 bits (depth-16 cells), then every
  // run of equal high bits is ordered by its low bits: the same stable order
  // as a full 64-bit sort; such runs are rare and short (at most 2 bodies in
  // the headline states), so this replaces four full passes
  int buf = radix_sort_u32(s, sort, n, nullptr, 0, 32, true, true, S.status, 0, true);
  sort_fix_low_bits32(s, sort, buf, n, S.codes, S.longRuns, &S.counters[9], n / 16 + 64,
                      S.status, true);
  mark(s, "build.sort");
  if (S.nseg > 1) {
    // stable passes on the instance id keep instances in their ranges
    k_seg_keys<<<grid_for(n), kBlock, 0, s>>>(S, sort.vals[buf], keys32(sort, buf));
    if (buf == 1) {
      cudaMemcpyAsync(keys32(sort, 0), keys32(sort, 1), sizeof(uint32_t) * n,
                      cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(sort.vals[0], sort.vals[1], sizeof(uint32_t) * n,
                      cudaMemcpyDeviceToDevice, s);
    }
    const int segBits = S.nseg <= 256 ? 8 : 16;
    buf = radix_sort_u32(s, sort, n, nullptr, 0, segBits, false, false, S.status);
  }
  k_gather_counts<<<grid_for(n), kBlock, 0, s>>>(S, sort.vals[buf]);
  mark(s, "build.gather");
  // swap the double-buffered state: the host mirrors this swap
  DevState T = S;
  T.pv = S.pv2;
  T.mr = S.mr2;
  T.id = S.id2;
  T.pv2 = S.pv;
  T.mr2 = S.mr;
  T.id2 = S.id;
  S = T;
  launch_trav_tree(s, S, scan, moments);
}

// The traversal layout straight from the sorted codes (the step path).
// moments: the cells' second moments, centres and sizes too (tM, tC: only
// the corrected forms and the network's harvest read them).
void launch_trav_tree(cudaStream_t s, const DevState &S, ScanScratch &scan, bool moments) {
  const uint32_t n = S.n;
  // per-record scratch in arrays only the breadth-first build uses
  uint32_t *owner = reinterpret_cast<uint32_t *>(S.start);
  uint4 *kids = reinterpret_cast<uint4 *>(S.moments);
  // the records per body (splitCount, splitLo) came with the gather
  // the scan also writes each record's first body (owner)
  exclusive_scan_u32(s, S.splitCount, S.splitStart, n, nullptr, &S.counters[6],
                     scan, S.status, owner, S.nodeCapacity, 3);
  mark(s, "tree.counts");
  if (moments)
    k_trav_nodes<true><<<grid_for(n / 2 + 64), kBlock, 0, s>>>(S, owner, kids);
  else
    k_trav_nodes<false><<<grid_for(n / 2 + 64), kBlock, 0, s>>>(S, owner, kids);
  mark(s, "tree.nodes");
  if (moments)
    k_trav_upward<true><<<grid_for(n / 4 + 64), kBlock, 0, s>>>(S, kids);
  else
    k_trav_upward<false><<<grid_for(n / 4 + 64), kBlock, 0, s>>>(S, kids);
  mark(s, "tree.upward");
}

// The reference's breadth-first node arrays (TreeKernels.cuh:88-95) of the
// last build, for introspection only: the step path does not need them.
// Uses the per-body split scratch and the sort scratch, and leaves the
// traversal layout as it is.
void launch_bfs_tree(cudaStream_t s, const DevState &S, ScanScratch &scan,
                     SortScratch &sort) {
  const uint32_t n = S.n;
  k_split_counts<<<grid_for(n), kBlock, 0, s>>>(S);
  exclusive_scan_u32(s, S.splitCount, S.splitStart, n, nullptr, &S.counters[3],
                     scan, S.status);
  k_split_emit<<<grid_for(n), kBlock, 0, s>>>(S, sort.keys[0], sort.vals[0]);
  const int depthBits = S.nseg <= 4 ? 8 : (S.nseg <= 1024 ? 16 : 24);
  const int eb = radix_sort_u64(s, sort, 2 * n + 64, &S.counters[3], 0,
                                depthBits, false, false, S.status);
  cudaMemsetAsync(S.groupStart, 0, sizeof(uint32_t) * S.nseg * kLevelSlots, s);
  cudaMemsetAsync(S.groupEnd, 0, sizeof(uint32_t) * S.nseg * kLevelSlots, s);
  k_groups<<<grid_for(2 * n), kBlock, 0, s>>>(S, sort.keys[eb]);
  k_levels<<<1, 1024, 0, s>>>(S);
  k_split_nodes<<<grid_for(n / 4 + 64), kBlock, 0, s>>>(S, sort.keys[eb],
                                                        sort.vals[eb]);
  k_upward<<<grid_for(n), kBlock, 0, s>>>(S);
}

} // namespace nbx
