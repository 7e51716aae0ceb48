// force.cu -- warp-cooperative stackless Barnes-Hut traversal.
//
// Each lane walks the tree for one body exactly as accelerationAt does
// (src/cuda/TreeKernels.cuh:197-245; QuadTree::acceleration,
// src/QuadTree.cpp:264-389): accept a node when size^2 < d^2*theta^2 and
// add m*d*fastInvSqrt(d^2)/(d^2+eps^2) (clamped to FLT_MAX), otherwise sum
// a leaf's bodies one by one, otherwise descend.  Per-lane acceptance is
// kept, so each body opens exactly the nodes the reference opens and sums
// them in the same order.
//
// The warp cooperates through the depth-first preorder layout (build.cu):
// along every lane's walk the preorder position only increases (descend =
// +1, skip = +subtree size), so the warp always serves the smallest
// position any lane is waiting at.  The node's record is read once per
// warp (one broadcast load through L1; staging 32-node tiles in shared
// memory measured 9-11% slower for the extra per-iteration bookkeeping);
// a leaf's bodies are staged in shared memory with one coalesced load.
//
// kExact = true evaluates every float operation as the reference writes
// it (no FMA contraction, IEEE reciprocal): the result is bit-identical to
// the host-compiled reference traversal on the same tree.  kExact = false
// lets the compiler contract and uses the hardware reciprocal
// approximation (relative difference ~1e-7 per term).
#include "mlp.cuh"
#include "nbx_state.cuh"

#include <float.h>

namespace nbx {
namespace {

constexpr int kForceBlock = 256;
constexpr int kWarps = kForceBlock / 32;
constexpr uint32_t kDone = 0xffffffffu;

// One traversal record with a single 256-bit read-only load (sm_100); the
// records are 32-byte aligned (TravNode).
__device__ __forceinline__ void ld_node(const TravNode *p, float4 &a, int4 &b) {
  asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z),
        "=r"(b.w)
      : "l"(p));
}

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <bool kExact>
__device__ __forceinline__ float inv_sqrt_law(float x) {
  if (kExact) {
    const float xhalf = __fmul_rn(0.5f, x);
    const float y = u2f(0x5f3759dfu - (f2u(x) >> 1));
    return __fmul_rn(y, __fsub_rn(1.5f, __fmul_rn(__fmul_rn(xhalf, y), y)));
  } else {
    return fast_inv_sqrt(x);
  }
}

// The tree force law's factor m * fastInvSqrt(d^2) / (d^2 + eps^2), clamped
// to FLT_MAX (the term is d * factor).  kClamp = false leaves the clamp out
// where it cannot act: fastInvSqrt never exceeds ~2e19 (its value at 0), so
// with eps > 0 and every |m| < 1.6e19 * min(1, eps^2) neither m * fastInvSqrt
// nor the factor reaches FLT_MAX (the host checks this before choosing it).
template <bool kExact, bool kClamp = true>
__device__ __forceinline__ float law_factor(float dSq, float m, float eSq) {
  if (kExact)
    return fminf(__fmul_rn(__fmul_rn(m, inv_sqrt_law<true>(dSq)),
                           __frcp_rn(__fadd_rn(dSq, eSq))),
                 FLT_MAX);
  const float f = m * inv_sqrt_law<false>(dSq) * rcp_approx(dSq + eSq);
  return kClamp ? fminf(f, FLT_MAX) : f;
}

// One interaction of the tree force law; accumulates into (ax, ay).
template <bool kExact, bool kClamp = true>
__device__ __forceinline__ void add_term(float dx, float dy, float dSq,
                                         float m, float eSq, float &ax,
                                         float &ay) {
  if (kExact) {
    const float f = fminf(__fmul_rn(__fmul_rn(m, inv_sqrt_law<true>(dSq)),
                                    __frcp_rn(__fadd_rn(dSq, eSq))),
                          FLT_MAX);
    ax = __fadd_rn(ax, __fmul_rn(dx, f));
    ay = __fadd_rn(ay, __fmul_rn(dy, f));
  } else {
    const float f = law_factor<false, kClamp>(dSq, m, eSq);
    ax = fmaf(dx, f, ax);
    ay = fmaf(dy, f, ay);
  }
}

template <bool kExact>
__device__ __forceinline__ float sq_dist(float dx, float dy) {
  if (kExact) return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  return fmaf(dx, dx, dy * dy);
}

// kCount: instead of writing accelerations, add the walk's far (accepted,
// mass > 0), near (leaf body terms) and visited-node counts to counts[0..2].
// Second-order (quadrupole) term of the softened law for a cell with mass
// M and second moments I about its centre of mass, relative to the kernel
// g(r) = 1/(r (r^2 + eps^2)) of the monopole M g d:
//   delta = 1/2 [ (g'/r)(2 I d + tr(I) d) + (g''/r^2 - g'/r^3) d (d'Id) ],
// returned divided by M g so that the cell term is fac * (d + delta/(M g)).
__device__ __forceinline__ void quad_term(float dx, float dy, float dSq,
                                          float eSq, float mass, float ixx,
                                          float iyy, float ixy, float &qx,
                                          float &qy) {
  const float q = dSq + eSq;
  // a correction term: the hardware reciprocal's ~1 ulp is far below its
  // own truncation error
  const float iq = rcp_approx(q), ir2 = rcp_approx(dSq);
  const float c3 = 3.0f * dSq + eSq;
  const float aOverG = -c3 * ir2 * iq;                        // g'/(r g)
  const float gpp = -6.0f * iq + c3 * (2.0f * ir2 * iq + 4.0f * iq * iq);
  const float bOverG = gpp * ir2 + c3 * ir2 * ir2 * iq;       // B / g
  const float Idx = ixx * dx + ixy * dy, Idy = ixy * dx + iyy * dy;
  const float tr = ixx + iyy;
  const float dId = dx * Idx + dy * Idy;
  const float h = 0.5f * rcp_approx(mass);
  qx = h * (aOverG * (2.0f * Idx + tr * dx) + bOverG * dx * dId);
  qy = h * (aOverG * (2.0f * Idy + tr * dy) + bOverG * dy * dId);
}

// One warp's walk: lane targets (x, y) start at node cur (kDone: none) and
// add their terms to (ax, ay); kCount adds the walk's counts instead.
// kCorr = 1: accepted cells with size^2 >= d^2 * band^2 get the learned
// correction (mlp.cuh), evaluated for the warp's rows on tensor cores;
// kCorr = 2: they get the analytic quadrupole term instead (the control).
template <bool kExact, bool kCount, int kCorr, bool kClamp>
__device__ __forceinline__ void walk_targets(
    const DevState &S, float tSq, float eSq, float bandSq, float eps, float x, float y,
    uint32_t cur, float4 *sBodyW, const MlpDev &sW, __nv_bfloat16 (*sStageW)[16],
    float &ax, float &ay, uint32_t &nFar, uint32_t &nNear, uint32_t &nVisit,
    uint32_t &nIter, uint32_t &nChunk) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    const uint32_t k = __reduce_min_sync(0xffffffffu, cur);
    if (k == kDone) break;
    if (kCount) ++nIter;
    // k is the same for the whole warp: one broadcast 256-bit load
    float4 A;
    int4 B;
    ld_node(&S.tN[k], A, B);
    // the node after k's subtree (kDone past the instance's last node)
    const uint32_t nxt = (uint32_t)B.x;
    // every lane evaluates the node; only the lanes waiting at it use it
    const bool at = cur == k;
    const float dx = kExact ? __fsub_rn(A.x, x) : A.x - x;
    const float dy = kExact ? __fsub_rn(A.y, y) : A.y - y;
    const float dSq = sq_dist<kExact>(dx, dy);
    const float far = kExact ? __fmul_rn(dSq, tSq) : dSq * tSq;
    const bool accept = at && A.w < far;
    const bool openLeaf = at && !accept && B.y == B.x; // leaf: open == next
    {
      // the reference adds a cell only if its mass is > 0; in the clamp-free
      // plain walk masses are >= 0 and every term is finite, so a massless
      // cell's term is exactly +-0 and the mass test can go
      constexpr bool kZeroMassAddsNothing = !kExact && !kClamp && kCorr == 0;
      const bool use = accept && (kZeroMassAddsNothing || A.z > 0.0f);
      const float fac = law_factor<kExact, kClamp>(dSq, A.z, eSq);
      float tx, ty;
      if (kExact) {
        tx = __fadd_rn(ax, __fmul_rn(dx, fac));
        ty = __fadd_rn(ay, __fmul_rn(dy, fac));
      } else {
        tx = fmaf(dx, fac, ax);
        ty = fmaf(dy, fac, ay);
      }
      if (kCorr == 2) {
        const bool band = use && A.w >= dSq * bandSq;
        if (__ballot_sync(0xffffffffu, band)) {
          const float4 M = S.tM[k];
          float qx, qy;
          quad_term(dx, dy, dSq, eSq, A.z, M.x, M.y, M.z, qx, qy);
          if (band) {
            tx = ax + fac * (dx + qx);
            ty = ay + fac * (dy + qy);
          }
        }
      }
      if (kCorr == 1) {
        const bool band = use && A.w >= dSq * bandSq;
        if (__ballot_sync(0xffffffffu, band)) {
          const float4 M = S.tM[k];
          const float2 Q = S.tC[k];
          float f[9], ux = 0.0f, uy = 0.0f;
          bool ok = band && mlp_features(dx, dy, dSq, A.z, M.w, Q.x, Q.y, A.x,
                                         A.y, M.x, M.y, M.z, 1.0f, eps, f, ux, uy);
          if (!ok)
            for (int q = 0; q < 9; ++q) f[q] = 0.0f;
          float o0, o1;
          mlp_warp(sW, f, sStageW, o0, o1);
          if (ok) {
            // |mono| * ((1 + t0) u + t1 w), w = (-uy, ux)
            const float r = dSq * rsqrtf(dSq);
            tx = ax + fac * (dx * (1.0f + o0) - r * o1 * uy);
            ty = ay + fac * (dy * (1.0f + o0) + r * o1 * ux);
          }
        }
      }
      ax = use ? tx : ax;
      ay = use ? ty : ay;
      if (kCount) nFar += use ? 1u : 0u;
    }
    if (kCount) nVisit += at ? 1u : 0u;
    // accepted: skip the subtree; opened: the node's open slot (skip a
    // leaf, descend into an interior node)
    cur = at ? (accept ? nxt : (uint32_t)B.y) : cur;
    const uint32_t leafLanes = __ballot_sync(0xffffffffu, openLeaf);
    if (leafLanes) {
      const uint32_t b0 = (uint32_t)B.z, b1 = (uint32_t)B.w;
      const uint32_t bEnd = b1 <= S.n ? b1 : S.n; // defensive bound
      for (uint32_t base = b0; base < bEnd; base += 32) {
        const uint32_t cnt = min(32u, bEnd - base);
        if (kCount) ++nChunk;
        __syncwarp();
        if ((uint32_t)lane < cnt) sBodyW[lane] = S.xym[base + lane];
        __syncwarp();
#pragma unroll 4
        for (uint32_t j = 0; j < cnt; ++j) {
          const float4 q = sBodyW[j];
          const float ex = kExact ? __fsub_rn(q.x, x) : q.x - x;
          const float ey = kExact ? __fsub_rn(q.y, y) : q.y - y;
          float tx = ax, ty = ay;
          add_term<kExact, kClamp>(ex, ey, sq_dist<kExact>(ex, ey), q.z, eSq, tx, ty);
          ax = openLeaf ? tx : ax;
          ay = openLeaf ? ty : ay;
        }
      }
      if (kCount && openLeaf) nNear += bEnd > b0 ? bEnd - b0 : 0u;
    }
  }
}

// Paired FP32 arithmetic (sm_100 f32x2: one instruction for two lanes of
// float math in a 64-bit register pair).
typedef unsigned long long f2x;
__device__ __forceinline__ f2x pk2(float a, float b) {
  f2x r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(f2x r, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f2x add2(f2x a, f2x b) {
  f2x r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2x sub2(f2x a, f2x b) {
  f2x r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
  f2x r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
  f2x r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// The default plain walk (contracted arithmetic, clamp-free law, no
// correction, no counting) with paired FP32 instructions: the cell term's
// {dx, dy} and its accumulation are one pair each, and a leaf's bodies are
// taken two at a time (structure-of-arrays staging, so one 64-bit shared
// load gives two bodies' x, y or mass).  Each body accepts, opens and skips
// exactly the nodes walk_targets does, and every term is the same float
// arithmetic; only the leaf terms' summation order changes (two running
// sums, added to the cell terms at the end).
__device__ __forceinline__ void walk_plain_x2(const DevState &S, float tSq, float eSq,
                                              float x, float y, uint32_t cur,
                                              float *sX, float *sY, float *sM,
                                              float &axOut, float &ayOut) {
  const int lane = threadIdx.x & 31;
  const f2x P = pk2(x, y), XX = pk2(x, x), YY = pk2(y, y), E2 = pk2(eSq, eSq);
  const f2x NHALF = pk2(-0.5f, -0.5f), THREEHALF = pk2(1.5f, 1.5f);
  f2x acc = pk2(0.0f, 0.0f);  // cell terms {ax, ay}
  f2x lx = pk2(0.0f, 0.0f), ly = pk2(0.0f, 0.0f); // leaf terms, two sums each
  for (;;) {
    const uint32_t k = __reduce_min_sync(0xffffffffu, cur);
    if (k == kDone) break;
    float4 A;
    int4 B;
    ld_node(&S.tN[k], A, B);
    const uint32_t nxt = (uint32_t)B.x;
    const bool at = cur == k;
    const f2x D = sub2(pk2(A.x, A.y), P);
    float dx, dy;
    upk2(D, dx, dy);
    const float dSq = fmaf(dx, dx, dy * dy);
    const bool accept = at && A.w < dSq * tSq;
    const bool openLeaf = at && !accept && B.y == B.x; // leaf: open == next
    // a massless cell adds exactly +-0 in the clamp-free law (masses >= 0,
    // finite terms), so no mass test
    float fac = A.z * fast_inv_sqrt(dSq) * rcp_approx(dSq + eSq);
    fac = accept ? fac : 0.0f;
    acc = fma2(D, pk2(fac, fac), acc);
    cur = at ? (accept ? nxt : (uint32_t)B.y) : cur;
    if (__ballot_sync(0xffffffffu, openLeaf)) {
      const uint32_t b0 = (uint32_t)B.z, b1 = (uint32_t)B.w;
      const uint32_t bEnd = b1 <= S.n ? b1 : S.n; // defensive bound
      for (uint32_t base = b0; base < bEnd; base += 32) {
        const uint32_t cnt = min(32u, bEnd - base);
        __syncwarp();
        if ((uint32_t)lane < cnt) {
          const float4 q = S.xym[base + lane];
          sX[lane] = q.x;
          sY[lane] = q.y;
          sM[lane] = q.z;
        } else if ((uint32_t)lane == cnt) { // odd count: a massless partner
          sX[lane] = 0.0f;
          sY[lane] = 0.0f;
          sM[lane] = 0.0f;
        }
        __syncwarp();
        if (openLeaf) {
          const uint32_t pairs = (cnt + 1) >> 1;
          for (uint32_t p = 0; p < pairs; ++p) {
            const f2x X2 = reinterpret_cast<const f2x *>(sX)[p];
            const f2x Y2 = reinterpret_cast<const f2x *>(sY)[p];
            const f2x M2 = reinterpret_cast<const f2x *>(sM)[p];
            const f2x EX = sub2(X2, XX), EY = sub2(Y2, YY);
            const f2x D2 = fma2(EX, EX, mul2(EY, EY));
            float d0, d1;
            upk2(D2, d0, d1);
            // fastInvSqrt of both: magic guess, one Newton step
            const f2x G = pk2(u2f(0x5f3759dfu - (f2u(d0) >> 1)),
                              u2f(0x5f3759dfu - (f2u(d1) >> 1)));
            const f2x T = mul2(mul2(D2, NHALF), G);
            const f2x IS = mul2(G, fma2(T, G, THREEHALF));
            float q0, q1;
            upk2(add2(D2, E2), q0, q1);
            const f2x F = mul2(mul2(M2, IS), pk2(rcp_approx(q0), rcp_approx(q1)));
            lx = fma2(EX, F, lx);
            ly = fma2(EY, F, ly);
          }
        }
      }
    }
  }
  float ax, ay, lx0, lx1, ly0, ly1;
  upk2(acc, ax, ay);
  upk2(lx, lx0, lx1);
  upk2(ly, ly0, ly1);
  axOut = ax + (lx0 + lx1);
  ayOut = ay + (ly0 + ly1);
}

// Every target of the launch, one warp per 32.  kPairs selects the paired
// leaf loop for the default plain walk.
template <bool kExact, bool kCount, int kCorr, bool kClamp, bool kPairs>
__device__ __forceinline__ void forces_walk(
    const DevState &S, float tSq, float eSq, unsigned long long *counts,
    float bandSq, float eps, const float2 *__restrict__ query, uint32_t nQuery,
    float2 *__restrict__ queryAcc, float4 (*sBody)[32], const MlpDev &sW,
    __nv_bfloat16 (*sStage)[32][16]) {
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const uint32_t warpsTotal = (gridDim.x * blockDim.x) >> 5;
  // query points (instance 0's tree) instead of the bodies, if given; for
  // the bodies, the launch's range of targets
  const uint32_t tBegin = query ? 0u : S.forceBegin;
  const uint32_t nTargets = query ? nQuery : (S.forceEnd ? min(S.forceEnd, S.n) : S.n);
  for (uint32_t wb = tBegin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
       wb < nTargets; wb += warpsTotal * 32) {
    const uint32_t i = wb + lane;
    const bool valid = i < nTargets;
    float x = 0.0f, y = 0.0f;
    uint32_t cur = kDone;
    bool wide = false;
    if (valid) {
      if (query) {
        const float2 q = query[i];
        x = q.x;
        y = q.y;
      } else {
        const float4 b = S.xym[i];
        x = b.x;
        y = b.y;
      }
      const SegDev &G = S.seg[query ? 0u : S.segOf[i]];
      if (G.travCount > 0) cur = G.travBase;
      wide = G.wide != 0u;
    }
    float ax = 0.0f, ay = 0.0f;
    uint32_t nFar = 0, nNear = 0, nVisit = 0, nIter = 0, nChunk = 0;
    // the clamp-free law only while no lane's instance reaches beyond the
    // coordinate limit (the build's per-instance flag)
    constexpr bool kPlainX2 = kPairs && !kExact && !kCount && kCorr == 0 && !kClamp;
    const bool anyWide = !kClamp && __any_sync(0xffffffffu, wide);
    if (anyWide)
      walk_targets<kExact, kCount, kCorr, true>(S, tSq, eSq, bandSq, eps, x, y, cur,
                                                sBody[w], sW, sStage[kCorr == 1 ? w : 0],
                                                ax, ay, nFar, nNear, nVisit, nIter, nChunk);
    else if (kPlainX2) {
      float *sX = reinterpret_cast<float *>(sBody[w]);
      walk_plain_x2(S, tSq, eSq, x, y, cur, sX, sX + 32, sX + 64, ax, ay);
    } else
      walk_targets<kExact, kCount, kCorr, kClamp>(S, tSq, eSq, bandSq, eps, x, y, cur,
                                                  sBody[w], sW, sStage[kCorr == 1 ? w : 0],
                                                  ax, ay, nFar, nNear, nVisit, nIter, nChunk);
    if (kCount) {
      unsigned long long f = nFar, nn = nNear, v = nVisit;
      for (int o = 16; o > 0; o >>= 1) {
        f += __shfl_xor_sync(0xffffffffu, f, o);
        nn += __shfl_xor_sync(0xffffffffu, nn, o);
        v += __shfl_xor_sync(0xffffffffu, v, o);
      }
      if (lane == 0) {
        atomicAdd(&counts[0], f);
        atomicAdd(&counts[1], nn);
        atomicAdd(&counts[2], v);
        atomicAdd(&counts[3], (unsigned long long)nIter);
        atomicAdd(&counts[4], (unsigned long long)nChunk);
      }
    } else if (valid) {
      if (query) {
        queryAcc[i] = make_float2(ax, ay);
      } else {
        add_attractor<kExact>(S.attr, x, y, ax, ay);
        S.acc[i] = make_float2(ax, ay);
        if (S.recOut) {
          // the body's whole record (nbx_body: pos, vel, acc, mass,
          // radius, id), for a copy to the host right after this launch
          const float4 p = S.pv[i];
          const float2 m = S.mr[i];
          uint32_t *r = S.recOut + (size_t)i * 9;
          r[0] = __float_as_uint(p.x);
          r[1] = __float_as_uint(p.y);
          r[2] = __float_as_uint(p.z);
          r[3] = __float_as_uint(p.w);
          r[4] = __float_as_uint(ax);
          r[5] = __float_as_uint(ay);
          r[6] = __float_as_uint(m.x);
          r[7] = __float_as_uint(m.y);
          r[8] = S.id[i];
        }
      }
    }
  }
}

// The force pass.  kClamp = false is the clamp-free law (see law_factor),
// which the host picks only for non-negative masses below its bound; a
// warp holding a target whose instance reaches beyond the coordinate limit
// stored at upload (the build's SegDev::wide), where distances could
// overflow, takes the clamped walk instead.  Launch bounds: a full SM of
// kBlock-thread blocks (2048 threads: at most 32 registers) for every walk
// but the learned correction's, whose MMA fragments keep it at 3 blocks of
// 256, and the default plain walk's: 1536 threads per SM (40 registers),
// 1% faster than 2048 at 32 registers and identical in results.  kBlock
// and kPairs vary only for the default plain walk (the autotuner's block
// shape and leaf width).
template <bool kExact, bool kCount = false, int kCorr = 0, bool kClamp = true,
          int kBlock = kForceBlock, bool kPairs = true>
__global__ void __launch_bounds__(kBlock, kCorr == 1 ? 3
                                          : (kPairs && !kExact && !kCount && kCorr == 0 &&
                                                     !kClamp
                                                 ? 1536 / kBlock
                                                 : 2048 / kBlock))
    k_forces(DevState S, float tSq, float eSq,
             unsigned long long *counts = nullptr,
             const MlpDev *__restrict__ mlp = nullptr, float bandSq = 0.0f,
             float eps = 0.0f, const float2 *__restrict__ query = nullptr,
             uint32_t nQuery = 0, float2 *__restrict__ queryAcc = nullptr) {
  constexpr int kBlockWarps = kBlock / 32;
  constexpr int kStage = kCorr == 1 ? kBlockWarps : 1;
  __shared__ float4 sBody[kBlockWarps][32];
  __shared__ MlpDev sW;
  __shared__ __nv_bfloat16 sStage[kStage][32][16];
  if (kCorr == 1) {
    for (int q = threadIdx.x; q < (int)(sizeof(MlpDev) / 4); q += blockDim.x)
      reinterpret_cast<uint32_t *>(&sW)[q] = reinterpret_cast<const uint32_t *>(mlp)[q];
    __syncthreads();
  }
  forces_walk<kExact, kCount, kCorr, kClamp, kPairs>(S, tSq, eSq, counts, bandSq, eps, query,
                                                     nQuery, queryAcc, sBody, sW, sStage);
}

// FMA throughput probe: 8 independent chains per thread.
__global__ void k_fma_probe(float *out, int iters) {
  float a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = threadIdx.x * 1e-7f + j;
  const float b = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = fmaf(a[j], b, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += a[j];
  if (s == 12345.0f) out[0] = s; // keeps the chains live
}

} // namespace

void launch_interaction_count(cudaStream_t s, const DevState &S,
                              unsigned long long *counts) {
  uint32_t warps = (S.n + 31) / 32;
  uint32_t b = (warps + kWarps - 1) / kWarps;
  cudaMemsetAsync(counts, 0, 5 * sizeof(unsigned long long), s);
  k_forces<false, true><<<b ? b : 1, kForceBlock, 0, s>>>(S, S.tSq, S.eSq, counts);
}

// FP32 FMA peak of the device in TFLOP/s (2 flops per FMA), timed with
// CUDA events around one large probe launch.
double fp32_fma_peak_tflops(cudaStream_t s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  if (cudaMalloc(&out, 4) != cudaSuccess) return 0.0;
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  k_fma_probe<<<blocks, threads, 0, s>>>(out, 64); // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  k_fma_probe<<<blocks, threads, 0, s>>>(out, iters);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  return ms > 0 ? flops / (ms * 1e-3) / 1e12 : 0.0;
}

// Accelerations at arbitrary points from instance 0's last tree
// (QuadTree::acceleration, QuadTree.cpp:264-389, for any query position).
void launch_query_forces(cudaStream_t s, const DevState &S, bool exact,
                         const float2 *query, uint32_t nq, float2 *out) {
  const uint32_t b = ((nq + 31) / 32 + kWarps - 1) / kWarps;
  if (exact)
    k_forces<true><<<b ? b : 1, kForceBlock, 0, s>>>(S, S.tSq, S.eSq, nullptr,
                                                     nullptr, 0.0f, 0.0f, query,
                                                     nq, out);
  else
    k_forces<false><<<b ? b : 1, kForceBlock, 0, s>>>(S, S.tSq, S.eSq, nullptr,
                                                      nullptr, 0.0f, 0.0f, query,
                                                      nq, out);
}

// Bodies a force launch over S covers (its target range, or all).
uint32_t force_targets(const DevState &S) {
  const uint32_t e = S.forceEnd ? (S.forceEnd < S.n ? S.forceEnd : S.n) : S.n;
  return e > S.forceBegin ? e - S.forceBegin : 0u;
}

// The default plain walk with kBlock threads per block and the paired or
// single-body leaf loop.
template <int kBlock>
void launch_plain(cudaStream_t s, const DevState &S, int blocks, bool pairs) {
  if (blocks <= 0) {
    const uint32_t warps = (force_targets(S) + 31) / 32, per = kBlock / 32;
    const uint32_t b = (warps + per - 1) / per;
    blocks = (int)(b ? b : 1);
  }
  if (pairs)
    k_forces<false, false, 0, false, kBlock, true><<<blocks, kBlock, 0, s>>>(S, S.tSq, S.eSq);
  else
    k_forces<false, false, 0, false, kBlock, false><<<blocks, kBlock, 0, s>>>(S, S.tSq, S.eSq);
}

void launch_forces(cudaStream_t s, const DevState &S, bool exact, int blocks,
                   const MlpDev *mlp, float band, int corr, bool noClamp, int threads,
                   bool pairs) {
  if (corr == 0 && !exact && noClamp) {
    if (threads == 128) launch_plain<128>(s, S, blocks, pairs);
    else if (threads == 512) launch_plain<512>(s, S, blocks, pairs);
    else launch_plain<256>(s, S, blocks, pairs);
    return;
  }
  if (blocks <= 0) {
    uint32_t warps = (force_targets(S) + 31) / 32;
    uint32_t b = (warps + kWarps - 1) / kWarps;
    blocks = (int)(b ? b : 1);
  }
  if (corr == 1 && mlp)
    k_forces<false, false, 1><<<blocks, kForceBlock, 0, s>>>(
        S, S.tSq, S.eSq, nullptr, mlp, band * band, sqrtf(S.eSq));
  else if (corr == 2 && noClamp)
    k_forces<false, false, 2, false><<<blocks, kForceBlock, 0, s>>>(
        S, S.tSq, S.eSq, nullptr, nullptr, band * band, sqrtf(S.eSq));
  else if (corr == 2)
    k_forces<false, false, 2><<<blocks, kForceBlock, 0, s>>>(
        S, S.tSq, S.eSq, nullptr, nullptr, band * band, sqrtf(S.eSq));
  else if (exact)
    k_forces<true><<<blocks, kForceBlock, 0, s>>>(S, S.tSq, S.eSq);
  else
    k_forces<false><<<blocks, kForceBlock, 0, s>>>(S, S.tSq, S.eSq);
}

} // namespace nbx
