// naive.cu -- direct all-pairs gravity: the force pass of NaiveSimulation
// (src/naive/NaiveSimulation.cpp:17-57) and CudaNaiveSimulation
// (src/cuda/CudaNaive.cu:17-57), selected by nbx_params.force_law = 1.
//
// Per pair, in the reference's order of operations:
//   d = pos_j - pos_i, s = |d|^2 + eps^2,
//   acc_i += d * (m_j * (1 / sqrt(s)) * (1 / s)),
// summed over every other body j of the same instance in array order.
//
// The step is iterate -> collide -> attract as for the tree, with an
// identity gather in place of the Morton gather so the state alternates
// between the two buffers exactly as a tree step does.
//
// Layout: blocks of 256 threads, two targets per thread (512 per block);
// the block's sources stream through shared memory in tiles of 256 bodies,
// one float4 {x, y, m, 0} per body, so each load from shared memory is a
// broadcast that serves two interactions.  A block whose targets all
// belong to one instance (every block of a single simulation) runs the
// unchecked loop; blocks that straddle instances, exact arithmetic and
// eps = 0 run a loop that checks each source's instance and skips j == i
// (the reference skips it explicitly; with eps > 0 it adds exactly zero).
//
// Bound: FP32 issue (9 FMA-pipe instructions and one MUFU rsqrt per
// interaction in the default arithmetic), 20 FLOP per interaction by the
// same convention as the tree force pass.
#include "nbx_state.cuh"

#include <float.h>

namespace nbx {
namespace {

constexpr int kNaiveThreads = 256;
constexpr int kNaiveTargets = 2; // per thread
constexpr int kNaiveBlockTargets = kNaiveThreads * kNaiveTargets;

// Exact: the reference's IEEE operations, no contraction.
__device__ __forceinline__ void naive_term_exact(float4 q, float x, float y,
                                                 float eSq, float &ax, float &ay) {
  const float dx = __fsub_rn(q.x, x), dy = __fsub_rn(q.y, y);
  const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), eSq);
  const float invSoft = __frcp_rn(s);
  const float invDist = __frcp_rn(__fsqrt_rn(s));
  const float f = __fmul_rn(__fmul_rn(q.z, invDist), invSoft);
  ax = __fadd_rn(ax, __fmul_rn(dx, f));
  ay = __fadd_rn(ay, __fmul_rn(dy, f));
}

// Default: contracted, one hardware rsqrt (s^-3/2 = r^3).
__device__ __forceinline__ void naive_term_fast(float4 q, float x, float y,
                                                float eSq, float &ax, float &ay) {
  const float dx = q.x - x, dy = q.y - y;
  const float s = fmaf(dx, dx, fmaf(dy, dy, eSq));
  const float r = rsqrtf(s);
  const float f = q.z * (r * r * r);
  ax = fmaf(dx, f, ax);
  ay = fmaf(dy, f, ay);
}

template <bool kExact>
__global__ void __launch_bounds__(kNaiveThreads)
    k_naive(DevState S, float eSq, int alwaysCheck) {
  __shared__ float4 tile[kNaiveThreads];
  __shared__ uint32_t sLo, sHi;
  __shared__ int sMixed;
  const uint32_t base0 = blockIdx.x * kNaiveBlockTargets;
  uint32_t idx[kNaiveTargets], j0[kNaiveTargets], j1[kNaiveTargets];
  float x[kNaiveTargets], y[kNaiveTargets], ax[kNaiveTargets], ay[kNaiveTargets];
  if (threadIdx.x == 0) {
    sLo = 0xffffffffu;
    sHi = 0u;
    sMixed = alwaysCheck;
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < kNaiveTargets; ++t) {
    idx[t] = base0 + t * kNaiveThreads + threadIdx.x;
    x[t] = y[t] = ax[t] = ay[t] = 0.0f;
    j0[t] = j1[t] = 0u;
    if (idx[t] < S.n) {
      const float4 b = S.xym[idx[t]];
      x[t] = b.x;
      y[t] = b.y;
      const SegDev &G = S.seg[S.segOf[idx[t]]];
      j0[t] = G.start;
      j1[t] = G.start + G.count;
      atomicMin(&sLo, j0[t]);
      atomicMax(&sHi, j1[t]);
    }
  }
  __syncthreads();
  const uint32_t lo = sLo, hi = sHi;
#pragma unroll
  for (int t = 0; t < kNaiveTargets; ++t)
    if (idx[t] < S.n && (j0[t] != lo || j1[t] != hi)) sMixed = 1;
  __syncthreads();
  const bool checked = kExact || sMixed != 0;
  for (uint32_t base = lo; base < hi; base += kNaiveThreads) {
    const uint32_t j = base + threadIdx.x;
    tile[threadIdx.x] = j < hi ? S.xym[j] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kNaiveThreads, hi - base);
    if (!checked && cnt == kNaiveThreads) {
#pragma unroll 8
      for (int k = 0; k < kNaiveThreads; ++k) {
        const float4 q = tile[k];
#pragma unroll
        for (int t = 0; t < kNaiveTargets; ++t) naive_term_fast(q, x[t], y[t], eSq, ax[t], ay[t]);
      }
    } else {
      for (uint32_t k = 0; k < cnt; ++k) {
        const float4 q = tile[k];
        const uint32_t jj = base + k;
#pragma unroll
        for (int t = 0; t < kNaiveTargets; ++t) {
          if (jj < j0[t] || jj >= j1[t] || jj == idx[t]) continue;
          if (kExact) naive_term_exact(q, x[t], y[t], eSq, ax[t], ay[t]);
          else naive_term_fast(q, x[t], y[t], eSq, ax[t], ay[t]);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < kNaiveTargets; ++t) {
    if (idx[t] >= S.n) continue;
    add_attractor<kExact>(S.attr, x[t], y[t], ax[t], ay[t]);
    S.acc[idx[t]] = make_float2(ax[t], ay[t]);
  }
}

// The naive step's stand-in for the Morton gather: the same buffer swap,
// bodies kept in their order.
__global__ void k_identity_gather(DevState S) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n;
       i += gridDim.x * blockDim.x) {
    const float4 v = S.pv[i];
    const float2 m = S.mr[i];
    S.pv2[i] = v;
    S.mr2[i] = m;
    S.id2[i] = S.id[i];
    S.xym[i] = make_float4(v.x, v.y, m.x, 0.0f);
  }
}

} // namespace

// Identity gather + buffer swap; returns the state after the swap.
DevState launch_naive_gather(cudaStream_t s, const DevState &S) {
  uint32_t b = (S.n + 255) / 256;
  if (b > 148u * 16u) b = 148u * 16u;
  k_identity_gather<<<b ? b : 1, 256, 0, s>>>(S);
  DevState T = S;
  T.pv = S.pv2;
  T.mr = S.mr2;
  T.id = S.id2;
  T.pv2 = S.pv;
  T.mr2 = S.mr;
  T.id2 = S.id;
  return T;
}

// All-pairs accelerations of the bodies in S.xym into S.acc.
void launch_naive_forces(cudaStream_t s, const DevState &S, bool exact) {
  if (S.n == 0) return;
  const uint32_t blocks = (S.n + kNaiveBlockTargets - 1) / kNaiveBlockTargets;
  const int check = S.eSq > 0.0f ? 0 : 1; // eps = 0: skip j == i explicitly
  if (exact)
    k_naive<true><<<blocks, kNaiveThreads, 0, s>>>(S, S.eSq, 1);
  else
    k_naive<false><<<blocks, kNaiveThreads, 0, s>>>(S, S.eSq, check);
}

} // namespace nbx
