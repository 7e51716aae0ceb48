// diag.cu -- FP64 checks on the GPU: direct-sum accelerations with the
// tree's force law for sampled targets (exactTreeLawForces,
// src/cuda/CheckCuda.cu:453-475) and compensated energy / momentum sums.
// These are the only FP64 arithmetic in the library.
#include "nbx_state.cuh"

namespace nbx {
namespace {

constexpr int kDirectThreads = 128;
constexpr int kDirectChunks = 64;

// What a direct sum adds per source: the force of the tree law
// m d / (|d| (d^2 + eps^2)) or of the Plummer law m d / (d^2 + eps^2)^1.5,
// or the potential of either (per unit target mass): the tree law's is
// -(m / eps) atan(eps / |d|) (its gradient is the tree force; -m / |d| for
// eps = 0), the Plummer law's -m / sqrt(d^2 + eps^2).
// kFastLawForce is the tree force law with the reference's fastInvSqrt
// (QuadTree.cpp:11-26) applied to the float distance squared, accumulated in
// FP64: the error of the reference's law itself, without any summation or
// tree error.
enum DirectKind { kTreeForce = 0, kPlummerForce = 1, kTreePotential = 2,
                  kPlummerPotential = 3, kFastLawForce = 4 };

// Partial FP64 sums: block (tb, chunk) adds sources of `chunk` for the
// targets tb*128 .. tb*128+127.  Sources staged through shared memory.
// Potentials go to .x (.y stays 0).
__global__ void __launch_bounds__(kDirectThreads)
    k_direct_partial(const float4 *__restrict__ pv, const float2 *__restrict__ mr,
                     uint32_t n, const uint32_t *__restrict__ targets,
                     const uint2 *__restrict__ ranges, uint32_t m, double eSq,
                     int kind, double2 *__restrict__ partial) {
  const double eps = sqrt(eSq);
  __shared__ float4 sSrc[kDirectThreads];
  const uint32_t t = blockIdx.x * kDirectThreads + threadIdx.x;
  const bool valid = t < m;
  const uint32_t ti = valid ? targets[t] : 0u;
  // sources: the target's own instance
  const uint2 rg = valid ? ranges[t] : make_uint2(0u, 0u);
  double x = 0.0, y = 0.0;
  if (valid) {
    const float4 p = pv[ti];
    x = p.x;
    y = p.y;
  }
  const uint32_t chunk = (n + gridDim.y - 1) / gridDim.y;
  const uint32_t j0 = blockIdx.y * chunk;
  const uint32_t j1 = min(n, j0 + chunk);
  double ax = 0.0, ay = 0.0;
  for (uint32_t base = j0; base < j1; base += kDirectThreads) {
    const uint32_t j = base + threadIdx.x;
    __syncthreads();
    if (j < j1) {
      const float4 p = pv[j];
      sSrc[threadIdx.x] = make_float4(p.x, p.y, mr[j].x, __uint_as_float(j));
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kDirectThreads, j1 - base);
    if (valid) {
      for (uint32_t k = 0; k < cnt; ++k) {
        const float4 s = sSrc[k];
        const uint32_t sj = __float_as_uint(s.w);
        if (sj == ti || sj < rg.x || sj >= rg.y) continue;
        const double dx = (double)s.x - x;
        const double dy = (double)s.y - y;
        const double dSq = dx * dx + dy * dy;
        if (dSq == 0.0) continue;
        const double q = dSq + eSq;
        if (kind == kFastLawForce) {
          const double f = (double)s.z * (double)fast_inv_sqrt((float)dSq) / (dSq + eSq);
          ax += dx * f;
          ay += dy * f;
        } else if (kind == kTreeForce || kind == kPlummerForce) {
          const double f = kind == kPlummerForce ? (double)s.z / (q * sqrt(q))
                                                 : (double)s.z / (sqrt(dSq) * q);
          ax += dx * f;
          ay += dy * f;
        } else if (kind == kPlummerPotential) {
          ax -= (double)s.z / sqrt(q);
        } else {
          const double r = sqrt(dSq);
          ax -= eps > 0.0 ? (double)s.z / eps * atan2(eps, r) : (double)s.z / r;
        }
      }
    }
  }
  if (valid) partial[(size_t)blockIdx.y * m + t] = make_double2(ax, ay);
}

__global__ void k_direct_reduce(const double2 *__restrict__ partial, uint32_t m,
                                int chunks, double *ax, double *ay) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  double sx = 0.0, sy = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const double2 v = partial[(size_t)c * m + t];
    sx += v.x;
    sy += v.y;
  }
  ax[t] = sx;
  ay[t] = sy;
}

// Neumaier accumulation in FP64.
struct KSum {
  double s = 0.0, c = 0.0;
  __device__ void add(double v) {
    const double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
  }
};

constexpr int kEmBlock = 256;

// Per-block compensated partial sums of {KE, px, py, Lz, M}.
__global__ void __launch_bounds__(kEmBlock)
    k_energy_partial(const float4 *__restrict__ pv, const float2 *__restrict__ mr,
                     uint32_t n, double *__restrict__ out) {
  KSum acc[5];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const float4 p = pv[i];
    const double m = mr[i].x, x = p.x, y = p.y, vx = p.z, vy = p.w;
    acc[0].add(0.5 * m * (vx * vx + vy * vy));
    acc[1].add(m * vx);
    acc[2].add(m * vy);
    acc[3].add(m * (x * vy - y * vx));
    acc[4].add(m);
  }
  __shared__ double sS[5][kEmBlock], sC[5][kEmBlock];
  for (int k = 0; k < 5; ++k) {
    sS[k][threadIdx.x] = acc[k].s;
    sC[k][threadIdx.x] = acc[k].c;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    const int k = threadIdx.x;
    KSum t;
    for (int j = 0; j < kEmBlock; ++j) {
      t.add(sS[k][j]);
      t.add(sC[k][j]);
    }
    out[(size_t)blockIdx.x * 10 + 2 * k] = t.s;
    out[(size_t)blockIdx.x * 10 + 2 * k + 1] = t.c;
  }
}

__global__ void k_energy_final(const double *__restrict__ part, int blocks,
                               double *out) {
  const int k = threadIdx.x;
  if (k >= 5) return;
  KSum t;
  for (int b = 0; b < blocks; ++b) {
    t.add(part[(size_t)b * 10 + 2 * k]);
    t.add(part[(size_t)b * 10 + 2 * k + 1]);
  }
  out[k] = t.s + t.c;
}

} // namespace

// partial must hold kDirectChunks * m double2.
// kind: 0 tree-law force, 1 Plummer force, 2 tree-law potential (to ax),
// 3 Plummer potential (to ax), 4 tree-law force with fastInvSqrt.
void launch_direct_fp64(cudaStream_t s, const float4 *pv, const float2 *mr,
                        uint32_t n, const uint32_t *targets, const uint2 *ranges,
                        uint32_t m, double eps, int kind, double2 *partial,
                        double *ax, double *ay) {
  if (m == 0) return;
  dim3 grid((m + kDirectThreads - 1) / kDirectThreads, kDirectChunks);
  k_direct_partial<<<grid, kDirectThreads, 0, s>>>(pv, mr, n, targets, ranges, m,
                                                   eps * eps, kind, partial);
  k_direct_reduce<<<(m + 255) / 256, 256, 0, s>>>(partial, m, kDirectChunks, ax,
                                                  ay);
}

size_t direct_partial_elems(uint32_t m) { return (size_t)kDirectChunks * m; }

// part must hold 10 * 592 doubles; out 5 doubles.
void launch_energy_momentum(cudaStream_t s, const float4 *pv, const float2 *mr,
                            uint32_t n, double *part, double *out) {
  const int blocks = 592;
  k_energy_partial<<<blocks, kEmBlock, 0, s>>>(pv, mr, n, part);
  k_energy_final<<<1, 32, 0, s>>>(part, blocks, out);
}

} // namespace nbx
