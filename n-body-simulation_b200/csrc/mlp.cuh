// mlp.cuh -- learned far-field correction: feature map, parameter layout and
// the warp-level BF16 tensor-core inference used inside the traversal.
//
// For an accepted cell (centre of mass C, mass M, square centre Q, side s,
// second moments I about C) seen from a target P, with d = C - P, r = |d|,
// u = d/r and w = (-u.y, u.x), the network reads 9 features
//   f0, f1 = ((Q - C).u, (Q - C).w) / s       cell-centre offset / size
//   f2     = log2(M) / 16                      log cell mass
//   f3..f5 = (u'Iu, w'Iw, u'Iw) / (M s^2)      second moments / size^2
//   f6     = s / r                             size / distance
//   f7     = (s / r)^2 / theta^2               opening ratio of the MAC
//   f8     = eps / r                           softening / distance
// and predicts (t0, t1): the cell's exact FP64 force minus its monopole, in
// the (u, w) frame, divided by the monopole's magnitude.  The corrected
// cell force is |a_mono| * ((1 + t0) u + t1 w).
//
// Network: 9 -> 32 SiLU -> 32 SiLU -> 2, BF16 weights, FP32 accumulate.
// Parameters (FP32 master copy, `kMlpParams` floats):
//   W1[32][9], b1[32], W2[32][32], b2[32], W3[2][32], b3[2].
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace nbx {

constexpr int kMlpIn = 9, kMlpHid = 32, kMlpOut = 2;
constexpr int kOffW1 = 0, kOffB1 = 288, kOffW2 = 320, kOffB2 = 1344,
              kOffW3 = 1376, kOffB3 = 1440, kMlpParams = 1442;
constexpr int kMlpRow = 12; // floats per training row: 9 features, 2 targets, weight

// Inference copy: BF16 weights laid out for mma.sync B fragments
// (row n of W holds the K inputs of output n, K padded to 16 / 32).
struct MlpDev {
  __nv_bfloat16 w1[32][16];
  __nv_bfloat16 w2[32][32];
  __nv_bfloat16 w3[8][32];
  float b1[32], b2[32], b3[8];
  float theta;     // MAC theta the features are normalised with
  float band;      // correct accepted cells with s/r >= band
  int32_t enabled; // weights loaded
  int32_t pad;
};

// Feature map; returns false if the cell is degenerate (no correction).
__host__ __device__ inline bool mlp_features(float dx, float dy, float dSq,
                                             float mass, float size, float qx,
                                             float qy, float cx, float cy,
                                             float ixx, float iyy, float ixy,
                                             float theta, float eps, float f[9],
                                             float &ux, float &uy) {
  if (!(dSq > 0.0f) || !(mass > 0.0f) || !(size > 0.0f)) return false;
  const float ir = 1.0f / sqrtf(dSq);
  ux = dx * ir;
  uy = dy * ir;
  const float wx = -uy, wy = ux;
  const float is = 1.0f / size;
  const float ox = (qx - cx) * is, oy = (qy - cy) * is;
  f[0] = ox * ux + oy * uy;
  f[1] = ox * wx + oy * wy;
  f[2] = log2f(mass) * (1.0f / 16.0f);
  const float inv = is * is / mass;
  f[3] = (ux * ux * ixx + 2.0f * ux * uy * ixy + uy * uy * iyy) * inv;
  f[4] = (wx * wx * ixx + 2.0f * wx * wy * ixy + wy * wy * iyy) * inv;
  f[5] = (ux * wx * ixx + (ux * wy + uy * wx) * ixy + uy * wy * iyy) * inv;
  f[6] = size * ir;
  f[7] = f[6] * f[6] / (theta * theta);
  f[8] = eps * ir;
  return true;
}

#if defined(__CUDACC__)

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4],
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SiLU of a bf16 pair: x * (0.5 + 0.5 tanh(x/2)).
__device__ __forceinline__ uint32_t silu_bf16x2(uint32_t x) {
  const __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162 *>(&x);
  const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f);
  __nv_bfloat162 t = __hmul2(h, half);
  uint32_t tu = *reinterpret_cast<uint32_t *>(&t), th;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(th) : "r"(tu));
  const __nv_bfloat162 tt = *reinterpret_cast<__nv_bfloat162 *>(&th);
  const __nv_bfloat162 s = __hfma2(tt, half, half);
  __nv_bfloat162 y = __hmul2(h, s);
  return *reinterpret_cast<uint32_t *>(&y);
}

// Warp-wide MLP on 32 rows, one per lane (row = lane).  `feat` holds the
// lane's 9 features (zeros for lanes without a row); `stage` is 32x16 bf16
// of per-warp shared memory.  Returns the lane's 2 outputs.  All 32 lanes
// must call it together.
__device__ __forceinline__ void mlp_warp(const MlpDev &W, const float feat[9],
                                         __nv_bfloat16 (*stage)[16], float &o0,
                                         float &o1) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // stage the input rows so each lane can read its A fragments
  uint32_t *row = reinterpret_cast<uint32_t *>(stage[lane]);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float lo = 2 * k < 9 ? feat[2 * k] : 0.0f;
    const float hi = 2 * k + 1 < 9 ? feat[2 * k + 1] : 0.0f;
    row[k] = pack_bf16(lo, hi);
  }
  __syncwarp();
  uint32_t a[2][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const uint32_t *r0 = reinterpret_cast<const uint32_t *>(stage[mt * 16 + g]);
    const uint32_t *r1 = reinterpret_cast<const uint32_t *>(stage[mt * 16 + g + 8]);
    a[mt][0] = r0[t];
    a[mt][1] = r1[t];
    a[mt][2] = r0[t + 4];
    a[mt][3] = r1[t + 4];
  }
  __syncwarp();
  // layer 1: [32 x 16] x [16 x 32]
  float acc[2][4][4];
  uint32_t h[2][4][2]; // bf16x2 activations: [mtile][ntile][row half]
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
    const uint32_t *wr = reinterpret_cast<const uint32_t *>(W.w1[nt * 8 + g]);
    const uint32_t b0 = wr[t], b1 = wr[t + 4];
    const float bias0 = W.b1[nt * 8 + 2 * t], bias1 = W.b1[nt * 8 + 2 * t + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      acc[mt][nt][0] = bias0;
      acc[mt][nt][1] = bias1;
      acc[mt][nt][2] = bias0;
      acc[mt][nt][3] = bias1;
      mma_bf16(acc[mt][nt], a[mt], b0, b1);
      h[mt][nt][0] = silu_bf16x2(pack_bf16(acc[mt][nt][0], acc[mt][nt][1]));
      h[mt][nt][1] = silu_bf16x2(pack_bf16(acc[mt][nt][2], acc[mt][nt][3]));
    }
  }
  // layer 2: [32 x 32] x [32 x 32]
  uint32_t h2[2][4][2];
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
    const uint32_t *wr = reinterpret_cast<const uint32_t *>(W.w2[nt * 8 + g]);
    const float bias0 = W.b2[nt * 8 + 2 * t], bias1 = W.b2[nt * 8 + 2 * t + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      float d[4] = {bias0, bias1, bias0, bias1};
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const uint32_t af[4] = {h[mt][2 * ks][0], h[mt][2 * ks][1],
                                h[mt][2 * ks + 1][0], h[mt][2 * ks + 1][1]};
        mma_bf16(d, af, wr[ks * 8 + t], wr[ks * 8 + t + 4]);
      }
      h2[mt][nt][0] = silu_bf16x2(pack_bf16(d[0], d[1]));
      h2[mt][nt][1] = silu_bf16x2(pack_bf16(d[2], d[3]));
    }
  }
  // layer 3: [32 x 32] x [32 x 8]
  float out[2][4];
  {
    const uint32_t *wr = reinterpret_cast<const uint32_t *>(W.w3[g]);
    const float bias0 = W.b3[2 * t], bias1 = W.b3[2 * t + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      out[mt][0] = bias0;
      out[mt][1] = bias1;
      out[mt][2] = bias0;
      out[mt][3] = bias1;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const uint32_t af[4] = {h2[mt][2 * ks][0], h2[mt][2 * ks][1],
                                h2[mt][2 * ks + 1][0], h2[mt][2 * ks + 1][1]};
        mma_bf16(out[mt], af, wr[ks * 8 + t], wr[ks * 8 + t + 4]);
      }
    }
  }
  // row r's outputs sit in lane 4*(r%8) of m-tile r/16, half (r%16)/8
  const int mt = lane >> 4, lr = lane & 15, src = 4 * (lr & 7);
  const bool hi = lr >= 8;
  const float x0 = __shfl_sync(0xffffffffu, out[0][0], src);
  const float x1 = __shfl_sync(0xffffffffu, out[0][1], src);
  const float x2 = __shfl_sync(0xffffffffu, out[0][2], src);
  const float x3 = __shfl_sync(0xffffffffu, out[0][3], src);
  const float y0 = __shfl_sync(0xffffffffu, out[1][0], src);
  const float y1 = __shfl_sync(0xffffffffu, out[1][1], src);
  const float y2 = __shfl_sync(0xffffffffu, out[1][2], src);
  const float y3 = __shfl_sync(0xffffffffu, out[1][3], src);
  o0 = mt == 0 ? (hi ? x2 : x0) : (hi ? y2 : y0);
  o1 = mt == 0 ? (hi ? x3 : x1) : (hi ? y3 : y1);
}

#endif

} // namespace nbx
