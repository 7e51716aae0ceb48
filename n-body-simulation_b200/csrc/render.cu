// render.cu -- headless splat renderer: the viewer's point-sprite drawing
// (src/viewer/Renderer.cpp:8-52, 113-147) rasterised by CUDA kernels into
// a float RGBA image in device memory, plus the viewer's body statistics
// (GlBodyBuffer::fill, src/viewer/Interop.cu:14-45, 80-104).  No graphics
// API is involved.
//
// Per body (vertex shader): p = (pos - centre) * scale pixels from the
// image centre (y up), point size = max(2 r scale pointScale, minPoint),
// alpha = clamp(size / minPoint, 0.08, 1), colour = the speed ramp
// (mode 0, "Speed") or (0.35, 0.75, 1) (mode 1, "Glow").  Per covered pixel
// centre c (fragment shader): d = (c - window position) / (point size / 2),
// r2 = |d|^2, discarded when r2 > 1, a = (1 - r2) alpha brightness, source
// (colour a, a) premultiplied.  Blending: Glow adds (ONE, ONE); Speed
// composites over in draw order (ONE, ONE_MINUS_SRC_ALPHA).  The image
// starts at the clear colour (0, 0, 0.02, 1); row 0 is the bottom row.
//
// GPU layout: bodies emit one (tile, body) entry per 16x16-pixel tile their
// point touches, in body order; a stable radix sort on the tile index groups
// them with each tile's entries still in draw order; one 256-thread block
// per tile then composites its pixels over the tile's entries, staged
// through shared memory.  So the over-blend sees the bodies in the order GL
// would draw them, and every pixel's arithmetic is sequential.
//
// This file is compiled with --fmad=false: each expression rounds as
// written, as in the C restatement of the same math.
#include "nbx_state.cuh"

#include <float.h>

namespace nbx {

namespace {

constexpr int kTilePx = 16;
constexpr int kVertexThreads = 256;

__device__ __forceinline__ float mixf(float x, float y, float a) {
  return x * (1.0f - a) + y * a; // GLSL mix
}

// ramp() of the vertex shader (Renderer.cpp:20-25)
__device__ __forceinline__ float3 speed_ramp(float t) {
  t = fminf(fmaxf(t, 0.0f), 1.0f);
  const float3 slow = make_float3(0.15f, 0.3f, 1.0f), mid = make_float3(0.2f, 0.95f, 1.0f),
               fast = make_float3(1.0f, 0.9f, 0.55f);
  if (t < 0.5f) {
    const float u = t * 2.0f;
    return make_float3(mixf(slow.x, mid.x, u), mixf(slow.y, mid.y, u), mixf(slow.z, mid.z, u));
  }
  const float u = t * 2.0f - 1.0f;
  return make_float3(mixf(mid.x, fast.x, u), mixf(mid.y, fast.y, u), mixf(mid.z, fast.z, u));
}

// Pixel range [lo, hi] of a point centred at w with half size hf along an
// axis of `extent` pixels; false when it misses the image.
__device__ __forceinline__ bool pixel_range(float w, float hf, uint32_t extent, int &lo,
                                            int &hi) {
  const float a = w - hf, b = w + hf;
  if (!(a < (float)extent) || !(b >= 0.0f)) return false; // also rejects NaN
  lo = a <= 0.0f ? 0 : (int)floorf(a);
  hi = b >= (float)(extent - 1) ? (int)extent - 1 : (int)floorf(b);
  return lo <= hi;
}

// One vertex per body: window position, half size, alpha, colour and the
// number of tiles touched; statistics partials per block.
__global__ void __launch_bounds__(kVertexThreads)
    k_render_vertices(const float4 *__restrict__ pv, const float2 *__restrict__ mr,
                      uint32_t n, RenderParams P, float4 *__restrict__ v0,
                      float4 *__restrict__ v1, uint32_t *__restrict__ tiles,
                      double4 *__restrict__ partial,
                      unsigned long long *__restrict__ total) {
  __shared__ double sMx[kVertexThreads / 32], sMy[kVertexThreads / 32], sM[kVertexThreads / 32];
  __shared__ float sV[kVertexThreads / 32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double mx = 0.0, my = 0.0, m = 0.0;
  float speed = 0.0f;
  if (i < n) {
    const float4 s = pv[i];
    const float2 q = mr[i];
    speed = sqrtf(s.z * s.z + s.w * s.w);
    m = q.x;
    mx = (double)q.x * s.x;
    my = (double)q.x * s.y;
    const float wx = (s.x - P.camX) * P.scale + P.halfW;
    const float wy = (s.y - P.camY) * P.scale + P.halfH;
    const float size = q.y * 2.0f * P.scale * P.pointScale;
    const float ps = fmaxf(size, P.minPoint);
    const float alpha = fminf(fmaxf(size / P.minPoint, 0.08f), 1.0f);
    const float hf = ps * 0.5f;
    const float3 c = P.mode == 0 ? speed_ramp(speed / P.speedMax)
                                 : make_float3(0.35f, 0.75f, 1.0f);
    v0[i] = make_float4(wx, wy, hf, alpha);
    v1[i] = make_float4(c.x, c.y, c.z, 0.0f);
    int x0, x1, y0, y1;
    uint32_t t = 0;
    if (pixel_range(wx, hf, P.width, x0, x1) && pixel_range(wy, hf, P.height, y0, y1))
      t = (uint32_t)(x1 / kTilePx - x0 / kTilePx + 1) * (uint32_t)(y1 / kTilePx - y0 / kTilePx + 1);
    tiles[i] = t;
  }
  {
    // 64-bit total of (tile, body) entries: the host checks it before
    // the 32-bit scan of the per-body counts
    unsigned long long t64 = i < n ? tiles[i] : 0ull;
    for (int o = 16; o > 0; o >>= 1) t64 += __shfl_down_sync(0xffffffffu, t64, o);
    if ((threadIdx.x & 31) == 0 && t64) atomicAdd(total, t64);
  }
  // deterministic block partials (fixed shuffle tree, then warp order)
  for (int o = 16; o > 0; o >>= 1) {
    mx += __shfl_down_sync(0xffffffffu, mx, o);
    my += __shfl_down_sync(0xffffffffu, my, o);
    m += __shfl_down_sync(0xffffffffu, m, o);
    speed = fmaxf(speed, __shfl_down_sync(0xffffffffu, speed, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sMx[w] = mx;
    sMy[w] = my;
    sM[w] = m;
    sV[w] = speed;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0;
    float v = 0.0f;
    for (int k = 0; k < kVertexThreads / 32; ++k) {
      a += sMx[k];
      b += sMy[k];
      c += sM[k];
      v = fmaxf(v, sV[k]);
    }
    partial[blockIdx.x] = make_double4(a, b, c, (double)v);
  }
}

// BodyStats from the block partials, in block order: {comX, comY, maxSpeed}.
__global__ void k_render_stats(const double4 *__restrict__ partial, uint32_t blocks,
                               float *__restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 0.0, b = 0.0, c = 0.0, v = 0.0;
  for (uint32_t k = 0; k < blocks; ++k) {
    a += partial[k].x;
    b += partial[k].y;
    c += partial[k].z;
    v = fmax(v, partial[k].w);
  }
  out[0] = c > 0.0 ? (float)(a / c) : 0.0f;
  out[1] = c > 0.0 ? (float)(b / c) : 0.0f;
  out[2] = v > 0.0 ? (float)v : 1.0f;
}

// Entries (tile, body) in body order, tiles row by row.
__global__ void k_render_emit(const float4 *__restrict__ v0, const uint32_t *__restrict__ off,
                              uint32_t n, RenderParams P, uint64_t *__restrict__ keys,
                              uint32_t *__restrict__ vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const float4 v = v0[i];
    int x0, x1, y0, y1;
    if (!pixel_range(v.x, v.z, P.width, x0, x1) || !pixel_range(v.y, v.z, P.height, y0, y1))
      continue;
    uint32_t o = off[i];
    for (int ty = y0 / kTilePx; ty <= y1 / kTilePx; ++ty)
      for (int tx = x0 / kTilePx; tx <= x1 / kTilePx; ++tx) {
        keys[o] = (uint64_t)ty * P.tilesX + tx;
        vals[o] = i;
        ++o;
      }
  }
}

// First and one-past-last sorted entry of every tile (tiles start empty).
__global__ void k_render_tile_bounds(const uint64_t *__restrict__ keys,
                                     const uint32_t *__restrict__ count,
                                     uint32_t *__restrict__ first, uint32_t *__restrict__ last) {
  const uint32_t m = *count;
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m;
       e += gridDim.x * blockDim.x) {
    const uint64_t k = keys[e];
    if (e == 0 || keys[e - 1] != k) first[k] = e;
    if (e + 1 == m || keys[e + 1] != k) last[k] = e + 1;
  }
}

// One block per tile, one thread per pixel, entries in draw order.
__global__ void __launch_bounds__(kTilePx *kTilePx)
    k_render_composite(const float4 *__restrict__ v0, const float4 *__restrict__ v1,
                       const uint32_t *__restrict__ bodies, const uint32_t *__restrict__ first,
                       const uint32_t *__restrict__ last, RenderParams P,
                       float4 *__restrict__ image) {
  __shared__ float4 sV0[kTilePx * kTilePx], sV1[kTilePx * kTilePx];
  const uint32_t tile = blockIdx.x;
  const uint32_t tx = tile % P.tilesX, ty = tile / P.tilesX;
  const uint32_t px = tx * kTilePx + (threadIdx.x % kTilePx);
  const uint32_t py = ty * kTilePx + (threadIdx.x / kTilePx);
  const bool inside = px < P.width && py < P.height;
  const float cx = (float)px + 0.5f, cy = (float)py + 0.5f;
  float4 acc = make_float4(0.0f, 0.0f, 0.02f, 1.0f);
  const uint32_t e0 = first[tile], e1 = last[tile];
  for (uint32_t base = e0; base < e1; base += kTilePx * kTilePx) {
    const uint32_t cnt = min((uint32_t)(kTilePx * kTilePx), e1 - base);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const uint32_t b = bodies[base + threadIdx.x];
      sV0[threadIdx.x] = v0[b];
      sV1[threadIdx.x] = v1[b];
    }
    __syncthreads();
    if (!inside) continue;
    for (uint32_t k = 0; k < cnt; ++k) {
      const float4 v = sV0[k];
      const float dx = (cx - v.x) / v.z, dy = (cy - v.y) / v.z;
      const float r2 = dx * dx + dy * dy;
      if (r2 > 1.0f) continue;
      const float a = (1.0f - r2) * v.w * P.brightness;
      const float4 c = sV1[k];
      const float sr = c.x * a, sg = c.y * a, sb = c.z * a;
      if (P.mode == 1) {
        acc.x = sr + acc.x;
        acc.y = sg + acc.y;
        acc.z = sb + acc.z;
        acc.w = a + acc.w;
      } else {
        const float k1 = 1.0f - a;
        acc.x = sr + acc.x * k1;
        acc.y = sg + acc.y * k1;
        acc.z = sb + acc.z * k1;
        acc.w = a + acc.w * k1;
      }
    }
  }
  if (inside) image[(size_t)py * P.width + px] = acc;
}

} // namespace

void render_vertices(cudaStream_t s, const float4 *pv, const float2 *mr, uint32_t n,
                     const RenderParams &P, float4 *v0, float4 *v1, uint32_t *tiles,
                     double4 *partial, unsigned long long *total, float *stats) {
  const uint32_t blocks = (n + kVertexThreads - 1) / kVertexThreads;
  cudaMemsetAsync(total, 0, sizeof(unsigned long long), s);
  if (blocks)
    k_render_vertices<<<blocks, kVertexThreads, 0, s>>>(pv, mr, n, P, v0, v1, tiles, partial,
                                                         total);
  k_render_stats<<<1, 32, 0, s>>>(partial, blocks, stats);
}

uint32_t render_vertex_blocks(uint32_t n) {
  return (n + kVertexThreads - 1) / kVertexThreads;
}

void render_emit(cudaStream_t s, const float4 *v0, const uint32_t *off, uint32_t n,
                 const RenderParams &P, uint64_t *keys, uint32_t *vals) {
  uint32_t b = (n + 255) / 256;
  if (b > 148u * 16u) b = 148u * 16u;
  if (n) k_render_emit<<<b, 256, 0, s>>>(v0, off, n, P, keys, vals);
}

void render_composite(cudaStream_t s, const float4 *v0, const float4 *v1,
                      const uint64_t *keys, const uint32_t *bodies, const uint32_t *count,
                      uint32_t maxEntries, uint32_t *first, uint32_t *last,
                      const RenderParams &P, float4 *image) {
  const uint32_t tiles = P.tilesX * P.tilesY;
  cudaMemsetAsync(first, 0, sizeof(uint32_t) * tiles, s);
  cudaMemsetAsync(last, 0, sizeof(uint32_t) * tiles, s);
  uint32_t b = (maxEntries + 255) / 256;
  if (b > 148u * 16u) b = 148u * 16u;
  if (maxEntries) k_render_tile_bounds<<<b, 256, 0, s>>>(keys, count, first, last);
  k_render_composite<<<tiles, kTilePx * kTilePx, 0, s>>>(v0, v1, bodies, first, last, P,
                                                          image);
}

} // namespace nbx
