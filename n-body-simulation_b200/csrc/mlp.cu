// mlp.cu -- harvesting, training and evaluation of the learned far-field
// correction (feature map and layout in mlp.cuh).
//
// Harvest: sampled targets walk the current tree with the MAC at theta;
// every accepted cell with s/r >= band yields a training row whose target
// is the cell's exact FP64 force on the target (direct sum over the cell's
// bodies with the tree force law, CheckCuda.cu:453-475) minus its FP64
// monopole, in the cell's (u, w) frame, divided by the monopole magnitude.
//
// Training: plain SIMT FP32 forward/backward with BF16-rounded weights and
// activations (the precision the tensor-core inference runs at), gradients
// summed in a fixed order (deterministic), Adam on an FP32 master copy that
// is re-packed to BF16 after every step.
#include "mlp.cuh"
#include "nbx_state.cuh"

#include <float.h>

#include <algorithm>

namespace nbx {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ float bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float sigmoidf(float z) { return 1.0f / (1.0f + expf(-z)); }

// One thread per target: walk the tree, emit (target, node) for accepted
// band cells.
__global__ void k_harvest_walk(DevState S, const uint32_t *__restrict__ targets,
                               uint32_t nt, float tSq, float bandSq,
                               uint2 *items, uint32_t cap, uint32_t *count) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nt;
       q += gridDim.x * blockDim.x) {
    const uint32_t t = targets[q];
    const float4 P = S.xym[t];
    const SegDev &G = S.seg[S.segOf[t]];
    uint32_t cur = G.travBase, end = G.travBase + G.travCount;
    uint32_t guard = 0;
    while (cur < end && ++guard < (1u << 24)) {
      const float4 A = S.tN[cur].a;
      const int4 B = S.tN[cur].b;
      const float dx = A.x - P.x, dy = A.y - P.y;
      const float dSq = dx * dx + dy * dy;
      const uint32_t nxt = (uint32_t)B.x > cur ? (uint32_t)B.x : end;
      if (A.w < dSq * tSq) {
        if (A.z > 0.0f && A.w >= dSq * bandSq) {
          const uint32_t slot = atomicAdd(count, 1u);
          if (slot < cap) items[slot] = make_uint2(t, cur);
        }
        cur = nxt;
      } else if (B.y == B.x) { // leaf
        cur = nxt;
      } else {
        cur = cur + 1;
      }
    }
  }
}

// One warp per item: FP64 exact cell force, features and target.
__global__ void k_harvest_rows(DevState S, const uint2 *__restrict__ items,
                               const uint32_t *count, uint32_t cap, float eps,
                               float *rows) {
  const int lane = threadIdx.x & 31;
  const uint32_t nItems = min(*count, cap);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nItems;
       it += warps) {
    const uint2 pr = items[it];
    const uint32_t t = pr.x, g = pr.y;
    const float4 P = S.xym[t];
    const float4 A = S.tN[g].a;
    const int4 B = S.tN[g].b;
    const float4 M = S.tM[g];
    const float2 Q = S.tC[g];
    const double e2 = (double)eps * eps;
    double sx = 0.0, sy = 0.0;
    for (int j = B.z + lane; j < B.w; j += 32) {
      if ((uint32_t)j == t) continue;
      const float4 b = S.xym[j];
      const double dx = (double)b.x - P.x, dy = (double)b.y - P.y;
      const double d2 = dx * dx + dy * dy;
      if (d2 == 0.0) continue;
      const double f = (double)b.z / (sqrt(d2) * (d2 + e2));
      sx += dx * f;
      sy += dy * f;
    }
    for (int o = 16; o > 0; o >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, o);
      sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (lane == 0) {
      const double dx = (double)A.x - P.x, dy = (double)A.y - P.y;
      const double d2 = dx * dx + dy * dy;
      const double r = sqrt(d2);
      const double fm = (double)A.z / (r * (d2 + e2));
      const double mx = dx * fm, my = dy * fm, mag = r * fm;
      float f[9], ux, uy;
      float *row = rows + (size_t)it * kMlpRow;
      const float fdx = A.x - P.x, fdy = A.y - P.y;
      const bool ok = mlp_features(fdx, fdy, fdx * fdx + fdy * fdy, A.z, M.w,
                                   Q.x, Q.y, A.x, A.y, M.x, M.y, M.z, 1.0f,
                                   eps, f, ux, uy) &&
                      mag > 0.0;
      if (ok) {
        const double ex = (sx - mx) / mag, ey = (sy - my) / mag;
        const double t0 = ex * ux + ey * uy;
        const double t1 = -ex * uy + ey * ux;
        for (int k = 0; k < 9; ++k) row[k] = fminf(fmaxf(f[k], -8.0f), 8.0f);
        row[9] = (float)fmin(fmax(t0, -8.0), 8.0);
        row[10] = (float)fmin(fmax(t1, -8.0), 8.0);
        row[11] = 1.0f;
      } else {
        for (int k = 0; k < kMlpRow; ++k) row[k] = 0.0f; // weight 0
      }
    }
  }
}

// Training: forward/backward for a block of 64 rows, then per-parameter
// gradient sums over those rows in a fixed order.
constexpr int kRowsPerBlock = 64;

struct RowCache {
  float x[kRowsPerBlock][9];
  float h1[kRowsPerBlock][32];
  float h2[kRowsPerBlock][32];
  float dz1[kRowsPerBlock][32];
  float dz2[kRowsPerBlock][32];
  float dy[kRowsPerBlock][2];
  float loss[kRowsPerBlock];
};

__global__ void __launch_bounds__(kBlock)
    k_mlp_grad_partial(const float *__restrict__ rows,
                       const uint32_t *__restrict__ order, uint32_t first,
                       uint32_t batch, float scale, const float *__restrict__ P,
                       float *__restrict__ partial, float *__restrict__ lossPart) {
  __shared__ float w[kMlpParams];
  __shared__ RowCache c;
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) {
    const bool isBias = (p >= kOffB1 && p < kOffW2) || (p >= kOffB2 && p < kOffW3) ||
                        p >= kOffB3;
    w[p] = isBias ? P[p] : bf16r(P[p]);
  }
  __syncthreads();
  const uint32_t r = threadIdx.x;
  const uint32_t local = blockIdx.x * kRowsPerBlock + r;
  if (r < kRowsPerBlock) {
    float x[9], z1[32], h1[32], z2[32], h2[32];
    float tgt[2] = {0.0f, 0.0f}, wt = 0.0f;
    if (local < batch) {
      const float *row = rows + (size_t)(order ? order[first + local] : first + local) * kMlpRow;
      for (int k = 0; k < 9; ++k) x[k] = bf16r(row[k]);
      tgt[0] = row[9];
      tgt[1] = row[10];
      wt = row[11];
    } else {
      for (int k = 0; k < 9; ++k) x[k] = 0.0f;
    }
    for (int j = 0; j < 32; ++j) {
      float s = w[kOffB1 + j];
      for (int k = 0; k < 9; ++k) s += w[kOffW1 + j * 9 + k] * x[k];
      z1[j] = s;
      h1[j] = bf16r(s * sigmoidf(s));
    }
    for (int j = 0; j < 32; ++j) {
      float s = w[kOffB2 + j];
      for (int k = 0; k < 32; ++k) s += w[kOffW2 + j * 32 + k] * h1[k];
      z2[j] = s;
      h2[j] = bf16r(s * sigmoidf(s));
    }
    float loss = 0.0f;
    for (int j = 0; j < 2; ++j) {
      float s = w[kOffB3 + j];
      for (int k = 0; k < 32; ++k) s += w[kOffW3 + j * 32 + k] * h2[k];
      const float e = s - tgt[j];
      loss += wt * e * e;
      c.dy[r][j] = scale * 2.0f * wt * e;
    }
    c.loss[r] = loss;
    // backward
    float dz2v[32];
    for (int k = 0; k < 32; ++k) {
      const float dh = w[kOffW3 + k] * c.dy[r][0] + w[kOffW3 + 32 + k] * c.dy[r][1];
      const float sg = sigmoidf(z2[k]);
      dz2v[k] = dh * sg * (1.0f + z2[k] * (1.0f - sg));
      c.dz2[r][k] = dz2v[k];
    }
    for (int k = 0; k < 32; ++k) {
      float dh = 0.0f;
      for (int j = 0; j < 32; ++j) dh += w[kOffW2 + j * 32 + k] * dz2v[j];
      const float sg = sigmoidf(z1[k]);
      c.dz1[r][k] = dh * sg * (1.0f + z1[k] * (1.0f - sg));
    }
    for (int k = 0; k < 9; ++k) c.x[r][k] = x[k];
    for (int k = 0; k < 32; ++k) {
      c.h1[r][k] = h1[k];
      c.h2[r][k] = h2[k];
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) {
    float s = 0.0f;
    if (p < kOffB1) {
      const int j = p / 9, k = p % 9;
      for (int q = 0; q < kRowsPerBlock; ++q) s += c.dz1[q][j] * c.x[q][k];
    } else if (p < kOffW2) {
      const int j = p - kOffB1;
      for (int q = 0; q < kRowsPerBlock; ++q) s += c.dz1[q][j];
    } else if (p < kOffB2) {
      const int j = (p - kOffW2) / 32, k = (p - kOffW2) % 32;
      for (int q = 0; q < kRowsPerBlock; ++q) s += c.dz2[q][j] * c.h1[q][k];
    } else if (p < kOffW3) {
      const int j = p - kOffB2;
      for (int q = 0; q < kRowsPerBlock; ++q) s += c.dz2[q][j];
    } else if (p < kOffB3) {
      const int j = (p - kOffW3) / 32, k = (p - kOffW3) % 32;
      for (int q = 0; q < kRowsPerBlock; ++q) s += c.dy[q][j] * c.h2[q][k];
    } else {
      const int j = p - kOffB3;
      for (int q = 0; q < kRowsPerBlock; ++q) s += c.dy[q][j];
    }
    partial[(size_t)blockIdx.x * kMlpParams + p] = s;
  }
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (int q = 0; q < kRowsPerBlock; ++q) s += c.loss[q];
    lossPart[blockIdx.x] = s;
  }
}

__global__ void k_mlp_grad_reduce(const float *__restrict__ partial, int blocks,
                                  const float *__restrict__ lossPart,
                                  float *grad, float *lossOut) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= kMlpParams;
       p += gridDim.x * blockDim.x) {
    float s = 0.0f;
    if (p < kMlpParams) {
      for (int b = 0; b < blocks; ++b) s += partial[(size_t)b * kMlpParams + p];
      grad[p] = s;
    } else {
      for (int b = 0; b < blocks; ++b) s += lossPart[b];
      if (lossOut) *lossOut = s;
    }
  }
}

__global__ void k_mlp_pack(const float *__restrict__ P, MlpDev *W) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < 32 * 16) {
    const int j = p / 16, k = p % 16;
    W->w1[j][k] = __float2bfloat16_rn(k < 9 ? P[kOffW1 + j * 9 + k] : 0.0f);
  }
  if (p < 32 * 32) W->w2[p / 32][p % 32] = __float2bfloat16_rn(P[kOffW2 + p]);
  if (p < 8 * 32) {
    const int j = p / 32, k = p % 32;
    W->w3[j][k] = __float2bfloat16_rn(j < 2 ? P[kOffW3 + j * 32 + k] : 0.0f);
  }
  if (p < 32) {
    W->b1[p] = P[kOffB1 + p];
    W->b2[p] = P[kOffB2 + p];
  }
  if (p < 8) W->b3[p] = p < 2 ? P[kOffB3 + p] : 0.0f;
}

__global__ void k_mlp_adam(float *P, const float *__restrict__ grad, float *m,
                           float *v, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float g = grad[p];
  m[p] = b1 * m[p] + (1.0f - b1) * g;
  v[p] = b2 * v[p] + (1.0f - b2) * g * g;
  P[p] -= lr * (m[p] / c1) / (sqrtf(v[p] / c2) + eps);
}

// Forward only: SIMT (training precision) or tensor cores (inference path).
__global__ void k_mlp_eval_simt(const float *__restrict__ feat, uint32_t n,
                                const float *__restrict__ P, float *out) {
  __shared__ float w[kMlpParams];
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) {
    const bool isBias = (p >= kOffB1 && p < kOffW2) || (p >= kOffB2 && p < kOffW3) ||
                        p >= kOffB3;
    w[p] = isBias ? P[p] : bf16r(P[p]);
  }
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[9], h1[32], h2[32];
  for (int k = 0; k < 9; ++k) x[k] = bf16r(feat[(size_t)i * 9 + k]);
  for (int j = 0; j < 32; ++j) {
    float s = w[kOffB1 + j];
    for (int k = 0; k < 9; ++k) s += w[kOffW1 + j * 9 + k] * x[k];
    h1[j] = bf16r(s * sigmoidf(s));
  }
  for (int j = 0; j < 32; ++j) {
    float s = w[kOffB2 + j];
    for (int k = 0; k < 32; ++k) s += w[kOffW2 + j * 32 + k] * h1[k];
    h2[j] = bf16r(s * sigmoidf(s));
  }
  for (int j = 0; j < 2; ++j) {
    float s = w[kOffB3 + j];
    for (int k = 0; k < 32; ++k) s += w[kOffW3 + j * 32 + k] * h2[k];
    out[(size_t)i * 2 + j] = s;
  }
}

__global__ void k_mlp_eval_mma(const float *__restrict__ feat, uint32_t n,
                               const MlpDev *__restrict__ Wg, float *out) {
  __shared__ MlpDev W;
  __shared__ __nv_bfloat16 stage[kBlock / 32][32][16];
  for (int i = threadIdx.x; i < (int)(sizeof(MlpDev) / 4); i += blockDim.x)
    reinterpret_cast<uint32_t *>(&W)[i] = reinterpret_cast<const uint32_t *>(Wg)[i];
  __syncthreads();
  const uint32_t warpsTotal = (gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n;
       base += warpsTotal * 32) {
    const uint32_t i = base + lane;
    float f[9];
    for (int k = 0; k < 9; ++k) f[k] = i < n ? feat[(size_t)i * 9 + k] : 0.0f;
    float o0, o1;
    mlp_warp(W, f, stage[wi], o0, o1);
    if (i < n) {
      out[(size_t)i * 2] = o0;
      out[(size_t)i * 2 + 1] = o1;
    }
  }
}

} // namespace

// ------------------------------------------------------------------ host
void mlp_harvest(cudaStream_t s, const DevState &S, const uint32_t *targets,
                 uint32_t nt, float theta, float band, float eps, uint2 *items,
                 uint32_t cap, uint32_t *count, float *rows) {
  cudaMemsetAsync(count, 0, 4, s);
  k_harvest_walk<<<(nt + 127) / 128, 128, 0, s>>>(S, targets, nt, theta * theta,
                                                 band * band, items, cap, count);
  k_harvest_rows<<<1184, kBlock, 0, s>>>(S, items, count, cap, eps, rows);
}

void mlp_pack(cudaStream_t s, const float *P, MlpDev *W) {
  k_mlp_pack<<<4, 256, 0, s>>>(P, W);
}

// Gradient of the mean weighted squared error over `batch` rows
// (order[first..first+batch) or rows first.. if order is null).
void mlp_gradient(cudaStream_t s, const float *rows, const uint32_t *order,
                  uint32_t first, uint32_t batch, const float *P, float *partial,
                  float *lossPart, float *grad, float *loss) {
  const int blocks = (batch + kRowsPerBlock - 1) / kRowsPerBlock;
  k_mlp_grad_partial<<<blocks, kBlock, 0, s>>>(rows, order, first, batch,
                                               1.0f / (float)batch, P, partial,
                                               lossPart);
  k_mlp_grad_reduce<<<8, 256, 0, s>>>(partial, blocks, lossPart, grad, loss);
}

void mlp_adam(cudaStream_t s, float *P, const float *grad, float *m, float *v,
              int step, float lr, MlpDev *W) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(P, grad, m, v, lr, b1, b2,
                                                      1e-8f, c1, c2);
  k_mlp_pack<<<4, 256, 0, s>>>(P, W);
}

void mlp_eval(cudaStream_t s, const float *feat, uint32_t n, const float *P,
              const MlpDev *W, float *out, bool tensor) {
  if (tensor)
    k_mlp_eval_mma<<<std::max(1u, std::min(1184u, (n + 255) / 256)), kBlock, 0, s>>>(feat, n, W, out);
  else
    k_mlp_eval_simt<<<(n + 255) / 256, 256, 0, s>>>(feat, n, P, out);
}

int mlp_rows_per_block() { return kRowsPerBlock; }

} // namespace nbx
