// nbx_math.h -- arithmetic shared by the device kernels and host code.
//
// Everything here is integer or single-precision float arithmetic and
// compiles for host and device alike, so host-side tests of these
// functions speak for the kernels too.
//
//  * sd_*: IEEE-754 binary64 add/sub/mul/div and floor done with 64-bit
//    integer arithmetic (round to nearest, ties to even).  The reference
//    quantises Morton coordinates in double
//    (src/cuda/TreeKernels.cuh:48-57, CudaQuadTree.cu:41-44); these
//    reproduce those doubles bit for bit anywhere, host included: the
//    per-instance Morton frame is made with them, and the host checks use
//    them.  The per-body quantisation of the step runs in native FP64
//    (build.cu), which rounds the same IEEE operations the same way.
//  * fast_inv_sqrt: the force law's bit-level inverse square root
//    (src/QuadTree.cpp:11-26, TreeKernels.cuh:180-195).
//  * float_order_key: a float's total-order key for radix sorting.
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define NBX_HD __host__ __device__ __forceinline__
#else
#define NBX_HD inline
#endif

namespace nbx {

NBX_HD uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}

NBX_HD float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

NBX_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
  return __clzll((long long)x);
#else
  return x ? __builtin_clzll(x) : 64;
#endif
}

NBX_HD int clz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __clz((int)x);
#else
  return x ? __builtin_clz(x) : 32;
#endif
}

// High 64 bits of a 64x64 product.
NBX_HD uint64_t umulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// ---------------------------------------------------------------------
// binary64 in integers.
constexpr uint64_t kSdSign = 0x8000000000000000ull;
constexpr uint64_t kSdExpMask = 0x7FF0000000000000ull;
constexpr uint64_t kSdFracMask = 0x000FFFFFFFFFFFFFull;
constexpr uint64_t kSdQNaN = 0x7FF8000000000000ull;
constexpr uint64_t kSdInf = 0x7FF0000000000000ull;

NBX_HD bool sd_isnan(uint64_t a) {
  return (a & kSdExpMask) == kSdExpMask && (a & kSdFracMask) != 0;
}
NBX_HD bool sd_isinf(uint64_t a) { return (a & ~kSdSign) == kSdInf; }
NBX_HD bool sd_iszero(uint64_t a) { return (a & ~kSdSign) == 0; }

// Exact float -> double conversion.
NBX_HD uint64_t sd_from_float(float f) {
  const uint32_t u = f2u(f);
  const uint64_t sign = (uint64_t)(u >> 31) << 63;
  const uint32_t e = (u >> 23) & 0xFFu;
  const uint32_t m = u & 0x7FFFFFu;
  if (e == 0xFFu) {
    return sign | kSdInf | ((uint64_t)m << 29) | (m ? (1ull << 51) : 0);
  }
  if (e == 0) {
    if (m == 0) return sign;
    const int p = 31 - clz32(m); // leading bit position, 0..22
    const uint64_t de = (uint64_t)(p - 149 + 1023);
    const uint64_t frac = ((uint64_t)m << (52 - p)) & kSdFracMask;
    return sign | (de << 52) | frac;
  }
  return sign | ((uint64_t)(e - 127 + 1023) << 52) | ((uint64_t)m << 29);
}

// Unpacks a finite non-zero value: mantissa with the implicit bit at
// position 52, unbiased-free exponent field (>= 1).
NBX_HD void sd_unpack(uint64_t a, int &e, uint64_t &m) {
  e = (int)((a >> 52) & 0x7FF);
  m = a & kSdFracMask;
  if (e == 0) {
    // subnormal: normalise so the leading bit is at 52
    const int sh = clz64(m) - 11;
    m <<= sh;
    e = 1 - sh;
  } else {
    m |= 1ull << 52;
  }
}

// Rounds a mantissa carrying 3 extra low bits (guard, round, sticky) with
// its leading bit at position 55, and packs it.  e is the exponent field of
// the leading bit; values below the normal range are denormalised first.
NBX_HD uint64_t sd_round_pack(uint64_t sign, int e, uint64_t m) {
  if (e <= 0) {
    // shift right into the subnormal range, keeping a sticky bit
    const int sh = 1 - e;
    if (sh >= 64) {
      m = (m != 0);
    } else {
      const uint64_t lost = m & ((1ull << sh) - 1);
      m = (m >> sh) | (lost != 0);
    }
    e = 0;
  }
  const uint32_t low = (uint32_t)(m & 7u);
  m >>= 3;
  if (low > 4u || (low == 4u && (m & 1u))) {
    m += 1;
    if (m == (1ull << 53)) {
      m >>= 1;
      e += 1;
    } else if (e == 0 && m == (1ull << 52)) {
      e = 1; // rounded up out of the subnormal range
    }
  }
  if (e >= 2047) return sign | kSdInf;
  if (e == 0) return sign | (m & kSdFracMask);
  return sign | ((uint64_t)e << 52) | (m & kSdFracMask);
}

NBX_HD uint64_t sd_add(uint64_t a, uint64_t b) {
  if (sd_isnan(a) || sd_isnan(b)) return kSdQNaN;
  if (sd_isinf(a)) {
    if (sd_isinf(b) && ((a ^ b) & kSdSign)) return kSdQNaN;
    return a;
  }
  if (sd_isinf(b)) return b;
  if (sd_iszero(a)) {
    if (sd_iszero(b)) return a & b & kSdSign; // -0 only if both are -0
    return b;
  }
  if (sd_iszero(b)) return a;
  // |a| >= |b|
  if ((a & ~kSdSign) < (b & ~kSdSign)) {
    const uint64_t t = a;
    a = b;
    b = t;
  }
  const uint64_t sa = a & kSdSign, sb = b & kSdSign;
  int ea, eb;
  uint64_t ma, mb;
  sd_unpack(a, ea, ma);
  sd_unpack(b, eb, mb);
  ma <<= 3;
  mb <<= 3;
  const int d = ea - eb;
  if (d > 0) {
    if (d >= 60) {
      mb = (mb != 0);
    } else {
      const uint64_t lost = mb & ((1ull << d) - 1);
      mb = (mb >> d) | (lost != 0);
    }
  }
  uint64_t m;
  int e = ea;
  if (sa == sb) {
    m = ma + mb;
    if (m >> 56) {
      m = (m >> 1) | (m & 1u);
      e += 1;
    }
  } else {
    m = ma - mb;
    if (m == 0) return 0; // exact cancellation gives +0
    const int sh = clz64(m) - 8; // bring the leading bit to 55
    if (sh > 0) {
      m <<= sh;
      e -= sh;
    }
  }
  return sd_round_pack(sa, e, m);
}

NBX_HD uint64_t sd_neg(uint64_t a) { return a ^ kSdSign; }
NBX_HD uint64_t sd_sub(uint64_t a, uint64_t b) { return sd_add(a, sd_neg(b)); }

NBX_HD uint64_t sd_mul(uint64_t a, uint64_t b) {
  const uint64_t sign = (a ^ b) & kSdSign;
  if (sd_isnan(a) || sd_isnan(b)) return kSdQNaN;
  if (sd_isinf(a) || sd_isinf(b)) {
    if (sd_iszero(a) || sd_iszero(b)) return kSdQNaN;
    return sign | kSdInf;
  }
  if (sd_iszero(a) || sd_iszero(b)) return sign;
  int ea, eb;
  uint64_t ma, mb;
  sd_unpack(a, ea, ma);
  sd_unpack(b, eb, mb);
  // 106-bit product; the leading bit is at 104 or 105.
  const uint64_t lo = ma * mb;
  const uint64_t hi = umulhi64(ma, mb);
  int e = ea + eb - 1023;
  // Take the top 56 bits (leading bit at 55) with a sticky bit.
  uint64_t m;
  uint64_t rest;
  if (hi >> 41) { // bit 105 set
    m = (hi << 14) | (lo >> 50);
    rest = lo & ((1ull << 50) - 1);
    e += 1;
  } else {
    m = (hi << 15) | (lo >> 49);
    rest = lo & ((1ull << 49) - 1);
  }
  m |= (rest != 0);
  return sd_round_pack(sign, e, m);
}

NBX_HD uint64_t sd_div(uint64_t a, uint64_t b) {
  const uint64_t sign = (a ^ b) & kSdSign;
  if (sd_isnan(a) || sd_isnan(b)) return kSdQNaN;
  if (sd_isinf(a)) return sd_isinf(b) ? kSdQNaN : (sign | kSdInf);
  if (sd_isinf(b)) return sign;
  if (sd_iszero(b)) return sd_iszero(a) ? kSdQNaN : (sign | kSdInf);
  if (sd_iszero(a)) return sign;
  int ea, eb;
  uint64_t ma, mb;
  sd_unpack(a, ea, ma);
  sd_unpack(b, eb, mb);
  int e = ea - eb + 1023;
  if (ma < mb) {
    ma <<= 1;
    e -= 1;
  }
  // ma/mb in [1, 2): 56 quotient bits by restoring division, leading bit 55.
  uint64_t q = 0, r = ma;
  for (int i = 0; i < 56; ++i) {
    q <<= 1;
    if (r >= mb) {
      r -= mb;
      q |= 1u;
    }
    r <<= 1;
  }
  q |= (r != 0);
  return sd_round_pack(sign, e, q);
}

// Reference quantise(): q = floor(p); !(q > 0) -> 0; q >= 2^32-1 -> 2^32-1.
NBX_HD uint32_t sd_quantise_floor(uint64_t p) {
  if (sd_isnan(p) || (p & kSdSign) || sd_iszero(p)) return 0u;
  const int E = (int)((p >> 52) & 0x7FF) - 1023;
  if (E < 0) return 0u;
  if (E >= 32) return 0xFFFFFFFFu;
  const uint64_t m = (p & kSdFracMask) | (1ull << 52);
  return (uint32_t)(m >> (52 - E));
}

// Per-root constants of mortonKernel (CudaQuadTree.cu:41-44):
// x0 = double(cx) - 0.5*size, y0 likewise, scale = 2^32/size (0 if !(size>0)).
struct MortonFrame {
  uint64_t x0, y0, scale;
};

NBX_HD MortonFrame sd_morton_frame(float cx, float cy, float size) {
  MortonFrame f;
  const uint64_t half = sd_mul(0x3FE0000000000000ull, sd_from_float(size));
  f.x0 = sd_sub(sd_from_float(cx), half);
  f.y0 = sd_sub(sd_from_float(cy), half);
  f.scale = (size > 0.0f) ? sd_div(0x41F0000000000000ull, sd_from_float(size))
                          : 0ull;
  return f;
}

NBX_HD uint32_t sd_quantise(float v, uint64_t lo, uint64_t scale) {
  return sd_quantise_floor(sd_mul(sd_sub(sd_from_float(v), lo), scale));
}

// spreadBits (TreeKernels.cuh:37-45).
NBX_HD uint64_t spread_bits(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

// mortonCode (TreeKernels.cuh:62-66): digit = 2*ybit + xbit.
NBX_HD uint64_t morton_code(float x, float y, const MortonFrame &f) {
  return (spread_bits(sd_quantise(y, f.y0, f.scale)) << 1) |
         spread_bits(sd_quantise(x, f.x0, f.scale));
}

// digitAt (TreeKernels.cuh:68-70).
NBX_HD int digit_at(uint64_t code, int depth) {
  return (int)((code >> (62 - 2 * depth)) & 3u);
}

// Common prefix length in 2-bit digits (32 for equal codes).
NBX_HD int lcp_digits(uint64_t a, uint64_t b) {
  return a == b ? 32 : (clz64(a ^ b) >> 1);
}

// fastInvSqrt (QuadTree.cpp:11-26): magic-constant guess + one Newton step.
NBX_HD float fast_inv_sqrt(float x) {
  const float xhalf = 0.5f * x;
  const uint32_t i = 0x5f3759dfu - (f2u(x) >> 1);
  const float y = u2f(i);
  return y * (1.5f - xhalf * y * y);
}

// Total-order key of a float for ascending radix sorts; -0 sorts as +0 so
// that key order matches the float comparison a < b.
NBX_HD uint32_t float_order_key(float f) {
  uint32_t u = f2u(f);
  if (u == 0x80000000u) u = 0;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

} // namespace nbx
