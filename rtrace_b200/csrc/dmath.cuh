// Double-precision vector math and Rust scalar semantics for the render
// kernels.  Every operation mirrors the reference's nalgebra operation
// order (dot = x*x' + y*y' + z*z' left to right, normalisation by division
// by the norm, gemv column accumulation) so that the device produces the
// same IEEE results as the reference's CPU code.  Compile with
// -fmad=false: a fused multiply-add would change the rounding.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#define RTB_HD __host__ __device__ __forceinline__

// float4 elements before node 0 of a single-precision BVH (the header
// holds the slab scale in element 0): 64 bytes, so that every 64-byte
// node lies in one 128-byte line of a 128-byte aligned array.
#define RTB_FBVH_HEAD 4

namespace rtb {

struct V3 {
  double x, y, z;
  RTB_HD double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
RTB_HD V3 mk(double x, double y, double z) { return V3{x, y, z}; }
RTB_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
RTB_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
RTB_HD V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
RTB_HD V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
RTB_HD V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
RTB_HD V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
RTB_HD V3 cmul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
RTB_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RTB_HD double norm(V3 a) { return sqrt(0.0 + dot(a, a)); }
RTB_HD V3 normalize(V3 a) { return a / norm(a); }
RTB_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
RTB_HD V3 ld3(const double* p) { return {p[0], p[1], p[2]}; }

// Bit casts between double and its IEEE encoding.
RTB_HD uint64_t dbits(double d) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  memcpy(&u, &d, 8);
  return u;
#endif
}
RTB_HD double bitsd(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, 8);
  return d;
#endif
}
// A packed int pair stored in the bits of a double (low word first).
RTB_HD int lo32(double d) { return (int)(uint32_t)(dbits(d) & 0xffffffffu); }
RTB_HD int hi32(double d) { return (int)(uint32_t)(dbits(d) >> 32); }
RTB_HD double pack2(int lo, int hi) { return bitsd((uint64_t)(uint32_t)lo | ((uint64_t)(uint32_t)hi << 32)); }

// f64::max / f64::min ignore NaN operands; CUDA fmax/fmin do the same.
RTB_HD double rmax(double a, double b) { return fmax(a, b); }
RTB_HD double rmin(double a, double b) { return fmin(a, b); }
RTB_HD double rclamp(double v, double lo, double hi) {
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}
RTB_HD double rfract(double v) { return v - trunc(v); }
// Saturating `as` casts (NaN -> 0)
RTB_HD uint64_t sat_u64(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551616.0) return ~0ULL;
  return (uint64_t)v;
}
RTB_HD uint8_t sat_u8(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 255.0) return 255;
  return (uint8_t)v;
}
RTB_HD int32_t sat_i32(double v) {
  if (v != v) return 0;
  if (v <= -2147483648.0) return (int32_t)0x80000000;
  if (v >= 2147483647.0) return 0x7fffffff;
  return (int32_t)v;
}

// Rows 0..2 of a 4x4 matrix (row-major, 12 doubles) applied by nalgebra's
// gemv to (v, w): y = m0*x; y = m1*y' + y; y = m2*z + y; y = m3*w + y.
RTB_HD V3 gemv34(const double* m, V3 v, double w) {
  double y0 = m[0] * v.x, y1 = m[4] * v.x, y2 = m[8] * v.x;
  y0 = m[1] * v.y + y0;
  y1 = m[5] * v.y + y1;
  y2 = m[9] * v.y + y2;
  y0 = m[2] * v.z + y0;
  y1 = m[6] * v.z + y1;
  y2 = m[10] * v.z + y2;
  y0 = m[3] * w + y0;
  y1 = m[7] * w + y1;
  y2 = m[11] * w + y2;
  return {y0, y1, y2};
}
RTB_HD V3 gemv33(const double* m, V3 v) {
  double y0 = m[0] * v.x, y1 = m[3] * v.x, y2 = m[6] * v.x;
  y0 = m[1] * v.y + y0;
  y1 = m[4] * v.y + y1;
  y2 = m[7] * v.y + y2;
  y0 = m[2] * v.z + y0;
  y1 = m[5] * v.z + y1;
  y2 = m[8] * v.z + y2;
  return {y0, y1, y2};
}

// reflect (src/lighting.rs:291-294)
RTB_HD V3 reflect(V3 i, V3 n) {
  double s = 2.0 * dot(i, n);
  return normalize(i - s * n);
}

// ------------------------------------------------------------------------
// rand 0.8 StdRng: ChaCha12 with a 64-bit block counter and stream 0,
// seeded by rand_core 0.6's PCG32 (XSH-RR) expansion of a u64.  The output
// is the concatenation of blocks 0, 1, 2, ...; next_u64 joins two
// consecutive words (low first), which holds across rand_core's 64-word
// buffer boundary as well.
// ------------------------------------------------------------------------
RTB_HD uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

RTB_HD void pcg32_key(uint64_t seed, uint32_t key[8]) {
  uint64_t st = seed;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    st = st * 6364136223846793005ULL + 11634580027462260723ULL;
    uint32_t xs = (uint32_t)(((st >> 18) ^ st) >> 27);
    uint32_t rot = (uint32_t)(st >> 59);
    key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
  }
}

RTB_HD void chacha_block(const uint32_t key[8], uint64_t counter, int double_rounds, uint32_t out[16]) {
  uint32_t x0 = 0x61707865u, x1 = 0x3320646eu, x2 = 0x79622d32u, x3 = 0x6b206574u;
  uint32_t x4 = key[0], x5 = key[1], x6 = key[2], x7 = key[3];
  uint32_t x8 = key[4], x9 = key[5], x10 = key[6], x11 = key[7];
  uint32_t x12 = (uint32_t)counter, x13 = (uint32_t)(counter >> 32), x14 = 0u, x15 = 0u;
#define RTB_QR(a, b, c, d)                 \
  a += b; d ^= a; d = rotl32(d, 16);       \
  c += d; b ^= c; b = rotl32(b, 12);       \
  a += b; d ^= a; d = rotl32(d, 8);        \
  c += d; b ^= c; b = rotl32(b, 7);
  for (int r = 0; r < double_rounds; r++) {
    RTB_QR(x0, x4, x8, x12) RTB_QR(x1, x5, x9, x13) RTB_QR(x2, x6, x10, x14) RTB_QR(x3, x7, x11, x15)
    RTB_QR(x0, x5, x10, x15) RTB_QR(x1, x6, x11, x12) RTB_QR(x2, x7, x8, x13) RTB_QR(x3, x4, x9, x14)
  }
#undef RTB_QR
  out[0] = x0 + 0x61707865u;
  out[1] = x1 + 0x3320646eu;
  out[2] = x2 + 0x79622d32u;
  out[3] = x3 + 0x6b206574u;
  out[4] = x4 + key[0];
  out[5] = x5 + key[1];
  out[6] = x6 + key[2];
  out[7] = x7 + key[3];
  out[8] = x8 + key[4];
  out[9] = x9 + key[5];
  out[10] = x10 + key[6];
  out[11] = x11 + key[7];
  out[12] = x12 + (uint32_t)counter;
  out[13] = x13 + (uint32_t)(counter >> 32);
  out[14] = x14;
  out[15] = x15;
}

struct StdRng {
  uint32_t key[8];
  uint32_t buf[16];
  uint64_t next_block;
  int pos;
  RTB_HD void init(uint64_t seed) {
    pcg32_key(seed, key);
    next_block = 0;
    pos = 16;
  }
  RTB_HD uint32_t u32() {
    if (pos >= 16) {
      chacha_block(key, next_block, 6, buf);
      next_block++;
      pos = 0;
    }
    return buf[pos++];
  }
  RTB_HD uint64_t u64() {
    uint64_t lo = u32();
    uint64_t hi = u32();
    return (hi << 32) | lo;
  }
  // Rng::gen::<f64>(): 53 high bits times 2^-53
  RTB_HD double f64() {
    const double scale = 1.0 / 9007199254740992.0;
    return scale * (double)(u64() >> 11);
  }
  // Rng::gen_range(low..high) for f64 (UniformFloat::sample_single).  The
  // caller has checked low < high and a finite range.  Returns false if the
  // retry bound ran out (cannot happen for finite, ordered bounds).
  RTB_HD bool range(double low, double high, double* out) {
    double scale = high - low;
    for (int it = 0; it < 64; it++) {
      double v12 = bitsd((u64() >> 12) | (1023ULL << 52));
      double res = (v12 - 1.0) * scale + low;
      if (res < high) {
        *out = res;
        return true;
      }
      scale = bitsd(dbits(scale) - 1);
    }
    return false;
  }
};

}  // namespace rtb
