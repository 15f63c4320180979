// rtrace_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A scalar, double-precision CPU restatement of the render path of
// SeaRyanC/rtrace (a Rust crate).  It exists so that the tests, the smoke
// check and the CPU-baseline leg of bench.py can compare the CUDA renderer
// against the reference's algorithm on the same inputs.  Nothing in the
// shipped library links, loads or calls this file.
//
// The reference cannot be compiled in this environment (no Rust toolchain),
// so this restatement follows its source file by file; every function names
// the reference lines it restates.  Arithmetic is written in the same
// operation order as the reference (nalgebra's left-to-right dot products,
// division-based normalisation, no fused multiply-add: build with
// -ffp-contract=off), with Rust's saturating float->int casts and
// NaN-ignoring f64::max/min.
//
// Third-party arithmetic that the reference pulls from crates that are not
// vendored (no Cargo.lock; versions are the newest semver-compatible ones):
//   * rand 0.8 / rand_chacha 0.3 / rand_core 0.6: StdRng = ChaCha12,
//     seed_from_u64 = PCG32 (XSH-RR) seed expansion, gen::<f64>() = 53-bit
//     multiply method, gen_range(f64..f64) = [1,2)-mantissa method with a
//     one-ulp scale decrease on rounding up to `high`.
//   * nalgebra 0.33: vector/matrix operation order (gemv column order,
//     4x4 cofactor inverse, 3x3 adjugate inverse, from_euler_angles).
//   * serde_json 1.0: default (non float_roundtrip) float parsing,
//     significand as f64 then one multiply/divide by a power of ten.
// These are restated from their published algorithms.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

namespace orc {

static const double INF = std::numeric_limits<double>::infinity();

struct Err : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------------------
// Rust scalar semantics
// ---------------------------------------------------------------------------
// f64::max / f64::min ignore a NaN operand (IEEE maxNum / minNum).
static inline double rmax(double a, double b) { return std::fmax(a, b); }
static inline double rmin(double a, double b) { return std::fmin(a, b); }
// f64::clamp: NaN passes through.
static inline double rclamp(double v, double lo, double hi) {
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}
// f64::fract = self - self.trunc()
static inline double rfract(double v) { return v - std::trunc(v); }
// `x as u64` (saturating, NaN -> 0)
static inline uint64_t sat_u64(double v) {
  if (!(v > 0.0)) return 0;  // NaN, negatives, zero
  if (v >= 18446744073709551616.0) return UINT64_MAX;
  return (uint64_t)v;
}
// `x as u8` (saturating, NaN -> 0)
static inline uint8_t sat_u8(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 255.0) return 255;
  return (uint8_t)v;
}
// `x as i32` (saturating, NaN -> 0)
static inline int32_t sat_i32(double v) {
  if (std::isnan(v)) return 0;
  if (v <= -2147483648.0) return INT32_MIN;
  if (v >= 2147483647.0) return INT32_MAX;
  return (int32_t)v;
}
// f64::to_radians: self * (PI / 180)
static inline double to_radians(double deg) {
  const double RADS_PER_DEG = M_PI / 180.0;
  return deg * RADS_PER_DEG;
}
// f64::round: half away from zero
static inline double rround(double v) { return std::round(v); }

// ---------------------------------------------------------------------------
// nalgebra Vector3 / Point3 in the reference's operation order
// ---------------------------------------------------------------------------
struct V3 {
  double x, y, z;
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
static inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
static inline V3 cmul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
// dot: a + b + c, evaluated left to right
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// norm_squared starts from zero and adds the dot product
static inline double norm(V3 a) { return std::sqrt(0.0 + dot(a, a)); }
// Unit::new_normalize / normalize divide each component by the norm
static inline V3 normalize(V3 a) { double n = norm(a); return a / n; }
static inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// 4x4 matrix, stored row-major m[r][c]; products follow nalgebra's gemv
// (column-by-column accumulation: y = a_0 x_0, then y = a_j x_j + y).
struct M4 {
  double m[4][4];
};
static M4 m4_identity() {
  M4 r;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) r.m[i][j] = (i == j) ? 1.0 : 0.0;
  return r;
}
static void m4_gemv(const M4& a, const double x[4], double y[4]) {
  for (int i = 0; i < 4; i++) y[i] = (1.0 * a.m[i][0]) * x[0];
  for (int j = 1; j < 4; j++)
    for (int i = 0; i < 4; i++) y[i] = (1.0 * a.m[i][j]) * x[j] + 1.0 * y[i];
}
static M4 m4_mul(const M4& a, const M4& b) {
  M4 r;
  for (int j = 0; j < 4; j++) {
    double col[4] = {b.m[0][j], b.m[1][j], b.m[2][j], b.m[3][j]};
    double y[4];
    m4_gemv(a, col, y);
    for (int i = 0; i < 4; i++) r.m[i][j] = y[i];
  }
  return r;
}
static V3 m4_point(const M4& a, V3 p) {  // (M * p.to_homogeneous()).xyz
  double x[4] = {p.x, p.y, p.z, 1.0}, y[4];
  m4_gemv(a, x, y);
  return {y[0], y[1], y[2]};
}
static V3 m4_vec(const M4& a, V3 v) {  // (M * v.to_homogeneous()).xyz (w = 0)
  double x[4] = {v.x, v.y, v.z, 0.0}, y[4];
  m4_gemv(a, x, y);
  return {y[0], y[1], y[2]};
}
static bool m4_is_identity(const M4& a) {
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      if (a.m[i][j] != ((i == j) ? 1.0 : 0.0)) return false;
  return true;
}
// nalgebra try_inverse for 4x4: cofactor expansion over the column-major
// slice m[k] = M[k % 4][k / 4], determinant from the first column of
// cofactors, then every entry multiplied by 1/det.
static bool m4_try_inverse(const M4& M, M4* out) {
  double m[16];
  for (int k = 0; k < 16; k++) m[k] = M.m[k % 4][k / 4];
  double inv[16];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] +
           m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] -
           m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] +
           m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] -
            m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  if (det == 0.0) return false;
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] -
           m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] +
           m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] -
           m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] +
            m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] +
           m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] -
           m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] +
            m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] -
            m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] -
           m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] +
           m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] -
            m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] +
            m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double inv_det = 1.0 / det;
  for (int k = 0; k < 16; k++) out->m[k % 4][k / 4] = inv[k] * inv_det;
  return true;
}
// nalgebra try_inverse for 3x3 (adjugate divided by the determinant).
static bool m3_try_inverse(const double a[3][3], double out[3][3]) {
  double m11 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double m12 = a[1][0] * a[2][2] - a[2][0] * a[1][2];
  double m13 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
  double det = a[0][0] * m11 - a[0][1] * m12 + a[0][2] * m13;
  if (det == 0.0) return false;
  double m21 = a[0][1] * a[2][2] - a[2][1] * a[0][2];
  double m22 = a[0][0] * a[2][2] - a[2][0] * a[0][2];
  double m23 = a[0][0] * a[2][1] - a[2][0] * a[0][1];
  double m31 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
  double m32 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
  double m33 = a[0][0] * a[1][1] - a[1][0] * a[0][1];
  out[0][0] = m11 / det;
  out[1][0] = -m12 / det;
  out[2][0] = m13 / det;
  out[0][1] = -m21 / det;
  out[1][1] = m22 / det;
  out[2][1] = -m23 / det;
  out[0][2] = m31 / det;
  out[1][2] = -m32 / det;
  out[2][2] = m33 / det;
  return true;
}
static V3 m3_vec(const double a[3][3], V3 v) {  // gemv order
  double y[3];
  for (int i = 0; i < 3; i++) y[i] = (1.0 * a[i][0]) * v.x;
  for (int i = 0; i < 3; i++) y[i] = (1.0 * a[i][1]) * v.y + 1.0 * y[i];
  for (int i = 0; i < 3; i++) y[i] = (1.0 * a[i][2]) * v.z + 1.0 * y[i];
  return {y[0], y[1], y[2]};
}
// Rotation3::from_euler_angles(roll, pitch, yaw).to_homogeneous()
static M4 m4_euler(double roll, double pitch, double yaw) {
  double sr = std::sin(roll), cr = std::cos(roll);
  double sp = std::sin(pitch), cp = std::cos(pitch);
  double sy = std::sin(yaw), cy = std::cos(yaw);
  M4 r = m4_identity();
  r.m[0][0] = cy * cp;
  r.m[0][1] = cy * sp * sr - sy * cr;
  r.m[0][2] = cy * sp * cr + sy * sr;
  r.m[1][0] = sy * cp;
  r.m[1][1] = sy * sp * sr + cy * cr;
  r.m[1][2] = sy * sp * cr - cy * sr;
  r.m[2][0] = -sp;
  r.m[2][1] = cp * sr;
  r.m[2][2] = cp * cr;
  return r;
}

// ---------------------------------------------------------------------------
// rand 0.8 StdRng (ChaCha12, 64-bit counter, stream 0) + rand_core 0.6
// seed_from_u64 (PCG32 expansion); rand's Standard f64 and
// UniformFloat::sample_single.
// ---------------------------------------------------------------------------
static inline uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }
static void chacha12_block(const uint32_t key[8], uint64_t counter, uint32_t out[16]) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                    key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                    (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u};
  uint32_t x[16];
  memcpy(x, s, sizeof x);
#define QR(a, b, c, d)           \
  x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 16); \
  x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 12); \
  x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 8);  \
  x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 7);
  for (int r = 0; r < 6; r++) {
    QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
    QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
  }
#undef QR
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}
static inline uint32_t pcg32_step(uint64_t& state) {
  const uint64_t MUL = 6364136223846793005ULL;
  const uint64_t INC = 11634580027462260723ULL;
  state = state * MUL + INC;
  uint64_t s = state;
  uint32_t xorshifted = (uint32_t)(((s >> 18) ^ s) >> 27);
  uint32_t rot = (uint32_t)(s >> 59);
  return (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
}

struct StdRng {
  uint32_t key[8];
  uint64_t counter = 0;  // next block to generate
  uint32_t buf[64];
  int idx = 64;
  explicit StdRng(uint64_t seed) {
    uint64_t st = seed;
    for (int i = 0; i < 8; i++) key[i] = pcg32_step(st);
  }
  void refill() {  // rand_chacha fills four consecutive blocks at a time
    for (int b = 0; b < 4; b++) chacha12_block(key, counter + b, buf + 16 * b);
    counter += 4;
  }
  uint32_t next_u32() {
    if (idx >= 64) { refill(); idx = 0; }
    return buf[idx++];
  }
  // rand_core BlockRng::next_u64
  uint64_t next_u64() {
    if (idx < 63) {
      uint64_t lo = buf[idx], hi = buf[idx + 1];
      idx += 2;
      return (hi << 32) | lo;
    } else if (idx >= 64) {
      refill();
      idx = 2;
      return ((uint64_t)buf[1] << 32) | buf[0];
    } else {
      uint64_t x = buf[63];
      refill();
      idx = 1;
      uint64_t y = buf[0];
      return (y << 32) | x;
    }
  }
  // Standard distribution for f64: (u64 >> 11) * 2^-53
  double gen_f64() {
    const double scale = 1.0 / (double)(1ULL << 53);
    uint64_t v = next_u64() >> 11;
    return scale * (double)v;
  }
  // Rng::gen_range(low..high) for f64
  double gen_range(double low, double high) {
    if (!(low < high)) throw Err("cannot sample empty range");
    double scale = high - low;
    if (!std::isfinite(scale)) throw Err("UniformSampler::sample_single: range overflow");
    for (;;) {
      uint64_t bits = next_u64() >> 12;
      uint64_t fb = (1023ULL << 52) | bits;
      double v12;
      memcpy(&v12, &fb, 8);
      double v01 = v12 - 1.0;
      double res = v01 * scale + low;
      if (res < high) return res;
      if (!(std::isfinite(low) && std::isfinite(high)))
        throw Err("Uniform::sample_single: low and high must be finite");
      uint64_t sb;
      memcpy(&sb, &scale, 8);
      sb -= 1;
      memcpy(&scale, &sb, 8);
    }
  }
};

// ---------------------------------------------------------------------------
// JSON reader with serde_json's default number semantics
// ---------------------------------------------------------------------------
struct JVal {
  enum Kind { NUL, BOOL, U64, I64, F64, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  uint64_t u = 0;
  int64_t i = 0;
  double d = 0;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal* get(const char* k) const {
    for (auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

static const double POW10[] = {
    1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
    1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22, 1e23, 1e24, 1e25, 1e26, 1e27, 1e28, 1e29,
    1e30, 1e31, 1e32, 1e33, 1e34, 1e35, 1e36, 1e37, 1e38, 1e39, 1e40, 1e41, 1e42, 1e43,
    1e44, 1e45, 1e46, 1e47, 1e48, 1e49, 1e50, 1e51, 1e52, 1e53, 1e54, 1e55, 1e56, 1e57,
    1e58, 1e59, 1e60, 1e61, 1e62, 1e63, 1e64, 1e65, 1e66, 1e67, 1e68, 1e69, 1e70, 1e71,
    1e72, 1e73, 1e74, 1e75, 1e76, 1e77, 1e78, 1e79, 1e80, 1e81, 1e82, 1e83, 1e84, 1e85,
    1e86, 1e87, 1e88, 1e89, 1e90, 1e91, 1e92, 1e93, 1e94, 1e95, 1e96, 1e97, 1e98, 1e99,
    1e100, 1e101, 1e102, 1e103, 1e104, 1e105, 1e106, 1e107, 1e108, 1e109, 1e110, 1e111,
    1e112, 1e113, 1e114, 1e115, 1e116, 1e117, 1e118, 1e119, 1e120, 1e121, 1e122, 1e123,
    1e124, 1e125, 1e126, 1e127, 1e128, 1e129, 1e130, 1e131, 1e132, 1e133, 1e134, 1e135,
    1e136, 1e137, 1e138, 1e139, 1e140, 1e141, 1e142, 1e143, 1e144, 1e145, 1e146, 1e147,
    1e148, 1e149, 1e150, 1e151, 1e152, 1e153, 1e154, 1e155, 1e156, 1e157, 1e158, 1e159,
    1e160, 1e161, 1e162, 1e163, 1e164, 1e165, 1e166, 1e167, 1e168, 1e169, 1e170, 1e171,
    1e172, 1e173, 1e174, 1e175, 1e176, 1e177, 1e178, 1e179, 1e180, 1e181, 1e182, 1e183,
    1e184, 1e185, 1e186, 1e187, 1e188, 1e189, 1e190, 1e191, 1e192, 1e193, 1e194, 1e195,
    1e196, 1e197, 1e198, 1e199, 1e200, 1e201, 1e202, 1e203, 1e204, 1e205, 1e206, 1e207,
    1e208, 1e209, 1e210, 1e211, 1e212, 1e213, 1e214, 1e215, 1e216, 1e217, 1e218, 1e219,
    1e220, 1e221, 1e222, 1e223, 1e224, 1e225, 1e226, 1e227, 1e228, 1e229, 1e230, 1e231,
    1e232, 1e233, 1e234, 1e235, 1e236, 1e237, 1e238, 1e239, 1e240, 1e241, 1e242, 1e243,
    1e244, 1e245, 1e246, 1e247, 1e248, 1e249, 1e250, 1e251, 1e252, 1e253, 1e254, 1e255,
    1e256, 1e257, 1e258, 1e259, 1e260, 1e261, 1e262, 1e263, 1e264, 1e265, 1e266, 1e267,
    1e268, 1e269, 1e270, 1e271, 1e272, 1e273, 1e274, 1e275, 1e276, 1e277, 1e278, 1e279,
    1e280, 1e281, 1e282, 1e283, 1e284, 1e285, 1e286, 1e287, 1e288, 1e289, 1e290, 1e291,
    1e292, 1e293, 1e294, 1e295, 1e296, 1e297, 1e298, 1e299, 1e300, 1e301, 1e302, 1e303,
    1e304, 1e305, 1e306, 1e307, 1e308};

struct JParser {
  const char* p;
  const char* end;
  [[noreturn]] void fail(const char* m) { throw Err(std::string("JSON parse error: ") + m); }
  void ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
  }
  int peek() { return p < end ? (unsigned char)*p : 0; }
  // serde_json f64_from_parts (default feature set)
  double from_parts(bool positive, uint64_t sig, int exponent) {
    double f = (double)sig;
    for (;;) {
      unsigned ae = (unsigned)(exponent < 0 ? -(int64_t)exponent : exponent);
      if (ae <= 308) {
        double pw = POW10[ae];
        if (exponent >= 0) {
          f *= pw;
          if (std::isinf(f)) fail("number out of range");
        } else {
          f /= pw;
        }
        break;
      }
      if (f == 0.0) break;
      if (exponent >= 0) fail("number out of range");
      f /= 1e308;
      exponent += 308;
    }
    return positive ? f : -f;
  }
  static bool ovf(uint64_t a, uint64_t b, uint64_t c) { return a >= c / 10 && (a > c / 10 || b > c % 10); }
  double parse_exponent(bool positive, uint64_t sig, int starting) {
    p++;  // e/E
    bool pos_exp = true;
    if (peek() == '+') { p++; } else if (peek() == '-') { p++; pos_exp = false; }
    if (!(peek() >= '0' && peek() <= '9')) fail("invalid number");
    int64_t e = *p++ - '0';
    while (peek() >= '0' && peek() <= '9') {
      int d = *p++ - '0';
      if (e >= INT32_MAX / 10 && (e > INT32_MAX / 10 || d > INT32_MAX % 10)) {
        while (peek() >= '0' && peek() <= '9') p++;
        if (sig == 0 || !pos_exp) return positive ? 0.0 : -0.0;
        fail("number out of range");
      }
      e = e * 10 + d;
    }
    int64_t fe = pos_exp ? (int64_t)starting + e : (int64_t)starting - e;
    if (fe > INT32_MAX) fe = INT32_MAX;
    if (fe < INT32_MIN) fe = INT32_MIN;
    return from_parts(positive, sig, (int)fe);
  }
  double parse_decimal(bool positive, uint64_t sig, int exp_before) {
    p++;  // '.'
    int exp_after = 0;
    while (peek() >= '0' && peek() <= '9') {
      uint64_t d = *p - '0';
      if (ovf(sig, d, UINT64_MAX)) {
        while (peek() >= '0' && peek() <= '9') p++;
        int e = exp_before + exp_after;
        if (peek() == 'e' || peek() == 'E') return parse_exponent(positive, sig, e);
        return from_parts(positive, sig, e);
      }
      p++;
      sig = sig * 10 + d;
      exp_after -= 1;
    }
    if (exp_after == 0) fail("invalid number");
    int e = exp_before + exp_after;
    if (peek() == 'e' || peek() == 'E') return parse_exponent(positive, sig, e);
    return from_parts(positive, sig, e);
  }
  void parse_number(JVal& v) {
    bool positive = true;
    if (peek() == '-') { positive = false; p++; }
    if (!(peek() >= '0' && peek() <= '9')) fail("invalid number");
    uint64_t sig = 0;
    if (peek() == '0') {
      p++;
      if (peek() >= '0' && peek() <= '9') fail("invalid number");
    } else {
      sig = *p++ - '0';
      while (peek() >= '0' && peek() <= '9') {
        uint64_t d = *p - '0';
        if (ovf(sig, d, UINT64_MAX)) {
          // parse_long_integer: count the remaining integer digits as
          // powers of ten
          int exponent = 0;
          while (peek() >= '0' && peek() <= '9') { p++; exponent++; }
          v.kind = JVal::F64;
          if (peek() == '.') { v.d = parse_decimal(positive, sig, exponent); return; }
          if (peek() == 'e' || peek() == 'E') { v.d = parse_exponent(positive, sig, exponent); return; }
          v.d = from_parts(positive, sig, exponent);
          return;
        }
        p++;
        sig = sig * 10 + d;
      }
    }
    if (peek() == '.') { v.kind = JVal::F64; v.d = parse_decimal(positive, sig, 0); return; }
    if (peek() == 'e' || peek() == 'E') { v.kind = JVal::F64; v.d = parse_exponent(positive, sig, 0); return; }
    if (positive) { v.kind = JVal::U64; v.u = sig; return; }
    int64_t neg = (int64_t)(0 - sig);
    if (neg >= 0) { v.kind = JVal::F64; v.d = -(double)sig; return; }
    v.kind = JVal::I64;
    v.i = neg;
  }
  static void put_utf8(std::string& out, uint32_t cp) {
    if (cp < 0x80) out += (char)cp;
    else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
    else if (cp < 0x10000) {
      out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F));
    } else {
      out += (char)(0xF0 | (cp >> 18)); out += (char)(0x80 | ((cp >> 12) & 0x3F));
      out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F));
    }
  }
  uint32_t hex4() {
    if (end - p < 4) fail("EOF while parsing a string");
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) {
      char c = *p++;
      v <<= 4;
      if (c >= '0' && c <= '9') v |= c - '0';
      else if (c >= 'a' && c <= 'f') v |= c - 'a' + 10;
      else if (c >= 'A' && c <= 'F') v |= c - 'A' + 10;
      else fail("invalid escape");
    }
    return v;
  }
  std::string parse_string() {
    p++;  // opening quote
    std::string out;
    for (;;) {
      if (p >= end) fail("EOF while parsing a string");
      char c = *p++;
      if (c == '"') return out;
      if ((unsigned char)c < 0x20) fail("control character in string");
      if (c != '\\') { out += c; continue; }
      if (p >= end) fail("EOF while parsing a string");
      char e = *p++;
      switch (e) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          uint32_t cp = hex4();
          if (cp >= 0xD800 && cp < 0xDC00) {
            if (end - p >= 2 && p[0] == '\\' && p[1] == 'u') {
              p += 2;
              uint32_t lo = hex4();
              cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
            } else fail("lone leading surrogate");
          }
          put_utf8(out, cp);
          break;
        }
        default: fail("invalid escape");
      }
    }
  }
  void parse_value(JVal& v, int depth) {
    if (depth > 128) fail("recursion limit exceeded");
    ws();
    int c = peek();
    if (c == '{') {
      p++;
      v.kind = JVal::OBJ;
      ws();
      if (peek() == '}') { p++; return; }
      for (;;) {
        ws();
        if (peek() != '"') fail("key must be a string");
        std::string k = parse_string();
        ws();
        if (peek() != ':') fail("expected `:`");
        p++;
        v.obj.emplace_back(k, JVal());
        parse_value(v.obj.back().second, depth + 1);
        ws();
        if (peek() == ',') { p++; continue; }
        if (peek() == '}') { p++; return; }
        fail("expected `,` or `}`");
      }
    } else if (c == '[') {
      p++;
      v.kind = JVal::ARR;
      ws();
      if (peek() == ']') { p++; return; }
      for (;;) {
        v.arr.emplace_back();
        parse_value(v.arr.back(), depth + 1);
        ws();
        if (peek() == ',') { p++; continue; }
        if (peek() == ']') { p++; return; }
        fail("expected `,` or `]`");
      }
    } else if (c == '"') {
      v.kind = JVal::STR;
      v.s = parse_string();
    } else if (c == 't' && end - p >= 4 && !strncmp(p, "true", 4)) {
      p += 4; v.kind = JVal::BOOL; v.b = true;
    } else if (c == 'f' && end - p >= 5 && !strncmp(p, "false", 5)) {
      p += 5; v.kind = JVal::BOOL; v.b = false;
    } else if (c == 'n' && end - p >= 4 && !strncmp(p, "null", 4)) {
      p += 4; v.kind = JVal::NUL;
    } else if (c == '-' || (c >= '0' && c <= '9')) {
      parse_number(v);
    } else {
      fail("expected value");
    }
  }
};

static JVal parse_json(const std::string& text) {
  JParser ps{text.data(), text.data() + text.size()};
  JVal v;
  ps.parse_value(v, 0);
  ps.ws();
  if (ps.p != ps.end) ps.fail("trailing characters");
  return v;
}

// serde field access helpers
static const JVal& req(const JVal& o, const char* k) {
  const JVal* v = o.get(k);
  if (!v) throw Err(std::string("missing field `") + k + "`");
  return *v;
}
static const JVal* opt(const JVal& o, const char* k) {
  const JVal* v = o.get(k);
  if (!v || v->kind == JVal::NUL) return nullptr;
  return v;
}
static double as_f64(const JVal& v) {
  switch (v.kind) {
    case JVal::U64: return (double)v.u;
    case JVal::I64: return (double)v.i;
    case JVal::F64: return v.d;
    default: throw Err("invalid type: expected f64");
  }
}
static std::string as_str(const JVal& v) {
  if (v.kind != JVal::STR) throw Err("invalid type: expected a string");
  return v.s;
}
static bool as_bool(const JVal& v) {
  if (v.kind != JVal::BOOL) throw Err("invalid type: expected a boolean");
  return v.b;
}
static V3 as_v3(const JVal& v) {
  if (v.kind != JVal::ARR) throw Err("invalid type: expected an array of length 3");
  if (v.arr.size() != 3) throw Err("invalid length, expected an array of length 3");
  return v3(as_f64(v.arr[0]), as_f64(v.arr[1]), as_f64(v.arr[2]));
}

// ---------------------------------------------------------------------------
// Scene model (src/scene.rs:15-458)
// ---------------------------------------------------------------------------
// hex_to_color (src/scene.rs:15-30)
static bool parse_u8_radix16(const std::string& s, uint8_t* out) {
  // u8::from_str_radix accepts an optional leading '+'
  size_t i = 0;
  if (s.size() > 1 && s[0] == '+') i = 1;
  if (i >= s.size()) return false;
  unsigned v = 0;
  for (; i < s.size(); i++) {
    char c = s[i];
    int d;
    if (c >= '0' && c <= '9') d = c - '0';
    else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
    else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
    else return false;
    v = v * 16 + d;
    if (v > 255) return false;
  }
  *out = (uint8_t)v;
  return true;
}
static bool hex_to_color(const std::string& in, V3* out, std::string* err) {
  size_t k = 0;
  while (k < in.size() && in[k] == '#') k++;
  std::string hex = in.substr(k);
  if (hex.size() != 6) { if (err) *err = "Invalid hex color format"; return false; }
  // slicing at byte offsets 0..2, 2..4, 4..6 requires char boundaries
  for (int b : {2, 4})
    if (((unsigned char)hex[b] & 0xC0) == 0x80) { if (err) *err = "Invalid hex color"; return false; }
  uint8_t r, g, b;
  if (!parse_u8_radix16(hex.substr(0, 2), &r) || !parse_u8_radix16(hex.substr(2, 2), &g) ||
      !parse_u8_radix16(hex.substr(4, 2), &b)) {
    if (err) *err = "Invalid hex color";
    return false;
  }
  *out = v3((double)r / 255.0, (double)g / 255.0, (double)b / 255.0);
  return true;
}
static V3 hex_or(const std::string& s, V3 fallback) {
  V3 c;
  return hex_to_color(s, &c, nullptr) ? c : fallback;
}
static V3 hex_req(const std::string& s) {
  V3 c;
  std::string e;
  if (!hex_to_color(s, &c, &e)) throw Err(e);
  return c;
}

struct Material {
  std::string color = "#FFFFFF";
  double ambient = 0.1, diffuse = 0.7, specular = 0.3, shininess = 32.0;
  bool has_reflectivity = false;
  double reflectivity = 0.0;
  int texture = 0;  // 0 none, 1 grid, 2 checkerboard
  std::string line_color;
  double line_width = 0, cell_size = 0;
  std::shared_ptr<Material> material_b;
};

static Material parse_material(const JVal& j) {
  if (j.kind != JVal::OBJ) throw Err("invalid type: expected struct Material");
  Material m;
  m.color = as_str(req(j, "color"));
  m.ambient = as_f64(req(j, "ambient"));
  m.diffuse = as_f64(req(j, "diffuse"));
  m.specular = as_f64(req(j, "specular"));
  m.shininess = as_f64(req(j, "shininess"));
  if (const JVal* r = opt(j, "reflectivity")) { m.has_reflectivity = true; m.reflectivity = as_f64(*r); }
  if (const JVal* t = opt(j, "texture")) {
    const JVal& ty = req(*t, "type");
    std::string tn = as_str(ty);
    if (tn == "grid") {
      m.texture = 1;
      m.line_color = as_str(req(*t, "line_color"));
      m.line_width = as_f64(req(*t, "line_width"));
      m.cell_size = as_f64(req(*t, "cell_size"));
    } else if (tn == "checkerboard") {
      m.texture = 2;
      m.material_b = std::make_shared<Material>(parse_material(req(*t, "material_b")));
    } else {
      throw Err("unknown variant `" + tn + "`, expected `grid` or `checkerboard`");
    }
  }
  return m;
}

// Transform::from_str (src/scene.rs:117-165)
static bool parse_f64_rust(const std::string& s, double* out) {
  // Rust f64::from_str: decimal or inf/nan literals; no leading/trailing
  // whitespace (the caller trims).  Correctly rounded.
  if (s.empty()) return false;
  std::string t = s;
  size_t i = 0;
  if (t[0] == '+' || t[0] == '-') i = 1;
  std::string body = t.substr(i);
  std::string lower;
  for (char c : body) lower += (char)tolower((unsigned char)c);
  if (lower == "inf" || lower == "infinity" || lower == "nan") {
    double v = (lower == "nan") ? NAN : INF;
    *out = (t[0] == '-') ? -v : v;
    return true;
  }
  bool digits = false, dot = false, exp = false;
  for (size_t k = 0; k < body.size(); k++) {
    char c = body[k];
    if (c >= '0' && c <= '9') digits = true;
    else if (c == '.' && !dot && !exp) dot = true;
    else if ((c == 'e' || c == 'E') && digits && !exp) {
      exp = true;
      if (k + 1 < body.size() && (body[k + 1] == '+' || body[k + 1] == '-')) k++;
      if (k + 1 >= body.size()) return false;
    } else return false;
  }
  if (!digits) return false;
  char* e2 = nullptr;
  *out = strtod(t.c_str(), &e2);
  return e2 && *e2 == 0;
}
static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}
static M4 transform_matrix(const std::string& in) {
  std::string s = trim(in);
  const char* kinds[3] = {"rotate(", "translate(", "scale("};
  for (int k = 0; k < 3; k++) {
    size_t n = strlen(kinds[k]);
    if (s.compare(0, n, kinds[k]) != 0) continue;
    std::string params = s.substr(n);
    if (params.empty() || params.back() != ')') throw Err("Missing closing parenthesis");
    params.pop_back();
    std::vector<double> vals;
    size_t st = 0;
    for (;;) {
      size_t c = params.find(',', st);
      std::string part = trim(params.substr(st, c == std::string::npos ? std::string::npos : c - st));
      double v;
      if (!parse_f64_rust(part, &v)) throw Err("Invalid transform parameters");
      vals.push_back(v);
      if (c == std::string::npos) break;
      st = c + 1;
    }
    if (vals.size() != 3) throw Err("Transform requires exactly 3 parameters (x, y, z)");
    if (k == 0) {
      // to_matrix: rz * ry * rx with from_euler_angles
      double xr = to_radians(vals[0]), yr = to_radians(vals[1]), zr = to_radians(vals[2]);
      M4 rx = m4_euler(xr, 0.0, 0.0), ry = m4_euler(0.0, yr, 0.0), rz = m4_euler(0.0, 0.0, zr);
      return m4_mul(m4_mul(rz, ry), rx);
    }
    M4 r = m4_identity();
    if (k == 1) { r.m[0][3] = vals[0]; r.m[1][3] = vals[1]; r.m[2][3] = vals[2]; }
    else { r.m[0][0] = vals[0]; r.m[1][1] = vals[1]; r.m[2][2] = vals[2]; }
    return r;
  }
  throw Err("Unknown transform type. Expected rotate(), translate(), or scale(), got: " + s);
}
// parse_transforms (src/scene.rs:191-203): later transforms multiply from the left
static bool parse_transforms(const std::vector<std::string>& ts, M4* out) {
  M4 comb = m4_identity();
  try {
    for (auto& t : ts) comb = m4_mul(transform_matrix(t), comb);
  } catch (const Err&) {
    return false;
  }
  *out = comb;
  return true;
}

// ---------------------------------------------------------------------------
// Mesh, STL and k-d tree (src/mesh.rs)
// ---------------------------------------------------------------------------
struct Triangle {
  V3 v[3];
  V3 normal;
  // center (src/mesh.rs:21-23): (v0 + v1 + v2) / 3
  V3 center() const { return (v[0] + v[1] + v[2]) / 3.0; }
  void bounds(V3* mn, V3* mx) const {  // src/mesh.rs:26-36 (inf / sup)
    *mn = v[0];
    *mx = v[0];
    for (int k = 1; k < 3; k++) {
      *mn = v3(rmin(mn->x, v[k].x), rmin(mn->y, v[k].y), rmin(mn->z, v[k].z));
      *mx = v3(rmax(mx->x, v[k].x), rmax(mx->y, v[k].y), rmax(mx->z, v[k].z));
    }
  }
};

struct KdNode {
  bool leaf = false;
  int axis = 0;
  double split = 0;
  std::unique_ptr<KdNode> left, right;
  std::vector<size_t> tris;
  V3 bmin, bmax;
};

struct KdTree {
  std::unique_ptr<KdNode> root;
  size_t max_depth = 16, max_leaf = 10;

  static void compute_bounds(const std::vector<Triangle>& t, const std::vector<size_t>& idx, V3* mn, V3* mx) {
    if (idx.empty()) { *mn = v3(0, 0, 0); *mx = v3(0, 0, 0); return; }
    *mn = v3(INF, INF, INF);
    *mx = v3(-INF, -INF, -INF);
    for (size_t i : idx) {
      V3 a, b;
      t[i].bounds(&a, &b);
      *mn = v3(rmin(mn->x, a.x), rmin(mn->y, a.y), rmin(mn->z, a.z));
      *mx = v3(rmax(mx->x, b.x), rmax(mx->y, b.y), rmax(mx->z, b.z));
    }
  }
  // build_recursive (src/mesh.rs:125-197)
  std::unique_ptr<KdNode> build(const std::vector<Triangle>& t, std::vector<size_t> idx, V3 bmin, V3 bmax,
                                size_t depth) {
    auto n = std::make_unique<KdNode>();
    n->bmin = bmin;
    n->bmax = bmax;
    if (depth >= max_depth || idx.size() <= max_leaf) {
      n->leaf = true;
      n->tris = std::move(idx);
      return n;
    }
    int axis = (int)(depth % 3);
    std::vector<std::pair<double, size_t>> pos;
    pos.reserve(idx.size());
    for (size_t i : idx) pos.emplace_back(t[i].center()[axis], i);
    for (auto& pr : pos)
      if (std::isnan(pr.first)) throw Err("called `Option::unwrap()` on a `None` value");
    std::stable_sort(pos.begin(), pos.end(),
                     [](const std::pair<double, size_t>& a, const std::pair<double, size_t>& b) {
                       return a.first < b.first;
                     });
    double split = pos[pos.size() / 2].first;
    std::vector<size_t> l, r;
    for (auto& pr : pos) {
      V3 mn, mx;
      t[pr.second].bounds(&mn, &mx);
      if (mn[axis] <= split) l.push_back(pr.second);
      if (mx[axis] > split) r.push_back(pr.second);
    }
    if (l.empty()) { l.push_back(r.back()); r.pop_back(); }
    else if (r.empty()) { r.push_back(l.back()); l.pop_back(); }
    V3 lmin, lmax, rmin_, rmax_;
    compute_bounds(t, l, &lmin, &lmax);
    compute_bounds(t, r, &rmin_, &rmax_);
    n->axis = axis;
    n->split = split;
    n->left = build(t, std::move(l), lmin, lmax, depth + 1);
    n->right = build(t, std::move(r), rmin_, rmax_, depth + 1);
    return n;
  }
  void construct(const std::vector<Triangle>& t) {
    root.reset();
    if (t.empty()) return;
    std::vector<size_t> idx(t.size());
    for (size_t i = 0; i < t.size(); i++) idx[i] = i;
    V3 mn, mx;
    compute_bounds(t, idx, &mn, &mx);
    root = build(t, std::move(idx), mn, mx, 0);
  }
  // ray_intersects_bounds (src/mesh.rs:218-255)
  static bool ray_hits_bounds(V3 o, V3 d, V3 mn, V3 mx) {
    double tmin = -INF, tmax = INF;
    for (int a = 0; a < 3; a++) {
      if (std::fabs(d[a]) < 1e-9) {
        if (o[a] < mn[a] || o[a] > mx[a]) return false;
      } else {
        double inv = 1.0 / d[a];
        double t0 = (mn[a] - o[a]) * inv;
        double t1 = (mx[a] - o[a]) * inv;
        if (t0 > t1) std::swap(t0, t1);
        tmin = rmax(tmin, t0);
        tmax = rmin(tmax, t1);
        if (tmin > tmax) return false;
      }
    }
    return tmax >= 0.0;
  }
  // traverse_recursive (src/mesh.rs:399-465)
  template <class F>
  void traverse(const KdNode* n, V3 o, V3 d, F& cb, uint64_t* visits) const {
    if (visits) (*visits)++;
    if (n->leaf) {
      if (ray_hits_bounds(o, d, n->bmin, n->bmax)) cb(n->tris);
      return;
    }
    double op = o[n->axis], dir = d[n->axis];
    if (std::fabs(dir) < 1e-9) {
      if (op <= n->split) traverse(n->left.get(), o, d, cb, visits);
      else traverse(n->right.get(), o, d, cb, visits);
      return;
    }
    double ts = (n->split - op) / dir;
    if (op <= n->split) {
      traverse(n->left.get(), o, d, cb, visits);
      if (ts >= 0.0) traverse(n->right.get(), o, d, cb, visits);
    } else {
      traverse(n->right.get(), o, d, cb, visits);
      if (ts >= 0.0) traverse(n->left.get(), o, d, cb, visits);
    }
  }
};

struct Mesh {
  std::vector<Triangle> tris;
  V3 bmin{INF, INF, INF}, bmax{-INF, -INF, -INF};
  KdTree kd;
  void add(const Triangle& t) {  // add_triangle (src/mesh.rs:1006-1014)
    for (int k = 0; k < 3; k++) {
      bmin = v3(rmin(bmin.x, t.v[k].x), rmin(bmin.y, t.v[k].y), rmin(bmin.z, t.v[k].z));
      bmax = v3(rmax(bmax.x, t.v[k].x), rmax(bmax.y, t.v[k].y), rmax(bmax.z, t.v[k].z));
    }
    tris.push_back(t);
  }
  void compute_bounds() {  // src/mesh.rs:1017-1033
    if (tris.empty()) { bmin = v3(0, 0, 0); bmax = v3(0, 0, 0); return; }
    bmin = v3(INF, INF, INF);
    bmax = v3(-INF, -INF, -INF);
    for (auto& t : tris)
      for (int k = 0; k < 3; k++) {
        bmin = v3(rmin(bmin.x, t.v[k].x), rmin(bmin.y, t.v[k].y), rmin(bmin.z, t.v[k].z));
        bmax = v3(rmax(bmax.x, t.v[k].x), rmax(bmax.y, t.v[k].y), rmax(bmax.z, t.v[k].z));
      }
  }
  void build_kdtree() { kd.construct(tris); }
};

// STL parsing (src/mesh.rs:751-1003)
static std::vector<std::string> split_lines(const std::string& s) {
  // str::lines: split on \n, strip a trailing \r
  std::vector<std::string> out;
  size_t st = 0;
  while (st < s.size()) {
    size_t e = s.find('\n', st);
    std::string line = s.substr(st, e == std::string::npos ? std::string::npos : e - st);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    out.push_back(line);
    if (e == std::string::npos) break;
    st = e + 1;
  }
  return out;
}
static std::vector<std::string> split_ws(const std::string& s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}
static bool starts_with(const std::string& s, const char* p) { return s.compare(0, strlen(p), p) == 0; }
static std::string trim_start(const std::string& s) {
  size_t a = 0;
  while (a < s.size() && isspace((unsigned char)s[a])) a++;
  return s.substr(a);
}
static bool is_ascii_stl(const std::string& bytes) {
  auto lines = split_lines(bytes);
  for (size_t i = 0; i < lines.size() && i < 10; i++) {
    std::string t = trim(lines[i]);
    if (starts_with(t, "facet normal") || t == "outer loop" || t == "endloop") return true;
  }
  return false;
}
static double parse_f64_req(const std::string& s) {
  double v;
  if (!parse_f64_rust(s, &v)) throw Err("invalid float literal");
  return v;
}
static Mesh load_ascii_stl(const std::string& bytes) {
  auto lines = split_lines(bytes);
  Mesh m;
  size_t i = 0;
  while (i < lines.size()) {
    std::string line = trim(lines[i]);
    if (starts_with(line, "facet normal")) {
      auto parts = split_ws(line);
      if (parts.size() != 5) throw Err("Invalid facet normal format");
      Triangle t;
      t.normal = v3(parse_f64_req(parts[2]), parse_f64_req(parts[3]), parse_f64_req(parts[4]));
      i++;
      if (i >= lines.size() || trim(lines[i]) != "outer loop") throw Err("Expected 'outer loop' after facet normal");
      for (int j = 0; j < 3; j++) {
        i++;
        if (i >= lines.size()) throw Err("Unexpected end of file while reading vertex");
        std::string vl = trim(lines[i]);
        if (!starts_with(vl, "vertex")) throw Err("Expected vertex line");
        auto vp = split_ws(vl);
        if (vp.size() != 4) throw Err("Invalid vertex format");
        t.v[j] = v3(parse_f64_req(vp[1]), parse_f64_req(vp[2]), parse_f64_req(vp[3]));
      }
      i++;
      if (i >= lines.size() || trim(lines[i]) != "endloop") throw Err("Expected 'endloop'");
      i++;
      if (i >= lines.size() || trim(lines[i]) != "endfacet") throw Err("Expected 'endfacet'");
      m.add(t);
    }
    i++;
  }
  m.compute_bounds();
  m.build_kdtree();
  return m;
}
static float le_f32(const unsigned char* b) {
  float f;
  uint32_t u = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
  memcpy(&f, &u, 4);
  return f;
}
static Mesh load_binary_stl(const std::string& bytes) {
  if (bytes.size() < 84) throw Err("Binary STL too short");
  const unsigned char* b = (const unsigned char*)bytes.data();
  size_t n = (size_t)b[80] | ((size_t)b[81] << 8) | ((size_t)b[82] << 16) | ((size_t)b[83] << 24);
  size_t expected = 84 + n * 50;
  if (bytes.size() < expected)
    throw Err("Binary STL size mismatch: expected " + std::to_string(expected) + ", got " + std::to_string(bytes.size()));
  Mesh m;
  size_t off = 84;
  for (size_t k = 0; k < n; k++) {
    Triangle t;
    t.normal = v3((double)le_f32(b + off), (double)le_f32(b + off + 4), (double)le_f32(b + off + 8));
    off += 12;
    for (int i = 0; i < 3; i++) {
      t.v[i] = v3((double)le_f32(b + off), (double)le_f32(b + off + 4), (double)le_f32(b + off + 8));
      off += 12;
    }
    off += 2;
    m.add(t);
  }
  m.compute_bounds();
  m.build_kdtree();
  return m;
}
static Mesh mesh_from_stl_bytes(const std::string& bytes) {  // from_stl_file / from_stl_bytes
  if (bytes.size() < 80) throw Err("failed to fill whole buffer");
  std::string header = bytes.substr(0, 80);
  if (starts_with(trim_start(header), "solid") && is_ascii_stl(bytes)) return load_ascii_stl(bytes);
  return load_binary_stl(bytes);
}
static std::string read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw Err("No such file or directory (os error 2): " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

// Scene description (src/scene.rs:311-458)
struct Light {
  V3 position;
  std::string color;
  double intensity = 1;
  bool has_diameter = false;
  double diameter = 0;
};
struct Fog {
  std::string color;
  double density, start, end;
};
struct Outline {
  bool enabled = false;
  double depth_weight = 1, normal_weight = 1, threshold = 0.1;
  std::string color = "#000000";
  double thickness = 1;
  bool use_8 = false;
};
struct CameraCfg {
  std::string kind;
  V3 position, target, up;
  double width = 10, height = 10;
  bool has_fov = false;
  double fov = 45;
  bool has_pitch = false, has_grid_color = false, has_thickness = false;
  double grid_pitch = 0, grid_thickness = 0;
  std::string grid_color;
};
struct SceneObject {
  int kind;  // 0 sphere 1 plane 2 cube 3 mesh
  V3 a, b;   // sphere: center,(radius in r); plane: point, normal; cube: center, size
  double radius = 0;
  Material material;
  bool has_transform = false;
  std::vector<std::string> transform;
  std::string filename;
  std::shared_ptr<Mesh> mesh;
};
struct Scene {
  CameraCfg camera;
  std::vector<SceneObject> objects;
  std::vector<Light> lights;
  std::string ambient_color;
  double ambient_intensity = 0.1;
  bool has_fog = false;
  Fog fog;
  bool has_background = false;
  std::string background;
  bool has_outline = false;
  Outline outline;
};

static Scene parse_scene(const std::string& text, const std::string& base_dir) {
  JVal j = parse_json(text);
  if (j.kind != JVal::OBJ) throw Err("invalid type: expected struct Scene");
  Scene s;
  const JVal& cam = req(j, "camera");
  if (cam.kind != JVal::OBJ) throw Err("invalid type: expected struct Camera");
  s.camera.kind = as_str(req(cam, "kind"));
  s.camera.position = as_v3(req(cam, "position"));
  s.camera.target = as_v3(req(cam, "target"));
  s.camera.up = as_v3(req(cam, "up"));
  s.camera.width = as_f64(req(cam, "width"));
  s.camera.height = as_f64(req(cam, "height"));
  if (const JVal* f = opt(cam, "fov")) { s.camera.has_fov = true; s.camera.fov = as_f64(*f); }
  if (const JVal* f = opt(cam, "grid_pitch")) { s.camera.has_pitch = true; s.camera.grid_pitch = as_f64(*f); }
  if (const JVal* f = opt(cam, "grid_color")) { s.camera.has_grid_color = true; s.camera.grid_color = as_str(*f); }
  if (const JVal* f = opt(cam, "grid_thickness")) { s.camera.has_thickness = true; s.camera.grid_thickness = as_f64(*f); }

  const JVal& objs = req(j, "objects");
  if (objs.kind != JVal::ARR) throw Err("invalid type: expected a sequence");
  for (const JVal& o : objs.arr) {
    if (o.kind != JVal::OBJ) throw Err("invalid type: expected internally tagged enum Object");
    std::string kind = as_str(req(o, "kind"));
    SceneObject so;
    if (kind == "sphere") {
      so.kind = 0;
      so.a = as_v3(req(o, "center"));
      so.radius = as_f64(req(o, "radius"));
    } else if (kind == "plane") {
      so.kind = 1;
      so.a = as_v3(req(o, "point"));
      so.b = as_v3(req(o, "normal"));
    } else if (kind == "cube") {
      so.kind = 2;
      so.a = as_v3(req(o, "center"));
      so.b = as_v3(req(o, "size"));
    } else if (kind == "mesh") {
      so.kind = 3;
      so.transform.clear();
    } else {
      throw Err("unknown variant `" + kind + "`, expected one of `sphere`, `plane`, `cube`, `mesh`");
    }
    so.material = parse_material(req(o, "material"));
    if (const JVal* t = opt(o, "transform")) {
      if (t->kind != JVal::ARR) throw Err("invalid type: expected a sequence");
      so.has_transform = true;
      for (auto& e : t->arr) so.transform.push_back(as_str(e));
    }
    if (kind == "mesh") so.filename = as_str(req(o, "filename"));
    s.objects.push_back(std::move(so));
  }
  const JVal& lights = req(j, "lights");
  if (lights.kind != JVal::ARR) throw Err("invalid type: expected a sequence");
  for (const JVal& l : lights.arr) {
    Light L;
    L.position = as_v3(req(l, "position"));
    L.color = as_str(req(l, "color"));
    L.intensity = as_f64(req(l, "intensity"));
    if (const JVal* d = opt(l, "diameter")) { L.has_diameter = true; L.diameter = as_f64(*d); }
    s.lights.push_back(L);
  }
  const JVal& ss = req(j, "scene_settings");
  const JVal& amb = req(ss, "ambient_illumination");
  s.ambient_color = as_str(req(amb, "color"));
  s.ambient_intensity = as_f64(req(amb, "intensity"));
  if (const JVal* f = opt(ss, "fog")) {
    s.has_fog = true;
    s.fog.color = as_str(req(*f, "color"));
    s.fog.density = as_f64(req(*f, "density"));
    s.fog.start = as_f64(req(*f, "start"));
    s.fog.end = as_f64(req(*f, "end"));
  }
  if (const JVal* b = opt(ss, "background_color")) { s.has_background = true; s.background = as_str(*b); }
  if (const JVal* o = opt(ss, "outline")) {
    s.has_outline = true;
    s.outline.enabled = as_bool(req(*o, "enabled"));
    if (const JVal* v = o->get("depth_weight")) s.outline.depth_weight = as_f64(*v);
    if (const JVal* v = o->get("normal_weight")) s.outline.normal_weight = as_f64(*v);
    if (const JVal* v = o->get("threshold")) s.outline.threshold = as_f64(*v);
    if (const JVal* v = o->get("color")) s.outline.color = as_str(*v);
    if (const JVal* v = o->get("thickness")) s.outline.thickness = as_f64(*v);
    if (const JVal* v = o->get("use_8_neighbors")) s.outline.use_8 = as_bool(*v);
  }
  // load_mesh_data (src/scene.rs:483-505) runs after deserialisation
  for (auto& so : s.objects) {
    if (so.kind != 3) continue;
    const std::string& fn = so.filename;
    std::string path = base_dir.empty() ? fn : (fn.size() && fn[0] == '/' ? fn : base_dir + "/" + fn);
    so.mesh = std::make_shared<Mesh>(mesh_from_stl_bytes(read_file(path)));
  }
  return s;
}

// ---------------------------------------------------------------------------
// Rays, hit records, primitives, world (src/ray.rs)
// ---------------------------------------------------------------------------
struct Ray {
  V3 o, d;
  Ray(V3 origin, V3 dir) : o(origin), d(normalize(dir)) {}  // Ray::new
  V3 at(double t) const { return o + t * d; }
};
struct Hit {
  V3 point, normal;
  double t;
  bool front_face;
  size_t material_index;
  bool has_uv = false;
  double u = 0, v = 0;
};
// HitRecord::new (src/ray.rs:39-64)
static Hit make_hit(V3 p, V3 outward, double t, const Ray& r, size_t mi) {
  Hit h;
  h.point = p;
  h.t = t;
  h.front_face = dot(r.d, outward) < 0.0;
  h.normal = h.front_face ? normalize(outward) : normalize(-outward);
  h.material_index = mi;
  return h;
}

struct Counters {
  std::atomic<uint64_t> primary{0}, reflection{0}, shadow{0}, kd_visits{0}, tri_tests{0}, sphere_tests{0};
};
// Per-thread tallies, added into the shared Counters when a worker finishes
// (keeps the timed CPU baseline free of atomic contention).
struct LocalCounts {
  uint64_t primary = 0, reflection = 0, shadow = 0, kd_visits = 0, tri_tests = 0, sphere_tests = 0;
};
static thread_local LocalCounts tlc;
static void flush_counts(Counters* c) {
  if (!c) return;
  c->primary += tlc.primary;
  c->reflection += tlc.reflection;
  c->shadow += tlc.shadow;
  c->kd_visits += tlc.kd_visits;
  c->tri_tests += tlc.tri_tests;
  c->sphere_tests += tlc.sphere_tests;
  tlc = LocalCounts();
}

struct Object {
  size_t mi;
  virtual ~Object() {}
  virtual bool hit(const Ray& r, double tmin, double tmax, Hit* h, Counters* c) const = 0;
};

struct Sphere : Object {  // src/ray.rs:88-120
  V3 c;
  double r;
  bool hit(const Ray& ray, double tmin, double tmax, Hit* h, Counters* ct) const override {
    if (ct) tlc.sphere_tests++;
    V3 oc = ray.o - c;
    double a = dot(ray.d, ray.d);
    double hb = dot(oc, ray.d);
    double cc = dot(oc, oc) - r * r;
    double disc = hb * hb - a * cc;
    if (disc < 0.0) return false;
    double sq = std::sqrt(disc);
    double root = (-hb - sq) / a;
    if (root < tmin || tmax < root) {
      root = (-hb + sq) / a;
      if (root < tmin || tmax < root) return false;
    }
    V3 p = ray.at(root);
    V3 outward = (p - c) / r;
    *h = make_hit(p, outward, root, ray, mi);
    return true;
  }
};

struct Plane : Object {  // src/ray.rs:135-176
  V3 p, n;
  bool hit(const Ray& ray, double tmin, double tmax, Hit* h, Counters*) const override {
    double denom = dot(n, ray.d);
    if (std::fabs(denom) < 1e-8) return false;
    double t = dot(p - ray.o, n) / denom;
    if (t < tmin || t > tmax) return false;
    V3 pt = ray.at(t);
    *h = make_hit(pt, n, t, ray, mi);
    V3 ua = std::fabs(n.x) > 0.9 ? v3(0, 1, 0) : v3(1, 0, 0);
    V3 uax = normalize(cross(ua, n));
    V3 vax = normalize(cross(n, uax));
    V3 rel = pt - p;
    h->has_uv = true;
    h->u = dot(rel, uax);
    h->v = dot(rel, vax);
    return true;
  }
};

struct Cube : Object {  // src/ray.rs:183-262, 410-491
  V3 c, half;
  M4 w2l, l2w;
  bool identity = true;
  double ntr[3][3];  // inverse-transpose of w2l's rotation part
  void init(V3 center, V3 size, const M4* tm) {
    c = center;
    half = size / 2.0;
    if (!tm) {
      w2l = m4_identity();
      l2w = w2l;
    } else {
      M4 inv;
      if (!m4_try_inverse(*tm, &inv)) inv = m4_identity();
      w2l = inv;
      l2w = *tm;
    }
    identity = m4_is_identity(w2l);
    double rot[3][3], ri[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) rot[i][j] = w2l.m[i][j];
    if (!m3_try_inverse(rot, ri))
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) ri[i][j] = (i == j) ? 1.0 : 0.0;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) ntr[i][j] = ri[j][i];
  }
  bool hit(const Ray& ray, double tmin, double tmax, Hit* h, Counters*) const override {
    V3 lo = m4_vec(w2l, ray.o - c);
    V3 ld = m4_vec(w2l, ray.d);
    if (norm(ld) < 1e-8) return false;
    Ray lr(lo, ld);
    double tminh = tmin, tmaxh = tmax;
    V3 normal = v3(0, 0, 0);
    for (int a = 0; a < 3; a++) {
      double inv = 1.0 / lr.d[a];
      double t0 = (-half[a] - lr.o[a]) * inv;
      double t1 = (half[a] - lr.o[a]) * inv;
      V3 an = v3(0, 0, 0);
      an[a] = inv < 0.0 ? 1.0 : -1.0;
      if (inv < 0.0) {
        std::swap(t0, t1);
        an[a] = -an[a];
      }
      if (t0 > tminh) { tminh = t0; normal = an; }
      if (t1 < tmaxh) tmaxh = t1;
      if (tminh > tmaxh) return false;
    }
    double t = tminh > tmin ? tminh : tmaxh;
    if (t < tmin || t > tmax) return false;
    V3 lhp = lr.at(t);
    V3 whp = c + m4_point(l2w, lhp);
    V3 wn = identity ? normal : m3_vec(ntr, normal);
    *h = make_hit(whp, wn, t, ray, mi);
    return true;
  }
};

struct MeshObj : Object {  // src/ray.rs:498-680
  std::shared_ptr<Mesh> mesh;
  bool use_kd = true;
  // intersect_triangle (src/ray.rs:527-583)
  static bool tri(const Ray& r, const Triangle& t, double tmin, double tmax, double* tout, V3* nout, double* uo,
                  double* vo) {
    V3 e1 = t.v[1] - t.v[0];
    V3 e2 = t.v[2] - t.v[0];
    V3 hh = cross(r.d, e2);
    double a = dot(e1, hh);
    if (a > -1e-8 && a < 1e-8) return false;
    double f = 1.0 / a;
    V3 s = r.o - t.v[0];
    double u = f * dot(s, hh);
    if (!(u >= 0.0 && u <= 1.0)) return false;
    V3 q = cross(s, e1);
    double v = f * dot(r.d, q);
    if (v < 0.0 || u + v > 1.0) return false;
    double tt = f * dot(e2, q);
    if (tt > tmin && tt < tmax) {
      V3 n = cross(e1, e2);
      if (norm(n) < 1e-8) return false;
      if (a < 0.0) n = -n;
      n = normalize(n);
      *tout = tt;
      *nout = n;
      *uo = u;
      *vo = v;
      return true;
    }
    return false;
  }
  // intersect_bounds (src/ray.rs:586-610)
  bool bounds_hit(const Ray& r, double tmin, double tmax) const {
    double tl = tmin, th = tmax;
    for (int a = 0; a < 3; a++) {
      double inv = 1.0 / r.d[a];
      double t0 = (mesh->bmin[a] - r.o[a]) * inv;
      double t1 = (mesh->bmax[a] - r.o[a]) * inv;
      if (inv < 0.0) std::swap(t0, t1);
      tl = rmax(tl, t0);
      th = rmin(th, t1);
      if (tl > th) return false;
    }
    return true;
  }
  bool hit(const Ray& r, double tmin, double tmax, Hit* h, Counters* ct) const override {
    if (!bounds_hit(r, tmin, tmax)) return false;
    bool found = false;
    double closest = tmax;
    auto visit = [&](const std::vector<size_t>& idx) {
      for (size_t ti : idx) {
        if (ct) tlc.tri_tests++;
        double t, u, v;
        V3 n;
        if (tri(r, mesh->tris[ti], tmin, closest, &t, &n, &u, &v)) {
          if (t < closest) {
            closest = t;
            *h = make_hit(r.at(t), n, t, r, mi);
            h->has_uv = true;
            h->u = u;
            h->v = v;
            found = true;
          }
        }
      }
    };
    if (use_kd) {
      if (mesh->kd.root) {
        uint64_t visits = 0;
        mesh->kd.traverse(mesh->kd.root.get(), r.o, r.d, visit, ct ? &visits : nullptr);
        if (ct) tlc.kd_visits += visits;
      }
    } else {
      std::vector<size_t> all(mesh->tris.size());
      for (size_t i = 0; i < all.size(); i++) all[i] = i;
      visit(all);
    }
    return found;
  }
};

struct World {  // src/ray.rs:683-712
  std::vector<std::unique_ptr<Object>> objects;
  bool hit(const Ray& r, double tmin, double tmax, Hit* out, Counters* c) const {
    bool any = false;
    double closest = tmax;
    Hit h;
    for (auto& o : objects) {
      if (o->hit(r, tmin, closest, &h, c)) {
        closest = h.t;
        *out = h;
        any = true;
      }
    }
    return any;
  }
};

// ---------------------------------------------------------------------------
// Camera (src/camera.rs:23-254)
// ---------------------------------------------------------------------------
struct Camera {
  V3 origin, horizontal, vertical, llc, view_dir;
  bool persp = false;
  bool has_pitch = false, has_gcolor = false, has_thick = false;
  double pitch = 0, thickness = 0;
  V3 gcolor;
};
static Camera make_camera(const CameraCfg& cfg, double aspect) {
  Camera c;
  V3 origin = cfg.position, target = cfg.target, up = cfg.up;
  V3 w = normalize(origin - target);
  V3 u = normalize(cross(up, w));
  V3 v = cross(w, u);
  V3 vd = normalize(-w);
  if (cfg.has_grid_color) { c.gcolor = hex_req(cfg.grid_color); c.has_gcolor = true; }
  c.has_pitch = cfg.has_pitch;
  c.pitch = cfg.grid_pitch;
  c.has_thick = cfg.has_thickness;
  c.thickness = cfg.grid_thickness;
  c.origin = origin;
  c.view_dir = vd;
  if (cfg.kind == "ortho") {
    double vh = cfg.height;
    double vw = rmax(cfg.width, vh * aspect);
    c.horizontal = vw * u;
    c.vertical = vh * v;
    c.llc = origin - c.horizontal / 2.0 - c.vertical / 2.0;
    c.persp = false;
  } else if (cfg.kind == "perspective") {
    double fov = cfg.has_fov ? cfg.fov : 45.0;
    if (fov <= 0.0 || fov >= 180.0) throw Err("Field of view must be between 0 and 180 degrees");
    double focal = 1.0;
    double theta = to_radians(fov);
    double hh = std::tan(theta / 2.0);
    double hw = aspect * hh;
    double vh = 2.0 * hh * focal;
    double vw = 2.0 * hw * focal;
    c.horizontal = vw * u;
    c.vertical = vh * v;
    V3 center = origin + focal * vd;
    c.llc = center - c.horizontal / 2.0 - c.vertical / 2.0;
    c.persp = true;
  } else {
    throw Err("Unsupported camera type: " + cfg.kind);
  }
  return c;
}
static Ray get_ray(const Camera& c, double u, double v) {  // src/camera.rs:155-167
  V3 vp = c.llc + u * c.horizontal + v * c.vertical;
  if (c.persp) {
    V3 dir = normalize(vp - c.origin);
    return Ray(c.origin, dir);
  }
  return Ray(vp, c.view_dir);
}
static bool grid_color(const Camera& c, const Ray& r, V3* out) {  // src/camera.rs:171-254
  if (c.persp) return false;
  if (!(c.has_pitch && c.has_gcolor && c.has_thick && c.pitch > 0.0 && c.thickness > 0.0)) return false;
  double p = c.pitch, half = c.thickness / 2.0;
  for (int plane = 0; plane < 3; plane++) {
    int ax = plane == 0 ? 2 : (plane == 1 ? 1 : 0);  // z=0, y=0, x=0
    int a1 = plane == 0 ? 0 : (plane == 1 ? 0 : 1);
    int a2 = plane == 0 ? 1 : (plane == 1 ? 2 : 2);
    if (std::fabs(r.d[ax]) > 1e-10) {
      double t = -r.o[ax] / r.d[ax];
      if (t > 0.0) {
        V3 ip = r.o + t * r.d;
        double m1 = std::fabs(rfract(ip[a1] / p));
        double m2 = std::fabs(rfract(ip[a2] / p));
        double d1 = rmin(m1 * p, (1.0 - m1) * p);
        double d2 = rmin(m2 * p, (1.0 - m2) * p);
        if (d1 <= half || d2 <= half) { *out = c.gcolor; return true; }
      }
    }
  }
  return false;
}

// ---------------------------------------------------------------------------
// Lighting (src/lighting.rs)
// ---------------------------------------------------------------------------
struct ShadeMat {  // effective material after apply_texture
  V3 color;        // parsed colour (fallback white)
  double ambient, diffuse, specular, shininess;
};
static V3 reflect(V3 i, V3 n) {  // src/lighting.rs:291-294
  double s = 2.0 * dot(i, n);
  return normalize(i - s * n);
}

struct Ctx {
  const World* world;
  const Scene* scene;
  const Camera* cam;   // non-null for ray_color_with_camera(Some(camera))
  V3 cam_pos;
  V3 background;
  std::vector<const Material*> materials;  // by object index
  Counters* ct;
  uint32_t disk_samples = 16;  // shadow rays per disk light; the reference's constant is 16
};

// apply_texture (src/lighting.rs:9-54) then hex_to_color of the effective colour
static ShadeMat effective_material(const Material& m, const Hit& h) {
  const Material* em = &m;
  std::string color = m.color;
  if (m.texture != 0 && h.has_uv) {
    if (m.texture == 1) {
      V3 gc = hex_or(m.line_color, v3(0, 0, 0));
      double half = m.line_width / 2.0;
      double um = std::fabs(rfract(h.u / m.cell_size));
      double vm = std::fabs(rfract(h.v / m.cell_size));
      bool onu = um <= half || um >= (1.0 - half);
      bool onv = vm <= half || vm >= (1.0 - half);
      if (onu || onv) {
        char buf[16];
        snprintf(buf, sizeof buf, "#%02X%02X%02X", sat_u8(gc.x * 255.0), sat_u8(gc.y * 255.0), sat_u8(gc.z * 255.0));
        color = buf;
      }
    } else {
      int32_t cu = sat_i32(std::floor(h.u)), cv = sat_i32(std::floor(h.v));
      int32_t sum = (int32_t)((uint32_t)cu + (uint32_t)cv);  // release build wraps
      if (sum % 2 != 0) {
        em = m.material_b.get();
        color = em->color;
      }
    }
  }
  ShadeMat s;
  s.color = hex_or(color, v3(1, 1, 1));
  s.ambient = em->ambient;
  s.diffuse = em->diffuse;
  s.specular = em->specular;
  s.shininess = em->shininess;
  return s;
}

static bool shadowed(const Ctx& c, V3 origin, V3 dir, double dist) {
  if (c.ct) tlc.shadow++;
  Ray sr(origin, dir);
  Hit tmp;
  return c.world->hit(sr, 0.001, dist, &tmp, c.ct);
}

// calculate_point_light_contribution (src/lighting.rs:100-142)
static V3 point_light(const Ctx& c, const Hit& h, const ShadeMat& m, V3 lp, V3 lc, double li) {
  V3 ld = normalize(lp - h.point);
  V3 so = h.point + 0.001 * h.normal;
  double dist = norm(lp - h.point);
  if (shadowed(c, so, ld, dist)) return v3(0, 0, 0);
  double ds = rmax(dot(h.normal, ld), 0.0);
  V3 diffuse = m.diffuse * ds * li * cmul(lc, m.color);
  V3 spec = v3(0, 0, 0);
  if (ds > 0.0) {
    V3 vd = normalize(c.cam_pos - h.point);
    V3 rd = reflect(-ld, h.normal);
    double ss = std::pow(rmax(dot(vd, rd), 0.0), m.shininess);
    spec = m.specular * ss * li * lc;
  }
  return diffuse + spec;
}

// calculate_diffuse_light_contribution (src/lighting.rs:145-217) with
// sample_disk_light_point (:69-97) and sample_disk_point (:57-66)
static V3 disk_light(const Ctx& c, const Hit& h, const ShadeMat& m, V3 lp, V3 lc, double li, double diameter,
                     uint64_t seed) {
  const uint32_t SAMPLES = c.disk_samples;
  uint64_t ls = seed * 0x9E3779B97F4A7C15ULL + sat_u64(h.point.x * 1000.0) * 0x85EBCA6BULL +
                sat_u64(h.point.y * 1000.0) * 0xC2B2AE35ULL + sat_u64(h.point.z * 1000.0) * 0x6C8E9CF5ULL;
  StdRng rng(ls);
  V3 total = v3(0, 0, 0);
  uint32_t visible = 0;
  for (uint32_t s = 0; s < SAMPLES; s++) {
    double radius = diameter / 2.0;
    V3 ldir = normalize(lp - h.point);
    V3 up = std::fabs(ldir.x) < 0.9 ? v3(1, 0, 0) : v3(0, 1, 0);
    V3 u = normalize(cross(up, ldir));
    V3 v = normalize(cross(ldir, u));
    double dx, dy;
    for (;;) {
      dx = rng.gen_range(-radius, radius);
      dy = rng.gen_range(-radius, radius);
      if (dx * dx + dy * dy <= radius * radius) break;
    }
    V3 sp = lp + dx * u + dy * v;
    V3 sd = normalize(sp - h.point);
    double dist = norm(sp - h.point);
    V3 so = h.point + 0.001 * h.normal;
    if (shadowed(c, so, sd, dist)) continue;
    visible++;
    double ds = rmax(dot(h.normal, sd), 0.0);
    V3 diffuse = m.diffuse * ds * li * cmul(lc, m.color);
    V3 spec = v3(0, 0, 0);
    if (ds > 0.0) {
      V3 vd = normalize(c.cam_pos - h.point);
      V3 rd = reflect(-sd, h.normal);
      double ss = std::pow(rmax(dot(vd, rd), 0.0), m.shininess);
      spec = m.specular * ss * li * lc;
    }
    total = total + (diffuse + spec);
  }
  return (total / (double)SAMPLES) * ((double)visible / (double)SAMPLES);
}

// phong_lighting (src/lighting.rs:220-288)
static V3 phong(const Ctx& c, const Hit& h, const Material& mat, uint64_t seed) {
  ShadeMat m = effective_material(mat, h);
  V3 ac = hex_or(c.scene->ambient_color, v3(1, 1, 1));
  V3 color = m.ambient * c.scene->ambient_intensity * cmul(ac, m.color);
  for (auto& L : c.scene->lights) {
    V3 lc = hex_or(L.color, v3(1, 1, 1));
    V3 contrib = L.has_diameter ? disk_light(c, h, m, L.position, lc, L.intensity, L.diameter, seed)
                                : point_light(c, h, m, L.position, lc, L.intensity);
    color = color + contrib;
  }
  return color;
}

// apply_fog (src/lighting.rs:297-319)
static V3 apply_fog(const Scene& s, V3 color, double dist) {
  if (!s.has_fog) return color;
  V3 fc = hex_or(s.fog.color, v3(0.5, 0.5, 0.5));
  double f;
  if (dist <= s.fog.start) f = 0.0;
  else if (dist >= s.fog.end) f = 1.0;
  else f = (dist - s.fog.start) / (s.fog.end - s.fog.start);
  f = 1.0 - std::exp(-s.fog.density * f);
  f = rclamp(f, 0.0, 1.0);
  return color * (1.0 - f) + fc * f;
}

// ray_color_with_camera / ray_color_with_data (src/lighting.rs:352-506).
// Both compute the same colour; the data variant also reports the first
// hit's camera distance and normal.
static V3 ray_color(const Ctx& c, const Ray& r, int depth, uint64_t seed, bool* has_data, double* dep, V3* nrm) {
  if (has_data) *has_data = false;
  if (depth <= 0) return v3(0, 0, 0);
  Hit h;
  if (c.world->hit(r, 0.001, INF, &h, c.ct)) {
    if (has_data) {
      *has_data = true;
      *dep = norm(h.point - c.cam_pos);
      *nrm = h.normal;
    }
    const Material& mat = *c.materials[h.material_index];
    V3 color = phong(c, h, mat, seed);
    double dist = norm(h.point - c.cam_pos);
    color = apply_fog(*c.scene, color, dist);
    if (mat.has_reflectivity) {
      double refl = mat.reflectivity;
      if (refl > 0.0 && depth > 1) {
        V3 vd = normalize(c.cam_pos - h.point);
        V3 rd = reflect(-vd, h.normal);
        Ray rr(h.point + 0.001 * h.normal, rd);
        if (c.ct) tlc.reflection++;
        V3 rc = ray_color(c, rr, depth - 1, seed, nullptr, nullptr, nullptr);
        color = color * (1.0 - refl) + rc * refl;
      }
    }
    return color;
  }
  if (c.cam) {
    V3 g;
    if (grid_color(*c.cam, r, &g)) return g;
  }
  return c.background;
}

// ---------------------------------------------------------------------------
// Outline post-process (src/outline.rs:86-278)
// ---------------------------------------------------------------------------
struct OutlineCfg {
  double wd, wn, thr;
  V3 color;
  bool use8;
  double thickness;
};
// Applied to rows [ya, yb) of the image (the whole image in the reference's
// render; a band of rows for bounded samples, whose first and last
// 1 + ceil(thickness - 1) rows then lack their neighbours' G-buffers).  The
// edge mask is computed only where the band's blend reads it.
static void apply_outline(std::vector<V3>& img, const std::vector<uint8_t>& valid, const std::vector<double>& depth,
                          const std::vector<V3>& normal, uint32_t W, uint32_t H, const OutlineCfg& cfg,
                          uint32_t ya = 0, uint32_t yb = UINT32_MAX) {
  yb = std::min(yb, H);
  auto fg = [&](int64_t x, int64_t y) -> bool {
    if (x < 0 || y < 0 || x >= (int64_t)W || y >= (int64_t)H) return false;
    return valid[(size_t)y * W + x];
  };
  int32_t radius = 0;
  if (cfg.thickness > 1.0) radius = std::max(0, sat_i32(std::ceil(cfg.thickness - 1.0)));
  const uint32_t my0 = ya > (uint32_t)radius ? ya - (uint32_t)radius : 0;
  const uint32_t my1 = (uint32_t)std::min<int64_t>((int64_t)H, (int64_t)yb + radius);
  std::vector<double> mask((size_t)W * H, 0.0);
  for (uint32_t y = my0; y < my1; y++)
    for (uint32_t x = 0; x < W; x++) {
      std::vector<std::pair<int64_t, int64_t>> nb;
      if (cfg.use8) {
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            if (dx == 0 && dy == 0) continue;
            int64_t nx = (int64_t)x + dx, ny = (int64_t)y + dy;
            if (nx >= 0 && ny >= 0) nb.emplace_back(nx, ny);
          }
      } else {
        if (x > 0) nb.emplace_back((int64_t)x - 1, y);
        nb.emplace_back((int64_t)x + 1, y);
        if (y > 0) nb.emplace_back(x, (int64_t)y - 1);
        nb.emplace_back(x, (int64_t)y + 1);
      }
      bool cf = fg(x, y);
      double maxe = 0.0;
      for (auto& q : nb) {
        bool nf = fg(q.first, q.second);
        double e;
        if (cf && nf) {
          size_t ci = (size_t)y * W + x, ni = (size_t)q.second * W + q.first;
          double dd = std::fabs(depth[ci] - depth[ni]);
          double ndd = dd / rmax(depth[ci] * 0.1, 0.1);
          double dp = rclamp(dot(normal[ci], normal[ni]), -1.0, 1.0);
          double nd = 1.0 - dp;
          e = cfg.wd * ndd + cfg.wn * nd;
        } else if (cf != nf) {
          e = cfg.wd * 2.0 + cfg.wn * 2.0;
        } else {
          e = 0.0;
        }
        maxe = rmax(maxe, e);
      }
      if (maxe > cfg.thr) mask[(size_t)y * W + x] = (maxe - cfg.thr) / rmax(1.0 - cfg.thr, 0.001);
    }
  std::vector<double> fin = mask;
  if (cfg.thickness > 1.0) {
    if (radius > 0) {
      for (uint32_t y = ya; y < yb; y++)
        for (uint32_t x = 0; x < W; x++) {
          size_t idx = (size_t)y * W + x;
          double ms = mask[idx];
          for (int32_t dy = -radius; dy <= radius; dy++)
            for (int32_t dx = -radius; dx <= radius; dx++) {
              int64_t nx = (int64_t)x + dx, ny = (int64_t)y + dy;
              if (nx >= 0 && ny >= 0 && nx < (int64_t)W && ny < (int64_t)H) {
                double dist = std::sqrt((double)(dx * dx + dy * dy));
                if (dist <= cfg.thickness) {
                  double fo = 1.0 - (dist / cfg.thickness);
                  double st = mask[(size_t)ny * W + nx] * fo;
                  ms = rmax(ms, st);
                }
              }
            }
          fin[idx] = ms;
        }
    }
  }
  for (size_t i = (size_t)ya * W; i < (size_t)yb * W; i++) {
    if (fin[i] > 0.0) {
      double w = rclamp(rmin(fin[i], 1.0), 0.0, 1.0);
      img[i] = v3(img[i].x * (1.0 - w) + cfg.color.x * w, img[i].y * (1.0 - w) + cfg.color.y * w,
                  img[i].z * (1.0 - w) + cfg.color.z * w);
    }
  }
}

// ---------------------------------------------------------------------------
// Renderer (src/renderer.rs:120-912)
// ---------------------------------------------------------------------------
struct RenderOpts {
  uint32_t width, height;
  int max_depth = 10;
  bool use_kdtree = true;
  uint32_t samples = 1;
  int aa = 1;  // 0 no-jitter, 1 quincunx, 2 stochastic
  uint64_t seed = 0;
  bool outline = false;  // apply the scene's outline settings
  int threads = 1;
  uint32_t y0 = 0, y1 = UINT32_MAX;  // render only rows [y0, y1) (CPU baseline samples)
  uint32_t disk_samples = 16;        // extension: shadow rays per disk light (16 in the reference)
};

static void build_world(const Scene& s, bool use_kd, World* w, std::vector<const Material*>* mats) {
  mats->assign(s.objects.size(), nullptr);
  for (size_t i = 0; i < s.objects.size(); i++) {
    const SceneObject& o = s.objects[i];
    M4 tm;
    bool ht = o.has_transform && parse_transforms(o.transform, &tm);
    if (o.kind == 0) {
      auto sp = std::make_unique<Sphere>();
      V3 c = o.a;
      double r = o.radius;
      if (ht) {
        c = m4_point(tm, c);
        double sx = norm(v3(tm.m[0][0], tm.m[1][0], tm.m[2][0]));
        double sy = norm(v3(tm.m[0][1], tm.m[1][1], tm.m[2][1]));
        double sz = norm(v3(tm.m[0][2], tm.m[1][2], tm.m[2][2]));
        r *= rmax(rmax(sx, sy), sz);
      }
      hex_req(o.material.color);
      sp->c = c;
      sp->r = r;
      sp->mi = i;
      w->objects.push_back(std::move(sp));
    } else if (o.kind == 1) {
      auto pl = std::make_unique<Plane>();
      V3 p = o.a, n = o.b;
      if (ht) {
        p = m4_point(tm, p);
        M4 inv;
        if (m4_try_inverse(tm, &inv)) {
          M4 it;
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) it.m[a][b] = inv.m[b][a];
          n = m4_vec(it, n);
        }
      }
      pl->p = p;
      pl->n = normalize(n);
      hex_req(o.material.color);
      pl->mi = i;
      w->objects.push_back(std::move(pl));
    } else if (o.kind == 2) {
      auto cb = std::make_unique<Cube>();
      hex_req(o.material.color);
      cb->init(o.a, o.b, ht ? &tm : nullptr);
      cb->mi = i;
      w->objects.push_back(std::move(cb));
    } else {
      if (!o.mesh) continue;
      auto mo = std::make_unique<MeshObj>();
      if (ht) {
        auto m = std::make_shared<Mesh>();
        m->tris = o.mesh->tris;
        for (auto& t : m->tris)
          for (int k = 0; k < 3; k++) t.v[k] = m4_point(tm, t.v[k]);
        m->compute_bounds();
        m->build_kdtree();
        mo->mesh = m;
      } else {
        mo->mesh = o.mesh;
      }
      hex_req(o.material.color);
      mo->use_kd = use_kd;
      mo->mi = i;
      w->objects.push_back(std::move(mo));
    }
    (*mats)[i] = &o.material;
  }
}

template <class F>
static void parallel_for(size_t n, int threads, F&& fn, Counters* ct) {
  if (threads <= 1) {
    for (size_t i = 0; i < n; i++) fn(i);
    flush_counts(ct);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> th;
  std::exception_ptr eptr;
  std::mutex em;
  for (int t = 0; t < threads; t++)
    th.emplace_back([&]() {
      try {
        for (;;) {
          size_t i = next.fetch_add(1);
          if (i >= n) break;
          fn(i);
        }
      } catch (...) {
        std::lock_guard<std::mutex> g(em);
        if (!eptr) eptr = std::current_exception();
        next.store(n);
      }
      flush_counts(ct);
    });
  for (auto& t : th) t.join();
  if (eptr) std::rethrow_exception(eptr);
}

struct PairHash {
  size_t operator()(const std::pair<uint32_t, uint32_t>& p) const {
    return std::hash<uint64_t>()(((uint64_t)p.first << 32) | p.second);
  }
};

static void render(const Scene& s, const RenderOpts& o, std::vector<V3>* out, Counters* ct) {
  if (o.samples == 0) throw Err("Samples must be greater than 0");
  double aspect = (double)o.width / (double)o.height;
  Camera cam = make_camera(s.camera, aspect);
  World world;
  std::vector<const Material*> mats;
  build_world(s, o.use_kdtree, &world, &mats);
  V3 bg = s.has_background ? hex_req(s.background) : v3(0, 0, 0);
  OutlineCfg ocfg{};
  bool outline = false;
  if (o.outline && s.has_outline && s.outline.enabled) {
    outline = true;
    ocfg.wd = s.outline.depth_weight;
    ocfg.wn = s.outline.normal_weight;
    ocfg.thr = s.outline.threshold;
    ocfg.color = hex_req(s.outline.color);
    ocfg.use8 = s.outline.use_8;
    ocfg.thickness = s.outline.thickness;
  }
  const uint32_t W = o.width, H = o.height;
  out->assign((size_t)W * H, v3(0, 0, 0));
  Ctx c{&world, &s, nullptr, s.camera.position, bg, mats, ct, o.disk_samples};
  const uint64_t GOLD = 0x9E3779B97F4A7C15ULL;

  if (o.aa == 1) {  // render_quincunx (src/renderer.rs:752-897)
    std::mutex mu;
    std::unordered_map<std::pair<uint32_t, uint32_t>, V3, PairHash> cache;
    double pw = 1.0 / (double)W, ph = 1.0 / (double)H;
    auto corner = [&](uint32_t cx, uint32_t cy) -> V3 {
      auto key = std::make_pair(cx, cy);
      {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
      }
      double cu = rclamp((double)cx * pw, 0.0, 1.0);
      double cv = rclamp(1.0 - (double)cy * ph, 0.0, 1.0);
      Ray r = get_ray(cam, cu, cv);
      uint64_t seed = o.seed * GOLD + (uint64_t)cx + (uint64_t)cy * 0x85EBCA6BULL;
      if (ct) tlc.primary++;
      V3 col = ray_color(c, r, o.max_depth, seed, nullptr, nullptr, nullptr);
      {
        std::lock_guard<std::mutex> g(mu);
        cache[key] = col;
      }
      return col;
    };
    uint32_t ya = std::min(o.y0, H), yb = std::min(o.y1, H);
    size_t base = (size_t)ya * W;
    parallel_for((size_t)W * (yb - ya), o.threads, [&](size_t k) {
      size_t i = base + k;
      uint32_t x = (uint32_t)(i % W), y = (uint32_t)(i / W);
      double u = ((double)x + 0.5) * pw;
      double v = 1.0 - ((double)y + 0.5) * ph;
      Ray r = get_ray(cam, u, v);
      uint64_t seed = o.seed * GOLD + (uint64_t)x * 0x85EBCA6BULL + (uint64_t)y * 0xC2B2AE35ULL + 0x12345678ULL;
      if (ct) tlc.primary++;
      V3 cc = ray_color(c, r, o.max_depth, seed, nullptr, nullptr, nullptr);
      V3 k0 = corner(x, y), k1 = corner(x + 1, y), k2 = corner(x, y + 1), k3 = corner(x + 1, y + 1);
      V3 tot = cc + k0 + k1 + k2 + k3;
      (*out)[i] = tot / 5.0;
    }, ct);
  } else {  // render_standard[_with_outline] (src/renderer.rs:445-749)
    Ctx cc = c;
    cc.cam = &cam;
    std::vector<uint8_t> valid(outline ? (size_t)W * H : 0, 0);
    std::vector<double> depth(outline ? (size_t)W * H : 0, 0.0);
    std::vector<V3> nrm(outline ? (size_t)W * H : 0, v3(0, 0, 0));
    double pwid = 1.0 / (double)(uint32_t)(W - 1), phei = 1.0 / (double)(uint32_t)(H - 1);
    uint32_t ya = std::min(o.y0, H), yb = std::min(o.y1, H);
    size_t base = (size_t)ya * W;
    parallel_for((size_t)W * (yb - ya), o.threads, [&](size_t k) {
      size_t i = base + k;
      uint32_t x = (uint32_t)(i % W), y = (uint32_t)(i / W);
      double pu = (double)x / (double)(uint32_t)(W - 1);
      double pv = (double)(uint32_t)(H - 1 - y) / (double)(uint32_t)(H - 1);
      V3 tot = v3(0, 0, 0);
      uint64_t pseed = o.seed * GOLD + (uint64_t)x * 0x85EBCA6BULL + (uint64_t)y * 0xC2B2AE35ULL;
      StdRng rng(pseed);
      bool have = false;
      double pd = 0;
      V3 pn = v3(0, 0, 0);
      for (uint32_t sidx = 0; sidx < o.samples; sidx++) {
        double su, sv;
        if (o.aa == 0) {
          su = pu;
          sv = pv;
        } else if (o.samples == 1) {
          double ju = rng.gen_f64() - 0.5;
          double jv = rng.gen_f64() - 0.5;
          su = pu + ju * pwid;
          sv = pv + jv * phei;
        } else {
          double ang = 2.0 * M_PI * (double)sidx / (double)o.samples;
          double ph_ = rng.gen_f64() * 2.0 * M_PI;
          double ra = ang + ph_;
          double rad = 0.5 * rng.gen_f64();
          double ju = rad * std::cos(ra);
          double jv = rad * std::sin(ra);
          su = pu + ju * pwid;
          sv = pv + jv * phei;
        }
        Ray r = get_ray(cam, su, sv);
        uint64_t sseed = pseed + (uint64_t)sidx * 0x1F845FEDULL;
        if (ct) tlc.primary++;
        bool hd = false;
        double d = 0;
        V3 n;
        V3 col = ray_color(cc, r, o.max_depth, sseed, outline ? &hd : nullptr, &d, &n);
        tot = tot + col;
        if (outline && hd) {
          if (!have || d < pd) { have = true; pd = d; pn = n; }
        }
      }
      (*out)[i] = tot / (double)o.samples;
      if (outline && have) { valid[i] = 1; depth[i] = pd; nrm[i] = pn; }
    }, ct);
    if (outline) apply_outline(*out, valid, depth, nrm, W, H, ocfg, ya, yb);
  }
}

// create_image_from_data (src/renderer.rs:899-912)
static void quantize(const std::vector<V3>& img, uint8_t* rgb) {
  for (size_t i = 0; i < img.size(); i++) {
    rgb[3 * i + 0] = sat_u8(rclamp(img[i].x, 0.0, 1.0) * 255.0);
    rgb[3 * i + 1] = sat_u8(rclamp(img[i].y, 0.0, 1.0) * 255.0);
    rgb[3 * i + 2] = sat_u8(rclamp(img[i].z, 0.0, 1.0) * 255.0);
  }
}

static std::string dir_of(const std::string& path) {
  size_t k = path.find_last_of('/');
  if (k == std::string::npos) return "";
  if (k == 0) return "/";
  return path.substr(0, k);
}

static void set_err(char* err, int len, const std::string& m) {
  if (!err || len <= 0) return;
  snprintf(err, (size_t)len, "%s", m.c_str());
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI used by the tests (ctypes)
// ---------------------------------------------------------------------------
extern "C" {

// Renders a scene file the way `Renderer::render` does.  aa: 0 no-jitter,
// 1 quincunx, 2 stochastic.  outline != 0 applies the scene's enabled
// outline settings (quincunx ignores them, as the reference does).
// Returns 0 on success, 1 on a reference-side error (message in err).
// counts (nullable) receives [primary, reflection, shadow, kd_visits,
// triangle_tests, sphere_tests].
int oracle_render_rows(const char* scene_path, const char* scene_json, uint32_t width, uint32_t height, int aa,
                       uint32_t samples, int max_depth, uint64_t seed, int use_kdtree, int outline, int threads,
                       uint32_t y0, uint32_t y1, uint8_t* out_rgb, double* out_linear, uint64_t* counts, char* err,
                       int err_len);

int oracle_render(const char* scene_path, const char* scene_json, uint32_t width, uint32_t height, int aa,
                  uint32_t samples, int max_depth, uint64_t seed, int use_kdtree, int outline, int threads,
                  uint8_t* out_rgb, double* out_linear, uint64_t* counts, char* err, int err_len) {
  return oracle_render_rows(scene_path, scene_json, width, height, aa, samples, max_depth, seed, use_kdtree, outline,
                            threads, 0, UINT32_MAX, out_rgb, out_linear, counts, err, err_len);
}

// As oracle_render, restricted to image rows [y0, y1): the pixels of other
// rows stay black.  The outline pass runs on the band's rows; its first and
// last 1 + ceil(thickness - 1) rows lack the neighbouring rows' depth and
// normals, so only the rows inside them are the reference's.  Used to time
// bounded samples of a frame (CPU baseline) and to check full-size frames.
int oracle_render_ex(const char* scene_path, const char* scene_json, uint32_t width, uint32_t height, int aa,
                     uint32_t samples, int max_depth, uint64_t seed, int use_kdtree, int outline, int threads,
                     uint32_t y0, uint32_t y1, uint32_t disk_samples, uint8_t* out_rgb, double* out_linear,
                     uint64_t* counts, char* err, int err_len);

int oracle_render_rows(const char* scene_path, const char* scene_json, uint32_t width, uint32_t height, int aa,
                       uint32_t samples, int max_depth, uint64_t seed, int use_kdtree, int outline, int threads,
                       uint32_t y0, uint32_t y1, uint8_t* out_rgb, double* out_linear, uint64_t* counts, char* err,
                       int err_len) {
  return oracle_render_ex(scene_path, scene_json, width, height, aa, samples, max_depth, seed, use_kdtree, outline,
                          threads, y0, y1, 16, out_rgb, out_linear, counts, err, err_len);
}

// As oracle_render_rows with disk_samples shadow rays per disk light and
// shading point (an extension: the reference always casts 16; the samples
// continue the same StdRng stream, so the first 16 are the reference's).
int oracle_render_ex(const char* scene_path, const char* scene_json, uint32_t width, uint32_t height, int aa,
                     uint32_t samples, int max_depth, uint64_t seed, int use_kdtree, int outline, int threads,
                     uint32_t y0, uint32_t y1, uint32_t disk_samples, uint8_t* out_rgb, double* out_linear,
                     uint64_t* counts, char* err, int err_len) {
  using namespace orc;
  if (disk_samples == 0) {
    set_err(err, err_len, "disk_samples must be positive");
    return 1;
  }
  try {
    Scene s = scene_path ? parse_scene(read_file(scene_path), dir_of(scene_path))
                         : parse_scene(std::string(scene_json), ".");
    RenderOpts o;
    o.width = width;
    o.height = height;
    o.aa = aa;
    o.samples = samples;
    o.max_depth = max_depth;
    o.seed = seed;
    o.use_kdtree = use_kdtree != 0;
    o.outline = outline != 0 && aa != 1;
    o.threads = threads;
    o.y0 = y0;
    o.y1 = y1;
    o.disk_samples = disk_samples;
    std::vector<V3> img;
    Counters ct;
    render(s, o, &img, counts ? &ct : nullptr);
    if (out_rgb) quantize(img, out_rgb);
    if (out_linear)
      for (size_t i = 0; i < img.size(); i++) {
        out_linear[3 * i] = img[i].x;
        out_linear[3 * i + 1] = img[i].y;
        out_linear[3 * i + 2] = img[i].z;
      }
    if (counts) {
      counts[0] = ct.primary;
      counts[1] = ct.reflection;
      counts[2] = ct.shadow;
      counts[3] = ct.kd_visits;
      counts[4] = ct.tri_tests;
      counts[5] = ct.sphere_tests;
    }
    return 0;
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return 1;
  }
}

// One ChaCha block with an explicit 64-bit counter and stream id (two
// words), for checking the block function against published test vectors.
void oracle_chacha_block(const uint32_t* key, uint64_t counter, const uint32_t* nonce, int double_rounds,
                         uint32_t* out) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                    key[4], key[5], key[6], key[7], (uint32_t)counter, (uint32_t)(counter >> 32), nonce[0],
                    nonce[1]};
  uint32_t x[16];
  memcpy(x, s, sizeof x);
#define QR2(a, b, c, d)                                 \
  x[a] += x[b]; x[d] ^= x[a]; x[d] = orc::rotl32(x[d], 16); \
  x[c] += x[d]; x[b] ^= x[c]; x[b] = orc::rotl32(x[b], 12); \
  x[a] += x[b]; x[d] ^= x[a]; x[d] = orc::rotl32(x[d], 8);  \
  x[c] += x[d]; x[b] ^= x[c]; x[b] = orc::rotl32(x[b], 7);
  for (int r = 0; r < double_rounds; r++) {
    QR2(0, 4, 8, 12) QR2(1, 5, 9, 13) QR2(2, 6, 10, 14) QR2(3, 7, 11, 15)
    QR2(0, 5, 10, 15) QR2(1, 6, 11, 12) QR2(2, 7, 8, 13) QR2(3, 4, 9, 14)
  }
#undef QR2
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// apply_outline_detection + create_image_from_data (src/outline.rs:86-110,
// src/renderer.rs:899-912) on caller buffers: colours, depths and normals
// planar (one double per pixel per plane), valid = 1 where the pixel has a
// depth and normal.
void oracle_outline(uint32_t W, uint32_t H, const double* r, const double* g, const double* b,
                    const uint8_t* valid, const double* depth, const double* nx, const double* ny, const double* nz,
                    double depth_weight, double normal_weight, double threshold, const double* edge_color,
                    int use_8_neighbors, double thickness, uint8_t* rgb) {
  using namespace orc;
  size_t n = (size_t)W * H;
  std::vector<V3> img(n), nrm(n);
  std::vector<uint8_t> val(valid, valid + n);
  std::vector<double> dep(depth, depth + n);
  for (size_t i = 0; i < n; i++) {
    img[i] = v3(r[i], g[i], b[i]);
    nrm[i] = v3(nx[i], ny[i], nz[i]);
  }
  OutlineCfg cfg{depth_weight, normal_weight, threshold, v3(edge_color[0], edge_color[1], edge_color[2]),
                 use_8_neighbors != 0, thickness};
  apply_outline(img, val, dep, nrm, W, H, cfg);
  quantize(img, rgb);
}

// The first n u32 words of StdRng::seed_from_u64(seed).
void oracle_stdrng_u32(uint64_t seed, int n, uint32_t* out) {
  orc::StdRng r(seed);
  for (int i = 0; i < n; i++) out[i] = r.next_u32();
}
// n draws of rng.gen::<f64>().
void oracle_stdrng_f64(uint64_t seed, int n, double* out) {
  orc::StdRng r(seed);
  for (int i = 0; i < n; i++) out[i] = r.gen_f64();
}
// n draws of rng.gen_range(lo..hi); returns 0, or 1 if the range is empty.
int oracle_stdrng_range(uint64_t seed, double lo, double hi, int n, double* out) {
  orc::StdRng r(seed);
  try {
    for (int i = 0; i < n; i++) out[i] = r.gen_range(lo, hi);
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}
// The 16 disk-light sample offsets (dx, dy) that one area-light shading
// point draws for the given light seed (src/lighting.rs:57-66, 170-173).
int oracle_disk_offsets(uint64_t light_seed, double radius, double* out32) {
  orc::StdRng r(light_seed);
  try {
    for (int s = 0; s < 16; s++) {
      double dx, dy;
      for (;;) {
        dx = r.gen_range(-radius, radius);
        dy = r.gen_range(-radius, radius);
        if (dx * dx + dy * dy <= radius * radius) break;
      }
      out32[2 * s] = dx;
      out32[2 * s + 1] = dy;
    }
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

// MeshObject::hit on an STL file for a batch of rays (origin, direction:
// 6 doubles each, the direction is normalised by Ray::new).  out: 8 doubles
// per ray [hit, t, px, py, pz, nx, ny, nz].  Returns the triangle count, or
// -1 on error.
long oracle_mesh_hit(const char* stl_path, int use_kdtree, long n, const double* rays, double tmin, double tmax,
                     double* out, char* err, int err_len) {
  using namespace orc;
  try {
    MeshObj mo;
    mo.mesh = std::make_shared<Mesh>(mesh_from_stl_bytes(read_file(stl_path)));
    mo.use_kd = use_kdtree != 0;
    mo.mi = 0;
    for (long i = 0; i < n; i++) {
      const double* r = rays + 6 * i;
      Ray ray(v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]));
      Hit h;
      double* o = out + 8 * i;
      if (mo.hit(ray, tmin, tmax, &h, nullptr)) {
        o[0] = 1;
        o[1] = h.t;
        o[2] = h.point.x; o[3] = h.point.y; o[4] = h.point.z;
        o[5] = h.normal.x; o[6] = h.normal.y; o[7] = h.normal.z;
      } else {
        for (int k = 0; k < 8; k++) o[k] = 0;
      }
    }
    return (long)mo.mesh->tris.size();
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return -1;
  }
}

// parse_transforms applied to a point (src/scene.rs:191-203); returns 0 or
// 1 when a transform string does not parse.
int oracle_transform_point(const char* const* transforms, int n, const double* p, double* out) {
  using namespace orc;
  std::vector<std::string> ts;
  for (int i = 0; i < n; i++) ts.push_back(transforms[i]);
  M4 m;
  if (!parse_transforms(ts, &m)) return 1;
  V3 r = m4_point(m, v3(p[0], p[1], p[2]));
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  return 0;
}

// hex_to_color; returns 0 or 1 on error.
int oracle_hex_to_color(const char* hex, double* out) {
  orc::V3 c;
  if (!orc::hex_to_color(hex, &c, nullptr)) return 1;
  out[0] = c.x;
  out[1] = c.y;
  out[2] = c.z;
  return 0;
}

// KdTree::new(triangles, 16, 10) (build_recursive, src/mesh.rs:125-197)
// over n triangles of 9 doubles (v0, v1, v2), flattened in preorder (left
// child next) into 72-byte records {int32 axis (-1 leaf), right, first,
// count; double split, bounds_min[3], bounds_max[3]} and the leaf lists in
// leaf order: the layout the CUDA library's rt_kd_build returns.  Call with
// null outputs to get the sizes, then again with buffers of those sizes.
// Returns 0, or 1 with the panic message in err.
int oracle_kd_build(const double* v, int64_t n, void* nodes_out, int32_t* idx_out, int64_t* n_nodes,
                    int64_t* n_idx, char* err, int err_len) {
  struct Rec {
    int32_t axis, right, first, count;
    double split, bmin[3], bmax[3];
  };
  static_assert(sizeof(Rec) == 72, "record layout");
  std::vector<orc::Triangle> t((size_t)n);
  for (int64_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) t[i].v[k] = orc::v3(v[9 * i + 3 * k], v[9 * i + 3 * k + 1], v[9 * i + 3 * k + 2]);
  orc::KdTree kd;
  try {
    kd.construct(t);
  } catch (const std::exception& e) {
    snprintf(err, err_len, "%s", e.what());
    return 1;
  }
  std::vector<Rec> recs;
  std::vector<int32_t> idx;
  std::function<void(const orc::KdNode*)> walk = [&](const orc::KdNode* nd) {
    Rec r{};
    for (int a = 0; a < 3; a++) {
      r.bmin[a] = nd->bmin[a];
      r.bmax[a] = nd->bmax[a];
    }
    size_t me = recs.size();
    if (nd->leaf) {
      r.axis = -1;
      r.first = (int32_t)idx.size();
      r.count = (int32_t)nd->tris.size();
      for (size_t i : nd->tris) idx.push_back((int32_t)i);
      recs.push_back(r);
      return;
    }
    r.axis = nd->axis;
    r.split = nd->split;
    recs.push_back(r);
    walk(nd->left.get());
    recs[me].right = (int32_t)recs.size();
    walk(nd->right.get());
  };
  if (kd.root) walk(kd.root.get());
  *n_nodes = (int64_t)recs.size();
  *n_idx = (int64_t)idx.size();
  if (nodes_out) memcpy(nodes_out, recs.data(), recs.size() * sizeof(Rec));
  if (idx_out) memcpy(idx_out, idx.data(), idx.size() * sizeof(int32_t));
  return 0;
}

// serde_json's default f64 parsing of one JSON number literal.
int oracle_json_f64(const char* text, double* out) {
  try {
    orc::JVal v = orc::parse_json(text);
    *out = orc::as_f64(v);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

}  // extern "C"
