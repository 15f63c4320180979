// Host-side scene loading for the B200 render path.
//
// Restates the reference's host work before rendering: serde_json
// deserialisation of the scene (src/scene.rs:311-458), STL loading
// (src/mesh.rs:751-1003), transform parsing and composition
// (src/scene.rs:115-203), the World build that transforms primitives
// (src/renderer.rs:138-317) and the k-d tree build (src/mesh.rs:73-215).
// The output is the flattened rt_scene_desc of include/rtrace_gpu.h.
//
// Arithmetic follows the reference's operation order (nalgebra gemv column
// accumulation, 4x4 cofactor inverse, euler-angle matrices); this file must
// be compiled without floating-point contraction.

#include "scene_loader.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <thread>

namespace rtb {
namespace {

const double INF = std::numeric_limits<double>::infinity();

struct LoadError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// f64::max / f64::min: a NaN argument is ignored.  When the arguments
// compare equal (+0 and -0) the reference's llvm.maxnum/minnum may return
// either, and a compiled std::fmax/fmin differs from call site to call
// site; these keep the first, as glibc's fmin/fmax do, everywhere (the
// device k-d build uses the same rule, so both builds give the same bytes).
inline double rmax(double a, double b) { return (b > a || a != a) ? b : a; }
inline double rmin(double a, double b) { return (b < a || a != a) ? b : a; }
inline double to_radians(double d) {
  const double k = M_PI / 180.0;
  return d * k;
}

struct V {
  double x, y, z;
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator/(V a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V operator*(double s, V a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V a) { return std::sqrt(0.0 + dot(a, a)); }
inline V normalize(V a) { return a / norm(a); }
inline V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// ---------------------------------------------------------------- JSON ----
struct J {
  enum K { NUL, BOOL, U64, I64, F64, STR, ARR, OBJ } k = NUL;
  bool b = false;
  uint64_t u = 0;
  int64_t i = 0;
  double d = 0;
  std::string s;
  std::vector<J> a;
  std::vector<std::pair<std::string, J>> o;
  const J* get(const char* key) const {
    for (auto& kv : o)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

// serde_json (default features) converts a decimal literal as
// significand-as-f64 followed by one multiply or divide by 10^|exp|.
double pow10_exact(unsigned e) {
  static double table[309];
  static bool init = false;
  if (!init) {
    for (unsigned k = 0; k < 309; k++) {
      char buf[16];
      snprintf(buf, sizeof buf, "1e%u", k);
      table[k] = strtod(buf, nullptr);  // the literal 1eK, correctly rounded
    }
    init = true;
  }
  return table[e];
}

struct JsonReader {
  const char* p;
  const char* e;
  [[noreturn]] void fail(const char* m) { throw LoadError(std::string("JSON parse error: ") + m); }
  void ws() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
  }
  int peek() const { return p < e ? (unsigned char)*p : 0; }
  static bool ovf(uint64_t a, uint64_t b) {
    const uint64_t c = UINT64_MAX;
    return a >= c / 10 && (a > c / 10 || b > c % 10);
  }
  double from_parts(bool pos, uint64_t sig, int exponent) {
    double f = (double)sig;
    for (;;) {
      int64_t ae = exponent < 0 ? -(int64_t)exponent : exponent;
      if (ae <= 308) {
        double pw = pow10_exact((unsigned)ae);
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
    return pos ? f : -f;
  }
  double exponent_part(bool pos, uint64_t sig, int start) {
    p++;
    bool pe = true;
    if (peek() == '+') p++;
    else if (peek() == '-') { p++; pe = false; }
    if (!(peek() >= '0' && peek() <= '9')) fail("invalid number");
    int64_t x = *p++ - '0';
    while (peek() >= '0' && peek() <= '9') {
      int dgt = *p++ - '0';
      if (x >= INT32_MAX / 10 && (x > INT32_MAX / 10 || dgt > INT32_MAX % 10)) {
        while (peek() >= '0' && peek() <= '9') p++;
        if (sig == 0 || !pe) return pos ? 0.0 : -0.0;
        fail("number out of range");
      }
      x = x * 10 + dgt;
    }
    int64_t fe = pe ? (int64_t)start + x : (int64_t)start - x;
    fe = std::max<int64_t>(INT32_MIN, std::min<int64_t>(INT32_MAX, fe));
    return from_parts(pos, sig, (int)fe);
  }
  double decimal_part(bool pos, uint64_t sig, int before) {
    p++;
    int after = 0;
    while (peek() >= '0' && peek() <= '9') {
      uint64_t dg = *p - '0';
      if (ovf(sig, dg)) {
        while (peek() >= '0' && peek() <= '9') p++;
        if (peek() == 'e' || peek() == 'E') return exponent_part(pos, sig, before + after);
        return from_parts(pos, sig, before + after);
      }
      p++;
      sig = sig * 10 + dg;
      after--;
    }
    if (after == 0) fail("invalid number");
    if (peek() == 'e' || peek() == 'E') return exponent_part(pos, sig, before + after);
    return from_parts(pos, sig, before + after);
  }
  void number(J& v) {
    bool pos = true;
    if (peek() == '-') { pos = false; p++; }
    if (!(peek() >= '0' && peek() <= '9')) fail("invalid number");
    uint64_t sig = 0;
    if (peek() == '0') {
      p++;
      if (peek() >= '0' && peek() <= '9') fail("invalid number");
    } else {
      sig = *p++ - '0';
      while (peek() >= '0' && peek() <= '9') {
        uint64_t dg = *p - '0';
        if (ovf(sig, dg)) {
          int ex = 0;
          while (peek() >= '0' && peek() <= '9') { p++; ex++; }
          v.k = J::F64;
          if (peek() == '.') v.d = decimal_part(pos, sig, ex);
          else if (peek() == 'e' || peek() == 'E') v.d = exponent_part(pos, sig, ex);
          else v.d = from_parts(pos, sig, ex);
          return;
        }
        p++;
        sig = sig * 10 + dg;
      }
    }
    if (peek() == '.') { v.k = J::F64; v.d = decimal_part(pos, sig, 0); return; }
    if (peek() == 'e' || peek() == 'E') { v.k = J::F64; v.d = exponent_part(pos, sig, 0); return; }
    if (pos) { v.k = J::U64; v.u = sig; return; }
    int64_t neg = (int64_t)(0 - sig);
    if (neg >= 0) { v.k = J::F64; v.d = -(double)sig; return; }
    v.k = J::I64;
    v.i = neg;
  }
  uint32_t hex4() {
    if (e - p < 4) fail("EOF while parsing a string");
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
  static void utf8(std::string& out, uint32_t cp) {
    if (cp < 0x80) out += (char)cp;
    else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
    else if (cp < 0x10000) {
      out += (char)(0xE0 | (cp >> 12));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    } else {
      out += (char)(0xF0 | (cp >> 18));
      out += (char)(0x80 | ((cp >> 12) & 0x3F));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    }
  }
  std::string str() {
    p++;
    std::string out;
    for (;;) {
      if (p >= e) fail("EOF while parsing a string");
      char c = *p++;
      if (c == '"') return out;
      if ((unsigned char)c < 0x20) fail("control character in string");
      if (c != '\\') { out += c; continue; }
      if (p >= e) fail("EOF while parsing a string");
      char x = *p++;
      switch (x) {
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
            if (e - p >= 2 && p[0] == '\\' && p[1] == 'u') {
              p += 2;
              uint32_t lo = hex4();
              cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
            } else {
              fail("lone leading surrogate");
            }
          }
          utf8(out, cp);
          break;
        }
        default: fail("invalid escape");
      }
    }
  }
  void value(J& v, int depth) {
    if (depth > 128) fail("recursion limit exceeded");
    ws();
    int c = peek();
    if (c == '{') {
      p++;
      v.k = J::OBJ;
      ws();
      if (peek() == '}') { p++; return; }
      for (;;) {
        ws();
        if (peek() != '"') fail("key must be a string");
        std::string key = str();
        ws();
        if (peek() != ':') fail("expected `:`");
        p++;
        v.o.emplace_back(key, J());
        value(v.o.back().second, depth + 1);
        ws();
        if (peek() == ',') { p++; continue; }
        if (peek() == '}') { p++; return; }
        fail("expected `,` or `}`");
      }
    } else if (c == '[') {
      p++;
      v.k = J::ARR;
      ws();
      if (peek() == ']') { p++; return; }
      for (;;) {
        v.a.emplace_back();
        value(v.a.back(), depth + 1);
        ws();
        if (peek() == ',') { p++; continue; }
        if (peek() == ']') { p++; return; }
        fail("expected `,` or `]`");
      }
    } else if (c == '"') {
      v.k = J::STR;
      v.s = str();
    } else if (c == 't' && e - p >= 4 && !strncmp(p, "true", 4)) {
      p += 4; v.k = J::BOOL; v.b = true;
    } else if (c == 'f' && e - p >= 5 && !strncmp(p, "false", 5)) {
      p += 5; v.k = J::BOOL; v.b = false;
    } else if (c == 'n' && e - p >= 4 && !strncmp(p, "null", 4)) {
      p += 4; v.k = J::NUL;
    } else if (c == '-' || (c >= '0' && c <= '9')) {
      number(v);
    } else {
      fail("expected value");
    }
  }
};

J parse_json(const std::string& text) {
  JsonReader r{text.data(), text.data() + text.size()};
  J v;
  r.value(v, 0);
  r.ws();
  if (r.p != r.e) r.fail("trailing characters");
  return v;
}

const J& req(const J& o, const char* k) {
  if (o.k != J::OBJ) throw LoadError(std::string("invalid type: expected a map containing `") + k + "`");
  const J* v = o.get(k);
  if (!v) throw LoadError(std::string("missing field `") + k + "`");
  return *v;
}
const J* opt(const J& o, const char* k) {
  const J* v = o.get(k);
  return (!v || v->k == J::NUL) ? nullptr : v;
}
double f64(const J& v) {
  if (v.k == J::U64) return (double)v.u;
  if (v.k == J::I64) return (double)v.i;
  if (v.k == J::F64) return v.d;
  throw LoadError("invalid type: expected f64");
}
std::string str(const J& v) {
  if (v.k != J::STR) throw LoadError("invalid type: expected a string");
  return v.s;
}
bool boolean(const J& v) {
  if (v.k != J::BOOL) throw LoadError("invalid type: expected a boolean");
  return v.b;
}
V vec3(const J& v) {
  if (v.k != J::ARR || v.a.size() != 3) throw LoadError("invalid length, expected an array of length 3");
  return {f64(v.a[0]), f64(v.a[1]), f64(v.a[2])};
}

// ------------------------------------------------------- Rust parsing -----
std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}
// f64::from_str (correctly rounded; accepts inf/infinity/nan)
bool parse_rust_f64(const std::string& t, double* out) {
  if (t.empty()) return false;
  size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
  std::string body = t.substr(i), low;
  for (char c : body) low += (char)tolower((unsigned char)c);
  if (low == "inf" || low == "infinity" || low == "nan") {
    double v = low == "nan" ? NAN : INF;
    *out = t[0] == '-' ? -v : v;
    return true;
  }
  bool digits = false, dot = false, ex = false;
  for (size_t k = 0; k < body.size(); k++) {
    char c = body[k];
    if (c >= '0' && c <= '9') digits = true;
    else if (c == '.' && !dot && !ex) dot = true;
    else if ((c == 'e' || c == 'E') && digits && !ex) {
      ex = true;
      if (k + 1 < body.size() && (body[k + 1] == '+' || body[k + 1] == '-')) k++;
      if (k + 1 >= body.size()) return false;
    } else {
      return false;
    }
  }
  if (!digits) return false;
  char* end = nullptr;
  *out = strtod(t.c_str(), &end);
  return end && *end == 0;
}

// ---------------------------------------------------------- matrices -----
struct M4 {
  double m[4][4];
};
M4 ident() {
  M4 r;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) r.m[i][j] = i == j ? 1.0 : 0.0;
  return r;
}
// nalgebra gemv: y = a_0 * x_0, then y = a_j * x_j + y for j = 1..3
void gemv4(const M4& a, const double x[4], double y[4]) {
  for (int i = 0; i < 4; i++) y[i] = a.m[i][0] * x[0];
  for (int j = 1; j < 4; j++)
    for (int i = 0; i < 4; i++) y[i] = a.m[i][j] * x[j] + y[i];
}
M4 mul(const M4& a, const M4& b) {
  M4 r;
  for (int j = 0; j < 4; j++) {
    double c[4] = {b.m[0][j], b.m[1][j], b.m[2][j], b.m[3][j]}, y[4];
    gemv4(a, c, y);
    for (int i = 0; i < 4; i++) r.m[i][j] = y[i];
  }
  return r;
}
V xform_point(const M4& a, V p) {
  double x[4] = {p.x, p.y, p.z, 1.0}, y[4];
  gemv4(a, x, y);
  return {y[0], y[1], y[2]};
}
V xform_vec(const M4& a, V p) {
  double x[4] = {p.x, p.y, p.z, 0.0}, y[4];
  gemv4(a, x, y);
  return {y[0], y[1], y[2]};
}
// nalgebra 4x4 try_inverse: cofactors over the column-major slice, det from
// the first column, then scale by 1/det.
bool inverse4(const M4& M, M4* out) {
  double m[16], inv[16];
  for (int k = 0; k < 16; k++) m[k] = M.m[k % 4][k / 4];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] +
           m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] -
           m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] +
           m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] -
            m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  if (det == 0.0) return false;
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] -
           m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] +
           m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] -
           m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] +
            m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] +
           m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] -
           m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] +
            m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] -
            m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] -
           m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] +
           m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] -
            m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] +
            m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double id = 1.0 / det;
  for (int k = 0; k < 16; k++) out->m[k % 4][k / 4] = inv[k] * id;
  return true;
}
// Rotation3::from_euler_angles(roll, pitch, yaw), homogeneous
M4 euler(double roll, double pitch, double yaw) {
  double sr = std::sin(roll), cr = std::cos(roll), sp = std::sin(pitch), cp = std::cos(pitch);
  double sy = std::sin(yaw), cy = std::cos(yaw);
  M4 r = ident();
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
// Transform::from_str + to_matrix (src/scene.rs:117-187)
M4 transform_matrix(const std::string& in) {
  std::string s = trim(in);
  static const char* kinds[3] = {"rotate(", "translate(", "scale("};
  for (int k = 0; k < 3; k++) {
    size_t n = strlen(kinds[k]);
    if (s.compare(0, n, kinds[k]) != 0) continue;
    std::string params = s.substr(n);
    if (params.empty() || params.back() != ')') throw LoadError("Missing closing parenthesis");
    params.pop_back();
    std::vector<double> v;
    size_t st = 0;
    for (;;) {
      size_t c = params.find(',', st);
      double x;
      if (!parse_rust_f64(trim(params.substr(st, c == std::string::npos ? std::string::npos : c - st)), &x))
        throw LoadError("Invalid transform parameters");
      v.push_back(x);
      if (c == std::string::npos) break;
      st = c + 1;
    }
    if (v.size() != 3) throw LoadError("Transform requires exactly 3 parameters (x, y, z)");
    if (k == 0) {
      M4 rx = euler(to_radians(v[0]), 0.0, 0.0);
      M4 ry = euler(0.0, to_radians(v[1]), 0.0);
      M4 rz = euler(0.0, 0.0, to_radians(v[2]));
      return mul(mul(rz, ry), rx);
    }
    M4 r = ident();
    if (k == 1) { r.m[0][3] = v[0]; r.m[1][3] = v[1]; r.m[2][3] = v[2]; }
    else { r.m[0][0] = v[0]; r.m[1][1] = v[1]; r.m[2][2] = v[2]; }
    return r;
  }
  throw LoadError("Unknown transform type");
}
// parse_transforms (src/scene.rs:191-203); false when a string does not parse
bool parse_transforms(const std::vector<std::string>& ts, M4* out) {
  M4 c = ident();
  try {
    for (auto& t : ts) c = mul(transform_matrix(t), c);
  } catch (const LoadError&) {
    return false;
  }
  *out = c;
  return true;
}

// -------------------------------------------------------------- STL -----
struct Tri {
  V v[3];
};
std::vector<std::string> lines_of(const std::string& s) {
  std::vector<std::string> out;
  size_t st = 0;
  while (st < s.size()) {
    size_t e = s.find('\n', st);
    std::string l = s.substr(st, e == std::string::npos ? std::string::npos : e - st);
    if (!l.empty() && l.back() == '\r') l.pop_back();
    out.push_back(std::move(l));
    if (e == std::string::npos) break;
    st = e + 1;
  }
  return out;
}
std::vector<std::string> words(const std::string& s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}
bool starts(const std::string& s, const char* p) { return s.compare(0, strlen(p), p) == 0; }
double must_f64(const std::string& s) {
  double v;
  if (!parse_rust_f64(s, &v)) throw LoadError("invalid float literal");
  return v;
}
std::vector<Tri> load_stl(const std::string& bytes) {
  if (bytes.size() < 80) throw LoadError("failed to fill whole buffer");
  std::string header = bytes.substr(0, 80);
  size_t a = 0;
  while (a < header.size() && isspace((unsigned char)header[a])) a++;
  bool ascii = false;
  if (header.compare(a, 5, "solid") == 0) {
    auto ls = lines_of(bytes);
    for (size_t i = 0; i < ls.size() && i < 10; i++) {
      std::string t = trim(ls[i]);
      if (starts(t, "facet normal") || t == "outer loop" || t == "endloop") { ascii = true; break; }
    }
  }
  std::vector<Tri> out;
  if (ascii) {
    auto ls = lines_of(bytes);
    size_t i = 0;
    while (i < ls.size()) {
      std::string line = trim(ls[i]);
      if (starts(line, "facet normal")) {
        auto parts = words(line);
        if (parts.size() != 5) throw LoadError("Invalid facet normal format");
        for (int k = 2; k < 5; k++) must_f64(parts[k]);
        i++;
        if (i >= ls.size() || trim(ls[i]) != "outer loop") throw LoadError("Expected 'outer loop' after facet normal");
        Tri t;
        for (int j = 0; j < 3; j++) {
          i++;
          if (i >= ls.size()) throw LoadError("Unexpected end of file while reading vertex");
          std::string vl = trim(ls[i]);
          if (!starts(vl, "vertex")) throw LoadError("Expected vertex line");
          auto vp = words(vl);
          if (vp.size() != 4) throw LoadError("Invalid vertex format");
          t.v[j] = {must_f64(vp[1]), must_f64(vp[2]), must_f64(vp[3])};
        }
        i++;
        if (i >= ls.size() || trim(ls[i]) != "endloop") throw LoadError("Expected 'endloop'");
        i++;
        if (i >= ls.size() || trim(ls[i]) != "endfacet") throw LoadError("Expected 'endfacet'");
        out.push_back(t);
      }
      i++;
    }
    return out;
  }
  if (bytes.size() < 84) throw LoadError("Binary STL too short");
  const unsigned char* b = (const unsigned char*)bytes.data();
  size_t n = (size_t)b[80] | ((size_t)b[81] << 8) | ((size_t)b[82] << 16) | ((size_t)b[83] << 24);
  size_t expected = 84 + n * 50;
  if (bytes.size() < expected)
    throw LoadError("Binary STL size mismatch: expected " + std::to_string(expected) + ", got " +
                    std::to_string(bytes.size()));
  out.resize(n);
  auto f32 = [&](size_t off) {
    uint32_t u = (uint32_t)b[off] | ((uint32_t)b[off + 1] << 8) | ((uint32_t)b[off + 2] << 16) |
                 ((uint32_t)b[off + 3] << 24);
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
  };
  // 50-byte facets: normal (unused by rendering), three vertices, attribute
  auto parse = [&](size_t k0, size_t k1) {
    for (size_t k = k0; k < k1; k++) {
      const size_t off = 84 + 50 * k + 12;
      for (int i = 0; i < 3; i++) out[k].v[i] = {f32(off + 12 * i), f32(off + 12 * i + 4), f32(off + 12 * i + 8)};
    }
  };
  const size_t parts = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), n / 65536 + 1);
  std::vector<std::thread> th;
  for (size_t p = 1; p < parts; p++) th.emplace_back(parse, n * p / parts, n * (p + 1) / parts);
  parse(0, n / parts);
  for (auto& t : th) t.join();
  return out;
}

// ----------------------------------------------------------- k-d tree -----
// KdTree::new(tris, 16, 10) / build_recursive (src/mesh.rs:75-197),
// emitted in preorder.  Subtrees above a size threshold build in parallel
// and are stitched together afterwards, which keeps the preorder layout.
struct KdOut {
  std::vector<rt_kd_node_desc> nodes;
  std::vector<int32_t> idx;
};
struct KdBuilder {
  const std::vector<Tri>& t;
  std::vector<V> tmin, tmax, center;
  explicit KdBuilder(const std::vector<Tri>& tris) : t(tris) {
    size_t n = t.size();
    tmin.resize(n);
    tmax.resize(n);
    center.resize(n);
    for (size_t i = 0; i < n; i++) {
      V mn = t[i].v[0], mx = t[i].v[0];
      for (int k = 1; k < 3; k++) {
        mn = {rmin(mn.x, t[i].v[k].x), rmin(mn.y, t[i].v[k].y), rmin(mn.z, t[i].v[k].z)};
        mx = {rmax(mx.x, t[i].v[k].x), rmax(mx.y, t[i].v[k].y), rmax(mx.z, t[i].v[k].z)};
      }
      tmin[i] = mn;
      tmax[i] = mx;
      center[i] = (t[i].v[0] + t[i].v[1] + t[i].v[2]) / 3.0;  // Triangle::center
    }
  }
  void bounds(const std::vector<int32_t>& idx, double bmin[3], double bmax[3]) const {
    if (idx.empty()) {
      for (int k = 0; k < 3; k++) bmin[k] = bmax[k] = 0.0;
      return;
    }
    double mn[3] = {INF, INF, INF}, mx[3] = {-INF, -INF, -INF};
    for (int32_t i : idx)
      for (int k = 0; k < 3; k++) {
        mn[k] = rmin(mn[k], tmin[i][k]);
        mx[k] = rmax(mx[k], tmax[i][k]);
      }
    for (int k = 0; k < 3; k++) { bmin[k] = mn[k]; bmax[k] = mx[k]; }
  }
  void build(std::vector<int32_t> idx, const double bmin[3], const double bmax[3], int depth, KdOut& out) const {
    rt_kd_node_desc nd{};
    for (int k = 0; k < 3; k++) { nd.bounds_min[k] = bmin[k]; nd.bounds_max[k] = bmax[k]; }
    if (depth >= 16 || idx.size() <= 10) {
      nd.axis = -1;
      nd.first = (int32_t)out.idx.size();
      nd.count = (int32_t)idx.size();
      out.idx.insert(out.idx.end(), idx.begin(), idx.end());
      out.nodes.push_back(nd);
      return;
    }
    int axis = depth % 3;
    std::vector<std::pair<double, int32_t>> pos;
    pos.reserve(idx.size());
    for (int32_t i : idx) {
      double c = center[i][axis];
      if (std::isnan(c)) throw LoadError("called `Option::unwrap()` on a `None` value");
      pos.emplace_back(c, i);
    }
    std::stable_sort(pos.begin(), pos.end(), [](const std::pair<double, int32_t>& a,
                                                const std::pair<double, int32_t>& b) { return a.first < b.first; });
    double split = pos[pos.size() / 2].first;
    std::vector<int32_t> l, r;
    for (auto& pr : pos) {
      if (tmin[pr.second][axis] <= split) l.push_back(pr.second);
      if (tmax[pr.second][axis] > split) r.push_back(pr.second);
    }
    if (l.empty()) { l.push_back(r.back()); r.pop_back(); }
    else if (r.empty()) { r.push_back(l.back()); l.pop_back(); }
    double lmin[3], lmax[3], rmn[3], rmx[3];
    bounds(l, lmin, lmax);
    bounds(r, rmn, rmx);
    nd.axis = axis;
    nd.split = split;
    size_t me = out.nodes.size();
    out.nodes.push_back(nd);
    if (depth < 4 && l.size() + r.size() > 20000) {
      KdOut ro;
      auto fut = std::async(std::launch::async, [&]() { build(std::move(r), rmn, rmx, depth + 1, ro); });
      build(std::move(l), lmin, lmax, depth + 1, out);
      fut.get();
      int32_t node_off = (int32_t)out.nodes.size(), idx_off = (int32_t)out.idx.size();
      out.nodes[me].right = node_off;
      for (auto n : ro.nodes) {
        if (n.axis >= 0) n.right += node_off;
        else n.first += idx_off;
        out.nodes.push_back(n);
      }
      out.idx.insert(out.idx.end(), ro.idx.begin(), ro.idx.end());
    } else {
      build(std::move(l), lmin, lmax, depth + 1, out);
      out.nodes[me].right = (int32_t)out.nodes.size();
      build(std::move(r), rmn, rmx, depth + 1, out);
    }
  }
};

void make_mesh(const std::vector<Tri>& tris, HostMesh* m, const KdBuildHook* kd) {
  m->vertices.resize(tris.size() * 9);
  // Mesh::compute_bounds (src/mesh.rs:1017-1033)
  if (tris.empty()) {
    for (int k = 0; k < 3; k++) m->bmin[k] = m->bmax[k] = 0.0;
    return;
  }
  // the vertex array and the bounds over contiguous ranges on host threads;
  // the ranges' bounds combine in range order, which is the sequential
  // fold (rmin/rmax keep the first of equal operands)
  const size_t n = tris.size();
  const size_t parts = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), n / 65536 + 1);
  std::vector<double> pmn(3 * parts, INF), pmx(3 * parts, -INF);
  auto work = [&](size_t p) {
    for (size_t i = n * p / parts; i < n * (p + 1) / parts; i++)
      for (int v = 0; v < 3; v++)
        for (int k = 0; k < 3; k++) {
          const double c = tris[i].v[v][k];
          m->vertices[9 * i + 3 * v + k] = c;
          pmn[3 * p + k] = rmin(pmn[3 * p + k], c);
          pmx[3 * p + k] = rmax(pmx[3 * p + k], c);
        }
  };
  std::vector<std::thread> th;
  for (size_t p = 1; p < parts; p++) th.emplace_back(work, p);
  work(0);
  for (auto& t : th) t.join();
  double mn[3] = {INF, INF, INF}, mx[3] = {-INF, -INF, -INF};
  for (size_t p = 0; p < parts; p++)
    for (int k = 0; k < 3; k++) {
      mn[k] = rmin(mn[k], pmn[3 * p + k]);
      mx[k] = rmax(mx[k], pmx[3 * p + k]);
    }
  for (int k = 0; k < 3; k++) { m->bmin[k] = mn[k]; m->bmax[k] = mx[k]; }
  if (kd && kd->build && tris.size() >= kd->min_triangles) {
    std::string e = kd->build(m->vertices.data(), tris.size(), &m->nodes, &m->tri_index);
    if (!e.empty()) throw LoadError(e);
    return;
  }
  KdBuilder kb(tris);
  std::vector<int32_t> all(tris.size());
  for (size_t i = 0; i < tris.size(); i++) all[i] = (int32_t)i;
  double bmin[3], bmax[3];
  kb.bounds(all, bmin, bmax);
  KdOut out;
  kb.build(std::move(all), bmin, bmax, 0, out);
  m->nodes = std::move(out.nodes);
  m->tri_index = std::move(out.idx);
}

// ----------------------------------------------------------- scene -----
struct MatIn {
  std::string color;
  double ambient, diffuse, specular, shininess;
  bool has_refl = false;
  double refl = 0;
  int texture = 0;
  std::string line_color;
  double line_width = 0, cell_size = 0;
  std::shared_ptr<MatIn> b;
};
MatIn parse_material(const J& j) {
  MatIn m;
  m.color = str(req(j, "color"));
  m.ambient = f64(req(j, "ambient"));
  m.diffuse = f64(req(j, "diffuse"));
  m.specular = f64(req(j, "specular"));
  m.shininess = f64(req(j, "shininess"));
  if (const J* r = opt(j, "reflectivity")) { m.has_refl = true; m.refl = f64(*r); }
  if (const J* t = opt(j, "texture")) {
    std::string ty = str(req(*t, "type"));
    if (ty == "grid") {
      m.texture = 1;
      m.line_color = str(req(*t, "line_color"));
      m.line_width = f64(req(*t, "line_width"));
      m.cell_size = f64(req(*t, "cell_size"));
    } else if (ty == "checkerboard") {
      m.texture = 2;
      m.b = std::make_shared<MatIn>(parse_material(req(*t, "material_b")));
    } else {
      throw LoadError("unknown variant `" + ty + "`, expected `grid` or `checkerboard`");
    }
  }
  return m;
}
void color_or(const std::string& s, const double fb[3], double out[3]) {
  if (!hex_to_color(s, out, nullptr))
    for (int k = 0; k < 3; k++) out[k] = fb[k];
}

struct ObjIn {
  int kind;
  V a{}, b{};
  double radius = 0;
  MatIn mat;
  bool has_transform = false;
  std::vector<std::string> transform;
  std::string filename;
};

// The scene's "objects" array (src/scene.rs:55-96 deserialisation).
std::vector<ObjIn> parse_objects(const J& j) {
  std::vector<ObjIn> objs;
  const J& oa = req(j, "objects");
  if (oa.k != J::ARR) throw LoadError("invalid type: expected a sequence");
  for (const J& o : oa.a) {
    ObjIn ob;
    std::string k = str(req(o, "kind"));
    if (k == "sphere") { ob.kind = RT_OBJ_SPHERE; ob.a = vec3(req(o, "center")); ob.radius = f64(req(o, "radius")); }
    else if (k == "plane") { ob.kind = RT_OBJ_PLANE; ob.a = vec3(req(o, "point")); ob.b = vec3(req(o, "normal")); }
    else if (k == "cube") { ob.kind = RT_OBJ_CUBE; ob.a = vec3(req(o, "center")); ob.b = vec3(req(o, "size")); }
    else if (k == "mesh") { ob.kind = RT_OBJ_MESH; ob.filename = str(req(o, "filename")); }
    else throw LoadError("unknown variant `" + k + "`, expected one of `sphere`, `plane`, `cube`, `mesh`");
    ob.mat = parse_material(req(o, "material"));
    if (const J* tr = opt(o, "transform")) {
      if (tr->k != J::ARR) throw LoadError("invalid type: expected a sequence");
      ob.has_transform = true;
      for (auto& e : tr->a) ob.transform.push_back(str(e));
    }
    objs.push_back(std::move(ob));
  }
  return objs;
}

}  // namespace

// --------------------------------------------------------- public API -----
std::string kd_build_host(const double* vertices, size_t n, std::vector<rt_kd_node_desc>* nodes,
                          std::vector<int32_t>* idx) {
  nodes->clear();
  idx->clear();
  if (n == 0) return "";  // make_mesh builds no tree for an empty mesh
  std::vector<Tri> tris(n);
  for (size_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) tris[i].v[k] = {vertices[9 * i + 3 * k], vertices[9 * i + 3 * k + 1], vertices[9 * i + 3 * k + 2]};
  try {
    KdBuilder kb(tris);
    std::vector<int32_t> all(n);
    for (size_t i = 0; i < n; i++) all[i] = (int32_t)i;
    double bmin[3], bmax[3];
    kb.bounds(all, bmin, bmax);
    KdOut out;
    kb.build(std::move(all), bmin, bmax, 0, out);
    *nodes = std::move(out.nodes);
    *idx = std::move(out.idx);
  } catch (const std::exception& e) {
    return e.what();
  }
  return "";
}

bool hex_to_color(const std::string& in, double out[3], std::string* err) {
  size_t k = 0;
  while (k < in.size() && in[k] == '#') k++;
  std::string hex = in.substr(k);
  if (hex.size() != 6) {
    if (err) *err = "Invalid hex color format";
    return false;
  }
  for (int bpos : {2, 4})
    if (((unsigned char)hex[bpos] & 0xC0) == 0x80) {
      if (err) *err = "Invalid hex color";
      return false;
    }
  unsigned vals[3];
  for (int c = 0; c < 3; c++) {
    std::string part = hex.substr(2 * c, 2);
    size_t i = (part.size() > 1 && part[0] == '+') ? 1 : 0;  // from_str_radix accepts '+'
    unsigned v = 0;
    bool ok = i < part.size();
    for (; ok && i < part.size(); i++) {
      char ch = part[i];
      int d = (ch >= '0' && ch <= '9') ? ch - '0'
              : (ch >= 'a' && ch <= 'f') ? ch - 'a' + 10
              : (ch >= 'A' && ch <= 'F') ? ch - 'A' + 10 : -1;
      if (d < 0) ok = false;
      else v = v * 16 + d;
    }
    if (!ok) {
      if (err) *err = "Invalid hex color";
      return false;
    }
    vals[c] = v;
  }
  for (int c = 0; c < 3; c++) out[c] = (double)vals[c] / 255.0;
  return true;
}

bool read_text_file(const std::string& path, std::string* out, std::string* err) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    *err = "No such file or directory (os error 2): " + path;
    return false;
  }
  const std::streamoff size = f.tellg();
  if (size >= 0) {  // one sized read (a 100 MB STL is read once, not copied through a stream)
    out->resize((size_t)size);
    f.seekg(0);
    if (size == 0 || f.read(&(*out)[0], size)) return true;
  }
  f.clear();
  f.seekg(0);
  std::stringstream ss;
  ss << f.rdbuf();
  *out = ss.str();
  return true;
}

std::string parent_dir(const std::string& path) {
  size_t k = path.find_last_of('/');
  if (k == std::string::npos) return "";
  if (k == 0) return "/";
  return path.substr(0, k);
}

void HostScene::finalize() {
  mesh_descs.clear();
  for (auto& m : meshes) {
    rt_mesh_desc d{};
    d.vertices = m->vertices.data();
    d.n_triangles = (int64_t)(m->vertices.size() / 9);
    for (int k = 0; k < 3; k++) { d.bounds_min[k] = m->bmin[k]; d.bounds_max[k] = m->bmax[k]; }
    d.nodes = m->nodes.empty() ? nullptr : m->nodes.data();
    d.n_nodes = (int64_t)m->nodes.size();
    d.tri_index = m->tri_index.empty() ? nullptr : m->tri_index.data();
    d.n_tri_index = (int64_t)m->tri_index.size();
    mesh_descs.push_back(d);
  }
  desc.objects = objects.data();
  desc.n_objects = (int32_t)objects.size();
  desc.materials = materials.data();
  desc.n_materials = (int32_t)materials.size();
  desc.lights = lights.data();
  desc.n_lights = (int32_t)lights.size();
  desc.meshes = mesh_descs.data();
  desc.n_meshes = (int32_t)mesh_descs.size();
  desc.render_error = render_error.empty() ? nullptr : render_error.c_str();
}

bool load_scene_json(const std::string& text, const std::string& base_dir, HostScene* hs, std::string* err,
                     const KdBuildHook* kd) {
  try {
    J j = parse_json(text);
    if (j.k != J::OBJ) throw LoadError("invalid type: expected struct Scene");
    rt_scene_desc& d = hs->desc;
    d = rt_scene_desc{};
    // camera (src/scene.rs:33-46)
    const J& cam = req(j, "camera");
    rt_camera_config& cc = d.camera;
    std::string kind = str(req(cam, "kind"));
    snprintf(cc.kind, sizeof cc.kind, "%s", kind.c_str());
    if (kind.size() >= sizeof cc.kind) snprintf(cc.kind, sizeof cc.kind, "%s", "<unsupported>");
    V p = vec3(req(cam, "position")), t = vec3(req(cam, "target")), u = vec3(req(cam, "up"));
    for (int k = 0; k < 3; k++) { cc.position[k] = p[k]; cc.target[k] = t[k]; cc.up[k] = u[k]; }
    cc.width = f64(req(cam, "width"));
    cc.height = f64(req(cam, "height"));
    if (const J* f = opt(cam, "fov")) { cc.has_fov = 1; cc.fov = f64(*f); }
    if (const J* f = opt(cam, "grid_pitch")) { cc.has_grid_pitch = 1; cc.grid_pitch = f64(*f); }
    if (const J* f = opt(cam, "grid_thickness")) { cc.has_grid_thickness = 1; cc.grid_thickness = f64(*f); }
    if (const J* f = opt(cam, "grid_color")) cc.grid_color_state = hex_to_color(str(*f), cc.grid_color, nullptr) ? 1 : 2;

    std::vector<ObjIn> objs = parse_objects(j);
    const J& la = req(j, "lights");
    if (la.k != J::ARR) throw LoadError("invalid type: expected a sequence");
    static const double WHITE[3] = {1, 1, 1}, BLACK[3] = {0, 0, 0}, GREY[3] = {0.5, 0.5, 0.5};
    hs->lights.clear();
    for (const J& l : la.a) {
      rt_light_desc ld{};
      V lp = vec3(req(l, "position"));
      for (int k = 0; k < 3; k++) ld.position[k] = lp[k];
      color_or(str(req(l, "color")), WHITE, ld.color);
      ld.intensity = f64(req(l, "intensity"));
      if (const J* dm = opt(l, "diameter")) { ld.has_diameter = 1; ld.diameter = f64(*dm); }
      hs->lights.push_back(ld);
    }
    const J& ss = req(j, "scene_settings");
    const J& amb = req(ss, "ambient_illumination");
    color_or(str(req(amb, "color")), WHITE, d.ambient_color);
    d.ambient_intensity = f64(req(amb, "intensity"));
    if (const J* f = opt(ss, "fog")) {
      d.has_fog = 1;
      color_or(str(req(*f, "color")), GREY, d.fog_color);
      d.fog_density = f64(req(*f, "density"));
      d.fog_start = f64(req(*f, "start"));
      d.fog_end = f64(req(*f, "end"));
    }
    std::string bg_error;
    bool has_bg = false;
    std::string bg;
    if (const J* b = opt(ss, "background_color")) { has_bg = true; bg = str(*b); }
    rt_outline_config& oc = d.outline;
    oc = rt_outline_config{};
    oc.depth_weight = 1.0;
    oc.normal_weight = 1.0;
    oc.threshold = 0.1;
    oc.line_thickness = 1.0;
    std::string outline_color_error;
    if (const J* o = opt(ss, "outline")) {
      bool en = boolean(req(*o, "enabled"));
      std::string ocol = "#000000";
      if (const J* v = o->get("depth_weight")) oc.depth_weight = f64(*v);
      if (const J* v = o->get("normal_weight")) oc.normal_weight = f64(*v);
      if (const J* v = o->get("threshold")) oc.threshold = f64(*v);
      if (const J* v = o->get("color")) ocol = str(*v);
      if (const J* v = o->get("thickness")) oc.line_thickness = f64(*v);
      if (const J* v = o->get("use_8_neighbors")) oc.use_8_neighbors = boolean(*v) ? 1 : 0;
      // extension, no key of the reference's schema (serde ignores it there)
      if (const J* v = o->get("object_id_weight")) oc.object_id_weight = f64(*v);
      if (en) {
        std::string e2;
        if (hex_to_color(ocol, oc.edge_color, &e2)) {
          oc.enabled = 1;
          d.has_outline = 1;
        } else {
          oc.enabled = 0;
          d.has_outline = 2;  // get_outline_config would fail with this colour
        }
      }
    }
    // load_mesh_data (src/scene.rs:483-505), after deserialisation
    std::vector<std::vector<Tri>> raw(objs.size());
    for (size_t i = 0; i < objs.size(); i++) {
      if (objs[i].kind != RT_OBJ_MESH) continue;
      const std::string& fn = objs[i].filename;
      std::string path = (base_dir.empty() || (!fn.empty() && fn[0] == '/')) ? fn : base_dir + "/" + fn;
      std::string bytes, e2;
      if (!read_text_file(path, &bytes, &e2)) throw LoadError(e2);
      raw[i] = load_stl(bytes);
    }
    // World build (src/renderer.rs:138-317)
    hs->objects.clear();
    hs->materials.clear();
    hs->meshes.clear();
    hs->render_error.clear();
    for (size_t i = 0; i < objs.size(); i++) {
      const ObjIn& o = objs[i];
      M4 tm;
      bool ht = o.has_transform && parse_transforms(o.transform, &tm);
      rt_object_desc od{};
      od.kind = o.kind;
      od.material = (int32_t)i;
      if (o.kind == RT_OBJ_SPHERE) {
        V c = o.a;
        double r = o.radius;
        if (ht) {
          c = xform_point(tm, c);
          double sx = norm({tm.m[0][0], tm.m[1][0], tm.m[2][0]});
          double sy = norm({tm.m[0][1], tm.m[1][1], tm.m[2][1]});
          double sz = norm({tm.m[0][2], tm.m[1][2], tm.m[2][2]});
          r *= rmax(rmax(sx, sy), sz);
        }
        for (int k = 0; k < 3; k++) od.a[k] = c[k];
        od.radius = r;
      } else if (o.kind == RT_OBJ_PLANE) {
        V pp = o.a, nn = o.b;
        if (ht) {
          pp = xform_point(tm, pp);
          M4 inv;
          if (inverse4(tm, &inv)) {
            M4 it;
            for (int a = 0; a < 4; a++)
              for (int b = 0; b < 4; b++) it.m[a][b] = inv.m[b][a];
            nn = xform_vec(it, nn);
          }
        }
        nn = normalize(nn);
        for (int k = 0; k < 3; k++) { od.a[k] = pp[k]; od.b[k] = nn[k]; }
      } else if (o.kind == RT_OBJ_CUBE) {
        for (int k = 0; k < 3; k++) { od.a[k] = o.a[k]; od.b[k] = o.b[k]; }
        if (ht) {
          od.has_transform = 1;
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) od.transform[4 * a + b] = tm.m[a][b];
        }
      } else {
        std::vector<Tri> tris = std::move(raw[i]);  // each mesh object reads its own file
        if (ht)
          for (auto& tr : tris)
            for (int k = 0; k < 3; k++) tr.v[k] = xform_point(tm, tr.v[k]);
        auto hm = std::make_unique<HostMesh>();
        make_mesh(tris, hm.get(), kd);
        od.mesh = (int32_t)hs->meshes.size();
        hs->meshes.push_back(std::move(hm));
      }
      std::string ce;
      double col[3];
      if (!hex_to_color(o.mat.color, col, &ce) && hs->render_error.empty()) hs->render_error = ce;
      rt_material_desc md{};
      for (int k = 0; k < 3; k++) md.color[k] = col[k];
      md.ambient = o.mat.ambient;
      md.diffuse = o.mat.diffuse;
      md.specular = o.mat.specular;
      md.shininess = o.mat.shininess;
      md.has_reflectivity = o.mat.has_refl ? 1 : 0;
      md.reflectivity = o.mat.refl;
      md.texture = o.mat.texture;
      if (o.mat.texture == 1) {
        color_or(o.mat.line_color, BLACK, md.grid_line_color);
        md.grid_line_width = o.mat.line_width;
        md.grid_cell_size = o.mat.cell_size;
      } else if (o.mat.texture == 2) {
        color_or(o.mat.b->color, WHITE, md.checker_color);
        md.checker_ambient = o.mat.b->ambient;
        md.checker_diffuse = o.mat.b->diffuse;
        md.checker_specular = o.mat.b->specular;
        md.checker_shininess = o.mat.b->shininess;
      }
      hs->objects.push_back(od);
      hs->materials.push_back(md);
    }
    if (has_bg) {
      std::string be;
      if (!hex_to_color(bg, d.background, &be) && hs->render_error.empty()) hs->render_error = be;
    }
    hs->finalize();
    return true;
  } catch (const std::exception& e) {
    *err = e.what();
    return false;
  }
}

// Camera::from_config (src/camera.rs:23-153)
bool make_camera(const rt_camera_config& cfg, double aspect, CameraBasis* c, std::string* err) {
  V origin{cfg.position[0], cfg.position[1], cfg.position[2]};
  V target{cfg.target[0], cfg.target[1], cfg.target[2]};
  V up{cfg.up[0], cfg.up[1], cfg.up[2]};
  V w = normalize(origin - target);
  V u = normalize(cross(up, w));
  V v = cross(w, u);
  V vd = normalize(V{-w.x, -w.y, -w.z});
  if (cfg.grid_color_state == 2) {
    *err = "Invalid hex color";
    return false;
  }
  std::string kind = cfg.kind;
  V hor, ver, llc;
  if (kind == "ortho") {
    double vh = cfg.height;
    double vw = rmax(cfg.width, vh * aspect);
    hor = vw * u;
    ver = vh * v;
    llc = origin - hor / 2.0 - ver / 2.0;
    c->persp = 0;
  } else if (kind == "perspective") {
    double fov = cfg.has_fov ? cfg.fov : 45.0;
    if (fov <= 0.0 || fov >= 180.0) {
      *err = "Field of view must be between 0 and 180 degrees";
      return false;
    }
    double focal = 1.0;
    double theta = to_radians(fov);
    double hh = std::tan(theta / 2.0);
    double hw = aspect * hh;
    double vh = 2.0 * hh * focal;
    double vw = 2.0 * hw * focal;
    hor = vw * u;
    ver = vh * v;
    V center = origin + focal * vd;
    llc = center - hor / 2.0 - ver / 2.0;
    c->persp = 1;
  } else {
    *err = "Unsupported camera type: " + kind;
    return false;
  }
  for (int k = 0; k < 3; k++) {
    c->origin[k] = origin[k];
    c->horizontal[k] = hor[k];
    c->vertical[k] = ver[k];
    c->llc[k] = llc[k];
    c->view_dir[k] = vd[k];
    c->grid_color[k] = cfg.grid_color[k];
  }
  // get_grid_color's preconditions (src/camera.rs:172-184)
  c->grid_enabled = (!c->persp && cfg.has_grid_pitch && cfg.grid_color_state == 1 && cfg.has_grid_thickness &&
                     cfg.grid_pitch > 0.0 && cfg.grid_thickness > 0.0)
                        ? 1
                        : 0;
  c->grid_pitch = cfg.grid_pitch;
  c->grid_half_thickness = cfg.grid_thickness / 2.0;
  return true;
}


// Scene::compute_finite_bounds (src/scene.rs:538-690) and
// AutoCamera::generate_cameras (src/auto_camera.rs:9-130).
bool auto_cameras(const std::string& text, const std::string& base_dir, rt_camera_config out[4], std::string* err) {
  try {
    J j = parse_json(text);
    if (j.k != J::OBJ) throw LoadError("invalid type: expected struct Scene");
    std::vector<ObjIn> objs = parse_objects(j);
    bool have = false;
    V mn{}, mx{};
    auto grow = [&](V a, V b) {
      if (!have) {
        mn = a;
        mx = b;
        have = true;
        return;
      }
      mn = {rmin(mn.x, a.x), rmin(mn.y, a.y), rmin(mn.z, a.z)};
      mx = {rmax(mx.x, b.x), rmax(mx.y, b.y), rmax(mx.z, b.z)};
    };
    for (const ObjIn& o : objs) {
      M4 tm;
      bool ht = o.has_transform && parse_transforms(o.transform, &tm);
      if (o.kind == RT_OBJ_SPHERE) {
        V c = o.a;
        double r = o.radius;
        if (ht) {
          c = xform_point(tm, c);
          double sx = norm({tm.m[0][0], tm.m[1][0], tm.m[2][0]});
          double sy = norm({tm.m[0][1], tm.m[1][1], tm.m[2][1]});
          double sz = norm({tm.m[0][2], tm.m[1][2], tm.m[2][2]});
          r *= rmax(rmax(sx, sy), sz);
        }
        V rv{r, r, r};
        grow(c - rv, c + rv);
      } else if (o.kind == RT_OBJ_CUBE) {
        // Cube::bounds (src/ray.rs:228-262)
        V h = o.b / 2.0;
        M4 inv;
        bool oriented = ht;
        if (ht && inverse4(tm, &inv)) {
          bool ident = true;
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) ident = ident && inv.m[a][b] == (a == b ? 1.0 : 0.0);
          oriented = !ident;
        } else if (ht) {
          oriented = false;  // try_inverse failed: the cube keeps the identity
        }
        if (!oriented) {
          grow(o.a - h, o.a + h);
        } else {
          const double INF = std::numeric_limits<double>::infinity();
          V cmn{INF, INF, INF}, cmx{-INF, -INF, -INF};
          for (int k = 0; k < 8; k++) {
            V corner{(k & 4) ? h.x : -h.x, (k & 2) ? h.y : -h.y, (k & 1) ? h.z : -h.z};
            V w = o.a + xform_point(tm, corner);
            cmn = {rmin(cmn.x, w.x), rmin(cmn.y, w.y), rmin(cmn.z, w.z)};
            cmx = {rmax(cmx.x, w.x), rmax(cmx.y, w.y), rmax(cmx.z, w.z)};
          }
          grow(cmn, cmx);
        }
      } else if (o.kind == RT_OBJ_MESH) {
        const std::string& fn = o.filename;
        std::string path = (base_dir.empty() || (!fn.empty() && fn[0] == '/')) ? fn : base_dir + "/" + fn;
        std::string bytes, e2;
        if (!read_text_file(path, &bytes, &e2)) throw LoadError(e2);
        std::vector<Tri> tris = load_stl(bytes);
        if (tris.empty()) continue;
        // Mesh::bounds (src/mesh.rs:26-36)
        V bmn = tris[0].v[0], bmx = tris[0].v[0];
        for (const Tri& t : tris)
          for (int k = 0; k < 3; k++) {
            bmn = {rmin(bmn.x, t.v[k].x), rmin(bmn.y, t.v[k].y), rmin(bmn.z, t.v[k].z)};
            bmx = {rmax(bmx.x, t.v[k].x), rmax(bmx.y, t.v[k].y), rmax(bmx.z, t.v[k].z)};
          }
        if (ht) {
          V c0 = xform_point(tm, {bmn.x, bmn.y, bmn.z});
          V tmn = c0, tmx = c0;
          for (int k = 1; k < 8; k++) {
            V corner{(k & 4) ? bmx.x : bmn.x, (k & 2) ? bmx.y : bmn.y, (k & 1) ? bmx.z : bmn.z};
            V w = xform_point(tm, corner);
            tmn = {rmin(tmn.x, w.x), rmin(tmn.y, w.y), rmin(tmn.z, w.z)};
            tmx = {rmax(tmx.x, w.x), rmax(tmx.y, w.y), rmax(tmx.z, w.z)};
          }
          grow(tmn, tmx);
        } else {
          grow(bmn, bmx);
        }
      }
    }
    if (!have) throw LoadError("Scene has no finite objects to compute bounds");
    V c{(mn.x + mx.x) / 2.0, (mn.y + mx.y) / 2.0, (mn.z + mx.z) / 2.0};
    V size = mx - mn;
    const double margin = 1.15;
    double vw = rmax(rmax(size.x, size.y), size.z) * margin;
    double dist = vw * 2.0;
    auto ortho = [&](rt_camera_config* cc, V pos, V up) {
      *cc = rt_camera_config{};
      snprintf(cc->kind, sizeof cc->kind, "%s", "ortho");
      double pp[3] = {pos.x, pos.y, pos.z}, tt[3] = {c.x, c.y, c.z}, uu[3] = {up.x, up.y, up.z};
      for (int k = 0; k < 3; k++) {
        cc->position[k] = pp[k];
        cc->target[k] = tt[k];
        cc->up[k] = uu[k];
      }
      cc->width = vw;
      cc->height = vw;
    };
    ortho(&out[0], {c.x, c.y - dist, c.z}, {0, 0, 1});  // left
    ortho(&out[1], {c.x - dist, c.y, c.z}, {0, 0, 1});  // front
    ortho(&out[2], {c.x, c.y, c.z + dist}, {0, 1, 0});  // top
    // perspective: 50 degree FOV, 35 degrees down, along the +x +y diagonal
    double maxd = rmax(rmax(size.x, size.y), size.z) * margin;
    double fov_rad = to_radians(50.0);
    double dfov = maxd / std::tan(fov_rad / 2.0);
    double xy = to_radians(45.0), down = to_radians(35.0);
    double hd = dfov * std::cos(down);
    rt_camera_config& pc = out[3];
    pc = rt_camera_config{};
    snprintf(pc.kind, sizeof pc.kind, "%s", "perspective");
    double pp[3] = {c.x + hd * std::cos(xy), c.y + hd * std::sin(xy), c.z + dfov * std::sin(down)};
    double tt[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; k++) {
      pc.position[k] = pp[k];
      pc.target[k] = tt[k];
      pc.up[k] = k == 2 ? 1.0 : 0.0;
    }
    pc.width = 1.0;
    pc.height = 1.0;
    pc.has_fov = 1;
    pc.fov = 50.0;
    return true;
  } catch (const std::exception& e) {
    if (err) *err = e.what();
    return false;
  }
}

}  // namespace rtb
