// Native scene-file loader: toaster scene JSON with its glTF/GLB meshes, PNG base-colour textures
// and Radiance (.hdr) or PNG environment maps, validated as the reference loader validates them
// and packed into the GPU records of toaster_cuda.h.
//
//   reading and validation  crates/toaster-scene/src/loader.rs:534-971 (load_scene, build_scene),
//                           loader.rs:1541-1610 (box_triangles, validate_*),
//                           crates/toaster-scene/src/environment.rs:42-128 (EnvironmentMap::new/load),
//                           crates/toaster-scene/src/texture.rs:13-35 (Texture::new)
//   glTF import             crates/toaster-assets/src/gltf_loader.rs:11-233
//   packing                 crates/toaster-gpu/src/scene_upload.rs:79-294 (scene_to_gpu without the
//                           hierarchy: the library builds it on upload), :352-405 (make_camera,
//                           material_to_gpu), :412-475 (lights_to_gpu),
//                           environment.rs:244-278 (importance CDF)
//
// Arithmetic is f32 in the reference's operation order (glam's scalar order for vector and matrix
// products); the host compiler runs with -ffp-contract=off so nothing is fused. JSON numbers are
// parsed to the nearest double and rounded to f32, as serde_json does for every number of at most
// 19 significant digits and decimal exponent within +-22 (all of the reference's scene files).
// Animation tracks, physics, triggers, spawn points and event reactions do not change the packed
// records and are skipped without validation.
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../../include/toaster_cuda.h"

namespace {

struct LoadError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

[[noreturn]] void bail(const std::string& message) { throw LoadError(message); }

constexpr float kF32Epsilon = 1.1920929e-7f;
constexpr float kPiF = 3.14159265358979323846f;

// ---------------------------------------------------------------------------------- f32 vectors
struct V3 {
  float x = 0.0f, y = 0.0f, z = 0.0f;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
float length(V3 a) { return std::sqrt(dot(a, a)); }
V3 normalize(V3 a) { return a * (1.0f / length(a)); }
bool finite(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

// glam's normalize_or_zero: the vector times 1/|v| when that reciprocal is finite and positive.
V3 normalize_or_zero(V3 a) {
  const float rcp = 1.0f / length(a);
  if (std::isfinite(rcp) && rcp > 0.0f) return a * rcp;
  return {};
}

// Column-major 4x4 (glam Mat4 / the glTF node matrix layout).
struct M4 {
  float c[4][4];  // c[column][row]
};

M4 identity4() {
  M4 m{};
  for (int i = 0; i < 4; ++i) m.c[i][i] = 1.0f;
  return m;
}

// a * b, column j = ((a.x * b[j].x + a.y * b[j].y) + a.z * b[j].z) + a.w * b[j].w.
M4 mul(const M4& a, const M4& b) {
  M4 r{};
  for (int j = 0; j < 4; ++j)
    for (int row = 0; row < 4; ++row) {
      float v = a.c[0][row] * b.c[j][0];
      v = v + a.c[1][row] * b.c[j][1];
      v = v + a.c[2][row] * b.c[j][2];
      v = v + a.c[3][row] * b.c[j][3];
      r.c[j][row] = v;
    }
  return r;
}

// glam Mat4::transform_point3: ((x_axis * p.x + y_axis * p.y) + z_axis * p.z) + w_axis.
V3 transform_point(const M4& m, V3 p) {
  float out[3];
  for (int row = 0; row < 3; ++row) {
    float v = m.c[0][row] * p.x;
    v = m.c[1][row] * p.y + v;
    v = m.c[2][row] * p.z + v;
    v = m.c[3][row] + v;
    out[row] = v;
  }
  return {out[0], out[1], out[2]};
}

// Mat3::from_mat4(m).inverse().transpose() as glam computes it: the columns are the cofactor
// crosses scaled by 1 / det.
struct M3 {
  V3 col[3];
};
M3 normal_matrix(const M4& m) {
  const V3 x{m.c[0][0], m.c[0][1], m.c[0][2]};
  const V3 y{m.c[1][0], m.c[1][1], m.c[1][2]};
  const V3 z{m.c[2][0], m.c[2][1], m.c[2][2]};
  const V3 t0 = cross(y, z), t1 = cross(z, x), t2 = cross(x, y);
  const float inv_det = 1.0f / dot(z, t2);
  return {{t0 * inv_det, t1 * inv_det, t2 * inv_det}};
}
V3 mul(const M3& m, V3 v) {
  V3 r = m.col[0] * v.x;
  r = r + m.col[1] * v.y;
  r = r + m.col[2] * v.z;
  return r;
}

// ---------------------------------------------------------------------------------------- JSON
struct Json {
  enum Kind : uint8_t { kNull, kBool, kNumber, kString, kArray, kObject };
  Kind kind = kNull;
  bool boolean = false;
  double number = 0.0;
  bool integral = false;   // integer text: no fraction, no exponent
  bool negative = false;
  bool overflow = false;   // integer magnitude above 2^64 - 1
  uint64_t magnitude = 0;
  std::string text;
  std::vector<Json> items;
  std::vector<std::pair<std::string, Json>> members;

  const Json* find(const char* key) const {
    for (const auto& m : members)
      if (m.first == key) return &m.second;
    return nullptr;
  }
};

class JsonParser {
 public:
  JsonParser(const char* data, size_t size, std::string what) : p_(data), end_(data + size), begin_(data), what_(std::move(what)) {}

  Json parse_document() {
    skip_ws();
    Json v = value(0);
    skip_ws();
    if (p_ != end_) fail("trailing characters");
    return v;
  }

 private:
  [[noreturn]] void fail(const char* why) const {
    size_t line = 1, col = 1;
    for (const char* q = begin_; q < p_ && q < end_; ++q) {
      if (*q == '\n') {
        ++line;
        col = 1;
      } else {
        ++col;
      }
    }
    bail(what_ + ": " + why + " at line " + std::to_string(line) + " column " + std::to_string(col));
  }

  void skip_ws() {
    while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
  }

  bool literal(const char* word) {
    const size_t n = std::strlen(word);
    if (size_t(end_ - p_) >= n && std::memcmp(p_, word, n) == 0) {
      p_ += n;
      return true;
    }
    return false;
  }

  Json value(int depth) {
    if (depth > 128) fail("recursion limit exceeded");
    if (p_ >= end_) fail("EOF while parsing a value");
    Json v;
    const char c = *p_;
    if (c == '{') {
      v.kind = Json::kObject;
      ++p_;
      skip_ws();
      if (p_ < end_ && *p_ == '}') {
        ++p_;
        return v;
      }
      for (;;) {
        skip_ws();
        if (p_ >= end_ || *p_ != '"') fail("key must be a string");
        std::string key = string();
        skip_ws();
        if (p_ >= end_ || *p_ != ':') fail("expected ':'");
        ++p_;
        skip_ws();
        for (const auto& m : v.members)
          if (m.first == key) fail(("duplicate field `" + key + "`").c_str());
        v.members.emplace_back(std::move(key), value(depth + 1));
        skip_ws();
        if (p_ < end_ && *p_ == ',') {
          ++p_;
          continue;
        }
        if (p_ < end_ && *p_ == '}') {
          ++p_;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = Json::kArray;
      ++p_;
      skip_ws();
      if (p_ < end_ && *p_ == ']') {
        ++p_;
        return v;
      }
      for (;;) {
        skip_ws();
        v.items.push_back(value(depth + 1));
        skip_ws();
        if (p_ < end_ && *p_ == ',') {
          ++p_;
          continue;
        }
        if (p_ < end_ && *p_ == ']') {
          ++p_;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = Json::kString;
      v.text = string();
      return v;
    }
    if (literal("true")) {
      v.kind = Json::kBool;
      v.boolean = true;
      return v;
    }
    if (literal("false")) {
      v.kind = Json::kBool;
      return v;
    }
    if (literal("null")) return v;
    if (c == '-' || (c >= '0' && c <= '9')) {
      number(v);
      return v;
    }
    fail("expected value");
  }

  static void put_utf8(std::string& out, uint32_t cp) {
    if (cp < 0x80) {
      out += char(cp);
    } else if (cp < 0x800) {
      out += char(0xC0 | (cp >> 6));
      out += char(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      out += char(0xE0 | (cp >> 12));
      out += char(0x80 | ((cp >> 6) & 0x3F));
      out += char(0x80 | (cp & 0x3F));
    } else {
      out += char(0xF0 | (cp >> 18));
      out += char(0x80 | ((cp >> 12) & 0x3F));
      out += char(0x80 | ((cp >> 6) & 0x3F));
      out += char(0x80 | (cp & 0x3F));
    }
  }

  uint32_t hex4() {
    if (end_ - p_ < 4) fail("EOF while parsing a string");
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) {
      const char h = *p_++;
      v <<= 4;
      if (h >= '0' && h <= '9') v |= uint32_t(h - '0');
      else if (h >= 'a' && h <= 'f') v |= uint32_t(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= uint32_t(h - 'A' + 10);
      else fail("invalid escape");
    }
    return v;
  }

  std::string string() {
    ++p_;  // opening quote
    std::string out;
    for (;;) {
      if (p_ >= end_) fail("EOF while parsing a string");
      const unsigned char c = static_cast<unsigned char>(*p_++);
      if (c == '"') return out;
      if (c < 0x20) fail("control character in string");
      if (c != '\\') {
        out += char(c);
        continue;
      }
      if (p_ >= end_) fail("EOF while parsing a string");
      const char e = *p_++;
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
            if (end_ - p_ < 6 || p_[0] != '\\' || p_[1] != 'u') fail("unpaired surrogate");
            p_ += 2;
            const uint32_t lo = hex4();
            if (lo < 0xDC00 || lo >= 0xE000) fail("unpaired surrogate");
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          } else if (cp >= 0xDC00 && cp < 0xE000) {
            fail("unpaired surrogate");
          }
          put_utf8(out, cp);
          break;
        }
        default: fail("invalid escape");
      }
    }
  }

  void number(Json& v) {
    const char* start = p_;
    v.kind = Json::kNumber;
    v.integral = true;
    if (*p_ == '-') {
      v.negative = true;
      ++p_;
    }
    if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) fail("invalid number");
    if (*p_ == '0') {
      ++p_;
    } else {
      while (p_ < end_ && *p_ >= '0' && *p_ <= '9') {
        const uint64_t d = uint64_t(*p_ - '0');
        if (v.magnitude > (UINT64_MAX - d) / 10) v.overflow = true;
        else v.magnitude = v.magnitude * 10 + d;
        ++p_;
      }
    }
    if (p_ < end_ && *p_ == '.') {
      v.integral = false;
      ++p_;
      if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) fail("invalid number");
      while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
    }
    if (p_ < end_ && (*p_ == 'e' || *p_ == 'E')) {
      v.integral = false;
      ++p_;
      if (p_ < end_ && (*p_ == '+' || *p_ == '-')) ++p_;
      if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) fail("invalid number");
      while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
    }
    const auto r = std::from_chars(start, p_, v.number);
    if (r.ec == std::errc::result_out_of_range) fail("number out of range");
    if (r.ec != std::errc() || r.ptr != p_) fail("invalid number");
  }

  const char* p_;
  const char* end_;
  const char* begin_;
  std::string what_;
};

// Typed reads with serde's meaning: a required field that is absent is an error, an optional one
// that is absent or null is None.
const Json& field(const Json& obj, const char* key, const std::string& ctx) {
  if (obj.kind != Json::kObject) bail(ctx + ": expected an object");
  const Json* v = obj.find(key);
  if (!v) bail(ctx + ": missing field `" + key + "`");
  return *v;
}

const Json* optional(const Json& obj, const char* key) {
  const Json* v = obj.find(key);
  return (v && v->kind != Json::kNull) ? v : nullptr;
}

float as_f32(const Json& v, const std::string& ctx) {
  if (v.kind != Json::kNumber) bail(ctx + ": expected a number");
  return float(v.number);
}

uint64_t as_index(const Json& v, const std::string& ctx, uint64_t limit) {
  if (v.kind != Json::kNumber || !v.integral || v.overflow || (v.negative && v.magnitude != 0) || v.magnitude > limit)
    bail(ctx + ": expected an integer in [0, " + std::to_string(limit) + "]");
  return v.magnitude;
}

uint32_t as_u32(const Json& v, const std::string& ctx) { return uint32_t(as_index(v, ctx, UINT32_MAX)); }

const std::string& as_str(const Json& v, const std::string& ctx) {
  if (v.kind != Json::kString) bail(ctx + ": expected a string");
  return v.text;
}

const std::vector<Json>& as_array(const Json& v, const std::string& ctx) {
  if (v.kind != Json::kArray) bail(ctx + ": expected an array");
  return v.items;
}

V3 as_vec3(const Json& v, const std::string& ctx) {
  const auto& a = as_array(v, ctx);
  if (a.size() != 3) bail(ctx + ": expected an array of 3 numbers");
  return {as_f32(a[0], ctx), as_f32(a[1], ctx), as_f32(a[2], ctx)};
}

// ------------------------------------------------------------------------------------ files
std::vector<uint8_t> read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) bail("failed to open " + path);
  f.seekg(0, std::ios::end);
  const std::streamoff n = f.tellg();
  if (n < 0) bail("failed to read " + path);
  f.seekg(0, std::ios::beg);
  std::vector<uint8_t> data(static_cast<size_t>(n));
  if (n && !f.read(reinterpret_cast<char*>(data.data()), n)) bail("failed to read " + path);
  return data;
}

std::string parent_dir(const std::string& path) {
  const size_t slash = path.find_last_of('/');
  return slash == std::string::npos ? std::string() : path.substr(0, slash);
}

// Path::join: an absolute path replaces the base.
std::string join(const std::string& dir, const std::string& rel) {
  if (!rel.empty() && rel[0] == '/') return rel;
  if (dir.empty()) return rel;
  return dir + "/" + rel;
}

std::vector<uint8_t> base64_decode(const std::string& s, const std::string& ctx) {
  auto val = [](char c) -> int {
    if (c >= 'A' && c <= 'Z') return c - 'A';
    if (c >= 'a' && c <= 'z') return c - 'a' + 26;
    if (c >= '0' && c <= '9') return c - '0' + 52;
    if (c == '+' || c == '-') return 62;
    if (c == '/' || c == '_') return 63;
    return -1;
  };
  std::vector<uint8_t> out;
  out.reserve(s.size() / 4 * 3);
  uint32_t acc = 0;
  int bits = 0;
  for (char c : s) {
    if (c == '=') break;
    const int v = val(c);
    if (v < 0) bail(ctx + ": invalid base64 data");
    acc = (acc << 6) | uint32_t(v);
    bits += 6;
    if (bits >= 8) {
      bits -= 8;
      out.push_back(uint8_t((acc >> bits) & 0xFF));
    }
  }
  return out;
}

std::string percent_decode(const std::string& s) {
  std::string out;
  for (size_t i = 0; i < s.size(); ++i) {
    if (s[i] == '%' && i + 2 < s.size() && std::isxdigit(static_cast<unsigned char>(s[i + 1])) &&
        std::isxdigit(static_cast<unsigned char>(s[i + 2]))) {
      out += char(std::stoi(s.substr(i + 1, 2), nullptr, 16));
      i += 2;
    } else {
      out += s[i];
    }
  }
  return out;
}

// ---------------------------------------------------------------------------------------- PNG
// 8-bit images as the image crate hands them to the glTF importer, after png's EXPAND transform:
// palettes become RGB (RGBA with a tRNS chunk), grey of depth 1/2/4 is scaled to 8 bits, a tRNS
// colour key becomes an alpha channel. 16-bit images are rejected, as image_to_rgba8 rejects them.
struct Image8 {
  uint32_t width = 0, height = 0;
  int channels = 0;  // 1 grey, 2 grey+alpha, 3 RGB, 4 RGBA
  std::vector<uint8_t> pixels;
};

uint32_t be32(const uint8_t* p) { return uint32_t(p[0]) << 24 | uint32_t(p[1]) << 16 | uint32_t(p[2]) << 8 | p[3]; }

bool is_png(const uint8_t* d, size_t n) {
  static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
  return n >= 8 && std::memcmp(d, sig, 8) == 0;
}

bool is_jpeg(const uint8_t* d, size_t n) { return n >= 3 && d[0] == 0xFF && d[1] == 0xD8 && d[2] == 0xFF; }

uint8_t paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return uint8_t(a);
  if (pb <= pc) return uint8_t(b);
  return uint8_t(c);
}

// Reverses the scanline filters of one (sub)image in place; rows are 1 + row_bytes long.
void unfilter(uint8_t* data, uint32_t rows, size_t row_bytes, size_t bpp, const std::string& ctx) {
  std::vector<uint8_t> zero(row_bytes, 0);
  const uint8_t* prev = zero.data();
  for (uint32_t y = 0; y < rows; ++y) {
    uint8_t* row = data + size_t(y) * (row_bytes + 1);
    const uint8_t type = row[0];
    uint8_t* cur = row + 1;
    switch (type) {
      case 0: break;
      case 1:
        for (size_t i = bpp; i < row_bytes; ++i) cur[i] = uint8_t(cur[i] + cur[i - bpp]);
        break;
      case 2:
        for (size_t i = 0; i < row_bytes; ++i) cur[i] = uint8_t(cur[i] + prev[i]);
        break;
      case 3:
        for (size_t i = 0; i < row_bytes; ++i) {
          const int left = i >= bpp ? cur[i - bpp] : 0;
          cur[i] = uint8_t(cur[i] + ((left + prev[i]) >> 1));
        }
        break;
      case 4:
        for (size_t i = 0; i < row_bytes; ++i) {
          const int left = i >= bpp ? cur[i - bpp] : 0;
          const int upleft = i >= bpp ? prev[i - bpp] : 0;
          cur[i] = uint8_t(cur[i] + paeth(left, prev[i], upleft));
        }
        break;
      default: bail(ctx + ": invalid PNG filter type");
    }
    prev = cur;
  }
}

Image8 decode_png(const uint8_t* d, size_t n, const std::string& ctx) {
  if (!is_png(d, n)) bail(ctx + ": not a PNG image");
  size_t pos = 8;
  uint32_t w = 0, h = 0;
  int depth = 0, color = -1, interlace = 0;
  std::vector<uint8_t> idat, palette, trns;
  bool have_ihdr = false, have_iend = false;
  while (pos + 12 <= n) {
    const uint32_t len = be32(d + pos);
    if (len > n - pos - 12) bail(ctx + ": truncated PNG chunk");
    const uint8_t* type = d + pos + 4;
    const uint8_t* body = d + pos + 8;
    const uint32_t crc = be32(body + len);
    if (uint32_t(crc32(crc32(0L, Z_NULL, 0), type, len + 4)) != crc) bail(ctx + ": PNG chunk CRC mismatch");
    if (std::memcmp(type, "IHDR", 4) == 0) {
      if (len != 13) bail(ctx + ": invalid PNG header");
      w = be32(body);
      h = be32(body + 4);
      depth = body[8];
      color = body[9];
      if (body[10] != 0 || body[11] != 0 || body[12] > 1) bail(ctx + ": unsupported PNG compression, filter or interlace method");
      interlace = body[12];
      have_ihdr = true;
    } else if (std::memcmp(type, "PLTE", 4) == 0) {
      palette.assign(body, body + len);
    } else if (std::memcmp(type, "tRNS", 4) == 0) {
      trns.assign(body, body + len);
    } else if (std::memcmp(type, "IDAT", 4) == 0) {
      idat.insert(idat.end(), body, body + len);
    } else if (std::memcmp(type, "IEND", 4) == 0) {
      have_iend = true;
      break;
    } else if (!(type[0] & 0x20)) {
      bail(ctx + ": unknown critical PNG chunk");
    }
    pos += size_t(len) + 12;
  }
  if (!have_ihdr || !have_iend) bail(ctx + ": truncated PNG");
  if (w == 0 || h == 0) bail(ctx + ": PNG dimensions must be nonzero");
  if (depth == 16) bail(ctx + ": unsupported 16-bit image; use an 8-bit image");
  int samples = 0;
  switch (color) {
    case 0: samples = 1; if (depth != 1 && depth != 2 && depth != 4 && depth != 8) bail(ctx + ": invalid PNG bit depth"); break;
    case 2: samples = 3; if (depth != 8) bail(ctx + ": invalid PNG bit depth"); break;
    case 3: samples = 1; if (depth != 1 && depth != 2 && depth != 4 && depth != 8) bail(ctx + ": invalid PNG bit depth"); break;
    case 4: samples = 2; if (depth != 8) bail(ctx + ": invalid PNG bit depth"); break;
    case 6: samples = 4; if (depth != 8) bail(ctx + ": invalid PNG bit depth"); break;
    default: bail(ctx + ": invalid PNG colour type");
  }
  if (color == 3 && (palette.empty() || palette.size() % 3 != 0)) bail(ctx + ": paletted PNG without a valid palette");
  if (uint64_t(w) * h > (uint64_t(1) << 28)) bail(ctx + ": PNG dimensions are too large");

  // Sub-images: one for a plain image, the seven Adam7 passes for an interlaced one.
  struct Pass {
    uint32_t x0, y0, dx, dy, w, h;
  };
  std::vector<Pass> passes;
  if (interlace == 0) {
    passes.push_back({0, 0, 1, 1, w, h});
  } else {
    static const uint32_t a7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                      {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    for (const auto& a : a7) {
      const uint32_t pw = w > a[0] ? (w - a[0] + a[2] - 1) / a[2] : 0;
      const uint32_t ph = h > a[1] ? (h - a[1] + a[3] - 1) / a[3] : 0;
      passes.push_back({a[0], a[1], a[2], a[3], pw, ph});
    }
  }
  size_t total = 0;
  for (const Pass& p : passes)
    if (p.w && p.h) total += size_t(p.h) * (1 + (size_t(p.w) * samples * depth + 7) / 8);
  std::vector<uint8_t> raw(total);
  {
    z_stream zs{};
    if (inflateInit(&zs) != Z_OK) bail(ctx + ": zlib initialisation failed");
    zs.next_in = idat.data();
    zs.avail_in = uInt(idat.size());
    zs.next_out = raw.data();
    zs.avail_out = uInt(raw.size());
    const int rc = inflate(&zs, Z_FINISH);
    const size_t produced = raw.size() - zs.avail_out;
    inflateEnd(&zs);
    if ((rc != Z_STREAM_END && rc != Z_BUF_ERROR && rc != Z_OK) || produced != raw.size())
      bail(ctx + ": corrupt PNG image data");
  }

  // Expanded output channels.
  int out_ch = 0;
  if (color == 0) out_ch = trns.size() >= 2 ? 2 : 1;
  else if (color == 2) out_ch = trns.size() >= 6 ? 4 : 3;
  else if (color == 3) out_ch = trns.empty() ? 3 : 4;
  else if (color == 4) out_ch = 2;
  else out_ch = 4;
  Image8 img;
  img.width = w;
  img.height = h;
  img.channels = out_ch;
  img.pixels.assign(size_t(w) * h * out_ch, 0);

  const size_t bpp = std::max<size_t>(1, size_t(samples) * depth / 8);
  size_t off = 0;
  for (const Pass& p : passes) {
    if (!p.w || !p.h) continue;
    const size_t row_bytes = (size_t(p.w) * samples * depth + 7) / 8;
    uint8_t* data = raw.data() + off;
    unfilter(data, p.h, row_bytes, bpp, ctx);
    for (uint32_t py = 0; py < p.h; ++py) {
      const uint8_t* row = data + size_t(py) * (row_bytes + 1) + 1;
      for (uint32_t px = 0; px < p.w; ++px) {
        const uint32_t x = p.x0 + px * p.dx, y = p.y0 + py * p.dy;
        uint8_t* o = img.pixels.data() + (size_t(y) * w + x) * out_ch;
        if (color == 0 || color == 3) {
          uint32_t v;
          if (depth == 8) {
            v = row[px];
          } else {
            const size_t bit = size_t(px) * depth;
            v = (row[bit >> 3] >> (8 - depth - (bit & 7))) & ((1u << depth) - 1u);
          }
          if (color == 0) {
            const uint32_t key = trns.size() >= 2 ? (uint32_t(trns[0]) << 8 | trns[1]) : 0xFFFFFFFFu;
            const uint8_t grey = uint8_t(depth == 8 ? v : v * (255u / ((1u << depth) - 1u)));
            o[0] = grey;
            if (out_ch == 2) o[1] = v == key ? 0 : 255;
          } else {
            if (size_t(v) * 3 + 2 >= palette.size()) bail(ctx + ": PNG palette index out of range");
            o[0] = palette[v * 3];
            o[1] = palette[v * 3 + 1];
            o[2] = palette[v * 3 + 2];
            if (out_ch == 4) o[3] = v < trns.size() ? trns[v] : 255;
          }
        } else if (color == 2) {
          const uint8_t* s = row + size_t(px) * 3;
          o[0] = s[0];
          o[1] = s[1];
          o[2] = s[2];
          if (out_ch == 4) {
            const bool keyed = s[0] == trns[1] && s[1] == trns[3] && s[2] == trns[5] && trns[0] == 0 && trns[2] == 0 && trns[4] == 0;
            o[3] = keyed ? 0 : 255;
          }
        } else {
          std::memcpy(o, row + size_t(px) * samples, size_t(samples));
        }
      }
    }
    off += size_t(p.h) * (row_bytes + 1);
  }
  return img;
}

// gltf_loader.rs:200-233 image_to_rgba8.
std::vector<uint8_t> to_rgba8(const Image8& img) {
  const size_t n = size_t(img.width) * img.height;
  std::vector<uint8_t> out(n * 4);
  for (size_t i = 0; i < n; ++i) {
    const uint8_t* s = img.pixels.data() + i * img.channels;
    uint8_t* o = out.data() + i * 4;
    switch (img.channels) {
      case 1: o[0] = o[1] = o[2] = s[0]; o[3] = 255; break;
      case 2: o[0] = o[1] = o[2] = s[0]; o[3] = s[1]; break;
      case 3: o[0] = s[0]; o[1] = s[1]; o[2] = s[2]; o[3] = 255; break;
      default: std::memcpy(o, s, 4); break;
    }
  }
  return out;
}

// ---------------------------------------------------------------------- Radiance RGBE (.hdr)
struct EnvImage {
  uint32_t width = 0, height = 0;
  std::vector<V3> pixels;
};

V3 rgbe_to_f32(const uint8_t* p) {
  if (p[3] == 0) return {};
  const float scale = std::ldexp(1.0f, int(p[3]) - 136);
  return {scale * float(p[0]), scale * float(p[1]), scale * float(p[2])};
}

bool is_hdr(const uint8_t* d, size_t n) {
  return (n >= 10 && std::memcmp(d, "#?RADIANCE", 10) == 0) || (n >= 6 && std::memcmp(d, "#?RGBE", 6) == 0);
}

EnvImage decode_hdr(const uint8_t* d, size_t n, const std::string& ctx) {
  size_t pos = 0;
  auto line = [&]() -> std::string {
    const size_t start = pos;
    while (pos < n && d[pos] != '\n') ++pos;
    if (pos >= n) bail(ctx + ": truncated Radiance header");
    std::string s(reinterpret_cast<const char*>(d + start), pos - start);
    ++pos;
    if (!s.empty() && s.back() == '\r') s.pop_back();
    return s;
  };
  if (!is_hdr(d, n)) bail(ctx + ": not a Radiance image");
  for (;;) {
    const std::string l = line();
    if (l.empty()) break;
    if (l.rfind("FORMAT=", 0) == 0 && l != "FORMAT=32-bit_rle_rgbe") bail(ctx + ": unsupported Radiance format " + l.substr(7));
  }
  const std::string dims = line();
  char ys[3] = {0}, xs[3] = {0};
  unsigned long hh = 0, ww = 0;
  if (std::sscanf(dims.c_str(), "%2s %lu %2s %lu", ys, &hh, xs, &ww) != 4 || std::strcmp(ys, "-Y") != 0 ||
      std::strcmp(xs, "+X") != 0)
    bail(ctx + ": unsupported Radiance orientation '" + dims + "'");
  if (ww == 0 || hh == 0 || ww > (1u << 20) || hh > (1u << 20) || uint64_t(ww) * hh > (uint64_t(1) << 28))
    bail(ctx + ": invalid Radiance dimensions");
  EnvImage img;
  img.width = uint32_t(ww);
  img.height = uint32_t(hh);
  img.pixels.resize(size_t(ww) * hh);
  std::vector<uint8_t> scan(size_t(ww) * 4);
  for (uint32_t y = 0; y < img.height; ++y) {
    const uint32_t w = img.width;
    const bool rle = w >= 8 && w < 0x8000 && pos + 4 <= n && d[pos] == 2 && d[pos + 1] == 2 && !(d[pos + 2] & 0x80) &&
                     ((uint32_t(d[pos + 2]) << 8) | d[pos + 3]) == w;
    if (rle) {
      pos += 4;
      for (int c = 0; c < 4; ++c) {
        uint32_t x = 0;
        while (x < w) {
          if (pos >= n) bail(ctx + ": truncated Radiance scanline");
          uint32_t count = d[pos++];
          if (count > 128) {
            count -= 128;
            if (count > w - x || pos >= n) bail(ctx + ": bad Radiance run length");
            const uint8_t v = d[pos++];
            for (uint32_t k = 0; k < count; ++k) scan[size_t(x + k) * 4 + c] = v;
          } else {
            if (count == 0 || count > w - x || n - pos < count) bail(ctx + ": bad Radiance run length");
            for (uint32_t k = 0; k < count; ++k) scan[size_t(x + k) * 4 + c] = d[pos++];
          }
          x += count;
        }
      }
    } else {
      // Flat pixels, with the original run-length form: (1, 1, 1, k) repeats the previous pixel
      // k << shift times, the shift growing by 8 for consecutive run pixels.
      uint32_t x = 0;
      int shift = 0;
      while (x < w) {
        if (n - pos < 4) bail(ctx + ": truncated Radiance scanline");
        const uint8_t* p = d + pos;
        pos += 4;
        if (p[0] == 1 && p[1] == 1 && p[2] == 1) {
          if (x == 0) bail(ctx + ": Radiance run without a preceding pixel");
          const uint64_t count = uint64_t(p[3]) << shift;
          if (count > w - x) bail(ctx + ": bad Radiance run length");
          for (uint64_t k = 0; k < count; ++k, ++x) std::memcpy(&scan[size_t(x) * 4], &scan[size_t(x - 1) * 4], 4);
          shift += 8;
        } else {
          std::memcpy(&scan[size_t(x) * 4], p, 4);
          ++x;
          shift = 0;
        }
      }
    }
    for (uint32_t x = 0; x < w; ++x) img.pixels[size_t(y) * w + x] = rgbe_to_f32(&scan[size_t(x) * 4]);
  }
  return img;
}

// texture.rs:84-91 srgb_to_linear.
float srgb_to_linear(uint8_t v) {
  const float x = float(v) / 255.0f;
  if (x <= 0.04045f) return x / 12.92f;
  return std::pow((x + 0.055f) / 1.055f, 2.4f);
}

// environment.rs:94-128 EnvironmentMap::load: Radiance images as linear f32, 8-bit images through
// the sRGB transfer function.
EnvImage load_environment_image(const std::string& path) {
  const std::vector<uint8_t> data = read_file(path);
  if (is_hdr(data.data(), data.size())) return decode_hdr(data.data(), data.size(), path);
  if (is_png(data.data(), data.size())) {
    const Image8 img = decode_png(data.data(), data.size(), path);
    EnvImage env;
    env.width = img.width;
    env.height = img.height;
    env.pixels.resize(size_t(img.width) * img.height);
    for (size_t i = 0; i < env.pixels.size(); ++i) {
      const uint8_t* s = img.pixels.data() + i * img.channels;
      const bool grey = img.channels <= 2;
      env.pixels[i] = {srgb_to_linear(s[0]), srgb_to_linear(grey ? s[0] : s[1]), srgb_to_linear(grey ? s[0] : s[2])};
    }
    return env;
  }
  bail("unsupported environment map format (Radiance .hdr and PNG are read): " + path);
}

// ---------------------------------------------------------------------------------------- glTF
struct MeshVertex {
  V3 position;
  bool has_normal = false, has_uv = false;
  V3 normal;
  float uv[2] = {0.0f, 0.0f};
};
struct MeshTriangle {
  uint32_t index[3];
  int64_t material = -1;  // glTF material index, -1 for none
};
struct MeshMaterial {
  float base_color[4] = {1.0f, 1.0f, 1.0f, 1.0f};
  int64_t texture = -1;  // glTF texture index, -1 for none
};
struct Texture {
  uint32_t width = 0, height = 0;
  std::vector<uint8_t> rgba8;
};
struct Mesh {
  std::vector<MeshVertex> vertices;
  std::vector<MeshTriangle> triangles;
  std::vector<MeshMaterial> materials;
  std::vector<Texture> textures;
};

class GltfReader {
 public:
  explicit GltfReader(const std::string& path) : path_(path), dir_(parent_dir(path)) {
    const std::vector<uint8_t> file = read_file(path);
    std::string json;
    if (file.size() >= 12 && std::memcmp(file.data(), "glTF", 4) == 0) {
      // Binary container: 12-byte header, a JSON chunk, an optional BIN chunk.
      auto le32 = [&](size_t at) {
        return uint32_t(file[at]) | uint32_t(file[at + 1]) << 8 | uint32_t(file[at + 2]) << 16 | uint32_t(file[at + 3]) << 24;
      };
      if (le32(4) != 2) bail(path + ": unsupported GLB version");
      const size_t total = std::min<size_t>(le32(8), file.size());
      size_t pos = 12;
      bool first = true;
      while (pos + 8 <= total) {
        const uint32_t len = le32(pos), type = le32(pos + 4);
        if (len > total - pos - 8) bail(path + ": truncated GLB chunk");
        if (first) {
          if (type != 0x4E4F534Au) bail(path + ": GLB does not start with a JSON chunk");
          json.assign(reinterpret_cast<const char*>(file.data() + pos + 8), len);
          first = false;
        } else if (type == 0x004E4942u && !have_bin_) {
          bin_.assign(file.begin() + long(pos + 8), file.begin() + long(pos + 8 + len));
          have_bin_ = true;
        }
        pos += 8 + size_t(len);
      }
      if (first) bail(path + ": GLB without a JSON chunk");
    } else {
      json.assign(file.begin(), file.end());
    }
    doc_ = JsonParser(json.data(), json.size(), path).parse_document();
    if (doc_.kind != Json::kObject) bail(path + ": glTF document is not an object");
    load_buffers();
  }

  Mesh load() {
    Mesh mesh;
    if (const Json* mats = optional(doc_, "materials")) {
      for (const Json& m : as_array(*mats, path_ + " materials")) {
        MeshMaterial mm;
        if (const Json* pbr = optional(m, "pbrMetallicRoughness")) {
          if (const Json* f = optional(*pbr, "baseColorFactor")) {
            const auto& a = as_array(*f, path_ + " baseColorFactor");
            if (a.size() != 4) bail(path_ + ": baseColorFactor must have 4 components");
            for (int i = 0; i < 4; ++i) mm.base_color[i] = as_f32(a[i], path_ + " baseColorFactor");
          }
          if (const Json* t = optional(*pbr, "baseColorTexture"))
            mm.texture = int64_t(as_index(field(*t, "index", path_ + " baseColorTexture"), path_ + " texture index", INT32_MAX));
        }
        mesh.materials.push_back(mm);
      }
    }
    // Every image is decoded, as the importer does, then each texture takes its source image.
    std::vector<Texture> images;
    if (const Json* imgs = optional(doc_, "images")) {
      size_t i = 0;
      for (const Json& im : as_array(*imgs, path_ + " images")) images.push_back(load_image(im, i++));
    }
    if (const Json* texs = optional(doc_, "textures")) {
      for (const Json& t : as_array(*texs, path_ + " textures")) {
        const Json* src = optional(t, "source");
        if (!src) bail(path_ + ": texture without a source image");
        const uint64_t s = as_index(*src, path_ + " texture source", UINT32_MAX);
        if (s >= images.size()) bail(path_ + ": texture references an unknown image");
        mesh.textures.push_back(images[s]);
      }
    }
    for (const MeshMaterial& m : mesh.materials)
      if (m.texture >= 0 && size_t(m.texture) >= mesh.textures.size()) bail(path_ + ": material references an unknown texture");

    const Json* scenes = optional(doc_, "scenes");
    const std::vector<Json> none;
    const auto& scene_list = scenes ? as_array(*scenes, path_ + " scenes") : none;
    auto load_scene_nodes = [&](const Json& scene) {
      if (const Json* roots = optional(scene, "nodes"))
        for (const Json& r : as_array(*roots, path_ + " scene nodes")) load_node(node_index(r), identity4(), mesh, 0);
    };
    if (const Json* s = optional(doc_, "scene")) {
      const uint64_t idx = as_index(*s, path_ + " scene", UINT32_MAX);
      if (idx >= scene_list.size()) bail(path_ + ": default scene index out of range");
      load_scene_nodes(scene_list[idx]);
    } else {
      for (const Json& sc : scene_list) load_scene_nodes(sc);
    }
    if (mesh.triangles.empty()) bail("glTF " + path_ + " contains no triangle primitives");
    return mesh;
  }

 private:
  std::vector<uint8_t> load_uri(const std::string& uri, const std::string& ctx) {
    if (uri.rfind("data:", 0) == 0) {
      const size_t comma = uri.find(',');
      if (comma == std::string::npos || uri.substr(0, comma).find(";base64") == std::string::npos)
        bail(ctx + ": only base64 data URIs are supported");
      return base64_decode(uri.substr(comma + 1), ctx);
    }
    if (uri.find("://") != std::string::npos) bail(ctx + ": unsupported URI scheme");
    return read_file(join(dir_, percent_decode(uri)));
  }

  void load_buffers() {
    const Json* bufs = optional(doc_, "buffers");
    if (!bufs) return;
    size_t i = 0;
    for (const Json& b : as_array(*bufs, path_ + " buffers")) {
      const std::string ctx = path_ + " buffer " + std::to_string(i);
      const uint64_t len = as_index(field(b, "byteLength", ctx), ctx + " byteLength", UINT32_MAX);
      std::vector<uint8_t> data;
      if (const Json* uri = optional(b, "uri")) {
        data = load_uri(as_str(*uri, ctx + " uri"), ctx);
      } else {
        if (i != 0 || !have_bin_) bail(ctx + ": buffer without a URI outside a GLB");
        data = bin_;
      }
      if (data.size() < len) bail(ctx + ": buffer is shorter than its byteLength");
      data.resize(size_t(len));
      buffers_.push_back(std::move(data));
      ++i;
    }
  }

  // The bytes of a buffer view: pointer, length and stride (0 when absent).
  struct View {
    const uint8_t* data;
    size_t length;
    size_t stride;
  };
  View view(uint64_t index, const std::string& ctx) {
    const auto& views = as_array(field(doc_, "bufferViews", ctx), ctx + " bufferViews");
    if (index >= views.size()) bail(ctx + ": bufferView index out of range");
    const Json& v = views[index];
    const uint64_t buf = as_index(field(v, "buffer", ctx), ctx + " buffer", UINT32_MAX);
    if (buf >= buffers_.size()) bail(ctx + ": buffer index out of range");
    const uint64_t off = optional(v, "byteOffset") ? as_index(*optional(v, "byteOffset"), ctx, UINT32_MAX) : 0;
    const uint64_t len = as_index(field(v, "byteLength", ctx), ctx + " byteLength", UINT32_MAX);
    const uint64_t stride = optional(v, "byteStride") ? as_index(*optional(v, "byteStride"), ctx, 252) : 0;
    if (off + len > buffers_[buf].size()) bail(ctx + ": bufferView exceeds its buffer");
    return {buffers_[buf].data() + off, size_t(len), size_t(stride)};
  }

  static int component_size(uint32_t type) {
    switch (type) {
      case 5120: case 5121: return 1;
      case 5122: case 5123: return 2;
      case 5125: case 5126: return 4;
      default: return 0;
    }
  }

  static double component(const uint8_t* p, uint32_t type) {
    switch (type) {
      case 5120: return double(int8_t(p[0]));
      case 5121: return double(p[0]);
      case 5122: { int16_t v; std::memcpy(&v, p, 2); return double(v); }
      case 5123: { uint16_t v; std::memcpy(&v, p, 2); return double(v); }
      case 5125: { uint32_t v; std::memcpy(&v, p, 4); return double(v); }
      default: { float v; std::memcpy(&v, p, 4); return double(v); }
    }
  }

  // Reads accessor `index` as `count` x `ncomp` raw component values (sparse substitution
  // applied); returns the component type.
  uint32_t read_accessor(uint64_t index, int ncomp, std::vector<double>& out, uint32_t& count, const std::string& ctx) {
    const auto& accs = as_array(field(doc_, "accessors", ctx), ctx + " accessors");
    if (index >= accs.size()) bail(ctx + ": accessor index out of range");
    const Json& a = accs[index];
    const uint32_t type = as_u32(field(a, "componentType", ctx), ctx + " componentType");
    const int csize = component_size(type);
    if (!csize) bail(ctx + ": invalid accessor component type");
    const std::string& shape = as_str(field(a, "type", ctx), ctx + " type");
    const int n_shape = shape == "SCALAR" ? 1 : shape == "VEC2" ? 2 : shape == "VEC3" ? 3 : shape == "VEC4" ? 4 : 0;
    if (n_shape != ncomp) bail(ctx + ": accessor has type " + shape);
    count = as_u32(field(a, "count", ctx), ctx + " count");
    out.assign(size_t(count) * ncomp, 0.0);
    const size_t elem = size_t(csize) * ncomp;
    if (const Json* bv = optional(a, "bufferView")) {
      const View v = view(as_index(*bv, ctx, UINT32_MAX), ctx);
      const uint64_t off = optional(a, "byteOffset") ? as_index(*optional(a, "byteOffset"), ctx, UINT32_MAX) : 0;
      const size_t stride = v.stride ? v.stride : elem;
      if (count && off + uint64_t(stride) * (count - 1) + elem > v.length) bail(ctx + ": accessor exceeds its bufferView");
      for (uint32_t i = 0; i < count; ++i)
        for (int c = 0; c < ncomp; ++c) out[size_t(i) * ncomp + c] = component(v.data + off + size_t(i) * stride + size_t(c) * csize, type);
    }
    if (const Json* sp = optional(a, "sparse")) {
      const uint32_t n = as_u32(field(*sp, "count", ctx), ctx + " sparse count");
      const Json& idx = field(*sp, "indices", ctx);
      const Json& val = field(*sp, "values", ctx);
      const uint32_t itype = as_u32(field(idx, "componentType", ctx), ctx + " sparse componentType");
      const int isize = component_size(itype);
      if (itype != 5121 && itype != 5123 && itype != 5125) bail(ctx + ": invalid sparse index type");
      const View iv = view(as_index(field(idx, "bufferView", ctx), ctx, UINT32_MAX), ctx);
      const View vv = view(as_index(field(val, "bufferView", ctx), ctx, UINT32_MAX), ctx);
      const uint64_t ioff = optional(idx, "byteOffset") ? as_index(*optional(idx, "byteOffset"), ctx, UINT32_MAX) : 0;
      const uint64_t voff = optional(val, "byteOffset") ? as_index(*optional(val, "byteOffset"), ctx, UINT32_MAX) : 0;
      if (ioff + uint64_t(n) * isize > iv.length || voff + uint64_t(n) * elem > vv.length) bail(ctx + ": sparse data exceeds its bufferView");
      for (uint32_t k = 0; k < n; ++k) {
        const uint64_t target = uint64_t(component(iv.data + ioff + size_t(k) * isize, itype));
        if (target >= count) bail(ctx + ": sparse index out of range");
        for (int c = 0; c < ncomp; ++c)
          out[size_t(target) * ncomp + c] = component(vv.data + voff + size_t(k) * elem + size_t(c) * csize, type);
      }
    }
    return type;
  }

  std::vector<float> read_floats(uint64_t index, int ncomp, uint32_t& count, const std::string& ctx) {
    std::vector<double> raw;
    const uint32_t type = read_accessor(index, ncomp, raw, count, ctx);
    if (type != 5126) bail(ctx + ": expected float components");
    std::vector<float> out(raw.size());
    for (size_t i = 0; i < raw.size(); ++i) out[i] = float(raw[i]);
    return out;
  }

  // TEXCOORD_0 as f32: floats as they are, normalised u8 / u16 divided by 255 / 65535 in f32.
  std::vector<float> read_tex_coords(uint64_t index, uint32_t& count, const std::string& ctx) {
    std::vector<double> raw;
    const uint32_t type = read_accessor(index, 2, raw, count, ctx);
    std::vector<float> out(raw.size());
    for (size_t i = 0; i < raw.size(); ++i) {
      if (type == 5126) out[i] = float(raw[i]);
      else if (type == 5121) out[i] = float(raw[i]) / 255.0f;
      else if (type == 5123) out[i] = float(raw[i]) / 65535.0f;
      else bail(ctx + ": invalid TEXCOORD_0 component type");
    }
    return out;
  }

  std::vector<uint32_t> read_indices(uint64_t index, const std::string& ctx) {
    std::vector<double> raw;
    uint32_t count = 0;
    const uint32_t type = read_accessor(index, 1, raw, count, ctx);
    if (type != 5121 && type != 5123 && type != 5125) bail(ctx + ": invalid index component type");
    std::vector<uint32_t> out(raw.size());
    for (size_t i = 0; i < raw.size(); ++i) out[i] = uint32_t(raw[i]);
    return out;
  }

  Texture load_image(const Json& im, size_t i) {
    const std::string ctx = path_ + " image " + std::to_string(i);
    std::vector<uint8_t> bytes;
    if (const Json* uri = optional(im, "uri")) {
      bytes = load_uri(as_str(*uri, ctx), ctx);
    } else if (const Json* bv = optional(im, "bufferView")) {
      const View v = view(as_index(*bv, ctx, UINT32_MAX), ctx);
      bytes.assign(v.data, v.data + v.length);
    } else {
      bail(ctx + ": image without a URI or bufferView");
    }
    if (is_jpeg(bytes.data(), bytes.size())) bail(ctx + ": JPEG textures are not supported by this loader; use PNG");
    const Image8 img = decode_png(bytes.data(), bytes.size(), ctx);
    Texture t;
    t.width = img.width;
    t.height = img.height;
    t.rgba8 = to_rgba8(img);
    return t;
  }

  uint64_t node_index(const Json& v) {
    const uint64_t i = as_index(v, path_ + " node index", UINT32_MAX);
    if (i >= as_array(field(doc_, "nodes", path_), path_ + " nodes").size()) bail(path_ + ": node index out of range");
    return i;
  }

  // The node's local matrix: `matrix` as given, else translation * rotation * scale with the
  // quaternion expanded as the importer's math does.
  M4 local_matrix(const Json& node) {
    const std::string ctx = path_ + " node";
    if (const Json* m = optional(node, "matrix")) {
      const auto& a = as_array(*m, ctx + " matrix");
      if (a.size() != 16) bail(ctx + ": matrix must have 16 components");
      M4 r{};
      for (int i = 0; i < 16; ++i) r.c[i / 4][i % 4] = as_f32(a[i], ctx + " matrix");
      return r;
    }
    float t[3] = {0, 0, 0}, q[4] = {0, 0, 0, 1}, s[3] = {1, 1, 1};
    auto read = [&](const char* key, float* dst, size_t n) {
      if (const Json* v = optional(node, key)) {
        const auto& a = as_array(*v, ctx + " " + key);
        if (a.size() != n) bail(ctx + ": " + key + " has the wrong length");
        for (size_t i = 0; i < n; ++i) dst[i] = as_f32(a[i], ctx + " " + key);
      }
    };
    read("translation", t, 3);
    read("rotation", q, 4);
    read("scale", s, 3);
    M4 tm = identity4();
    tm.c[3][0] = t[0];
    tm.c[3][1] = t[1];
    tm.c[3][2] = t[2];
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx2 = x2 * x, xy2 = x2 * y, xz2 = x2 * z;
    const float yy2 = y2 * y, yz2 = y2 * z, zz2 = z2 * z;
    const float sy2 = y2 * w, sz2 = z2 * w, sx2 = x2 * w;
    M4 rm{};
    rm.c[0][0] = 1.0f - yy2 - zz2;
    rm.c[0][1] = xy2 + sz2;
    rm.c[0][2] = xz2 - sy2;
    rm.c[1][0] = xy2 - sz2;
    rm.c[1][1] = 1.0f - xx2 - zz2;
    rm.c[1][2] = yz2 + sx2;
    rm.c[2][0] = xz2 + sy2;
    rm.c[2][1] = yz2 - sx2;
    rm.c[2][2] = 1.0f - xx2 - yy2;
    rm.c[3][3] = 1.0f;
    M4 sm{};
    sm.c[0][0] = s[0];
    sm.c[1][1] = s[1];
    sm.c[2][2] = s[2];
    sm.c[3][3] = 1.0f;
    return mul(mul(tm, rm), sm);
  }

  // gltf_loader.rs:63-197 load_node: the node's primitives, then its children, depth first.
  void load_node(uint64_t index, const M4& parent, Mesh& out, int depth) {
    if (depth > 256) bail(path_ + ": node hierarchy is too deep or cyclic");
    const Json& node = as_array(field(doc_, "nodes", path_), path_ + " nodes")[index];
    const M4 world = mul(parent, local_matrix(node));
    if (const Json* mesh_ref = optional(node, "mesh")) {
      const auto& meshes = as_array(field(doc_, "meshes", path_), path_ + " meshes");
      const uint64_t mi = as_index(*mesh_ref, path_ + " mesh index", UINT32_MAX);
      if (mi >= meshes.size()) bail(path_ + ": mesh index out of range");
      const auto& prims = as_array(field(meshes[mi], "primitives", path_), path_ + " primitives");
      for (size_t pi = 0; pi < prims.size(); ++pi) {
        const Json& prim = prims[pi];
        const std::string ctx = "glTF mesh " + std::to_string(mi) + " primitive " + std::to_string(pi);
        const uint32_t mode = optional(prim, "mode") ? as_u32(*optional(prim, "mode"), ctx + " mode") : 4u;
        if (mode != 4) bail(ctx + " uses unsupported mode " + std::to_string(mode) + "; only triangles are supported");
        const Json& attrs = field(prim, "attributes", ctx);
        const Json* pos_ref = optional(attrs, "POSITION");
        if (!pos_ref) bail(ctx + " has no POSITION attribute");
        uint32_t n_pos = 0, n_nrm = 0, n_uv = 0;
        const std::vector<float> pos = read_floats(as_index(*pos_ref, ctx, UINT32_MAX), 3, n_pos, ctx + " POSITION");
        std::vector<V3> positions(n_pos);
        for (uint32_t i = 0; i < n_pos; ++i) {
          positions[i] = transform_point(world, {pos[i * 3], pos[i * 3 + 1], pos[i * 3 + 2]});
          if (!finite(positions[i])) bail(ctx + " produces non-finite positions");
        }
        const Json* nrm_ref = optional(attrs, "NORMAL");
        const Json* uv_ref = optional(attrs, "TEXCOORD_0");
        std::vector<float> nrm, uv;
        if (nrm_ref) nrm = read_floats(as_index(*nrm_ref, ctx, UINT32_MAX), 3, n_nrm, ctx + " NORMAL");
        if (uv_ref) uv = read_tex_coords(as_index(*uv_ref, ctx, UINT32_MAX), n_uv, ctx + " TEXCOORD_0");
        if ((nrm_ref && n_nrm != n_pos) || (uv_ref && n_uv != n_pos)) bail(ctx + " has mismatched vertex attribute counts");
        const M3 nm = nrm_ref ? normal_matrix(world) : M3{};
        std::vector<uint32_t> indices;
        if (const Json* ind = optional(prim, "indices")) {
          indices = read_indices(as_index(*ind, ctx, UINT32_MAX), ctx + " indices");
        } else {
          indices.resize(n_pos);
          for (uint32_t i = 0; i < n_pos; ++i) indices[i] = i;
        }
        if (indices.size() % 3 != 0) bail(ctx + " has an index count that is not divisible by three");
        for (uint32_t i : indices)
          if (i >= n_pos) bail(ctx + " contains an out-of-bounds index");
        if (out.vertices.size() + n_pos > UINT32_MAX) bail("glTF mesh has too many vertices");
        const uint32_t base = uint32_t(out.vertices.size());
        for (uint32_t i = 0; i < n_pos; ++i) {
          MeshVertex v;
          v.position = positions[i];
          if (nrm_ref) {
            const V3 n = normalize_or_zero(mul(nm, V3{nrm[i * 3], nrm[i * 3 + 1], nrm[i * 3 + 2]}));
            if (!finite(n) || (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f)) bail(ctx + " produces an invalid normal");
            v.has_normal = true;
            v.normal = n;
          }
          if (uv_ref) {
            v.uv[0] = uv[i * 2];
            v.uv[1] = uv[i * 2 + 1];
            if (!std::isfinite(v.uv[0]) || !std::isfinite(v.uv[1])) bail(ctx + " contains non-finite texture coordinates");
            v.has_uv = true;
          }
          out.vertices.push_back(v);
        }
        int64_t material = -1;
        if (const Json* m = optional(prim, "material")) {
          material = int64_t(as_index(*m, ctx + " material", INT32_MAX));
          if (size_t(material) >= out.materials.size()) bail(ctx + " references an unknown material");
        }
        for (size_t k = 0; k < indices.size(); k += 3)
          out.triangles.push_back({{base + indices[k], base + indices[k + 1], base + indices[k + 2]}, material});
      }
    }
    if (const Json* children = optional(node, "children"))
      for (const Json& c : as_array(*children, path_ + " children")) load_node(node_index(c), world, out, depth + 1);
  }

  std::string path_, dir_;
  Json doc_;
  std::vector<uint8_t> bin_;
  bool have_bin_ = false;
  std::vector<std::vector<uint8_t>> buffers_;
};

// ------------------------------------------------------------------------------- scene model
enum class MatKind { kDiffuse, kTexturedDiffuse, kMetal, kDielectric, kEmissive };
struct Material {
  MatKind kind = MatKind::kDiffuse;
  V3 albedo{1.0f, 1.0f, 1.0f};
  float roughness = 0.0f, ior = 0.0f, strength = 0.0f;
  size_t texture = 0;
};
struct Sphere {
  V3 center;
  float radius;
  uint32_t material;
};
struct Triangle {
  V3 v[3];
  uint32_t material;
};
struct Attributes {
  bool has_normals = false, has_uvs = false;
  V3 n[3];
  float uv[3][2] = {{0, 0}, {0, 0}, {0, 0}};
};

void validate_color(const std::string& name, const char* what, V3 c) {
  if (!finite(c) || c.x < 0.0f || c.y < 0.0f || c.z < 0.0f || c.x > 1.0f || c.y > 1.0f || c.z > 1.0f)
    bail("material '" + name + "' " + what + " must be between 0 and 1");
}

void validate_triangle(const V3 v[3]) {
  if (!finite(v[0]) || !finite(v[1]) || !finite(v[2])) bail("triangle vertices must be finite");
  const V3 c = cross(v[1] - v[0], v[2] - v[0]);
  if (dot(c, c) <= kF32Epsilon) bail("triangle vertices must not be collinear");
}

// loader.rs:1541-1568: the eight corners and twelve faces in the reference's order.
void box_triangles(V3 center, V3 size, V3 out[12][3]) {
  const V3 h = size * 0.5f;
  const V3 corners[8] = {center + V3{-h.x, -h.y, -h.z}, center + V3{-h.x, -h.y, h.z}, center + V3{-h.x, h.y, -h.z},
                         center + V3{-h.x, h.y, h.z},   center + V3{h.x, -h.y, -h.z}, center + V3{h.x, -h.y, h.z},
                         center + V3{h.x, h.y, -h.z},   center + V3{h.x, h.y, h.z}};
  static const int faces[12][3] = {{1, 5, 7}, {1, 7, 3}, {4, 0, 2}, {4, 2, 6}, {0, 1, 3}, {0, 3, 2},
                                   {5, 4, 6}, {5, 6, 7}, {3, 7, 6}, {3, 6, 2}, {0, 4, 5}, {0, 5, 1}};
  for (int f = 0; f < 12; ++f)
    for (int k = 0; k < 3; ++k) out[f][k] = corners[faces[f][k]];
}

float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

void set4(float* dst, V3 v, float w = 0.0f) {
  dst[0] = v.x;
  dst[1] = v.y;
  dst[2] = v.z;
  dst[3] = w;
}

}  // namespace

struct tc_loaded_scene {
  tc_scene_data data{};
  float exposure_stops = 0.0f;
  std::vector<tc_gpu_sphere> spheres;
  std::vector<tc_gpu_triangle> triangles;
  std::vector<tc_gpu_triangle_attributes> attributes;
  std::vector<tc_gpu_material> materials;
  std::vector<tc_gpu_light> lights;
  std::vector<uint32_t> texels;
  std::vector<float> environment;
};

namespace {

void build(const std::string& path, tc_loaded_scene& out) {
  const std::vector<uint8_t> text = read_file(path);
  const Json doc = JsonParser(reinterpret_cast<const char*>(text.data()), text.size(), path).parse_document();
  const std::string dir = parent_dir(path);
  if (doc.kind != Json::kObject) bail(path + ": the scene must be a JSON object");

  // Camera and render settings (loader.rs:107-135, validated at :548-570).
  const Json& cam = field(doc, "camera", "camera");
  const V3 position = as_vec3(field(cam, "position", "camera"), "camera position");
  const V3 look_at = as_vec3(field(cam, "look_at", "camera"), "camera look_at");
  const V3 up = optional(cam, "up") ? as_vec3(*optional(cam, "up"), "camera up") : V3{0.0f, 1.0f, 0.0f};
  const Json* fov_j = cam.find("fov_degrees");
  if (!fov_j) fov_j = cam.find("vertical_fov_degrees");
  if (!fov_j) bail("camera: missing field `fov_degrees`");
  const float fov = as_f32(*fov_j, "camera fov_degrees");
  const Json& render = field(doc, "render", "render");
  const uint32_t width = as_u32(field(render, "width", "render"), "render width");
  const uint32_t height = as_u32(field(render, "height", "render"), "render height");
  const Json* spp_j = render.find("samples");
  if (!spp_j) spp_j = render.find("samples_per_pixel");
  if (!spp_j) bail("render: missing field `samples`");
  const uint32_t samples = as_u32(*spp_j, "render samples");
  const uint32_t max_bounces = as_u32(field(render, "max_bounces", "render"), "render max_bounces");
  if (width == 0 || height == 0) bail("render width and height must be greater than zero");
  if (samples == 0) bail("render samples must be greater than zero");
  if (!(fov >= 0.0f && fov < 180.0f)) bail("camera fov_degrees must be between 0 and 180");
  const V3 view = position - look_at;
  if (!finite(position) || !finite(look_at) || !finite(up) ||
      (std::fabs(view.x) <= kF32Epsilon && std::fabs(view.y) <= kF32Epsilon && std::fabs(view.z) <= kF32Epsilon))
    bail("camera vectors are invalid");
  {
    const V3 c = cross(up, view);
    if (dot(c, c) <= kF32Epsilon) bail("camera up vector must not be parallel to its view direction");
  }

  // Display block (loader.rs:56-75): exposure and the ACES tone mapper, no other fields.
  if (const Json* disp = optional(doc, "display")) {
    if (disp->kind != Json::kObject) bail("display: expected an object");
    for (const auto& m : disp->members)
      if (m.first != "exposure_stops" && m.first != "tone_mapper") bail("display: unknown field `" + m.first + "`");
    if (const Json* e = optional(*disp, "exposure_stops")) out.exposure_stops = as_f32(*e, "display exposure_stops");
    if (const Json* t = optional(*disp, "tone_mapper"))
      if (as_str(*t, "display tone_mapper") != "aces") bail("display: unknown tone mapper `" + t->text + "`");
  }
  if (!std::isfinite(out.exposure_stops)) bail("display exposure_stops must be finite");

  // Materials (loader.rs:583-631).
  std::vector<Material> materials;
  std::unordered_map<std::string, size_t> names;
  for (const Json& m : as_array(field(doc, "materials", "scene"), "materials")) {
    const std::string& name = as_str(field(m, "name", "material"), "material name");
    if (names.count(name)) bail("duplicate material name '" + name + "'");
    const std::string& type = as_str(field(m, "type", "material '" + name + "'"), "material type");
    const std::string ctx = "material '" + name + "'";
    Material mat;
    if (type == "diffuse") {
      mat.kind = MatKind::kDiffuse;
      mat.albedo = as_vec3(field(m, "albedo", ctx), ctx + " albedo");
      validate_color(name, "albedo", mat.albedo);
    } else if (type == "metal") {
      mat.kind = MatKind::kMetal;
      mat.albedo = as_vec3(field(m, "albedo", ctx), ctx + " albedo");
      const float r = as_f32(field(m, "roughness", ctx), ctx + " roughness");
      validate_color(name, "albedo", mat.albedo);
      if (!std::isfinite(r)) bail(ctx + " roughness must be finite");
      mat.roughness = std::min(std::max(r, 0.0f), 1.0f);
    } else if (type == "dielectric") {
      mat.kind = MatKind::kDielectric;
      mat.ior = as_f32(field(m, "ior", ctx), ctx + " ior");
      if (!std::isfinite(mat.ior) || mat.ior <= 0.0f) bail(ctx + " ior must be finite and greater than zero");
    } else if (type == "emissive") {
      mat.kind = MatKind::kEmissive;
      mat.albedo = as_vec3(field(m, "color", ctx), ctx + " color");
      mat.strength = as_f32(field(m, "strength", ctx), ctx + " strength");
      validate_color(name, "color", mat.albedo);
      if (!std::isfinite(mat.strength) || mat.strength < 0.0f) bail(ctx + " strength must be finite and non-negative");
    } else {
      bail(ctx + ": unknown material type `" + type + "`");
    }
    names.emplace(name, materials.size());
    materials.push_back(mat);
  }
  auto material_of = [&](const Json& obj, const char* what) -> uint32_t {
    const std::string& name = as_str(field(obj, "material", what), std::string(what) + " material");
    const auto it = names.find(name);
    if (it == names.end()) bail(std::string(what) + " references unknown material '" + name + "'");
    return uint32_t(it->second);
  };

  // Objects (loader.rs:633-865).
  std::vector<Sphere> spheres;
  std::vector<Triangle> triangles;
  std::vector<Attributes> attributes;
  std::vector<Texture> textures;
  std::unordered_set<std::string> ids;
  for (const Json& obj : as_array(field(doc, "objects", "scene"), "objects")) {
    const std::string& type = as_str(field(obj, "type", "object"), "object type");
    const bool has_physics = optional(obj, "physics") != nullptr;
    if (type != "sphere" && type != "box" && type != "triangle" && type != "mesh") bail("unknown object type `" + type + "`");
    if (const Json* id = optional(obj, "id")) {
      const std::string& s = as_str(*id, type + " id");
      if (s.empty()) bail("physics entity id must not be empty");
      if (!ids.insert(s).second) bail("duplicate physics entity id '" + s + "'");
    } else if (has_physics && type != "triangle") {
      bail("physics objects require a nonempty object id");
    }
    if (const Json* g = optional(obj, "group"))
      if (as_str(*g, type + " group").empty()) bail("object group name must not be empty");
    if (type == "sphere") {
      const V3 c = as_vec3(field(obj, "center", "sphere"), "sphere center");
      const float r = as_f32(field(obj, "radius", "sphere"), "sphere radius");
      if (!finite(c) || !std::isfinite(r) || r <= 0.0f) bail("sphere radius must be positive and its center must be finite");
      spheres.push_back({c, r, material_of(obj, "sphere")});
    } else if (type == "box") {
      const V3 c = as_vec3(field(obj, "center", "box"), "box center");
      const V3 s = as_vec3(field(obj, "size", "box"), "box size");
      if (!finite(c) || !finite(s) || s.x <= 0.0f || s.y <= 0.0f || s.z <= 0.0f)
        bail("box center must be finite and size components must be positive");
      const uint32_t mi = material_of(obj, "box");
      V3 tris[12][3];
      box_triangles(c, s, tris);
      for (auto& t : tris) {
        triangles.push_back({{t[0], t[1], t[2]}, mi});
        attributes.push_back({});
      }
    } else if (type == "triangle") {
      if (has_physics) bail("triangle objects do not support physics in the rigid-body MVP");
      const auto& vs = as_array(field(obj, "vertices", "triangle"), "triangle vertices");
      if (vs.size() != 3) bail("triangle vertices: expected an array of 3 points");
      Triangle t;
      for (int k = 0; k < 3; ++k) t.v[k] = as_vec3(vs[k], "triangle vertex");
      validate_triangle(t.v);
      t.material = material_of(obj, "triangle");
      triangles.push_back(t);
      attributes.push_back({});
    } else {
      int64_t override_material = -1;
      if (optional(obj, "material")) override_material = material_of(obj, "mesh");
      const std::string mesh_path = join(dir, as_str(field(obj, "path", "mesh"), "mesh path"));
      Mesh mesh;
      try {
        mesh = GltfReader(mesh_path).load();
      } catch (const LoadError& e) {
        bail("failed to load mesh object " + mesh_path + ": " + e.what());
      }
      std::vector<size_t> imported;
      if (override_material < 0) {
        const size_t texture_base = textures.size();
        for (Texture& t : mesh.textures) {
          if (t.width == 0 || t.height == 0) bail("texture dimensions must be nonzero");
          textures.push_back(std::move(t));
        }
        for (const MeshMaterial& mm : mesh.materials) {
          Material mat;
          mat.albedo = {mm.base_color[0], mm.base_color[1], mm.base_color[2]};
          if (mm.texture >= 0) {
            const size_t ti = texture_base + size_t(mm.texture);
            if (ti >= textures.size()) bail("glTF material references an unknown texture");
            mat.kind = MatKind::kTexturedDiffuse;
            mat.texture = ti;
          } else {
            mat.kind = MatKind::kDiffuse;
          }
          materials.push_back(mat);
          imported.push_back(materials.size() - 1);
        }
      }
      int64_t default_material = -1;
      if (override_material < 0)
        for (const MeshTriangle& t : mesh.triangles)
          if (t.material < 0) {
            materials.push_back(Material{});  // diffuse, albedo (1, 1, 1)
            default_material = int64_t(materials.size() - 1);
            break;
          }
      for (size_t ti = 0; ti < mesh.triangles.size(); ++ti) {
        const MeshTriangle& mt = mesh.triangles[ti];
        const MeshVertex* v[3] = {&mesh.vertices[mt.index[0]], &mesh.vertices[mt.index[1]], &mesh.vertices[mt.index[2]]};
        Triangle t;
        for (int k = 0; k < 3; ++k) t.v[k] = v[k]->position;
        try {
          validate_triangle(t.v);
        } catch (const LoadError& e) {
          bail("mesh " + mesh_path + " contains invalid triangle " + std::to_string(ti) + ": " + e.what());
        }
        Attributes a;
        a.has_normals = v[0]->has_normal && v[1]->has_normal && v[2]->has_normal;
        a.has_uvs = v[0]->has_uv && v[1]->has_uv && v[2]->has_uv;
        for (int k = 0; k < 3; ++k) {
          if (a.has_normals) a.n[k] = v[k]->normal;
          if (a.has_uvs) {
            a.uv[k][0] = v[k]->uv[0];
            a.uv[k][1] = v[k]->uv[1];
          }
        }
        size_t mi;
        if (override_material >= 0) {
          mi = size_t(override_material);
        } else if (mt.material >= 0) {
          if (size_t(mt.material) >= imported.size()) bail("glTF primitive references an unknown material");
          mi = imported[size_t(mt.material)];
        } else {
          mi = size_t(default_material);
        }
        if (materials[mi].kind == MatKind::kTexturedDiffuse && !a.has_uvs)
          bail("mesh " + mesh_path + " triangle " + std::to_string(ti) + " uses a base-color texture without TEXCOORD_0");
        t.material = uint32_t(mi);
        triangles.push_back(t);
        attributes.push_back(a);
      }
    }
  }

  // Background (loader.rs:137-182, :901-924) and the environment map (environment.rs:42-92).
  uint32_t background = 0;
  EnvImage env;
  float env_intensity = 0.0f, env_rotation = 0.0f;
  if (const Json* bg = optional(render, "background")) {
    if (bg->kind == Json::kString) {
      if (bg->text == "sky") background = 0;
      else if (bg->text == "black") background = 1;
      else bail("render background: unknown variant `" + bg->text + "`");
    } else if (bg->kind == Json::kObject) {
      const std::string& t = as_str(field(*bg, "type", "render background"), "render background type");
      if (t != "environment") bail("render background: unknown variant `" + t + "`");
      const std::string env_path = join(dir, as_str(field(*bg, "path", "environment background"), "environment path"));
      const float intensity = optional(*bg, "intensity") ? as_f32(*optional(*bg, "intensity"), "environment intensity") : 1.0f;
      const float rotation = optional(*bg, "rotation_degrees") ? as_f32(*optional(*bg, "rotation_degrees"), "environment rotation_degrees") : 0.0f;
      try {
        env = load_environment_image(env_path);
      } catch (const LoadError& e) {
        bail("failed to load environment background " + env_path + ": " + e.what());
      }
      for (const V3& p : env.pixels)
        if (!finite(p) || p.x < 0.0f || p.y < 0.0f || p.z < 0.0f) bail("environment pixels must be finite and non-negative");
      if (!std::isfinite(intensity) || intensity < 0.0f) bail("environment intensity must be finite and non-negative");
      if (!std::isfinite(rotation)) bail("environment rotation_degrees must be finite");
      env_intensity = intensity;
      float r = std::fmod(rotation, 360.0f);  // f32::rem_euclid(360.0)
      if (r < 0.0f) r = r + 360.0f;
      env_rotation = r;
      background = 2;
    } else {
      bail("render background: data did not match any variant");
    }
  }

  // ------------------------------------------------------------ packing (scene_upload.rs:79-294)
  if (spheres.empty() && triangles.empty()) bail("GPU renderer requires at least one object");
  if (materials.empty()) bail("GPU renderer requires at least one material");
  if (spheres.size() > UINT32_MAX || triangles.size() > UINT32_MAX || materials.size() > UINT32_MAX) bail("too many primitives for GPU");

  tc_gpu_camera& camera = out.data.camera;
  {
    const float aspect = float(width) / float(height);
    const V3 backward = normalize(position - look_at);
    const V3 right = normalize(cross(up, backward));
    const V3 true_up = cross(backward, right);
    const float radians = fov * (kPiF / 180.0f);
    const float vh = 2.0f * float(std::tan(double(0.5f * radians)));
    const float vw = aspect * vh;
    const V3 horizontal = vw * right;
    const V3 vertical = vh * true_up;
    const V3 lower_left = position - horizontal * 0.5f - vertical * 0.5f - backward;
    set4(camera.origin, position);
    set4(camera.lower_left_corner, lower_left);
    set4(camera.horizontal, horizontal);
    set4(camera.vertical, vertical);
  }

  out.spheres.resize(spheres.size());
  for (size_t i = 0; i < spheres.size(); ++i) {
    tc_gpu_sphere s{};
    set4(s.center_radius, spheres[i].center, spheres[i].radius);
    s.material_index = spheres[i].material;
    out.spheres[i] = s;
  }
  out.triangles.resize(triangles.size());
  out.attributes.resize(triangles.size());
  for (size_t i = 0; i < triangles.size(); ++i) {
    tc_gpu_triangle t{};
    set4(t.v0, triangles[i].v[0]);
    set4(t.v1, triangles[i].v[1]);
    set4(t.v2, triangles[i].v[2]);
    t.material_index = triangles[i].material;
    out.triangles[i] = t;
    const Attributes& a = attributes[i];
    tc_gpu_triangle_attributes g{};
    if (a.has_normals) {
      set4(g.n0, a.n[0]);
      set4(g.n1, a.n[1]);
      set4(g.n2, a.n[2]);
      g.flags |= 1u;
    }
    if (a.has_uvs) {
      float* uv[3] = {g.uv0, g.uv1, g.uv2};
      for (int k = 0; k < 3; ++k) {
        uv[k][0] = a.uv[k][0];
        uv[k][1] = a.uv[k][1];
      }
      g.flags |= 2u;
    }
    out.attributes[i] = g;
  }

  // Texture atlas: textures back to back, one little-endian RGBA8 word per texel.
  std::vector<uint32_t> tex_offset(textures.size());
  size_t texel_count = 0;
  for (size_t i = 0; i < textures.size(); ++i) {
    if (texel_count > UINT32_MAX) bail("texture atlas is too large");
    tex_offset[i] = uint32_t(texel_count);
    texel_count += textures[i].rgba8.size() / 4;
  }
  out.texels.reserve(texel_count);
  for (const Texture& t : textures)
    for (size_t k = 0; k + 3 < t.rgba8.size(); k += 4)
      out.texels.push_back(uint32_t(t.rgba8[k]) | uint32_t(t.rgba8[k + 1]) << 8 | uint32_t(t.rgba8[k + 2]) << 16 |
                           uint32_t(t.rgba8[k + 3]) << 24);

  out.materials.resize(materials.size());
  for (size_t i = 0; i < materials.size(); ++i) {
    const Material& m = materials[i];
    tc_gpu_material g{};
    V3 albedo = m.albedo;
    switch (m.kind) {
      case MatKind::kDiffuse: g.kind = 0; break;
      case MatKind::kTexturedDiffuse:
        g.kind = 0;
        g.texture_offset = tex_offset[m.texture];
        g.texture_width = textures[m.texture].width;
        g.texture_height = textures[m.texture].height;
        break;
      case MatKind::kMetal: g.kind = 1; g.params[0] = m.roughness; break;
      case MatKind::kDielectric: g.kind = 2; albedo = {1.0f, 1.0f, 1.0f}; g.params[1] = m.ior; break;
      case MatKind::kEmissive: g.kind = 3; g.params[2] = m.strength; break;
    }
    set4(g.albedo, albedo, 1.0f);
    out.materials[i] = g;
  }

  // Emissive primitives with their power weights, triangles first (scene_upload.rs:412-475).
  float cumulative = 0.0f;
  for (const Triangle& t : triangles) {
    const Material& m = materials[t.material];
    if (m.kind != MatKind::kEmissive) continue;
    const float area = 0.5f * length(cross(t.v[1] - t.v[0], t.v[2] - t.v[0]));
    const float weight = area * luminance(m.albedo) * m.strength;
    if (weight <= 0.0f) continue;
    cumulative += weight;
    tc_gpu_light l{};
    l.kind = 0;
    l.material_index = t.material;
    set4(l.v0, t.v[0]);
    set4(l.v1, t.v[1]);
    set4(l.v2, t.v[2]);
    l.area_weight_cumulative[0] = area;
    l.area_weight_cumulative[1] = weight;
    l.area_weight_cumulative[2] = cumulative;
    out.lights.push_back(l);
  }
  for (const Sphere& s : spheres) {
    const Material& m = materials[s.material];
    if (m.kind != MatKind::kEmissive) continue;
    const float area = 4.0f * kPiF * s.radius * s.radius;
    const float weight = area * luminance(m.albedo) * m.strength;
    if (weight <= 0.0f) continue;
    cumulative += weight;
    tc_gpu_light l{};
    l.kind = 1;
    l.material_index = s.material;
    set4(l.center_radius, s.center, s.radius);
    l.area_weight_cumulative[0] = area;
    l.area_weight_cumulative[1] = weight;
    l.area_weight_cumulative[2] = cumulative;
    out.lights.push_back(l);
  }

  // Environment texels with the importance CDF in lane w (environment.rs:244-278).
  if (background == 2) {
    const size_t n = env.pixels.size();
    std::vector<double> weights(n);
    double total = 0.0;
    for (size_t i = 0; i < n; ++i) {
      const size_t y = i / env.width;
      const double theta = 3.14159265358979323846 * (double(y) + 0.5) / double(env.height);
      const V3 p = env.pixels[i];
      const double lum = 0.2126 * double(p.x) + 0.7152 * double(p.y) + 0.0722 * double(p.z);
      weights[i] = lum * std::sin(theta) * double(env_intensity);
      total += weights[i];
    }
    out.environment.assign(n * 4, 0.0f);
    const bool usable = total > 0.0 && std::isfinite(total);
    double acc = 0.0;
    for (size_t i = 0; i < n; ++i) {
      out.environment[i * 4] = env.pixels[i].x;
      out.environment[i * 4 + 1] = env.pixels[i].y;
      out.environment[i * 4 + 2] = env.pixels[i].z;
      if (usable) {
        acc += weights[i] / total;
        out.environment[i * 4 + 3] = i + 1 == n ? 1.0f : float(acc);
      }
    }
  }

  tc_gpu_render_params& p = out.data.params;
  p.width = width;
  p.height = height;
  p.samples = samples;
  p.max_bounces = max_bounces;
  p.sphere_count = uint32_t(spheres.size());
  p.triangle_count = uint32_t(triangles.size());
  p.material_count = uint32_t(materials.size());
  p.background_kind = background;
  p.light_count = uint32_t(out.lights.size());
  p.total_light_weight = cumulative;
  if (background == 2) {
    p.environment_width = env.width;
    p.environment_height = env.height;
    p.environment_intensity = env_intensity;
    p.environment_rotation_degrees = env_rotation;
  }

  tc_scene_data& sd = out.data;
  sd.spheres = out.spheres.data();
  sd.sphere_count = out.spheres.size();
  sd.triangles = out.triangles.data();
  sd.triangle_count = out.triangles.size();
  sd.triangle_attributes = out.attributes.data();
  sd.triangle_attribute_count = out.attributes.size();
  sd.materials = out.materials.data();
  sd.material_count = out.materials.size();
  sd.lights = out.lights.data();
  sd.light_count = out.lights.size();
  sd.texture_pixels = out.texels.empty() ? nullptr : out.texels.data();
  sd.texture_pixel_count = out.texels.size();
  sd.environment_pixels = out.environment.empty() ? nullptr : out.environment.data();
  sd.environment_pixel_count = out.environment.size() / 4;
}

void write_error(char* error, size_t capacity, const char* message) {
  if (!error || capacity == 0) return;
  std::snprintf(error, capacity, "%s", message);
}

}  // namespace

extern "C" int tc_scene_load(const char* path, tc_loaded_scene** out, char* error, size_t error_capacity) {
  if (error && error_capacity) error[0] = '\0';
  if (!path || !out) {
    write_error(error, error_capacity, "path and out must not be null");
    return TC_ERR_INVALID;
  }
  *out = nullptr;
  tc_loaded_scene* scene = new (std::nothrow) tc_loaded_scene();
  if (!scene) {
    write_error(error, error_capacity, "out of host memory");
    return TC_ERR_INVALID;
  }
  try {
    build(path, *scene);
  } catch (const std::exception& e) {
    write_error(error, error_capacity, e.what());
    delete scene;
    return TC_ERR_INVALID;
  }
  *out = scene;
  return TC_OK;
}

extern "C" const tc_scene_data* tc_loaded_scene_data(const tc_loaded_scene* scene) {
  return scene ? &scene->data : nullptr;
}

extern "C" int tc_loaded_scene_display(const tc_loaded_scene* scene, float* exposure_stops) {
  if (!scene || !exposure_stops) return TC_ERR_INVALID;
  *exposure_stops = scene->exposure_stops;
  return TC_OK;
}

extern "C" int tc_loaded_scene_free(tc_loaded_scene* scene) {
  delete scene;
  return TC_OK;
}
