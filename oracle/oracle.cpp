// TEST INFRASTRUCTURE ONLY — the CPU oracle for toaster's GPU path-tracing path.
//
// This file is a C++17 restatement of the reference CPU renderer and BVH that the
// CUDA path is checked against. Only the tests, the smoke check and the benchmark's
// CPU-baseline / reference arm load it; the product library never links it.
//
// What it restates (paths are relative to the toaster project root):
//   crates/toaster-bvh/src/aabb.rs, bvh.rs, flatten.rs           (whole: median-split build)
//   crates/toaster-cpu/src/intersect.rs:28-338                    (sphere, triangle, ordered traversal)
//   crates/toaster-cpu/src/integrator.rs:24-389                   (recursive estimator, BSDFs, NEE, MIS)
//   crates/toaster-cpu/src/light.rs:57-170                        (power-weighted area lights)
//   crates/toaster-scene/src/environment.rs:132-287               (lat-long map, flat CDF, pdf)
//   crates/toaster-core/src/camera.rs:54-99, light.rs:6-13, color.rs:33-74
//
// Arithmetic: glam 0.30.10 scalar Vec3 semantics are assumed (dot = x*x'+y*y'+z*z' left to
// right, cross = (a.y*b.z - b.y*a.z, ...), normalize = v * (1/sqrt(dot))). The file must be
// compiled with -ffp-contract=off so no multiply-add is fused, matching Rust's IEEE f32.
// Transcendentals use glibc's f32 functions, which is what Rust's std calls on Linux.
//
// Pinning: the known-answer tests of intersect.rs, integrator.rs, light.rs, environment.rs,
// bvh.rs, flatten.rs and aabb.rs are restated in tests/test_oracle_known_answers.py. The
// reference's random stream (rand 0.9.4 ChaCha12 StdRng) is not reproduced: this oracle uses
// PCG32 (O'Neill 2014) per pixel, so image parity against it is statistical by design.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kRayEpsilon = 0.001f;  // integrator.rs:11
constexpr float kTrianglePadding = 1e-5f;  // intersect.rs:8
constexpr float kF32Epsilon = std::numeric_limits<float>::epsilon();

struct V3 {
  float x, y, z;
  float operator[](int axis) const { return axis == 0 ? x : (axis == 1 ? y : z); }
};
static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 splat(float s) { return V3{s, s, s}; }
static inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
static inline V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
static inline V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
static inline V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
static inline float length_squared(V3 a) { return dot(a, a); }
static inline float length(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 normalize(V3 a) { return a * (1.0f / length(a)); }
static inline V3 normalize_or_zero(V3 a) {
  float rcp = 1.0f / length(a);
  if (std::isfinite(rcp) && rcp > 0.0f) return a * rcp;
  return splat(0.0f);
}
static inline V3 vmin(V3 a, V3 b) { return V3{std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
static inline V3 vmax(V3 a, V3 b) { return V3{std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
static inline V3 lerp(V3 a, V3 b, float s) { return a + (b - a) * s; }
static inline bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

// ---------------------------------------------------------------- aabb.rs
struct Aabb {
  V3 min, max;
  static Aabb empty() {
    float inf = std::numeric_limits<float>::infinity();
    return Aabb{splat(inf), splat(-inf)};
  }
  Aabb unite(const Aabb& o) const { return Aabb{vmin(min, o.min), vmax(max, o.max)}; }
  Aabb expand(float amount) const { V3 d = splat(amount); return Aabb{min - d, max + d}; }
  V3 centroid() const { return 0.5f * (min + max); }
  V3 extent() const { return max - min; }
  int longest_axis() const {  // aabb.rs:62-71: ties prefer the lower axis
    V3 e = extent();
    if (e.x >= e.y && e.x >= e.z) return 0;
    if (e.y >= e.z) return 1;
    return 2;
  }
  // aabb.rs:74-110: slab test in [min_distance, max_distance]; an infinite inverse
  // direction component means the ray is parallel to that slab.
  bool intersects_ray(V3 origin, V3 inv, float min_distance, float max_distance) const {
    float t_min = min_distance, t_max = max_distance;
    for (int axis = 0; axis < 3; ++axis) {
      float o = origin[axis], lo = min[axis], hi = max[axis], id = inv[axis];
      if (std::isinf(id)) {
        if (o < lo || o > hi) return false;
        continue;
      }
      float near_t = (lo - o) * id;
      float far_t = (hi - o) * id;
      if (near_t > far_t) std::swap(near_t, far_t);
      t_min = std::fmax(t_min, near_t);
      t_max = std::fmin(t_max, far_t);
      if (t_max < t_min) return false;
    }
    return true;
  }
};

// intersect.rs:322-338
static float entry_distance(const Aabb& b, V3 origin, V3 inv) {
  float entry = -std::numeric_limits<float>::infinity();
  for (int axis = 0; axis < 3; ++axis) {
    if (std::isinf(inv[axis])) continue;
    float near_t = (b.min[axis] - origin[axis]) * inv[axis];
    float far_t = (b.max[axis] - origin[axis]) * inv[axis];
    if (near_t > far_t) std::swap(near_t, far_t);
    entry = std::fmax(entry, near_t);
  }
  return entry;
}

// ---------------------------------------------------------------- bvh.rs / flatten.rs
enum PrimKind : uint32_t { kSphere = 0, kTriangle = 1 };
struct PrimRef { uint32_t kind, index; };
struct PrimInfo { Aabb bounds; V3 centroid; PrimRef prim; };
struct FlatNode { Aabb bounds; uint32_t first_or_right; uint32_t count; };

// f32::total_cmp key (IEEE totalOrder as a signed integer).
static inline int32_t total_key(float f) {
  int32_t bits;
  std::memcpy(&bits, &f, 4);
  bits ^= static_cast<int32_t>(static_cast<uint32_t>(bits >> 31) >> 1);
  return bits;
}

struct BuildNode {
  Aabb bounds;
  bool leaf;
  uint32_t first, count;
  std::unique_ptr<BuildNode> left, right;
};

// bvh.rs:92-139 (recursive median split; stable sort by total_cmp; split at n/2).
static std::unique_ptr<BuildNode> build_recursive(PrimInfo* info, size_t n, std::vector<PrimRef>& ordered,
                                                  size_t max_leaf) {
  if (n == 0) return nullptr;
  Aabb bounds = Aabb::empty();
  for (size_t i = 0; i < n; ++i) bounds = bounds.unite(info[i].bounds);
  auto make_leaf = [&]() {
    auto node = std::make_unique<BuildNode>();
    node->bounds = bounds;
    node->leaf = true;
    node->first = static_cast<uint32_t>(ordered.size());
    node->count = static_cast<uint32_t>(n);
    for (size_t i = 0; i < n; ++i) ordered.push_back(info[i].prim);
    return node;
  };
  if (n <= max_leaf) return make_leaf();
  Aabb cb = Aabb::empty();
  for (size_t i = 0; i < n; ++i) cb = cb.unite(Aabb{info[i].centroid, info[i].centroid});
  int axis = cb.longest_axis();
  if (cb.extent()[axis] <= kF32Epsilon) return make_leaf();
  std::stable_sort(info, info + n, [axis](const PrimInfo& a, const PrimInfo& b) {
    return total_key(a.centroid[axis]) < total_key(b.centroid[axis]);
  });
  size_t split = n / 2;
  auto node = std::make_unique<BuildNode>();
  node->bounds = bounds;
  node->leaf = false;
  node->left = build_recursive(info, split, ordered, max_leaf);
  node->right = build_recursive(info + split, n - split, ordered, max_leaf);
  return node;
}

// flatten.rs:72-97 (depth first; left child = parent + 1; right index stored).
static uint32_t flatten_node(const BuildNode* node, std::vector<FlatNode>& nodes) {
  uint32_t index = static_cast<uint32_t>(nodes.size());
  nodes.push_back(FlatNode{node->bounds, 0, 0});
  if (node->leaf) {
    nodes[index].first_or_right = node->first;
    nodes[index].count = node->count;
  } else {
    flatten_node(node->left.get(), nodes);
    uint32_t right = flatten_node(node->right.get(), nodes);
    nodes[index].first_or_right = right;
  }
  return index;
}

struct FlatBvh {
  std::vector<FlatNode> nodes;
  std::vector<PrimRef> prims;
};

static FlatBvh build_flat_bvh(std::vector<PrimInfo> info, size_t max_leaf) {
  FlatBvh bvh;
  bvh.prims.reserve(info.size());
  auto root = build_recursive(info.data(), info.size(), bvh.prims, std::max<size_t>(max_leaf, 1));
  if (root) flatten_node(root.get(), bvh.nodes);
  return bvh;
}

// ---------------------------------------------------------------- scene model
enum MaterialKind : uint32_t { kDiffuse = 0, kMetal = 1, kDielectric = 2, kEmissive = 3 };
struct Material {
  uint32_t kind;
  V3 albedo;  // diffuse/metal albedo; emissive colour
  float roughness, ior, strength;
  uint32_t tex_offset, tex_width, tex_height;
};
struct Sphere { V3 center; float radius; uint32_t material; };
struct Triangle { V3 v[3]; uint32_t material; };
struct TriAttr { bool has_normals, has_uvs; V3 n[3]; float uv[3][2]; };
enum Background : uint32_t { kSky = 0, kBlack = 1, kEnvironment = 2 };

struct Environment {
  uint32_t width = 0, height = 0;
  std::vector<V3> pixels;
  float intensity = 0.0f, rotation_degrees = 0.0f;
  std::vector<float> cdf;

  static float rem_euclid(float a, float b) {
    float r = std::fmod(a, b);
    return r < 0.0f ? r + std::fabs(b) : r;
  }
  static float unit_interval(float v) {  // environment.rs:281-287
    if (std::isfinite(v)) return std::fmin(std::fmax(v, 0.0f), 1.0f - kF32Epsilon);
    return 0.0f;
  }
  // environment.rs:42-88 and :245-278 (f64 accumulation, f32 storage, last entry = 1).
  void init(uint32_t w, uint32_t h, const float* rgb, float inten, float rot) {
    width = w; height = h; intensity = inten;
    rotation_degrees = rem_euclid(rot, 360.0f);
    pixels.resize(size_t(w) * h);
    for (size_t i = 0; i < pixels.size(); ++i) pixels[i] = v3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
    std::vector<double> weights(pixels.size());
    double total = 0.0;
    for (size_t i = 0; i < pixels.size(); ++i) {
      size_t y = i / w;
      double theta = double(kPi) * (double(y) + 0.5) / double(h);
      const V3& p = pixels[i];
      double lum = 0.2126 * double(p.x) + 0.7152 * double(p.y) + 0.0722 * double(p.z);
      double weight = lum * std::sin(theta) * double(inten);
      weights[i] = weight;
      total += weight;
    }
    cdf.assign(pixels.size(), 0.0f);
    if (!(total > 0.0) || !std::isfinite(total)) return;
    double acc = 0.0;
    for (size_t i = 0; i < pixels.size(); ++i) {
      acc += weights[i] / total;
      cdf[i] = float(acc);
    }
    if (!cdf.empty()) cdf.back() = 1.0f;
  }
  V3 texel(int x, int y) const {
    int xi = int(((x % int(width)) + int(width)) % int(width));
    int yi = std::min(std::max(y, 0), int(height) - 1);
    return pixels[size_t(yi) * width + size_t(xi)];
  }
  // environment.rs:132-152
  V3 sample(V3 direction) const {
    V3 d = normalize_or_zero(direction);
    if (is_zero(d)) return splat(0.0f);
    float u = rem_euclid(std::atan2(d.z, d.x) / (2.0f * kPi) + 0.5f + rotation_degrees / 360.0f, 1.0f);
    float v = std::acos(std::fmin(std::fmax(d.y, -1.0f), 1.0f)) / kPi;
    float x = u * float(width) - 0.5f;
    float y = v * float(height) - 0.5f;
    int x0 = int(std::floor(x)), y0 = int(std::floor(y));
    float ax = x - std::floor(x), ay = y - std::floor(y);
    V3 top = lerp(texel(x0, y0), texel(x0 + 1, y0), ax);
    V3 bottom = lerp(texel(x0, y0 + 1), texel(x0 + 1, y0 + 1), ax);
    return lerp(top, bottom, ay) * intensity;
  }
  float texel_pdf_solid_angle(size_t index, float sin_theta) const {  // :225-234
    float prev = index == 0 ? 0.0f : cdf[index - 1];
    float p = std::fmax(cdf[index] - prev, 0.0f);
    if (p <= 0.0f || sin_theta <= 0.0f) return 0.0f;
    return p * float(width) * float(height) / (2.0f * kPi * kPi * sin_theta);
  }
  bool direction_to_uv(V3 direction, float& u, float& v, float& sin_theta) const {  // :213-222
    V3 d = normalize_or_zero(direction);
    if (is_zero(d)) return false;
    u = rem_euclid(std::atan2(d.z, d.x) / (2.0f * kPi) + 0.5f + rotation_degrees / 360.0f, 1.0f);
    float theta = std::acos(std::fmin(std::fmax(d.y, -1.0f), 1.0f));
    v = theta / kPi;
    sin_theta = std::sin(theta);
    return true;
  }
  float pdf_solid_angle(V3 direction) const {  // :193-200
    float u, v, s;
    if (!direction_to_uv(direction, u, v, s)) return 0.0f;
    size_t x = size_t(std::floor(u * float(width))) % width;
    size_t y = std::min(size_t(std::floor(v * float(height))), size_t(height) - 1);
    return texel_pdf_solid_angle(y * width + x, s);
  }
  // environment.rs:159-189
  bool sample_importance(float selection, float ju, float jv, V3& dir, V3& radiance, float& pdf) const {
    if (cdf.empty() || cdf.back() <= 0.0f) return false;
    float sel = unit_interval(selection);
    size_t index = size_t(std::upper_bound(cdf.begin(), cdf.end(), sel) - cdf.begin());
    index = std::min(index, cdf.size() - 1);
    size_t x = index % width, y = index / width;
    float u = (float(x) + unit_interval(ju)) / float(width);
    float v = (float(y) + unit_interval(jv)) / float(height);
    float theta = kPi * v;
    float phi = 2.0f * kPi * (u - 0.5f - rotation_degrees / 360.0f);
    float st = std::sin(theta);
    dir = v3(st * std::cos(phi), std::cos(theta), st * std::sin(phi));
    pdf = texel_pdf_solid_angle(index, st);
    radiance = sample(dir);
    return true;
  }
};

// ---------------------------------------------------------------- camera.rs:54-99
struct Camera {
  V3 origin, lower_left, horizontal, vertical;
  bool init(V3 position, V3 look_at, V3 up, float fov_degrees, float aspect) {
    if (!(fov_degrees >= 0.0f && fov_degrees < 180.0f) || !std::isfinite(aspect) || aspect <= 0.0f) return false;
    V3 view = position - look_at;
    if (length_squared(view) <= kF32Epsilon) return false;
    V3 backward = normalize(view);
    V3 right = cross(up, backward);
    if (length_squared(right) <= kF32Epsilon) return false;
    right = normalize(right);
    V3 true_up = cross(backward, right);
    float radians = fov_degrees * (kPi / 180.0f);
    float vh = 2.0f * std::tan(0.5f * radians);
    float vw = aspect * vh;
    horizontal = vw * right;
    vertical = vh * true_up;
    lower_left = position - horizontal * 0.5f - vertical * 0.5f - backward;
    origin = position;
    return true;
  }
  void ray(float u, float v, V3& o, V3& d) const {
    o = origin;
    d = normalize(lower_left + u * horizontal + v * vertical - origin);
  }
};

// ---------------------------------------------------------------- RNG (documented substitute)
// PCG32 (O'Neill 2014, XSH-RR output, 64-bit LCG) seeded through SplitMix64.
struct Rng {
  uint64_t state, inc;
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed) {
    uint64_t s = seed;
    state = splitmix(s);
    inc = splitmix(s) | 1ull;
  }
  uint32_t next_u32() {
    uint64_t old = state;
    state = old * 6364136223846793005ull + inc;
    uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
  }
  float uniform() { return float(next_u32() >> 8) * (1.0f / 16777216.0f); }  // [0,1)
  float range(float lo, float hi) { return lo + (hi - lo) * uniform(); }
};

// ---------------------------------------------------------------- scene + traversal
struct Hit {
  float distance;
  V3 point, normal;
  bool front_face;
  uint32_t material;
  float uv[2];
  PrimRef prim;
};

struct Counters {
  uint64_t rays = 0, node_tests = 0, sphere_tests = 0, triangle_tests = 0, interior_visits = 0, leaf_visits = 0;
  void add(const Counters& o) {
    rays += o.rays; node_tests += o.node_tests; sphere_tests += o.sphere_tests;
    triangle_tests += o.triangle_tests; interior_visits += o.interior_visits; leaf_visits += o.leaf_visits;
  }
};

struct Scene {
  std::vector<Sphere> spheres;
  std::vector<Triangle> triangles;
  std::vector<TriAttr> attrs;
  std::vector<Material> materials;
  std::vector<uint32_t> texture_pixels;
  Camera camera;
  uint32_t width = 1, height = 1, samples = 1, max_bounces = 1, background = kSky;
  Environment env;
  bool has_env = false;
  FlatBvh bvh;
  // light.rs:14-53
  struct AreaLight { bool is_triangle; Triangle tri; V3 center; float radius; V3 normal, emission; float area, weight, cumulative; };
  std::vector<AreaLight> lights;
  float total_light_weight = 0.0f;

  void build_bvh(size_t max_leaf = 4) {  // intersect.rs:158-163, :291-320
    std::vector<PrimInfo> info;
    info.reserve(spheres.size() + triangles.size());
    for (size_t i = 0; i < spheres.size(); ++i) {
      V3 r = splat(spheres[i].radius);
      Aabb b{spheres[i].center - r, spheres[i].center + r};
      info.push_back(PrimInfo{b, b.centroid(), PrimRef{kSphere, uint32_t(i)}});
    }
    for (size_t i = 0; i < triangles.size(); ++i) {
      const Triangle& t = triangles[i];
      Aabb b = Aabb{vmin(vmin(t.v[0], t.v[1]), t.v[2]), vmax(vmax(t.v[0], t.v[1]), t.v[2])}.expand(kTrianglePadding);
      info.push_back(PrimInfo{b, b.centroid(), PrimRef{kTriangle, uint32_t(i)}});
    }
    bvh = build_flat_bvh(std::move(info), max_leaf);
  }

  void collect_lights() {  // light.rs:57-113
    lights.clear();
    total_light_weight = 0.0f;
    for (const Triangle& t : triangles) {
      const Material& m = materials[t.material];
      if (m.kind != kEmissive) continue;
      V3 e1 = t.v[1] - t.v[0], e2 = t.v[2] - t.v[0];
      V3 c = cross(e1, e2);
      float area = 0.5f * length(c);
      float weight = area * (0.2126f * m.albedo.x + 0.7152f * m.albedo.y + 0.0722f * m.albedo.z) * m.strength;
      if (weight <= 0.0f) continue;
      total_light_weight += weight;
      lights.push_back(AreaLight{true, t, splat(0), 0.0f, normalize(c), m.albedo * m.strength, area, weight, total_light_weight});
    }
    for (const Sphere& s : spheres) {
      const Material& m = materials[s.material];
      if (m.kind != kEmissive) continue;
      float area = 4.0f * kPi * s.radius * s.radius;
      float weight = area * (0.2126f * m.albedo.x + 0.7152f * m.albedo.y + 0.0722f * m.albedo.z) * m.strength;
      if (weight <= 0.0f) continue;
      total_light_weight += weight;
      lights.push_back(AreaLight{false, Triangle{}, s.center, s.radius, splat(0), m.albedo * m.strength, area, weight, total_light_weight});
    }
  }

  // intersect.rs:28-68
  bool intersect_sphere(V3 o, V3 d, const Sphere& s, float tmin, float tmax, Hit& hit) const {
    V3 offset = o - s.center;
    float a = length_squared(d);
    float half_b = dot(offset, d);
    float c = length_squared(offset) - s.radius * s.radius;
    float disc = half_b * half_b - a * c;
    if (disc < 0.0f) return false;
    float sq = std::sqrt(disc);
    float t = (-half_b - sq) / a;
    if (t < tmin || t > tmax) {
      t = (-half_b + sq) / a;
      if (t < tmin || t > tmax) return false;
    }
    V3 p = o + t * d;
    V3 outward = (p - s.center) / s.radius;
    bool front = dot(d, outward) < 0.0f;
    hit.distance = t; hit.point = p; hit.normal = front ? outward : -outward; hit.front_face = front;
    hit.material = s.material; hit.uv[0] = hit.uv[1] = 0.0f;
    return true;
  }

  // intersect.rs:87-148 (Moller-Trumbore, double sided, optional attributes)
  bool intersect_triangle(V3 o, V3 d, uint32_t index, float tmin, float tmax, Hit& hit) const {
    const Triangle& tri = triangles[index];
    const float eps = 1e-8f;
    V3 e1 = tri.v[1] - tri.v[0];
    V3 e2 = tri.v[2] - tri.v[0];
    V3 p = cross(d, e2);
    float det = dot(e1, p);
    if (std::fabs(det) < eps) return false;
    float inv = 1.0f / det;
    V3 s = o - tri.v[0];
    float u = dot(s, p) * inv;
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    V3 q = cross(s, e1);
    float v = dot(d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    float t = dot(e2, q) * inv;
    if (t < tmin || t > tmax) return false;
    V3 gn = normalize(cross(e1, e2));
    bool front = dot(d, gn) < 0.0f;
    float w0 = 1.0f - u - v;
    V3 outward = gn;
    const TriAttr* at = index < attrs.size() ? &attrs[index] : nullptr;
    if (at && at->has_normals) outward = normalize(w0 * at->n[0] + u * at->n[1] + v * at->n[2]);
    if (dot(outward, gn) < 0.0f) outward = -outward;
    hit.uv[0] = hit.uv[1] = 0.0f;
    if (at && at->has_uvs) {
      hit.uv[0] = w0 * at->uv[0][0] + u * at->uv[1][0] + v * at->uv[2][0];
      hit.uv[1] = w0 * at->uv[0][1] + u * at->uv[1][1] + v * at->uv[2][1];
    }
    hit.distance = t; hit.point = o + t * d; hit.normal = front ? outward : -outward; hit.front_face = front;
    hit.material = tri.material;
    return true;
  }

  bool test_prim(V3 o, V3 d, PrimRef pr, float tmin, float tmax, Hit& h, Counters* c) const {
    bool ok;
    if (pr.kind == kSphere) {
      if (c) c->sphere_tests++;
      ok = intersect_sphere(o, d, spheres[pr.index], tmin, tmax, h);
    } else {
      if (c) c->triangle_tests++;
      ok = intersect_triangle(o, d, pr.index, tmin, tmax, h);
    }
    if (ok) h.prim = pr;
    return ok;
  }

  // intersect.rs:172-263: ordered (front-to-back by entry distance) closest hit.
  bool intersect(V3 o, V3 d, float tmin, Hit& hit, Counters* c = nullptr) const {
    if (c) c->rays++;
    if (bvh.nodes.empty()) return false;
    V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float closest = std::numeric_limits<float>::infinity();
    bool found = false;
    std::vector<uint32_t> stack;
    stack.reserve(64);
    stack.push_back(0);
    Hit cand;
    while (!stack.empty()) {
      uint32_t ni = stack.back();
      stack.pop_back();
      const FlatNode& node = bvh.nodes[ni];
      if (c) c->node_tests++;
      if (!node.bounds.intersects_ray(o, inv, tmin, closest)) continue;
      if (node.count > 0) {
        if (c) c->leaf_visits++;
        for (uint32_t i = node.first_or_right; i < node.first_or_right + node.count; ++i) {
          if (test_prim(o, d, bvh.prims[i], tmin, closest, cand, c)) {
            closest = cand.distance;
            hit = cand;
            found = true;
          }
        }
      } else {
        if (c) { c->interior_visits++; c->node_tests += 2; }
        uint32_t li = ni + 1, ri = node.first_or_right;
        const FlatNode& l = bvh.nodes[li];
        const FlatNode& r = bvh.nodes[ri];
        bool lh = l.bounds.intersects_ray(o, inv, tmin, closest);
        bool rh = r.bounds.intersects_ray(o, inv, tmin, closest);
        if (lh && rh) {
          float ld = entry_distance(l.bounds, o, inv);
          float rd = entry_distance(r.bounds, o, inv);
          if (ld < rd) { stack.push_back(ri); stack.push_back(li); }
          else { stack.push_back(li); stack.push_back(ri); }
        } else if (lh) {
          stack.push_back(li);
        } else if (rh) {
          stack.push_back(ri);
        }
      }
    }
    return found;
  }

  // intersect.rs:266-289
  bool intersect_linear(V3 o, V3 d, float tmin, Hit& hit) const {
    float closest = std::numeric_limits<float>::infinity();
    bool found = false;
    Hit cand;
    for (uint32_t i = 0; i < spheres.size(); ++i)
      if (test_prim(o, d, PrimRef{kSphere, i}, tmin, closest, cand, nullptr)) { closest = cand.distance; hit = cand; found = true; }
    for (uint32_t i = 0; i < triangles.size(); ++i)
      if (test_prim(o, d, PrimRef{kTriangle, i}, tmin, closest, cand, nullptr)) { closest = cand.distance; hit = cand; found = true; }
    return found;
  }

  // light.rs:126-170
  bool sample_light(Rng& rng, V3& pos, V3& normal, V3& emission, float& pdf_area) const {
    if (lights.empty() || total_light_weight <= 0.0f) return false;
    float target = rng.uniform() * total_light_weight;
    const AreaLight* sel = &lights.back();
    for (const AreaLight& l : lights) {
      if (target < l.cumulative) { sel = &l; break; }
    }
    if (sel->is_triangle) {
      float su = std::sqrt(rng.uniform());
      float v = rng.uniform();
      float w0 = 1.0f - su, w1 = su * (1.0f - v), w2 = su * v;
      pos = sel->tri.v[0] * w0 + sel->tri.v[1] * w1 + sel->tri.v[2] * w2;
      normal = sel->normal;
    } else {
      float z = rng.range(-1.0f, 1.0f);
      float az = rng.range(0.0f, 2.0f * kPi);
      float radial = std::sqrt(std::fmax(1.0f - z * z, 0.0f));
      normal = v3(radial * std::cos(az), radial * std::sin(az), z);
      pos = sel->center + sel->radius * normal;
    }
    emission = sel->emission;
    float selection_pdf = sel->weight / total_light_weight;
    pdf_area = selection_pdf / sel->area;
    return true;
  }

  V3 texel_srgb(const Material& m, int x, int y) const {
    int w = int(m.tex_width), h = int(m.tex_height);
    int xi = ((x % w) + w) % w, yi = ((y % h) + h) % h;
    uint32_t px = texture_pixels[m.tex_offset + uint32_t(yi) * m.tex_width + uint32_t(xi)];
    auto lin = [](float s) { return s <= 0.04045f ? s / 12.92f : std::pow((s + 0.055f) / 1.055f, 2.4f); };
    return v3(lin(float(px & 255u) / 255.0f), lin(float((px >> 8) & 255u) / 255.0f), lin(float((px >> 16) & 255u) / 255.0f));
  }
  // Bilinear repeated texture lookup used by textured diffuse materials.
  V3 albedo_at(const Material& m, const Hit& h) const {
    if (m.tex_width == 0 || m.tex_height == 0) return m.albedo;
    float u = h.uv[0] - std::floor(h.uv[0]), v = h.uv[1] - std::floor(h.uv[1]);
    float px = u * float(m.tex_width) - 0.5f, py = v * float(m.tex_height) - 0.5f;
    int bx = int(std::floor(px)), by = int(std::floor(py));
    float ax = px - std::floor(px), ay = py - std::floor(py);
    V3 top = lerp(texel_srgb(m, bx, by), texel_srgb(m, bx + 1, by), ax);
    V3 bottom = lerp(texel_srgb(m, bx, by + 1), texel_srgb(m, bx + 1, by + 1), ax);
    return m.albedo * lerp(top, bottom, ay);
  }
};

// ---------------------------------------------------------------- integrator.rs
static float power_heuristic(float a, float b) {  // :247-256
  float a2 = a * a, b2 = b * b, den = a2 + b2;
  return den > 0.0f ? a2 / den : 0.0f;
}
static V3 reflect(V3 d, V3 n) { return d - 2.0f * dot(d, n) * n; }  // :353-355
static V3 refract(V3 d, V3 n, float ratio) {  // :358-363
  float cos_theta = std::fmin(dot(-d, n), 1.0f);
  V3 perp = ratio * (d + cos_theta * n);
  V3 par = -std::sqrt(std::fabs(1.0f - length_squared(perp))) * n;
  return perp + par;
}
static float reflectance(float cosine, float ratio) {  // :366-369
  float r0 = (1.0f - ratio) / (1.0f + ratio);
  r0 = r0 * r0;
  float m = 1.0f - cosine;
  return r0 + (1.0f - r0) * (m * m * m * m * m);
}
static V3 random_in_unit_sphere(Rng& rng) {  // :377-389
  for (;;) {
    V3 v = v3(rng.range(-1.0f, 1.0f), rng.range(-1.0f, 1.0f), rng.range(-1.0f, 1.0f));
    float l2 = length_squared(v);
    if (l2 >= 1e-8f && l2 <= 1.0f) return v;
  }
}
static V3 random_unit_vector(Rng& rng) { return normalize(random_in_unit_sphere(rng)); }

struct Scatter { V3 origin, direction, attenuation; bool has_pdf; float pdf; };

// integrator.rs:270-337
static bool scatter(V3 in_dir, const Hit& hit, const Material& m, V3 albedo, Rng& rng, Scatter& s) {
  s.origin = hit.point;
  if (m.kind == kDiffuse) {
    V3 dir = hit.normal + random_unit_vector(rng);
    if (length_squared(dir) < 1e-8f) dir = hit.normal;
    s.direction = normalize(dir);
    s.attenuation = albedo;
    s.has_pdf = true;
    s.pdf = std::fmax(dot(hit.normal, normalize(dir)), 0.0f) / kPi;
    return true;
  }
  if (m.kind == kMetal) {
    V3 refl = reflect(normalize(in_dir), hit.normal);
    float rough = std::fmin(std::fmax(m.roughness, 0.0f), 1.0f);
    V3 dir = refl + rough * random_in_unit_sphere(rng);
    if (dot(dir, hit.normal) <= 0.0f) return false;
    s.direction = normalize(dir);
    s.attenuation = m.albedo;
    s.has_pdf = false;
    return true;
  }
  if (m.kind == kDielectric) {
    float ratio = hit.front_face ? 1.0f / m.ior : m.ior;
    V3 unit = normalize(in_dir);
    float cos_theta = std::fmin(dot(-unit, hit.normal), 1.0f);
    float sin_theta = std::sqrt(1.0f - cos_theta * cos_theta);
    bool cannot = ratio * sin_theta > 1.0f;
    V3 dir;
    if (cannot || reflectance(cos_theta, ratio) > rng.uniform()) dir = reflect(unit, hit.normal);
    else dir = refract(unit, hit.normal, ratio);
    s.direction = normalize(dir);
    s.attenuation = splat(1.0f);
    s.has_pdf = false;
    return true;
  }
  return false;
}

struct Tracer {
  const Scene& sc;
  Counters* counters;

  // integrator.rs:168-205
  V3 direct_area_light(const Hit& hit, V3 albedo, Rng& rng) const {
    V3 pos, ln, emission;
    float pdf_area;
    if (!sc.sample_light(rng, pos, ln, emission, pdf_area)) return splat(0.0f);
    V3 so = hit.point + hit.normal * kRayEpsilon;
    V3 to_light = pos - so;
    float d2 = length_squared(to_light);
    if (d2 <= kRayEpsilon * kRayEpsilon) return splat(0.0f);
    float dist = std::sqrt(d2);
    V3 dir = to_light / dist;
    float cs = std::fmax(dot(hit.normal, dir), 0.0f);
    float cl = std::fmax(dot(ln, -dir), 0.0f);
    if (cs <= 0.0f || cl <= 0.0f) return splat(0.0f);
    Hit blocker;
    if (sc.intersect(so, dir, kRayEpsilon, blocker, counters) && blocker.distance < dist - 2.0f * kRayEpsilon)
      return splat(0.0f);
    V3 brdf = albedo / kPi;
    return brdf * emission * cs * cl / (d2 * pdf_area);
  }

  // integrator.rs:208-244
  V3 direct_environment(const Hit& hit, V3 albedo, Rng& rng) const {
    if (sc.background != kEnvironment || !sc.has_env) return splat(0.0f);
    float u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
    V3 dir, rad;
    float pdf;
    if (!sc.env.sample_importance(u1, u2, u3, dir, rad, pdf)) return splat(0.0f);
    float cs = std::fmax(dot(hit.normal, dir), 0.0f);
    if (cs <= 0.0f || pdf <= 0.0f) return splat(0.0f);
    Hit blocker;
    if (sc.intersect(hit.point + hit.normal * kRayEpsilon, dir, kRayEpsilon, blocker, counters)) return splat(0.0f);
    float bsdf_pdf = cs / kPi;
    float mis = power_heuristic(pdf, bsdf_pdf);
    V3 brdf = albedo / kPi;
    return brdf * rad * cs * mis / pdf;
  }

  // integrator.rs:99-165
  V3 ray_color(V3 o, V3 d, Rng& rng, uint32_t depth, bool include_emission, bool has_bsdf_pdf, float bsdf_pdf) const {
    if (depth == 0) return splat(0.0f);
    Hit hit;
    if (sc.intersect(o, d, kRayEpsilon, hit, counters)) {
      const Material& m = sc.materials[hit.material];
      if (m.kind == kEmissive) return include_emission ? m.albedo * m.strength : splat(0.0f);
      V3 albedo = m.kind == kDiffuse ? sc.albedo_at(m, hit) : m.albedo;
      Scatter s;
      if (scatter(d, hit, m, albedo, rng, s)) {
        bool next_include = m.kind != kDiffuse;
        V3 indirect = s.attenuation * ray_color(s.origin, s.direction, rng, depth - 1, next_include, s.has_pdf, s.pdf);
        V3 direct = splat(0.0f);
        if (m.kind == kDiffuse) direct = direct_area_light(hit, albedo, rng) + direct_environment(hit, albedo, rng);
        return direct + indirect;
      }
      return splat(0.0f);
    }
    if (sc.background == kSky) {
      V3 dir = normalize(d);
      float blend = 0.5f * (dir.y + 1.0f);
      return lerp(splat(1.0f), v3(0.35f, 0.65f, 1.0f), blend);
    }
    if (sc.background == kBlack || !sc.has_env) return splat(0.0f);
    V3 rad = sc.env.sample(d);
    float w = has_bsdf_pdf ? power_heuristic(bsdf_pdf, sc.env.pdf_solid_angle(d)) : 1.0f;
    return rad * w;
  }
};

}  // namespace orc

using namespace orc;

// ================================================================ C API (ctypes)
// Records use the byte layout of crates/toaster-gpu/src/gpu_types.rs (GpuSphere 32 B,
// GpuTriangle 64 B, GpuTriangleAttributes 80 B, GpuMaterial 48 B) so the oracle and the CUDA
// library consume the same packed arrays.
struct OrcSphereRec { float center_radius[4]; uint32_t material; uint32_t pad[3]; };
struct OrcTriangleRec { float v0[4], v1[4], v2[4]; uint32_t material; uint32_t pad[3]; };
struct OrcAttrRec { float n0[4], n1[4], n2[4]; float uv0[2], uv1[2], uv2[2]; uint32_t flags; uint32_t pad; };
struct OrcMaterialRec { uint32_t kind, tex_offset, tex_width, tex_height; float albedo[4]; float params[4]; };
static_assert(sizeof(OrcSphereRec) == 32, "GpuSphere layout");
static_assert(sizeof(OrcTriangleRec) == 64, "GpuTriangle layout");
static_assert(sizeof(OrcAttrRec) == 80, "GpuTriangleAttributes layout");
static_assert(sizeof(OrcMaterialRec) == 48, "GpuMaterial layout");

extern "C" {

struct OrcRenderSettings {
  float camera_position[3], camera_look_at[3], camera_up[3], fov_degrees;
  uint32_t width, height, samples, max_bounces, background;
};

void* orc_scene_create(const OrcSphereRec* spheres, uint32_t n_spheres, const OrcTriangleRec* tris, uint32_t n_tris,
                       const OrcAttrRec* attrs, const OrcMaterialRec* mats, uint32_t n_mats,
                       const uint32_t* texture_pixels, uint32_t n_texture_pixels,
                       const OrcRenderSettings* settings, const float* env_rgb, uint32_t env_w, uint32_t env_h,
                       float env_intensity, float env_rotation, uint32_t max_leaf) {
  auto* sc = new Scene();
  for (uint32_t i = 0; i < n_spheres; ++i) {
    const auto& r = spheres[i];
    sc->spheres.push_back(Sphere{v3(r.center_radius[0], r.center_radius[1], r.center_radius[2]), r.center_radius[3], r.material});
  }
  for (uint32_t i = 0; i < n_tris; ++i) {
    const auto& r = tris[i];
    sc->triangles.push_back(Triangle{{v3(r.v0[0], r.v0[1], r.v0[2]), v3(r.v1[0], r.v1[1], r.v1[2]), v3(r.v2[0], r.v2[1], r.v2[2])}, r.material});
    TriAttr a{};
    if (attrs) {
      const auto& ar = attrs[i];
      a.has_normals = (ar.flags & 1u) != 0;
      a.has_uvs = (ar.flags & 2u) != 0;
      a.n[0] = v3(ar.n0[0], ar.n0[1], ar.n0[2]);
      a.n[1] = v3(ar.n1[0], ar.n1[1], ar.n1[2]);
      a.n[2] = v3(ar.n2[0], ar.n2[1], ar.n2[2]);
      a.uv[0][0] = ar.uv0[0]; a.uv[0][1] = ar.uv0[1];
      a.uv[1][0] = ar.uv1[0]; a.uv[1][1] = ar.uv1[1];
      a.uv[2][0] = ar.uv2[0]; a.uv[2][1] = ar.uv2[1];
    }
    sc->attrs.push_back(a);
  }
  for (uint32_t i = 0; i < n_mats; ++i) {
    const auto& r = mats[i];
    Material m{};
    m.kind = r.kind;
    m.albedo = v3(r.albedo[0], r.albedo[1], r.albedo[2]);
    m.roughness = r.params[0];
    m.ior = r.params[1];
    m.strength = r.params[2];
    m.tex_offset = r.tex_offset; m.tex_width = r.tex_width; m.tex_height = r.tex_height;
    sc->materials.push_back(m);
  }
  if (texture_pixels && n_texture_pixels) sc->texture_pixels.assign(texture_pixels, texture_pixels + n_texture_pixels);
  if (settings) {
    sc->width = settings->width; sc->height = settings->height;
    sc->samples = settings->samples; sc->max_bounces = settings->max_bounces;
    sc->background = settings->background;
    const float* p = settings->camera_position;
    const float* l = settings->camera_look_at;
    const float* u = settings->camera_up;
    sc->camera.init(v3(p[0], p[1], p[2]), v3(l[0], l[1], l[2]), v3(u[0], u[1], u[2]), settings->fov_degrees,
                    float(settings->width) / float(settings->height));
  }
  if (env_rgb && env_w && env_h) {
    sc->env.init(env_w, env_h, env_rgb, env_intensity, env_rotation);
    sc->has_env = true;
  }
  sc->build_bvh(max_leaf ? max_leaf : 4);
  sc->collect_lights();
  return sc;
}

void orc_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

uint32_t orc_bvh_node_count(void* s) { return uint32_t(static_cast<Scene*>(s)->bvh.nodes.size()); }
uint32_t orc_bvh_prim_count(void* s) { return uint32_t(static_cast<Scene*>(s)->bvh.prims.size()); }

// Writes the flat hierarchy in GpuBvhNode order (gpu_types.rs:172-184): per node 8 floats
// (min.xyz, 0, max.xyz, 0) into `bounds`, and (first_or_right, count) into `links`;
// primitive references as (kind, index) pairs.
void orc_bvh_export(void* s, float* bounds, uint32_t* links, uint32_t* prims) {
  const Scene* sc = static_cast<Scene*>(s);
  for (size_t i = 0; i < sc->bvh.nodes.size(); ++i) {
    const FlatNode& n = sc->bvh.nodes[i];
    float* b = bounds + 8 * i;
    b[0] = n.bounds.min.x; b[1] = n.bounds.min.y; b[2] = n.bounds.min.z; b[3] = 0.0f;
    b[4] = n.bounds.max.x; b[5] = n.bounds.max.y; b[6] = n.bounds.max.z; b[7] = 0.0f;
    links[2 * i] = n.first_or_right;
    links[2 * i + 1] = n.count;
  }
  for (size_t i = 0; i < sc->bvh.prims.size(); ++i) {
    prims[2 * i] = sc->bvh.prims[i].kind;
    prims[2 * i + 1] = sc->bvh.prims[i].index;
  }
}

// Closest hit for n rays (origin.xyz, direction.xyz) with min distance `tmin`.
// prim[i] = kind << 31 | index, or 0xFFFFFFFF on a miss; t[i] = distance or +inf.
// hit_info (optional, 8 floats per ray): normal.xyz, front_face, material, uv.xy, 0.
// counts (optional, 6 u64): rays, node tests, sphere tests, triangle tests, interior, leaf.
void orc_trace_closest(void* s, const float* rays, uint64_t n, float tmin, uint32_t* prim, float* t,
                       float* hit_info, uint64_t* counts, int linear) {
  const Scene* sc = static_cast<Scene*>(s);
  Counters total;
#pragma omp parallel
  {
    Counters local;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < int64_t(n); ++i) {
      const float* r = rays + 6 * i;
      Hit h;
      bool ok = linear ? sc->intersect_linear(v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), tmin, h)
                       : sc->intersect(v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), tmin, h, counts ? &local : nullptr);
      if (ok) {
        prim[i] = (h.prim.kind << 31) | h.prim.index;
        t[i] = h.distance;
      } else {
        prim[i] = 0xFFFFFFFFu;
        t[i] = std::numeric_limits<float>::infinity();
      }
      if (hit_info) {
        float* hi = hit_info + 8 * i;
        if (ok) {
          hi[0] = h.normal.x; hi[1] = h.normal.y; hi[2] = h.normal.z; hi[3] = h.front_face ? 1.0f : 0.0f;
          hi[4] = float(h.material); hi[5] = h.uv[0]; hi[6] = h.uv[1]; hi[7] = 0.0f;
        } else {
          for (int k = 0; k < 8; ++k) hi[k] = 0.0f;
        }
      }
    }
#pragma omp critical
    total.add(local);
  }
  if (counts) {
    counts[0] = total.rays; counts[1] = total.node_tests; counts[2] = total.sphere_tests;
    counts[3] = total.triangle_tests; counts[4] = total.interior_visits; counts[5] = total.leaf_visits;
  }
}

// One recursive radiance estimate per ray (integrator.rs:73-93 semantics) with caller seeds.
// out: 3 floats per ray. bsdf_pdf < 0 means "None" for the environment MIS weight.
void orc_ray_color(void* s, const float* rays, uint64_t n, uint32_t depth, int include_emission, float bsdf_pdf,
                   uint64_t seed, float* out) {
  const Scene* sc = static_cast<Scene*>(s);
  Tracer tr{*sc, nullptr};
  for (uint64_t i = 0; i < n; ++i) {
    Rng rng(seed ^ (i * 0x9E3779B97F4A7C15ull));
    const float* r = rays + 6 * i;
    V3 c = tr.ray_color(v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), rng, depth, include_emission != 0,
                        bsdf_pdf >= 0.0f, bsdf_pdf);
    out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
  }
}

// Renders rows [row0, row1) stepping by row_step (integrator.rs:24-67 per pixel), writing the
// per-pixel mean (3 floats) and, optionally, the per-pixel sum of squared sample values
// (3 doubles) for variance estimates. Seeds are per pixel so any thread count gives the same
// image. threads <= 0 uses all OpenMP threads. counts (optional, 6 u64) as in orc_trace_closest.
void orc_render(void* s, uint64_t seed, uint32_t row0, uint32_t row1, uint32_t row_step, int threads, float* mean,
                double* sumsq, uint64_t* counts) {
  const Scene* sc = static_cast<Scene*>(s);
  uint32_t w = sc->width, spp = sc->samples;
  std::vector<uint32_t> rows;
  for (uint32_t y = row0; y < row1; y += (row_step ? row_step : 1)) rows.push_back(y);
  Counters total;
#ifdef _OPENMP
  int nt = threads > 0 ? threads : omp_get_max_threads();
#else
  int nt = 1;
  (void)threads;
#endif
#pragma omp parallel num_threads(nt)
  {
    Counters local;
    Tracer tr{*sc, counts ? &local : nullptr};
#pragma omp for schedule(dynamic, 16)
    for (int64_t item = 0; item < int64_t(rows.size()) * int64_t(w); ++item) {
      const int64_t ri = item / int64_t(w);
      const uint32_t y = rows[size_t(ri)];
      const uint32_t x = uint32_t(item - ri * int64_t(w));
      {
        uint64_t pix = uint64_t(y) * w + x;
        Rng rng(seed * 0xD1B54A32D192ED03ull + pix);
        V3 sum = splat(0.0f);
        double sq[3] = {0.0, 0.0, 0.0};
        for (uint32_t k = 0; k < spp; ++k) {
          float u = (float(x) + rng.uniform()) / float(sc->width);
          float v = 1.0f - (float(y) + rng.uniform()) / float(sc->height);
          V3 o, d;
          sc->camera.ray(u, v, o, d);
          V3 c = tr.ray_color(o, d, rng, sc->max_bounces, true, false, 0.0f);
          sum += c;
          sq[0] += double(c.x) * c.x; sq[1] += double(c.y) * c.y; sq[2] += double(c.z) * c.z;
        }
        V3 m = sum / float(spp);
        size_t o3 = size_t(ri) * w * 3 + size_t(x) * 3;
        mean[o3] = m.x; mean[o3 + 1] = m.y; mean[o3 + 2] = m.z;
        if (sumsq) { sumsq[o3] = sq[0]; sumsq[o3 + 1] = sq[1]; sumsq[o3 + 2] = sq[2]; }
      }
    }
#pragma omp critical
    total.add(local);
  }
  if (counts) {
    counts[0] = total.rays; counts[1] = total.node_tests; counts[2] = total.sphere_tests;
    counts[3] = total.triangle_tests; counts[4] = total.interior_visits; counts[5] = total.leaf_visits;
  }
}

// ---- known-answer hooks (restated reference unit tests call these directly)

// aabb.rs:74-110 on explicit bounds and inverse direction.
int orc_aabb_intersects(const float* mn, const float* mx, const float* origin, const float* inv, float tmin,
                        float tmax) {
  Aabb b{v3(mn[0], mn[1], mn[2]), v3(mx[0], mx[1], mx[2])};
  return b.intersects_ray(v3(origin[0], origin[1], origin[2]), v3(inv[0], inv[1], inv[2]), tmin, tmax) ? 1 : 0;
}

// Camera basis (camera.rs:54-91): out = origin, lower_left, horizontal, vertical (12 floats).
int orc_camera_basis(const float* pos, const float* look, const float* up, float fov, float aspect, float* out) {
  Camera c;
  if (!c.init(v3(pos[0], pos[1], pos[2]), v3(look[0], look[1], look[2]), v3(up[0], up[1], up[2]), fov, aspect)) return 0;
  const V3 vs[4] = {c.origin, c.lower_left, c.horizontal, c.vertical};
  for (int i = 0; i < 4; ++i) { out[3 * i] = vs[i].x; out[3 * i + 1] = vs[i].y; out[3 * i + 2] = vs[i].z; }
  return 1;
}

// Scatter one incoming direction off a synthetic hit (integrator.rs:270-337).
// hit: point.xyz, normal.xyz, front_face; material: kind, albedo.xyz, roughness, ior.
// out: direction.xyz, attenuation.xyz, pdf (or -1). Returns 0 when absorbed.
int orc_scatter(const float* in_dir, const float* hit, const float* material, uint64_t seed, float* out) {
  Hit h{};
  h.point = v3(hit[0], hit[1], hit[2]);
  h.normal = v3(hit[3], hit[4], hit[5]);
  h.front_face = hit[6] != 0.0f;
  Material m{};
  m.kind = uint32_t(material[0]);
  m.albedo = v3(material[1], material[2], material[3]);
  m.roughness = material[4];
  m.ior = material[5];
  Rng rng(seed);
  Scatter s;
  if (!scatter(v3(in_dir[0], in_dir[1], in_dir[2]), h, m, m.albedo, rng, s)) return 0;
  out[0] = s.direction.x; out[1] = s.direction.y; out[2] = s.direction.z;
  out[3] = s.attenuation.x; out[4] = s.attenuation.y; out[5] = s.attenuation.z;
  out[6] = s.has_pdf ? s.pdf : -1.0f;
  return 1;
}

void orc_refract(const float* d, const float* n, float ratio, float* out) {
  V3 r = refract(v3(d[0], d[1], d[2]), v3(n[0], n[1], n[2]), ratio);
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
float orc_reflectance(float cosine, float ratio) { return reflectance(cosine, ratio); }
float orc_power_heuristic(float a, float b) { return power_heuristic(a, b); }

// Direct lighting at a synthetic hit (integrator.rs:168-244). which: 0 = area light, 1 = environment.
void orc_direct(void* s, const float* hit, const float* albedo, int which, uint64_t seed, uint32_t draws, float* out) {
  const Scene* sc = static_cast<Scene*>(s);
  Hit h{};
  h.point = v3(hit[0], hit[1], hit[2]);
  h.normal = v3(hit[3], hit[4], hit[5]);
  h.front_face = true;
  Tracer tr{*sc, nullptr};
  Rng rng(seed);
  V3 sum = splat(0.0f);
  for (uint32_t i = 0; i < draws; ++i) {
    V3 a = v3(albedo[0], albedo[1], albedo[2]);
    sum += which == 0 ? tr.direct_area_light(h, a, rng) : tr.direct_environment(h, a, rng);
  }
  out[0] = sum.x; out[1] = sum.y; out[2] = sum.z;
}

// Light list (light.rs:57-113): per light 4 floats (area, weight, cumulative, kind) + total.
uint32_t orc_lights(void* s, float* out, float* total) {
  const Scene* sc = static_cast<Scene*>(s);
  for (size_t i = 0; i < sc->lights.size(); ++i) {
    out[4 * i] = sc->lights[i].area; out[4 * i + 1] = sc->lights[i].weight;
    out[4 * i + 2] = sc->lights[i].cumulative; out[4 * i + 3] = sc->lights[i].is_triangle ? 0.0f : 1.0f;
  }
  if (total) *total = sc->total_light_weight;
  return uint32_t(sc->lights.size());
}

// Draws n light samples: per draw (pos.xyz, normal.xyz, emission.xyz, pdf_area).
void orc_sample_lights(void* s, uint64_t seed, uint32_t n, float* out) {
  const Scene* sc = static_cast<Scene*>(s);
  Rng rng(seed);
  for (uint32_t i = 0; i < n; ++i) {
    V3 p, nn, e;
    float pdf = 0.0f;
    if (!sc->sample_light(rng, p, nn, e, pdf)) { std::memset(out + 10 * i, 0, 40); continue; }
    float* o = out + 10 * i;
    o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = nn.x; o[4] = nn.y; o[5] = nn.z;
    o[6] = e.x; o[7] = e.y; o[8] = e.z; o[9] = pdf;
  }
}

// ---- environment hooks (environment.rs)
void* orc_env_create(uint32_t w, uint32_t h, const float* rgb, float intensity, float rotation) {
  auto* e = new Environment();
  e->init(w, h, rgb, intensity, rotation);
  return e;
}
void orc_env_destroy(void* e) { delete static_cast<Environment*>(e); }
void orc_env_cdf(void* e, float* out) {
  const Environment* env = static_cast<Environment*>(e);
  std::copy(env->cdf.begin(), env->cdf.end(), out);
}
float orc_env_rotation(void* e) { return static_cast<Environment*>(e)->rotation_degrees; }
void orc_env_lookup(void* e, const float* dirs, uint32_t n, float* out_rgb, float* out_pdf) {
  const Environment* env = static_cast<Environment*>(e);
  for (uint32_t i = 0; i < n; ++i) {
    V3 d = v3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    V3 r = env->sample(d);
    out_rgb[3 * i] = r.x; out_rgb[3 * i + 1] = r.y; out_rgb[3 * i + 2] = r.z;
    if (out_pdf) out_pdf[i] = env->pdf_solid_angle(d);
  }
}
// uniforms: 3 per sample; out: direction.xyz, radiance.xyz, pdf, valid (8 floats).
void orc_env_sample(void* e, const float* uniforms, uint32_t n, float* out) {
  const Environment* env = static_cast<Environment*>(e);
  for (uint32_t i = 0; i < n; ++i) {
    V3 d, r;
    float pdf = 0.0f;
    bool ok = env->sample_importance(uniforms[3 * i], uniforms[3 * i + 1], uniforms[3 * i + 2], d, r, pdf);
    float* o = out + 8 * i;
    o[0] = d.x; o[1] = d.y; o[2] = d.z; o[3] = r.x; o[4] = r.y; o[5] = r.z; o[6] = pdf; o[7] = ok ? 1.0f : 0.0f;
  }
}
// Direction -> (u, v, sin_theta) per environment.rs:213-222; returns 0 for a zero direction.
int orc_env_direction_to_uv(void* e, const float* d, float* out) {
  const Environment* env = static_cast<Environment*>(e);
  return env->direction_to_uv(v3(d[0], d[1], d[2]), out[0], out[1], out[2]) ? 1 : 0;
}

// crates/toaster-core/src/color.rs:24-74 and crates/toaster-gpu/src/image_output.rs:57-88: exposure,
// ACES fitted tone map, clamp, sRGB transfer, round to bytes; alpha clamped and rounded.
static float aces_channel(float c) {
  if (std::isnan(c)) return 0.0f;
  if (!std::isfinite(c)) return c > 0.0f ? 1.0f : 0.0f;
  c = std::fmax(c, 0.0f);
  return (c * (2.51f * c + 0.03f)) / (c * (2.43f * c + 0.59f) + 0.14f);
}
static float linear_to_srgb(float c) {
  return c <= 0.0031308f ? 12.92f * c : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
}
static uint8_t channel_to_u8(float c) { return uint8_t(std::round(std::fmin(std::fmax(c, 0.0f), 1.0f) * 255.0f)); }

void orc_display_rgba8(const float* rgba, uint64_t n, float exposure_stops, uint8_t* out) {
  const float scale = std::exp2(exposure_stops);
  for (uint64_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      float t = aces_channel(rgba[4 * i + c] * scale);
      t = std::fmin(std::fmax(t, 0.0f), 1.0f);
      out[4 * i + c] = channel_to_u8(linear_to_srgb(t));
    }
    out[4 * i + 3] = channel_to_u8(rgba[4 * i + 3]);
  }
}

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
