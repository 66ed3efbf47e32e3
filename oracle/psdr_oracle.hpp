// psdr_oracle.hpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A CPU restatement of the differentiable path tracer of LiuLinyun/torch_psdr,
// templated on the scalar type:
//   float      -> the FP32 instance: timed CPU baseline, bit-exact intersection KAT;
//   double     -> the FP64 oracle every GPU image/gradient is compared against;
//   Dual<K>    -> forward-mode derivatives (K tangent directions) of the same
//                 estimator, reproducing the reference's detach() semantics, used to
//                 check the hand-written GPU adjoint.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
// The product (torch_psdr_b200) never links, calls or executes anything here.
//
// PARITY UNPINNED. The reference ships no tests, golden images or known-answer
// vectors, and it cannot be built or run here (bazel, clang-15/libc++, the unpinned
// enoki master.zip and the OptiX SDK are all absent). Each function below cites the
// reference file:line it restates. Third-party arithmetic the reference calls is
// restated from its published definition:
//   * enoki::PCG32 (enoki master, unpinned; WORKSPACE:17-22): O'Neill's PCG32
//     XSH-RR 64/32 with the pcg-basic default constants, masked advance, float
//     mapping (x>>9)|0x3f800000 - 1.
//   * enoki::binary_search: fixed log2(n)+1 bisection steps.
//   * OptiX closest hit (scene_optix.cc:240-277, device_programs.cu:13-47): replaced
//     by the watertight ray/triangle test of Woop, Benthin & Wald (JCGT 2013) with
//     tmin = 1e-3 and ties broken by the smaller triangle id.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <utility>
#include <vector>

namespace orc {

// ------------------------------------------------------------------ scalars
template <int K> struct Dual {
  double v;
  double d[K];
  Dual() : v(0) { for (int i = 0; i < K; ++i) d[i] = 0; }
  Dual(double x) : v(x) { for (int i = 0; i < K; ++i) d[i] = 0; }
};
template <int K> inline Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v + b.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <int K> inline Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v - b.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <int K> inline Dual<K> operator-(const Dual<K>& a) { Dual<K> r(-a.v); for (int i = 0; i < K; ++i) r.d[i] = -a.d[i]; return r; }
template <int K> inline Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v * b.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int K> inline Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v / b.v); double ib = 1.0 / b.v; for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib; return r; }
template <int K> inline Dual<K>& operator+=(Dual<K>& a, const Dual<K>& b) { a = a + b; return a; }
template <int K> inline Dual<K>& operator-=(Dual<K>& a, const Dual<K>& b) { a = a - b; return a; }
template <int K> inline Dual<K>& operator*=(Dual<K>& a, const Dual<K>& b) { a = a * b; return a; }
template <int K> inline Dual<K>& operator/=(Dual<K>& a, const Dual<K>& b) { a = a / b; return a; }

template <class S> struct Traits { using R = S; };
template <int K> struct Traits<Dual<K>> { using R = double; };

inline double val(double x) { return x; }
inline float val(float x) { return x; }
template <int K> inline double val(const Dual<K>& x) { return x.v; }
inline double detach(double x) { return x; }
inline float detach(float x) { return x; }
template <int K> inline Dual<K> detach(const Dual<K>& x) { return Dual<K>(x.v); }

inline float sqrt_(float x) { return std::sqrt(x); }
inline double sqrt_(double x) { return std::sqrt(x); }
template <int K> inline Dual<K> sqrt_(const Dual<K>& x) {
  Dual<K> r(std::sqrt(x.v));
  double g = r.v > 0 ? 0.5 / r.v : 0.0;
  for (int i = 0; i < K; ++i) r.d[i] = x.d[i] * g;
  return r;
}
template <class S> inline S safe_sqrt(const S& x) { return val(x) > 0 ? sqrt_(x) : S(0); }
inline float sin_(float x) { return std::sin(x); }
inline double sin_(double x) { return std::sin(x); }
inline float cos_(float x) { return std::cos(x); }
inline double cos_(double x) { return std::cos(x); }
template <class S> inline S abs_(const S& x) { return val(x) < 0 ? -x : x; }
template <class S> inline S max0(const S& x) { return val(x) > 0 ? x : S(0); }
// enoki::clamp = max(min(x, hi), lo): the derivative passes only strictly inside.
template <class S> inline S clamp_(const S& x, double lo, double hi) {
  if (val(x) < lo) return S(lo);
  if (val(x) > hi) return S(hi);
  return x;
}

// ------------------------------------------------------------------ vectors
template <class S> struct V3 {
  S x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(S a, S b, S c) : x(a), y(b), z(c) {}
  S& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const S& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class S> inline V3<S> operator+(const V3<S>& a, const V3<S>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> inline V3<S> operator-(const V3<S>& a, const V3<S>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> inline V3<S> operator-(const V3<S>& a) { return {-a.x, -a.y, -a.z}; }
template <class S> inline V3<S> operator*(const V3<S>& a, const S& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S> inline V3<S> operator*(const S& s, const V3<S>& a) { return {a.x * s, a.y * s, a.z * s}; }
template <class S> inline V3<S> mul(const V3<S>& a, const V3<S>& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class S> inline V3<S> operator/(const V3<S>& a, const S& s) { return {a.x / s, a.y / s, a.z / s}; }
template <class S> inline S dot(const V3<S>& a, const V3<S>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> inline V3<S> cross(const V3<S>& a, const V3<S>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class S> inline S sqnorm(const V3<S>& a) { return dot(a, a); }
template <class S> inline S norm(const V3<S>& a) { return sqrt_(sqnorm(a)); }
template <class S> inline V3<S> normalize(const V3<S>& a) { return a / norm(a); }
template <class S> inline V3<S> detach(const V3<S>& a) { return {detach(a.x), detach(a.y), detach(a.z)}; }
template <class S> inline V3<typename Traits<S>::R> valv(const V3<S>& a) {
  using R = typename Traits<S>::R;
  return {R(val(a.x)), R(val(a.y)), R(val(a.z))};
}
template <class S> inline V3<double> val3(const V3<S>& a) { return {double(val(a.x)), double(val(a.y)), double(val(a.z))}; }
template <class S, class T> inline V3<S> cvt(const V3<T>& a) { return {S(a.x), S(a.y), S(a.z)}; }
template <class S> inline bool finite3(const V3<S>& a) { return std::isfinite(val(sqnorm(a))); }

// ------------------------------------------------------------------ PCG32 + TEA
// enoki/random.h PCG32 (third-party, restated from the PCG paper / pcg-basic).
constexpr uint64_t PCG32_DEFAULT_STATE = 0x853c49e6748fea9bULL;
constexpr uint64_t PCG32_DEFAULT_STREAM = 0xda3e39cb94b95bdbULL;
constexpr uint64_t PCG32_MULT = 0x5851f42d4c957f2dULL;

struct Pcg32 {
  uint64_t state = 0, inc = 0;
  uint32_t next(bool advance = true) {
    uint64_t old = state;
    if (advance) state = old * PCG32_MULT + inc;
    uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
    uint32_t rot = (uint32_t)(old >> 59);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  void seed(uint64_t initstate, uint64_t initseq) {
    state = 0;
    inc = (initseq << 1) | 1u;
    next();
    state += initstate;
    next();
  }
  float next_float(bool advance = true) {
    uint32_t bits = (next(advance) >> 9) | 0x3f800000u;
    float f;
    std::memcpy(&f, &bits, 4);
    return f - 1.0f;
  }
};

// sampler.h:70-80 sample_tea_64 (4 rounds)
inline uint64_t tea64(uint32_t v0, uint32_t v1) {
  uint32_t sum = 0;
  for (int i = 0; i < 4; ++i) {
    sum += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return (uint64_t)v0 + ((uint64_t)v1 << 32);
}

// sampler.h:11-17: stream i is seeded with tea(i + DEFAULT_STATE, i) / tea(i, i + DEFAULT_STATE),
// both arguments truncated to 32 bits.
inline Pcg32 make_sampler(uint64_t i) {
  uint32_t a = (uint32_t)(i + PCG32_DEFAULT_STATE);
  uint32_t b = (uint32_t)i;
  Pcg32 p;
  p.seed(tea64(a, b), tea64(b, a));
  return p;
}

// ------------------------------------------------------------------ discrete sampler
// sampler.h:86-117 DiscreteSampler: pmf = w / sum(w), cmf = inclusive prefix sum.
// pmf/cmf are formed in double and rounded to the working precision R.
template <class R> struct Discrete {
  int n = 0;
  std::vector<R> pmf, cmf;
  double sum = 0;
  void build(const std::vector<double>& w) {
    n = (int)w.size();
    sum = 0;
    for (double x : w) sum += x;
    pmf.resize(n);
    cmf.resize(n);
    double acc = 0;
    for (int i = 0; i < n; ++i) {
      acc += w[i];
      pmf[i] = R(w[i] / sum);
      cmf[i] = R(acc / sum);
    }
  }
  // sample_reuse: binary search for the first cmf >= s, then rescale s in place.
  int sample_reuse(R& s, R& pdf) const {
    if (n == 1) { pdf = R(1); return 0; }
    int start = 0, end = n - 1;
    int span = end - start;
    int iters = 0;
    while ((1 << (iters)) <= span) ++iters;  // floor(log2(span)) + 1
    for (int it = 0; it < iters; ++it) {
      int mid = (start + end) >> 1;
      bool cond = cmf[mid] < s;
      if (cond) start = std::min(mid + 1, end);
      else end = mid;
    }
    int idx = start;
    pdf = pmf[idx];
    R prev = idx > 0 ? cmf[idx - 1] : R(0);
    s = (s - prev) / pdf;
    return idx;
  }
};

// ------------------------------------------------------------------ ray/triangle
// Watertight test (Woop, Benthin, Wald 2013). Evaluated in R with a fixed order of
// IEEE operations; the GPU kernel performs the identical sequence (no contraction).
template <class R> struct RayPre {
  R o[3];
  int kx, ky, kz;
  R Sx, Sy, Sz;
};
template <class R> inline RayPre<R> ray_pre(const R o[3], const R d[3]) {
  RayPre<R> p;
  for (int i = 0; i < 3; ++i) p.o[i] = o[i];
  R ax = std::fabs(d[0]), ay = std::fabs(d[1]), az = std::fabs(d[2]);
  int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  if (d[kz] < R(0)) std::swap(kx, ky);
  p.kx = kx; p.ky = ky; p.kz = kz;
  p.Sx = d[kx] / d[kz];
  p.Sy = d[ky] / d[kz];
  p.Sz = R(1) / d[kz];
  return p;
}
template <class R>
inline bool tri_test(const RayPre<R>& r, const R* p0, const R* p1, const R* p2, R tmin, R tmax,
                     R& t, R& b1, R& b2) {
  const int kx = r.kx, ky = r.ky, kz = r.kz;
  R A[3], B[3], C[3];
  for (int i = 0; i < 3; ++i) { A[i] = p0[i] - r.o[i]; B[i] = p1[i] - r.o[i]; C[i] = p2[i] - r.o[i]; }
  R Ax = A[kx] - r.Sx * A[kz], Ay = A[ky] - r.Sy * A[kz];
  R Bx = B[kx] - r.Sx * B[kz], By = B[ky] - r.Sy * B[kz];
  R Cx = C[kx] - r.Sx * C[kz], Cy = C[ky] - r.Sy * C[kz];
  R U = Cx * By - Cy * Bx;
  R V = Ax * Cy - Ay * Cx;
  R W = Bx * Ay - By * Ax;
  if ((U < R(0) || V < R(0) || W < R(0)) && (U > R(0) || V > R(0) || W > R(0))) return false;
  R det = (U + V) + W;
  if (det == R(0)) return false;
  R Az = r.Sz * A[kz], Bz = r.Sz * B[kz], Cz = r.Sz * C[kz];
  R T = (U * Az + V * Bz) + W * Cz;
  R tt = T / det;
  if (!(tt > tmin && tt <= tmax)) return false;
  t = tt;
  b1 = V / det;
  b2 = W / det;
  return true;
}

// ------------------------------------------------------------------ scene inputs (C layout)
extern "C" {
struct OrcTexture {
  int kind;  // 0 constant, 1 uv map
  int h, w, c;
  const float* data;  // constant: c floats; uv: (h, w, c) in the caller's row order
};
struct OrcMesh {
  const float* V; int nV;
  const int* F; int nF;
  const float* uv; int nUV;   // may be null
  const int* uvi;             // may be null
  int mat;                    // 0 DiffuseMaterial, 1 DiffuseBsdfMaterial
  OrcTexture color;
  OrcTexture rough;           // DiffuseBsdfMaterial: 1 channel
  OrcTexture normal;          // DiffuseBsdfMaterial: 3 channels, kind -1 = none
};
struct OrcLight {
  const float* V; int nV;     // area light mesh (environment lights: ignored)
  const int* F; int nF;
  float emit[3];
  int type;                   // 0 AreaLight, 1 EnvLight (cube map), 2 SH9Light
  OrcTexture cube_map;        // EnvLight: UV3f texture
  float sh9[27];              // SH9Light: 9 x 3 coefficients, row-major
  float box_min[3], box_max[3];  // environment lights: the bounding box (scene.cc:31-49)
};
struct OrcCamera {
  float look_from[3], look_at[3], up[3];
  float fov;   // perspective: vertical field of view; orthographic: view width
  int h, w;
  int type;    // 0 perspective, 1 orthographic
};
struct OrcConfig {
  int n_pass, spp_interior, enable_light_visable, spp_primary_edge, spp_secondary_edge;
  int max_bounce, mis_light_samples, mis_bsdf_samples;
  int pe_rounds, se_rounds, pe_res, se_res[3];
  int mode;  // 0: reference formulas, 1: unbiased estimator
  int spp_pixel_boundary;  // pixel-border samples per border segment (unbiased estimator)
  uint64_t seed;  // stream offset seed * 2654435761 of every non-preprocess stream (the GPU's seed)
};
}

// ------------------------------------------------------------------ camera
struct M4 { double m[4][4]; };
inline M4 mmul(const M4& a, const M4& b) {
  M4 r{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a.m[i][k] * b.m[k][j];
      r.m[i][j] = s;
    }
  return r;
}
inline M4 minv(const M4& a) {
  double m[4][8];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 8; ++j) m[i][j] = j < 4 ? a.m[i][j] : (j - 4 == i ? 1.0 : 0.0);
  for (int c = 0; c < 4; ++c) {
    int p = c;
    for (int r = c + 1; r < 4; ++r) if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
    for (int j = 0; j < 8; ++j) std::swap(m[c][j], m[p][j]);
    double iv = 1.0 / m[c][c];
    for (int j = 0; j < 8; ++j) m[c][j] *= iv;
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      double f = m[r][c];
      for (int j = 0; j < 8; ++j) m[r][j] -= f * m[c][j];
    }
  }
  M4 r{};
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) r.m[i][j] = m[i][j + 4];
  return r;
}

// camera.h:7-64 (perspective, orthographic, look_at), :111-124 (BaseCamera), psdr.cc:24-37
// (near -0.01, far -1000), camera.h:290-300 (orthographic view box: width view_width,
// height view_width H / W).
template <class R> struct Camera {
  R r2c[4][4], c2w[4][4], w2c[4][4], c2r[4][4];
  int H, W;
  int ortho = 0;
  V3<double> pos_d;
  void setup(const OrcCamera& c) {
    H = c.h; W = c.w;
    double o[3] = {c.look_from[0], c.look_from[1], c.look_from[2]};
    double t[3] = {c.look_at[0], c.look_at[1], c.look_at[2]};
    double u[3] = {c.up[0], c.up[1], c.up[2]};
    auto nrm = [](double* v) { double n = std::sqrt(v[0]*v[0]+v[1]*v[1]+v[2]*v[2]); v[0]/=n; v[1]/=n; v[2]/=n; };
    auto crs = [](const double* a, const double* b, double* r) {
      r[0] = a[1]*b[2]-a[2]*b[1]; r[1] = a[2]*b[0]-a[0]*b[2]; r[2] = a[0]*b[1]-a[1]*b[0]; };
    double dir[3] = {o[0]-t[0], o[1]-t[1], o[2]-t[2]};
    nrm(dir); nrm(u);
    double right[3], nup[3];
    crs(u, dir, right);
    crs(dir, right, nup);
    M4 cw{};
    for (int i = 0; i < 3; ++i) { cw.m[i][0] = right[i]; cw.m[i][1] = nup[i]; cw.m[i][2] = dir[i]; cw.m[i][3] = o[i]; }
    cw.m[3][3] = 1;
    double nearv = -0.01, farv = -1000.0;
    M4 cs{};
    ortho = c.type == 1;
    if (ortho) {
      // orthographic(left, right, bottom, top, near, far) = scale * translate
      double hw = double(c.fov) / 2, hh = double(H) * hw / double(W);
      cs.m[0][0] = 2 / (2 * hw);
      cs.m[1][1] = 2 / (2 * hh);
      cs.m[2][2] = 2 / (nearv - farv);
      cs.m[2][3] = cs.m[2][2] * (-(nearv + farv) / 2);
      cs.m[3][3] = 1;
    } else {
      double inv_nf = 1.0 / (nearv - farv);
      double cot = 1.0 / std::tan(double(c.fov) * 0.5);
      cs.m[0][0] = -cot; cs.m[1][1] = -cot; cs.m[2][2] = (nearv + farv) * inv_nf;
      cs.m[2][3] = -2 * farv * nearv * inv_nf; cs.m[3][2] = 1;
    }
    M4 sr{};
    sr.m[0][0] = 0.5 * W; sr.m[1][1] = -0.5 * H; sr.m[2][2] = 1; sr.m[3][3] = 1;
    M4 tr{};
    tr.m[0][0] = tr.m[1][1] = tr.m[2][2] = tr.m[3][3] = 1; tr.m[0][3] = 1; tr.m[1][3] = -1;
    M4 c2r_ = mmul(mmul(sr, tr), cs);
    M4 r2c_ = minv(c2r_);
    M4 w2c_ = minv(cw);
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) {
      r2c[i][j] = R(r2c_.m[i][j]); c2w[i][j] = R(cw.m[i][j]); w2c[i][j] = R(w2c_.m[i][j]); c2r[i][j] = R(c2r_.m[i][j]);
    }
    pos_d = V3<double>(o[0], o[1], o[2]);
  }
  template <class S> static V3<S> xpos(const R m[4][4], const V3<S>& p) {
    S w = S(m[3][0]) * p.x + S(m[3][1]) * p.y + S(m[3][2]) * p.z + S(m[3][3]);
    V3<S> r(S(m[0][0]) * p.x + S(m[0][1]) * p.y + S(m[0][2]) * p.z + S(m[0][3]),
            S(m[1][0]) * p.x + S(m[1][1]) * p.y + S(m[1][2]) * p.z + S(m[1][3]),
            S(m[2][0]) * p.x + S(m[2][1]) * p.y + S(m[2][2]) * p.z + S(m[2][3]));
    return r / w;
  }
  template <class S> static V3<S> xdir(const R m[4][4], const V3<S>& p) {
    return V3<S>(S(m[0][0]) * p.x + S(m[0][1]) * p.y + S(m[0][2]) * p.z,
                 S(m[1][0]) * p.x + S(m[1][1]) * p.y + S(m[1][2]) * p.z,
                 S(m[2][0]) * p.x + S(m[2][1]) * p.y + S(m[2][2]) * p.z);
  }
};

// ------------------------------------------------------------------ scene
template <class S> struct Tri {
  V3<S> p0, p1, p2, n, t;
  S area;
  double uv[6];
  int obj;
};
template <class S> struct Edge {
  V3<S> p0, p1, out, nl, nr;
  S len;
  int v0, v1;  // global vertex ids
};

template <class S> struct Scene {
  using R = typename Traits<S>::R;
  std::vector<V3<S>> verts;          // global vertex list (objects then light meshes)
  std::vector<std::array<int, 3>> faces;
  std::vector<Tri<S>> tris;
  std::vector<Edge<S>> edges;
  Discrete<R> edge_cdf;
  // objects: first n_obj are meshes, the rest are light meshes
  int n_obj = 0;
  std::vector<int> obj_light;        // light index or -1
  std::vector<int> obj_tex_kind, obj_tex_h, obj_tex_w, obj_tex_off;
  // DiffuseBsdfMaterial: roughness (1 channel) and normal map (3 channels) in `tex`
  struct TexRef { int kind = -1, h = 0, w = 0, c = 0, off = -1; };
  std::vector<int> obj_mat;
  std::vector<TexRef> obj_rough, obj_nrm;
  std::vector<S> tex;                // all textures concatenated (caller row order, 3 channels)
  std::vector<int> obj_vert_off;
  // lights
  std::vector<V3<S>> emit;
  std::vector<int> light_kind;          // 0 area, 1 env cube map, 2 SH9
  std::vector<TexRef> light_tex;        // env: cube map; SH9: the 27 coefficients (c = 27)
  std::vector<int> light_tri0, light_ntri;
  std::vector<Discrete<R>> light_tri_cdf;
  std::vector<double> light_area, light_power;
  Discrete<R> light_cdf;
  double all_power = 0;
  // acceleration (values only)
  std::vector<R> tv;                 // 9 per triangle (value positions)
  struct Node { R lo[3], hi[3]; int left, right, first, count; };
  std::vector<Node> nodes;
  std::vector<int> order;
};

// mesh.cc:27-67 triangle attributes.
template <class S>
inline void tri_attrs(Tri<S>& t) {
  V3<S> a = t.p2 - t.p1, b = t.p0 - t.p2, c = t.p1 - t.p0;
  t.n = normalize(cross(c, b));
  using R = typename Traits<S>::R;
  // uv are the float inputs stored as doubles; differences are formed in S.
  S du1y = S(R(t.uv[3])) - S(R(t.uv[1]));
  S du2y = S(R(t.uv[5])) - S(R(t.uv[1]));
  t.t = normalize(du2y * c + du1y * b);
  S la = norm(a), lb = norm(b), lc = norm(c);
  S p = (la + lb + lc) / S(2);
  t.area = safe_sqrt(p * (p - la) * (p - lb) * (p - lc));
}

// mesh.cc:97-204 build_edges, in (min, max) vertex-id order per mesh.
template <class S>
inline void build_edges(Scene<S>& sc, int vbase, const int* F, int nF) {
  struct Info { int l, kl, r, kr, cnt; };
  std::map<std::pair<int, int>, Info> m;
  auto add = [&](int i, int j, int k, int f) {
    auto key = std::make_pair(std::min(i, j), std::max(i, j));
    auto it = m.find(key);
    if (it == m.end()) m.emplace(key, Info{f, k, -1, -1, 1});
    else { it->second.r = f; it->second.kr = k; it->second.cnt++; }
  };
  for (int f = 0; f < nF; ++f) {
    int i = F[3 * f], j = F[3 * f + 1], k = F[3 * f + 2];
    add(i, j, k, f); add(j, k, i, f); add(k, i, j, f);
  }
  const S eps = S(1e-5);
  for (auto& kv : m) {
    const Info& in = kv.second;
    int r = in.r == -1 ? in.l : in.r;
    int kr = in.r == -1 ? in.kl : in.kr;
    Edge<S> e;
    e.v0 = vbase + kv.first.first; e.v1 = vbase + kv.first.second;
    e.p0 = sc.verts[e.v0]; e.p1 = sc.verts[e.v1];
    V3<S> p2l = sc.verts[vbase + in.kl], p2r = sc.verts[vbase + kr];
    V3<S> nl = normalize(cross(e.p1 - e.p0, p2l - e.p1));
    V3<S> nr = normalize(cross(p2r - e.p1, e.p1 - e.p0));
    bool shared = in.l != r;
    V3<S> out = shared ? normalize(nl + nr) : normalize(cross(e.p1 - e.p0, nl));
    V3<S> mid_p = e.p0 + e.p1, mid_c = p2l + p2r;
    V3<S> cp = normalize(mid_p - mid_c);
    if (val(dot(cp, out)) < 0 && shared && val(norm(nl - nr)) > val(eps)) { nl = -nl; nr = -nr; out = -out; }
    e.nl = nl; e.nr = nr; e.out = out;
    e.len = norm(e.p0 - e.p1);
    sc.edges.push_back(e);
  }
}

// Top-down median BVH over the value positions (the oracle's own, independent of the GPU LBVH).
template <class S>
inline void build_bvh(Scene<S>& sc) {
  using R = typename Traits<S>::R;
  int n = (int)sc.tris.size();
  sc.tv.resize(9 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    const auto& t = sc.tris[i];
    const V3<S>* p[3] = {&t.p0, &t.p1, &t.p2};
    for (int v = 0; v < 3; ++v) for (int k = 0; k < 3; ++k) sc.tv[9 * i + 3 * v + k] = R(val((*p[v])[k]));
  }
  sc.order.resize(n);
  for (int i = 0; i < n; ++i) sc.order[i] = i;
  sc.nodes.clear();
  std::vector<double> cen(3 * (size_t)n);
  for (int i = 0; i < n; ++i) for (int k = 0; k < 3; ++k)
    cen[3 * i + k] = (double(sc.tv[9 * i + k]) + sc.tv[9 * i + 3 + k] + sc.tv[9 * i + 6 + k]) / 3.0;
  struct Job { int node, lo, hi; };
  sc.nodes.push_back({});
  std::vector<Job> st{{0, 0, n}};
  while (!st.empty()) {
    Job j = st.back(); st.pop_back();
    auto& nd = sc.nodes[j.node];
    R lo[3] = {std::numeric_limits<R>::infinity(), std::numeric_limits<R>::infinity(), std::numeric_limits<R>::infinity()};
    R hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (int i = j.lo; i < j.hi; ++i) {
      int t = sc.order[i];
      for (int v = 0; v < 3; ++v) for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], sc.tv[9 * t + 3 * v + k]);
        hi[k] = std::max(hi[k], sc.tv[9 * t + 3 * v + k]);
      }
    }
    for (int k = 0; k < 3; ++k) { nd.lo[k] = lo[k]; nd.hi[k] = hi[k]; }
    if (j.hi - j.lo <= 4) { nd.left = nd.right = -1; nd.first = j.lo; nd.count = j.hi - j.lo; continue; }
    int ax = 0;
    double ext[3];
    for (int k = 0; k < 3; ++k) ext[k] = double(hi[k]) - double(lo[k]);
    if (ext[1] > ext[ax]) ax = 1;
    if (ext[2] > ext[ax]) ax = 2;
    int mid = (j.lo + j.hi) / 2;
    std::nth_element(sc.order.begin() + j.lo, sc.order.begin() + mid, sc.order.begin() + j.hi,
                     [&](int a, int b) { return cen[3 * a + ax] < cen[3 * b + ax] || (cen[3 * a + ax] == cen[3 * b + ax] && a < b); });
    int l = (int)sc.nodes.size();
    sc.nodes.push_back({});
    sc.nodes.push_back({});
    sc.nodes[j.node].left = l; sc.nodes[j.node].right = l + 1; sc.nodes[j.node].count = 0;
    st.push_back({l, j.lo, mid});
    st.push_back({l + 1, mid, j.hi});
  }
}

template <class R> struct Hit { int tri = -1; R b1 = 0, b2 = 0, t = 0; };

// Closest hit, t in (1e-3, tmax], ties -> smaller triangle id. Brute force or BVH.
template <class S>
inline Hit<typename Traits<S>::R> intersect(const Scene<S>& sc, const typename Traits<S>::R o[3],
                                            const typename Traits<S>::R d[3], bool use_bvh = true,
                                            typename Traits<S>::R tmax = std::numeric_limits<typename Traits<S>::R>::infinity()) {
  using R = typename Traits<S>::R;
  const R tmin = R(1e-3);
  Hit<R> h;
  h.t = tmax;
  RayPre<R> rp = ray_pre(o, d);
  auto test = [&](int t) {
    R tt, b1, b2;
    if (tri_test(rp, &sc.tv[9 * t], &sc.tv[9 * t + 3], &sc.tv[9 * t + 6], tmin, h.t, tt, b1, b2)) {
      if (tt < h.t || h.tri < 0 || t < h.tri) { h.t = tt; h.tri = t; h.b1 = b1; h.b2 = b2; }
    }
  };
  int n = (int)sc.tris.size();
  if (!use_bvh || sc.nodes.empty()) {
    for (int t = 0; t < n; ++t) test(t);
    return h;
  }
  double inv[3];
  for (int k = 0; k < 3; ++k) inv[k] = 1.0 / (std::fabs(double(d[k])) > 1e-30 ? double(d[k]) : (d[k] < 0 ? -1e-30 : 1e-30));
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const auto& nd = sc.nodes[stack[--sp]];
    double tn = double(tmin), tf = double(h.t) * (1 + 1e-5) + 1e-9;
    bool miss = false;
    for (int k = 0; k < 3 && !miss; ++k) {
      double lo = double(nd.lo[k]) - 1e-6 * (std::fabs(double(nd.lo[k])) + 1.0);
      double hi = double(nd.hi[k]) + 1e-6 * (std::fabs(double(nd.hi[k])) + 1.0);
      double t0 = (lo - double(o[k])) * inv[k], t1 = (hi - double(o[k])) * inv[k];
      if (t0 > t1) std::swap(t0, t1);
      tn = std::max(tn, t0); tf = std::min(tf, t1);
      if (tn > tf) miss = true;
    }
    if (miss) continue;
    if (nd.count > 0) {
      for (int i = nd.first; i < nd.first + nd.count; ++i) test(sc.order[i]);
    } else {
      stack[sp++] = nd.left;
      stack[sp++] = nd.right;
    }
  }
  return h;
}

// ------------------------------------------------------------------ scene construction
// scene.cc:3-104 (flatten objects then emitter meshes, light power CDF, edge CDF).
template <class S>
struct Seeds {
  // Optional tangent seeds for Dual scalars; each pointer is K doubles per scalar.
  const double* verts = nullptr;   // (V_total, 3, K)
  const double* tex = nullptr;     // concatenated textures (elements, K)
  const double* emit = nullptr;    // (n_lights, 3, K)
  const double* campos = nullptr;  // (n_cams, 3, K)
};

template <class S> inline S seeded(double v, const double* seed) { (void)seed; return S(v); }
template <int K> inline Dual<K> seeded_dual(double v, const double* seed) {
  Dual<K> r(v);
  if (seed) for (int i = 0; i < K; ++i) r.d[i] = seed[i];
  return r;
}
template <class S> struct Seeder { static S make(double v, const double*, int) { return S(typename Traits<S>::R(v)); } };
template <int K> struct Seeder<Dual<K>> { static Dual<K> make(double v, const double* s, int k) { return seeded_dual<K>(v, s ? s + (size_t)k * K : nullptr); } };

// emitter.cc:103-119 bounding-box mesh of the environment lights: vertex v has
// x = max if bit 2, y = max if bit 1, z = max if bit 0; faces and cube-map uvs (a 4 x 3
// cross layout) as the reference lists them.
static const int env_box_faces[36] = {
    0, 1, 2, 3, 2, 1, 4, 5, 6, 7, 6, 5, 0, 4, 1, 5, 1, 4,
    2, 6, 3, 7, 3, 6, 4, 0, 6, 2, 6, 0, 5, 1, 7, 3, 7, 1};
static const float env_box_uvs[28] = {0.25f, 0.f, 0.5f, 0.f, 0.f, 1.f / 3, 0.25f, 1.f / 3, 0.5f, 1.f / 3,
                                      0.75f, 1.f / 3, 1.f, 1.f / 3, 0.f, 2.f / 3, 0.25f, 2.f / 3, 0.5f, 2.f / 3,
                                      0.75f, 2.f / 3, 1.f, 2.f / 3, 0.25f, 1.f, 0.5f, 1.f};
static const int env_box_uv_indices[36] = {
    2, 3, 7, 8, 7, 3, 5, 4, 10, 9, 10, 4, 0, 1, 3, 4, 3, 1,
    12, 13, 8, 9, 8, 13, 5, 6, 10, 11, 10, 6, 4, 3, 9, 8, 9, 3};

template <class S>
inline Scene<S> build_scene(const OrcMesh* meshes, int nm, const OrcLight* lights, int nl, const Seeds<S>& seeds) {
  using R = typename Traits<S>::R;
  Scene<S> sc;
  sc.n_obj = nm + nl;
  int vglob = 0, texoff = 0, tex_elem = 0;
  auto add_mesh = [&](const float* V, int nV, const int* F, int nF, const float* uv, const int* uvi,
                      int light_id, const OrcTexture* tex, bool edges = true) {
    int obj = (int)sc.obj_light.size();
    sc.obj_light.push_back(light_id);
    sc.obj_vert_off.push_back(vglob);
    for (int v = 0; v < nV; ++v) {
      V3<S> p;
      for (int k = 0; k < 3; ++k) p[k] = Seeder<S>::make(V[3 * v + k], seeds.verts, 3 * (vglob + v) + k);
      sc.verts.push_back(p);
    }
    if (tex) {
      sc.obj_tex_kind.push_back(tex->kind);
      sc.obj_tex_h.push_back(tex->kind ? tex->h : 1);
      sc.obj_tex_w.push_back(tex->kind ? tex->w : 1);
      sc.obj_tex_off.push_back(texoff);
      int cnt = tex->kind ? tex->h * tex->w * 3 : 3;
      for (int e = 0; e < cnt; ++e) sc.tex.push_back(Seeder<S>::make(tex->data[tex->kind ? e : (tex->c == 1 ? 0 : e)], seeds.tex, tex_elem + e));
      texoff += cnt; tex_elem += cnt;
    } else {
      sc.obj_tex_kind.push_back(-1); sc.obj_tex_h.push_back(0); sc.obj_tex_w.push_back(0); sc.obj_tex_off.push_back(-1);
    }
    for (int f = 0; f < nF; ++f) {
      Tri<S> t;
      int i0 = F[3 * f], i1 = F[3 * f + 1], i2 = F[3 * f + 2];
      sc.faces.push_back({vglob + i0, vglob + i1, vglob + i2});
      t.p0 = sc.verts[vglob + i0]; t.p1 = sc.verts[vglob + i1]; t.p2 = sc.verts[vglob + i2];
      if (uv && uvi) {
        for (int c = 0; c < 3; ++c) { int u = uvi[3 * f + c]; t.uv[2 * c] = uv[2 * u]; t.uv[2 * c + 1] = uv[2 * u + 1]; }
      } else {
        t.uv[0] = 0; t.uv[1] = 0; t.uv[2] = 0; t.uv[3] = 1; t.uv[4] = 1; t.uv[5] = 0;
      }
      t.obj = obj;
      tri_attrs(t);
      sc.tris.push_back(t);
    }
    if (edges) build_edges(sc, vglob, F, nF);
    vglob += nV;
  };
  for (int m = 0; m < nm; ++m) {
    const auto& M = meshes[m];
    add_mesh(M.V, M.nV, M.F, M.nF, M.uv, M.uvi, -1, &M.color);
  }
  // roughness and normal maps of DiffuseBsdfMaterial meshes, after every color texture
  // (their derivative seeds follow the colors' in the same order)
  auto add_tex = [&](const OrcTexture& t, int ch) {
    typename Scene<S>::TexRef r;
    if (t.kind < 0 || !t.data) return r;
    r.kind = t.kind; r.h = t.kind ? t.h : 1; r.w = t.kind ? t.w : 1; r.c = ch; r.off = texoff;
    int cnt = r.h * r.w * ch;
    for (int e = 0; e < cnt; ++e) sc.tex.push_back(Seeder<S>::make(t.data[t.kind ? e : (t.c == 1 ? 0 : e % t.c)], seeds.tex, tex_elem + e));
    texoff += cnt; tex_elem += cnt;
    return r;
  };
  for (int m = 0; m < nm; ++m) {
    const auto& M = meshes[m];
    sc.obj_mat.push_back(M.mat);
    sc.obj_rough.push_back(M.mat == 1 ? add_tex(M.rough, 1) : typename Scene<S>::TexRef{});
    sc.obj_nrm.push_back(M.mat == 1 ? add_tex(M.normal, 3) : typename Scene<S>::TexRef{});
  }
  std::vector<double> powers;
  for (int l = 0; l < nl; ++l) {
    const auto& Lg = lights[l];
    V3<S> e;
    for (int k = 0; k < 3; ++k) e[k] = Seeder<S>::make(Lg.emit[k], seeds.emit, 3 * l + k);
    sc.emit.push_back(e);
    sc.light_kind.push_back(Lg.type);
    sc.light_tri0.push_back((int)sc.tris.size());
    if (Lg.type == 0) {
      sc.light_tex.push_back(typename Scene<S>::TexRef{});
      sc.light_ntri.push_back(Lg.nF);
      add_mesh(Lg.V, Lg.nV, Lg.F, Lg.nF, nullptr, nullptr, l, nullptr);
    } else {
      // emitter.cc:97-131 / 221-244 set_aabb: the bounding box as a 12-triangle mesh
      // (cube-map uvs for EnvLight), outside the edge list (scene.cc:59-62)
      float bv[24];
      for (int v = 0; v < 8; ++v) {
        bv[3 * v] = (v & 4) ? Lg.box_max[0] : Lg.box_min[0];
        bv[3 * v + 1] = (v & 2) ? Lg.box_max[1] : Lg.box_min[1];
        bv[3 * v + 2] = (v & 1) ? Lg.box_max[2] : Lg.box_min[2];
      }
      if (Lg.type == 1) {
        sc.light_tex.push_back(add_tex(Lg.cube_map, 3));
      } else {
        typename Scene<S>::TexRef r;
        r.kind = 0; r.h = 1; r.w = 1; r.c = 27; r.off = texoff;
        for (int k = 0; k < 27; ++k) sc.tex.push_back(Seeder<S>::make(Lg.sh9[k], seeds.tex, tex_elem + k));
        texoff += 27; tex_elem += 27;
        sc.light_tex.push_back(r);
      }
      sc.light_ntri.push_back(12);
      add_mesh(bv, 8, env_box_faces, 12, Lg.type == 1 ? env_box_uvs : nullptr,
               Lg.type == 1 ? env_box_uv_indices : nullptr, l, nullptr, false);
    }
    sc.obj_mat.push_back(0);
    sc.obj_rough.push_back(typename Scene<S>::TexRef{});
    sc.obj_nrm.push_back(typename Scene<S>::TexRef{});
    std::vector<double> areas;
    double tot = 0;
    for (int f = 0; f < sc.light_ntri[l]; ++f) { double a = double(R(val(sc.tris[sc.light_tri0[l] + f].area))); areas.push_back(a); tot += a; }
    Discrete<R> d; d.build(areas);
    sc.light_tri_cdf.push_back(d);
    // emitter.cc:10-11 power = 2*pi*luminance(emit)*area; environment lights 4*pi
    // (emitter.cc:130, 243)
    double lum = double(Lg.emit[0]) * 0.2126 + double(Lg.emit[1]) * 0.7152 + double(Lg.emit[2]) * 0.0722;
    double pw = Lg.type == 0 ? 2 * M_PI * lum * tot : 4 * M_PI;
    sc.light_area.push_back(tot);
    sc.light_power.push_back(pw);
    powers.push_back(pw);
  }
  if (nl > 0) sc.light_cdf.build(powers);
  sc.all_power = 0;
  for (double p : powers) sc.all_power += p;
  std::vector<double> lens;
  for (auto& e : sc.edges) lens.push_back(double(R(val(e.len))));
  if (!lens.empty()) sc.edge_cdf.build(lens);
  build_bvh(sc);
  return sc;
}

// ------------------------------------------------------------------ intersection record
template <class S> struct Its {
  bool valid = false, is_front = false, is_light = false;
  V3<S> p, n, t, wi;
  S sqd = S(0), jac = S(1), area = S(0);
  double u = 0, v = 0;    // texture coordinates (no derivatives)
  double b1 = 0, b2 = 0;  // barycentrics of the hit
  int tri = -1, obj = -1, light = -1;
};

// scene.cc:106-161 Scene::hit (OptiX barycentrics are not differentiated).
template <class S, bool AD>
inline Its<S> scene_hit(const Scene<S>& sc, const V3<S>& o, const V3<S>& d, bool valid,
                        typename Traits<S>::R tmax = std::numeric_limits<typename Traits<S>::R>::infinity()) {
  using R = typename Traits<S>::R;
  Its<S> its;
  if (!valid) return its;
  R oo[3] = {R(val(o.x)), R(val(o.y)), R(val(o.z))};
  R dd[3] = {R(val(d.x)), R(val(d.y)), R(val(d.z))};
  Hit<R> h = intersect(sc, oo, dd, true, tmax);
  if (h.tri < 0) return its;
  const Tri<S>& tr = sc.tris[h.tri];
  its.valid = true;
  its.tri = h.tri;
  its.b1 = double(h.b1);
  its.b2 = double(h.b2);
  S bu = S(h.b1), bv = S(h.b2);
  its.p = tr.p0 + bu * (tr.p1 - tr.p0) + bv * (tr.p2 - tr.p0);
  R u0 = R(tr.uv[0]), v0 = R(tr.uv[1]);
  its.u = double(u0 + R(h.b1) * (R(tr.uv[2]) - u0) + R(h.b2) * (R(tr.uv[4]) - u0));
  its.v = double(v0 + R(h.b1) * (R(tr.uv[3]) - v0) + R(h.b2) * (R(tr.uv[5]) - v0));
  V3<S> wun = its.p - o;
  its.wi = -normalize(wun);
  its.sqd = sqnorm(wun);
  its.is_front = val(dot(its.wi, tr.n)) > 0;
  its.n = its.is_front ? tr.n : -tr.n;
  its.t = its.is_front ? tr.t : -tr.t;
  its.obj = tr.obj;
  its.light = sc.obj_light[tr.obj];
  its.is_light = its.light >= 0;
  its.area = tr.area;
  its.jac = AD ? tr.area / detach(tr.area) : S(1);
  return its;
}

// texture.h:65-74 UVTexture::at_nearest (rows flipped by torch_psdr.py:250), :24-31 constant.
template <class S>
inline V3<S> tex_at(const Scene<S>& sc, int obj, double u, double v) {
  using R = typename Traits<S>::R;
  int kind = sc.obj_tex_kind[obj];
  int off = sc.obj_tex_off[obj];
  if (kind == 0) return V3<S>(sc.tex[off], sc.tex[off + 1], sc.tex[off + 2]);
  if (kind < 0) return V3<S>();
  int H = sc.obj_tex_h[obj], W = sc.obj_tex_w[obj];
  R uu = R(u) * R(W) - R(0.5), vv = R(v) * R(H) - R(0.5);
  R ru = std::nearbyint(uu), rv = std::nearbyint(vv);
  ru = std::min(std::max(ru, R(-1)), R(W)); rv = std::min(std::max(rv, R(-1)), R(H));
  int u0 = std::min(std::max((int)ru, 0), W - 1);
  int v0 = std::min(std::max((int)rv, 0), H - 1);
  int row = H - 1 - v0;
  int e = off + 3 * (row * W + u0);
  return V3<S>(sc.tex[e], sc.tex[e + 1], sc.tex[e + 2]);
}
inline int tex_index(int kind, int H, int W, double u, double v, bool f32) {
  if (kind == 0) return 0;
  double uu, vv;
  if (f32) { float a = float(u) * float(W) - 0.5f, b = float(v) * float(H) - 0.5f; uu = std::nearbyint(a); vv = std::nearbyint(b); }
  else { uu = std::nearbyint(u * W - 0.5); vv = std::nearbyint(v * H - 0.5); }
  int u0 = std::min(std::max((int)std::max(std::min(uu, double(W)), -1.0), 0), W - 1);
  int v0 = std::min(std::max((int)std::max(std::min(vv, double(H)), -1.0), 0), H - 1);
  return 3 * ((H - 1 - v0) * W + u0);
}

template <class S> inline S inv_pi() { return S(typename Traits<S>::R(1.0 / M_PI)); }

// diffuse_material.cc:3-30 cosine-weighted sample in the (T, N x T, N) frame.
template <class S>
inline V3<S> diffuse_sample_dir(const Its<S>& its, typename Traits<S>::R ru, typename Traits<S>::R rv,
                                typename Traits<S>::R& cos_theta) {
  using R = typename Traits<S>::R;
  V3<S> B = cross(its.n, its.t);
  R ct = ru > 0 ? std::sqrt(ru) : R(0);
  R st = (R(1) - ru) > 0 ? std::sqrt(R(1) - ru) : R(0);
  R phi = rv * R(2 * M_PI);
  R sp = std::sin(phi), cp = std::cos(phi);
  R uu = cp * st, vv = sp * st;
  cos_theta = ct;
  return normalize(its.t * S(uu) + B * S(vv) + its.n * S(ct));
}

// texture.h:24-31, 65-74: nearest texel of a roughness / normal texture (c channels).
template <class S>
inline V3<S> tex_fetch(const Scene<S>& sc, const typename Scene<S>::TexRef& t, double u, double v) {
  if (t.kind < 0) return V3<S>();
  int e = t.off;
  if (t.kind == 1) e += tex_index(1, t.h, t.w, u, v, std::is_same<typename Traits<S>::R, float>::value) / 3 * t.c;
  if (t.c == 1) return V3<S>(sc.tex[e], S(0), S(0));
  return V3<S>(sc.tex[e], sc.tex[e + 1], sc.tex[e + 2]);
}

// diffuse_bsdf.cc:10-20 shading normal: the normal map in the (T, Ng x T, Ng) frame,
// or the (flipped) geometric normal.
template <class S>
inline V3<S> shading_normal(const Scene<S>& sc, const Its<S>& its) {
  if (sc.obj_mat[its.obj] != 1 || sc.obj_nrm[its.obj].kind < 0) return its.n;
  V3<S> m = tex_fetch(sc, sc.obj_nrm[its.obj], its.u, its.v);
  V3<S> B = cross(its.n, its.t);
  return normalize(its.t * (m.x * S(2) - S(1)) + B * (m.y * S(2) - S(1)) + its.n * (m.z * S(2) - S(1)));
}

// BSDF value for outgoing direction L (the incoming one is its.wi): DiffuseMaterial
// color / pi (diffuse_material.cc:33-37); DiffuseBsdfMaterial's rough-diffuse model
// (diffuse_bsdf.cc:56-88) with its sign rule on t.
template <class S>
inline V3<S> bsdf_eval(const Scene<S>& sc, const Its<S>& its, const V3<S>& L) {
  using R = typename Traits<S>::R;
  V3<S> color = tex_at(sc, its.obj, its.u, its.v);
  if (sc.obj_mat[its.obj] != 1) return color * inv_pi<S>();
  V3<S> N = shading_normal(sc, its);
  S sigma = tex_fetch(sc, sc.obj_rough[its.obj], its.u, its.v).x;
  S a = S(R(1)) / (S(R(M_PI)) + S(R((3 * M_PI - 4) / 6)) * sigma);
  S b = sigma * a;
  S nl = dot(N, L), nv = dot(N, its.wi);
  if (val(nl) < 0) nl = S(0);
  if (val(nv) < 0) nv = S(0);
  S t = dot(its.wi, L) - nl * nv;
  if (val(t) > 0) t = (val(nl) >= val(nv) ? nl : nv) + S(R(1e-5));
  return color * (a + b * t);
}

// Material sampling (diffuse_material.cc:3-30, diffuse_bsdf.cc:3-53): cosine-weighted
// around the shading normal in the (T, Ng x T, N) frame; pdf = cos_theta / pi.
template <class S>
inline V3<S> material_sample_dir(const Scene<S>& sc, const Its<S>& its, typename Traits<S>::R ru,
                                 typename Traits<S>::R rv, typename Traits<S>::R& cos_theta) {
  using R = typename Traits<S>::R;
  V3<S> N = shading_normal(sc, its);
  V3<S> B = cross(its.n, its.t);
  R ct = ru > 0 ? std::sqrt(ru) : R(0);
  R st = (R(1) - ru) > 0 ? std::sqrt(R(1) - ru) : R(0);
  R phi = rv * R(2 * M_PI);
  R sp = std::sin(phi), cp = std::cos(phi);
  cos_theta = ct;
  return normalize(its.t * S(cp * st) + B * S(sp * st) + N * S(ct));
}

// Radiance of a light hit: AreaLight's constant (emitter.cc:17-28), EnvLight's cube map
// at the box uv (emitter.cc:134-141; diffuse_material.h:53-58), SH9Light's second-order
// real spherical harmonics at the hit's incoming direction (emitter.cc:246-283).
template <class S>
inline V3<S> light_emit(const Scene<S>& sc, const Its<S>& its) {
  using R = typename Traits<S>::R;
  const int l = its.light;
  const int kind = sc.light_kind[l];
  if (kind == 0) return sc.emit[l];
  if (kind == 1) return tex_fetch(sc, sc.light_tex[l], its.u, its.v);
  const S x = its.wi.x, y = its.wi.y, z = its.wi.z;
  const R c0 = R(std::sqrt(1.0 / (4 * M_PI))), c1 = R(std::sqrt(0.75 / M_PI)), c2 = R(std::sqrt(3.75 / M_PI));
  const R c3 = R(std::sqrt(5.0 / 16.0 / M_PI)), c4 = R(std::sqrt(15.0 / 16.0 / M_PI));
  const S Y[9] = {S(c0), S(c1) * y, S(c1) * z, S(c1) * x, S(c2) * (x * y), S(c2) * (y * z),
                  S(c3) * (S(R(2)) * (z * z) - x * x - y * y), S(c2) * (z * x), S(c4) * (x * x - y * y)};
  const int off = sc.light_tex[l].off;
  V3<S> e;
  for (int k = 0; k < 9; ++k)
    for (int ch = 0; ch < 3; ++ch) e[ch] = e[ch] + sc.tex[off + 3 * k + ch] * Y[k];
  return e;
}

// path_integrator.cc:3-9 (power heuristic, n1/n2 sample counts)
template <class R> inline R mis_w(R w1, R w2, R n1, R n2) {
  R a = (n1 * w1) * (n1 * w1), b = (n2 * w2) * (n2 * w2);
  return a / (a + b);
}

// emitter.cc:29-59 AreaLight::sample_light_point
template <class S>
inline V3<S> light_sample_point(const Scene<S>& sc, int l, typename Traits<S>::R rx, typename Traits<S>::R ry,
                                typename Traits<S>::R& pdf) {
  using R = typename Traits<S>::R;
  R pdf_tri;
  int idx = sc.light_tri_cdf[l].sample_reuse(rx, pdf_tri);
  const Tri<S>& t = sc.tris[sc.light_tri0[l] + idx];
  R sv = ry > 0 ? std::sqrt(ry) : R(0);
  R u = rx * sv, v = R(1) - sv;
  pdf = R(1) / R(sc.light_area[l]);
  return t.p0 + (t.p1 - t.p0) * S(u) + (t.p2 - t.p0) * S(v);
}

// ------------------------------------------------------------------ trace2light
// path_integrator.cc:80-186. AD=true reproduces renderD's tape semantics (detached
// pdfs and MIS weights, jacobi = area/detach(area)); AD=false is the plain render.
// geo_dirs (the unbiased estimator) forms the G terms of BSDF-sampled segments from
// the segment's end points instead of the sampled direction (same value, the
// derivative of the material-form path integral).
template <class S, bool AD>
inline V3<S> trace2light(const Scene<S>& sc, Pcg32& rng, Its<S> its, bool valid, int nL, int nB, int D, bool light_vis,
                         bool geo_dirs = false) {
  using R = typename Traits<S>::R;
  V3<S> T(S(1), S(1), S(1)), L;
  valid = valid && its.valid;
  const R eps = R(1e-5);
  for (int depth = 0; depth < D; ++depth) {
    bool hit_light = valid && its.is_light;
    if (light_vis && depth == 0 && hit_light) L = L + mul(T, light_emit(sc, its));
    valid = valid && !hit_light;
    for (int i = 0; i < nL; ++i) {
      R rx = rng.next_float(valid), ry = rng.next_float(valid);
      if (!valid) continue;
      R pch = R(1);
      int l = 0;
      if ((int)sc.emit.size() > 0) l = sc.light_cdf.sample_reuse(rx, pch);
      R pl;
      V3<S> y = light_sample_point(sc, l, rx, ry, pl);
      R pdf_light = pl * pch;
      V3<S> dir = normalize(y - its.p);
      Its<S> il = scene_hit<S, AD>(sc, its.p, dir, true);
      bool is_hit = il.valid && il.is_light && val(sqnorm(il.p - y)) < double(eps);
      if (!is_hit) continue;
      V3<S> emit = light_emit(sc, il);
      V3<S> bsdf = bsdf_eval(sc, its, dir);
      S tmp = dot(il.n, -dir) / il.sqd;
      S G = dot(its.n, dir) * tmp;
      V3<S> value = mul(emit, bsdf) * (G * il.jac / S(pdf_light));
      R weight = R(1) / R(nL);
      if (nB > 0) {
        R pdf_bsdf = R(val(dot(its.n, dir) * inv_pi<S>() * tmp));
        weight *= mis_w<R>(pdf_light, pdf_bsdf, R(nL), R(nB));
      }
      L = L + mul(T, value) * S(weight);
    }
    for (int i = 0; i < nB; ++i) {
      R rx = rng.next_float(valid), ry = rng.next_float(valid);
      if (!valid) continue;
      R ct;
      V3<S> wo = material_sample_dir(sc, its, rx, ry, ct);
      Its<S> il = scene_hit<S, AD>(sc, its.p, wo, true);
      bool is_hit = il.valid && il.is_light;
      if (!is_hit) continue;
      V3<S> emit = light_emit(sc, il);
      S tmp = dot(il.n, -wo) / il.sqd;
      S G = dot(its.n, wo) * tmp;
      V3<S> Lb = wo;
      if (geo_dirs) {
        const V3<S> wg = normalize(il.p - its.p);
        G = dot(its.n, wg) * (dot(il.n, -wg) / il.sqd);
        Lb = wg;
      }
      V3<S> bsdf = bsdf_eval(sc, its, Lb);
      R pdf_bsdf = R(ct) * R(1.0 / M_PI) * R(val(tmp));
      V3<S> value = mul(emit, bsdf) * (G * il.jac / S(pdf_bsdf));
      R weight = R(1) / R(nB);
      if (nL > 0) {
        R pch = R(sc.light_power[il.light] / sc.all_power);
        R pdf_light = pch * (R(1) / R(sc.light_area[il.light]));
        weight *= mis_w<R>(pdf_bsdf, pdf_light, R(nB), R(nL));
      }
      L = L + mul(T, value) * S(weight);
    }
    // indirect (always drawn; the ray of the final depth is never used)
    R rx = rng.next_float(valid), ry = rng.next_float(valid);
    if (depth + 1 == D) break;
    if (!valid) break;
    R ct;
    V3<S> wo = material_sample_dir(sc, its, rx, ry, ct);
    Its<S> nx = scene_hit<S, AD>(sc, its.p, wo, true);
    valid = valid && nx.valid;
    if (!valid) break;
    S tmp = dot(nx.n, -wo) / nx.sqd;
    S G = dot(its.n, wo) * tmp;
    V3<S> Lb = wo;
    if (geo_dirs) {
      const V3<S> wg = normalize(nx.p - its.p);
      G = dot(its.n, wg) * (dot(nx.n, -wg) / nx.sqd);
      Lb = wg;
    }
    V3<S> bsdf = bsdf_eval(sc, its, Lb);
    R pdf = R(ct) * R(1.0 / M_PI) * R(val(tmp));
    T = mul(T, bsdf) * (nx.jac * G / S(pdf));
    its = nx;
  }
  if (!finite3(L)) L = V3<S>();
  return L;
}

}  // namespace orc
