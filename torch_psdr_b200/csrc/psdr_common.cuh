// psdr_common.cuh -- device-side building blocks shared by every kernel file:
// vector math, the PCG32/TEA sampler streams, scene records in HBM, the watertight
// ray/triangle test and the LBVH traversal.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define PSDR_HD __host__ __device__ __forceinline__
#define PSDR_D __device__ __forceinline__

namespace psdr {

// ------------------------------------------------------------------ float3 math
PSDR_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
PSDR_HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
PSDR_HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
PSDR_HD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
PSDR_HD float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
PSDR_HD float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
PSDR_HD float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
PSDR_HD float3 mul(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
PSDR_HD float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
PSDR_HD float3& operator-=(float3& a, float3 b) { a = a - b; return a; }
PSDR_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PSDR_HD float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PSDR_HD float sqnorm(float3 a) { return dot(a, a); }
PSDR_HD float norm(float3 a) { return sqrtf(sqnorm(a)); }
PSDR_HD float3 normalize(float3 a) { return a * (1.0f / sqrtf(sqnorm(a))); }
PSDR_HD float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }
PSDR_HD float sel3(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
PSDR_HD float comp(float3 v, int k) { return sel3(v, k); }
PSDR_HD bool finite3(float3 v) { return isfinite(sqnorm(v)); }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float k2Pi = 6.28318530717958647692f;
constexpr float kEps = 1e-5f;       // types.h:114 REAL_EPS
constexpr float kTmin = 1e-3f;      // device_programs.cu:8 tmin of every trace
constexpr int kEdgeNonManifold = -2;  // DevScene::edge_f of an edge with more than two faces

// ------------------------------------------------------------------ PCG32 + TEA
// One PCG32 stream per sample index (sampler.h:8-84), seeded through 4-round TEA.
constexpr uint64_t kPcgState = 0x853c49e6748fea9bULL;
constexpr uint64_t kPcgMult = 0x5851f42d4c957f2dULL;

PSDR_HD uint64_t tea64(uint32_t v0, uint32_t v1) {
  uint32_t sum = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    sum += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return (uint64_t)v0 + ((uint64_t)v1 << 32);
}

struct Rng {
  uint64_t state, inc;
  PSDR_HD uint32_t next(bool advance) {
    uint64_t old = state;
    if (advance) state = old * kPcgMult + inc;
    uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
    uint32_t rot = (uint32_t)(old >> 59);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  PSDR_HD float next_float(bool advance = true) {
    uint32_t bits = (next(advance) >> 9) | 0x3f800000u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(bits) - 1.0f;
#else
    float f;
    __builtin_memcpy(&f, &bits, 4);
    return f - 1.0f;
#endif
  }
};

// sampler.h:11-17; `seed` != 0 shifts the stream index (an extension: 0 reproduces
// the reference's streams).
PSDR_HD Rng make_rng(uint64_t i) {
  uint32_t a = (uint32_t)(i + kPcgState), b = (uint32_t)i;
  uint64_t initstate = tea64(a, b), initseq = tea64(b, a);
  Rng r;
  r.state = 0;
  r.inc = (initseq << 1) | 1u;
  r.next(true);
  r.state += initstate;
  r.next(true);
  return r;
}

// ------------------------------------------------------------------ gradient accumulators
// Exact, order-independent gradient sum: a fixed-point value in two int64 limbs,
// value = hi 2^-20 + lo 2^-52. A contribution v adds sign(v) floor(|v| 2^20) to hi and
// sign(v) round(frac(|v| 2^20) 2^32) to lo with integer atomics (fire-and-forget
// reductions). Integer additions commute, so the sum does not depend on the order in
// which threads reach it: backward passes are bitwise reproducible for any tile size and
// scheduling. Each contribution is rounded once, to 2^-52 (2.2e-16); the only other
// rounding is the final conversion. Limits: a contribution's magnitude saturates at 2^42,
// the hi limb holds totals below 2^43, the lo limb absorbs 2^31 contributions per entry;
// non-finite contributions are dropped.
struct GradAcc {
  long long hi, lo;
};
PSDR_D void acc_add(GradAcc* a, float v) {
  if (!(v != 0.f) || !isfinite(v)) return;
  const double q = fmin(fabs((double)v) * 1048576.0, 4398046511104.0 * 1048576.0);  // |v| 2^20, at most 2^62
  const double fh = floor(q);
  const long long dh = (long long)fh;
  const long long dl = __double2ll_rn((q - fh) * 4294967296.0);  // in [0, 2^32]
  const bool neg = v < 0.f;
  if (dh) atomicAdd(reinterpret_cast<unsigned long long*>(&a->hi), (unsigned long long)(neg ? -dh : dh));
  if (dl) atomicAdd(reinterpret_cast<unsigned long long*>(&a->lo), (unsigned long long)(neg ? -dl : dl));
}
PSDR_HD double acc_value(long long hi, long long lo) {
  return (double)hi * 9.5367431640625e-07 + (double)lo * 2.220446049250313e-16;  // 2^-20, 2^-52
}

// ------------------------------------------------------------------ scene records
struct DevTex {
  int kind;  // -1 none, 0 constant, 1 uv
  int ch;
  int h, w;
  const float* data;
  GradAcc* grad;  // accumulator with the same layout, or null
};
struct DevObj {
  int mat;
  int light;  // light index or -1
  DevTex color, rough, normal;
};
struct DevLight {
  int tri0, ntri;
  float emit[3];
  float area, inv_area, power;
  GradAcc* grad_emit;  // 3 accumulators or null
  int kind;           // PSDR_LIGHT_AREA, _ENV (cube map in tex), _SH9 (coefficients in sh)
  DevTex tex;         // ENV cube map (tex.grad: its accumulator or null)
  float sh[27];       // SH9 (9,3) coefficients
  GradAcc* grad_sh;   // SH9: 27 accumulators or null
};

// Per-triangle shading record, 6 x float4 (96 B) in original triangle order:
//  [0] p0.xyz, area   [1] p1.xyz, obj(bits)   [2] p2.xyz, uv0.x
//  [3] n.xyz, uv0.y   [4] t.xyz, uv1.x        [5] uv1.y, uv2.x, uv2.y, 0
// BVH node (4-wide, child boxes stored in the parent), 7 x float4 (112 B):
//  [0] lo.x of children 0..3 [1] hi.x [2] lo.y [3] hi.y [4] lo.z [5] hi.z [6] links (int)
// link >= 0: internal node; link < 0: leaf ~((first << 3) | (count-1)); 0x7fffffff: empty.
// Leaf triangles, 3 x float4 (48 B) in BVH order: p0.xyz + id(bits), p1.xyz, p2.xyz.
struct DevScene {
  int ntri, nvert, nobj, nlight;
  const float4* tri;
  const int4* tri_v;       // global vertex ids (x,y,z) + object (w)
  const float* verts;      // (nvert, 3)
  const DevObj* objs;
  const DevLight* lights;
  const float* light_pmf;
  const float* light_cmf;
  const float* ltri_pmf;   // per-light triangle CDFs, indexed by tri - ltri_base
  const float* ltri_cmf;
  int ltri_base;
  int edge_cap;
  const int* n_edges;      // device scalar
  const float4* edge;      // 4 x float4: (p0,len) (p1,out.x) (out.yz,nl.xy) (nl.z,nr)
  const int2* edge_v;
  // the edge's faces (global triangle ids; y = -1 for a boundary edge); kEdgeNonManifold in x
  // for an edge of more than two faces
  const int2* edge_f;
  const float* edge_pmf;
  const float* edge_cmf;
  int root;
  const float4* nodes;
  const float4* leaf;
  GradAcc* grad_verts;     // (nvert, 3) or null
  const unsigned char* vmask;  // (nvert): 1 = the caller wants this vertex's gradient
  int* err;                // device error word (bit 0: traversal stack overflow)
};

// ------------------------------------------------------------------ discrete sampling
// sampler.h:98-117 DiscreteSampler::sample_reuse with enoki::binary_search's fixed
// floor(log2(n-1))+1 bisection steps; rescales s in place.
PSDR_D int discrete_sample(const float* __restrict__ pmf, const float* __restrict__ cmf, int n, float& s,
                           float& pdf) {
  if (n <= 1) { pdf = 1.0f; return 0; }
  int start = 0, end = n - 1;
  int iters = 32 - __clz(end);
  for (int it = 0; it < iters; ++it) {
    int mid = (start + end) >> 1;
    if (__ldg(cmf + mid) < s) start = min(mid + 1, end);
    else end = mid;
  }
  pdf = __ldg(pmf + start);
  float prev = start > 0 ? __ldg(cmf + start - 1) : 0.0f;
  s = (s - prev) / pdf;
  return start;
}

// ------------------------------------------------------------------ watertight test
// Woop, Benthin & Wald (JCGT 2013). Every arithmetic step is an explicitly rounded
// IEEE operation so the device result is bit-identical to the float oracle.
struct RayPre {
  float3 o;
  int kx, ky, kz;
  float Sx, Sy, Sz;
};
PSDR_D RayPre ray_pre(float3 o, float3 d) {
  RayPre r;
  r.o = o;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  float dz = sel3(d, kz);
  if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
  r.kx = kx; r.ky = ky; r.kz = kz;
  r.Sx = __fdiv_rn(sel3(d, kx), dz);
  r.Sy = __fdiv_rn(sel3(d, ky), dz);
  r.Sz = __fdiv_rn(1.0f, dz);
  return r;
}
PSDR_D bool tri_test(const RayPre& r, float3 p0, float3 p1, float3 p2, float tmin, float tmax, float& t,
                     float& b1, float& b2) {
  float3 A = f3(__fsub_rn(p0.x, r.o.x), __fsub_rn(p0.y, r.o.y), __fsub_rn(p0.z, r.o.z));
  float3 B = f3(__fsub_rn(p1.x, r.o.x), __fsub_rn(p1.y, r.o.y), __fsub_rn(p1.z, r.o.z));
  float3 C = f3(__fsub_rn(p2.x, r.o.x), __fsub_rn(p2.y, r.o.y), __fsub_rn(p2.z, r.o.z));
  float Akz = sel3(A, r.kz), Bkz = sel3(B, r.kz), Ckz = sel3(C, r.kz);
  float Ax = __fsub_rn(sel3(A, r.kx), __fmul_rn(r.Sx, Akz)), Ay = __fsub_rn(sel3(A, r.ky), __fmul_rn(r.Sy, Akz));
  float Bx = __fsub_rn(sel3(B, r.kx), __fmul_rn(r.Sx, Bkz)), By = __fsub_rn(sel3(B, r.ky), __fmul_rn(r.Sy, Bkz));
  float Cx = __fsub_rn(sel3(C, r.kx), __fmul_rn(r.Sx, Ckz)), Cy = __fsub_rn(sel3(C, r.ky), __fmul_rn(r.Sy, Ckz));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
  float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  float tt = __fdiv_rn(T, det);
  if (!(tt > tmin && tt <= tmax)) return false;
  t = tt;
  b1 = __fdiv_rn(V, det);
  b2 = __fdiv_rn(W, det);
  return true;
}

// ------------------------------------------------------------------ explicitly rounded ops
// Used where a result must be bit-identical to the float oracle (the edge-sample rays
// of the primary boundary term graze silhouettes, so their construction is exact).
PSDR_D float3 sub_rn(float3 a, float3 b) { return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
PSDR_D float3 add_rn(float3 a, float3 b) { return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
PSDR_D float3 scale_rn(float3 a, float s) { return f3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
PSDR_D float dot_rn(float3 a, float3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
PSDR_D float norm_rn(float3 a) { return __fsqrt_rn(dot_rn(a, a)); }
PSDR_D float3 normalize_rn(float3 a) {
  const float n = norm_rn(a);
  return f3(__fdiv_rn(a.x, n), __fdiv_rn(a.y, n), __fdiv_rn(a.z, n));
}
PSDR_D float3 cross_rn(float3 a, float3 b) {
  return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
// row-major 4x4 affine/projective transform of a point, summed left to right
PSDR_D float3 xform_pos_rn(const float* m, float3 p) {
  auto row = [&](int r) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4 * r], p.x), __fmul_rn(m[4 * r + 1], p.y)),
                               __fmul_rn(m[4 * r + 2], p.z)), m[4 * r + 3]);
  };
  const float w = row(3);
  return f3(__fdiv_rn(row(0), w), __fdiv_rn(row(1), w), __fdiv_rn(row(2), w));
}

// ------------------------------------------------------------------ traversal
constexpr int kStack = 96;

struct HitRec {
  int tri;
  float b1, b2, t;
};

PSDR_D float safe_inv(float d) { return 1.0f / (fabsf(d) > 1e-30f ? d : copysignf(1e-30f, d)); }

// Closest hit in (tmin, tmax], ties broken by the smaller triangle id. Node boxes are
// expanded at build time and the cull bound is relaxed by 1e-5 relative so that no
// triangle the exact test would accept is culled (the KAT checks this against brute
// force on every ray).
//
// t_occ turns the query into an occlusion test below t_occ: the first triangle hit
// with t < t_occ ends the traversal and the ray reports a miss. Shadow rays use it
// with t_occ = |y - x| - 4e-3: any such hit lies >= 4e-3 from the light point y, so
// the reference's test |hit - y|^2 < 1e-5 (path_integrator.cc:114-116) fails for it
// exactly as it would for the true closest hit; hits at or beyond t_occ are resolved
// as closest hits.
PSDR_D void cswap(float& ka, int& va, float& kb, int& vb) {
  if (kb < ka) {
    const float tk = ka; ka = kb; kb = tk;
    const int tv = va; va = vb; vb = tv;
  }
}

// Not inlined: kernels that trace from several places (shadow-boundary samples trace
// up to seven times) then hold one copy of the traversal loop, which keeps their code
// inside the instruction cache.
static __device__ __noinline__ HitRec trace_closest(const DevScene& sc, float3 o, float3 d, float tmin, float tmax,
                                                    float t_occ = -INFINITY) {
  const RayPre rp = ray_pre(o, d);
  const float3 inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
  const float3 oi = f3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
  HitRec h;
  h.tri = -1; h.b1 = 0.f; h.b2 = 0.f; h.t = tmax;
  int stack[kStack];
  int sp = 0;
  int node = sc.root;
  if (sc.ntri <= 0) return h;
  while (true) {
    if (node >= 0) {
      // 4-wide node: six float4 of child bounds (SoA) + the four child links
      const float4* nd = sc.nodes + 7 * (size_t)node;
      const float4 lx = __ldg(nd), hx = __ldg(nd + 1), ly = __ldg(nd + 2), hy = __ldg(nd + 3);
      const float4 lz = __ldg(nd + 4), hz = __ldg(nd + 5);
      const int4 e = __ldg(reinterpret_cast<const int4*>(nd + 6));
      const float cull = h.t * 1.00001f + 1e-12f;
      auto slab = [&](float l_x, float h_x, float l_y, float h_y, float l_z, float h_z, int c) {
        const float ax = fmaf(l_x, inv.x, -oi.x), bx = fmaf(h_x, inv.x, -oi.x);
        const float ay = fmaf(l_y, inv.y, -oi.y), by = fmaf(h_y, inv.y, -oi.y);
        const float az = fmaf(l_z, inv.z, -oi.z), bz = fmaf(h_z, inv.z, -oi.z);
        const float tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), tmin));
        const float tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), cull));
        return (c != 0x7fffffff && tn <= tf * 1.0000005f) ? tn : INFINITY;
      };
      float k0 = slab(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, e.x);
      float k1 = slab(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, e.y);
      float k2 = slab(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, e.z);
      float k3 = slab(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, e.w);
      int c0 = e.x, c1 = e.y, c2 = e.z, c3 = e.w;
      // sort the four (distance, child) pairs, nearest first
      cswap(k0, c0, k1, c1);
      cswap(k2, c2, k3, c3);
      cswap(k0, c0, k2, c2);
      cswap(k1, c1, k3, c3);
      cswap(k1, c1, k2, c2);
      if (k0 == INFINITY) {
        if (sp == 0) break;
        node = stack[--sp];
        continue;
      }
      node = c0;
      if (sp + 3 <= kStack) {
        if (k3 != INFINITY) stack[sp++] = c3;
        if (k2 != INFINITY) stack[sp++] = c2;
        if (k1 != INFINITY) stack[sp++] = c1;
      } else {
        atomicOr(sc.err, 1);
      }
    } else {
      const int code = ~node;
      const int first = code >> 3, cnt = (code & 7) + 1;
      for (int k = 0; k < cnt; ++k) {
        const float4* lt = sc.leaf + 3 * (size_t)(first + k);
        const float4 q0 = __ldg(lt), q1 = __ldg(lt + 1), q2 = __ldg(lt + 2);
        float tt, b1, b2;
        if (tri_test(rp, xyz(q0), xyz(q1), xyz(q2), tmin, h.t, tt, b1, b2)) {
          if (tt < t_occ) {  // occluded before the target: report a miss
            h.tri = -1;
            h.t = tt;
            return h;
          }
          const int id = __float_as_int(q0.w);
          if (tt < h.t || h.tri < 0 || id < h.tri) { h.t = tt; h.tri = id; h.b1 = b1; h.b2 = b2; }
        }
      }
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
  return h;
}

// Resumable form of trace_closest for kernels that interleave many rays per thread
// (dynamic ray fetch): the same visiting order, tests and tie rule, so the same hit.
struct TraceState {
  RayPre rp;
  float3 inv, oi;
  float tmin, t_occ;
  HitRec h;
  int node, sp;
};

PSDR_D void trace_begin(TraceState& s, float3 o, float3 d, float tmin, float tmax, float t_occ, int root) {
  s.rp = ray_pre(o, d);
  s.inv = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
  s.oi = f3(o.x * s.inv.x, o.y * s.inv.y, o.z * s.inv.z);
  s.tmin = tmin;
  s.t_occ = t_occ;
  s.h.tri = -1; s.h.b1 = 0.f; s.h.b2 = 0.f; s.h.t = tmax;
  s.node = root;
  s.sp = 0;
}

// One node or leaf visit; returns true when the query is finished (s.h holds the hit).
// Stk stores the traversal stack: push(i, node), pop(i).
template <class Stk>
PSDR_D bool trace_step(const DevScene& sc, TraceState& s, Stk& stack) {
  if (s.node >= 0) {
    const float4* nd = sc.nodes + 7 * (size_t)s.node;
    const float4 lx = __ldg(nd), hx = __ldg(nd + 1), ly = __ldg(nd + 2), hy = __ldg(nd + 3);
    const float4 lz = __ldg(nd + 4), hz = __ldg(nd + 5);
    const int4 e = __ldg(reinterpret_cast<const int4*>(nd + 6));
    const float cull = s.h.t * 1.00001f + 1e-12f;
    const float3 inv = s.inv, oi = s.oi;
    const float tmin = s.tmin;
    auto slab = [&](float l_x, float h_x, float l_y, float h_y, float l_z, float h_z, int c) {
      const float ax = fmaf(l_x, inv.x, -oi.x), bx = fmaf(h_x, inv.x, -oi.x);
      const float ay = fmaf(l_y, inv.y, -oi.y), by = fmaf(h_y, inv.y, -oi.y);
      const float az = fmaf(l_z, inv.z, -oi.z), bz = fmaf(h_z, inv.z, -oi.z);
      const float tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), tmin));
      const float tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), cull));
      return (c != 0x7fffffff && tn <= tf * 1.0000005f) ? tn : INFINITY;
    };
    float k0 = slab(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, e.x);
    float k1 = slab(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, e.y);
    float k2 = slab(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, e.z);
    float k3 = slab(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, e.w);
    int c0 = e.x, c1 = e.y, c2 = e.z, c3 = e.w;
    cswap(k0, c0, k1, c1);
    cswap(k2, c2, k3, c3);
    cswap(k0, c0, k2, c2);
    cswap(k1, c1, k3, c3);
    cswap(k1, c1, k2, c2);
    if (k0 == INFINITY) {
      if (s.sp == 0) return true;
      s.node = stack.pop(--s.sp);
      return false;
    }
    s.node = c0;
    if (s.sp + 3 <= kStack) {
      if (k3 != INFINITY) stack.push(s.sp++, c3);
      if (k2 != INFINITY) stack.push(s.sp++, c2);
      if (k1 != INFINITY) stack.push(s.sp++, c1);
    } else {
      atomicOr(sc.err, 1);
    }
    return false;
  }
  const int code = ~s.node;
  const int first = code >> 3, cnt = (code & 7) + 1;
  for (int k = 0; k < cnt; ++k) {
    const float4* lt = sc.leaf + 3 * (size_t)(first + k);
    const float4 q0 = __ldg(lt), q1 = __ldg(lt + 1), q2 = __ldg(lt + 2);
    float tt, b1, b2;
    if (tri_test(s.rp, xyz(q0), xyz(q1), xyz(q2), s.tmin, s.h.t, tt, b1, b2)) {
      if (tt < s.t_occ) {
        s.h.tri = -1;
        s.h.t = tt;
        return true;
      }
      const int id = __float_as_int(q0.w);
      if (tt < s.h.t || s.h.tri < 0 || id < s.h.tri) { s.h.t = tt; s.h.tri = id; s.h.b1 = b1; s.h.b2 = b2; }
    }
  }
  if (s.sp == 0) return true;
  s.node = stack.pop(--s.sp);
  return false;
}


// ------------------------------------------------------------------ surface points
// scene.cc:106-161 Scene::hit: the point is re-formed from the triangle and the
// barycentrics; the normal and tangent face the incoming ray (is_front flip).
struct Surf {
  float3 p, n, t;
  float3 wi;     // unit direction toward the ray origin (the incoming direction V)
  float u, v;
  float area;
  float sqd;     // squared distance to the ray origin
  int tri, obj, light;
  bool valid, is_light, front;
};

PSDR_D Surf make_surf(const DevScene& sc, int tri, float b1, float b2, float3 org) {
  Surf s;
  s.valid = tri >= 0;
  s.tri = tri;
  s.is_light = false;
  s.light = -1;
  s.obj = -1;
  if (!s.valid) return s;
  const float4* r = sc.tri + 6 * (size_t)tri;
  const float4 q0 = __ldg(r), q1 = __ldg(r + 1), q2 = __ldg(r + 2), q3 = __ldg(r + 3), q4 = __ldg(r + 4),
               q5 = __ldg(r + 5);
  const float3 p0 = xyz(q0), p1 = xyz(q1), p2 = xyz(q2);
  s.p = p0 + b1 * (p1 - p0) + b2 * (p2 - p0);
  const float u0 = q2.w, v0 = q3.w, u1 = q4.w, v1 = q5.x, u2 = q5.y, v2 = q5.z;
  s.u = u0 + b1 * (u1 - u0) + b2 * (u2 - u0);
  s.v = v0 + b1 * (v1 - v0) + b2 * (v2 - v0);
  const float3 wun = s.p - org;
  s.sqd = sqnorm(wun);
  const float3 wi = -normalize(wun);
  s.wi = wi;
  const float3 n = xyz(q3), t = xyz(q4);
  s.front = dot(wi, n) > 0.0f;
  s.n = s.front ? n : -n;
  s.t = s.front ? t : -t;
  s.area = q0.w;
  s.obj = __float_as_int(q1.w);
  s.light = __ldg(&sc.objs[s.obj].light);
  s.is_light = s.light >= 0;
  return s;
}

// texture.h:65-74 UVTexture::at_nearest on the caller's (H,W,C) tensor with the row
// flip of torch_psdr.py:250; returns the element offset of the texel.
PSDR_D int texel_offset(const DevTex& tx, float u, float v) {
  if (tx.kind != 1) return 0;
  float uu = rintf(fminf(fmaxf(u * (float)tx.w - 0.5f, -1.0f), (float)tx.w));
  float vv = rintf(fminf(fmaxf(v * (float)tx.h - 0.5f, -1.0f), (float)tx.h));
  int u0 = min(max((int)uu, 0), tx.w - 1);
  int v0 = min(max((int)vv, 0), tx.h - 1);
  return tx.ch * ((tx.h - 1 - v0) * tx.w + u0);
}
PSDR_D float3 tex_rgb(const DevTex& tx, int off) {
  if (tx.kind < 0) return f3(0.f, 0.f, 0.f);
  const float* p = tx.data + off;
  if (tx.ch == 1) { float x = __ldg(p); return f3(x, x, x); }
  return f3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// diffuse_material.cc:3-30: cosine-weighted direction in the (T, N x T, N) frame.
PSDR_D float3 diffuse_dir(float3 N, float3 T, float ru, float rv, float& cos_theta, float& sin_theta,
                          float& sphi, float& cphi) {
  const float3 B = cross(N, T);
  cos_theta = ru > 0.f ? sqrtf(ru) : 0.f;
  sin_theta = (1.0f - ru) > 0.f ? sqrtf(1.0f - ru) : 0.f;
  sincosf(rv * k2Pi, &sphi, &cphi);
  const float uu = cphi * sin_theta, vv = sphi * sin_theta;
  return normalize(T * uu + B * vv + N * cos_theta);
}

// ------------------------------------------------------------------ materials
constexpr int kMatDiffuseBsdf = 1;                      // PSDR_MAT_DIFFUSE_BSDF
constexpr float kOrenC = (3.0f * kPi - 4.0f) / 6.0f;    // diffuse_bsdf.cc:36

// Shading normal (diffuse_bsdf.cc:10-20): DiffuseBsdfMaterial's normal map in the
// (T, Ng x T, Ng) frame, else the flipped geometric normal; m = 2 texel - 1.
PSDR_D float3 shading_normal(const DevObj& ob, const Surf& x, float3& m, bool& mapped) {
  mapped = ob.mat == kMatDiffuseBsdf && ob.normal.kind >= 0;
  m = f3(0.f, 0.f, 1.f);
  if (!mapped) return x.n;
  const float3 tx = tex_rgb(ob.normal, texel_offset(ob.normal, x.u, x.v));
  m = f3(tx.x * 2.f - 1.f, tx.y * 2.f - 1.f, tx.z * 2.f - 1.f);
  const float3 B = cross(x.n, x.t);
  return normalize(x.t * m.x + B * m.y + x.n * m.z);
}

// Roughness of a DiffuseBsdfMaterial point (1-channel texture).
PSDR_D float material_sigma(const DevObj& ob, const Surf& x) {
  if (ob.mat != kMatDiffuseBsdf) return 0.f;
  return tex_rgb(ob.rough, texel_offset(ob.rough, x.u, x.v)).x;
}

// BSDF value toward L for the incoming direction V: DiffuseMaterial color / pi
// (diffuse_material.cc:33-37); DiffuseBsdfMaterial's rough-diffuse model with its rule
// on t (diffuse_bsdf.cc:56-88).
PSDR_D float3 bsdf_value(const DevObj& ob, float3 color, float sigma, float3 N, float3 V, float3 L) {
  if (ob.mat != kMatDiffuseBsdf) return color * kInvPi;
  const float a = 1.0f / (kPi + kOrenC * sigma), b = sigma * a;
  const float nl = fmaxf(dot(N, L), 0.f), nv = fmaxf(dot(N, V), 0.f);
  float t = dot(V, L) - nl * nv;
  if (t > 0.f) t = fmaxf(nl, nv) + kEps;
  return color * (a + b * t);
}

// Material sampling (diffuse_material.cc:3-30, diffuse_bsdf.cc:3-53): cosine-weighted
// about the shading normal N in the (T, Ng x T, N) frame; pdf = cos_theta / pi.
PSDR_D float3 material_dir(const Surf& x, float3 N, float ru, float rv, float& cos_theta, float& sin_theta,
                           float& sphi, float& cphi) {
  const float3 B = cross(x.n, x.t);
  cos_theta = ru > 0.f ? sqrtf(ru) : 0.f;
  sin_theta = (1.0f - ru) > 0.f ? sqrtf(1.0f - ru) : 0.f;
  sincosf(rv * k2Pi, &sphi, &cphi);
  const float uu = cphi * sin_theta, vv = sphi * sin_theta;
  return normalize(x.t * uu + B * vv + N * cos_theta);
}

// BSDF of surface point x toward L (incoming direction x.wi), any material.
PSDR_D float3 surf_bsdf(const DevScene& sc, const Surf& x, float3 L) {
  const DevObj& ob = sc.objs[x.obj];
  const float3 color = tex_rgb(ob.color, texel_offset(ob.color, x.u, x.v));
  if (ob.mat != kMatDiffuseBsdf) return color * kInvPi;
  float3 m;
  bool mapped;
  const float3 N = shading_normal(ob, x, m, mapped);
  return bsdf_value(ob, color, material_sigma(ob, x), N, x.wi, L);
}

// ------------------------------------------------------------------ light emission
constexpr int kLightArea = 0, kLightEnv = 1, kLightSh9 = 2;  // PSDR_LIGHT_*

// Second-order real spherical harmonics (emitter.cc:246-266): Y(0,0), Y(1,-1..1), Y(2,-2..2).
constexpr float kSh0 = 0.28209479177387814f;   // sqrt(1 / (4 pi))
constexpr float kSh1 = 0.48860251190291992f;   // sqrt(3 / (4 pi))
constexpr float kSh2 = 1.09254843059207907f;   // sqrt(15 / (4 pi))
constexpr float kSh3 = 0.31539156525252005f;   // sqrt(5 / (16 pi))
constexpr float kSh4 = 0.54627421529603953f;   // sqrt(15 / (16 pi))
PSDR_D void sh9_basis(float3 d, float Y[9]) {
  Y[0] = kSh0;
  Y[1] = kSh1 * d.y;
  Y[2] = kSh1 * d.z;
  Y[3] = kSh1 * d.x;
  Y[4] = kSh2 * (d.x * d.y);
  Y[5] = kSh2 * (d.y * d.z);
  Y[6] = kSh3 * (2.f * (d.z * d.z) - d.x * d.x - d.y * d.y);
  Y[7] = kSh2 * (d.z * d.x);
  Y[8] = kSh4 * (d.x * d.x - d.y * d.y);
}

// Radiance of an environment light hit at box uv (u, v) reached along incoming direction
// wi: EnvLight's cube map (emitter.cc:134-141), SH9Light's harmonics of wi
// (emitter.cc:268-275). Out of line: area-light kernels keep their register budgets.
static __device__ __noinline__ float3 env_emit(const DevLight* L, float u, float v, float3 wi) {
  if (L->kind == kLightEnv) return tex_rgb(L->tex, texel_offset(L->tex, u, v));
  float Y[9];
  sh9_basis(wi, Y);
  float3 e = f3(0.f, 0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 9; ++k) e += f3(L->sh[3 * k], L->sh[3 * k + 1], L->sh[3 * k + 2]) * Y[k];
  return e;
}

// Radiance of the light hit q (light L). EXT: the kernel instance for scenes with an
// environment light (or a DiffuseBsdfMaterial); the other instance has area lights only.
template <bool EXT>
PSDR_D float3 light_emit(const DevLight& L, const Surf& q) {
  if (!EXT || L.kind == kLightArea) return f3(L.emit[0], L.emit[1], L.emit[2]);
  return env_emit(&L, q.u, q.v, q.wi);
}

PSDR_D float mis_power(float w1, float w2, float n1, float n2) {
  const float a = (n1 * w1) * (n1 * w1), b = (n2 * w2) * (n2 * w2);
  return a / (a + b);
}

// emitter.cc:29-59 AreaLight::sample_light_point (triangle by area, sqrt warp).
struct LightSample {
  float3 y;
  float pdf;     // pdf_light * pdf_choose (detached)
  int light;
  int tri;       // global triangle id the point lies on
  float su, sv;  // y = p0 + (p1-p0) su + (p2-p0) sv
};
PSDR_D LightSample sample_light(const DevScene& sc, float rx, float ry) {
  LightSample ls;
  float pch = 1.0f;
  int l = discrete_sample(sc.light_pmf, sc.light_cmf, sc.nlight, rx, pch);
  const DevLight& L = sc.lights[l];
  float ptri;
  const int base = L.tri0 - sc.ltri_base;
  int k = discrete_sample(sc.ltri_pmf + base, sc.ltri_cmf + base, L.ntri, rx, ptri);
  const int tri = L.tri0 + k;
  const float4* r = sc.tri + 6 * (size_t)tri;
  const float3 p0 = xyz(__ldg(r)), p1 = xyz(__ldg(r + 1)), p2 = xyz(__ldg(r + 2));
  const float sq = ry > 0.f ? sqrtf(ry) : 0.f;
  ls.su = rx * sq;
  ls.sv = 1.0f - sq;
  ls.y = p0 + (p1 - p0) * ls.su + (p2 - p0) * ls.sv;
  ls.pdf = L.inv_area * pch;
  ls.light = l;
  ls.tri = tri;
  return ls;
}

}  // namespace psdr
