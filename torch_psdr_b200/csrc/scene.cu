// scene.cu -- scene construction on the device.
//
// Replaces Scene::Scene (scene.cc:3-104), TriangleMesh (mesh.cc:5-204) and the OptiX
// GAS build (scene_optix.cc:187-238):
//  * flattened vertex array and 96-byte per-triangle shading records,
//  * the edge list via a stable sort of half-edges by (min,max) vertex id (the
//    reference hashes them on the host; grouping by sorted key gives the same
//    left/right face assignment, in (min,max) order per mesh),
//  * discrete CDFs over edges (length), lights (power) and light triangles (area),
//  * an LBVH: 30-bit Morton codes of triangle-box centres (large triangles split off
//    by a top key bit), radix sort, Karras (2012) hierarchy, bottom-up boxes, then a
//    4-wide layout (pairwise collapse of the binary tree) with child boxes in the
//    parent and leaves of up to `leaf_size` triangles.
#include <algorithm>
#include <cmath>

#include "psdr_internal.h"

namespace psdr {

namespace {

// mesh.cc:27-67 triangle attributes (normal, uv tangent, Heron area).
__global__ void k_tri_records(int nF, const int* __restrict__ faces, int vbase, int tri_off, int obj,
                              const float* __restrict__ verts, const float* __restrict__ uvs,
                              const int* __restrict__ uvi, float4* __restrict__ out, int4* __restrict__ out_v) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nF) return;
  const int i0 = faces[3 * f] + vbase, i1 = faces[3 * f + 1] + vbase, i2 = faces[3 * f + 2] + vbase;
  const float3 p0 = f3(verts[3 * i0], verts[3 * i0 + 1], verts[3 * i0 + 2]);
  const float3 p1 = f3(verts[3 * i1], verts[3 * i1 + 1], verts[3 * i1 + 2]);
  const float3 p2 = f3(verts[3 * i2], verts[3 * i2 + 1], verts[3 * i2 + 2]);
  float uv[6] = {0.f, 0.f, 0.f, 1.f, 1.f, 0.f};
  if (uvs && uvi) {
    for (int c = 0; c < 3; ++c) {
      const int u = uvi[3 * f + c];
      uv[2 * c] = uvs[2 * u];
      uv[2 * c + 1] = uvs[2 * u + 1];
    }
  }
  const float3 a = p2 - p1, b = p0 - p2, c = p1 - p0;
  const float3 cr = cross(c, b);
  const float3 n = cr / sqrtf(sqnorm(cr));
  const float du1y = uv[3] - uv[1], du2y = uv[5] - uv[1];
  const float3 tw = c * du2y + b * du1y;
  const float3 t = tw / sqrtf(sqnorm(tw));
  const float la = norm(a), lb = norm(b), lc = norm(c);
  const float s = (la + lb + lc) / 2.0f;
  const float q = s * (s - la) * (s - lb) * (s - lc);
  const float area = q > 0.f ? sqrtf(q) : 0.f;
  float4* r = out + 6 * (size_t)(tri_off + f);
  r[0] = make_float4(p0.x, p0.y, p0.z, area);
  r[1] = make_float4(p1.x, p1.y, p1.z, __int_as_float(obj));
  r[2] = make_float4(p2.x, p2.y, p2.z, uv[0]);
  r[3] = make_float4(n.x, n.y, n.z, uv[1]);
  r[4] = make_float4(t.x, t.y, t.z, uv[2]);
  r[5] = make_float4(uv[3], uv[4], uv[5], 0.f);
  out_v[tri_off + f] = make_int4(i0, i1, i2, obj);
}

// emitter.cc:4-14 + sampler.h:86-96: per-light area, power and triangle CDF.
__global__ void k_light_setup(DevLight* lights, int nlight, const float4* __restrict__ tri, float* ltri_pmf,
                              float* ltri_cmf, int ltri_base, float* light_pmf, float* light_cmf) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double all_power = 0;
  for (int l = 0; l < nlight; ++l) {
    DevLight& L = lights[l];
    double tot = 0;
    for (int k = 0; k < L.ntri; ++k) tot += (double)tri[6 * (size_t)(L.tri0 + k)].w;
    double acc = 0;
    for (int k = 0; k < L.ntri; ++k) {
      double a = (double)tri[6 * (size_t)(L.tri0 + k)].w;
      acc += a;
      ltri_pmf[L.tri0 - ltri_base + k] = (float)(a / tot);
      ltri_cmf[L.tri0 - ltri_base + k] = (float)(acc / tot);
    }
    L.area = (float)tot;
    L.inv_area = 1.0f / (float)tot;
    const double lum = (double)L.emit[0] * 0.2126 + (double)L.emit[1] * 0.7152 + (double)L.emit[2] * 0.0722;
    // environment lights: 4 pi (emitter.cc:130, 243)
    const double pw = L.kind == 0 ? 2.0 * 3.14159265358979323846 * lum * tot : 4.0 * 3.14159265358979323846;
    L.power = (float)pw;
    all_power += pw;
  }
  double acc = 0;
  for (int l = 0; l < nlight; ++l) {
    const double lum = (double)lights[l].emit[0] * 0.2126 + (double)lights[l].emit[1] * 0.7152 +
                       (double)lights[l].emit[2] * 0.0722;
    const double p = lights[l].kind == 0 ? 2.0 * 3.14159265358979323846 * lum * (double)lights[l].area
                                         : 4.0 * 3.14159265358979323846;
    acc += p;
    light_pmf[l] = (float)(p / all_power);
    light_cmf[l] = (float)(acc / all_power);
  }
}

// ---------------------------------------------------------------- edges
// Half-edge h = 3f + slot: slot 0 (F0,F1,third F2), 1 (F1,F2,F0), 2 (F2,F0,F1).
__global__ void k_halfedges(int nF, const int4* __restrict__ tri_v, int tri_lo, int tri_hi,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  int n = 3 * nF;
  if (h >= n) return;
  const int f = h / 3, slot = h - 3 * f;
  const int4 v = tri_v[f];
  const int a = slot == 0 ? v.x : (slot == 1 ? v.y : v.z);
  const int b = slot == 0 ? v.y : (slot == 1 ? v.z : v.x);
  const uint32_t lo = (uint32_t)min(a, b), hi = (uint32_t)max(a, b);
  keys[h] = ((uint64_t)lo << 32) | hi;
  vals[h] = (uint32_t)h;
}

__global__ void k_edge_flags(const uint64_t* __restrict__ keys, int n, int* __restrict__ flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

PSDR_D float3 ldv(const float* v, int i) { return f3(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }

// mesh.cc:97-204 build_edges: left face = first half-edge of the group, right face =
// last one (a boundary edge uses the left face twice), normals, out direction and the
// orientation fix, length.
__global__ void k_edge_build(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, int n,
                             const int* __restrict__ flags, const int* __restrict__ eidx,
                             const int4* __restrict__ tri_v, const float* __restrict__ verts,
                             float4* __restrict__ edge, int2* __restrict__ edge_v, int2* __restrict__ edge_f,
                             float* __restrict__ elen, int* __restrict__ n_edges) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == n - 1) *n_edges = eidx[i] + flags[i];
  if (i >= n || !flags[i]) return;
  int j = i;
  while (j + 1 < n && keys[j + 1] == keys[i]) ++j;
  const uint32_t hl = vals[i], hr = vals[j];
  auto third = [&](uint32_t h) {
    const int f = h / 3, slot = h - 3 * f;
    const int4 v = tri_v[f];
    return slot == 0 ? v.z : (slot == 1 ? v.x : v.y);
  };
  const int fl = hl / 3, fr = hr / 3;
  const bool shared = j > i && fl != fr;
  const int kl = third(hl), kr = j > i ? third(hr) : kl;
  const int v0 = (int)(keys[i] >> 32), v1 = (int)(keys[i] & 0xffffffffu);
  const float3 p0 = ldv(verts, v0), p1 = ldv(verts, v1), p2l = ldv(verts, kl), p2r = ldv(verts, kr);
  float3 nl = normalize(cross(p1 - p0, p2l - p1));
  float3 nr = normalize(cross(p2r - p1, p1 - p0));
  float3 out = shared ? normalize(nl + nr) : normalize(cross(p1 - p0, nl));
  const float3 cp = normalize((p0 + p1) - (p2l + p2r));
  if (dot(cp, out) < 0.f && shared && norm(nl - nr) > kEps) { nl = -nl; nr = -nr; out = -out; }
  const float len = norm_rn(sub_rn(p0, p1));  // exact: the edge CDF matches the float oracle
  const int e = eidx[i];
  edge[4 * e + 0] = make_float4(p0.x, p0.y, p0.z, len);
  edge[4 * e + 1] = make_float4(p1.x, p1.y, p1.z, out.x);
  edge[4 * e + 2] = make_float4(out.y, out.z, nl.x, nl.y);
  edge[4 * e + 3] = make_float4(nl.z, nr.x, nr.y, nr.z);
  edge_v[e] = make_int2(v0, v1);
  edge_f[e] = j > i + 1 ? make_int2(kEdgeNonManifold, -1) : make_int2(fl, shared ? fr : -1);
  elen[e] = len;
}

__global__ void k_to_double(const float* __restrict__ in, const int* __restrict__ n_dev, int cap,
                            double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cap) return;
  out[i] = i < *n_dev ? (double)in[i] : 0.0;
}

__global__ void k_cdf_finalize(const double* __restrict__ w, const double* __restrict__ pre,
                               const int* __restrict__ n_dev, int cap, float* __restrict__ pmf,
                               float* __restrict__ cmf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *n_dev;
  if (i >= n || i >= cap) return;
  const double tot = pre[n - 1];
  pmf[i] = (float)(w[i] / tot);
  cmf[i] = (float)(pre[i] / tot);
}

// ---------------------------------------------------------------- LBVH
PSDR_D unsigned int f2ord(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
PSDR_D float ord2f(unsigned int u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

// n_core: triangles before the environment light's box (the box, 1000 times the scene,
// would squeeze the scene into a few Morton cells); the geometry box covers all n.
__global__ void k_centroid_box(int n, int n_core, const float4* __restrict__ tri, unsigned int* __restrict__ cbox) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float3 lo = f3(INFINITY, INFINITY, INFINITY), hi = f3(-INFINITY, -INFINITY, -INFINITY);
  float3 glo = lo, ghi = hi;
  if (i < n) {
    const float4* r = tri + 6 * (size_t)i;
    const float3 p0 = xyz(r[0]), p1 = xyz(r[1]), p2 = xyz(r[2]);
    const float3 bl = f3(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)), fminf(p0.z, fminf(p1.z, p2.z)));
    const float3 bh = f3(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)), fmaxf(p0.z, fmaxf(p1.z, p2.z)));
    const float3 c = (bl + bh) * 0.5f;
    if (i < n_core) { lo = c; hi = c; }
    glo = bl; ghi = bh;
  }
  for (int o = 16; o; o >>= 1) {
    lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
    lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
    lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
    glo.x = fminf(glo.x, __shfl_xor_sync(0xffffffffu, glo.x, o));
    glo.y = fminf(glo.y, __shfl_xor_sync(0xffffffffu, glo.y, o));
    glo.z = fminf(glo.z, __shfl_xor_sync(0xffffffffu, glo.z, o));
    ghi.x = fmaxf(ghi.x, __shfl_xor_sync(0xffffffffu, ghi.x, o));
    ghi.y = fmaxf(ghi.y, __shfl_xor_sync(0xffffffffu, ghi.y, o));
    ghi.z = fmaxf(ghi.z, __shfl_xor_sync(0xffffffffu, ghi.z, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(cbox + 0, f2ord(lo.x)); atomicMin(cbox + 1, f2ord(lo.y)); atomicMin(cbox + 2, f2ord(lo.z));
    atomicMax(cbox + 3, f2ord(hi.x)); atomicMax(cbox + 4, f2ord(hi.y)); atomicMax(cbox + 5, f2ord(hi.z));
    atomicMin(cbox + 6, f2ord(glo.x)); atomicMin(cbox + 7, f2ord(glo.y)); atomicMin(cbox + 8, f2ord(glo.z));
    atomicMax(cbox + 9, f2ord(ghi.x)); atomicMax(cbox + 10, f2ord(ghi.y)); atomicMax(cbox + 11, f2ord(ghi.z));
  }
}

__global__ void k_cbox_init(unsigned int* cbox) {
  int i = threadIdx.x;
  if (i < 12) cbox[i] = ((i % 6) < 3) ? 0xffffffffu : 0u;
}

PSDR_D unsigned int expand_bits(unsigned int v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_morton(int n, int n_core, const float4* __restrict__ tri, const unsigned int* __restrict__ cbox,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float3 lo = f3(ord2f(cbox[0]), ord2f(cbox[1]), ord2f(cbox[2]));
  const float3 hi = f3(ord2f(cbox[3]), ord2f(cbox[4]), ord2f(cbox[5]));
  const float4* r = tri + 6 * (size_t)i;
  const float3 p0 = xyz(r[0]), p1 = xyz(r[1]), p2 = xyz(r[2]);
  const float3 bl = f3(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)), fminf(p0.z, fminf(p1.z, p2.z)));
  const float3 bh = f3(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)), fmaxf(p0.z, fmaxf(p1.z, p2.z)));
  const float3 c = (bl + bh) * 0.5f;
  const float3 ext = hi - lo;
  auto q = [](float x, float l, float e) {
    float t = e > 0.f ? (x - l) / e : 0.5f;
    return (unsigned int)fminf(fmaxf(t * 1024.0f, 0.0f), 1023.0f);
  };
  unsigned int m = (expand_bits(q(c.x, lo.x, ext.x)) << 2) | (expand_bits(q(c.y, lo.y, ext.y)) << 1) |
                   expand_bits(q(c.z, lo.z, ext.z));
  // Triangles whose box spans more than a quarter of the scene (ground planes, walls)
  // get the top key bit, so the root splits them off instead of letting them inflate
  // the box of whatever small-triangle cluster shares their centroid cell.
  const float3 glo = f3(ord2f(cbox[6]), ord2f(cbox[7]), ord2f(cbox[8]));
  const float3 ghi = f3(ord2f(cbox[9]), ord2f(cbox[10]), ord2f(cbox[11]));
  const float sext = fmaxf(fmaxf(ghi.x - glo.x, ghi.y - glo.y), ghi.z - glo.z);
  const float text = fmaxf(fmaxf(bh.x - bl.x, bh.y - bl.y), bh.z - bl.z);
  if (text > 0.25f * sext || i >= n_core) m |= 1u << 30;
  keys[i] = m;
  vals[i] = (uint32_t)i;
}

// Common prefix of the (morton, index) pair keys at sorted positions i and j.
PSDR_D int delta(const uint64_t* __restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = (uint32_t)k[i], b = (uint32_t)k[j];
  if (a == b) return 32 + __clz((unsigned)(i ^ j));
  return __clz(a ^ b);
}

// Karras 2012: internal node i covers sorted leaves [first, last]; children are
// internal nodes (< n-1) or leaves (n-1 + k) in `parent`/`child` index space.
__global__ void k_karras(int n, const uint64_t* __restrict__ k, int2* __restrict__ child,
                         int2* __restrict__ range, int* __restrict__ parent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(k, n, i, i - d);
  int lmax = 2;
  while (delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(k, n, i, j);
  int s = 0;
  for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
    if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    if (t == 1) break;
  }
  const int g = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int left = (lo == g) ? (n - 1 + g) : g;
  const int right = (hi == g + 1) ? (n - 1 + g + 1) : (g + 1);
  child[i] = make_int2(left, right);
  range[i] = make_int2(lo, hi);
  parent[left] = i;
  parent[right] = i;
}

__global__ void k_bottom_up(int n, const uint32_t* __restrict__ order, const float4* __restrict__ tri,
                            const int2* __restrict__ child, const int* __restrict__ parent,
                            float* __restrict__ aabb, int* __restrict__ flags) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int t = order[k];
  const float4* r = tri + 6 * (size_t)t;
  const float3 p0 = xyz(r[0]), p1 = xyz(r[1]), p2 = xyz(r[2]);
  float* b = aabb + 6 * (size_t)(n - 1 + k);
  b[0] = fminf(p0.x, fminf(p1.x, p2.x)); b[1] = fminf(p0.y, fminf(p1.y, p2.y)); b[2] = fminf(p0.z, fminf(p1.z, p2.z));
  b[3] = fmaxf(p0.x, fmaxf(p1.x, p2.x)); b[4] = fmaxf(p0.y, fmaxf(p1.y, p2.y)); b[5] = fmaxf(p0.z, fmaxf(p1.z, p2.z));
  if (n == 1) return;
  int node = parent[n - 1 + k];
  while (true) {
    __threadfence();
    if (atomicAdd(&flags[node], 1) == 0) return;
    __threadfence();
    const int2 c = child[node];
    const volatile float* a = aabb + 6 * (size_t)c.x;
    const volatile float* bb = aabb + 6 * (size_t)c.y;
    float* o = aabb + 6 * (size_t)node;
    o[0] = fminf(a[0], bb[0]); o[1] = fminf(a[1], bb[1]); o[2] = fminf(a[2], bb[2]);
    o[3] = fmaxf(a[3], bb[3]); o[4] = fmaxf(a[4], bb[4]); o[5] = fmaxf(a[5], bb[5]);
    if (node == 0) return;
    node = parent[node];
  }
}

// ---- 4-wide BVH: greedy collapse of the binary tree. Starting from the root, a 4-wide
// node takes the two children of its binary node and keeps replacing the internal child
// with the largest surface area by that child's two children until it holds four (or
// only leaves are left); every internal child left in it becomes a 4-wide node of the
// next level. A binary node whose range holds at most leaf_size triangles is a leaf.
// One block walks the tree level by level; within a level the nodes take their indices
// in queue order through a block-wide scan, so the layout is the same on every build.
__device__ __forceinline__ float box_area(const float* b) {
  const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  return dx * dy + dy * dz + dz * dx;
}

__global__ void __launch_bounds__(1024) k_collapse4(int n, int leaf_size, const int2* __restrict__ child,
                                                    const int2* __restrict__ range, const float* __restrict__ aabb,
                                                    int* __restrict__ flag, int* __restrict__ idx4,
                                                    int* __restrict__ slots4, int* __restrict__ qa,
                                                    int* __restrict__ qb) {
  __shared__ int warp_sum[32];
  __shared__ int level_n, next_n, next_idx;
  auto expandable = [&](int c) {
    if (c >= n - 1) return false;
    const int2 r = range[c];
    return r.y - r.x + 1 > leaf_size;
  };
  if (threadIdx.x == 0) {
    qa[0] = 0;
    flag[0] = 1;
    idx4[0] = 0;
    level_n = 1;
    next_idx = 1;
  }
  __syncthreads();
  int* cur = qa;
  int* nxt = qb;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  while (level_n > 0) {
    const int m = level_n;
    if (threadIdx.x == 0) next_n = 0;
    __syncthreads();
    for (int base = 0; base < m; base += blockDim.x) {
      const int q = base + threadIdx.x;
      int sl[4] = {-1, -1, -1, -1};
      int cnt = 0;
      if (q < m) {
        const int i = cur[q];
        const int2 ch = child[i];
        sl[0] = ch.x;
        sl[1] = ch.y;
        int ns = 2;
        while (ns < 4) {
          int best = -1;
          float ba = -1.f;
          for (int k = 0; k < ns; ++k)
            if (expandable(sl[k])) {
              const float a = box_area(aabb + 6 * (size_t)sl[k]);
              if (a > ba) { ba = a; best = k; }
            }
          if (best < 0) break;
          const int2 g = child[sl[best]];
          sl[best] = g.x;
          sl[ns++] = g.y;
        }
        for (int k = 0; k < 4; ++k) {
          slots4[4 * (size_t)i + k] = sl[k];
          if (sl[k] >= 0 && expandable(sl[k])) ++cnt;
        }
      }
      // block-wide exclusive scan of cnt (queue order)
      int x = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) warp_sum[wid] = x;
      __syncthreads();
      if (wid == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, w, o);
          if (lane >= o) w += y;
        }
        warp_sum[lane] = w;  // inclusive over warps
      }
      __syncthreads();
      const int excl = x - cnt + (wid > 0 ? warp_sum[wid - 1] : 0);
      const int total = warp_sum[(blockDim.x >> 5) - 1];
      if (cnt > 0) {
        int k2 = excl;
        for (int k = 0; k < 4; ++k)
          if (sl[k] >= 0 && expandable(sl[k])) {
            const int c = sl[k];
            flag[c] = 1;
            idx4[c] = next_idx + k2;
            nxt[next_n + k2] = c;
            ++k2;
          }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        next_idx += total;
        next_n += total;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) level_n = next_n;
    int* t = cur;
    cur = nxt;
    nxt = t;
    __syncthreads();
  }
}

__global__ void k_layout4(int n, int leaf_size, const int* __restrict__ slots4, const int2* __restrict__ range,
                          const float* __restrict__ aabb, const unsigned int* __restrict__ cbox,
                          const int* __restrict__ flag, const int* __restrict__ idx4, float4* __restrict__ nodes4) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1 || !flag[i]) return;
  const float3 glo = f3(ord2f(cbox[6]), ord2f(cbox[7]), ord2f(cbox[8]));
  const float3 ghi = f3(ord2f(cbox[9]), ord2f(cbox[10]), ord2f(cbox[11]));
  const float ext = fmaxf(fmaxf(ghi.x - glo.x, ghi.y - glo.y), ghi.z - glo.z);
  const float apad = ext * 2e-6f + 1e-20f;
  auto is_leaf = [&](int c) {
    if (c >= n - 1) return true;
    const int2 r = range[c];
    return r.y - r.x + 1 <= leaf_size;
  };
  auto leaf_code = [&](int c) {
    if (c >= n - 1) return ~((c - (n - 1)) << 3);
    const int2 r = range[c];
    return ~((r.x << 3) | (r.y - r.x));
  };
  int slot[4];
  int ns = 0;
  for (int k = 0; k < 4; ++k) {
    const int c = slots4[4 * (size_t)i + k];
    if (c >= 0) slot[ns++] = c;
  }
  float lo[3][4], hi[3][4];
  int enc[4];
  for (int k = 0; k < 4; ++k) {
    if (k >= ns) {
      for (int q = 0; q < 3; ++q) { lo[q][k] = INFINITY; hi[q][k] = -INFINITY; }
      enc[k] = 0x7fffffff;
      continue;
    }
    const int c = slot[k];
    const float* b = aabb + 6 * (size_t)c;
    for (int q = 0; q < 3; ++q) {
      lo[q][k] = b[q] - (fabsf(b[q]) * 2e-6f + apad);
      hi[q][k] = b[3 + q] + (fabsf(b[3 + q]) * 2e-6f + apad);
    }
    enc[k] = is_leaf(c) ? leaf_code(c) : idx4[c];
  }
  float4* o = nodes4 + 7 * (size_t)idx4[i];
  o[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
  o[1] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
  o[2] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
  o[3] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
  o[4] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
  o[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
  o[6] = make_float4(__int_as_float(enc[0]), __int_as_float(enc[1]), __int_as_float(enc[2]), __int_as_float(enc[3]));
}

__global__ void k_leaf_tris(int n, const uint32_t* __restrict__ order, const float4* __restrict__ tri,
                            float4* __restrict__ leaf) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int t = order[k];
  const float4* r = tri + 6 * (size_t)t;
  const float4 a = r[0], b = r[1], c = r[2];
  leaf[3 * (size_t)k + 0] = make_float4(a.x, a.y, a.z, __int_as_float(t));
  leaf[3 * (size_t)k + 1] = make_float4(b.x, b.y, b.z, 0.f);
  leaf[3 * (size_t)k + 2] = make_float4(c.x, c.y, c.z, 0.f);
}

inline int nblk(int64_t n, int t = 256) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

}  // namespace

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Builds everything that depends on vertex positions (records, edges, CDFs, BVH) on
// stream `st`. Device work only (after the first build sized the scratch), so it can
// also be recorded into a graph.
// Vertices, triangle records, light tables and the edge list (everything but the BVH).
// Returns the number of triangles outside the environment light's box.
static int build_records_and_edges(psdr_scene* s, cudaStream_t st, int& vbits_out) {
  // vertices
  for (int o = 0; o < s->nobj; ++o) {
    const float* src = o < (int)s->meshes.size() ? s->meshes[o].vertices : s->lights[o - s->meshes.size()].vertices;
    PSDR_CUDA(cudaMemcpyAsync(s->verts.as<float>() + 3 * (size_t)s->obj_vert_off[o], src,
                              sizeof(float) * 3 * (size_t)s->obj_nvert[o], cudaMemcpyDeviceToDevice, st));
  }
  for (int o = 0; o < s->nobj; ++o) {
    const bool is_mesh = o < (int)s->meshes.size();
    const int* faces = is_mesh ? s->meshes[o].faces : s->lights[o - s->meshes.size()].faces;
    const float* uvs = is_mesh ? s->meshes[o].uvs : nullptr;
    const int* uvi = is_mesh ? s->meshes[o].uv_indices : nullptr;
    if (is_mesh && (!uvs || !uvi)) { uvs = nullptr; uvi = nullptr; }
    // the EnvLight box carries the cube-map uvs
    if (!is_mesh && o - (int)s->meshes.size() == s->env_light && s->lights[s->env_light].type == PSDR_LIGHT_ENV) {
      uvs = s->env_uv.as<float>();
      uvi = s->env_uvi.as<int>();
    }
    const int nF = s->obj_ntri[o];
    if (nF == 0) continue;
    k_tri_records<<<nblk(nF), 256, 0, st>>>(nF, faces, s->obj_vert_off[o], s->obj_tri_off[o], o, s->verts.as<float>(),
                                            uvs, uvi, s->tri.as<float4>(), s->tri_v.as<int4>());
  }
  PSDR_CUDA(cudaGetLastError());
  // lights (the table was uploaded at creation; area, power and CDFs are recomputed)
  if (s->nlight > 0) {
    k_light_setup<<<1, 1, 0, st>>>(s->lights_buf.as<DevLight>(), s->nlight, s->tri.as<float4>(), s->ltri_pmf.as<float>(),
                                   s->ltri_cmf.as<float>(), s->dev.ltri_base, s->light_pmf.as<float>(),
                                   s->light_cmf.as<float>());
  }
  // edges: sort half-edges by (min,max) vertex id; the environment light's box (the last
  // triangles) has no edges (scene.cc:59-62 takes them from the other meshes only)
  const int n_edge_tri = s->env_light >= 0 ? s->obj_tri_off[s->meshes.size() + s->env_light] : s->ntri;
  const int nh = 3 * n_edge_tri;
  uint64_t* keys = s->keys.as<uint64_t>();
  uint32_t* vals = s->vals.as<uint32_t>();
  k_halfedges<<<nblk(std::max(1, nh)), 256, 0, st>>>(n_edge_tri, s->tri_v.as<int4>(), 0, n_edge_tri, keys, vals);
  int vbits = 1;
  while ((1ll << vbits) < (long long)s->nvert) ++vbits;
  radix_sort_pairs(keys, vals, nh, 32 + vbits, s->sort_tmp, st);
  int* flags = s->aux_i.as<int>();
  int* eidx = s->aux_i2.as<int>();
  k_edge_flags<<<nblk(nh), 256, 0, st>>>(keys, nh, flags);
  exclusive_scan_int(flags, eidx, nh, s->flags.as<int>(), st);
  float* elen = reinterpret_cast<float*>(s->aux_d2.as<double>() + nh);  // scratch tail
  k_edge_build<<<nblk(nh), 256, 0, st>>>(keys, vals, nh, flags, eidx, s->tri_v.as<int4>(), s->verts.as<float>(),
                                         s->edge.as<float4>(), s->edge_v.as<int2>(), s->edge_f.as<int2>(), elen,
                                         s->n_edges.as<int>());
  k_to_double<<<nblk(nh), 256, 0, st>>>(elen, s->n_edges.as<int>(), nh, s->aux_d.as<double>());
  inclusive_scan_double(s->aux_d.as<double>(), s->aux_d2.as<double>(), nh,
                        reinterpret_cast<double*>(s->flags.as<int>()), st);
  k_cdf_finalize<<<nblk(nh), 256, 0, st>>>(s->aux_d.as<double>(), s->aux_d2.as<double>(), s->n_edges.as<int>(), nh,
                                           s->edge_pmf.as<float>(), s->edge_cmf.as<float>());
  PSDR_CUDA(cudaGetLastError());
  vbits_out = vbits;
  return n_edge_tri;
}

void scene_build_geometry(psdr_scene* s, cudaStream_t st) {
  int vbits = 1;
  const int n_edge_tri = build_records_and_edges(s, st, vbits);
  uint64_t* keys = s->keys.as<uint64_t>();
  uint32_t* vals = s->vals.as<uint32_t>();
  // BVH
  const int n = s->ntri;
  unsigned int* cbox = s->cbox.as<unsigned int>();
  k_cbox_init<<<1, 32, 0, st>>>(cbox);
  k_centroid_box<<<nblk(n), 256, 0, st>>>(n, n_edge_tri, s->tri.as<float4>(), cbox);
  k_morton<<<nblk(n), 256, 0, st>>>(n, n_edge_tri, s->tri.as<float4>(), cbox, keys, vals);
  radix_sort_pairs(keys, vals, n, 31, s->sort_tmp, st);
  int2* child = s->aux_i.as<int2>();
  int2* range = s->range.as<int2>();
  int* parent = s->parent.as<int>();
  float* aabb = s->aabb.as<float>();
  int* bflags = s->flags.as<int>();
  PSDR_CUDA(cudaMemsetAsync(bflags, 0, sizeof(int) * std::max(1, n), st));
  if (n > 1) k_karras<<<nblk(n - 1), 256, 0, st>>>(n, keys, child, range, parent);
  k_bottom_up<<<nblk(n), 256, 0, st>>>(n, vals, s->tri.as<float4>(), child, parent, aabb, bflags);
  if (n > 1) {
    // 4-wide nodes: flags (even depth), exclusive scan for their indices, layout. The
    // root (node 0) must stay an internal node: leaves hold fewer than n triangles.
    const int leaf = std::min(s->leaf_size, n - 1);
    int* f4 = s->aux_i2.as<int>();
    int* idx4 = s->aux_i2.as<int>() + n;
    int* slots4 = s->bvh_slots.as<int>();
    PSDR_CUDA(cudaMemsetAsync(f4, 0, sizeof(int) * (size_t)n, st));
    // the Morton keys are no longer needed: their storage holds the two level queues
    int* qa = reinterpret_cast<int*>(keys);
    k_collapse4<<<1, 1024, 0, st>>>(n, leaf, child, range, aabb, f4, idx4, slots4, qa, qa + n);
    k_layout4<<<nblk(n - 1), 256, 0, st>>>(n, leaf, slots4, range, aabb, cbox, f4, idx4, s->nodes.as<float4>());
    PSDR_CUDA(cudaMemcpyAsync(s->bvh_child.p, child, sizeof(int2) * (n - 1), cudaMemcpyDeviceToDevice, st));
    PSDR_CUDA(cudaMemcpyAsync(s->bvh_f4.p, f4, sizeof(int) * 2 * (size_t)n, cudaMemcpyDeviceToDevice, st));
  }
  k_leaf_tris<<<nblk(n), 256, 0, st>>>(n, vals, s->tri.as<float4>(), s->leaf.as<float4>());
  PSDR_CUDA(cudaMemcpyAsync(s->bvh_order.p, vals, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  // records + lights + half-edge sort (2 x passes x 5) + edge build/CDF (8) + BVH (9 + morton sort)
  count_launches(s->nobj + (s->nlight > 0) + 3 + 3 * ((32 + vbits + 7) / 8) + 8 + 8 + 3 * 4);
  PSDR_CUDA(cudaGetLastError());
}

// Same as scene_build_geometry for records, lights and edges, but the BVH keeps the tree
// of the last full build and only its boxes are recomputed (bottom-up over the saved
// child links and leaf order, then the 4-wide layout with the saved node indices). Any
// tree whose boxes bound their triangles gives the same closest hits.
void scene_refit_geometry(psdr_scene* s, cudaStream_t st) {
  int vbits = 1;
  const int n_edge_tri = build_records_and_edges(s, st, vbits);
  const int n = s->ntri;
  unsigned int* cbox = s->cbox.as<unsigned int>();
  k_cbox_init<<<1, 32, 0, st>>>(cbox);  // the scene extent pads the node boxes
  k_centroid_box<<<nblk(n), 256, 0, st>>>(n, n_edge_tri, s->tri.as<float4>(), cbox);
  const int2* child = s->bvh_child.as<int2>();
  const uint32_t* order = s->bvh_order.as<uint32_t>();
  float* aabb = s->aabb.as<float>();
  int* bflags = s->flags.as<int>();
  PSDR_CUDA(cudaMemsetAsync(bflags, 0, sizeof(int) * std::max(1, n), st));
  k_bottom_up<<<nblk(n), 256, 0, st>>>(n, order, s->tri.as<float4>(), child, s->parent.as<int>(), aabb, bflags);
  if (n > 1) {
    const int leaf = std::min(s->leaf_size, n - 1);
    const int* f4 = s->bvh_f4.as<int>();
    k_layout4<<<nblk(n - 1), 256, 0, st>>>(n, leaf, s->bvh_slots.as<int>(), s->range.as<int2>(), aabb, cbox, f4,
                                           f4 + n, s->nodes.as<float4>());
  }
  k_leaf_tris<<<nblk(n), 256, 0, st>>>(n, order, s->tri.as<float4>(), s->leaf.as<float4>());
  count_launches(s->nobj + (s->nlight > 0) + 3 + 3 * ((32 + vbits + 7) / 8) + 8 + 6);
  PSDR_CUDA(cudaGetLastError());
}

void psdr_scene_alloc(psdr_scene* s) {
  cudaStream_t st = s->stream;
  const int n = std::max(1, s->ntri), nh = 3 * n;
  s->verts.alloc(sizeof(float) * 3 * std::max(1, s->nvert), st);
  s->tri.alloc(sizeof(float4) * 6 * n, st);
  s->tri_v.alloc(sizeof(int4) * n, st);
  s->objs.alloc(sizeof(DevObj) * std::max(1, s->nobj), st);
  s->lights_buf.alloc(sizeof(DevLight) * std::max(1, s->nlight), st);
  s->light_pmf.alloc(sizeof(float) * std::max(1, s->nlight), st);
  s->light_cmf.alloc(sizeof(float) * std::max(1, s->nlight), st);
  int nlt = 0;
  for (auto& l : s->h_lights) nlt += l.ntri;
  s->ltri_pmf.alloc(sizeof(float) * std::max(1, nlt), st);
  s->ltri_cmf.alloc(sizeof(float) * std::max(1, nlt), st);
  s->n_edges.alloc(sizeof(int), st);
  s->edge.alloc(sizeof(float4) * 4 * nh, st);
  s->edge_v.alloc(sizeof(int2) * nh, st);
  s->edge_f.alloc(sizeof(int2) * nh, st);
  s->edge_pmf.alloc(sizeof(float) * nh, st);
  s->edge_cmf.alloc(sizeof(float) * nh, st);
  s->nodes.alloc(sizeof(float4) * 7 * n, st);
  s->leaf.alloc(sizeof(float4) * 3 * n, st);
  s->err.alloc(sizeof(int), st);
  s->keys.alloc(sizeof(uint64_t) * nh, st);
  s->vals.alloc(sizeof(uint32_t) * nh, st);
  s->aux_i.alloc(sizeof(int2) * nh, st);
  s->aux_i2.alloc(sizeof(int) * std::max<size_t>(nh, 2 * (size_t)n), st);
  s->aux_d.alloc(sizeof(double) * nh, st);
  s->aux_d2.alloc(sizeof(double) * nh + sizeof(float) * nh, st);
  s->aabb.alloc(sizeof(float) * 6 * (2 * (size_t)n), st);
  s->parent.alloc(sizeof(int) * 2 * (size_t)n, st);
  s->range.alloc(sizeof(int2) * n, st);
  s->flags.alloc(sizeof(int) * (2 * (size_t)n + std::max<size_t>(2 * (size_t)n, 2 * scan_tmp_ints(nh) + 64)), st);
  s->cbox.alloc(sizeof(unsigned int) * 12, st);
  s->bvh_child.alloc(sizeof(int2) * n, st);
  s->bvh_order.alloc(sizeof(uint32_t) * n, st);
  s->bvh_f4.alloc(sizeof(int) * 2 * (size_t)n, st);
  s->bvh_slots.alloc(sizeof(int) * 4 * (size_t)n, st);
  s->d_dev.alloc(sizeof(DevScene), st);
  PSDR_CUDA(cudaMemsetAsync(s->err.p, 0, sizeof(int), st));
  DevScene& d = s->dev;
  d.ntri = s->ntri; d.nvert = s->nvert; d.nobj = s->nobj; d.nlight = s->nlight;
  d.tri = s->tri.as<float4>(); d.tri_v = s->tri_v.as<int4>(); d.verts = s->verts.as<float>();
  d.objs = s->objs.as<DevObj>(); d.lights = s->lights_buf.as<DevLight>();
  d.light_pmf = s->light_pmf.as<float>(); d.light_cmf = s->light_cmf.as<float>();
  d.ltri_pmf = s->ltri_pmf.as<float>(); d.ltri_cmf = s->ltri_cmf.as<float>();
  d.edge_cap = nh; d.n_edges = s->n_edges.as<int>(); d.edge = s->edge.as<float4>(); d.edge_v = s->edge_v.as<int2>();
  d.edge_f = s->edge_f.as<int2>();
  d.edge_pmf = s->edge_pmf.as<float>(); d.edge_cmf = s->edge_cmf.as<float>();
  d.nodes = s->nodes.as<float4>(); d.leaf = s->leaf.as<float4>();
  d.root = s->ntri > 1 ? 0 : ~0;  // a single triangle makes the root a leaf
  d.grad_verts = nullptr;
  d.vmask = nullptr;
  d.err = s->err.as<int>();
}

}  // namespace psdr

// Host -> device uploads of the object and light tables and the scene record; done
// once at creation so that the geometry rebuild (psdr_scene_update, or a rebuild
// recorded into a batch graph) is made of device work only.
void psdr_scene::upload_tables() {
  using namespace psdr;
  PSDR_CUDA(cudaMemcpyAsync(objs.p, h_objs.data(), sizeof(DevObj) * std::max<size_t>(1, h_objs.size()),
                            cudaMemcpyHostToDevice, stream));
  if (nlight > 0)
    PSDR_CUDA(cudaMemcpyAsync(lights_buf.p, h_lights.data(), sizeof(DevLight) * nlight, cudaMemcpyHostToDevice,
                              stream));
  PSDR_CUDA(cudaMemcpyAsync(d_dev.p, &dev, sizeof(DevScene), cudaMemcpyHostToDevice, stream));
}
