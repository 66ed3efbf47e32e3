// render.cu -- wavefront path tracing, path-replay adjoint and edge sampling.
//
// Forward (path_integrator.cc:80-186 trace2light, :355-372 render_interior,
// camera.h:75-87 Film::add) as wavefront kernels over a tile of path samples:
//   k_camera  : sampler stream, pixel jitter, camera ray, primary closest hit
//   per depth : k_shade (hit-light test, light / BSDF / indirect sampling, ray write
//               with warp-aggregated compaction) -> k_trace (closest hit per ray)
//               -> k_accum (NEE + MIS contributions, throughput, compaction)
//   k_film    : per-pixel average of its spp paths (deterministic, no atomics).
// Backward (Wrap2torch.backward + enoki reverse sweep, torch_psdr.py:48-72): the tile
// is re-traced from the stored seeds recording only hit records, then k_adjoint
// replays every path's sampler stream and applies the hand-written adjoint of the
// estimator, scattering into fp64 accumulators (warp-aggregated where a warp shares
// the target). Primary-edge (path_integrator.cc:188-272) and direct-edge (:274-353)
// boundary terms follow the reference formulas (PSDR_EST_REFERENCE).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "render.h"

namespace psdr {

// ------------------------------------------------------------------ helpers
PSDR_D unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp-aggregated append: all lanes of the warp must call it together.
PSDR_D int warp_append(int* counter, bool pred) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return -1;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  return pred ? base + __popc(m & lanemask_lt()) : -1;
}

PSDR_D void xform_pos(const float* m, float3 p, float3& out) {
  const float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
  out = f3((m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3]) / w, (m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7]) / w,
           (m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]) / w);
}
PSDR_D float3 xform_dir(const float* m, float3 p) {
  return f3(m[0] * p.x + m[1] * p.y + m[2] * p.z, m[4] * p.x + m[5] * p.y + m[6] * p.z,
            m[8] * p.x + m[9] * p.y + m[10] * p.z);
}

// camera.h:260-276 gen_camera_ray_with_point: visibility in the raster + pixel.
PSDR_D bool project(const DevView& V, float3 pt, int& px, int& py) {
  float3 pc, p;
  xform_pos(V.w2c, pt, pc);
  xform_pos(V.c2r, pc, p);
  px = (int)floorf(p.x);
  py = (int)floorf(p.y);
  return pc.z < 0.f && p.x > 0.f && p.x < (float)V.W && p.y > 0.f && p.y < (float)V.H;
}

// camera.h:121 look direction c2w (0, 0, -1).
PSDR_D float3 view_look_dir(const DevView& V) { return f3(-V.c2w[2], -V.c2w[6], -V.c2w[10]); }

// camera.h:336-353 orthographic ray toward world point pt: origin c2w (w2c pt).xy0 (in
// the same rounded operations as the float oracle), direction the look direction.
PSDR_D float3 ortho_origin_rn(const DevView& V, float3 pt) {
  const float3 pc = xform_pos_rn(V.w2c, pt);
  return xform_pos_rn(V.c2w, f3(pc.x, pc.y, 0.f));
}

// Transposed Jacobian of that origin w.r.t. the point, applied to a: M^T a with
// M = C diag(1, 1, 0) W (C, W the rotation parts of c2w, w2c).
PSDR_D float3 ortho_origin_jt(const DevView& V, float3 a) {
  const float ux = V.c2w[0] * a.x + V.c2w[4] * a.y + V.c2w[8] * a.z;
  const float uy = V.c2w[1] * a.x + V.c2w[5] * a.y + V.c2w[9] * a.z;
  return f3(V.w2c[0] * ux + V.w2c[4] * uy, V.w2c[1] * ux + V.w2c[5] * uy, V.w2c[2] * ux + V.w2c[6] * uy);
}

PSDR_D int find_view(const DevView* __restrict__ views, int nv, long long g) {
  int lo = 0, hi = nv - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (views[mid].sample_off <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}
PSDR_D int find_view_pix(const DevView* __restrict__ views, int nv, long long g) {
  int lo = 0, hi = nv - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (views[mid].pix_off <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

PSDR_D float4 hit4(const HitRec& h) { return make_float4(__int_as_float(h.tri), h.b1, h.b2, h.t); }

// Out of line: the adjoint kernels scatter vertex and texel gradients from many call
// sites, and one copy of the three fixed-point conversions keeps their loops smaller in
// the instruction cache.
static __device__ __noinline__ void atomic_add3(GradAcc* p, float3 v) {
  acc_add(p, v.x);
  acc_add(p + 1, v.y);
  acc_add(p + 2, v.z);
}

// Vertex gradients are accumulated only for the vertices the caller asked for.
PSDR_D bool vert_wanted(const DevScene& sc, int v) { return sc.grad_verts && (!sc.vmask || sc.vmask[v]); }
PSDR_D void vert_add(const DevScene& sc, int v, float3 a) {
  if (vert_wanted(sc, v)) atomic_add3(sc.grad_verts + 3 * (size_t)v, a);
}

// ------------------------------------------------------------------ camera kernel
// ORTHO: the instance for jobs with an orthographic view (it handles both camera types).
// The replay instance is held to 4 blocks per SM (64 registers): its record writes
// otherwise take it to 76 registers and 3 blocks.
template <int MODE, bool ORTHO>
__global__ void __launch_bounds__(256, MODE != MODE_FWD ? 4 : 1) k_camera(WF w, const DevScene* __restrict__ scenes,
                                                const DevView* __restrict__ views, Tile tile) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (tile.n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    if (s < tile.n) {
      const long long g = tile.begin + s;
      const int v = find_view(views, w.nviews, g);
      const DevView& V = views[v];
      const DevScene& sc = scenes[V.scene];
      const long long i = g - V.sample_off;
      Rng rng = make_rng((unsigned long long)i + w.seed);
      const float jx = rng.next_float(), jy = rng.next_float();
      const int pix = V.spp > 1 ? (int)(i / V.spp) : (int)i;
      const int x = pix % V.W, y = pix / V.W;
      float3 pc;
      xform_pos(V.r2c, f3(jx + (float)x, jy + (float)y, 1.0f), pc);
      float3 o = V.pos, d;
      if (ORTHO && V.ortho) {
        // camera.h:313-334: origin on the camera plane, direction the look direction
        xform_pos(V.c2w, f3(pc.x, pc.y, 0.f), o);
        d = view_look_dir(V);
      } else {
        d = normalize(xform_dir(V.c2w, pc));
      }
      w.org[s] = make_float4(o.x, o.y, o.z, 0.f);  // before the out-of-line trace: o dies there
      const HitRec h = trace_closest(sc, o, d, kTmin, INFINITY);
      w.rs[s] = rng.state;
      w.ri[s] = rng.inc;
      w.view[s] = v;
      w.pix[s] = pix;
      w.T[s] = make_float4(1.f, 1.f, 1.f, 0.f);
      w.L[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      w.cur[s] = hit4(h);
      if (MODE != MODE_FWD) {
        float4* rec = w.rec + (size_t)s * w.rec_stride;
        rec[0] = hit4(h);
        float4* cb = rec + 1 + (size_t)w.D * w.R;
        for (int q = 0; q < 2 * w.D; ++q) cb[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      alive = h.tri >= 0;
    }
    const int k = warp_append(&w.cnt[0], alive);
    if (alive) w.q0[k] = s;
  }
}

// ------------------------------------------------------------------ shade kernel
// Hit-light test and all samples of one depth; rays are written to the shaded slot.
template <int MODE, bool BSDF>
__global__ void __launch_bounds__(256) k_shade(WF w, const DevScene* __restrict__ scenes,
                                               const DevView* __restrict__ views, int d) {
  const int* qin = (d & 1) ? w.q1 : w.q0;
  const int n = w.cnt[2 * d];
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const bool last = d == w.D - 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) w.cnt[2 * w.D + 2] = 0;  // ray fetch counter of k_trace
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n32; q += stride) {
    bool go = false;
    int s = -1;
    Surf x;
    const DevScene* sc = nullptr;
    if (q < n) {
      s = qin[q];
      sc = &scenes[views[w.view[s]].scene];
      const float4 c = w.cur[s];
      x = make_surf(*sc, __float_as_int(c.x), c.y, c.z, xyz(w.org[s]));
      if (x.is_light) {
        if (MODE != MODE_REPLAY && w.light_vis && d == 0) {
          const DevLight& Lt = sc->lights[x.light];
          float4 L = w.L[s];
          const float4 T = w.T[s];
          const float3 e = light_emit<BSDF>(Lt, x);
          L.x += T.x * e.x; L.y += T.y * e.y; L.z += T.z * e.z;
          w.L[s] = L;
        }
      } else {
        go = true;
      }
    }
    const int k = warp_append(&w.cnt[2 * d + 1], go);
    if (!go) continue;
    w.qs[k] = s;
    Rng rng{w.rs[s], w.ri[s]};
    float3 mm;
    bool mapped;
    const float3 Ns = BSDF ? shading_normal(sc->objs[x.obj], x, mm, mapped) : x.n;
    // rays are stored type-major (slot r * cap + k): a warp of k_trace then traces
    // rays of one kind from neighbouring paths
    const size_t cs = (size_t)w.cap;
    for (int i = 0; i < w.nL; ++i) {
      const float rx = rng.next_float(), ry = rng.next_float();
      const LightSample ls = sample_light(*sc, rx, ry);
      const float3 dv = ls.y - x.p;
      const float3 dir = normalize(dv);
      const float dist = norm(dv);
      const size_t slot = i * cs + k;
      w.ro[slot] = make_float4(x.p.x, x.p.y, x.p.z, dist * 1.0001f + 4e-3f);
      w.rd[slot] = make_float4(dir.x, dir.y, dir.z, __int_as_float(ls.light));
      w.ra[slot] = make_float4(ls.y.x, ls.y.y, ls.y.z, ls.pdf);
    }
    for (int j = 0; j < w.nB; ++j) {
      const float rx = rng.next_float(), ry = rng.next_float();
      float ct, st, sp, cp;
      const float3 wo = BSDF ? material_dir(x, Ns, rx, ry, ct, st, sp, cp) : diffuse_dir(x.n, x.t, rx, ry, ct, st, sp, cp);
      const size_t slot = (w.nL + j) * cs + k;
      w.ro[slot] = make_float4(x.p.x, x.p.y, x.p.z, INFINITY);
      w.rd[slot] = make_float4(wo.x, wo.y, wo.z, 0.f);
      w.ra[slot] = make_float4(ct, 0.f, 0.f, 0.f);
    }
    {
      const float rx = rng.next_float(), ry = rng.next_float();
      if (!last) {
        float ct, st, sp, cp;
        const float3 wo =
            BSDF ? material_dir(x, Ns, rx, ry, ct, st, sp, cp) : diffuse_dir(x.n, x.t, rx, ry, ct, st, sp, cp);
        const size_t slot = (w.nL + w.nB) * cs + k;
        w.ro[slot] = make_float4(x.p.x, x.p.y, x.p.z, INFINITY);
        w.rd[slot] = make_float4(wo.x, wo.y, wo.z, 0.f);
        w.ra[slot] = make_float4(ct, 0.f, 0.f, 0.f);
      }
    }
    w.rs[s] = rng.state;
  }
}

// ------------------------------------------------------------------ trace kernel
// Closest hit of every queued ray of a depth (light-sample rays r < nL stop at the first
// hit short of the light). Persistent warps with dynamic ray fetch: a lane whose ray
// has finished takes the next unclaimed ray of the queue after every 8 traversal steps,
// so a warp keeps its lanes busy instead of waiting for its longest ray (the rays of a
// warp differ in traversal length by an order of magnitude). The fetch counter is
// w.cnt[2D+2], reset by k_shade.
constexpr int kTraceSteps = 8;
// Lights of at most this many triangles in all let k_trace answer MIS BSDF-sample rays
// with a light test and a bounded occlusion query.
constexpr int kMisLightTris = 16;
__global__ void __launch_bounds__(128) k_trace(WF w, const DevScene* __restrict__ scenes,
                                                   const DevView* __restrict__ views, int d,
                                                   unsigned long long* __restrict__ ray_count) {
  const int nk = w.cnt[2 * d + 1];
  const int Rd = (d == w.D - 1) ? w.R - 1 : w.R;
  const long long total = (long long)nk * Rd;
  if (ray_count && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(ray_count, (unsigned long long)total);
  int* fetch = w.cnt + 2 * w.D + 2;
  // traversal stack: the first kShort entries of each lane in shared memory (one column per
  // lane, so a warp's pushes and pops hit 32 banks), the deeper ones in local memory
  constexpr int kShort = 16;
  __shared__ int sst[kShort][128];
  struct Stk {
    int (*sh)[128];
    int lane;
    int deep[kStack - kShort];
    __device__ __forceinline__ void push(int i, int v) { if (i < kShort) sh[i][lane] = v; else deep[i - kShort] = v; }
    __device__ __forceinline__ int pop(int i) const { return i < kShort ? sh[i][lane] : deep[i - kShort]; }
  } stack;
  stack.sh = sst;
  stack.lane = threadIdx.x;
  TraceState s;
  const DevScene* sc = nullptr;
  size_t slot = 0;
  bool live = false, done = false;
  while (true) {
    const unsigned want = __ballot_sync(0xffffffffu, !live && !done);
    if (want) {
      const int lane = threadIdx.x & 31, leader = __ffs(want) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(fetch, __popc(want));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!live && !done) {
        const long long idx = (long long)base + __popc(want & lanemask_lt());
        if (idx < total) {
          const int r = (int)(idx / nk);
          const int k = (int)(idx - (long long)r * nk);
          slot = (size_t)r * w.cap + k;
          sc = &scenes[views[w.view[w.qs[k]]].scene];
          const float4 o = w.ro[slot], dd = w.rd[slot];
          const float t_occ = r < w.nL ? (o.w - 4e-3f) / 1.0001f - 4e-3f : -INFINITY;
          trace_begin(s, xyz(o), xyz(dd), kTmin, o.w, t_occ, sc->root);
          live = sc->ntri > 0;
          if (live && r >= w.nL && r < w.nL + w.nB && sc->nlight > 0) {
            // MIS BSDF-sample ray: only a light hit contributes (the shade, accumulate and
            // adjoint kernels skip any other hit). The closest light triangle along the ray
            // (the traversal's test and tie rule) bounds an occlusion query: a nearer hit is
            // reported as a miss, and with no light along the ray nothing is traversed.
            int nlt = 0;
            for (int l = 0; l < sc->nlight; ++l) nlt += sc->lights[l].ntri;
            if (nlt <= kMisLightTris) {
              float tl = o.w;
              int best = -1;
              for (int l = 0; l < sc->nlight; ++l) {
                const DevLight& Lt = sc->lights[l];
                for (int t = Lt.tri0; t < Lt.tri0 + Lt.ntri; ++t) {
                  const float4* q = sc->tri + 6 * (size_t)t;
                  float tt, b1, b2;
                  if (tri_test(s.rp, xyz(__ldg(q)), xyz(__ldg(q + 1)), xyz(__ldg(q + 2)), kTmin, tl, tt, b1, b2) &&
                      (tt < tl || best < 0 || t < best)) {
                    tl = tt;
                    best = t;
                  }
                }
              }
              if (best < 0) {
                live = false;
                w.hit[slot] = make_float4(__int_as_float(-1), 0.f, 0.f, o.w);
              } else {
                s.h.t = tl;
                s.t_occ = tl;
              }
            }
          }
          if (!live && sc->ntri <= 0) w.hit[slot] = make_float4(__int_as_float(-1), 0.f, 0.f, o.w);
        } else {
          done = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, live)) {
      if (__all_sync(0xffffffffu, done)) break;
      continue;
    }
    if (live) {
#pragma unroll 1
      for (int it = 0; it < kTraceSteps; ++it) {
        if (trace_step(*sc, s, stack)) {
          w.hit[slot] = make_float4(__int_as_float(s.h.tri), s.h.b1, s.h.b2, s.h.t);
          live = false;
          break;
        }
      }
    }
  }
}

// ------------------------------------------------------------------ accumulate kernel
// Per shaded path: the depth's contribution C (light samples + MIS-weighted BSDF
// samples, path_integrator.cc:103-160) and throughput factor beta (indirect bounce,
// :163-181). FWD folds them into L and T; REPLAY also stores the hit records and
// (C, beta) of the depth, which is all the adjoint needs besides the sampler stream.
template <int MODE, bool BSDF>
__global__ void __launch_bounds__(256) k_accum(WF w, const DevScene* __restrict__ scenes,
                                               const DevView* __restrict__ views, int d) {
  const int n = w.cnt[2 * d + 1];
  int* qout = (d & 1) ? w.q0 : w.q1;
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const bool last = d == w.D - 1;
  const float fL = (float)w.nL, fB = (float)w.nB;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n32; k += stride) {
    bool cont = false;
    int s = -1;
    if (k < n) {
      s = w.qs[k];
      const DevScene& sc = scenes[views[w.view[s]].scene];
      const size_t cs = (size_t)w.cap;
      const float4 c = w.cur[s];
      const Surf x = make_surf(sc, __float_as_int(c.x), c.y, c.z, xyz(w.org[s]));
      const DevObj& ob = sc.objs[x.obj];
      const float3 color = tex_rgb(ob.color, texel_offset(ob.color, x.u, x.v));
      const float3 bsdf = color * kInvPi;
      // DiffuseBsdfMaterial: the value depends on the outgoing direction
      const bool rough = BSDF && ob.mat == kMatDiffuseBsdf;
      float3 Ns = x.n;
      float sigma = 0.f;
      if (rough) {
        float3 mm;
        bool mapped;
        Ns = shading_normal(ob, x, mm, mapped);
        sigma = material_sigma(ob, x);
      }
      auto fr = [&](float3 L) { return rough ? bsdf_value(ob, color, sigma, Ns, x.wi, L) : bsdf; };
      float3 C = f3(0.f, 0.f, 0.f), beta = f3(0.f, 0.f, 0.f);
      for (int i = 0; i < w.nL; ++i) {
        const float4 h = w.hit[i * cs + k];
        const int tri = __float_as_int(h.x);
        if (tri < 0) continue;
        const float4 dd = w.rd[i * cs + k], aux = w.ra[i * cs + k];
        const float3 dir = xyz(dd);
        const Surf q = make_surf(sc, tri, h.y, h.z, x.p);
        if (!(q.is_light && sqnorm(q.p - xyz(aux)) < kEps)) continue;
        const DevLight& Lt = sc.lights[__float_as_int(dd.w)];
        const float tmp = dot(q.n, -dir) / q.sqd;
        const float G = dot(x.n, dir) * tmp;
        const float pdf_l = aux.w;
        float wgt = 1.0f / fL;
        if (w.nB > 0) wgt *= mis_power(pdf_l, dot(x.n, dir) * kInvPi * tmp, fL, fB);
        const float3 f = fr(dir);
        C += mul(light_emit<BSDF>(Lt, q), f) * (G / pdf_l * wgt);
      }
      for (int j = 0; j < w.nB; ++j) {
        const size_t slot = (w.nL + j) * cs + k;
        const float4 h = w.hit[slot];
        const int tri = __float_as_int(h.x);
        if (tri < 0) continue;
        const float3 wo = xyz(w.rd[slot]);
        const float ct = w.ra[slot].x;
        const Surf q = make_surf(sc, tri, h.y, h.z, x.p);
        if (!q.is_light) continue;
        const DevLight& Lt = sc.lights[q.light];
        const float tmp = dot(q.n, -wo) / q.sqd;
        const float G = dot(x.n, wo) * tmp;
        const float pdf_b = ct * kInvPi * tmp;
        float wgt = 1.0f / fB;
        if (w.nL > 0) wgt *= mis_power(pdf_b, __ldg(sc.light_pmf + q.light) * Lt.inv_area, fB, fL);
        const float3 f = fr(wo);
        C += mul(light_emit<BSDF>(Lt, q), f) * (G / pdf_b * wgt);
      }
      float4 hn = make_float4(__int_as_float(-1), 0.f, 0.f, 0.f);
      if (!last) {
        const size_t slot = (w.nL + w.nB) * cs + k;
        hn = w.hit[slot];
        const int tri = __float_as_int(hn.x);
        if (tri >= 0) {
          const float3 wo = xyz(w.rd[slot]);
          const float ct = w.ra[slot].x;
          const Surf nx = make_surf(sc, tri, hn.y, hn.z, x.p);
          const float tmp = dot(nx.n, -wo) / nx.sqd;
          const float G = dot(x.n, wo) * tmp;
          const float pdf = ct * kInvPi * tmp;
          beta = fr(wo) * (G / pdf);
          w.cur[s] = hn;
          w.org[s] = make_float4(x.p.x, x.p.y, x.p.z, 0.f);
          cont = true;
        }
      }
      if (MODE != MODE_FWD) {
        float4* rec = w.rec + (size_t)s * w.rec_stride;
        float4* rh = rec + 1 + (size_t)d * w.R;
        const int Rd = last ? w.R - 1 : w.R;
        for (int r = 0; r < Rd; ++r) rh[r] = w.hit[r * cs + k];
        float4* cb = rec + 1 + (size_t)w.D * w.R + 2 * d;
        cb[0] = make_float4(C.x, C.y, C.z, 0.f);
        cb[1] = make_float4(beta.x, beta.y, beta.z, 0.f);
      }
      if (MODE != MODE_REPLAY) {
        const float3 T = xyz(w.T[s]);
        const float3 L = xyz(w.L[s]) + mul(T, C);
        const float3 Tn = mul(T, beta);
        w.T[s] = make_float4(Tn.x, Tn.y, Tn.z, 0.f);
        w.L[s] = make_float4(L.x, L.y, L.z, 0.f);
      }
    }
    const int kk = warp_append(&w.cnt[2 * (d + 1)], cont);
    if (cont) qout[kk] = s;
  }
}

// ------------------------------------------------------------------ film
// Per pixel: sum of its spp path radiances (non-finite paths count as 0), / spp,
// then the n_pass average of identical passes (path_integrator.cc:381-406).
__global__ void k_film(WF w, const DevView* __restrict__ views, Tile tile, int n_pass, float* samples_out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < tile.npix; p += gridDim.x * blockDim.x) {
    const long long gp = tile.pix_begin + p;
    const int v = find_view_pix(views, w.nviews, gp);
    const DevView& V = views[v];
    const long long lp = gp - V.pix_off;
    const long long s0 = V.sample_off + lp * V.spp - tile.begin;
    float3 acc = f3(0.f, 0.f, 0.f);
    for (int k = 0; k < V.spp; ++k) {
      const long long s = s0 + k;
      float3 L = xyz(w.L[s]);
      if (!finite3(L) || __float_as_int(w.cur[s].x) == -2) L = f3(0.f, 0.f, 0.f);
      if (samples_out) {
        samples_out[3 * (lp * V.spp + k)] = L.x;
        samples_out[3 * (lp * V.spp + k) + 1] = L.y;
        samples_out[3 * (lp * V.spp + k) + 2] = L.z;
      }
      acc += L;
    }
    float3 val = acc / (float)V.spp;
    if (n_pass > 1) {
      float3 a = f3(0.f, 0.f, 0.f);
      for (int i = 0; i < n_pass; ++i) a += val;
      val = a / (float)n_pass;
    }
    if (V.image) {
      float* o = V.image + 3 * lp;
      o[0] = val.x; o[1] = val.y; o[2] = val.z;
    }
  }
}

// ------------------------------------------------------------------ adjoint helpers
struct SurfAdj {
  float3 p, n, t;
  float area;
};
PSDR_D SurfAdj zero_adj() {
  SurfAdj a;
  a.p = a.n = a.t = f3(0.f, 0.f, 0.f);
  a.area = 0.f;
  return a;
}

// Light vertices accumulated in registers (single area light with <= 8 vertices).
struct HotAcc {
  int lv0, nlv;   // vertex range of the light mesh; nlv = 0 disables
  bool emit_hot;  // single light: accumulate its emission gradient in e[]
  float g[kMaxLightVerts * 3];
  float e[3];
};

// Adjoint ae of an environment light's radiance at box uv (u, v), incoming direction wi:
// scatters into the cube-map texel or the SH coefficients and returns the adjoint of wi.
static __device__ __noinline__ float3 env_emit_adj(const DevLight* L, float u, float v, float3 wi, float3 ae) {
  if (L->kind == kLightEnv) {
    if (L->tex.grad) atomic_add3(L->tex.grad + texel_offset(L->tex, u, v), ae);
    return f3(0.f, 0.f, 0.f);
  }
  float Y[9];
  sh9_basis(wi, Y);
  float s[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    if (L->grad_sh) atomic_add3(L->grad_sh + 3 * k, ae * Y[k]);
    s[k] = ae.x * L->sh[3 * k] + ae.y * L->sh[3 * k + 1] + ae.z * L->sh[3 * k + 2];
  }
  const float x = wi.x, y = wi.y, z = wi.z;
  return f3(kSh1 * s[3] + kSh2 * (s[4] * y + s[7] * z) - 2.f * kSh3 * s[6] * x + 2.f * kSh4 * s[8] * x,
            kSh1 * s[1] + kSh2 * (s[4] * x + s[5] * z) - 2.f * kSh3 * s[6] * y - 2.f * kSh4 * s[8] * y,
            kSh1 * s[2] + kSh2 * (s[5] * y + s[7] * x) + 4.f * kSh3 * s[6] * z);
}

// Emission adjoint of light hit q reached from x: area lights into the emission
// accumulator, environment lights into their parameters, and the SH9 direction's share
// into the point x (wi = -normalize(q - x)).
PSDR_D void add_emit(HotAcc& hot, GradAcc* grad_emit, float3 a) {
  if (!grad_emit) return;
  if (hot.emit_hot) { hot.e[0] += a.x; hot.e[1] += a.y; hot.e[2] += a.z; }
  else atomic_add3(grad_emit, a);
}

template <bool EXT>
PSDR_D void add_light_emit(HotAcc& hot, const DevLight& Lt, const Surf& q, float3 ae, SurfAdj& ax) {
  if (!EXT || Lt.kind == kLightArea) {
    add_emit(hot, Lt.grad_emit, ae);
    return;
  }
  const float3 aw = env_emit_adj(&Lt, q.u, q.v, q.wi, ae);
  if (Lt.kind == kLightSh9) ax.p += (aw - q.wi * dot(q.wi, aw)) / sqrtf(q.sqd);
}

PSDR_D void add_vertex(const DevScene& sc, HotAcc& hot, int v, float3 a) {
  if (!sc.grad_verts) return;
  const int rel = v - hot.lv0;
  if (hot.nlv > 0 && rel >= 0 && rel < hot.nlv) {
    // dynamic index: the accumulators live in local memory (L1), which keeps this code
    // short at each of the adjoint's scatter sites
    hot.g[3 * rel] += a.x;
    hot.g[3 * rel + 1] += a.y;
    hot.g[3 * rel + 2] += a.z;
    return;
  }
  vert_add(sc, v, a);
}

// Adjoint of Scene::hit's surface attributes (point, flipped normal and tangent,
// area) w.r.t. the triangle vertices (mesh.cc:27-67; area via |cross|/2, the same
// function as Heron's formula).
static __device__ __noinline__ void surf_vertex_adj(const DevScene& sc, int tri, float b1, float b2, bool front,
                                                    const SurfAdj& a, float3& g0, float3& g1, float3& g2) {
  const float4* r = sc.tri + 6 * (size_t)tri;
  const float4 q0 = __ldg(r), q1 = __ldg(r + 1), q2 = __ldg(r + 2), q3 = __ldg(r + 3), q5 = __ldg(r + 5);
  const float3 p0 = xyz(q0), p1 = xyz(q1), p2 = xyz(q2);
  const float sgn = front ? 1.f : -1.f;
  g0 = a.p * (1.f - b1 - b2);
  g1 = a.p * b1;
  g2 = a.p * b2;
  const float3 c = p1 - p0, b = p0 - p2;
  const float3 cr = cross(c, b);
  const float crn = norm(cr);
  const float3 n = cr / crn;
  const float3 an = a.n * sgn;
  float3 acr = (an - n * dot(n, an)) / crn + n * (0.5f * a.area);
  // tangent
  const float du1y = q5.x - q3.w, du2y = q5.z - q3.w;
  const float3 tw = c * du2y + b * du1y;
  const float twn = norm(tw);
  const float3 t = tw / twn;
  const float3 at = a.t * sgn;
  const float3 atw = (at - t * dot(t, at)) / twn;
  float3 ac = cross(b, acr) + atw * du2y;
  float3 ab = cross(acr, c) + atw * du1y;
  g1 += ac; g0 -= ac;
  g0 += ab; g2 -= ab;
}

PSDR_D void scatter_surf(const DevScene& sc, HotAcc& hot, int tri, float b1, float b2, bool front,
                         const SurfAdj& a) {
  if (!sc.grad_verts) return;
  const int4 tv = __ldg(sc.tri_v + tri);
  if (!vert_wanted(sc, tv.x) && !vert_wanted(sc, tv.y) && !vert_wanted(sc, tv.z)) return;
  float3 g0, g1, g2;
  surf_vertex_adj(sc, tri, b1, b2, front, a, g0, g1, g2);
  add_vertex(sc, hot, tv.x, g0);
  add_vertex(sc, hot, tv.y, g1);
  add_vertex(sc, hot, tv.z, g2);
}

// scatter_surf for a triangle that is not a light's: path vertices past the camera hit
// (paths end at lights), whose vertices never fall in the light-vertex register range.
// Out of line: the adjoint scatters from several depths' call sites.
static __device__ __noinline__ void scatter_mesh(const DevScene& sc, int tri, float b1, float b2, bool front,
                                                 SurfAdj a) {
  if (!sc.grad_verts) return;
  const int4 tv = __ldg(sc.tri_v + tri);
  if (!vert_wanted(sc, tv.x) && !vert_wanted(sc, tv.y) && !vert_wanted(sc, tv.z)) return;
  float3 g0, g1, g2;
  surf_vertex_adj(sc, tri, b1, b2, front, a, g0, g1, g2);
  vert_add(sc, tv.x, g0);
  vert_add(sc, tv.y, g1);
  vert_add(sc, tv.z, g2);
}

PSDR_D void scatter_tex(const DevTex& tx, int off, float3 a, bool /*unused*/) {
  if (!tx.grad) return;
  if (tx.ch == 1) acc_add(tx.grad + off, a.x + a.y + a.z);
  else atomic_add3(tx.grad + off, a);
}

// Adjoint of G = dot(Nx, w) dot(Nq, -w) / d2 with d2 = |q - x|^2, w given.
PSDR_D void geom_adj(float adjG, float3 Nx, float3 Nq, float3 w, float3 xp, float3 qp, float d2, float G,
                     SurfAdj& ax, SurfAdj& aq, float3& adj_w) {
  const float a = dot(Nx, w), bq = -dot(Nq, w);
  const float adj_a = adjG * bq / d2, adj_b = adjG * a / d2, adj_d2 = -adjG * G / d2;
  ax.n += w * adj_a;
  aq.n += w * (-adj_b);
  adj_w = Nx * adj_a - Nq * adj_b;
  const float3 dq = (qp - xp) * (2.f * adj_d2);
  aq.p += dq;
  ax.p -= dq;
}

// Adjoint of wo = normalize(u T + v B + ct N), B = N x T, w.r.t. N and T.
PSDR_D void dir_adj(float3 adj_wo, float3 wo, float3 N, float3 T, float u, float v, float ct, SurfAdj& ax) {
  const float3 B = cross(N, T);
  const float3 m = T * u + B * v + N * ct;
  const float3 am = (adj_wo - wo * dot(wo, adj_wo)) / norm(m);
  const float3 aB = am * v;
  ax.t += am * u + cross(aB, N);
  ax.n += am * ct + cross(T, aB);
}

// ------------------------------------------------------------------ material adjoints
// Material state of a shaded vertex (DiffuseBsdfMaterial, diffuse_bsdf.cc:3-88).
struct MatPt {
  float3 color;  // color texel
  float3 N;      // shading normal
  float3 m;      // normal-map vector 2 texel - 1
  float sigma;   // roughness texel
  bool rough, mapped;
};
PSDR_D MatPt mat_point(const DevObj& ob, const Surf& x) {
  MatPt mp;
  mp.color = tex_rgb(ob.color, texel_offset(ob.color, x.u, x.v));
  mp.rough = ob.mat == kMatDiffuseBsdf;
  mp.N = shading_normal(ob, x, mp.m, mp.mapped);
  mp.sigma = material_sigma(ob, x);
  return mp;
}

// Adjoints gathered at a vertex before they are folded into the surface and textures.
struct MatAdj {
  float3 color, N, V;
  float sigma;
};
PSDR_D MatAdj zero_mat_adj() {
  MatAdj a;
  a.color = a.N = a.V = f3(0.f, 0.f, 0.f);
  a.sigma = 0.f;
  return a;
}

// f = bsdf_value(color, sigma, N, V, L): returns f and accumulates the adjoints of
// color, sigma, N, V (ma) and L (adj_L) for the adjoint adj_f of f.
PSDR_D float3 bsdf_adj(const MatPt& mp, float3 V, float3 L, float3 adj_f, MatAdj& ma, float3& adj_L) {
  if (!mp.rough) {
    ma.color += adj_f * kInvPi;
    return mp.color * kInvPi;
  }
  const float a = 1.0f / (kPi + kOrenC * mp.sigma), b = mp.sigma * a;
  const float nlr = dot(mp.N, L), nvr = dot(mp.N, V);
  const float nl = fmaxf(nlr, 0.f), nv = fmaxf(nvr, 0.f);
  const float t0 = dot(V, L) - nl * nv;
  const float t = t0 > 0.f ? fmaxf(nl, nv) + kEps : t0;
  const float g = a + b * t;
  ma.color += adj_f * g;
  const float adj_g = dot(adj_f, mp.color);
  const float da = -kOrenC * a * a, db = a + mp.sigma * da;
  ma.sigma += adj_g * (da + db * t);
  const float adj_t = adj_g * b;
  float adj_nl = 0.f, adj_nv = 0.f;
  if (t0 > 0.f) {
    if (nl >= nv) adj_nl = adj_t;
    else adj_nv = adj_t;
  } else {
    adj_L += V * adj_t;
    ma.V += L * adj_t;
    adj_nl = -adj_t * nv;
    adj_nv = -adj_t * nl;
  }
  if (nlr >= 0.f) { ma.N += L * adj_nl; adj_L += mp.N * adj_nl; }
  if (nvr >= 0.f) { ma.N += V * adj_nv; ma.V += mp.N * adj_nv; }
  return mp.color * g;
}

// Adjoint of a sampled direction wo = normalize(u T + v B + ct N), B = Ng x T, about
// the shading normal N (its adjoint goes to adjN).
PSDR_D void dir_adj_mat(float3 adj_wo, float3 wo, const Surf& x, float3 N, float u, float v, float ct, SurfAdj& ax,
                        float3& adjN) {
  const float3 B = cross(x.n, x.t);
  const float3 m = x.t * u + B * v + N * ct;
  const float3 am = (adj_wo - wo * dot(wo, adj_wo)) / norm(m);
  const float3 aB = am * v;
  ax.t += am * u + cross(aB, x.n);
  ax.n += cross(x.t, aB);
  adjN += am * ct;
}

// Folds a vertex's material adjoints into its surface adjoint (shading normal through
// the normal map's frame, incoming direction into the point and the ray origin) and
// scatters the roughness and normal-map texel adjoints. Returns the ray origin's adjoint.
PSDR_D float3 mat_finalize(const DevObj& ob, const Surf& x, const MatPt& mp, const MatAdj& ma, SurfAdj& ax) {
  if (mp.mapped) {
    const float3 B = cross(x.n, x.t);
    const float3 nn = x.t * mp.m.x + B * mp.m.y + x.n * mp.m.z;
    const float3 am = (ma.N - mp.N * dot(mp.N, ma.N)) / norm(nn);
    const float3 aB = am * mp.m.y;
    ax.t += am * mp.m.x + cross(aB, x.n);
    ax.n += am * mp.m.z + cross(x.t, aB);
    if (ob.normal.grad)
      atomic_add3(ob.normal.grad + texel_offset(ob.normal, x.u, x.v), f3(dot(am, x.t), dot(am, B), dot(am, x.n)) * 2.f);
  } else {
    ax.n += ma.N;
  }
  if (mp.rough && ob.rough.grad && ma.sigma != 0.f)
    acc_add(ob.rough.grad + texel_offset(ob.rough, x.u, x.v), ma.sigma);
  // V = -normalize(x.p - o)
  const float3 au = (ma.V - x.wi * dot(x.wi, ma.V)) * (-1.f / sqrtf(x.sqd));
  ax.p += au;
  return -au;
}

struct DepthVals {
  float3 C, beta;
  bool has_next;
};

// Adjoint of a BSDF-sampled segment's G in the unbiased estimator: the direction is
// that of the segment's end points, w = normalize(q - x), so it back-propagates into
// both points instead of the sampling frame.
PSDR_D void geom_adj_points(float adjG, const Surf& x, const Surf& q, SurfAdj& ax, SurfAdj& aq,
                            float3 adj_w_extra = f3(0.f, 0.f, 0.f)) {
  const float3 rv = q.p - x.p;
  const float rn = norm(rv);
  const float3 wg = rv / rn;
  const float G = dot(x.n, wg) * (dot(q.n, -wg) / q.sqd);
  float3 adj_w;
  geom_adj(adjG, x.n, q.n, wg, x.p, q.p, q.sqd, G, ax, aq, adj_w);
  adj_w += adj_w_extra;
  const float3 ar = (adj_w - wg * dot(wg, adj_w)) / rn;
  aq.p += ar;
  ax.p -= ar;
}

// One depth of trace2light, recomputed from the sampler stream and the hit records.
// ADJ=false returns the contribution C and the throughput factor beta; ADJ=true
// back-propagates adjC / adjB into the surfaces, the texture, the emission and the
// light vertices (carry = adjoint of the next vertex, passed to the next depth).
// UNB (unbiased estimator): BSDF-sampled segments differentiate G through their end
// points (geom_adj_points); the reference differentiates it through the sampled
// direction's frame.
// BSDF (DiffuseBsdfMaterial in the scene): the BSDF value depends on the shading normal
// (mp), the incoming direction x.wi and the outgoing direction; their adjoints and the
// color / roughness adjoints gather in ma (adj_tex is unused).
template <bool ADJ, bool UNB = false, bool BSDF = false>
PSDR_D DepthVals depth_eval(const WF& w, const DevScene& sc, const Surf& x, Rng& rng, const float4* rec, bool last,
                            float3 adjC, float3 adjB, SurfAdj& ax, SurfAdj& carry, HotAcc& hot, float3& adj_tex,
                            const MatPt* mp = nullptr, MatAdj* ma = nullptr) {
  DepthVals out;
  out.C = f3(0.f, 0.f, 0.f);
  out.beta = f3(0.f, 0.f, 0.f);
  out.has_next = false;
  const float fL = (float)w.nL, fB = (float)w.nB;
  const DevObj& ob = sc.objs[x.obj];
  const float3 tex = tex_rgb(ob.color, texel_offset(ob.color, x.u, x.v));
  const float3 bsdf = tex * kInvPi;
  // DiffuseBsdfMaterial (BSDF): sampling about the shading normal, the value per direction
  const float3 Ns = BSDF ? mp->N : x.n;
  for (int i = 0; i < w.nL; ++i) {
    const float rx = rng.next_float(), ry = rng.next_float();
    const LightSample ls = sample_light(sc, rx, ry);
    const float4 h = rec[i];
    const int tri = __float_as_int(h.x);
    if (tri < 0) continue;
    const float3 rv = ls.y - x.p;
    const float3 dir = normalize(rv);
    const Surf q = make_surf(sc, tri, h.y, h.z, x.p);
    if (!(q.is_light && sqnorm(q.p - ls.y) < kEps)) continue;
    const DevLight& Lt = sc.lights[ls.light];
    const float3 emit = light_emit<BSDF>(Lt, q);
    const float tmp = dot(q.n, -dir) / q.sqd;
    const float G = dot(x.n, dir) * tmp;
    float wgt = 1.0f / fL;
    if (w.nB > 0) wgt *= mis_power(ls.pdf, dot(x.n, dir) * kInvPi * tmp, fL, fB);
    const float k = G / ls.pdf * wgt;
    if (!ADJ) {
      const float3 f = BSDF ? bsdf_value(ob, mp->color, mp->sigma, Ns, x.wi, dir) : bsdf;
      out.C += mul(emit, f) * k;
    } else {
      const float3 av = adjC * wgt;
      const float s_ = G / ls.pdf;
      float3 adjL = f3(0.f, 0.f, 0.f);
      float3 f = bsdf;
      if (BSDF) f = bsdf_adj(*mp, x.wi, dir, mul(av, emit) * s_, *ma, adjL);
      else adj_tex += mul(av, emit) * (s_ * kInvPi);
      const float3 eb = mul(emit, f);
      const float3 ae = mul(av, f) * s_;
      add_light_emit<BSDF>(hot, Lt, q, ae, ax);
      const float adj_gam = dot(av, eb) / ls.pdf;
      SurfAdj aq = zero_adj();
      aq.area = adj_gam * G / q.area;
      float3 adj_dir;
      geom_adj(adj_gam, x.n, q.n, dir, x.p, q.p, q.sqd, G, ax, aq, adj_dir);
      if (BSDF) adj_dir += adjL;
      const float3 ar = (adj_dir - dir * dot(dir, adj_dir)) / norm(rv);
      ax.p -= ar;
      // light sample point y = p0 + (p1-p0) su + (p2-p0) sv
      if (sc.grad_verts) {
        const int4 tv = __ldg(sc.tri_v + ls.tri);
        add_vertex(sc, hot, tv.x, ar * (1.f - ls.su - ls.sv));
        add_vertex(sc, hot, tv.y, ar * ls.su);
        add_vertex(sc, hot, tv.z, ar * ls.sv);
      }
      scatter_surf(sc, hot, tri, h.y, h.z, q.front, aq);
    }
  }
  for (int j = 0; j < w.nB; ++j) {
    const float rx = rng.next_float(), ry = rng.next_float();
    float ct, st, sp, cp;
    const float3 wo = BSDF ? material_dir(x, Ns, rx, ry, ct, st, sp, cp) : diffuse_dir(x.n, x.t, rx, ry, ct, st, sp, cp);
    const float4 h = rec[w.nL + j];
    const int tri = __float_as_int(h.x);
    if (tri < 0) continue;
    const Surf q = make_surf(sc, tri, h.y, h.z, x.p);
    if (!q.is_light) continue;
    const DevLight& Lt = sc.lights[q.light];
    const float3 emit = light_emit<BSDF>(Lt, q);
    const float tmp = dot(q.n, -wo) / q.sqd;
    const float G = dot(x.n, wo) * tmp;
    const float pdf_b = ct * kInvPi * tmp;
    float wgt = 1.0f / fB;
    if (w.nL > 0) wgt *= mis_power(pdf_b, __ldg(sc.light_pmf + q.light) * Lt.inv_area, fB, fL);
    if (!ADJ) {
      const float3 f = BSDF ? bsdf_value(ob, mp->color, mp->sigma, Ns, x.wi, wo) : bsdf;
      out.C += mul(emit, f) * (G / pdf_b * wgt);
    } else {
      const float3 av = adjC * wgt;
      const float s_ = G / pdf_b;
      // the BSDF's outgoing direction: the sampled one, or the segment's (unbiased)
      float3 adjL = f3(0.f, 0.f, 0.f);
      float3 f = bsdf;
      if (BSDF) f = bsdf_adj(*mp, x.wi, UNB ? normalize(q.p - x.p) : wo, mul(av, emit) * s_, *ma, adjL);
      else adj_tex += mul(av, emit) * (s_ * kInvPi);
      const float3 eb = mul(emit, f);
      const float3 ae = mul(av, f) * s_;
      add_light_emit<BSDF>(hot, Lt, q, ae, ax);
      const float adj_gam = dot(av, eb) / pdf_b;
      SurfAdj aq = zero_adj();
      aq.area = adj_gam * G / q.area;
      if (UNB) {
        geom_adj_points(adj_gam, x, q, ax, aq, adjL);
      } else {
        float3 adj_wo;
        geom_adj(adj_gam, x.n, q.n, wo, x.p, q.p, q.sqd, G, ax, aq, adj_wo);
        if (BSDF) dir_adj_mat(adj_wo + adjL, wo, x, Ns, cp * st, sp * st, ct, ax, ma->N);
        else dir_adj(adj_wo, wo, x.n, x.t, cp * st, sp * st, ct, ax);
      }
      scatter_surf(sc, hot, tri, h.y, h.z, q.front, aq);
    }
  }
  {
    const float rx = rng.next_float(), ry = rng.next_float();
    if (!last) {
      float ct, st, sp, cp;
      const float3 wo =
          BSDF ? material_dir(x, Ns, rx, ry, ct, st, sp, cp) : diffuse_dir(x.n, x.t, rx, ry, ct, st, sp, cp);
      const float4 h = rec[w.nL + w.nB];
      const int tri = __float_as_int(h.x);
      if (tri >= 0) {
        out.has_next = true;
        const Surf nx = make_surf(sc, tri, h.y, h.z, x.p);
        const float tmp = dot(nx.n, -wo) / nx.sqd;
        const float G = dot(x.n, wo) * tmp;
        const float pdf = ct * kInvPi * tmp;
        const float s_ = G / pdf;
        if (!ADJ) {
          out.beta = (BSDF ? bsdf_value(ob, mp->color, mp->sigma, Ns, x.wi, wo) : bsdf) * s_;
        } else {
          float3 adjL = f3(0.f, 0.f, 0.f);
          float3 f = bsdf;
          if (BSDF) f = bsdf_adj(*mp, x.wi, UNB ? normalize(nx.p - x.p) : wo, adjB * s_, *ma, adjL);
          else adj_tex += adjB * (s_ * kInvPi);
          const float adj_gam = dot(adjB, f) / pdf;
          carry = zero_adj();
          carry.area = adj_gam * G / nx.area;
          if (UNB) {
            geom_adj_points(adj_gam, x, nx, ax, carry, adjL);
          } else {
            float3 adj_wo;
            geom_adj(adj_gam, x.n, nx.n, wo, x.p, nx.p, nx.sqd, G, ax, carry, adj_wo);
            if (BSDF) dir_adj_mat(adj_wo + adjL, wo, x, Ns, cp * st, sp * st, ct, ax, ma->N);
            else dir_adj(adj_wo, wo, x.n, x.t, cp * st, sp * st, ct, ax);
          }
        }
      }
    }
  }
  return out;
}


// Warp-aggregated scatter of a surface adjoint: reduced over the warp when every
// lane targets the same triangle of the same scene (the spp samples of a pixel).
PSDR_D void scatter_surf_warp(const DevScene* scp, HotAcc& hot, int tri, float b1, float b2, bool front,
                              const SurfAdj& a, bool active) {
  const int t0 = __shfl_sync(0xffffffffu, active ? tri : -1, 0);
  const unsigned long long p0 = __shfl_sync(0xffffffffu, (unsigned long long)scp, 0);
  const bool uni = __all_sync(0xffffffffu, active && tri == t0 && (unsigned long long)scp == p0);
  if (!uni) {
    if (active) scatter_surf(*scp, hot, tri, b1, b2, front, a);
    return;
  }
  if (!scp->grad_verts) return;
  {
    const int4 tv = __ldg(scp->tri_v + tri);
    if (!vert_wanted(*scp, tv.x) && !vert_wanted(*scp, tv.y) && !vert_wanted(*scp, tv.z)) return;
  }
  float3 g0, g1, g2;
  surf_vertex_adj(*scp, tri, b1, b2, front, a, g0, g1, g2);
  float v[9] = {g0.x, g0.y, g0.z, g1.x, g1.y, g1.z, g2.x, g2.y, g2.z};
#pragma unroll
  for (int o = 16; o; o >>= 1)
#pragma unroll
    for (int k = 0; k < 9; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0) {
    const int4 tv = __ldg(scp->tri_v + tri);
    add_vertex(*scp, hot, tv.x, f3(v[0], v[1], v[2]));
    add_vertex(*scp, hot, tv.y, f3(v[3], v[4], v[5]));
    add_vertex(*scp, hot, tv.z, f3(v[6], v[7], v[8]));
  }
}

PSDR_D void scatter_tex_warp(const DevTex* tx, int off, float3 a, bool active) {
  const bool has = active && tx && tx->grad;
  const unsigned long long key = has ? (unsigned long long)(tx->grad + off) : 0ull;
  const unsigned long long k0 = __shfl_sync(0xffffffffu, key, 0);
  const bool uni = __all_sync(0xffffffffu, has && key == k0);
  if (!uni) {
    if (has) scatter_tex(*tx, off, a, false);
    return;
  }
  float v0 = a.x, v1 = a.y, v2 = a.z;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
    v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    v2 += __shfl_xor_sync(0xffffffffu, v2, o);
  }
  if ((threadIdx.x & 31) == 0) scatter_tex(*tx, off, f3(v0, v1, v2), false);
}

// ------------------------------------------------------------------ adjoint kernel
// One thread per path of the tile: the replay stored each depth's contribution C_d
// and throughput factor beta_d, so the suffix radiances S_d = C_d + beta_d S_{d+1}
// come straight from the records; the path is then walked forward once, replaying
// its sampler stream, and every depth's reverse-mode adjoint is applied
// (PSDR_EST_REFERENCE: pdfs and MIS weights are constants, jacobi = area/detach(area),
// barycentrics are not differentiated), scattering into fp64 accumulators.
PSDR_D float3 suffix_radiance(const float4* __restrict__ cb, int from, int D) {
  float3 S = f3(0.f, 0.f, 0.f);
  for (int k = D - 1; k >= from; --k) S = xyz(cb[2 * k]) + mul(xyz(cb[2 * k + 1]), S);
  return S;
}

// Camera-origin adjoint kept in registers while consecutive samples share a view.
struct CamAcc {
  const DevView* v = nullptr;
  float3 g;
  PSDR_D void add(const DevView* view, float3 a) {
    if (view != v) {
      flush();
      v = view;
      g = f3(0.f, 0.f, 0.f);
    }
    g += a;
  }
  PSDR_D void flush() {
    if (v && v->grad_pos && (g.x != 0.f || g.y != 0.f || g.z != 0.f)) atomic_add3(v->grad_pos, g);
    v = nullptr;
  }
  // End of a kernel: one atomic per warp when the warp shares the view.
  PSDR_D void flush_warp() {
    const unsigned long long key = (unsigned long long)v;
    const unsigned long long k0 = __shfl_sync(0xffffffffu, key, 0);
    if (!__all_sync(0xffffffffu, key == k0) || !v) { flush(); return; }
    float3 s = g;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      s.z += __shfl_xor_sync(0xffffffffu, s.z, o);
    }
    if ((threadIdx.x & 31) == 0) { g = s; flush(); }
    v = nullptr;
  }
};

// Viewing direction (camera -z axis in world space) and fx*fy of the map from world
// directions to raster coordinates: the camera's right and up axes are not normalised
// (camera.h:7-40), so c2r's scale is multiplied by the norms of w2c's first two rows.
PSDR_D float3 view_look(const DevView& V) { return f3(-V.c2w[2], -V.c2w[6], -V.c2w[10]); }
PSDR_D float view_fxfy(const DevView& V) {
  const float r0 = sqrtf(V.w2c[0] * V.w2c[0] + V.w2c[1] * V.w2c[1] + V.w2c[2] * V.w2c[2]);
  const float r1 = sqrtf(V.w2c[4] * V.w2c[4] + V.w2c[5] * V.w2c[5] + V.w2c[6] * V.w2c[6]);
  return fabsf(V.c2r[0] * V.c2r[5]) * r0 * r1;
}

// Unbiased estimator, primary vertex: adjoint of the camera Jacobian ratio J/detach(J),
// J = |n.(x-o)| / z^3, z = (x-o).look, scaled by phi = dot(dI, L).
PSDR_D void cam_jacobian_adj(const DevView& V, const Surf& x, float phi, SurfAdj& ax, CamAcc& cam) {
  if (V.ortho) {
    // J = |n.look|: only the normal moves it
    const float3 look = view_look(V);
    ax.n += look * (phi / dot(x.n, look));
    return;
  }
  const float3 rel = x.p - V.pos;
  const float nr = dot(x.n, rel);
  const float3 look = view_look(V);
  const float z = dot(rel, look);
  ax.n += rel * (phi / nr);
  const float3 ap = x.n * (phi / nr) - look * (3.f * phi / z);
  ax.p += ap;
  cam.add(&V, -ap);
}

// BSDF: DiffuseBsdfMaterial in the scene. The incoming direction of a vertex depends on
// the previous vertex (or the camera origin), so a vertex's surface adjoint is scattered
// one depth later.
template <bool UNB, bool BSDF = false>
__global__ void __launch_bounds__(128, BSDF ? 2 : 4) k_adjoint(WF w, const DevScene* __restrict__ scenes,
                                                 const DevView* __restrict__ views, Tile tile, int hot_lv0,
                                                 int hot_nlv, int emit_hot) {
  const int stride = gridDim.x * blockDim.x;
  CamAcc cam;
  const int n32 = (tile.n + 31) & ~31;
  HotAcc hot;
  hot.lv0 = hot_lv0;
  hot.nlv = hot_nlv;
  hot.emit_hot = emit_hot != 0;
#pragma unroll
  for (int k = 0; k < kMaxLightVerts * 3; ++k) hot.g[k] = 0.f;
  hot.e[0] = hot.e[1] = hot.e[2] = 0.f;
  const DevScene* flush_sc = nullptr;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool has0 = false;
    int tri0 = -1;
    float b10 = 0.f, b20 = 0.f;
    bool front0 = true;
    SurfAdj ax0 = zero_adj();
    float3 atex0 = f3(0.f, 0.f, 0.f);
    const DevTex* tx0 = nullptr;
    int toff0 = 0;
    const DevScene* scp = nullptr;
    if (s < tile.n) {
      const DevView& V = views[w.view[s]];
      scp = &scenes[V.scene];
      const float4* rec = w.rec + (size_t)s * w.rec_stride;
      const float4 h0 = rec[0];
      tri0 = __float_as_int(h0.x);
      if (tri0 >= 0 && V.dimage) {
        const DevScene& sc = *scp;
        flush_sc = scp;
        const float* gp = V.dimage + 3 * (size_t)w.pix[s];
        const float3 g = f3(gp[0], gp[1], gp[2]) / (float)V.spp;
        float3 o0 = V.pos;
        if (V.ortho) {
          // the camera ray's origin on the camera plane, as k_camera formed it
          Rng r0 = make_rng((unsigned long long)(tile.begin + s - V.sample_off) + w.seed);
          const float jx = r0.next_float(), jy = r0.next_float();
          const int pix = w.pix[s];
          float3 pc;
          xform_pos(V.r2c, f3(jx + (float)(pix % V.W), jy + (float)(pix / V.W), 1.0f), pc);
          xform_pos(V.c2w, f3(pc.x, pc.y, 0.f), o0);
        }
        const Surf x0 = make_surf(sc, tri0, h0.y, h0.z, o0);
        b10 = h0.y; b20 = h0.z; front0 = x0.front;
        const float4* hits = rec + 1;
        const float4* cb = rec + 1 + (size_t)w.D * w.R;
        if (x0.is_light) {
          // camera ray on a light: L = emit at depth 0 when lights are visible
          if (w.light_vis) {
            const DevLight& Lt = sc.lights[x0.light];
            const float3 L = light_emit<BSDF>(Lt, x0);
            has0 = true;
            ax0.area = dot(g, L) / x0.area;
            if (UNB) cam_jacobian_adj(V, x0, dot(g, L), ax0, cam);
            if (!BSDF || Lt.kind == kLightArea) {
              add_emit(hot, Lt.grad_emit, g);
            } else {
              // an SH9 light's radiance depends on wi = -normalize(x0 - o): its share goes
              // to the ray origin, which moves with the camera
              const float3 aw = env_emit_adj(&Lt, x0.u, x0.v, x0.wi, g);
              if (Lt.kind == kLightSh9) cam.add(&V, (aw - x0.wi * dot(x0.wi, aw)) / sqrtf(x0.sqd));
            }
          }
        } else {
          const float3 L = suffix_radiance(cb, 0, w.D);
          if (finite3(L)) {
            has0 = true;
            const long long i = tile.begin + s - V.sample_off;
            Rng rng = make_rng((unsigned long long)i + w.seed);
            rng.next_float();
            rng.next_float();
            SurfAdj ax = zero_adj();
            ax.area = dot(g, L) / x0.area;  // jacobi of the primary hit
            if (UNB) cam_jacobian_adj(V, x0, dot(g, L), ax, cam);
            Surf xc = x0;
            int tric = tri0;
            float4 hc = h0;
            float3 T = f3(1.f, 1.f, 1.f);
            // BSDF: the surface adjoint of depth d-1 >= 1, scattered after depth d
            SurfAdj axq = zero_adj();
            int triq = -1;
            float4 hq = h0;
            bool frontq = true;
            for (int d = 0; d < w.D; ++d) {
              const float3 adjC = mul(g, T);
              const float3 adjB = mul(adjC, suffix_radiance(cb, d + 1, w.D));
              SurfAdj nextc = zero_adj();
              float3 atx = f3(0.f, 0.f, 0.f);
              const DevObj& ob = sc.objs[xc.obj];
              if (BSDF) {
                const MatPt mp = mat_point(ob, xc);
                MatAdj ma = zero_mat_adj();
                const DepthVals dv = depth_eval<true, UNB, true>(w, sc, xc, rng, hits + (size_t)d * w.R,
                                                                 d == w.D - 1, adjC, adjB, ax, nextc, hot, atx, &mp,
                                                                 &ma);
                atx = ma.color;
                const float3 aorg = mat_finalize(ob, xc, mp, ma, ax);
                if (d == 0) cam.add(&V, aorg);
                else if (d == 1) ax0.p += aorg;
                else axq.p += aorg;
                if (triq >= 0) scatter_mesh(sc, triq, hq.y, hq.z, frontq, axq);
                triq = -1;
                const int off = texel_offset(ob.color, xc.u, xc.v);
                if (d == 0) {
                  ax0 = ax;
                  atex0 = atx;
                  tx0 = &ob.color;
                  toff0 = off;
                } else {
                  if (ob.color.grad) scatter_tex(ob.color, off, atx, false);
                  axq = ax;
                  triq = tric;
                  hq = hc;
                  frontq = xc.front;
                }
                if (!dv.has_next) break;
              } else {
                const DepthVals dv = depth_eval<true, UNB>(w, sc, xc, rng, hits + (size_t)d * w.R, d == w.D - 1,
                                                           adjC, adjB, ax, nextc, hot, atx);
                const int off = texel_offset(ob.color, xc.u, xc.v);
                if (d == 0) {
                  ax0 = ax;
                  atex0 = atx;
                  tx0 = &ob.color;
                  toff0 = off;
                } else {
                  if (ob.color.grad) scatter_tex(ob.color, off, atx, false);
                  scatter_mesh(sc, tric, hc.y, hc.z, xc.front, ax);
                }
                if (!dv.has_next) break;
              }
              T = mul(T, xyz(cb[2 * d + 1]));
              hc = hits[(size_t)d * w.R + w.nL + w.nB];
              tric = __float_as_int(hc.x);
              const float3 org = xc.p;
              xc = make_surf(sc, tric, hc.y, hc.z, org);
              if (xc.is_light) break;  // the path ends on a light: nothing downstream
              ax = nextc;
            }
            if (BSDF && triq >= 0) scatter_mesh(sc, triq, hq.y, hq.z, frontq, axq);
          }
        }
      }
    }
    scatter_surf_warp(scp, hot, tri0, b10, b20, front0, ax0, has0);
    scatter_tex_warp(tx0, toff0, atex0, has0);
  }
  if (UNB || BSDF) cam.flush_warp();
  // flush register accumulators: warp reduce, one atomic per warp
#pragma unroll
  for (int k = 0; k < kMaxLightVerts * 3; ++k) {
    float v = hot.g[k];
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    hot.g[k] = v;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float v = hot.e[k];
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    hot.e[k] = v;
  }
  const unsigned have = __ballot_sync(0xffffffffu, flush_sc != nullptr);
  if (!have) return;
  const unsigned long long addr = __shfl_sync(0xffffffffu, (unsigned long long)flush_sc, __ffs(have) - 1);
  const DevScene* fsc = reinterpret_cast<const DevScene*>(addr);
  if ((threadIdx.x & 31) == 0) {
    if (hot_nlv > 0 && vert_wanted(*fsc, hot_lv0))
      for (int k = 0; k < hot_nlv * 3; ++k)
        if (hot.g[k] != 0.f) acc_add(fsc->grad_verts + 3 * (size_t)hot_lv0 + k, hot.g[k]);
    if (emit_hot && fsc->nlight > 0 && fsc->lights[0].grad_emit)
      for (int k = 0; k < 3; ++k)
        if (hot.e[k] != 0.f) acc_add(fsc->lights[0].grad_emit + k, hot.e[k]);
  }
}

// ------------------------------------------------------------------ hypercube
struct HCube {
  const float* pmf;
  const float* cmf;
  const double* w;    // cell masses (double)
  const double* pre;  // inclusive prefix sums of w
  int ncells;
  int res[3];
  float unit[3];
};

// Unbiased estimator: the cell is the first whose double-precision prefix sum exceeds
// s * total (a float CDF cannot resolve cells below 2^-24 of the mass nor place a sample
// inside them); the caller draws a fresh uniform for the position inside the cell.
PSDR_D int hc_cell_unb(const HCube& hc, float s, double& pmf) {
  const double tot = hc.pre[hc.ncells - 1];
  const double t = (double)s * tot;
  int lo = 0, hi = hc.ncells - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (hc.pre[mid] > t) hi = mid;
    else lo = mid + 1;
  }
  pmf = hc.w[lo] / tot;
  return lo;
}

// ------------------------------------------------------------------ primary edges
// True when triangle tri is one of the faces of the edge with vertices ev.
PSDR_D bool tri_has_edge(const DevScene& sc, int tri, int2 ev) {
  if (tri < 0) return false;
  const int4 tv = __ldg(sc.tri_v + tri);
  return (tv.x == ev.x || tv.y == ev.x || tv.z == ev.x) && (tv.x == ev.y || tv.y == ev.y || tv.z == ev.y);
}

// path_integrator.cc:188-272. PRE=true is the preprocess pass over the hypercube
// cells (sample index = cell, the sampler stream persists across rounds); PRE=false
// samples the cell from the preprocessed mass.
// unb (unbiased estimator, PRE=false): one offset ray must hit a face of the edge
// (foreground); the path of the other side (background, possibly a miss) is traced,
// and eb.hb keeps that background hit with flag 1 (background on the +eps side) or 2.
template <bool PRE>
__global__ void __launch_bounds__(256, 3) k_edge_init(WF w, const DevScene* __restrict__ scenes,
                                                   const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                   long long begin, int n, HCube hc, int round, int unb) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    if (s < n) {
      const long long i = begin + s;
      const DevView& V = views[v];
      const DevScene& sc = scenes[V.scene];
      Rng rng;
      float s1, hpdf = 1.f;
      bool ok = true;
      if (PRE) {
        if (round == 0) rng = make_rng((unsigned long long)i);
        else { rng.state = w.rs[s]; rng.inc = w.ri[s]; }
        s1 = ((float)i + rng.next_float()) * hc.unit[0];
      } else {
        rng = make_rng((unsigned long long)i + w.seed);
        s1 = rng.next_float();
        if (unb) {
          double pm;
          const int cell = hc_cell_unb(hc, s1, pm);
          hpdf = (float)pm;
          ok = pm > 0.0;
          s1 = (rng.next_float() + (float)cell) * hc.unit[0];
        } else {
          const int cell = discrete_sample(hc.pmf, hc.cmf, hc.ncells, s1, hpdf);
          ok = hpdf > 0.f;
          s1 = (s1 + (float)cell) * hc.unit[0];
        }
      }
      const int ne = *sc.n_edges;
      float ss = s1, pe;
      const int e = discrete_sample(sc.edge_pmf, sc.edge_cmf, ne, ss, pe);
      const float4 E0 = __ldg(sc.edge + 4 * (size_t)e), E1 = __ldg(sc.edge + 4 * (size_t)e + 1);
      // ray construction in explicitly rounded ops (bit-identical to the float oracle)
      const float3 p0 = xyz(E0), p1 = xyz(E1);
      const float3 xe = add_rn(p0, scale_rn(sub_rn(p1, p0), ss));
      const float pdf_e = __fdiv_rn(pe, E0.w);
      const float3 pc = xform_pos_rn(V.w2c, xe);
      const float3 pr = xform_pos_rn(V.c2r, pc);
      const int px = (int)floorf(pr.x), py = (int)floorf(pr.y);
      bool valid = ok && pc.z < 0.f && pr.x > 0.f && pr.x < (float)V.W && pr.y > 0.f && pr.y < (float)V.H;
      // camera.h:260-276 / 336-353: the ray through the edge point
      const bool ortho = V.ortho;
      const float3 eo = ortho ? xform_pos_rn(V.c2w, f3(pc.x, pc.y, 0.f)) : V.pos;
      const float3 rd = ortho ? view_look_dir(V) : normalize_rn(sub_rn(xe, V.pos));
      const float3 nrm = cross_rn(rd, normalize_rn(sub_rn(p1, p0)));
      HitRec ha, hb;
      ha.tri = hb.tri = -1;
      ha.b1 = ha.b2 = hb.b1 = hb.b2 = 0.f;
      if (valid) {
        const float3 da = sub_rn(rd, scale_rn(nrm, kEps)), db = add_rn(rd, scale_rn(nrm, kEps));
        const int2 ef = (!PRE && unb) ? __ldg(sc.edge_f + e) : make_int2(kEdgeNonManifold, -1);
        if (ef.x == kEdgeNonManifold) {
          ha = trace_closest(sc, eo, da, kTmin, INFINITY);
          hb = trace_closest(sc, eo, db, kTmin, INFINITY);
        } else {
          // Unbiased silhouette sample: valid only when exactly one offset ray's closest hit
          // is a face of the edge. Test each ray against the edge's faces first (the
          // traversal's test and tie rule): a ray that misses both cannot have one as its
          // closest hit, and for a ray that hits one at t an occlusion query bounded at t
          // decides. Only the other ray of a valid sample needs its full closest hit (its
          // background).
          auto face_hit = [&](float3 d, float& tf) {
            const RayPre rp = ray_pre(eo, d);
            int best = -1;
            tf = INFINITY;
            for (int k = 0; k < 2; ++k) {
              const int f = k == 0 ? ef.x : ef.y;
              if (f < 0) continue;
              const float4* q = sc.tri + 6 * (size_t)f;
              float tt, b1, b2;
              if (tri_test(rp, xyz(__ldg(q)), xyz(__ldg(q + 1)), xyz(__ldg(q + 2)), kTmin, tf, tt, b1, b2) &&
                  (tt < tf || best < 0 || f < best)) {
                tf = tt;
                best = f;
              }
            }
            return best >= 0;
          };
          float tfa, tfb;
          const bool fa = face_hit(da, tfa), fb = face_hit(db, tfb);
          if (fa && fb) {
            // both rays reach the faces: bounded queries decide each ray; only a ray whose
            // face is hidden while the other's is seen needs its full closest hit
            const int2 ev = __ldg(sc.edge_v + e);
            ha = trace_closest(sc, eo, da, kTmin, tfa, tfa);
            hb = trace_closest(sc, eo, db, kTmin, tfb, tfb);
            const bool na = tri_has_edge(sc, ha.tri, ev), nb = tri_has_edge(sc, hb.tri, ev);
            if (na && !nb) hb = trace_closest(sc, eo, db, kTmin, INFINITY);
            else if (nb && !na) ha = trace_closest(sc, eo, da, kTmin, INFINITY);
          } else if (fa) {
            ha = trace_closest(sc, eo, da, kTmin, tfa, tfa);
            if (tri_has_edge(sc, ha.tri, __ldg(sc.edge_v + e))) hb = trace_closest(sc, eo, db, kTmin, INFINITY);
          } else if (fb) {
            hb = trace_closest(sc, eo, db, kTmin, tfb, tfb);
            if (tri_has_edge(sc, hb.tri, __ldg(sc.edge_v + e))) ha = trace_closest(sc, eo, da, kTmin, INFINITY);
          }
        }
      }
      int flag;
      HitRec hcur = ha;
      if (!PRE && unb) {
        const int2 ev = __ldg(sc.edge_v + e);
        const bool na = tri_has_edge(sc, ha.tri, ev), nb = tri_has_edge(sc, hb.tri, ev);
        const HitRec& hg = na ? hb : ha;
        valid = valid && na != nb && hg.tri >= 0;
        flag = valid ? (na ? 1 : 2) : 0;
        hcur = hg;
        eb.hb[s] = make_float4(__int_as_float(hg.tri), hg.b1, hg.b2, __int_as_float(flag));
      } else {
        const Surf a = make_surf(sc, ha.tri, ha.b1, ha.b2, eo);
        const Surf b = make_surf(sc, hb.tri, hb.b1, hb.b2, eo);
        valid = valid && a.valid && b.valid && (norm(a.p - xe) < 10.f * kEps || norm(b.p - xe) < 10.f * kEps);
        flag = valid ? 1 : 0;
        eb.hb[s] = make_float4(__int_as_float(hb.tri), hb.b1, hb.b2, __int_as_float(flag));
      }
      eb.a[s] = make_float4(__int_as_float(e), ss, pdf_e, hpdf);
      eb.n[s] = make_float4(nrm.x, nrm.y, nrm.z, __int_as_float(py * V.W + px));
      w.rs[s] = rng.state;
      w.ri[s] = rng.inc;
      w.view[s] = v;
      w.T[s] = make_float4(1.f, 1.f, 1.f, 0.f);
      w.L[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      w.cur[s] = hit4(hcur);
      w.org[s] = make_float4(eo.x, eo.y, eo.z, 0.f);
      eb.La[s] = w.org[s];  // the ray origin, for the second path (k_edge_mid)
      alive = valid;
    }
    const int k = warp_append(&w.cnt[0], alive);
    if (alive) w.q0[k] = s;
  }
}

// Unbiased silhouette term: -sgn L_bg K (d_rel . n) with d_rel = (dx_e - do) -
// (r_e / r_bg)(dx_bg - do), K = fx fy r_e / z_e^3 / (pdf_e hc_density H W spp); the
// background point moves with its triangle, the edge point with the edge's vertices.
__global__ void __launch_bounds__(256) k_edge_final_unb(WF w, const DevScene* __restrict__ scenes,
                                                        const DevView* __restrict__ views, int v, EdgeBuf eb, int n,
                                                        float cells, int spp) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  const float3 look = view_look(V);
  const float fxfy = view_fxfy(V);
  float3 go = f3(0.f, 0.f, 0.f);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= n || !V.dimage) continue;
    const float4 hg = eb.hb[s];
    const int flag = __float_as_int(hg.w);
    if (flag == 0) continue;
    const float4 a = eb.a[s], nn = eb.n[s];
    const float* gp = V.dimage + 3 * (size_t)__float_as_int(nn.w);
    const float3 L = xyz(w.L[s]);
    const float phi = gp[0] * L.x + gp[1] * L.y + gp[2] * L.z;
    if (!(phi != 0.f) || !isfinite(phi)) continue;
    const int e = __float_as_int(a.x);
    const float ss = a.y;
    const float4 E0 = __ldg(sc.edge + 4 * (size_t)e), E1 = __ldg(sc.edge + 4 * (size_t)e + 1);
    const float3 xe = add_rn(xyz(E0), scale_rn(sub_rn(xyz(E1), xyz(E0)), ss));
    const float3 re3 = xe - V.pos;
    const float re = norm(re3), z = dot(re3, look);
    const int tri = __float_as_int(hg.x);
    const Surf g = make_surf(sc, tri, hg.y, hg.z, V.pos);
    // orthographic: no depth scaling, and a camera translation moves both points alike
    const float ratio = V.ortho ? 1.f : re / sqrtf(g.sqd);
    const float K = fxfy * (V.ortho ? 1.f : re / (z * z * z)) / (a.z * a.w * cells * (float)V.H * (float)V.W *
                                                                  (float)spp);
    const float3 av = xyz(nn) * (-(flag == 1 ? 1.f : -1.f) * phi * K);
    if (!finite3(av)) continue;
    if (sc.grad_verts) {
      const int2 ev = __ldg(sc.edge_v + e);
      vert_add(sc, ev.x, av * (1.f - ss));
      vert_add(sc, ev.y, av * ss);
      const int4 tv = __ldg(sc.tri_v + tri);
      const float3 ag = av * (-ratio);
      vert_add(sc, tv.x, ag * (1.f - hg.y - hg.z));
      vert_add(sc, tv.y, ag * hg.y);
      vert_add(sc, tv.z, ag * hg.z);
    }
    go -= av * (1.f - ratio);
  }
  if (V.grad_pos) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      go.x += __shfl_xor_sync(0xffffffffu, go.x, o);
      go.y += __shfl_xor_sync(0xffffffffu, go.y, o);
      go.z += __shfl_xor_sync(0xffffffffu, go.z, o);
    }
    if ((threadIdx.x & 31) == 0 && (go.x != 0.f || go.y != 0.f || go.z != 0.f)) atomic_add3(V.grad_pos, go);
  }
}

// Between the two trace2light calls: keep L_a, restart the slot at the +eps hit with
// the sampler stream continuing where the first path left it.
__global__ void __launch_bounds__(256) k_edge_mid(WF w, const DevView* __restrict__ views, int v, EdgeBuf eb, int n) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    if (s < n) {
      const float4 hb = eb.hb[s];
      alive = __float_as_int(hb.w) != 0;
      if (alive) {
        const float4 eo = eb.La[s];  // the ray origin k_edge_init left there
        eb.La[s] = w.L[s];
        w.T[s] = make_float4(1.f, 1.f, 1.f, 0.f);
        w.L[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        w.cur[s] = make_float4(hb.x, hb.y, hb.z, 0.f);
        w.org[s] = eo;
      }
    }
    const int k = warp_append(&w.cnt[0], alive);
    if (alive) w.q0[k] = s;
  }
}

// PRE: mass[cell] += |dL / pdf_e|. Otherwise the gradient of the zero-valued term
// (x_e - detach(x_e)).n + (o - detach(o)).(n*[1,1,-1]) times dL / pdf_e / pdf_hc / spp.
template <bool PRE>
__global__ void __launch_bounds__(256) k_edge_final(WF w, const DevScene* __restrict__ scenes,
                                                    const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                    long long begin, int n, float* mass, int spp) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  float3 go = f3(0.f, 0.f, 0.f);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= n) continue;
    const float4 hb = eb.hb[s];
    if (__float_as_int(hb.w) == 0) continue;
    const float3 La = xyz(eb.La[s]), Lb = xyz(w.L[s]);
    const float3 dL = sub_rn(La, Lb);
    const float4 a = eb.a[s];
    const float pdf_e = a.z;
    if (PRE) {
      const float3 val = f3(__fdiv_rn(dL.x, pdf_e), __fdiv_rn(dL.y, pdf_e), __fdiv_rn(dL.z, pdf_e));
      if (finite3(val)) mass[begin + s] = __fadd_rn(mass[begin + s], norm_rn(val));
    } else {
      if (!finite3(dL * 0.0f)) continue;
      const float4 nn = eb.n[s];
      const int pix = __float_as_int(nn.w);
      if (!V.dimage) continue;
      const float* gp = V.dimage + 3 * (size_t)pix;
      const float K = (gp[0] * dL.x + gp[1] * dL.y + gp[2] * dL.z) / (pdf_e * a.w * (float)spp);
      const float3 nrm = xyz(nn);
      // x_dot_n = (x_e - detach(x_e)).n + (o - detach(o)).nflip; an orthographic ray's
      // origin o is x_e's foot on the camera plane and moves with x_e as well
      const float3 nflip = f3(nrm.x, nrm.y, -nrm.z);
      const float3 jo = V.ortho ? ortho_origin_jt(V, nflip) : f3(0.f, 0.f, 0.f);
      const float3 ax = (nrm + jo) * K;
      const int e = __float_as_int(a.x);
      const float ss = a.y;
      if (sc.grad_verts) {
        const int2 ev = __ldg(sc.edge_v + e);
        vert_add(sc, ev.x, ax * (1.f - ss));
        vert_add(sc, ev.y, ax * ss);
      }
      go += (nflip - jo) * K;
    }
  }
  if (!PRE && V.grad_pos) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      go.x += __shfl_xor_sync(0xffffffffu, go.x, o);
      go.y += __shfl_xor_sync(0xffffffffu, go.y, o);
      go.z += __shfl_xor_sync(0xffffffffu, go.z, o);
    }
    if ((threadIdx.x & 31) == 0 && (go.x != 0.f || go.y != 0.f || go.z != 0.f)) atomic_add3(V.grad_pos, go);
  }
}

// ------------------------------------------------------------------ pixel borders
// Unbiased estimator: material crossing the pixel borders. The border segments are the
// (W+1) x H vertical and W x (H+1) horizontal unit segments of the pixel grid; segment q
// contributes (dI[hi] - dI[lo]) . Int L v dl, L the radiance seen through the border
// point and v the raster velocity of its primary vertex across the segment (material
// flows into pixel hi and out of pixel lo; outside the image dI = 0). Segments are
// importance-sampled by m_q = |dI[hi] - dI[lo]|_1 (zero where the term is zero) with
// stratified inversion of the double-precision CDF: sample i of N takes
// u = (i + xi) / N, its segment is the first with prefix > u * total and its position
// along the segment the remainder, so every segment gets N m_q / total samples spread
// evenly along it.
PSDR_D void border_pixels(const DevView& V, long long q, bool& vert, int& k, int& j, int& lo, int& hi) {
  const long long nv = (long long)(V.W + 1) * V.H;
  vert = q < nv;
  lo = hi = -1;
  if (vert) {
    k = (int)(q % (V.W + 1));
    j = (int)(q / (V.W + 1));
    if (k >= 1) lo = j * V.W + k - 1;
    if (k < V.W) hi = j * V.W + k;
  } else {
    const long long r = q - nv;
    k = (int)(r % V.W);
    j = (int)(r / V.W);
    if (j >= 1) lo = (j - 1) * V.W + k;
    if (j < V.H) hi = j * V.W + k;
  }
}

PSDR_D float3 dimage_at(const DevView& V, int p) {
  if (p < 0) return f3(0.f, 0.f, 0.f);
  const float* g = V.dimage + 3 * (size_t)p;
  return f3(g[0], g[1], g[2]);
}

__global__ void k_border_mass(const DevView* __restrict__ views, int v, float* __restrict__ mass, long long S) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= S) return;
  const DevView& V = views[v];
  bool vert;
  int k, j, lo, hi;
  border_pixels(V, q, vert, k, j, lo, hi);
  const float3 d = dimage_at(V, hi) - dimage_at(V, lo);
  mass[q] = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
}

// Segment and position of border sample i of N (explicitly rounded double arithmetic,
// identical in the oracle).
PSDR_D long long border_locate(const double* __restrict__ w, const double* __restrict__ pre, long long S,
                               long long i, long long N, float xi, float& t, double& pmf) {
  const double tot = pre[S - 1];
  const double u = __ddiv_rn(__dadd_rn((double)i, (double)xi), (double)N);
  const double tt = __dmul_rn(u, tot);
  long long lo = 0, hi = S - 1;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (pre[mid] > tt) hi = mid;
    else lo = mid + 1;
  }
  const double base = lo > 0 ? pre[lo - 1] : 0.0;
  double r = __ddiv_rn(__dsub_rn(tt, base), w[lo]);
  r = r < 0.0 ? 0.0 : r;
  t = fminf((float)r, 0.99999994f);
  pmf = __ddiv_rn(w[lo], tot);
  return lo;
}

__global__ void __launch_bounds__(256) k_border_init(WF w, const DevScene* __restrict__ scenes,
                                                     const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                     const double* __restrict__ mw, const double* __restrict__ mpre,
                                                     long long S, long long begin, int n, long long N) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    if (s < n) {
      const long long i = begin + s;
      const DevView& V = views[v];
      const DevScene& sc = scenes[V.scene];
      Rng rng = make_rng((unsigned long long)i + w.seed);
      const float xi = rng.next_float();
      float t;
      double pmf;
      const long long q = border_locate(mw, mpre, S, i, N, xi, t, pmf);
      bool vert;
      int k, j, lo, hi;
      border_pixels(V, q, vert, k, j, lo, hi);
      const float3 fp = vert ? f3((float)k, t + (float)j, 1.0f) : f3(t + (float)k, (float)j, 1.0f);
      float3 pc;
      xform_pos(V.r2c, fp, pc);
      float3 o = V.pos, d;
      if (V.ortho) {
        xform_pos(V.c2w, f3(pc.x, pc.y, 0.f), o);
        d = view_look_dir(V);
      } else {
        d = normalize(xform_dir(V.c2w, pc));
      }
      const HitRec h = trace_closest(sc, o, d, kTmin, INFINITY);
      w.rs[s] = rng.state;
      w.ri[s] = rng.inc;
      w.view[s] = v;
      w.pix[s] = -1;
      w.T[s] = make_float4(1.f, 1.f, 1.f, 0.f);
      w.L[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      w.cur[s] = hit4(h);
      w.org[s] = make_float4(o.x, o.y, o.z, 0.f);
      eb.hb[s] = hit4(h);
      eb.a[s] = make_float4(__int_as_float((int)q), t, (float)pmf, 0.f);
      alive = h.tri >= 0 && pmf > 0.0;
    }
    const int k = warp_append(&w.cnt[0], alive);
    if (alive) w.q0[k] = s;
  }
}

__global__ void __launch_bounds__(256) k_border_final(WF w, const DevScene* __restrict__ scenes,
                                                      const DevView* __restrict__ views, int v, EdgeBuf eb, int n,
                                                      long long N) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  float3 go = f3(0.f, 0.f, 0.f);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= n || !V.dimage) continue;
    const float4 h = eb.hb[s];
    const int tri = __float_as_int(h.x);
    if (tri < 0) continue;
    const float4 a = eb.a[s];
    if (!(a.z > 0.f)) continue;
    bool vert;
    int k, j, lo, hi;
    border_pixels(V, __float_as_int(a.x), vert, k, j, lo, hi);
    const float3 L = xyz(w.L[s]);
    const float3 dg = dimage_at(V, hi) - dimage_at(V, lo);
    const float wgt = dot(dg, L) / ((float)N * a.z);
    if (!(wgt != 0.f) || !isfinite(wgt)) continue;
    // raster coordinate c (x for vertical borders, y for horizontal) of the material
    // point and its gradient w.r.t. the point
    const Surf x = make_surf(sc, tri, h.y, h.z, V.pos);
    float3 pc;
    xform_pos(V.w2c, x.p, pc);
    const float* m = V.c2r;
    const int c = vert ? 0 : 1;
    const float wden = m[12] * pc.x + m[13] * pc.y + m[14] * pc.z + m[15];
    const float u = (m[4 * c] * pc.x + m[4 * c + 1] * pc.y + m[4 * c + 2] * pc.z + m[4 * c + 3]) / wden;
    const float3 gpc = f3(m[4 * c] - u * m[12], m[4 * c + 1] - u * m[13], m[4 * c + 2] - u * m[14]) / wden;
    const float* r = V.w2c;
    const float3 gx = f3(r[0] * gpc.x + r[4] * gpc.y + r[8] * gpc.z, r[1] * gpc.x + r[5] * gpc.y + r[9] * gpc.z,
                         r[2] * gpc.x + r[6] * gpc.y + r[10] * gpc.z);
    const float3 ag = gx * wgt;
    if (!finite3(ag)) continue;
    if (sc.grad_verts) {
      const int4 tv = __ldg(sc.tri_v + tri);
      vert_add(sc, tv.x, ag * (1.f - h.y - h.z));
      vert_add(sc, tv.y, ag * h.y);
      vert_add(sc, tv.z, ag * h.z);
    }
    go -= ag;
  }
  if (V.grad_pos) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      go.x += __shfl_xor_sync(0xffffffffu, go.x, o);
      go.y += __shfl_xor_sync(0xffffffffu, go.y, o);
      go.z += __shfl_xor_sync(0xffffffffu, go.z, o);
    }
    if ((threadIdx.x & 31) == 0 && (go.x != 0.f || go.y != 0.f || go.z != 0.f)) atomic_add3(V.grad_pos, go);
  }
}

// ------------------------------------------------------------------ camera lens
// Unbiased estimator, perspective views: derivative of the image with respect to the
// camera's basis and field of view (look_at, up, fov, and look_from through the basis).
// With the camera origin fixed, the world direction seen at raster point u (taken from
// the image centre) is M [u; 1], M = C diag(2 tan(fov/2) / W, -2 tan(fov/2) / H, -1), C the
// camera basis (right, up, dir) of camera.h:35-52. A change dM moves the image content
// with the raster velocity V(u) = (h_3 u_x - h_1, h_3 u_y - h_2), h = G [u; 1],
// G = M^-1 dM. A box-filtered pixel then changes by the content flowing in across its
// borders (the integral the pixel-border samples estimate, with V in place of the
// material point's raster velocity) plus Int_P L div V du, where
// div V = 3 (G_31 u_x + G_32 u_y) + 2 G_33 - G_11 - G_22.
// Per view: grad_lens[0..2] = sum over camera samples of g.L {1, u_x, u_y} / spp (g the
// pixel's dPhi/dI), grad_lens[3..11] = dPhi/dG of the border part (row-major 3x3).
struct LensAcc {
  const DevView* v = nullptr;
  float s0 = 0.f, sx = 0.f, sy = 0.f;
  PSDR_D void add(const DevView* view, float gl, float ux, float uy) {
    if (view != v) {
      flush();
      v = view;
      s0 = sx = sy = 0.f;
    }
    s0 += gl;
    sx += gl * ux;
    sy += gl * uy;
  }
  PSDR_D void flush() {
    if (v && v->grad_lens && (s0 != 0.f || sx != 0.f || sy != 0.f)) {
      acc_add(v->grad_lens, s0);
      acc_add(v->grad_lens + 1, sx);
      acc_add(v->grad_lens + 2, sy);
    }
    v = nullptr;
  }
  PSDR_D void flush_warp() {
    const unsigned long long key = (unsigned long long)v;
    const unsigned long long k0 = __shfl_sync(0xffffffffu, key, 0);
    if (!__all_sync(0xffffffffu, key == k0) || !v) { flush(); return; }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      sx += __shfl_xor_sync(0xffffffffu, sx, o);
      sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if ((threadIdx.x & 31) == 0) flush();
    v = nullptr;
  }
};

// Interior moments from the replay records of a tile (after its adjoint): the sample's
// radiance is the film's value (the emission of a visible light, or the path's suffix
// radiance from depth 0); its raster position replays the two jitter draws of k_camera.
template <bool BSDF>
__global__ void __launch_bounds__(256) k_lens_interior(WF w, const DevScene* __restrict__ scenes,
                                                       const DevView* __restrict__ views, Tile tile) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (tile.n + 31) & ~31;
  LensAcc acc;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= tile.n) continue;
    const DevView& V = views[w.view[s]];
    if (!V.grad_lens || !V.dimage) continue;
    const float4* rec = w.rec + (size_t)s * w.rec_stride;
    const float4 h0 = rec[0];
    const int tri0 = __float_as_int(h0.x);
    if (tri0 < 0) continue;
    const DevScene& sc = scenes[V.scene];
    const Surf x0 = make_surf(sc, tri0, h0.y, h0.z, V.pos);
    float3 L;
    if (x0.is_light) {
      if (!w.light_vis) continue;
      L = light_emit<BSDF>(sc.lights[x0.light], x0);
    } else {
      L = suffix_radiance(rec + 1 + (size_t)w.D * w.R, 0, w.D);
    }
    if (!finite3(L)) continue;
    const int pix = w.pix[s];
    const float* gp = V.dimage + 3 * (size_t)pix;
    const float gl = (gp[0] * L.x + gp[1] * L.y + gp[2] * L.z) / (float)V.spp;
    Rng rng = make_rng((unsigned long long)(tile.begin + s - V.sample_off) + w.seed);
    const float jx = rng.next_float(), jy = rng.next_float();
    acc.add(&V, gl, jx + (float)(pix % V.W) - 0.5f * (float)V.W, jy + (float)(pix / V.W) - 0.5f * (float)V.H);
  }
  acc.flush_warp();
}

// Border part from the pixel-border samples of view v (after k_border_final): the
// sample's weight times dV_c/dG at its raster point, c the coordinate across the border.
__global__ void __launch_bounds__(256) k_lens_border(WF w, const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                     int n, long long N) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const DevView& V = views[v];
  float b0 = 0.f, b1 = 0.f, b2 = 0.f, b3 = 0.f, b4 = 0.f, b5 = 0.f, b6 = 0.f, b7 = 0.f, b8 = 0.f;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= n || !V.dimage || !V.grad_lens) continue;
    if (__float_as_int(eb.hb[s].x) < 0) continue;  // the border ray left the scene: no radiance
    const float4 a = eb.a[s];
    if (!(a.z > 0.f)) continue;
    bool vert;
    int k, j, lo, hi;
    border_pixels(V, __float_as_int(a.x), vert, k, j, lo, hi);
    const float3 L = xyz(w.L[s]);
    const float3 dg = dimage_at(V, hi) - dimage_at(V, lo);
    const float wgt = dot(dg, L) / ((float)N * a.z);
    if (!(wgt != 0.f) || !isfinite(wgt)) continue;
    const float ux = (vert ? (float)k : a.y + (float)k) - 0.5f * (float)V.W;
    const float uy = (vert ? a.y + (float)j : (float)j) - 0.5f * (float)V.H;
    const float wc = wgt * (vert ? ux : uy);
    if (vert) { b0 -= wgt * ux; b1 -= wgt * uy; b2 -= wgt; }
    else { b3 -= wgt * ux; b4 -= wgt * uy; b5 -= wgt; }
    b6 += wc * ux;
    b7 += wc * uy;
    b8 += wc;
  }
  float b[9] = {b0, b1, b2, b3, b4, b5, b6, b7, b8};
#pragma unroll
  for (int o = 16; o; o >>= 1)
#pragma unroll
    for (int m = 0; m < 9; ++m) b[m] += __shfl_xor_sync(0xffffffffu, b[m], o);
  if ((threadIdx.x & 31) == 0 && V.grad_lens) {
#pragma unroll
    for (int m = 0; m < 9; ++m)
      if (b[m] != 0.f) acc_add(V.grad_lens + 3 + m, b[m]);
  }
}

// dPhi/dtheta_j = <Gamma, P_j>, Gamma = B + the interior part of dPhi/dG.
__global__ void k_lens_out(const GradAcc* __restrict__ acc, LensChain ch, float* __restrict__ out, int accumulate) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double G[9];
  for (int m = 0; m < 9; ++m) G[m] = acc_value(acc[3 + m].hi, acc[3 + m].lo);
  const double s0 = acc_value(acc[0].hi, acc[0].lo), sx = acc_value(acc[1].hi, acc[1].lo),
               sy = acc_value(acc[2].hi, acc[2].lo);
  G[0] -= s0;
  G[4] -= s0;
  G[6] += 3.0 * sx;
  G[7] += 3.0 * sy;
  G[8] += 2.0 * s0;
  for (int j = 0; j < 10; ++j) {
    double d = 0.0;
    for (int m = 0; m < 9; ++m) d += G[m] * ch.P[j][m];
    out[j] = accumulate ? out[j] + (float)d : (float)d;
  }
}

// ------------------------------------------------------------------ interpenetration creases
// Unbiased estimator: where the surfaces of two different meshes cut into each other (a
// noisy icosphere sunk into the ground), the visible surface switches from one mesh to the
// other along their intersection curve. That curve is not a mesh edge, so neither the
// silhouette nor the shadow-boundary samples see it; it moves when either mesh moves. Its
// term (primary visibility): with surface 1 seen on one side of the projected curve and
// surface 2 on the other, n the raster normal from 1 to 2, the image changes by
//   Int_curve g [L1 (v_c - v_1) - L2 (v_c - v_2)] . n dl
// (raster velocities: v_c of the curve, v_k of surface k's material point at it). With
// J = d(raster)/d(world), w = J^T n, c = n1.n2 and the curve's world velocity taken in the
// plane of the two normals (it stays on both surfaces), the adjoint of surface k's material
// point is K [(G1 - G2) A_k n_k -+ G_k w] (minus for 1), A_1 = (w.n1 - c w.n2) / (1 - c^2),
// A_2 = (w.n2 - c w.n1) / (1 - c^2), G_k = g . L_k, K = raster length per sample.
constexpr int kCreaseCap = 16384;          // intersection segments kept per scene
constexpr int kCreaseSamplesPerSpp = 16384;  // crease samples per primary-edge spp
constexpr unsigned long long kCreaseStream = 0xC0000000ull;  // sampler streams of the crease samples

// Meshes whose boxes the crease extraction keeps (a triangle of a mesh beyond this many
// walks the tree without the box test).
constexpr int kCreaseBoxObjs = 4096;

struct CreaseBuf {
  float4* a;   // segment start xyz, length (ordered by the triangle pair)
  float4* b;   // segment end xyz, -
  int2* tris;  // the two triangles (different meshes)
  float4* ra;  // the same, in the order the extraction found them
  float4* rb;
  int2* rtris;
  int* count;  // segments found (may exceed kCreaseCap: the rest are dropped)
  int* obox;   // per mesh: its box (min xyz, max xyz as order-preserving ints), kCreaseBoxObjs
  int* later;  // per mesh m: the box of meshes m+1 .. (the ones its triangles are tested against)
};

// Order-preserving int image of a float (for atomicMin / atomicMax on boxes).
PSDR_D int f2ord(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
PSDR_D float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_crease_box_init(const DevScene* __restrict__ scenes, int si, CreaseBuf cb) {
  const int n = min(scenes[si].nobj, kCreaseBoxObjs);
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n; o += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      cb.obox[6 * o + k] = 0x7fffffff;
      cb.obox[6 * o + 3 + k] = (int)0x80000000;
    }
}

// Box of every mesh (lights excluded): one thread per triangle, reduced over the warp when
// its triangles belong to one mesh (meshes are contiguous ranges of triangles).
__global__ void k_crease_boxes(const DevScene* __restrict__ scenes, int si, CreaseBuf cb) {
  const DevScene& sc = scenes[si];
  const int nmesh = min(sc.nobj - sc.nlight, kCreaseBoxObjs);
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (sc.ntri + 31) & ~31;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n32; t += stride) {
    int o = -1;
    int v[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000, (int)0x80000000, (int)0x80000000};
    if (t < sc.ntri) {
      o = __ldg(sc.tri_v + t).w;
      if (o < nmesh) {
        const float4* R = sc.tri + 6 * (size_t)t;
        const float3 p0 = xyz(__ldg(R)), p1 = xyz(__ldg(R + 1)), p2 = xyz(__ldg(R + 2));
        v[0] = f2ord(fminf(p0.x, fminf(p1.x, p2.x)));
        v[1] = f2ord(fminf(p0.y, fminf(p1.y, p2.y)));
        v[2] = f2ord(fminf(p0.z, fminf(p1.z, p2.z)));
        v[3] = f2ord(fmaxf(p0.x, fmaxf(p1.x, p2.x)));
        v[4] = f2ord(fmaxf(p0.y, fmaxf(p1.y, p2.y)));
        v[5] = f2ord(fmaxf(p0.z, fmaxf(p1.z, p2.z)));
      } else {
        o = -1;
      }
    }
    const int o0 = __shfl_sync(0xffffffffu, o, 0);
    if (__all_sync(0xffffffffu, o == o0)) {
      if (o0 < 0) continue;
      for (int k = 0; k < 3; ++k) {
        const int mn = __reduce_min_sync(0xffffffffu, v[k]);
        const int mx = __reduce_max_sync(0xffffffffu, v[3 + k]);
        if ((threadIdx.x & 31) == 0) {
          atomicMin(cb.obox + 6 * o0 + k, mn);
          atomicMax(cb.obox + 6 * o0 + 3 + k, mx);
        }
      }
    } else if (o >= 0) {
      for (int k = 0; k < 3; ++k) {
        atomicMin(cb.obox + 6 * o + k, v[k]);
        atomicMax(cb.obox + 6 * o + 3 + k, v[3 + k]);
      }
    }
  }
}

// later[m] = union of the boxes of meshes m+1 .. nmesh-1 (empty for the last).
__global__ void k_crease_later(const DevScene* __restrict__ scenes, int si, CreaseBuf cb) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const DevScene& sc = scenes[si];
  const int nmesh = min(sc.nobj - sc.nlight, kCreaseBoxObjs);
  int u[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int m = nmesh - 1; m >= 0; --m) {
    for (int k = 0; k < 6; ++k) cb.later[6 * m + k] = u[k];
    for (int k = 0; k < 3; ++k) {
      u[k] = min(u[k], cb.obox[6 * m + k]);
      u[3 + k] = max(u[3 + k], cb.obox[6 * m + 3 + k]);
    }
  }
}

// The segment where triangles a and b cross (false when they do not, or are coplanar).
// Double precision; a vertex exactly on the other plane counts as on its positive side.
PSDR_D bool tri_tri_segment(const double3* A, const double3* B, double3& s0, double3& s1) {
  auto sub = [](double3 p, double3 q) { return make_double3(p.x - q.x, p.y - q.y, p.z - q.z); };
  auto dotd = [](double3 p, double3 q) { return p.x * q.x + p.y * q.y + p.z * q.z; };
  auto crs = [](double3 p, double3 q) {
    return make_double3(p.y * q.z - p.z * q.y, p.z * q.x - p.x * q.z, p.x * q.y - p.y * q.x);
  };
  // the two points where triangle T's edges cross the plane (n, d); false if none
  auto cut = [&](const double3* T, double3 n, double d, double3& p, double3& q) {
    double s[3];
    for (int k = 0; k < 3; ++k) s[k] = dotd(n, T[k]) + d;
    const bool pos0 = s[0] >= 0.0, pos1 = s[1] >= 0.0, pos2 = s[2] >= 0.0;
    if (pos0 == pos1 && pos1 == pos2) return false;
    // the lone vertex on its side
    const int k = (pos0 != pos1 && pos0 != pos2) ? 0 : (pos1 != pos0 && pos1 != pos2) ? 1 : 2;
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const double ti = s[k] / (s[k] - s[i]), tj = s[k] / (s[k] - s[j]);
    p = make_double3(T[k].x + (T[i].x - T[k].x) * ti, T[k].y + (T[i].y - T[k].y) * ti, T[k].z + (T[i].z - T[k].z) * ti);
    q = make_double3(T[k].x + (T[j].x - T[k].x) * tj, T[k].y + (T[j].y - T[k].y) * tj, T[k].z + (T[j].z - T[k].z) * tj);
    return true;
  };
  const double3 na = crs(sub(A[1], A[0]), sub(A[2], A[0])), nb = crs(sub(B[1], B[0]), sub(B[2], B[0]));
  const double3 D = crs(na, nb);
  const double dd = dotd(D, D);
  if (!(dd > 1e-30 * dotd(na, na) * dotd(nb, nb))) return false;
  double3 pa, qa, pb, qb;
  if (!cut(A, nb, -dotd(nb, B[0]), pa, qa) || !cut(B, na, -dotd(na, A[0]), pb, qb)) return false;
  double ta0 = dotd(pa, D), ta1 = dotd(qa, D), tb0 = dotd(pb, D), tb1 = dotd(qb, D);
  if (ta0 > ta1) { const double t = ta0; ta0 = ta1; ta1 = t; const double3 x = pa; pa = qa; qa = x; }
  if (tb0 > tb1) { const double t = tb0; tb0 = tb1; tb1 = t; const double3 x = pb; pb = qb; qb = x; }
  const double lo = fmax(ta0, tb0), hi = fmin(ta1, tb1);
  if (!(lo < hi)) return false;
  s0 = ta0 >= tb0 ? pa : pb;
  s1 = ta1 <= tb1 ? qa : qb;
  return true;
}

// One thread per triangle of a mesh: the LBVH is walked with the triangle's box, and every
// triangle of a later mesh (lights excluded) that it crosses adds one segment.
__global__ void __launch_bounds__(128) k_crease_pairs(const DevScene* __restrict__ scenes, int si, CreaseBuf cb) {
  const DevScene& sc = scenes[si];
  const int nmesh = sc.nobj - sc.nlight;
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < sc.ntri; t += stride) {
    const int4 tv = __ldg(sc.tri_v + t);
    if (tv.w >= nmesh || sc.root == 0x7fffffff) continue;
    const float4* R = sc.tri + 6 * (size_t)t;
    const float3 p0 = xyz(__ldg(R)), p1 = xyz(__ldg(R + 1)), p2 = xyz(__ldg(R + 2));
    const float3 lo = f3(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)), fminf(p0.z, fminf(p1.z, p2.z)));
    const float3 hi = f3(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)), fmaxf(p0.z, fmaxf(p1.z, p2.z)));
    if (tv.w < kCreaseBoxObjs) {
      // a triangle clear of every later mesh's box crosses none of its triangles
      const int* L = cb.later + 6 * tv.w;
      if (__ldg(L) == 0x7fffffff || ord2f(__ldg(L)) > hi.x || ord2f(__ldg(L + 3)) < lo.x || ord2f(__ldg(L + 1)) > hi.y ||
          ord2f(__ldg(L + 4)) < lo.y || ord2f(__ldg(L + 2)) > hi.z || ord2f(__ldg(L + 5)) < lo.z)
        continue;
    }
    const double3 A[3] = {make_double3(p0.x, p0.y, p0.z), make_double3(p1.x, p1.y, p1.z), make_double3(p2.x, p2.y, p2.z)};
    int stack[64];
    int sp = 0;
    int node = sc.root;
    while (true) {
      if (node >= 0) {
        const float4* nd = sc.nodes + 7 * (size_t)node;
        const float4 lx = __ldg(nd), hx = __ldg(nd + 1), ly = __ldg(nd + 2), hy = __ldg(nd + 3);
        const float4 lz = __ldg(nd + 4), hz = __ldg(nd + 5);
        const int4 e = __ldg(reinterpret_cast<const int4*>(nd + 6));
        const float clx[4] = {lx.x, lx.y, lx.z, lx.w}, chx[4] = {hx.x, hx.y, hx.z, hx.w};
        const float cly[4] = {ly.x, ly.y, ly.z, ly.w}, chy[4] = {hy.x, hy.y, hy.z, hy.w};
        const float clz[4] = {lz.x, lz.y, lz.z, lz.w}, chz[4] = {hz.x, hz.y, hz.z, hz.w};
        const int ch[4] = {e.x, e.y, e.z, e.w};
        for (int c = 0; c < 4; ++c) {
          if (ch[c] == 0x7fffffff) continue;
          if (clx[c] > hi.x || chx[c] < lo.x || cly[c] > hi.y || chy[c] < lo.y || clz[c] > hi.z || chz[c] < lo.z)
            continue;
          if (sp < 64) stack[sp++] = ch[c];
          else atomicOr(sc.err, 1);
        }
      } else {
        const int code = ~node;
        const int first = code >> 3, cnt = (code & 7) + 1;
        for (int k = 0; k < cnt; ++k) {
          const float4* lt = sc.leaf + 3 * (size_t)(first + k);
          const float4 q0 = __ldg(lt), q1 = __ldg(lt + 1), q2 = __ldg(lt + 2);
          const int u = __float_as_int(q0.w);
          const int ou = __ldg(sc.tri_v + u).w;
          if (ou <= tv.w || ou >= nmesh) continue;
          const double3 B[3] = {make_double3(q0.x, q0.y, q0.z), make_double3(q1.x, q1.y, q1.z),
                                make_double3(q2.x, q2.y, q2.z)};
          double3 s0, s1;
          if (!tri_tri_segment(A, B, s0, s1)) continue;
          const double len = sqrt((s1.x - s0.x) * (s1.x - s0.x) + (s1.y - s0.y) * (s1.y - s0.y) +
                                  (s1.z - s0.z) * (s1.z - s0.z));
          if (!(len > 0.0)) continue;
          const int slot = atomicAdd(cb.count, 1);
          if (slot >= kCreaseCap) continue;
          cb.ra[slot] = make_float4((float)s0.x, (float)s0.y, (float)s0.z, (float)len);
          cb.rb[slot] = make_float4((float)s1.x, (float)s1.y, (float)s1.z, 0.f);
          cb.rtris[slot] = make_int2(t, u);
        }
      }
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
}

// The extraction appends in whatever order the threads reach the counter; each segment's
// rank by its (triangle, triangle) pair puts them in one fixed order, so the samples (and
// the gradients) do not depend on scheduling.
__global__ void k_crease_order(CreaseBuf cb) {
  const int n = min(*cb.count, kCreaseCap);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 ti = cb.rtris[i];
    const unsigned long long ki = ((unsigned long long)(unsigned)ti.x << 32) | (unsigned)ti.y;
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const int2 tj = cb.rtris[j];
      const unsigned long long kj = ((unsigned long long)(unsigned)tj.x << 32) | (unsigned)tj.y;
      rank += kj < ki;
    }
    cb.a[rank] = cb.ra[i];
    cb.b[rank] = cb.rb[i];
    cb.tris[rank] = ti;
  }
}

// Segment lengths (0 past the segments found) as the masses of the length CDF.
__global__ void k_crease_mass(CreaseBuf cb, double* __restrict__ w) {
  const int n = min(*cb.count, kCreaseCap);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kCreaseCap; i += gridDim.x * blockDim.x)
    w[i] = i < n ? (double)cb.a[i].w : 0.0;
}

// World-space gradients of the raster coordinates (J's rows) at camera-space point pc.
PSDR_D void raster_grad(const DevView& V, float3 pc, float3& gx, float3& gy) {
  const float* m = V.c2r;
  const float* r = V.w2c;
  const float wden = m[12] * pc.x + m[13] * pc.y + m[14] * pc.z + m[15];
  float3 g[2];
  for (int c = 0; c < 2; ++c) {
    const float u = (m[4 * c] * pc.x + m[4 * c + 1] * pc.y + m[4 * c + 2] * pc.z + m[4 * c + 3]) / wden;
    const float3 gpc = f3(m[4 * c] - u * m[12], m[4 * c + 1] - u * m[13], m[4 * c + 2] - u * m[14]) / wden;
    g[c] = f3(r[0] * gpc.x + r[4] * gpc.y + r[8] * gpc.z, r[1] * gpc.x + r[5] * gpc.y + r[9] * gpc.z,
              r[2] * gpc.x + r[6] * gpc.y + r[10] * gpc.z);
  }
  gx = g[0];
  gy = g[1];
}

// Crease point of sample i (stratified by length over all segments) and its projection.
struct CreasePt {
  float3 x, tang;
  float2 u;     // raster position
  float2 n;     // unit raster normal of the projected curve
  float rlen;   // raster length per unit world length along the curve
  float wgt;    // world length per sample (total length / N)
  int seg;
  bool ok;
};

PSDR_D CreasePt crease_point(const DevView& V, CreaseBuf cb, const double* mw, const double* mpre, long long i,
                             long long N, float xi) {
  CreasePt c;
  c.ok = false;
  if (!(mpre[kCreaseCap - 1] > 0.0)) return c;
  float t;
  double pmf;
  c.seg = (int)border_locate(mw, mpre, kCreaseCap, i, N, xi, t, pmf);
  if (!(pmf > 0.0)) return c;
  const float4 a = cb.a[c.seg], b = cb.b[c.seg];
  const float3 s0 = xyz(a), s1 = xyz(b);
  c.x = s0 + (s1 - s0) * t;
  c.tang = (s1 - s0) * (1.f / a.w);
  c.wgt = (float)(mw[c.seg] / (pmf * (double)N));
  float3 pc, pr;
  xform_pos(V.w2c, c.x, pc);
  xform_pos(V.c2r, pc, pr);
  if (!(pc.z < 0.f && pr.x > 0.f && pr.x < (float)V.W && pr.y > 0.f && pr.y < (float)V.H)) return c;
  c.u = make_float2(pr.x, pr.y);
  float3 gx, gy;
  raster_grad(V, pc, gx, gy);
  const float mx = dot(gx, c.tang), my = dot(gy, c.tang);
  c.rlen = sqrtf(mx * mx + my * my);
  if (!(c.rlen > 0.f)) return c;
  c.n = make_float2(-my / c.rlen, mx / c.rlen);
  c.ok = true;
  return c;
}

// Offset rays on both sides of the projected curve; both must reach the two meshes next to
// the crease point (else something hides it). Paths from both hits give L1 and L2 (slots
// 2s: the -n side, surface 1; 2s + 1: the +n side, surface 2). The offset is 5 ray epsilons
// (tmin) in world units: closer to the crease, rays leaving one surface skip the other
// within tmin and the rendered radiance there is not the image's limit at the crease.
constexpr float kCreaseOffset = 5.f * kTmin;  // world units
__global__ void __launch_bounds__(256) k_crease_init(WF w, const DevScene* __restrict__ scenes,
                                                     const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                     CreaseBuf cb, const double* __restrict__ mw,
                                                     const double* __restrict__ mpre, long long begin, int n,
                                                     long long N) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    HitRec hs[2];
    hs[0].tri = hs[1].tri = -1;
    const DevView& V = views[v];
    if (s < n && !V.ortho) {
      const long long i = begin + s;
      const DevScene& sc = scenes[V.scene];
      Rng rng = make_rng(kCreaseStream + (unsigned long long)i + w.seed);
      const CreasePt c = crease_point(V, cb, mw, mpre, i, N, rng.next_float());
      bool ok = c.ok;
      int flag = 0;
      if (ok) {
        const int2 tp = cb.tris[c.seg];
        const int oa = __ldg(sc.tri_v + tp.x).w, ob = __ldg(sc.tri_v + tp.y).w;
        const float tol = 10.f * kCreaseOffset;
        int objs[2];
        for (int side = 0; side < 2; ++side) {
          const float sg = (side ? kCreaseOffset : -kCreaseOffset) * c.rlen;  // pixels
          float3 pcam;
          xform_pos(V.r2c, f3(c.u.x + sg * c.n.x, c.u.y + sg * c.n.y, 1.0f), pcam);
          const float3 d = normalize(xform_dir(V.c2w, pcam));
          hs[side] = trace_closest(sc, V.pos, d, kTmin, INFINITY);
          objs[side] = -1;
          if (hs[side].tri >= 0) {
            const Surf x = make_surf(sc, hs[side].tri, hs[side].b1, hs[side].b2, V.pos);
            if (norm(x.p - c.x) < tol) objs[side] = x.obj;
          }
        }
        ok = objs[0] >= 0 && objs[1] >= 0 && objs[0] != objs[1] && (objs[0] == oa || objs[0] == ob) &&
             (objs[1] == oa || objs[1] == ob);
        flag = ok ? (objs[0] == oa ? 1 : 2) : 0;  // 1: surface 1 is the segment's first triangle
      }
      const int px = ok ? min(V.W - 1, (int)floorf(c.u.x)) : 0, py = ok ? min(V.H - 1, (int)floorf(c.u.y)) : 0;
      eb.a[s] = make_float4(__int_as_float(c.seg), c.wgt * c.rlen, c.n.x, c.n.y);
      eb.n[s] = make_float4(c.x.x, c.x.y, c.x.z, __int_as_float(py * V.W + px));
      eb.hb[s] = make_float4(0.f, 0.f, 0.f, __int_as_float(flag));
      for (int side = 0; side < 2; ++side) {
        const int slot = 2 * s + side;
        const Rng r = make_rng(kCreaseStream + 0x10000000ull + 2 * (unsigned long long)i + side + w.seed);
        w.rs[slot] = r.state;
        w.ri[slot] = r.inc;
        w.view[slot] = v;
        w.pix[slot] = -1;
        w.T[slot] = make_float4(1.f, 1.f, 1.f, 0.f);
        w.L[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
        w.cur[slot] = hit4(hs[side]);
        w.org[slot] = make_float4(V.pos.x, V.pos.y, V.pos.z, 0.f);
      }
      alive = ok;
    }
    for (int side = 0; side < 2; ++side) {
      const int k = warp_append(&w.cnt[0], alive);
      if (alive) w.q0[k] = 2 * s + side;
    }
  }
}

// Barycentric weights of point x in triangle tri (of its vertices v0, v1, v2).
PSDR_D float3 bary_of(const DevScene& sc, int tri, float3 x) {
  const float4* R = sc.tri + 6 * (size_t)tri;
  const float3 p0 = xyz(__ldg(R)), p1 = xyz(__ldg(R + 1)), p2 = xyz(__ldg(R + 2));
  const float3 e1 = p1 - p0, e2 = p2 - p0, q = x - p0;
  const float d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2), q1 = dot(q, e1), q2 = dot(q, e2);
  const float den = d11 * d22 - d12 * d12;
  const float b1 = (d22 * q1 - d12 * q2) / den, b2 = (d11 * q2 - d12 * q1) / den;
  return f3(1.f - b1 - b2, b1, b2);
}

__global__ void __launch_bounds__(256) k_crease_final(WF w, const DevScene* __restrict__ scenes,
                                                      const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                      CreaseBuf cb, int n) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  float3 go = f3(0.f, 0.f, 0.f);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= n || !V.dimage) continue;
    const int flag = __float_as_int(eb.hb[s].w);
    if (flag == 0) continue;
    const float4 a = eb.a[s], xn = eb.n[s];
    const float* gp = V.dimage + 3 * (size_t)__float_as_int(xn.w);
    const float3 L1 = xyz(w.L[2 * s]), L2 = xyz(w.L[2 * s + 1]);
    const float G1 = gp[0] * L1.x + gp[1] * L1.y + gp[2] * L1.z, G2 = gp[0] * L2.x + gp[1] * L2.y + gp[2] * L2.z;
    if (!isfinite(G1) || !isfinite(G2) || (G1 == 0.f && G2 == 0.f)) continue;
    const int2 tp = cb.tris[__float_as_int(a.x)];
    const int t1 = flag == 1 ? tp.x : tp.y, t2 = flag == 1 ? tp.y : tp.x;
    const float3 x = xyz(xn);
    const float3 n1 = normalize(xyz(__ldg(sc.tri + 6 * (size_t)t1 + 3)));
    const float3 n2 = normalize(xyz(__ldg(sc.tri + 6 * (size_t)t2 + 3)));
    float3 pc, gx, gy;
    xform_pos(V.w2c, x, pc);
    raster_grad(V, pc, gx, gy);
    const float3 wv = gx * a.z + gy * a.w;  // J^T n
    const float c = dot(n1, n2), sn2 = 1.f - c * c;
    if (!(sn2 > 1e-6f)) continue;
    const float w1 = dot(wv, n1), w2 = dot(wv, n2);
    const float A1 = (w1 - c * w2) / sn2, A2 = (w2 - c * w1) / sn2;
    const float K = a.y;
    const float3 a1 = (n1 * ((G1 - G2) * A1) - wv * G1) * K;
    const float3 a2 = (n2 * ((G1 - G2) * A2) + wv * G2) * K;
    if (!finite3(a1) || !finite3(a2)) continue;
    if (sc.grad_verts) {
      const float3 b1 = bary_of(sc, t1, x), b2 = bary_of(sc, t2, x);
      const int4 v1 = __ldg(sc.tri_v + t1), v2 = __ldg(sc.tri_v + t2);
      vert_add(sc, v1.x, a1 * b1.x);
      vert_add(sc, v1.y, a1 * b1.y);
      vert_add(sc, v1.z, a1 * b1.z);
      vert_add(sc, v2.x, a2 * b2.x);
      vert_add(sc, v2.y, a2 * b2.y);
      vert_add(sc, v2.z, a2 * b2.z);
    }
    go -= a1 + a2;  // moving the camera by d is moving both surfaces by -d
  }
  if (V.grad_pos) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      go.x += __shfl_xor_sync(0xffffffffu, go.x, o);
      go.y += __shfl_xor_sync(0xffffffffu, go.y, o);
      go.z += __shfl_xor_sync(0xffffffffu, go.z, o);
    }
    if ((threadIdx.x & 31) == 0 && (go.x != 0.f || go.y != 0.f || go.z != 0.f)) atomic_add3(V.grad_pos, go);
  }
}

// ------------------------------------------------------------------ BSDF jumps
// Unbiased estimator, DiffuseBsdfMaterial with roughness > 0 (diffuse_bsdf.cc:56-88).
// With N.L >= 0 and N.V >= 0 the rough-diffuse value jumps by color b (max(N.L, N.V) +
// 1e-5) where t = m.L crosses 0, m = V - (N.V) N: over the shading hemisphere, the half
// great circle through N perpendicular to m. The rendered value at x_k changes at
// Int_arc dF L_i (Ng.L) d/dtheta[m . L_att] / |m| dl, L_att the direction from the material
// point x_k to the material point x_{k+1} seen along L. One pass per depth k:
// k_jump_init replays camera sample i to its k-th vertex (stream i: 2 jitter draws, then
// per vertex the arc draw and two direction draws), draws the arc direction there
// (uniform, pdf 1/pi) and starts a path along it on stream 16 i + k; the path kernels
// estimate L_i with D - k bounces; k_jump_final scatters the adjoint of the carrier
// m . normalize(x_{k+1} - x_k). Side buffers: a = weight (prefix throughput x color x dF x
// (Ng.L) pi / (|m| spp)) and pixel; n = x_k's hit (w: 1 when the sample is live);
// hb = x_{k+1}'s hit; La = x_{k-1}'s hit (tri -1: the camera).
constexpr unsigned long long kJumpStreams = 16;  // max_bounce <= 16

__global__ void __launch_bounds__(256) k_jump_init(WF w, const DevScene* __restrict__ scenes,
                                                   const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                   long long begin, int n, int k, int D) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    if (s < n) {
      const long long i = begin + s;
      const DevView& V = views[v];
      const DevScene& sc = scenes[V.scene];
      Rng rng = make_rng((unsigned long long)i + w.seed);
      const float jx = rng.next_float(), jy = rng.next_float();
      const int pix = V.spp > 1 ? (int)(i / V.spp) : (int)i;
      float3 pc;
      xform_pos(V.r2c, f3(jx + (float)(pix % V.W), jy + (float)(pix / V.W), 1.0f), pc);
      float3 o = V.pos, d;
      if (V.ortho) {
        xform_pos(V.c2w, f3(pc.x, pc.y, 0.f), o);
        d = view_look_dir(V);
      } else {
        d = normalize(xform_dir(V.c2w, pc));
      }
      HitRec h = trace_closest(sc, o, d, kTmin, INFINITY);
      Surf x = make_surf(sc, h.tri, h.b1, h.b2, o);
      HitRec hp;
      hp.tri = -1; hp.b1 = hp.b2 = hp.t = 0.f;
      float3 T = f3(1.f, 1.f, 1.f);
      eb.n[s] = make_float4(__int_as_float(-1), 0.f, 0.f, __int_as_float(0));
      w.L[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int kk = 1; kk <= k; ++kk) {
        if (!x.valid || x.is_light) break;
        const float u_arc = rng.next_float();
        const DevObj& ob = sc.objs[x.obj];
        const MatPt mp = mat_point(ob, x);
        if (kk == k) {
          const float nv = dot(mp.N, x.wi);
          const float3 m = x.wi - mp.N * nv;
          const float mlen = norm(m);
          if (!(mp.rough && mp.sigma > 0.f && nv >= 0.f && mlen > 1e-7f)) break;
          const float3 wa = normalize(cross(mp.N, m));
          float sp, cp;
          sincosf((u_arc - 0.5f) * kPi, &sp, &cp);
          const float3 L = normalize(mp.N * cp + wa * sp);
          const float nl = fmaxf(dot(mp.N, L), 0.f);
          const float a = 1.0f / (kPi + kOrenC * mp.sigma);
          const float dF = mp.sigma * a * (fmaxf(nl, nv) + kEps);
          const float3 wv = mul(T, mp.color) * (dF * dot(x.n, L) * kPi / (mlen * (float)V.spp));
          const HitRec ha = trace_closest(sc, x.p, L, kTmin, INFINITY);
          if (ha.tri < 0 || !finite3(wv)) break;
          eb.a[s] = make_float4(wv.x, wv.y, wv.z, __int_as_float(pix));
          eb.n[s] = make_float4(__int_as_float(h.tri), h.b1, h.b2, __int_as_float(1));
          eb.hb[s] = hit4(ha);
          eb.La[s] = hit4(hp);
          const Surf xa = make_surf(sc, ha.tri, ha.b1, ha.b2, x.p);
          if (k < D && !xa.is_light) {
            const Rng rl = make_rng((unsigned long long)i * kJumpStreams + (unsigned long long)k + w.seed);
            w.rs[s] = rl.state;
            w.ri[s] = rl.inc;
            w.view[s] = v;
            w.pix[s] = -1;
            w.T[s] = make_float4(1.f, 1.f, 1.f, 0.f);
            w.cur[s] = hit4(ha);
            w.org[s] = make_float4(x.p.x, x.p.y, x.p.z, 0.f);
            alive = true;
          }
          break;
        }
        // continue the camera path: cosine sampling about the shading normal
        const float rx = rng.next_float(), ry = rng.next_float();
        float ct, st, sphi, cphi;
        const float3 wo = material_dir(x, mp.N, rx, ry, ct, st, sphi, cphi);
        const HitRec hn = trace_closest(sc, x.p, wo, kTmin, INFINITY);
        const Surf nx = make_surf(sc, hn.tri, hn.b1, hn.b2, x.p);
        if (!nx.valid) break;
        const float tmp = dot(nx.n, -wo) / nx.sqd;
        const float G = dot(x.n, wo) * tmp;
        const float pdf = ct * kInvPi * tmp;
        T = mul(T, surf_bsdf(sc, x, wo)) * (G / pdf);
        if (!finite3(T)) break;
        hp = h;
        h = hn;
        x = nx;
      }
    }
    const int kq = warp_append(&w.cnt[0], alive);
    if (alive) w.q0[kq] = s;
  }
}

__global__ void __launch_bounds__(256) k_jump_final(WF w, const DevScene* __restrict__ scenes,
                                                    const DevView* __restrict__ views, int v, EdgeBuf eb, int n,
                                                    int k) {
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  HotAcc hot;
  hot.lv0 = 0;
  hot.nlv = 0;
  hot.emit_hot = false;
  float3 go = f3(0.f, 0.f, 0.f);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    if (s >= n || !V.dimage) continue;
    const float4 hk = eb.n[s];
    if (__float_as_int(hk.w) != 1) continue;
    const float4 a = eb.a[s], hn = eb.hb[s], hp = eb.La[s];
    const int pix = __float_as_int(a.w);
    const int tp = __float_as_int(hp.x);
    // the vertex before x_k: the camera (k = 1) or the material point of the last hit
    float3 op = V.pos;
    if (tp >= 0) op = make_surf(sc, tp, hp.y, hp.z, V.pos).p;
    const int tk = __float_as_int(hk.x);
    float3 ok = op;
    if (tp < 0 && V.ortho) {
      const Surf x0 = make_surf(sc, tk, hk.y, hk.z, V.pos);
      ok = ortho_origin_rn(V, x0.p);
    }
    const Surf x = make_surf(sc, tk, hk.y, hk.z, ok);
    const int ta = __float_as_int(hn.x);
    const Surf xa = make_surf(sc, ta, hn.y, hn.z, x.p);
    if (!x.valid || !xa.valid) continue;
    const float3 Li = xa.is_light ? light_emit<true>(sc.lights[xa.light], xa) : xyz(w.L[s]);
    const float* gp = V.dimage + 3 * (size_t)pix;
    const float wgt = gp[0] * a.x * Li.x + gp[1] * a.y * Li.y + gp[2] * a.z * Li.z;
    if (!(wgt != 0.f) || !isfinite(wgt)) continue;
    // q = m . l, m = V - (N.V) N, l = normalize(x_{k+1} - x_k)
    const DevObj& ob = sc.objs[x.obj];
    const MatPt mp = mat_point(ob, x);
    const bool fixed_v = tp < 0 && V.ortho;  // orthographic primary vertex: V = -look
    const float3 Vd = fixed_v ? -view_look_dir(V) : x.wi;
    const float3 u = xa.p - x.p;
    const float r = norm(u);
    const float3 l = u / r;
    const float nv = dot(mp.N, Vd), nl = dot(mp.N, l);
    const float3 m = Vd - mp.N * nv;
    const float3 du = (m - l * dot(m, l)) * (wgt / r);
    MatAdj ma = zero_mat_adj();
    ma.N = (Vd * nl + l * nv) * (-wgt);
    if (!fixed_v) ma.V = (l - mp.N * nl) * wgt;
    if (!finite3(du) || !finite3(ma.N) || !finite3(ma.V)) continue;
    SurfAdj ax = zero_adj(), aa = zero_adj();
    aa.p = du;
    ax.p = -du;
    const float3 ao = mat_finalize(ob, x, mp, ma, ax);
    scatter_surf(sc, hot, tk, hk.y, hk.z, x.front, ax);
    scatter_surf(sc, hot, ta, hn.y, hn.z, xa.front, aa);
    if (tp >= 0) {
      SurfAdj ap = zero_adj();
      ap.p = ao;
      scatter_surf(sc, hot, tp, hp.y, hp.z, true, ap);
    } else if (!fixed_v) {
      go += ao;
    }
  }
  if (V.grad_pos) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      go.x += __shfl_xor_sync(0xffffffffu, go.x, o);
      go.y += __shfl_xor_sync(0xffffffffu, go.y, o);
      go.z += __shfl_xor_sync(0xffffffffu, go.z, o);
    }
    if ((threadIdx.x & 31) == 0 && (go.x != 0.f || go.y != 0.f || go.z != 0.f)) atomic_add3(V.grad_pos, go);
  }
}

// ------------------------------------------------------------------ direct edges
// path_integrator.cc:274-353 and the boundary_term / hit_triangle adjoint (:11-78).
// UNB (unbiased estimator, PRE=false): the same samples and edge/light visibility
// tests; the edge point x_b, light point y and receiver x_d lie on one line and the
// shadow boundary moves over the receiver at d_eff = dx_b - dx_d / lam - dy (1 - 1/lam),
// lam = |x_d - y| / |x_b - y|. Per camera connection: -T |n_y.w| / |x_b - y|^2 J_cam
// (d_eff . (w x e)) / (pdf_e pdf_y hc_density H W spp), e oriented by the edge's outward
// vector so that the occluding faces lie on the -(w x e) side, T = f_r(x_d) L_e times the
// albedos of the diffuse bounces between x_d and the camera-visible vertex.
// BSDF: the DiffuseBsdfMaterial instance (direction-dependent f at the receiver and
// along the bounce chain); the other instance is the DiffuseMaterial one.
// The draws of shadow-boundary sample i: hypercube cell and position (PRE: the cell's
// sampler stream, persisted in w.rs / w.ri from the second preprocess round on), edge point x_b,
// light point y; returns the silhouette test (the edge's faces see y on opposite sides).
// PRE leaves the sampler state after the draws in `rng`; the caller persists it.
struct DirDraw {
  Rng rng;
  float hpdf, sx, pdf_e;
  int e;
  float3 p0, p1, out, nl, nr, xb, dir;
  LightSample ls;
};

template <bool PRE, bool UNB>
PSDR_D bool direct_draw(const WF& w, const DevScene& sc, const HCube& hc, int round, long long i, DirDraw& o) {
  float s3[3];
  o.hpdf = 1.f;
  if (PRE) {
    if (round == 0) o.rng = make_rng((unsigned long long)i);
    else { o.rng.state = w.rs[i]; o.rng.inc = w.ri[i]; }
    const int r12 = hc.res[1] * hc.res[2];
    const int c0 = (int)(i / r12);
    const int rem = (int)(i - (long long)c0 * r12);
    const int c1 = rem / hc.res[2], c2 = rem - c1 * hc.res[2];
    const float d0 = o.rng.next_float(), d1 = o.rng.next_float(), d2 = o.rng.next_float();
    s3[0] = ((float)c0 + d0) * hc.unit[0];
    s3[1] = ((float)c1 + d1) * hc.unit[1];
    s3[2] = ((float)c2 + d2) * hc.unit[2];
  } else {
    o.rng = make_rng((unsigned long long)i + w.seed);
    s3[0] = o.rng.next_float(); s3[1] = o.rng.next_float(); s3[2] = o.rng.next_float();
    int cell;
    if (UNB) {
      double pm;
      cell = hc_cell_unb(hc, s3[2], pm);
      o.hpdf = (float)pm;
      s3[2] = o.rng.next_float();
    } else {
      cell = discrete_sample(hc.pmf, hc.cmf, hc.ncells, s3[2], o.hpdf);
    }
    if (!(o.hpdf > 0.f)) return false;
    const int r12 = hc.res[1] * hc.res[2];
    const int c0 = cell / r12, rem = cell - c0 * r12;
    const int c1 = rem / hc.res[2], c2 = rem - c1 * hc.res[2];
    s3[0] = (s3[0] + (float)c0) * hc.unit[0];
    s3[1] = (s3[1] + (float)c1) * hc.unit[1];
    s3[2] = (s3[2] + (float)c2) * hc.unit[2];
  }
  const int ne = *sc.n_edges;
  float pe;
  o.sx = s3[0];
  o.e = discrete_sample(sc.edge_pmf, sc.edge_cmf, ne, o.sx, pe);
  const float4 E0 = __ldg(sc.edge + 4 * (size_t)o.e), E1 = __ldg(sc.edge + 4 * (size_t)o.e + 1),
               E2 = __ldg(sc.edge + 4 * (size_t)o.e + 2), E3 = __ldg(sc.edge + 4 * (size_t)o.e + 3);
  o.p0 = xyz(E0);
  o.p1 = xyz(E1);
  o.out = f3(E1.w, E2.x, E2.y);
  o.nl = f3(E2.z, E2.w, E3.x);
  o.nr = f3(E3.y, E3.z, E3.w);
  o.xb = o.p0 + (o.p1 - o.p0) * o.sx;
  o.pdf_e = pe / E0.w;
  o.ls = sample_light(sc, s3[1], s3[2]);
  o.dir = normalize(o.xb - o.ls.y);
  return dot(o.nl, o.dir) * dot(o.nr, o.dir) < 0.f && norm(o.nl - o.nr) > kEps;
}

// First stage of the shadow-boundary samples [begin, begin + n): the draws and the
// silhouette test only; the samples that pass are queued (w.q0, count in w.cnt[0]) for
// k_direct, whose warps then start with every lane on a sample that traces (most samples
// fail the test, and a lane that fails would idle while its warp traces). PRE persists the
// sampler state of the cells that fail; k_direct does it for the others.
template <bool PRE, bool UNB>
__global__ void __launch_bounds__(256) k_direct_pick(WF w, const DevScene* __restrict__ scenes,
                                                     const DevView* __restrict__ views, int v, long long begin,
                                                     int n, HCube hc, int round) {
  const DevScene& sc = scenes[views[v].scene];
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n32; k += stride) {
    bool ok = false;
    if (k < n) {
      const long long i = begin + k;
      DirDraw o;
      ok = direct_draw<PRE, UNB>(w, sc, hc, round, i, o);
      if (PRE && !ok) {
        w.rs[i] = o.rng.state;
        w.ri[i] = o.rng.inc;
      }
    }
    const int q = warp_append(&w.cnt[0], ok);
    if (ok) w.q0[q] = k;
  }
}

template <bool PRE, bool UNB, bool BSDF>
__global__ void __launch_bounds__(128) k_direct(WF w, const DevScene* __restrict__ scenes,
                                                const DevView* __restrict__ views, int v, long long begin, HCube hc,
                                                int round, float* mass, int spp) {
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  const int nq = w.cnt[0];
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += stride) {
    const long long i = begin + w.q0[q];
    DirDraw o;
    if (!direct_draw<PRE, UNB>(w, sc, hc, round, i, o)) continue;
    Rng& rng = o.rng;
    if (PRE) {
      w.rs[i] = rng.state;
      w.ri[i] = rng.inc;
    }
    const float hpdf = o.hpdf, sx = o.sx, pdf_e = o.pdf_e;
    const int e = o.e;
    const float3 p0 = o.p0, p1 = o.p1, out = o.out, xb = o.xb, dir = o.dir;
    const LightSample& ls = o.ls;
    // edge -> light: the same occlusion shortcut as the NEE rays (valid needs the
    // closest hit to be the light within sqrt(1e-5) of y)
    const float dist_l = norm(xb - ls.y);
    const HitRec hs = trace_closest(sc, xb, -dir, kTmin, dist_l * 1.0001f + 4e-3f, dist_l - 4e-3f);
    const Surf s0 = make_surf(sc, hs.tri, hs.b1, hs.b2, xb);
    if (!(s0.valid && s0.is_light && sqnorm(s0.p - ls.y) < kEps)) continue;
    const HitRec hd = trace_closest(sc, xb, dir, kTmin, INFINITY);
    const Surf d0 = make_surf(sc, hd.tri, hd.b1, hd.b2, xb);
    if (!(d0.valid && !d0.is_light)) continue;
    if (UNB) {
      // PRE: the guiding mass is the sum over camera connections of |weight| |w x e|
      // (the bounce chain draws from the sampler after its persisted state)
      if (!PRE && (!V.dimage || !sc.grad_verts)) continue;
      float3 ev = normalize(p1 - p0);
      if (dot(cross(dir, ev), out) < 0.f) ev = -ev;
      const float3 nsv = cross(dir, ev);
      const float dby = norm(xb - ls.y), lam = norm(d0.p - ls.y) / dby;
      const float cos_y = fabsf(dot(s0.n, dir));
      const float k0 = -cos_y / (dby * dby) / (pdf_e * ls.pdf * (float)V.H * (float)V.W);
      const float fxfy = view_fxfy(V);
      const float3 look = view_look(V);
      const DevLight& Lt = sc.lights[s0.light];
      // running throughput: the emission times pi f_r at every vertex the chain leaves
      // (DiffuseMaterial: f_r / pi of the receiver folded in up front, then the albedos)
      float3 T = light_emit<BSDF>(Lt, s0);
      if (!BSDF) {
        const DevObj& ob = sc.objs[d0.obj];
        T = mul(tex_rgb(ob.color, texel_offset(ob.color, d0.u, d0.v)) * kInvPi, T);
      }
      float wsum = 0.f, msum = 0.f;
      // camera connection of a vertex whose reflection hemisphere faces the camera:
      // T times its BSDF toward the camera times its camera Jacobian
      auto connect = [&](const Surf& v) {
        // from the camera position, or (orthographic) from v's foot on the camera plane
        // along the look direction
        const float3 co = V.ortho ? ortho_origin_rn(V, v.p) : V.pos;
        const float3 rel = v.p - co;
        const float dist = norm(rel);
        const float3 dir = V.ortho ? look : rel / dist;
        if (dot(v.n, dir) >= 0.f) return;
        int qx, qy;
        if (!project(V, v.p, qx, qy)) return;
        // the closest hit must be v itself: stop at the first hit short of it (same
        // outcome as a full closest-hit query followed by the distance test)
        const HitRec hc2 = trace_closest(sc, co, dir, kTmin, dist * 1.0001f + 4e-3f, dist - 4e-3f);
        const Surf iv = make_surf(sc, hc2.tri, hc2.b1, hc2.b2, co);
        if (!(iv.valid && !iv.is_light && sqnorm(iv.p - v.p) < kEps)) return;
        const float z = dot(rel, look);
        const float Jc = V.ortho ? fxfy * fabsf(dot(v.n, look)) : fxfy * fabsf(dot(v.n, rel)) / (z * z * z);
        const float3 Tf = BSDF ? mul(T, surf_bsdf(sc, v, -dir)) : T;
        if (PRE) {
          msum += norm(Tf) * fabsf(k0 * Jc);
        } else {
          const float* gp = V.dimage + 3 * ((size_t)qy * V.W + qx);
          wsum += (gp[0] * Tf.x + gp[1] * Tf.y + gp[2] * Tf.z) * (k0 * Jc);
        }
      };
      connect(d0);
      // the change of the radiance leaving the receiver, carried to the camera through
      // up to max_bounce - 1 bounces cosine-sampled about the geometric normal (each
      // multiplies pi f_r: G / pdf = pi)
      Surf v = d0;
      for (int j = 1; j < w.D; ++j) {
        const float ru = rng.next_float(), rv = rng.next_float();
        float ct, st, sp, cp;
        const float3 wo = diffuse_dir(v.n, v.t, ru, rv, ct, st, sp, cp);
        const HitRec hn = trace_closest(sc, v.p, wo, kTmin, INFINITY);
        const Surf nx = make_surf(sc, hn.tri, hn.b1, hn.b2, v.p);
        if (!nx.valid || nx.is_light) break;
        if (BSDF) {
          T = mul(T, surf_bsdf(sc, v, wo)) * kPi;
        } else {
          const DevObj& on = sc.objs[nx.obj];
          T = mul(T, tex_rgb(on.color, texel_offset(on.color, nx.u, nx.v)));
        }
        connect(nx);
        v = nx;
      }
      if (PRE) {
        const float m = msum * norm(nsv);
        if (isfinite(m)) mass[i] = mass[i] + m;
        continue;
      }
      const float3 a = nsv * (wsum / (hpdf * (float)hc.ncells * (float)spp));
      if (!finite3(a) || wsum == 0.f) continue;
      const int2 evv = __ldg(sc.edge_v + e);
      vert_add(sc, evv.x, a * (1.f - sx));
      vert_add(sc, evv.y, a * sx);
      const int4 td = __ldg(sc.tri_v + hd.tri);
      const float3 ad = a * (-1.f / lam);
      vert_add(sc, td.x, ad * (1.f - hd.b1 - hd.b2));
      vert_add(sc, td.y, ad * hd.b1);
      vert_add(sc, td.z, ad * hd.b2);
      const int4 tl = __ldg(sc.tri_v + ls.tri);
      const float3 al = a * (1.f / lam - 1.f);
      vert_add(sc, tl.x, al * (1.f - ls.su - ls.sv));
      vert_add(sc, tl.y, al * ls.su);
      vert_add(sc, tl.z, al * ls.sv);
      continue;
    }
    int px, py;
    if (!project(V, d0.p, px, py)) continue;
    float3 co = V.pos, cd;
    if (V.ortho) {
      co = ortho_origin_rn(V, d0.p);
      cd = view_look_dir(V);
    } else {
      cd = normalize(d0.p - V.pos);
    }
    const HitRec h2 = trace_closest(sc, co, cd, kTmin, INFINITY);
    const Surf i2 = make_surf(sc, h2.tri, h2.b1, h2.b2, co);
    if (!(i2.valid && !i2.is_light && sqnorm(i2.p - d0.p) < kEps)) continue;
    const float pdf_xw = s0.sqd * pdf_e * ls.pdf / dot(s0.n, dir);
    // boundary_term (detached quantities)
    const float3 xs = s0.p, xd = d0.p, ns = s0.n, nd = d0.n;
    const float3 rb = xb - xs;
    const float3 db = normalize(rb);
    float3 ev = normalize(p1 - p0);
    if (dot(cross(db, ev), out) < 0.f) ev = -ev;
    const float3 npl = cross(db, ev);
    const float3 ep = cross(nd, npl);
    const float cos_s = fabsf(dot(ns, db));
    const float cos_b = dot(ev, db), cos_d = dot(ep, db);
    const float sb2 = 1.f - cos_b * cos_b, sd2 = 1.f - cos_d * cos_d;
    const float sin_b = sb2 > 0.f ? sqrtf(sb2) : 0.f, sin_d = sd2 > 0.f ? sqrtf(sd2) : 0.f;
    const float len_sb = norm(xb - xs), len_sd = norm(xd - xs);
    const float Jb = len_sd * len_sb * sin_b / (sin_d * cos_s);
    const float dG = cos_s * dot(nd, -db) / (len_sd * len_sd);
    const DevLight& Lt = sc.lights[s0.light];
    const float3 Ts = light_emit<BSDF>(Lt, s0);
    float3 Td;
    if (BSDF) {
      Td = surf_bsdf(sc, d0, -cd);
    } else {
      const DevObj& ob = sc.objs[d0.obj];
      Td = tex_rgb(ob.color, texel_offset(ob.color, d0.u, d0.v)) * kInvPi;
    }
    if (PRE) {
      float3 val = mul(mul(f3(dG, dG, dG) * Jb / pdf_xw, Ts), Td);
      if (!finite3(val)) continue;
      val.x = val.x < kEps ? kEps : val.x;
      val.y = val.y < kEps ? kEps : val.y;
      val.z = val.z < kEps ? kEps : val.z;
      mass[i] = mass[i] + norm(val);
    } else {
      const float3 nep = cross(nd, ep);
      const float3 z = mul(mul(mul(f3(0.f, 0.f, 0.f), nep * dG) * Jb / pdf_xw, Ts), Td);
      if (!finite3(z) || !V.dimage || !sc.grad_verts) continue;
      const float* gp = V.dimage + 3 * ((size_t)py * V.W + px);
      const float c = Jb / pdf_xw * dG / (hpdf * (float)spp);
      const float3 wv = f3(gp[0] * nep.x * Ts.x * Td.x, gp[1] * nep.y * Ts.y * Td.y, gp[2] * nep.z * Ts.z * Td.z) * c;
      // hit_triangle(xs, d, xd, ep, nep) adjoint w.r.t. d
      const float3 e1 = ep, e2 = nep;
      const float3 T = xs - xd;
      const float3 P = cross(db, e2), Q = cross(T, e1);
      const float det = dot(P, e1);
      const float dcl = fminf(fmaxf(det, kEps), 1.f - kEps);
      const float inv = 1.f / dcl;
      const float u = dot(P, T) * inv, vv = dot(Q, db) * inv;
      const float au = dot(wv, e1), avv = dot(wv, e2);
      float3 ad = cross(e2, T) * (au * inv) + Q * (avv * inv);
      if (det > kEps && det < 1.f - kEps) ad += cross(e2, e1) * (-(au * u + avv * vv) * inv);
      const float3 axb = (ad - db * dot(db, ad)) / norm(rb);
      const int2 evv = __ldg(sc.edge_v + e);
      vert_add(sc, evv.x, axb * (1.f - sx));
      vert_add(sc, evv.y, axb * sx);
    }
  }
}

// ------------------------------------------------------------------ indirect shadow boundaries
// Unbiased estimator: shadow boundaries of light that other surfaces reflect. The geometry
// is the shadow-boundary term's with the light point replaced by the first surface y seen
// from the edge point x_b in a direction w sampled inside the edge's silhouette lune: the
// directions w = cos(t) e + sin(t) m(psi) for which exactly one of the two faces at the edge
// faces w, two opposite wedges of angle alpha (the angle between the face normals) around
// the edge, solid angle 4 alpha, sampled uniformly (pdf 1 / (4 alpha)). Measured this way
// the geometric factor cos_y / |x_b - y|^2 of the area form cancels, so sample weights stay
// bounded. y must be a mesh surface (light sources are the shadow-boundary term's); the
// receiver x_d is the first hit from x_b away from y and must be seen by the camera. The
// radiance leaving y toward x_b is a path traced from y with max_bounce - 1 bounces (y is
// the second vertex of the camera path through x_d); the boundary moves over the receiver at
// d_eff = dx_b - dx_d / lam - dy (1 - 1/lam) as for the light. Receivers that reach the
// camera only through further bounces are left out (their source paths would be one bounce
// shorter per chain vertex).
constexpr unsigned long long kIndirectStream = 0xE0000000ull;  // streams of the source paths
// Its per-sample variance is an order of magnitude below the light-source term's, so it takes
// a quarter of the shadow-boundary samples and a quarter of the guiding cells along the edge
// axis.
constexpr int kIndirectSampleDiv = 4, kIndirectCellDiv = 4;
// Preprocess rounds of the unbiased estimator's light-source shadow-boundary guide per
// requested round. One sample per cell (the reference's preprocess) leaves most of the 360k
// cells of the default guide with a single noisy estimate; the term's per-sample weights
// are heavy-tailed, and with four samples per cell its standard deviation on the 512²
// icosphere workload drops by a third (about 2.5x less variance) for ~1 ms.
constexpr int kDirectGuideRounds = 4;

// Direction of lune coordinates (u2, u3) in [0, 1)^2 at an edge with unit direction ev and
// unit face normals nl, nr (both perpendicular to ev); alpha gets the wedge angle.
PSDR_D float3 lune_dir(float3 ev, float3 nl, float3 nr, float u2, float u3, float& alpha) {
  const float3 b = cross(ev, nl);
  const float ar = atan2f(dot(nr, b), dot(nr, nl));  // nr's angle from nl around ev
  alpha = fabsf(ar);
  const bool second = u2 >= 0.5f;
  const float t = second ? 2.f * u2 - 1.f : 2.f * u2;
  const float psi = (second ? -0.5f * kPi : 0.5f * kPi) + t * ar;
  const float ct = 1.f - 2.f * u3, st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  float sp, cp;
  sincosf(psi, &sp, &cp);
  return ev * ct + (nl * cp + b * sp) * st;
}

// PRE: guiding mass per hypercube cell (|k0 J_cam| |f_r(x_d)| |w x e|; the source radiance
// is not known yet). Otherwise: one sample per thread, side buffers for k_indirect_final and
// a path from y (slot s) whose radiance toward x_b the depth loop computes.
template <bool PRE>
__global__ void __launch_bounds__(128) k_indirect(WF w, const DevScene* __restrict__ scenes,
                                                  const DevView* __restrict__ views, int v, EdgeBuf eb,
                                                  long long begin, int n, HCube hc, int round, float* mass) {
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  const int stride = gridDim.x * blockDim.x;
  const int n32 = (n + 31) & ~31;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n32; s += stride) {
    bool alive = false;
    if (s < n) {
      const long long i = begin + s;
      Rng rng;
      float s3[3], hpdf = 1.f;
      bool ok = true;
      if (PRE) {
        if (round == 0) rng = make_rng(kIndirectStream + (unsigned long long)i);
        else { rng.state = w.rs[s]; rng.inc = w.ri[s]; }
        const int r12 = hc.res[1] * hc.res[2];
        const int c0 = (int)(i / r12);
        const int rem = (int)(i - (long long)c0 * r12);
        const int c1 = rem / hc.res[2], c2 = rem - c1 * hc.res[2];
        const float d0 = rng.next_float(), d1 = rng.next_float(), d2 = rng.next_float();
        s3[0] = ((float)c0 + d0) * hc.unit[0];
        s3[1] = ((float)c1 + d1) * hc.unit[1];
        s3[2] = ((float)c2 + d2) * hc.unit[2];
        w.rs[s] = rng.state;
        w.ri[s] = rng.inc;
      } else {
        rng = make_rng(kIndirectStream + (unsigned long long)i + w.seed);
        s3[0] = rng.next_float(); s3[1] = rng.next_float(); s3[2] = rng.next_float();
        double pm;
        const int cell = hc_cell_unb(hc, s3[2], pm);
        hpdf = (float)pm;
        ok = pm > 0.0;
        s3[2] = rng.next_float();
        const int r12 = hc.res[1] * hc.res[2];
        const int c0 = cell / r12, rem = cell - c0 * r12;
        const int c1 = rem / hc.res[2], c2 = rem - c1 * hc.res[2];
        s3[0] = (s3[0] + (float)c0) * hc.unit[0];
        s3[1] = (s3[1] + (float)c1) * hc.unit[1];
        s3[2] = (s3[2] + (float)c2) * hc.unit[2];
      }
      const int ne = *sc.n_edges;
      float sx = s3[0], pe;
      const int e = ok ? discrete_sample(sc.edge_pmf, sc.edge_cmf, ne, sx, pe) : 0;
      float3 xb = f3(0.f, 0.f, 0.f), nsv = f3(0.f, 0.f, 0.f);
      HitRec hy, hd;
      hy.tri = hd.tri = -1;
      hy.b1 = hy.b2 = 0.f;
      if (ok) {
        const float4 E0 = __ldg(sc.edge + 4 * (size_t)e), E1 = __ldg(sc.edge + 4 * (size_t)e + 1),
                     E2 = __ldg(sc.edge + 4 * (size_t)e + 2), E3 = __ldg(sc.edge + 4 * (size_t)e + 3);
        const float3 p0 = xyz(E0), p1 = xyz(E1);
        const float3 out = f3(E1.w, E2.x, E2.y), nl = f3(E2.z, E2.w, E3.x), nr = f3(E3.y, E3.z, E3.w);
        xb = p0 + (p1 - p0) * sx;
        const float pdf_e = pe / E0.w;
        float3 ev = normalize(p1 - p0);
        float alpha;
        const float3 wy = lune_dir(ev, nl, nr, s3[1], s3[2], alpha);  // toward the source
        const float3 dir = -wy;                                       // from the source through x_b
        ok = alpha > kEps && dot(nl, dir) * dot(nr, dir) < 0.f;
        if (ok) {
          hy = trace_closest(sc, xb, wy, kTmin, INFINITY);
          const Surf s0 = make_surf(sc, hy.tri, hy.b1, hy.b2, xb);
          ok = s0.valid && !s0.is_light;
          if (ok) {
            hd = trace_closest(sc, xb, dir, kTmin, INFINITY);
            const Surf d0 = make_surf(sc, hd.tri, hd.b1, hd.b2, xb);
            ok = d0.valid && !d0.is_light;
            if (ok) {
              if (dot(cross(dir, ev), out) < 0.f) ev = -ev;
              nsv = cross(dir, ev);
              // the receiver seen by the camera (perspective views)
              const float3 rel = d0.p - V.pos;
              const float dist = norm(rel);
              const float3 cd = rel / dist;
              int qx = 0, qy = 0;
              ok = !V.ortho && dot(d0.n, cd) < 0.f && project(V, d0.p, qx, qy);
              if (ok) {
                const HitRec hc2 = trace_closest(sc, V.pos, cd, kTmin, dist * 1.0001f + 4e-3f, dist - 4e-3f);
                const Surf iv = make_surf(sc, hc2.tri, hc2.b1, hc2.b2, V.pos);
                ok = iv.valid && !iv.is_light && sqnorm(iv.p - d0.p) < kEps;
              }
              if (ok) {
                const float3 look = view_look(V);
                const float z = dot(rel, look);
                const float Jc = view_fxfy(V) * fabsf(dot(d0.n, rel)) / (z * z * z);
                const float k0 = -4.f * alpha / (pdf_e * (float)V.H * (float)V.W) * Jc;
                const float lam = norm(d0.p - s0.p) / norm(xb - s0.p);
                if (PRE) {
                  const float3 fr = surf_bsdf(sc, d0, -cd);
                  const float m = fabsf(k0) * norm(fr) * norm(nsv);
                  if (isfinite(m)) mass[i] = mass[i] + m;
                  ok = false;  // no path in the preprocess
                } else {
                  eb.a[s] = make_float4(__int_as_float(e), sx, hpdf, __int_as_float(qy * V.W + qx));
                  eb.n[s] = make_float4(__int_as_float(hy.tri), hy.b1, hy.b2, k0);
                  eb.hb[s] = make_float4(__int_as_float(hd.tri), hd.b1, hd.b2, lam);
                  eb.La[s] = make_float4(nsv.x, nsv.y, nsv.z, 0.f);
                }
              }
            }
          }
        }
      }
      if (!PRE) {
        eb.La[s].w = __int_as_float(ok ? 1 : 0);
        const Rng r = make_rng(kIndirectStream + 0x10000000ull + (unsigned long long)i + w.seed);
        w.rs[s] = r.state;
        w.ri[s] = r.inc;
        w.view[s] = v;
        w.pix[s] = -1;
        w.T[s] = make_float4(1.f, 1.f, 1.f, 0.f);
        w.L[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        w.cur[s] = make_float4(__int_as_float(ok ? hy.tri : -1), hy.b1, hy.b2, 0.f);
        w.org[s] = make_float4(xb.x, xb.y, xb.z, 0.f);
        alive = ok;
      }
    }
    if (!PRE) {
      const int k = warp_append(&w.cnt[0], alive);
      if (alive) w.q0[k] = s;
    }
  }
}

// N: the samples of the view (the per-sample estimate is divided by N / (H W)).
__global__ void __launch_bounds__(128) k_indirect_final(WF w, const DevScene* __restrict__ scenes,
                                                        const DevView* __restrict__ views, int v, EdgeBuf eb, int n,
                                                        float cells, long long N) {
  const DevView& V = views[v];
  const DevScene& sc = scenes[V.scene];
  const int stride = gridDim.x * blockDim.x;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    if (!V.dimage || !sc.grad_verts) continue;
    const float4 nv = eb.La[s];
    if (__float_as_int(nv.w) != 1) continue;
    const float4 a = eb.a[s], yn = eb.n[s], hd = eb.hb[s];
    const float3 Lo = xyz(w.L[s]);
    const int dtri = __float_as_int(hd.x);
    const float4 E0 = __ldg(sc.edge + 4 * (size_t)__float_as_int(a.x)), E1 = __ldg(sc.edge + 4 * (size_t)__float_as_int(a.x) + 1);
    const float3 xb = xyz(E0) + (xyz(E1) - xyz(E0)) * a.y;
    // the receiver lit from the edge side, reflecting toward the camera
    const Surf d0 = make_surf(sc, dtri, hd.y, hd.z, xb);
    const float3 fr = surf_bsdf(sc, d0, normalize(V.pos - d0.p));
    const float* gp = V.dimage + 3 * (size_t)__float_as_int(a.w);
    const float wsum = (gp[0] * fr.x * Lo.x + gp[1] * fr.y * Lo.y + gp[2] * fr.z * Lo.z) * yn.w;
    const float3 ag = xyz(nv) * (wsum / (a.z * cells * (float)((double)N / ((double)V.H * V.W))));
    if (!finite3(ag) || wsum == 0.f) continue;
    const int e = __float_as_int(a.x);
    const float sx = a.y, lam = hd.w;
    const int2 evv = __ldg(sc.edge_v + e);
    vert_add(sc, evv.x, ag * (1.f - sx));
    vert_add(sc, evv.y, ag * sx);
    const int4 td = __ldg(sc.tri_v + dtri);
    const float3 ad = ag * (-1.f / lam);
    vert_add(sc, td.x, ad * (1.f - hd.y - hd.z));
    vert_add(sc, td.y, ad * hd.y);
    vert_add(sc, td.z, ad * hd.z);
    const int4 ty = __ldg(sc.tri_v + __float_as_int(yn.x));
    const float3 ay = ag * (1.f / lam - 1.f);
    vert_add(sc, ty.x, ay * (1.f - yn.y - yn.z));
    vert_add(sc, ty.y, ay * yn.y);
    vert_add(sc, ty.z, ay * yn.z);
  }
}

// ------------------------------------------------------------------ small utilities
__global__ void k_mass_cdf(const float* __restrict__ mass, int n, double* __restrict__ w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = (double)mass[i];
}
// Unbiased estimator: add a uniform share (a quarter of the mean mass, 20% of the
// samples) to every cell, bounding sample weights at 5x the uniform one.
__global__ void k_mass_floor(float* __restrict__ mass, const double* __restrict__ pre, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double tot = pre[n - 1];
  const float f = tot > 0.0 ? (float)(0.25 * tot / (double)n) : 1.0f;
  mass[i] = mass[i] + f;
}
__global__ void k_mass_finalize(const double* __restrict__ w, const double* __restrict__ pre, int n,
                                float* __restrict__ pmf, float* __restrict__ cmf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double tot = pre[n - 1];
  if (!(tot > 0.0)) { pmf[i] = 0.f; cmf[i] = 1.f; return; }
  pmf[i] = (float)(w[i] / tot);
  cmf[i] = (float)(pre[i] / tot);
}
__global__ void k_grad_out(const GradAcc* __restrict__ acc, float* __restrict__ out, long long n, int accumulate) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const longlong2 a = __ldg(reinterpret_cast<const longlong2*>(acc) + i);
  out[i] = (accumulate ? out[i] : 0.f) + (float)acc_value(a.x, a.y);
}


// ================================================================== host side
namespace {
inline int grid_for(long long n, int threads, int per_sm) {
  const long long want = (n + threads - 1) / threads;
  const long long cap = (long long)num_sms() * per_sm;
  return (int)std::max<long long>(1, std::min(want, cap));
}
}  // namespace

// camera.h:7-64, :111-124; psdr.cc:24-29 (near -0.01, far -1000). Row-major floats.
void make_view(const psdr_camera_desc& c, int spp, DevView& v) {
  auto nrm = [](double* a) { double n = std::sqrt(a[0]*a[0]+a[1]*a[1]+a[2]*a[2]); a[0]/=n; a[1]/=n; a[2]/=n; };
  auto crs = [](const double* a, const double* b, double* r) {
    r[0] = a[1]*b[2]-a[2]*b[1]; r[1] = a[2]*b[0]-a[0]*b[2]; r[2] = a[0]*b[1]-a[1]*b[0]; };
  double o[3] = {c.look_from[0], c.look_from[1], c.look_from[2]};
  double t[3] = {c.look_at[0], c.look_at[1], c.look_at[2]};
  double u[3] = {c.up[0], c.up[1], c.up[2]};
  double dir[3] = {o[0]-t[0], o[1]-t[1], o[2]-t[2]};
  nrm(dir); nrm(u);
  double right[3], nup[3];
  crs(u, dir, right);
  crs(dir, right, nup);
  double cw[4][4] = {{0}}, cs[4][4] = {{0}}, sr[4][4] = {{0}}, tr[4][4] = {{0}};
  for (int i = 0; i < 3; ++i) { cw[i][0] = right[i]; cw[i][1] = nup[i]; cw[i][2] = dir[i]; cw[i][3] = o[i]; }
  cw[3][3] = 1;
  const double nearv = -0.01, farv = -1000.0, inv_nf = 1.0 / (nearv - farv);
  v.ortho = c.type == PSDR_CAM_ORTHOGRAPHIC;
  if (v.ortho) {
    // camera.h:19-31 orthographic(left, right, bottom, top, near, far) = scale * translate
    // over the view box of camera.h:290-300 (width fov = view_width, height width H / W)
    const double hw = (double)c.fov / 2, hh = (double)c.height * hw / (double)c.width;
    cs[0][0] = 2 / (2 * hw);
    cs[1][1] = 2 / (2 * hh);
    cs[2][2] = 2 / (nearv - farv);
    cs[2][3] = cs[2][2] * (-(nearv + farv) / 2);
    cs[3][3] = 1;
  } else {
    const double cot = 1.0 / std::tan((double)c.fov * 0.5);
    cs[0][0] = -cot; cs[1][1] = -cot; cs[2][2] = (nearv + farv) * inv_nf; cs[2][3] = -2 * farv * nearv * inv_nf;
    cs[3][2] = 1;
  }
  sr[0][0] = 0.5 * c.width; sr[1][1] = -0.5 * c.height; sr[2][2] = 1; sr[3][3] = 1;
  tr[0][0] = tr[1][1] = tr[2][2] = tr[3][3] = 1; tr[0][3] = 1; tr[1][3] = -1;
  auto mm = [](const double a[4][4], const double b[4][4], double r[4][4]) {
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) { double s = 0; for (int k = 0; k < 4; ++k) s += a[i][k] * b[k][j]; r[i][j] = s; } };
  auto inv = [](const double a[4][4], double r[4][4]) {
    double m[4][8];
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 8; ++j) m[i][j] = j < 4 ? a[i][j] : (j - 4 == i ? 1.0 : 0.0);
    for (int col = 0; col < 4; ++col) {
      int p = col;
      for (int rr = col + 1; rr < 4; ++rr) if (std::fabs(m[rr][col]) > std::fabs(m[p][col])) p = rr;
      for (int j = 0; j < 8; ++j) std::swap(m[col][j], m[p][j]);
      const double iv = 1.0 / m[col][col];
      for (int j = 0; j < 8; ++j) m[col][j] *= iv;
      for (int rr = 0; rr < 4; ++rr) { if (rr == col) continue; const double f = m[rr][col]; for (int j = 0; j < 8; ++j) m[rr][j] -= f * m[col][j]; }
    }
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) r[i][j] = m[i][j + 4];
  };
  double t1[4][4], c2r[4][4], r2c[4][4], w2c[4][4];
  mm(sr, tr, t1);
  mm(t1, cs, c2r);
  inv(c2r, r2c);
  inv(cw, w2c);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      v.r2c[4 * i + j] = (float)r2c[i][j];
      v.c2w[4 * i + j] = (float)cw[i][j];
      v.w2c[4 * i + j] = (float)w2c[i][j];
      v.c2r[4 * i + j] = (float)c2r[i][j];
    }
  v.pos = make_float3(c.look_from[0], c.look_from[1], c.look_from[2]);
  v.H = c.height;
  v.W = c.width;
  v.spp = spp;
  v.scene = 0;
  v.image = nullptr;
  v.dimage = nullptr;
  v.grad_pos = nullptr;
  v.grad_lens = nullptr;
  v.scene_ntri = 0;
}

// Forward-mode derivative of the raster-to-direction map M = C diag(2 t / W, -2 t / H, -1),
// t = tan(fov / 2), C = (right, up, dir) built as camera.h:35-52 does (dir = normalize(from -
// at), right = cross(normalize(up), dir) unnormalised, up' = cross(dir, right)), with
// respect to the ten camera parameters (from, at, up, fov); P_j = M^-1 dM/dtheta_j.
namespace {
struct Dual10 {
  double v;
  double d[10];
};
Dual10 dconst(double v) { Dual10 r{v, {0}}; return r; }
Dual10 dvar(double v, int j) { Dual10 r = dconst(v); r.d[j] = 1.0; return r; }
Dual10 operator+(const Dual10& a, const Dual10& b) { Dual10 r{a.v + b.v, {0}}; for (int j = 0; j < 10; ++j) r.d[j] = a.d[j] + b.d[j]; return r; }
Dual10 operator-(const Dual10& a, const Dual10& b) { Dual10 r{a.v - b.v, {0}}; for (int j = 0; j < 10; ++j) r.d[j] = a.d[j] - b.d[j]; return r; }
Dual10 operator*(const Dual10& a, const Dual10& b) { Dual10 r{a.v * b.v, {0}}; for (int j = 0; j < 10; ++j) r.d[j] = a.d[j] * b.v + a.v * b.d[j]; return r; }
Dual10 operator*(const Dual10& a, double k) { Dual10 r{a.v * k, {0}}; for (int j = 0; j < 10; ++j) r.d[j] = a.d[j] * k; return r; }
Dual10 dinv(const Dual10& a) { Dual10 r{1.0 / a.v, {0}}; for (int j = 0; j < 10; ++j) r.d[j] = -a.d[j] / (a.v * a.v); return r; }
Dual10 dsqrt(const Dual10& a) { Dual10 r{std::sqrt(a.v), {0}}; for (int j = 0; j < 10; ++j) r.d[j] = a.d[j] / (2.0 * r.v); return r; }
Dual10 dtan(const Dual10& a) {
  const double t = std::tan(a.v);
  Dual10 r{t, {0}};
  for (int j = 0; j < 10; ++j) r.d[j] = a.d[j] * (1.0 + t * t);
  return r;
}
void dnormalize(Dual10* a) {
  const Dual10 n = dinv(dsqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
  for (int k = 0; k < 3; ++k) a[k] = a[k] * n;
}
void dcross(const Dual10* a, const Dual10* b, Dual10* r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
bool inv3(const double* m, double* r) {
  const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
  const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
  const double id = 1.0 / det;
  r[0] = c00 * id; r[1] = (m[2] * m[7] - m[1] * m[8]) * id; r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = c01 * id; r[4] = (m[0] * m[8] - m[2] * m[6]) * id; r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = c02 * id; r[7] = (m[1] * m[6] - m[0] * m[7]) * id; r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return true;
}
}  // namespace

void lens_chain(const psdr_camera_desc& c, LensChain& out, double* m9) {
  Dual10 from[3], at[3], up[3];
  for (int k = 0; k < 3; ++k) {
    from[k] = dvar(c.look_from[k], k);
    at[k] = dvar(c.look_at[k], 3 + k);
    up[k] = dvar(c.up[k], 6 + k);
  }
  const Dual10 fov = dvar(c.fov, 9);
  Dual10 dir[3] = {from[0] - at[0], from[1] - at[1], from[2] - at[2]};
  dnormalize(dir);
  dnormalize(up);
  Dual10 right[3], nup[3];
  dcross(up, dir, right);
  dcross(dir, right, nup);
  const Dual10 t = dtan(fov * 0.5);
  const Dual10 sx = t * (2.0 / c.width), sy = t * (-2.0 / c.height);
  Dual10 M[9];
  for (int i = 0; i < 3; ++i) {
    M[3 * i] = right[i] * sx;
    M[3 * i + 1] = nup[i] * sy;
    M[3 * i + 2] = dir[i] * -1.0;
  }
  double m[9], mi[9];
  for (int q = 0; q < 9; ++q) m[q] = M[q].v;
  if (m9) std::copy(m, m + 9, m9);
  PSDR_CHECK(inv3(m, mi), "degenerate camera basis (look_at equals look_from, or up parallel to the view)");
  for (int j = 0; j < 10; ++j)
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q) {
        double acc = 0.0;
        for (int k = 0; k < 3; ++k) acc += mi[3 * r + k] * M[3 * k + q].d[j];
        out.P[j][3 * r + q] = acc;
      }
}

void lens_out(const GradAcc* acc, const LensChain& ch, float* out, int accumulate, cudaStream_t st) {
  k_lens_out<<<1, 32, 0, st>>>(acc, ch, out, accumulate);
  profiler().launches += 1;
  PSDR_CUDA(cudaGetLastError());
}

std::vector<Tile> plan_tiles(const std::vector<DevView>& views, int cap) {
  std::vector<Tile> tiles;
  Tile cur{0, 0, 0, 0};
  for (const DevView& v : views) {
    long long rem = (long long)v.H * v.W;
    while (rem > 0) {
      const long long room = (cap - cur.n) / v.spp;
      if (room <= 0) {
        tiles.push_back(cur);
        cur = Tile{cur.begin + cur.n, 0, cur.pix_begin + cur.npix, 0};
        continue;
      }
      const long long take = std::min(room, rem);
      cur.n += (int)(take * v.spp);
      cur.npix += (int)take;
      rem -= take;
    }
  }
  if (cur.n > 0) tiles.push_back(cur);
  return tiles;
}

void assign_offsets(std::vector<DevView>& views) {
  long long so = 0, po = 0;
  for (DevView& v : views) {
    v.sample_off = so;
    v.pix_off = po;
    so += (long long)v.H * v.W * v.spp;
    po += (long long)v.H * v.W;
  }
}

Profiler& profiler() {
  static Profiler p;
  return p;
}
void Profiler::begin_trace(cudaStream_t st) {
  if (!on) return;
  if (capture_ev) {
    cudaEvent_t a, b;
    PSDR_CUDA(cudaEventCreate(&a));
    PSDR_CUDA(cudaEventCreate(&b));
    capture_ev->emplace_back(a, b);
    // External: becomes an event-record node of the graph (re-recorded every replay)
    PSDR_CUDA(cudaEventRecordWithFlags(a, st, cudaEventRecordExternal));
    return;
  }
  if (used == ev.size()) {
    cudaEvent_t a, b;
    PSDR_CUDA(cudaEventCreate(&a));
    PSDR_CUDA(cudaEventCreate(&b));
    ev.emplace_back(a, b);
  }
  PSDR_CUDA(cudaEventRecord(ev[used].first, st));
}
void Profiler::end_trace(cudaStream_t st) {
  if (!on) return;
  if (capture_ev) {
    PSDR_CUDA(cudaEventRecordWithFlags(capture_ev->back().second, st, cudaEventRecordExternal));
    return;
  }
  PSDR_CUDA(cudaEventRecord(ev[used].second, st));
  ++used;
  ++trace_launches;
}
void Profiler::replayed(std::vector<EvPair>* graph_ev, long long n_trace) {
  if (!on || graph_ev->empty()) return;
  trace_launches += n_trace;
  for (auto& r : replays)
    if (r.first == graph_ev) { ++r.second; return; }
  replays.emplace_back(graph_ev, 1);
}
#define PSDR_LAUNCHED(n) (profiler().launches += (n))
void count_launches(int n) { profiler().launches += n; }

static int any_ortho(const std::vector<DevView>& views) {
  for (const DevView& v : views)
    if (v.ortho) return 1;
  return 0;
}

// Shadow-boundary samples [0, n) in chunks of the tile capacity: the pick stage queues the
// samples that pass the silhouette test, then the k_direct instance for the job's
// materials (w.bsdf) traces them.
template <bool PRE, bool UNB>
static void launch_direct(const WF& w, cudaStream_t st, const DevScene* scenes, const DevView* vd, int v,
                          long long n, const HCube& hc, int round, float* mass, int spp) {
  for (long long b = 0; b < n; b += w.cap) {
    const int nb = (int)std::min<long long>(w.cap, n - b);
    PSDR_CUDA(cudaMemsetAsync(w.cnt, 0, sizeof(int), st));
    k_direct_pick<PRE, UNB><<<grid_for(nb, 256, 8), 256, 0, st>>>(w, scenes, vd, v, b, nb, hc, round);
    const int g = grid_for(nb, 128, 16);
    if (w.bsdf) k_direct<PRE, UNB, true><<<g, 128, 0, st>>>(w, scenes, vd, v, b, hc, round, mass, spp);
    else k_direct<PRE, UNB, false><<<g, 128, 0, st>>>(w, scenes, vd, v, b, hc, round, mass, spp);
    PSDR_LAUNCHED(2);
  }
  PSDR_CUDA(cudaGetLastError());
}

// Zeroes the queue counters of a wavefront before a new set of paths enters its depth
// loop (k_shade resets the ray fetch counter of k_trace itself).
static void clear_counts(const WF& w, cudaStream_t st) {
  PSDR_CUDA(cudaMemsetAsync(w.cnt, 0, sizeof(int) * 2 * (w.D + 1), st));
}

template <int MODE>
static void depth_loop_t(WF& w, const DevScene* scenes, const DevView* views, cudaStream_t st) {
  const int cap = w.cap;
  Profiler& pf = profiler();
  for (int d = 0; d < w.D; ++d) {
    const int gs = grid_for(cap, 256, 8);
    if (w.bsdf) k_shade<MODE, true><<<gs, 256, 0, st>>>(w, scenes, views, d);
    else k_shade<MODE, false><<<gs, 256, 0, st>>>(w, scenes, views, d);
    pf.begin_trace(st);
    k_trace<<<num_sms() * w.trace_bps, 128, 0, st>>>(w, scenes, views, d, pf.on ? pf.d_rays : nullptr);
    pf.end_trace(st);
    PSDR_LAUNCHED(3);
    if (w.bsdf) k_accum<MODE, true><<<gs, 256, 0, st>>>(w, scenes, views, d);
    else k_accum<MODE, false><<<gs, 256, 0, st>>>(w, scenes, views, d);
  }
  PSDR_CUDA(cudaGetLastError());
}

static void depth_loop(WF& w, const DevScene* scenes, const DevView* views, int mode, cudaStream_t st) {
  if (mode == MODE_REPLAY) depth_loop_t<MODE_REPLAY>(w, scenes, views, st);
  else if (mode == MODE_KEEP) depth_loop_t<MODE_KEEP>(w, scenes, views, st);
  else depth_loop_t<MODE_FWD>(w, scenes, views, st);
}

template <int MODE>
static void launch_camera(const WF& w, const DevScene* scenes, const DevView* views, const Tile& tile, int g,
                          cudaStream_t st) {
  if (w.ortho) k_camera<MODE, true><<<g, 256, 0, st>>>(w, scenes, views, tile);
  else k_camera<MODE, false><<<g, 256, 0, st>>>(w, scenes, views, tile);
}

static void run_tile(WF& w, const DevScene* scenes, const DevView* views, const Tile& tile, int mode,
                     cudaStream_t st) {
  clear_counts(w, st);
  const int g = grid_for(tile.n, 256, 8);
  if (mode == MODE_REPLAY) launch_camera<MODE_REPLAY>(w, scenes, views, tile, g, st);
  else if (mode == MODE_KEEP) launch_camera<MODE_KEEP>(w, scenes, views, tile, g, st);
  else launch_camera<MODE_FWD>(w, scenes, views, tile, g, st);
  PSDR_LAUNCHED(1);
  depth_loop(w, scenes, views, mode, st);
}

int choose_cap(const psdr_config& cfg, const std::vector<DevView>& views, bool backward) {
  int maxspp = 1;
  long long total = 0;
  for (auto& v : views) { maxspp = std::max(maxspp, v.spp); total += (long long)v.H * v.W * v.spp; }
  long long cap = cfg.tile_paths > 0 ? cfg.tile_paths : (1 << 20);
  if (backward) {
    long long cells = std::max<long long>(cfg.primary_edge_hypercube_resolution,
                                          (long long)cfg.secondary_edge_hypercube_resolution[0] *
                                              cfg.secondary_edge_hypercube_resolution[1] *
                                              cfg.secondary_edge_hypercube_resolution[2]);
    cap = std::max(cap, cells);
  } else {
    cap = std::min<long long>(cap, std::max<long long>(total, maxspp));
  }
  cap = std::max<long long>(cap, maxspp);
  cap = (cap + 31) / 32 * 32;
  return (int)cap;
}

}  // namespace psdr

// Mass / prefix-sum buffers of the hypercube cells and pixel-border segments.
void psdr_workspace::ensure_mass(long long n, cudaStream_t st) {
  if (n <= mass_cap) return;
  mass_cap = n;
  mass.alloc(4 * (size_t)n, st);
  mass_d.alloc(8 * (size_t)n, st);
  mass_pre.alloc(8 * (size_t)n, st);
  scan_tmp.alloc(8 * (psdr::scan_tmp_doubles((int)n) + 64), st);
}

void psdr_workspace::ensure(int c, int r, int d, int nv, int rec_needed, cudaStream_t st) {
  using namespace psdr;
  stream = st;
  if (c > cap || r > R || d > D) {
    cap = std::max(c, cap);
    R = std::max(r, R);
    D = std::max(d, D);
    const size_t n = (size_t)cap;
    rs.alloc(8 * n, st); ri.alloc(8 * n, st); view.alloc(4 * n, st); pix.alloc(4 * n, st);
    T.alloc(16 * n, st); L.alloc(16 * n, st); cur.alloc(16 * n, st); org.alloc(16 * n, st);
    q0.alloc(4 * n, st); q1.alloc(4 * n, st); qs.alloc(4 * n, st);
    cnt.alloc(sizeof(int) * 2 * (kMaxDepth + 2), st);
    ro.alloc(16 * n * R, st); rd.alloc(16 * n * R, st); ra.alloc(16 * n * R, st); hit.alloc(16 * n * R, st);
    eb_a.alloc(16 * n, st); eb_n.alloc(16 * n, st); eb_hb.alloc(16 * n, st); eb_La.alloc(16 * n, st);
    hc_pmf.alloc(4 * n, st); hc_cmf.alloc(4 * n, st);
  }
  ensure_mass(cap, st);
  if (rec_needed) rec.alloc(16 * (size_t)cap * (1 + (size_t)D * R + 2 * (size_t)D), st);
  if (nv > nviews_cap) {
    nviews_cap = nv;
    views.alloc(sizeof(DevView) * nv, st);
  }
  wf.cap = cap;
  wf.rs = rs.as<unsigned long long>(); wf.ri = ri.as<unsigned long long>();
  wf.view = view.as<int>(); wf.pix = pix.as<int>();
  wf.T = T.as<float4>(); wf.L = L.as<float4>(); wf.cur = cur.as<float4>(); wf.org = org.as<float4>();
  wf.q0 = q0.as<int>(); wf.q1 = q1.as<int>(); wf.qs = qs.as<int>(); wf.cnt = cnt.as<int>();
  wf.ro = ro.as<float4>(); wf.rd = rd.as<float4>(); wf.ra = ra.as<float4>(); wf.hit = hit.as<float4>();
  wf.rec = rec.as<float4>();
}

namespace psdr {

void upload_views(psdr_workspace* ws, const std::vector<DevView>& views, cudaStream_t st) {
  ws->h_views = views;
  PSDR_CUDA(cudaMemcpyAsync(ws->views.p, ws->h_views.data(), sizeof(DevView) * views.size(), cudaMemcpyHostToDevice, st));
}

void set_wf(WF& w, const psdr_config& cfg, int nviews, int nB_override, int light_vis) {
  w.D = cfg.max_bounce;
  w.nL = cfg.mis_light_samples;
  w.nB = nB_override >= 0 ? nB_override : cfg.mis_bsdf_samples;
  w.R = w.nL + w.nB + 1;
  w.light_vis = light_vis;
  w.nviews = nviews;
  // seed s offsets every sample stream by s * 2654435761 (mod 2^32, the width of the
  // stream index): jobs of different seeds draw from disjoint stream ranges
  w.seed = cfg.seed * 2654435761ull;
  w.rec_stride = 1 + w.D * w.R + 2 * w.D;  // primary hit, hits per depth, (C, beta) per depth
  w.trace_bps = cfg.trace_queue > 0 ? cfg.trace_queue : 8;
}

void forward_tile(const DevScene* scenes_dev, const std::vector<DevView>& views, const DevView* vd, const Tile& t,
                  const psdr_config& cfg, psdr_workspace* ws, cudaStream_t st, float* samples_out,
                  const KeptRecords* keep) {
  WF w = ws->wf;
  w.cap = ws->cap;
  set_wf(w, cfg, (int)views.size(), -1, cfg.enable_light_visable);
  w.bsdf = ws->bsdf;
  w.ortho = any_ortho(views);
  if (keep) {
    w.rec = keep->rec + (size_t)t.begin * w.rec_stride;
    w.view = keep->view + t.begin;
    w.pix = keep->pix + t.begin;
  }
  run_tile(w, scenes_dev, vd, t, keep ? MODE_KEEP : MODE_FWD, st);
  k_film<<<grid_for(t.npix, 256, 8), 256, 0, st>>>(w, vd, t, std::max(1, cfg.n_pass), samples_out);
  PSDR_LAUNCHED(1);
  PSDR_CUDA(cudaGetLastError());
}

// Forward: the interior estimate of every view into V.image (and per-sample radiance
// of view 0 into samples_out when given).
// Device work of a forward job whose views are already in ws->views (tiles of `cap`
// paths). Makes no allocation and no host copy, so it can be recorded into a graph.
void forward_launch(const DevScene* scenes_dev, const std::vector<DevView>& views, const psdr_config& cfg, int cap,
                    psdr_workspace* ws, cudaStream_t st, float* samples_out) {
  const DevView* vd = ws->views.as<DevView>();
  for (const Tile& t : plan_tiles(views, cap)) forward_tile(scenes_dev, views, vd, t, cfg, ws, st, samples_out);
}

void render_forward_impl(const DevScene* scenes_dev, std::vector<DevView>& views, const psdr_config& cfg,
                         psdr_workspace* ws, cudaStream_t st, float* samples_out) {
  assign_offsets(views);
  const int cap = choose_cap(cfg, views, false);
  const int R = cfg.mis_light_samples + cfg.mis_bsdf_samples + 1;
  ws->ensure(cap, R, cfg.max_bounce, (int)views.size(), 0, st);
  upload_views(ws, views, st);
  forward_launch(scenes_dev, views, cfg, cap, ws, st, samples_out);
}

static void edge_phase(WF w, const DevScene* scenes, const DevView* vd, int v, const EdgeBuf& eb, long long begin,
                       int n, const HCube& hc, int round, bool pre, float* mass, int spp, cudaStream_t st) {
  clear_counts(w, st);
  if (pre) k_edge_init<true><<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, begin, n, hc, round, 0);
  else k_edge_init<false><<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, begin, n, hc, round, 0);
  PSDR_LAUNCHED(1);
  depth_loop(w, scenes, vd, MODE_FWD, st);
  clear_counts(w, st);
  k_edge_mid<<<grid_for(n, 256, 8), 256, 0, st>>>(w, vd, v, eb, n);
  PSDR_LAUNCHED(1);
  depth_loop(w, scenes, vd, MODE_FWD, st);
  if (pre) k_edge_final<true><<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, begin, n, mass, spp);
  else k_edge_final<false><<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, begin, n, mass, spp);
  PSDR_LAUNCHED(1);
  PSDR_CUDA(cudaGetLastError());
}

// Unbiased silhouette samples: one path per sample (the background side).
static void edge_phase_unb(WF w, const DevScene* scenes, const DevView* vd, int v, const EdgeBuf& eb,
                           long long begin, int n, const HCube& hc, int spp, cudaStream_t st) {
  clear_counts(w, st);
  k_edge_init<false><<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, begin, n, hc, 0, 1);
  PSDR_LAUNCHED(2);
  depth_loop(w, scenes, vd, MODE_FWD, st);
  k_edge_final_unb<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, n, (float)hc.ncells, spp);
  PSDR_CUDA(cudaGetLastError());
}

// Pixel-border samples [begin, begin + n) of the N of view v (segment masses in w/pre).
static void border_phase(WF w, const DevScene* scenes, const DevView* vd, int v, const EdgeBuf& eb,
                         const double* mw, const double* mpre, long long S, long long begin, int n, long long N,
                         bool lens, cudaStream_t st) {
  clear_counts(w, st);
  k_border_init<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, mw, mpre, S, begin, n, N);
  PSDR_LAUNCHED(2);
  depth_loop(w, scenes, vd, MODE_FWD, st);
  k_border_final<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, n, N);
  if (lens) {
    k_lens_border<<<grid_for(n, 256, 8), 256, 0, st>>>(w, vd, v, eb, n, N);
    PSDR_LAUNCHED(1);
  }
  PSDR_CUDA(cudaGetLastError());
}

// Indirect shadow-boundary samples [begin, begin + n) of view v: one source path each.
static void indirect_phase(WF w, const DevScene* scenes, const DevView* vd, int v, const EdgeBuf& eb,
                           long long begin, int n, const HCube& hc, long long N, cudaStream_t st) {
  clear_counts(w, st);
  k_indirect<false><<<grid_for(n, 128, 16), 128, 0, st>>>(w, scenes, vd, v, eb, begin, n, hc, 0, nullptr);
  PSDR_LAUNCHED(1);
  WF wy = w;
  wy.D = w.D - 1;  // the source y is the second vertex of the camera path
  wy.light_vis = 0;
  depth_loop(wy, scenes, vd, MODE_FWD, st);
  k_indirect_final<<<grid_for(n, 128, 16), 128, 0, st>>>(w, scenes, vd, v, eb, n, (float)hc.ncells, N);
  PSDR_LAUNCHED(1);
  PSDR_CUDA(cudaGetLastError());
}

// Interpenetration-crease samples [begin, begin + n) of the N of view v: two paths per
// sample (slots 2s, 2s + 1), so n is at most half the tile.
static void crease_phase(WF w, const DevScene* scenes, const DevView* vd, int v, const EdgeBuf& eb,
                         const CreaseBuf& cb, const double* mw, const double* mpre, long long begin, int n,
                         long long N, cudaStream_t st) {
  clear_counts(w, st);
  k_crease_init<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, cb, mw, mpre, begin, n, N);
  PSDR_LAUNCHED(1);
  depth_loop(w, scenes, vd, MODE_FWD, st);
  k_crease_final<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, cb, n);
  PSDR_LAUNCHED(1);
  PSDR_CUDA(cudaGetLastError());
}

static CreaseBuf crease_buf(psdr_workspace* ws) {
  unsigned char* p = ws->crease.as<unsigned char>();
  CreaseBuf cb;
  cb.a = reinterpret_cast<float4*>(p);
  cb.b = reinterpret_cast<float4*>(p + 16 * (size_t)kCreaseCap);
  cb.tris = reinterpret_cast<int2*>(p + 32 * (size_t)kCreaseCap);
  cb.ra = reinterpret_cast<float4*>(p + 40 * (size_t)kCreaseCap);
  cb.rb = reinterpret_cast<float4*>(p + 56 * (size_t)kCreaseCap);
  cb.rtris = reinterpret_cast<int2*>(p + 72 * (size_t)kCreaseCap);
  cb.count = reinterpret_cast<int*>(p + 80 * (size_t)kCreaseCap);
  cb.obox = reinterpret_cast<int*>(p + 80 * (size_t)kCreaseCap + 256);
  cb.later = cb.obox + 6 * kCreaseBoxObjs;
  return cb;
}

// BSDF-jump samples [begin, begin + n) of view v at depth k (1 <= k <= D): the arc
// paths run D - k bounces (none at k = D, where only a light seen along the arc counts).
static void jump_phase(WF w, const DevScene* scenes, const DevView* vd, int v, const EdgeBuf& eb, long long begin,
                       int n, int k, cudaStream_t st) {
  const int D = w.D;
  clear_counts(w, st);
  k_jump_init<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, begin, n, k, D);
  PSDR_LAUNCHED(1);
  if (k < D) {
    WF wk = w;
    wk.D = D - k;
    wk.light_vis = 0;
    depth_loop(wk, scenes, vd, MODE_FWD, st);
  }
  k_jump_final<<<grid_for(n, 256, 8), 256, 0, st>>>(w, scenes, vd, v, eb, n, k);
  PSDR_LAUNCHED(1);
  PSDR_CUDA(cudaGetLastError());
}

long long border_segments(const DevView& V) {
  return (long long)(V.W + 1) * V.H + (long long)V.W * (V.H + 1);
}

void ensure_border(psdr_workspace* ws, const psdr_config& cfg, const std::vector<DevView>& views, cudaStream_t st) {
  if (cfg.estimator != PSDR_EST_UNBIASED) return;
  long long s = kCreaseCap, nt = 1;
  for (const DevView& v : views) {
    s = std::max(s, border_segments(v));
    nt = std::max<long long>(nt, v.scene_ntri);
  }
  ws->ensure_mass(std::max(s, nt), st);
  ws->crease.alloc(80 * (size_t)kCreaseCap + 256 + 2 * 24 * (size_t)kCreaseBoxObjs, st);
}

void set_scene_ntri(std::vector<DevView>& views, const psdr_scene* const* scenes) {
  for (DevView& v : views) v.scene_ntri = scenes[v.scene]->ntri;
}

static HCube build_hcube(psdr_workspace* ws, int ncells, const int* res, int N, bool floor, cudaStream_t st) {
  HCube hc;
  const int b = (ncells + 255) / 256;
  if (floor) {
    k_mass_cdf<<<b, 256, 0, st>>>(ws->mass.as<float>(), ncells, ws->mass_d.as<double>());
    PSDR_LAUNCHED(5);
    inclusive_scan_double(ws->mass_d.as<double>(), ws->mass_pre.as<double>(), ncells, ws->scan_tmp.as<double>(), st);
    k_mass_floor<<<b, 256, 0, st>>>(ws->mass.as<float>(), ws->mass_pre.as<double>(), ncells);
  }
  k_mass_cdf<<<b, 256, 0, st>>>(ws->mass.as<float>(), ncells, ws->mass_d.as<double>());
  PSDR_LAUNCHED(5);
  inclusive_scan_double(ws->mass_d.as<double>(), ws->mass_pre.as<double>(), ncells, ws->scan_tmp.as<double>(), st);
  k_mass_finalize<<<b, 256, 0, st>>>(ws->mass_d.as<double>(), ws->mass_pre.as<double>(), ncells,
                                     ws->hc_pmf.as<float>(), ws->hc_cmf.as<float>());
  PSDR_CUDA(cudaGetLastError());
  hc.pmf = ws->hc_pmf.as<float>();
  hc.cmf = ws->hc_cmf.as<float>();
  hc.w = ws->mass_d.as<double>();
  hc.pre = ws->mass_pre.as<double>();
  hc.ncells = ncells;
  for (int k = 0; k < 3; ++k) {
    hc.res[k] = k < N ? res[k] : 1;
    hc.unit[k] = 1.0f / (float)hc.res[k];
  }
  return hc;
}

// Backward: interior path replay + adjoint, then the primary- and direct-edge terms
// of every view. Views must carry dimage (and grad_pos when wanted).
void backward_launch(const DevScene* scenes_dev, const std::vector<DevView>& views, const psdr_config& cfg,
                     int cap, psdr_workspace* ws, const SceneGradInfo& gi, cudaStream_t st);

void render_backward_impl(const DevScene* scenes_dev, std::vector<DevView>& views, const psdr_config& cfg,
                          psdr_workspace* ws, const SceneGradInfo& gi, cudaStream_t st) {
  assign_offsets(views);
  const int cap = choose_cap(cfg, views, true);
  const int Rmax = cfg.mis_light_samples + std::max(cfg.mis_bsdf_samples, 1) + 1;
  ws->ensure(cap, Rmax, cfg.max_bounce, (int)views.size(), 1, st);
  ensure_border(ws, cfg, views, st);
  upload_views(ws, views, st);
  backward_launch(scenes_dev, views, cfg, cap, ws, gi, st);
}

// The terms of a backward job: cfg.terms, or by default interior + primary + direct edges
// (reference estimator), and for the unbiased estimator also the pixel borders, creases,
// indirect shadow boundaries and, when a DiffuseBsdfMaterial mesh is in the job, its BRDF
// jumps.
static int job_terms(const psdr_config& cfg, const SceneGradInfo& gi) {
  if (cfg.terms) return cfg.terms;
  return cfg.estimator == PSDR_EST_UNBIASED ? (111 | (gi.jump ? 16 : 0)) : 7;
}

// The units of a backward job, in the serial order: every interior tile, then per view
// its boundary terms (primary edges, direct edges, pixel borders, indirect shadow
// boundaries, creases, BRDF jumps). Costs count traced rays.
std::vector<BwdUnit> backward_units(const std::vector<DevView>& views, const psdr_config& cfg, int cap,
                                    const SceneGradInfo& gi) {
  std::vector<BwdUnit> u;
  const bool unb = cfg.estimator == PSDR_EST_UNBIASED;
  const int terms = job_terms(cfg, gi);
  const double D = cfg.max_bounce;
  const double R = cfg.mis_light_samples + cfg.mis_bsdf_samples + 1;
  const double R1 = cfg.mis_light_samples + 2;  // boundary paths of the reference estimator: one BSDF sample
  if (terms & 1)
    for (const Tile& t : plan_tiles(views, cap)) u.push_back(BwdUnit{1, -1, t, 2.0 * t.n * (1 + D * R)});
  for (int v = 0; v < (int)views.size(); ++v) {
    const DevView& V = views[v];
    const double px = (double)V.H * V.W;
    if (terms & 2) {
      const double pre = (double)cfg.primary_edge_hypercube_resolution * cfg.primary_edge_preprocess_rounds *
                         2.0 * (1 + D * R1);
      const double n = px * cfg.spp_primary_edge * (unb ? 2 + D * R : 2.0 * (1 + D * R1));
      u.push_back(BwdUnit{2, v, Tile{}, pre + n});
    }
    if (terms & 4) {
      const int* r3 = cfg.secondary_edge_hypercube_resolution;
      const double per = unb ? 3.0 + 2.0 * (D - 1) : 3.0;
      const double pre = (double)r3[0] * r3[1] * r3[2] * cfg.secondary_edge_preprocess_rounds *
                         (unb ? kDirectGuideRounds : 1) * per;
      u.push_back(BwdUnit{4, v, Tile{}, pre + px * cfg.spp_secondary_edge * per});
    }
    if (unb && (terms & 8) && cfg.spp_pixel_boundary > 0 && V.dimage)
      u.push_back(BwdUnit{8, v, Tile{}, (double)border_segments(V) * cfg.spp_pixel_boundary * (1 + D * R)});
    if (unb && (terms & 64) && V.dimage && !V.ortho && cfg.max_bounce >= 2) {
      const int* rs = cfg.secondary_edge_hypercube_resolution;
      const double cells = (double)std::max(1, rs[0] / kIndirectCellDiv) * rs[1] * rs[2];
      const double n = std::max(1.0, px * cfg.spp_secondary_edge / kIndirectSampleDiv);
      u.push_back(BwdUnit{64, v, Tile{}, (cells * cfg.secondary_edge_preprocess_rounds + n) * 3.0 +
                                             n * (D - 1) * R});
    }
    if (unb && (terms & 32) && V.dimage && !V.ortho)
      u.push_back(BwdUnit{32, v, Tile{}, 8.0 * V.scene_ntri +
                                             (double)cfg.spp_primary_edge * kCreaseSamplesPerSpp * 2.0 * (1 + D * R)});
    if (unb && (terms & 16) && gi.bsdf && V.dimage) {
      double c = 0.0;
      for (int k = 1; k <= cfg.max_bounce; ++k) c += k + 1 + (D - k) * R;
      u.push_back(BwdUnit{16, v, Tile{}, px * V.spp * c});
    }
  }
  return u;
}

std::vector<std::vector<BwdUnit>> schedule_units(const std::vector<BwdUnit>& units, int lanes) {
  lanes = std::max(1, lanes);
  std::vector<int> order(units.size());
  for (size_t i = 0; i < units.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return units[a].cost > units[b].cost; });
  std::vector<double> load(lanes, 0.0);
  std::vector<int> lane_of(units.size(), 0);
  for (int i : order) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lane_of[i] = k;
    load[k] += units[i].cost;
  }
  std::vector<std::vector<BwdUnit>> out(lanes);
  for (size_t i = 0; i < units.size(); ++i) out[lane_of[i]].push_back(units[i]);
  return out;
}

std::vector<std::vector<Tile>> schedule_tiles(const std::vector<Tile>& tiles, int lanes) {
  std::vector<BwdUnit> u;
  for (const Tile& t : tiles) u.push_back(BwdUnit{1, -1, t, (double)t.n});
  std::vector<std::vector<Tile>> out;
  for (const auto& l : schedule_units(u, lanes)) {
    out.emplace_back();
    for (const BwdUnit& x : l) out.back().push_back(x.tile);
  }
  return out;
}

// Device work of one backward unit on workspace ws (views at vd); no allocation, no
// host copy.
void backward_unit(const DevScene* scenes_dev, const std::vector<DevView>& views, const DevView* vd,
                   const BwdUnit& u, const psdr_config& cfg, int cap, psdr_workspace* ws, const SceneGradInfo& gi,
                   cudaStream_t st, const KeptRecords* keep) {
  const bool unb = cfg.estimator == PSDR_EST_UNBIASED;
  bool lens = false;  // a view wants the camera-lens gradient
  for (const DevView& V : views) lens = lens || V.grad_lens != nullptr;
  // ---- interior tile
  if (u.term == 1) {
    WF w = ws->wf;
    w.cap = ws->cap;
    set_wf(w, cfg, (int)views.size(), -1, cfg.enable_light_visable);
    w.bsdf = ws->bsdf;
    w.ortho = any_ortho(views);
    const Tile& t = u.tile;
    if (keep) {
      w.rec = keep->rec + (size_t)t.begin * w.rec_stride;
      w.view = keep->view + t.begin;
      w.pix = keep->pix + t.begin;
    } else {
      run_tile(w, scenes_dev, vd, t, MODE_REPLAY, st);
    }
    const int g = grid_for(t.n, 128, 16);
    if (gi.bsdf) {
      if (unb) k_adjoint<true, true><<<g, 128, 0, st>>>(w, scenes_dev, vd, t, gi.hot_lv0, gi.hot_nlv, gi.emit_hot);
      else k_adjoint<false, true><<<g, 128, 0, st>>>(w, scenes_dev, vd, t, gi.hot_lv0, gi.hot_nlv, gi.emit_hot);
    } else {
      if (unb) k_adjoint<true><<<g, 128, 0, st>>>(w, scenes_dev, vd, t, gi.hot_lv0, gi.hot_nlv, gi.emit_hot);
      else k_adjoint<false><<<g, 128, 0, st>>>(w, scenes_dev, vd, t, gi.hot_lv0, gi.hot_nlv, gi.emit_hot);
    }
    PSDR_LAUNCHED(1);
    if (lens) {
      if (gi.bsdf) k_lens_interior<true><<<grid_for(t.n, 256, 8), 256, 0, st>>>(w, scenes_dev, vd, t);
      else k_lens_interior<false><<<grid_for(t.n, 256, 8), 256, 0, st>>>(w, scenes_dev, vd, t);
      PSDR_LAUNCHED(1);
    }
    PSDR_CUDA(cudaGetLastError());
    return;
  }
  // ---- boundary terms of view v
  WF w = ws->wf;
  w.cap = ws->cap;
  set_wf(w, cfg, (int)views.size(), 1, 0);
  w.bsdf = ws->bsdf;
  w.ortho = any_ortho(views);
  // paths of the unbiased boundary samples carry the interior estimator's radiance
  WF wi = ws->wf;
  wi.cap = ws->cap;
  set_wf(wi, cfg, (int)views.size(), -1, cfg.enable_light_visable);
  wi.bsdf = ws->bsdf;
  wi.ortho = any_ortho(views);
  EdgeBuf eb{ws->eb_a.as<float4>(), ws->eb_n.as<float4>(), ws->eb_hb.as<float4>(), ws->eb_La.as<float4>(), nullptr};
  const int v = u.view;
  const DevView& V = views[v];
  switch (u.term) {
    case 2: {  // primary edges: preprocess over the hypercube cells, then the edge samples
      const int cells = cfg.primary_edge_hypercube_resolution;
      PSDR_CUDA(cudaMemsetAsync(ws->mass.p, 0, sizeof(float) * cells, st));
      HCube none{};
      none.unit[0] = 1.0f / (float)cells;
      for (int r = 0; r < cfg.primary_edge_preprocess_rounds; ++r)
        edge_phase(w, scenes_dev, vd, v, eb, 0, cells, none, r, true, ws->mass.as<float>(), 1, st);
      const int res[1] = {cells};
      const HCube hc = build_hcube(ws, cells, res, 1, unb, st);
      const long long N = (long long)V.H * V.W * cfg.spp_primary_edge;
      for (long long b = 0; b < N; b += cap) {
        const int nb = (int)std::min<long long>(cap, N - b);
        if (unb) edge_phase_unb(wi, scenes_dev, vd, v, eb, b, nb, hc, cfg.spp_primary_edge, st);
        else edge_phase(w, scenes_dev, vd, v, eb, b, nb, hc, 0, false, nullptr, cfg.spp_primary_edge, st);
      }
      break;
    }
    case 4: {  // direct edges
      const int* r3 = cfg.secondary_edge_hypercube_resolution;
      const int cells = r3[0] * r3[1] * r3[2];
      PSDR_CUDA(cudaMemsetAsync(ws->mass.p, 0, sizeof(float) * cells, st));
      HCube pre{};
      for (int k = 0; k < 3; ++k) { pre.res[k] = r3[k]; pre.unit[k] = 1.0f / (float)r3[k]; }
      const int rounds = cfg.secondary_edge_preprocess_rounds * (unb ? kDirectGuideRounds : 1);
      PSDR_LAUNCHED(1);
      for (int r = 0; r < rounds; ++r) {
        if (unb) launch_direct<true, true>(w, st, scenes_dev, vd, v, cells, pre, r, ws->mass.as<float>(), 1);
        else launch_direct<true, false>(w, st, scenes_dev, vd, v, cells, pre, r, ws->mass.as<float>(), 1);
      }
      const HCube hc = build_hcube(ws, cells, r3, 3, unb, st);
      const long long N = (long long)V.H * V.W * cfg.spp_secondary_edge;
      if (unb) launch_direct<false, true>(w, st, scenes_dev, vd, v, N, hc, 0, nullptr, cfg.spp_secondary_edge);
      else launch_direct<false, false>(w, st, scenes_dev, vd, v, N, hc, 0, nullptr, cfg.spp_secondary_edge);
      PSDR_CUDA(cudaGetLastError());
      break;
    }
    case 8: {  // pixel borders (unbiased estimator): segment masses, their prefix sums, samples
      const long long S = border_segments(V);
      const long long N = S * cfg.spp_pixel_boundary;
      const int b = (int)((S + 255) / 256);
      k_border_mass<<<b, 256, 0, st>>>(vd, v, ws->mass.as<float>(), S);
      k_mass_cdf<<<b, 256, 0, st>>>(ws->mass.as<float>(), (int)S, ws->mass_d.as<double>());
      PSDR_LAUNCHED(2);
      inclusive_scan_double(ws->mass_d.as<double>(), ws->mass_pre.as<double>(), (int)S, ws->scan_tmp.as<double>(),
                            st);
      for (long long b0 = 0; b0 < N; b0 += cap)
        border_phase(wi, scenes_dev, vd, v, eb, ws->mass_d.as<double>(), ws->mass_pre.as<double>(), S, b0,
                     (int)std::min<long long>(cap, N - b0), N, V.grad_lens != nullptr, st);
      break;
    }
    case 64: {  // indirect shadow boundaries: the guiding preprocess, then the samples
      const int* rs = cfg.secondary_edge_hypercube_resolution;
      const int r3[3] = {std::max(1, rs[0] / kIndirectCellDiv), rs[1], rs[2]};
      const int cells = r3[0] * r3[1] * r3[2];
      PSDR_CUDA(cudaMemsetAsync(ws->mass.p, 0, sizeof(float) * cells, st));
      HCube pre{};
      for (int k = 0; k < 3; ++k) { pre.res[k] = r3[k]; pre.unit[k] = 1.0f / (float)r3[k]; }
      for (int r = 0; r < cfg.secondary_edge_preprocess_rounds; ++r) {
        k_indirect<true><<<grid_for(cells, 128, 16), 128, 0, st>>>(w, scenes_dev, vd, v, eb, 0, cells, pre, r,
                                                                   ws->mass.as<float>());
        PSDR_LAUNCHED(1);
      }
      const HCube hc = build_hcube(ws, cells, r3, 3, true, st);
      const long long N = std::max(1LL, (long long)V.H * V.W * cfg.spp_secondary_edge / kIndirectSampleDiv);
      for (long long b0 = 0; b0 < N; b0 += cap)
        indirect_phase(wi, scenes_dev, vd, v, eb, b0, (int)std::min<long long>(cap, N - b0), hc, N, st);
      break;
    }
    case 32: {  // creases: the segments where two meshes cross, a length CDF over them, samples
      const CreaseBuf cb = crease_buf(ws);
      PSDR_CUDA(cudaMemsetAsync(cb.count, 0, sizeof(int), st));
      k_crease_box_init<<<kCreaseBoxObjs / 256, 256, 0, st>>>(scenes_dev, V.scene, cb);
      k_crease_boxes<<<grid_for(V.scene_ntri, 256, 8), 256, 0, st>>>(scenes_dev, V.scene, cb);
      k_crease_later<<<1, 32, 0, st>>>(scenes_dev, V.scene, cb);
      PSDR_LAUNCHED(3);
      k_crease_pairs<<<num_sms() * 4, 128, 0, st>>>(scenes_dev, V.scene, cb);
      k_crease_order<<<kCreaseCap / 128, 128, 0, st>>>(cb);
      k_crease_mass<<<kCreaseCap / 256, 256, 0, st>>>(cb, ws->mass_d.as<double>());
      PSDR_LAUNCHED(3);
      inclusive_scan_double(ws->mass_d.as<double>(), ws->mass_pre.as<double>(), kCreaseCap,
                            ws->scan_tmp.as<double>(), st);
      const long long N = (long long)cfg.spp_primary_edge * kCreaseSamplesPerSpp;
      const int chunk = cap / 2;
      for (long long b0 = 0; b0 < N; b0 += chunk)
        crease_phase(wi, scenes_dev, vd, v, eb, cb, ws->mass_d.as<double>(), ws->mass_pre.as<double>(), b0,
                     (int)std::min<long long>(chunk, N - b0), N, st);
      break;
    }
    case 16: {  // BSDF jumps (DiffuseBsdfMaterial scenes)
      const long long N = (long long)V.H * V.W * V.spp;
      for (int k = 1; k <= cfg.max_bounce; ++k)
        for (long long b0 = 0; b0 < N; b0 += cap)
          jump_phase(wi, scenes_dev, vd, v, eb, b0, (int)std::min<long long>(cap, N - b0), k, st);
      break;
    }
    default:
      throw Error{PSDR_ERR_INVALID_ARG, "unknown backward unit"};
  }
}

// Device work of a backward job (views already uploaded); no allocation, no host copy.
// The units run one after another on st with one workspace.
void backward_launch(const DevScene* scenes_dev, const std::vector<DevView>& views, const psdr_config& cfg,
                     int cap, psdr_workspace* ws, const SceneGradInfo& gi, cudaStream_t st) {
  const DevView* vd = ws->views.as<DevView>();
  for (const BwdUnit& u : backward_units(views, cfg, cap, gi))
    backward_unit(scenes_dev, views, vd, u, cfg, cap, ws, gi, st);
}

void grad_out(const GradAcc* acc, float* out, long long n, int accumulate, cudaStream_t st) {
  if (!out || n <= 0) return;
  k_grad_out<<<(int)((n + 255) / 256), 256, 0, st>>>(acc, out, n, accumulate);
  PSDR_LAUNCHED(1);
}

}  // namespace psdr

// ---------------------------------------------------------------- profiler C entry points
using psdr::profiler;
extern "C" {
PSDR_API psdr_status psdr_profile_enable(int32_t on) {
  try {
    psdr::Profiler& p = profiler();
    if (on && !p.d_rays) {
      PSDR_CUDA(cudaMalloc(&p.d_rays, sizeof(unsigned long long)));
      PSDR_CUDA(cudaMemset(p.d_rays, 0, sizeof(unsigned long long)));
    }
    p.on = on != 0;
  } catch (const psdr::Error& e) {
    psdr::set_error(e.msg);
    return e.code;
  }
  return PSDR_OK;
}
PSDR_API psdr_status psdr_profile_reset(void) {
  try {
    psdr::Profiler& p = profiler();
    p.used = 0;
    p.launches = 0;
    p.trace_launches = 0;
    p.replays.clear();
    if (p.d_rays) PSDR_CUDA(cudaMemset(p.d_rays, 0, sizeof(unsigned long long)));
  } catch (const psdr::Error& e) {
    psdr::set_error(e.msg);
    return e.code;
  }
  return PSDR_OK;
}
PSDR_API psdr_status psdr_profile_read(int64_t* out3, double* trace_ms) {
  try {
    psdr::Profiler& p = profiler();
    double ms = 0;
    for (size_t i = 0; i < p.used; ++i) {
      PSDR_CUDA(cudaEventSynchronize(p.ev[i].second));
      float t = 0;
      PSDR_CUDA(cudaEventElapsedTime(&t, p.ev[i].first, p.ev[i].second));
      ms += t;
    }
    for (auto& r : p.replays) {
      double g = 0;
      for (auto& e : *r.first) {
        PSDR_CUDA(cudaEventSynchronize(e.second));
        float t = 0;
        PSDR_CUDA(cudaEventElapsedTime(&t, e.first, e.second));
        g += t;
      }
      ms += g * (double)r.second;
    }
    unsigned long long rays = 0;
    if (p.d_rays) PSDR_CUDA(cudaMemcpy(&rays, p.d_rays, sizeof(rays), cudaMemcpyDeviceToHost));
    if (out3) { out3[0] = p.launches; out3[1] = p.trace_launches; out3[2] = (int64_t)rays; }
    if (trace_ms) *trace_ms = ms;
  } catch (const psdr::Error& e) {
    psdr::set_error(e.msg);
    return e.code;
  }
  return PSDR_OK;
}
}

// ================================================================== allocation-free forward
// psdr_render_fwd_noalloc renders one camera without allocating device memory: the
// wavefront buffers of each tile live in one file-scope __device__ array that every
// GPU loading this library holds until the process exits. It exists for callers that
// cannot call cudaMalloc at render time -- hosts that hand the library a fixed memory
// budget up front (plugin hosts, engines with their own pools), and latency-critical
// loops where cudaMalloc's implicit device synchronisation is not acceptable.
namespace psdr {
namespace {

// Writes the view record into the scratch from a kernel argument, so the call issues no
// host-to-device copy from host memory.
__global__ void k_put_view(DevView* dst, DevView v) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *dst = v;
}

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array for the current device. The first call on a
// device looks it up with cudaGetSymbolAddress (the host-side symbol is only a
// stand-in and must never be passed to a kernel).
unsigned char* noalloc_scratch() {
  int dev = 0;
  PSDR_CUDA(cudaGetDevice(&dev));
  PSDR_CHECK(dev >= 0 && dev < kNoAllocMaxDevices, "device index out of range for the allocation-free path");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    PSDR_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  return g_noalloc_ptr[dev];
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bytes of scratch a tile of `cap` paths needs with R rays per path and depth D.
size_t noalloc_bytes(size_t cap, int R, int D) {
  size_t b = align256(sizeof(DevView));
  b += align256(sizeof(int) * 2 * (D + 2));
  b += 2 * align256(8 * cap);              // sampler state, stream increment
  b += 2 * align256(4 * cap);              // view, pixel
  b += 4 * align256(16 * cap);             // T, L, current vertex, origin
  b += 3 * align256(4 * cap);              // queues
  b += 4 * align256(16 * cap * (size_t)R); // ray origin/direction/aux, hits
  return b;
}

}  // namespace
}  // namespace psdr

extern "C" PSDR_API psdr_status psdr_render_fwd_noalloc(psdr_scene* scene, const psdr_camera_desc* cam,
                                                        const psdr_config* cfg, float* image, void* stream) {
  using namespace psdr;
  try {
    PSDR_CHECK(scene != nullptr && cam != nullptr && cfg != nullptr && image != nullptr, "null argument");
    PSDR_CHECK(cfg->n_pass > 0 && cfg->spp_interior > 0, "n_pass and spp_interior must be > 0");
    PSDR_CHECK(cfg->max_bounce > 0 && cfg->max_bounce <= kMaxDepth, "max_bounce must be in [1, 16]");
    PSDR_CHECK(cfg->mis_light_samples >= 0 && cfg->mis_bsdf_samples >= 0, "mis sample counts must be >= 0");
    PSDR_CHECK(cam->type == PSDR_CAM_PERSPECTIVE, "only perspective cameras are supported");
    PSDR_CHECK(cam->height > 0 && cam->width > 0, "camera height and width must be > 0");
    PSDR_CHECK(scene->nlight > 0 || cfg->mis_light_samples == 0, "scene has no light to sample");
    const int R = cfg->mis_light_samples + cfg->mis_bsdf_samples + 1;
    PSDR_CHECK(R <= kMaxRays, "too many mis samples");
    const int D = cfg->max_bounce;
    // largest tile (multiple of 32 paths) that fits the fixed scratch
    size_t cap = kNoAllocScratchBytes / (100 + 64 * (size_t)R);
    cap &= ~size_t(31);
    while (cap > 32 && noalloc_bytes(cap, R, D) > kNoAllocScratchBytes) cap -= 32;
    if ((size_t)cfg->spp_interior > cap) {
      set_error("psdr_render_fwd_noalloc: spp_interior " + std::to_string(cfg->spp_interior) +
                " exceeds the allocation-free tile of " + std::to_string(cap) + " paths (32 MiB scratch)");
      return PSDR_ERR_INVALID_ARG;
    }
    int cur_dev = 0;
    PSDR_CUDA(cudaGetDevice(&cur_dev));
    if (cur_dev != scene->device) {
      set_error("psdr_render_fwd_noalloc: the scene was created on device " + std::to_string(scene->device) +
                " but device " + std::to_string(cur_dev) + " is current");
      return PSDR_ERR_INVALID_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char* base = noalloc_scratch();
    size_t off = 0;
    auto take = [&](size_t bytes) { unsigned char* p = base + off; off += align256(bytes); return p; };
    DevView* vd = reinterpret_cast<DevView*>(take(sizeof(DevView)));
    WF w{};
    w.cap = (int)cap;
    w.cnt = reinterpret_cast<int*>(take(sizeof(int) * 2 * (D + 2)));
    w.rs = reinterpret_cast<unsigned long long*>(take(8 * cap));
    w.ri = reinterpret_cast<unsigned long long*>(take(8 * cap));
    w.view = reinterpret_cast<int*>(take(4 * cap));
    w.pix = reinterpret_cast<int*>(take(4 * cap));
    w.T = reinterpret_cast<float4*>(take(16 * cap));
    w.L = reinterpret_cast<float4*>(take(16 * cap));
    w.cur = reinterpret_cast<float4*>(take(16 * cap));
    w.org = reinterpret_cast<float4*>(take(16 * cap));
    w.q0 = reinterpret_cast<int*>(take(4 * cap));
    w.q1 = reinterpret_cast<int*>(take(4 * cap));
    w.qs = reinterpret_cast<int*>(take(4 * cap));
    w.ro = reinterpret_cast<float4*>(take(16 * cap * R));
    w.rd = reinterpret_cast<float4*>(take(16 * cap * R));
    w.ra = reinterpret_cast<float4*>(take(16 * cap * R));
    w.hit = reinterpret_cast<float4*>(take(16 * cap * R));
    w.rec = nullptr;
    set_wf(w, *cfg, 1, -1, cfg->enable_light_visable);
    w.bsdf = scene->has_bsdf || scene->env_light >= 0 ? 1 : 0;
    w.ortho = cam->type == PSDR_CAM_ORTHOGRAPHIC ? 1 : 0;
    // the view record goes into the scratch too (the previous call's view is overwritten)
    DevView V;
    make_view(*cam, cfg->spp_interior, V);
    V.sample_off = 0;
    V.pix_off = 0;
    V.image = image;
    k_put_view<<<1, 32, 0, st>>>(vd, V);
    count_launches(1);
    // tiles of whole pixels, walked without building a host-side list
    const long long npix = (long long)cam->height * cam->width;
    const long long pix_per_tile = (long long)cap / cfg->spp_interior;
    for (long long p0 = 0; p0 < npix; p0 += pix_per_tile) {
      const long long np = std::min(pix_per_tile, npix - p0);
      Tile t{p0 * cfg->spp_interior, (int)(np * cfg->spp_interior), p0, (int)np};
      run_tile(w, scene->d_dev.as<DevScene>(), vd, t, MODE_FWD, st);  // clears the queue counters first
      k_film<<<grid_for(t.npix, 256, 8), 256, 0, st>>>(w, vd, t, std::max(1, cfg->n_pass), nullptr);
    }
    PSDR_CUDA(cudaGetLastError());
  } catch (const psdr::Error& e) {
    psdr::set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    psdr::set_error(e.what());
    return PSDR_ERR_CUDA;
  }
  return PSDR_OK;
}
