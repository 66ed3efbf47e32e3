// oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY (the oracle's C entry points for ctypes).
//
// Render drivers for the oracle: interior term (path_integrator.cc:355-372), primary
// boundary (:188-272) and direct boundary (:274-353), in float, double or Dual<K>, with
// the reference's derivative formulas (mode 0) or the unbiased estimator (mode 1).
// PARITY UNPINNED (see psdr_oracle.hpp). Built by oracle/build.py into
// oracle/_build/liborc.so; loaded only by tests, smoke() and the bench CPU baseline.
#include <omp.h>

#include <cstdio>
#include <memory>

#include "psdr_oracle.hpp"

namespace orc {

template <class S, bool AD> struct Ctx {
  using R = typename Traits<S>::R;
  const Scene<S>& sc;    // scene in S (Dual when differentiating)
  const Scene<R>& scv;   // value scene for the non-AD evaluations
  Camera<R> cam;
  V3<S> cam_pos;
  OrcConfig cfg;
  // Float scene/camera for the primary-edge term: its +-1e-5 rays graze silhouette
  // edges, so they are formed in float exactly as the GPU forms them.
  const Scene<float>* scf = nullptr;
  Camera<float> camf;
  V3<float> posf;
  double hc_cells = 1.0;  // hypercube cell count of the term being evaluated
};

// Raster area per unit surface area at x with normal n (up to fx*fy): |n.(x-o)|/z^3;
// orthographic: |n.look| (parallel projection).
template <class S, class R>
inline S cam_jacobian(const Camera<R>& cam, const V3<S>& x, const V3<S>& n, const V3<S>& o) {
  V3<S> rel = x - o;
  V3<S> look(S(-cam.c2w[0][2]), S(-cam.c2w[1][2]), S(-cam.c2w[2][2]));
  if (cam.ortho) return abs_(dot(n, look));
  S z = dot(rel, look);
  return abs_(dot(n, rel)) / (z * z * z);
}

// fx*fy of the map from world directions to raster coordinates. The camera's right
// and up axes are not normalised (camera.h:7-40: right = up x dir), so the raster scale
// of camera space (c2r) is divided by their lengths (the norms of w2c's first rows
// are their inverses).
template <class R>
inline double raster_fxfy(const Camera<R>& cam) {
  double r0 = 0, r1 = 0;
  for (int j = 0; j < 3; ++j) {
    r0 += double(cam.w2c[0][j]) * double(cam.w2c[0][j]);
    r1 += double(cam.w2c[1][j]) * double(cam.w2c[1][j]);
  }
  return std::fabs(double(cam.c2r[0][0]) * double(cam.c2r[1][1])) * std::sqrt(r0 * r1);
}

// Raster position of x seen from o (camera rotation fixed, translation o).
template <class S, class R>
inline V3<S> raster_of(const Camera<R>& cam, const V3<S>& x, const V3<S>& o) {
  V3<S> rel = x - o;
  V3<S> pc(S(cam.w2c[0][0]) * rel.x + S(cam.w2c[0][1]) * rel.y + S(cam.w2c[0][2]) * rel.z,
           S(cam.w2c[1][0]) * rel.x + S(cam.w2c[1][1]) * rel.y + S(cam.w2c[1][2]) * rel.z,
           S(cam.w2c[2][0]) * rel.x + S(cam.w2c[2][1]) * rel.y + S(cam.w2c[2][2]) * rel.z);
  return Camera<R>::xpos(cam.c2r, pc);
}

// camera.h:336-353 OrthographicCamera::gen_camera_ray_with_point_: the ray origin is x's
// foot on the camera plane, c2w (w2c x).xy0, here with the camera translated to o (the
// rotation fixed), so that it carries the derivatives of x and o.
template <class S, class R>
inline V3<S> ortho_origin(const Camera<R>& cam, const V3<S>& x, const V3<S>& o) {
  V3<S> rel = x - o;
  S px = S(cam.w2c[0][0]) * rel.x + S(cam.w2c[0][1]) * rel.y + S(cam.w2c[0][2]) * rel.z;
  S py = S(cam.w2c[1][0]) * rel.x + S(cam.w2c[1][1]) * rel.y + S(cam.w2c[1][2]) * rel.z;
  return o + V3<S>(S(cam.c2w[0][0]) * px + S(cam.c2w[0][1]) * py, S(cam.c2w[1][0]) * px + S(cam.c2w[1][1]) * py,
                   S(cam.c2w[2][0]) * px + S(cam.c2w[2][1]) * py);
}
// camera.h:121 look direction: c2w (0, 0, -1).
template <class S, class R> inline V3<S> look_dir(const Camera<R>& cam) {
  return V3<S>(S(-cam.c2w[0][2]), S(-cam.c2w[1][2]), S(-cam.c2w[2][2]));
}

// camera.h:235-258 PerspectiveCamera::gen_camera_ray_ (camera.h:313-334 orthographic:
// origin c2w (r2c film).xy0, direction the look direction) for sample i.
template <class S, bool AD>
inline V3<S> interior_sample(const Ctx<S, AD>& c, uint64_t i, int& pix, bool& valid) {
  using R = typename Traits<S>::R;
  const int W = c.cam.W;
  const int spp = c.cfg.spp_interior;
  Pcg32 rng = make_sampler(i + c.cfg.seed * 2654435761ull);
  R jx = rng.next_float(), jy = rng.next_float();
  pix = spp > 1 ? int(i / (uint64_t)spp) : int(i);
  int x = pix % W, y = pix / W;
  V3<R> fp(jx + R(x), jy + R(y), R(1));
  V3<R> pc = Camera<R>::xpos(c.cam.r2c, fp);
  V3<S> org = c.cam_pos;
  V3<R> d;
  if (c.cam.ortho) {
    V3<R> o = Camera<R>::xpos(c.cam.c2w, V3<R>(pc.x, pc.y, R(0)));
    org = V3<S>(S(o.x), S(o.y), S(o.z)) + (c.cam_pos - detach(c.cam_pos));
    d = look_dir<R>(c.cam);
  } else {
    d = normalize(Camera<R>::xdir(c.cam.c2w, pc));
  }
  V3<S> ds(S(d.x), S(d.y), S(d.z));
  Its<S> its = scene_hit<S, AD>(c.sc, org, ds, true);
  valid = its.valid;
  const bool unb = c.cfg.mode == 1;
  V3<S> L = trace2light<S, AD>(c.sc, rng, its, its.valid, c.cfg.mis_light_samples, c.cfg.mis_bsdf_samples,
                               c.cfg.max_bounce, c.cfg.enable_light_visable != 0, unb && AD);
  S jac = its.jac;
  if (unb && AD && its.valid) {
    // raster area per surface area at the primary vertex, as a ratio with its detached value
    S J = cam_jacobian(c.cam, its.p, its.n, c.cam_pos);
    jac = jac * (J / detach(J));
  }
  return L * jac;
}

template <class S, class R>
inline void project(const Camera<R>& cam, const V3<S>& pt, bool& valid, int& rx, int& ry) {
  V3<S> pc = Camera<R>::xpos(cam.w2c, pt);
  V3<S> p = Camera<R>::xpos(cam.c2r, pc);
  double px = val(p.x), py = val(p.y);
  valid = valid && val(pc.z) < 0 && px > 0 && px < cam.W && py > 0 && py < cam.H;
  rx = (int)std::floor(px);
  ry = (int)std::floor(py);
}

// path_integrator.cc:203-251 eval_primary_boundary. The sampled point, the offset
// rays and the two trace2light<false> paths are evaluated in float; in AD mode the
// zero-valued x_dot_n carries the derivatives of the edge vertices and camera origin.
template <class S, bool AD>
inline V3<S> eval_primary(const Ctx<S, AD>& c, Pcg32& rng, float s1, int& rx, int& ry, bool& valid) {
  const Scene<float>& sf = *c.scf;
  float s = s1, pe;
  int ei = sf.edge_cdf.sample_reuse(s, pe);
  const Edge<float>& E = sf.edges[ei];
  V3<float> xe = E.p0 + (E.p1 - E.p0) * s;
  float pdf_e = pe / E.len;
  valid = true;
  project(c.camf, xe, valid, rx, ry);
  V3<float> of = c.posf, rd;
  if (c.camf.ortho) {
    V3<float> pcf = Camera<float>::xpos(c.camf.w2c, xe);
    of = Camera<float>::xpos(c.camf.c2w, V3<float>(pcf.x, pcf.y, 0.f));
    rd = look_dir<float>(c.camf);
  } else {
    rd = normalize(xe - c.posf);
  }
  V3<float> n = cross(rd, normalize(E.p1 - E.p0));
  const float eps = 1e-5f;
  V3<float> da = rd - n * eps, db = rd + n * eps;
  Its<float> ia = scene_hit<float, false>(sf, of, da, valid);
  Its<float> ib = scene_hit<float, false>(sf, of, db, valid);
  valid = valid && ia.valid && ib.valid && (norm(ia.p - xe) < 1e-4f || norm(ib.p - xe) < 1e-4f);
  V3<float> La = trace2light<float, false>(sf, rng, ia, valid, c.cfg.mis_light_samples, 1, c.cfg.max_bounce, false);
  V3<float> Lb = trace2light<float, false>(sf, rng, ib, valid, c.cfg.mis_light_samples, 1, c.cfg.max_bounce, false);
  V3<float> dL = La - Lb;
  V3<S> value;
  if (AD) {
    const Edge<S>& Es = c.sc.edges[ei];
    V3<S> xes = Es.p0 + (Es.p1 - Es.p0) * S(s);
    V3<S> ns(S(n.x), S(n.y), S(n.z));
    V3<S> nflip(S(n.x), S(n.y), S(-n.z));
    // the ray origin: the camera position, or (orthographic) the edge point's foot on
    // the camera plane, which moves with the edge point too
    V3<S> org = c.cam.ortho ? ortho_origin(c.cam, xes, c.cam_pos) : c.cam_pos;
    S xdn = dot(xes - detach(xes), ns) + dot(org - detach(org), nflip);
    V3<S> dLs(S(dL.x), S(dL.y), S(dL.z));
    value = dLs * (xdn / S(pdf_e));
  } else {
    V3<float> v = dL / pdf_e;
    value = V3<S>(S(v.x), S(v.y), S(v.z));
  }
  valid = valid && finite3(value);
  return value;
}

// path_integrator.cc:11-24 hit_triangle
template <class S>
inline V3<S> hit_triangle(const V3<S>& o, const V3<S>& d, const V3<S>& p0, const V3<S>& e1, const V3<S>& e2) {
  V3<S> T = o - p0;
  V3<S> P = cross(d, e2), Q = cross(T, e1);
  S inv = S(1) / clamp_(dot(P, e1), 1e-5, 1 - 1e-5);
  S u = dot(P, T) * inv, v = dot(Q, d) * inv;
  return p0 + e1 * u + e2 * v;
}

// path_integrator.cc:31-78 boundary_term
template <class S, bool AD>
inline V3<S> boundary_term(const V3<S>& xs, const V3<S>& xd, const V3<S>& xb, const V3<S>& ns, const V3<S>& nd,
                           const Edge<S>& E) {
  V3<S> xs_ = detach(xs), xd_ = detach(xd), xb_ = detach(xb), ns_ = detach(ns), nd_ = detach(nd);
  V3<S> dir = normalize(xb - xs_);
  V3<S> dir_ = detach(dir);
  V3<S> ev = normalize(detach(E.p1) - detach(E.p0));
  if (val(dot(cross(dir_, ev), detach(E.out))) < 0) ev = -ev;
  V3<S> n_plane = cross(dir_, ev);
  V3<S> eproj = cross(nd_, n_plane);
  S cos_s = abs_(dot(ns_, dir_));
  S cos_b = dot(ev, dir_), cos_d = dot(eproj, dir_);
  S sin_b = safe_sqrt(S(1) - cos_b * cos_b), sin_d = safe_sqrt(S(1) - cos_d * cos_d);
  S len_sb = norm(xb_ - xs_), len_sd = norm(xd_ - xs_);
  S Jb = len_sd * len_sb * sin_b / (sin_d * cos_s);
  S dG = cos_s * dot(nd_, -dir_) / (len_sd * len_sd);
  V3<S> fb;
  if (AD) {
    V3<S> nep = cross(nd_, eproj);
    V3<S> xh = hit_triangle(xs_, dir, xd_, eproj, nep);
    xh = xh - detach(xh);
    fb = mul(xh, nep * dG);
  } else {
    fb = V3<S>(dG, dG, dG);
  }
  return fb * Jb;
}

// path_integrator.cc:288-329 eval_direct_boundary
template <class S, bool AD>
inline V3<S> eval_direct(const Ctx<S, AD>& c, typename Traits<S>::R s3[3], int& rx, int& ry, bool& valid) {
  using R = typename Traits<S>::R;
  const Scene<S>& sc = c.sc;
  R s = s3[0], pe;
  int ei = sc.edge_cdf.sample_reuse(s, pe);
  const Edge<S>& E = sc.edges[ei];
  V3<S> xb = E.p0 + (E.p1 - E.p0) * S(s);
  S pdf_e = S(pe) / E.len;
  R sy = s3[1], sz = s3[2], pch = R(1);
  int l = sc.light_cdf.sample_reuse(sy, pch);
  R pl;
  V3<S> yl = light_sample_point(sc, l, sy, sz, pl);
  R pdf_l = pl * pch;
  V3<S> dir = normalize(xb - yl);
  valid = val(dot(E.nl, dir)) * val(dot(E.nr, dir)) < 0 && val(norm(E.nl - E.nr)) > 1e-5;
  rx = ry = 0;
  Its<S> is0 = scene_hit<S, AD>(sc, xb, -dir, valid);
  valid = valid && is0.valid && is0.is_light && val(sqnorm(is0.p - yl)) < double(R(1e-5));
  Its<S> id0 = scene_hit<S, AD>(sc, xb, dir, valid);
  valid = valid && id0.valid && !id0.is_light;
  project(c.cam, id0.p, valid, rx, ry);
  V3<S> corg = c.cam_pos, cd;
  if (c.cam.ortho) {
    corg = ortho_origin(c.cam, id0.p, c.cam_pos);
    cd = look_dir<S>(c.cam);
  } else {
    cd = normalize(id0.p - c.cam_pos);
  }
  Its<S> i2 = scene_hit<S, AD>(sc, corg, cd, valid);
  valid = valid && i2.valid && !i2.is_light && val(sqnorm(i2.p - id0.p)) < double(R(1e-5));
  V3<S> value;
  if (!valid) return value;
  S pdf_xw = is0.sqd * pdf_e * S(pdf_l) / dot(is0.n, dir);
  V3<S> Tb = boundary_term<S, AD>(is0.p, id0.p, xb, is0.n, id0.n, E) / pdf_xw;
  V3<S> Ts = detach(light_emit(sc, is0));
  V3<S> Td = detach(bsdf_eval(sc, id0, -cd));
  value = mul(mul(Tb, Ts), Td);
  valid = valid && finite3(value);
  return value;
}

// ---------------------------------------------------------------- unbiased estimator
// The derivative of the image in the material form of the path integral: every path
// vertex moves with its triangle (fixed barycentrics), so the interior term differentiates
// the measurement contribution times the area and camera Jacobians. Three boundary terms
// complete it: material crossing the pixel borders, silhouettes sliding over the
// background, and shadow boundaries sliding over the receivers of direct light. All are
// zero-valued in the forward image; only their derivatives are used.

// Material point of a hit found in the value scene, in the differentiated scene.
template <class S, class T>
inline V3<S> material_point(const Scene<S>& sc, const Its<T>& h) {
  const Tri<S>& t = sc.tris[h.tri];
  return t.p0 + (t.p1 - t.p0) * S(h.b1) + (t.p2 - t.p0) * S(h.b2);
}

constexpr int kMaxChainOut = 16;  // camera connections of one shadow-boundary sample

// True when triangle tri is one of the faces of edge E.
template <class S, class T>
inline bool tri_has_edge(const Scene<S>& sc, int tri, const Edge<T>& E) {
  if (tri < 0) return false;
  const auto& f = sc.faces[tri];
  const bool h0 = f[0] == E.v0 || f[1] == E.v0 || f[2] == E.v0;
  const bool h1 = f[0] == E.v1 || f[1] == E.v1 || f[2] == E.v1;
  return h0 && h1;
}

// Silhouette term. The edge sample and its two offset rays are those of eval_primary;
// one side must land on a face of the edge (foreground), the other side (background,
// possibly empty) changes visibility at the raster velocity of the edge relative to the
// background point: -L_bg (v_edge - v_bg).n_bg per unit raster length.
template <class S, bool AD>
inline V3<S> eval_primary_unb(const Ctx<S, AD>& c, Pcg32& rng, float s1, int& rx, int& ry, bool& valid) {
  const Scene<float>& sf = *c.scf;
  float s = s1, pe;
  int ei = sf.edge_cdf.sample_reuse(s, pe);
  const Edge<float>& E = sf.edges[ei];
  V3<float> xe = E.p0 + (E.p1 - E.p0) * s;
  float pdf_e = pe / E.len;
  valid = true;
  project(c.camf, xe, valid, rx, ry);
  V3<float> of = c.posf, rd;
  if (c.camf.ortho) {
    V3<float> pcf = Camera<float>::xpos(c.camf.w2c, xe);
    of = Camera<float>::xpos(c.camf.c2w, V3<float>(pcf.x, pcf.y, 0.f));
    rd = look_dir<float>(c.camf);
  } else {
    rd = normalize(xe - c.posf);
  }
  V3<float> n = cross(rd, normalize(E.p1 - E.p0));
  const float eps = 1e-5f;
  V3<float> da = rd - n * eps, db = rd + n * eps;
  Its<float> ia = scene_hit<float, false>(sf, of, da, valid);
  Its<float> ib = scene_hit<float, false>(sf, of, db, valid);
  const bool na = ia.valid && tri_has_edge(sf, ia.tri, E), nb = ib.valid && tri_has_edge(sf, ib.tri, E);
  valid = valid && na != nb;
  const Its<float>& ig = na ? ib : ia;
  valid = valid && ig.valid;
  V3<float> Lg = trace2light<float, false>(sf, rng, ig, valid, c.cfg.mis_light_samples, c.cfg.mis_bsdf_samples,
                                           c.cfg.max_bounce, c.cfg.enable_light_visable != 0);
  V3<S> value;
  if (!valid) return value;
  if constexpr (AD) {
    const Edge<S>& Es = c.sc.edges[ei];
    V3<S> xes = Es.p0 + (Es.p1 - Es.p0) * S(s);
    V3<S> xg = material_point(c.sc, ig);
    V3<double> o(c.posf.x, c.posf.y, c.posf.z);
    V3<double> rel_e(double(xe.x) - o.x, double(xe.y) - o.y, double(xe.z) - o.z);
    V3<double> rel_g(double(ig.p.x) - o.x, double(ig.p.y) - o.y, double(ig.p.z) - o.z);
    double re = norm(rel_e), rg = norm(rel_g);
    V3<double> look(-double(c.camf.c2w[0][2]), -double(c.camf.c2w[1][2]), -double(c.camf.c2w[2][2]));
    double z = dot(rel_e, look);
    // raster area swept per unit of (normal velocity x edge length): fx fy r_e / z^3, or
    // fx fy for the parallel projection, where a translation of the camera moves the
    // edge point and the background alike and depth does not scale velocities
    const bool ortho = c.cam.ortho;
    double k = raster_fxfy(c.cam) * (ortho ? 1.0 : re / (z * z * z)) / (double(pdf_e) * c.cam.H * c.cam.W);
    V3<S> dso = c.cam_pos - detach(c.cam_pos);
    V3<S> vrel = ortho ? (xes - detach(xes)) - (xg - detach(xg))
                       : (xes - detach(xes) - dso) - (xg - detach(xg) - dso) * S(re / rg);
    V3<S> ns(S(n.x), S(n.y), S(n.z));
    S vn = dot(vrel, ns) * S(na ? 1.0 : -1.0);
    value = V3<S>(S(Lg.x), S(Lg.y), S(Lg.z)) * (vn * S(-k));
  }
  valid = valid && finite3(value);
  return value;
}

// Shadow-boundary term of direct light. Sampling and the edge/light visibility tests
// are those of eval_direct; the edge point x_b, light point y and receiver x_d lie on
// one line. The shadow boundary moves over the receiver's material at the relative
// velocity d_eff = dx_b - dx_d/lam - dy (1 - 1/lam), lam = |x_d-y|/|x_b-y|; the
// occluding faces lie on the side opposite the edge's outward vector. The change of
// the radiance leaving x_d reaches the camera directly (x_d seen from the camera) and
// through up to max_bounce-1 diffuse reflections: a chain of cosine-sampled bounces
// from x_d connects each of its vertices to the camera; each bounce multiplies the
// albedo for diffuse surfaces (pi f_r against the cosine pdf about the geometric
// normal), and the camera-visible end adds its BSDF toward the camera and its camera
// Jacobian. Returns the common derivative carrier d_eff . (w x e) and fills one
// (pixel, RGB weight) pair per camera connection (in value mode too, for the guiding
// masses: sum of |weight| |w x e| over the connections).
struct DirectOut {
  int n = 0;
  int pix[kMaxChainOut];
  V3<double> w[kMaxChainOut];
  double nsn = 0;  // |w x e|
};

template <class S, bool AD>
inline S eval_direct_unb(const Ctx<S, AD>& c, typename Traits<S>::R s3[3], Pcg32& rng, DirectOut& out) {
  using R = typename Traits<S>::R;
  const Scene<S>& sc = c.sc;
  out.n = 0;
  R s = s3[0], pe;
  int ei = sc.edge_cdf.sample_reuse(s, pe);
  const Edge<S>& E = sc.edges[ei];
  V3<S> xb = E.p0 + (E.p1 - E.p0) * S(s);
  double pdf_e = double(pe) / val(E.len);
  R sy = s3[1], sz = s3[2], pch = R(1);
  int l = sc.light_cdf.sample_reuse(sy, pch);
  R pl;
  V3<S> yl = light_sample_point(sc, l, sy, sz, pl);
  double pdf_l = double(pl) * double(pch);
  V3<S> dir = normalize(xb - yl);
  bool valid = val(dot(E.nl, dir)) * val(dot(E.nr, dir)) < 0 && val(norm(E.nl - E.nr)) > 1e-5;
  Its<S> is0 = scene_hit<S, AD>(sc, xb, -dir, valid);
  valid = valid && is0.valid && is0.is_light && val(sqnorm(is0.p - yl)) < double(R(1e-5));
  Its<S> id0 = scene_hit<S, AD>(sc, xb, dir, valid);
  valid = valid && id0.valid && !id0.is_light;
  S dn = S(0);
  if (!valid) return dn;
  {
    V3<double> xbv = val3(xb), yv = val3(yl), xdv = val3(id0.p);
    V3<double> w = normalize(xbv - yv);
    V3<double> ev = normalize(val3(E.p1) - val3(E.p0));
    if (dot(cross(w, ev), val3(E.out)) < 0) ev = -ev;
    V3<double> ns = cross(w, ev);
    out.nsn = norm(ns);
    double dby = norm(xbv - yv), lam = norm(xdv - yv) / dby;
    if constexpr (AD) {
      V3<S> deff = (xb - detach(xb)) - (id0.p - detach(id0.p)) * S(1.0 / lam) - (yl - detach(yl)) * S(1.0 - 1.0 / lam);
      dn = dot(deff, V3<S>(S(ns.x), S(ns.y), S(ns.z)));
    }
    const double cos_y = std::fabs(dot(val3(is0.n), w));
    const double k0 = -cos_y / (dby * dby) / (pdf_e * pdf_l * c.cam.H * c.cam.W);
    const double fxfy = raster_fxfy(c.cam);
    const V3<double> o = val3(c.cam_pos);
    // running throughput: the emission, times pi f_r at every vertex the chain leaves
    V3<double> T = val3(light_emit(sc, is0));
    // camera connection of a vertex whose reflection hemisphere (its normal) faces the
    // camera: T times its BSDF toward the camera times its camera Jacobian
    auto connect = [&](const Its<S>& v) {
      // toward the camera: its position, or (orthographic) against the look direction
      // from the point's foot on the camera plane
      const V3<S> to_cam = c.cam.ortho ? -look_dir<S>(c.cam) : normalize(c.cam_pos - v.p);
      if (val(dot(v.n, to_cam)) <= 0) return;
      bool vis = true;
      int rx, ry;
      project(c.cam, v.p, vis, rx, ry);
      const V3<S> co = c.cam.ortho ? ortho_origin(c.cam, v.p, c.cam_pos) : c.cam_pos;
      Its<S> iv = scene_hit<S, AD>(sc, co, -to_cam, vis);
      vis = vis && iv.valid && !iv.is_light && val(sqnorm(iv.p - v.p)) < double(R(1e-5));
      if (!vis || out.n >= kMaxChainOut) return;
      const double Jc = fxfy * val(cam_jacobian(c.cam, val3(v.p), val3(v.n), o));
      const V3<double> fr = val3(bsdf_eval(sc, v, to_cam));
      out.pix[out.n] = ry * c.cam.W + rx;
      out.w[out.n] = mul(T, fr) * (k0 * Jc);
      ++out.n;
    };
    connect(id0);
    Its<S> v = id0;
    for (int j = 1; j < c.cfg.max_bounce; ++j) {
      R ru = rng.next_float(), rv = rng.next_float(), ct;
      V3<S> wo = diffuse_sample_dir(v, ru, rv, ct);
      Its<S> nx = scene_hit<S, AD>(sc, v.p, wo, true);
      if (!nx.valid || nx.is_light) break;
      T = mul(T, val3(bsdf_eval(sc, v, wo))) * M_PI;  // cosine sampling around Ng: G / pdf = pi
      connect(nx);
      v = nx;
    }
  }
  return dn;
}

// Indirect shadow-boundary term (test restatement of the GPU term): the shadow-boundary
// geometry of eval_direct_unb with the light point replaced by the first mesh surface y seen
// from the edge point x_b in a direction w drawn uniformly inside the edge's silhouette lune
// (the directions for which exactly one of the two faces at the edge faces w: two opposite
// wedges of angle alpha between the face normals, solid angle 4 alpha; coordinates (u2, u3):
// the wedge and the position across it from u2, cos(theta) = 1 - 2 u3 along the edge). The
// radiance leaving y toward x_b comes from a path of max_bounce - 1 bounces from y (stream
// kIndirectStream + 2^28 + i); the receiver connects to the camera directly (perspective).
constexpr uint64_t kIndirectStream = 0xE0000000ull;
// a quarter of the shadow-boundary samples and of the guiding cells along the edge axis
constexpr int kIndirectSampleDiv = 4, kIndirectCellDiv = 4;
// the unbiased estimator's light-source shadow-boundary guide: four preprocess rounds per
// requested round (the reference estimator keeps one)
constexpr int kDirectGuideRounds = 4;

// Intersection record of the point with barycentrics (b1, b2) on triangle tri, reached from o
// (the construction of scene_hit for a given hit).
template <class S>
inline Its<S> its_at(const Scene<S>& sc, int tri, double b1, double b2, const V3<S>& o) {
  using R = typename Traits<S>::R;
  Its<S> its;
  const Tri<S>& tr = sc.tris[tri];
  its.valid = true;
  its.tri = tri;
  its.b1 = b1;
  its.b2 = b2;
  its.p = tr.p0 + S(R(b1)) * (tr.p1 - tr.p0) + S(R(b2)) * (tr.p2 - tr.p0);
  R u0 = R(tr.uv[0]), v0 = R(tr.uv[1]);
  its.u = double(u0 + R(b1) * (R(tr.uv[2]) - u0) + R(b2) * (R(tr.uv[4]) - u0));
  its.v = double(v0 + R(b1) * (R(tr.uv[3]) - v0) + R(b2) * (R(tr.uv[5]) - v0));
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
  its.jac = S(1);
  return its;
}

// Returns the derivative carrier d_eff . (w x e); out gets the camera connection of the
// receiver (weight without the source radiance) and the source hit.
struct IndirectOut {
  bool ok = false;
  int pix = 0;
  V3<double> w;  // k0 J_cam f_r(x_d) (the source radiance multiplies it)
  double nsn = 0;
  int ytri = -1;
  double yb1 = 0, yb2 = 0;
  V3<float> xb;
};
template <class S, bool AD>
inline S eval_indirect_unb(const Ctx<S, AD>& c, typename Traits<S>::R s3[3], IndirectOut& out) {
  using R = typename Traits<S>::R;
  const Scene<S>& sc = c.sc;
  out.ok = false;
  S dn = S(0);
  R s = s3[0], pe;
  int ei = sc.edge_cdf.sample_reuse(s, pe);
  const Edge<S>& E = sc.edges[ei];
  V3<S> xb = E.p0 + (E.p1 - E.p0) * S(s);
  double pdf_e = double(pe) / val(E.len);
  // the lune direction toward the source
  const V3<double> evd = normalize(val3(E.p1) - val3(E.p0)), nl = val3(E.nl), nr = val3(E.nr);
  const V3<double> bb = cross(evd, nl);
  const double ar = std::atan2(dot(nr, bb), dot(nr, nl)), alpha = std::fabs(ar);
  const bool second = double(s3[1]) >= 0.5;
  const double t = second ? 2 * double(s3[1]) - 1 : 2 * double(s3[1]);
  const double psi = (second ? -0.5 * M_PI : 0.5 * M_PI) + t * ar;
  const double ct = 1 - 2 * double(s3[2]), st = std::sqrt(std::max(0.0, 1 - ct * ct));
  const V3<double> wyd = evd * ct + (nl * std::cos(psi) + bb * std::sin(psi)) * st;
  const V3<S> wy(S(wyd.x), S(wyd.y), S(wyd.z));
  const V3<S> dir = -wy;
  bool valid = alpha > 1e-5 && val(dot(E.nl, dir)) * val(dot(E.nr, dir)) < 0 && !c.cam.ortho;
  Its<S> is0 = scene_hit<S, AD>(sc, xb, wy, valid);
  valid = valid && is0.valid && !is0.is_light;
  Its<S> id0 = scene_hit<S, AD>(sc, xb, dir, valid);
  valid = valid && id0.valid && !id0.is_light;
  if (!valid) return dn;
  const V3<S> yl = is0.p;
  V3<double> xbv = val3(xb), yv = val3(yl), xdv = val3(id0.p);
  V3<double> w = val3(dir);
  V3<double> ev = evd;
  if (dot(cross(w, ev), val3(E.out)) < 0) ev = -ev;
  V3<double> ns = cross(w, ev);
  double lam = norm(xdv - yv) / norm(xbv - yv);
  // the receiver seen by the camera
  const V3<S> to_cam = normalize(c.cam_pos - id0.p);
  if (val(dot(id0.n, to_cam)) <= 0) return dn;
  bool vis = true;
  int rx, ry;
  project(c.cam, id0.p, vis, rx, ry);
  Its<S> iv = scene_hit<S, AD>(sc, c.cam_pos, -to_cam, vis);
  vis = vis && iv.valid && !iv.is_light && val(sqnorm(iv.p - id0.p)) < double(R(1e-5));
  if (!vis) return dn;
  if constexpr (AD) {
    V3<S> deff = (xb - detach(xb)) - (id0.p - detach(id0.p)) * S(1.0 / lam) - (yl - detach(yl)) * S(1.0 - 1.0 / lam);
    dn = dot(deff, V3<S>(S(ns.x), S(ns.y), S(ns.z)));
  }
  const double k0 = -4 * alpha / (pdf_e * c.cam.H * c.cam.W);
  const double Jc = raster_fxfy(c.cam) * val(cam_jacobian(c.cam, val3(id0.p), val3(id0.n), val3(c.cam_pos)));
  const V3<double> fr = val3(bsdf_eval(sc, id0, to_cam));
  out.ok = true;
  out.pix = ry * c.cam.W + rx;
  out.w = fr * (k0 * Jc);
  out.nsn = norm(ns);
  out.ytri = is0.tri;
  out.yb1 = is0.b1;
  out.yb2 = is0.b2;
  out.xb = V3<float>(float(xbv.x), float(xbv.y), float(xbv.z));
  return dn;
}

// Pixel-border term. Segment q of the (W+1) x H vertical and W x (H+1) horizontal unit
// segments of the pixel grid contributes (dI[hi] - dI[lo]) . Int L v dl: L is the
// radiance seen through the border point, v the raster velocity of its primary vertex
// across the segment (material flows into pixel hi and out of pixel lo; outside the
// image dI = 0). Segments are importance-sampled by m_q = |dI[hi] - dI[lo]|_1 (float)
// with stratified inversion of the double-precision CDF: sample i of N takes
// u = (i + xi) / N, the first segment whose prefix sum exceeds u * total, and the
// remainder as its position along the segment.
struct Border {
  int H = 0, W = 0;
  long long S = 0;
  std::vector<double> w, pre;
  void pixels(long long q, bool& vert, int& k, int& j, int& lo, int& hi) const {
    const long long nv = (long long)(W + 1) * H;
    vert = q < nv;
    lo = hi = -1;
    if (vert) {
      k = int(q % (W + 1)); j = int(q / (W + 1));
      if (k >= 1) lo = j * W + k - 1;
      if (k < W) hi = j * W + k;
    } else {
      const long long r = q - nv;
      k = int(r % W); j = int(r / W);
      if (j >= 1) lo = (j - 1) * W + k;
      if (j < H) hi = j * W + k;
    }
  }
  void build(int h, int wd, const double* dLdI) {
    H = h; W = wd;
    S = (long long)(W + 1) * H + (long long)W * (H + 1);
    w.resize(S); pre.resize(S);
    double acc = 0;
    for (long long q = 0; q < S; ++q) {
      bool vert; int k, j, lo, hi;
      pixels(q, vert, k, j, lo, hi);
      float d[3];
      for (int c = 0; c < 3; ++c)
        d[c] = (hi >= 0 ? float(dLdI[3 * hi + c]) : 0.f) - (lo >= 0 ? float(dLdI[3 * lo + c]) : 0.f);
      const float m = std::fabs(d[0]) + std::fabs(d[1]) + std::fabs(d[2]);
      w[q] = double(m);
      acc += w[q];
      pre[q] = acc;
    }
  }
  long long locate(long long i, long long N, float xi, float& t, double& pmf) const {
    const double tot = pre[S - 1];
    const double u = (double(i) + double(xi)) / double(N);
    const double tt = u * tot;
    long long q = (long long)(std::upper_bound(pre.begin(), pre.end(), tt) - pre.begin());
    if (q >= S) q = S - 1;
    const double base = q > 0 ? pre[q - 1] : 0.0;
    double r = (tt - base) / w[q];
    r = r < 0.0 ? 0.0 : r;
    t = std::min(float(r), 0.99999994f);
    pmf = w[q] / tot;
    return q;
  }
};

// Border sample i of N: adds dPhi/dtheta . seed_k to dphi.
template <class S, bool AD>
inline void pixel_border_sample(const Ctx<S, AD>& c, const Border& B, uint64_t i, uint64_t N, const double* dLdI,
                                double* dphi) {
  using R = typename Traits<S>::R;
  if constexpr (AD) {
    constexpr int KD = sizeof(S) / sizeof(double) - 1;
    Pcg32 rng = make_sampler(i + c.cfg.seed * 2654435761ull);
    const float xi = rng.next_float();
    float t;
    double pmf;
    const long long q = B.locate((long long)i, (long long)N, xi, t, pmf);
    if (!(pmf > 0)) return;
    bool vert; int k, j, lo, hi;
    B.pixels(q, vert, k, j, lo, hi);
    V3<R> fp = vert ? V3<R>(R(float(k)), R(t + float(j)), R(1)) : V3<R>(R(t + float(k)), R(float(j)), R(1));
    V3<R> pc = Camera<R>::xpos(c.cam.r2c, fp);
    V3<R> o(R(val(c.cam_pos.x)), R(val(c.cam_pos.y)), R(val(c.cam_pos.z))), d;
    if (c.cam.ortho) {
      o = Camera<R>::xpos(c.cam.c2w, V3<R>(pc.x, pc.y, R(0)));
      d = look_dir<R>(c.cam);
    } else {
      d = normalize(Camera<R>::xdir(c.cam.c2w, pc));
    }
    Its<R> its = scene_hit<R, false>(c.scv, o, d, true);
    if (!its.valid) return;
    V3<R> L = trace2light<R, false>(c.scv, rng, its, true, c.cfg.mis_light_samples, c.cfg.mis_bsdf_samples,
                                    c.cfg.max_bounce, c.cfg.enable_light_visable != 0);
    V3<S> x = material_point(c.sc, its);
    V3<S> r = raster_of(c.cam, x, c.cam_pos);
    S vel = vert ? r.x - detach(r.x) : r.y - detach(r.y);
    double wgt = 0;
    for (int ch = 0; ch < 3; ++ch) {
      double g = (hi >= 0 ? dLdI[3 * hi + ch] : 0.0) - (lo >= 0 ? dLdI[3 * lo + ch] : 0.0);
      wgt += g * double(L[ch]);
    }
    wgt /= double(N) * pmf;
    if (!std::isfinite(wgt)) return;
    for (int qd = 0; qd < KD; ++qd) dphi[qd] += wgt * vel.d[qd];
  }
}

// Intersection record of a value-scene hit with the differentiated scene's frame (the
// hit triangle's normal and tangent, flipped to the side the value hit faces).
template <class S, class T>
inline Its<S> material_its(const Scene<S>& sc, const Its<T>& h) {
  Its<S> r;
  const Tri<S>& tr = sc.tris[h.tri];
  r.valid = true;
  r.is_front = h.is_front;
  r.p = material_point(sc, h);
  r.n = h.is_front ? tr.n : -tr.n;
  r.t = h.is_front ? tr.t : -tr.t;
  r.u = h.u; r.v = h.v; r.b1 = h.b1; r.b2 = h.b2;
  r.tri = h.tri; r.obj = h.obj; r.light = h.light; r.is_light = h.is_light;
  return r;
}

// BSDF-jump term of DiffuseBsdfMaterial (diffuse_bsdf.cc:56-88). With N.L >= 0 and
// N.V >= 0 the rule on t makes the value jump by color b (max(N.L, N.V) + 1e-5) where
// t = V.L - (N.L)(N.V) = m.L crosses 0, m = V - (N.V) N: over the shading hemisphere, on
// the half great circle through N perpendicular to m. In the material form the rendered
// value at x_k changes at Int_arc dF L_i (Ng.L) d/dtheta[m . L_att] / |m| dl, where L_att is
// the direction from the material point x_k to the material point x_{k+1} seen along L
// (the arc's velocity relative to the surface it sweeps, per unit arc length). Sample i
// follows one camera path of its pixel (the interior term's sampling); at each of its
// vertices on a DiffuseBsdfMaterial with roughness > 0 it draws one arc direction
// uniformly (pdf 1/pi), traces L_i with the path's remaining bounces and adds
// dPhi/dtheta . seed_k to dphi through the zero-valued carrier m . L_att. The camera
// path draws from stream i (2 jitter draws, then per vertex the arc draw and two
// direction draws); the L_i of vertex k draws from its own stream 16 i + k, so that a
// wavefront renderer can estimate each depth's L_i in a pass of its own.
constexpr uint64_t kJumpStreams = 16;  // max_bounce <= 16
template <class S, bool AD>
inline void bsdf_jump_sample(const Ctx<S, AD>& c, uint64_t i, const double* dLdI, double* dphi) {
  using R = typename Traits<S>::R;
  if constexpr (AD) {
    constexpr int KD = sizeof(S) / sizeof(double) - 1;
    const int W = c.cam.W, spp = c.cfg.spp_interior, D = c.cfg.max_bounce;
    const int nL = c.cfg.mis_light_samples, nB = c.cfg.mis_bsdf_samples;
    Pcg32 rng = make_sampler(i + c.cfg.seed * 2654435761ull);
    R jx = rng.next_float(), jy = rng.next_float();
    const int pix = spp > 1 ? int(i / (uint64_t)spp) : int(i);
    V3<R> fp(jx + R(pix % W), jy + R(pix / W), R(1));
    V3<R> pc = Camera<R>::xpos(c.cam.r2c, fp);
    V3<R> o(R(val(c.cam_pos.x)), R(val(c.cam_pos.y)), R(val(c.cam_pos.z))), d;
    if (c.cam.ortho) {
      o = Camera<R>::xpos(c.cam.c2w, V3<R>(pc.x, pc.y, R(0)));
      d = look_dir<R>(c.cam);
    } else {
      d = normalize(Camera<R>::xdir(c.cam.c2w, pc));
    }
    Its<R> its = scene_hit<R, false>(c.scv, o, d, true);
    V3<R> T(R(1), R(1), R(1));
    V3<S> xprev = c.cam_pos;  // previous material vertex (the camera for x_1)
    for (int k = 1; k <= D; ++k) {
      if (!its.valid || its.is_light) break;
      const R sigma = c.scv.obj_mat[its.obj] == 1 ? R(tex_fetch(c.scv, c.scv.obj_rough[its.obj], its.u, its.v).x) : R(0);
      const V3<R> N = shading_normal(c.scv, its);
      const R nv = dot(N, its.wi);
      const V3<R> m = its.wi - N * nv;
      const R mlen = norm(m);
      const R u_arc = rng.next_float();
      if (sigma > 0 && nv >= 0 && mlen > R(1e-7)) {
        const V3<R> w = normalize(cross(N, m));
        const R psi = (u_arc - R(0.5)) * R(M_PI);
        const V3<R> L = normalize(N * R(std::cos(psi)) + w * R(std::sin(psi)));
        const R nl = std::max(dot(N, L), R(0));
        const R a = R(1) / (R(M_PI) + R((3 * M_PI - 4) / 6) * sigma);
        const R dF = sigma * a * (std::max(nl, nv) + R(1e-5));
        Its<R> nx = scene_hit<R, false>(c.scv, its.p, L, true);
        V3<R> Li;
        if (nx.valid) {
          if (nx.is_light) Li = light_emit(c.scv, nx);
          else if (k < D) {
            Pcg32 rli = make_sampler(i * kJumpStreams + (uint64_t)k + c.cfg.seed * 2654435761ull);
            Li = trace2light<R, false>(c.scv, rli, nx, true, nL, nB, D - k, false);
          }
        }
        const V3<R> wv = mul(mul(T, tex_at(c.scv, its.obj, its.u, its.v)), Li) *
                         (dF * dot(its.n, L) * R(M_PI) / mlen / R(spp));
        double wgt = 0;
        for (int ch = 0; ch < 3; ++ch) wgt += dLdI[3 * pix + ch] * double(wv[ch]);
        if (nx.valid && wgt != 0 && std::isfinite(wgt)) {
          const Its<S> xk = material_its(c.sc, its);
          const V3<S> xn = material_point(c.sc, nx);
          V3<S> Vd = (k == 1 && c.cam.ortho) ? -V3<S>(S(d.x), S(d.y), S(d.z)) : normalize(xprev - xk.p);
          const V3<S> Nd = shading_normal(c.sc, xk);
          const V3<S> md = Vd - Nd * dot(Nd, Vd);
          const S q = dot(md, normalize(xn - xk.p));
          for (int qd = 0; qd < KD; ++qd) dphi[qd] += wgt * q.d[qd];
        }
      }
      if (k == D) break;
      // continue the camera path (cosine sampling about the shading normal)
      const R rx = rng.next_float(), ry = rng.next_float();
      R ct;
      const V3<R> wo = material_sample_dir(c.scv, its, rx, ry, ct);
      Its<R> nx = scene_hit<R, false>(c.scv, its.p, wo, true);
      if (!nx.valid) break;
      const R tmp = dot(nx.n, -wo) / nx.sqd;
      const R G = dot(its.n, wo) * tmp;
      const R pdf = ct * R(1.0 / M_PI) * tmp;
      T = mul(T, bsdf_eval(c.scv, its, wo)) * (G / pdf);
      if (!finite3(T)) break;
      xprev = material_point(c.sc, its);
      its = nx;
    }
  }
}

// sampler.h:201-247 HyperCubeSampler: cells in row-major order of the resolution.
template <class R> struct HyperCube {
  int N = 1;
  int res[3] = {1, 1, 1};
  int cells = 1;
  R unit[3];
  Discrete<R> d;
  void init(int n, const int* r) {
    N = n;
    cells = 1;
    for (int i = 0; i < n; ++i) { res[i] = r[i]; cells *= r[i]; unit[i] = R(1) / R(r[i]); }
  }
  void cell_coords(int c, int* out) const {
    int cnt = cells, rem = c;
    for (int i = 0; i < N; ++i) { cnt /= res[i]; out[i] = rem / cnt; rem -= out[i] * cnt; }
  }
  R sample_reuse(R* s) const {
    R pdf;
    int idx = d.sample_reuse(s[N - 1], pdf);
    int cc[3];
    cell_coords(idx, cc);
    for (int i = 0; i < N; ++i) s[i] = (s[i] + R(cc[i])) * unit[i];
    return pdf;
  }
  // Unbiased estimator: the cell is the first whose double-precision prefix sum exceeds
  // s_last * total (a float CDF cannot resolve cells below 2^-24 of the mass nor place a
  // sample inside them), and the position inside the cell along the last dimension is
  // a fresh uniform. Returns the cell's probability.
  std::vector<double> w, pre;
  void build_unb(const std::vector<double>& m) {
    w = m;
    pre.resize(m.size());
    double acc = 0;
    for (size_t i = 0; i < m.size(); ++i) { acc += m[i]; pre[i] = acc; }
  }
  double sample_unb(R* s, Pcg32& rng) const {
    const double tot = pre.back();
    const double t = double(s[N - 1]) * tot;
    int idx = int(std::upper_bound(pre.begin(), pre.end(), t) - pre.begin());
    if (idx >= cells) idx = cells - 1;
    int cc[3];
    cell_coords(idx, cc);
    s[N - 1] = R(rng.next_float());
    for (int i = 0; i < N; ++i) s[i] = (s[i] + R(cc[i])) * unit[i];
    return w[idx] / tot;
  }
};

// The unbiased estimator mixes a uniform share into the guiding masses (a quarter of the
// mean mass per cell, 20% of the samples): no cell whose preprocessing sample happened
// to be invalid is left unsampled, and no sample weight exceeds 5x the uniform one.
inline void mass_floor(std::vector<double>& m) {
  double tot = 0;
  for (double x : m) tot += x;
  const double f = tot > 0 ? 0.25 * tot / double(m.size()) : 1.0;
  for (double& x : m) x = double(float(float(x) + float(f)));
}

// path_integrator.cc:253-272 preprocess_primary_boundary (value mode, float)
template <class R>
inline HyperCube<R> preprocess_primary(const Ctx<R, false>& c) {
  static_assert(std::is_same<R, float>::value, "the primary-edge term is evaluated in float");
  HyperCube<R> hc;
  int r = c.cfg.pe_res;
  hc.init(1, &r);
  std::vector<double> rst(hc.cells, 0.0);
  std::vector<Pcg32> rngs(hc.cells);
  for (int i = 0; i < hc.cells; ++i) rngs[i] = make_sampler(i);
  for (int round = 0; round < c.cfg.pe_rounds; ++round) {
    std::vector<double> add(hc.cells, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < hc.cells; ++i) {
      R s1 = (R(i) + rngs[i].next_float()) * hc.unit[0];
      int rx, ry;
      bool valid;
      V3<R> v = eval_primary<R, false>(c, rngs[i], s1, rx, ry, valid);
      if (valid) add[i] = double(R(norm(v)));
    }
    for (int i = 0; i < hc.cells; ++i) rst[i] = double(R(R(rst[i]) + R(add[i])));
  }
  if (c.cfg.mode == 1) {
    mass_floor(rst);
    hc.build_unb(rst);
  }
  hc.d.build(rst);
  return hc;
}

// path_integrator.cc:331-353 preprocess_direct_boundary (value mode)
template <class R>
inline HyperCube<R> preprocess_direct(const Ctx<R, false>& c) {
  HyperCube<R> hc;
  hc.init(3, c.cfg.se_res);
  std::vector<double> rst(hc.cells, 0.0);
  std::vector<Pcg32> rngs(hc.cells);
  for (int i = 0; i < hc.cells; ++i) rngs[i] = make_sampler(i);
  const int rounds = c.cfg.se_rounds * (c.cfg.mode == 1 ? kDirectGuideRounds : 1);
  for (int round = 0; round < rounds; ++round) {
    std::vector<double> add(hc.cells, 0.0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < hc.cells; ++i) {
      int cc[3];
      hc.cell_coords(i, cc);
      R s3[3];
      for (int k = 0; k < 3; ++k) s3[k] = rngs[i].next_float();
      for (int k = 0; k < 3; ++k) s3[k] = (R(cc[k]) + s3[k]) * hc.unit[k];
      int rx, ry;
      bool valid;
      if (c.cfg.mode == 1) {
        // unbiased estimator: the magnitude of its own per-sample weights (camera
        // connections of the receiver and of its bounce chain, which uses a copy of the
        // cell's sampler so that the rounds draw the same hypercube positions)
        Pcg32 rc = rngs[i];
        DirectOut o;
        eval_direct_unb<R, false>(c, s3, rc, o);
        double m = 0;
        for (int q = 0; q < o.n; ++q) m += norm(o.w[q]);
        add[i] = double(float(m * o.nsn));
        continue;
      }
      V3<R> v = eval_direct<R, false>(c, s3, rx, ry, valid);
      for (int k = 0; k < 3; ++k) if (v[k] < R(1e-5)) v[k] = R(1e-5);
      if (valid) add[i] = double(R(norm(v)));
    }
    for (int i = 0; i < hc.cells; ++i) rst[i] = double(R(R(rst[i]) + R(add[i])));
  }
  if (c.cfg.mode == 1) {
    mass_floor(rst);
    hc.build_unb(rst);
  }
  hc.d.build(rst);
  return hc;
}

// Guiding preprocess of the indirect shadow-boundary term: per cell the magnitude of its
// sample's camera weight without the source radiance (|k0 J_cam| |f_r| |w x e|).
template <class R>
inline HyperCube<R> preprocess_indirect(const Ctx<R, false>& c) {
  HyperCube<R> hc;
  const int res[3] = {std::max(1, c.cfg.se_res[0] / kIndirectCellDiv), c.cfg.se_res[1], c.cfg.se_res[2]};
  hc.init(3, res);
  std::vector<double> rst(hc.cells, 0.0);
  std::vector<Pcg32> rngs(hc.cells);
  for (int i = 0; i < hc.cells; ++i) rngs[i] = make_sampler(kIndirectStream + (uint64_t)i);
  for (int round = 0; round < c.cfg.se_rounds; ++round) {
    std::vector<double> add(hc.cells, 0.0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < hc.cells; ++i) {
      int cc[3];
      hc.cell_coords(i, cc);
      R s3[3];
      for (int k = 0; k < 3; ++k) s3[k] = rngs[i].next_float();
      for (int k = 0; k < 3; ++k) s3[k] = (R(cc[k]) + s3[k]) * hc.unit[k];
      IndirectOut o;
      eval_indirect_unb<R, false>(c, s3, o);
      if (o.ok) add[i] = double(float(std::fabs(norm(o.w)) * o.nsn));
    }
    for (int i = 0; i < hc.cells; ++i) rst[i] = double(R(R(rst[i]) + R(add[i])));
  }
  mass_floor(rst);
  hc.build_unb(rst);
  hc.d.build(rst);
  return hc;
}

}  // namespace orc

using namespace orc;

// Interpenetration creases (unbiased estimator; test restatement of the GPU term): the
// curves where triangles of two different meshes cross. Along the projected curve the
// visible surface switches from surface 1 (the -n side) to surface 2, and the image
// changes by Int g [L1 (v_c - v_1) - L2 (v_c - v_2)] . n dl in raster units, v_c the
// curve's raster velocity (the curve stays on both surfaces: its world velocity in the
// plane of the two normals n1, n2 satisfies n_k . dx_c = n_k . dx_k) and v_k the velocity
// of surface k's material point at the crease point. The derivative is carried by
//   (G1 - G2) (A1 n1 . (X1 - o) + A2 n2 . (X2 - o)) - G1 w . (X1 - o) + G2 w . (X2 - o),
// with w = J^T n (J the raster Jacobian), c = n1 . n2, A1 = (w.n1 - c w.n2) / (1 - c^2),
// A2 = (w.n2 - c w.n1) / (1 - c^2), G_k = g . L_k, and X_k, o the differentiated material
// points and camera origin. Segments are ordered by their triangle pair and sampled by
// length, N = spp_primary_edge x 16384 stratified samples.
constexpr uint64_t kCreaseStream = 0xC0000000ull;
constexpr uint64_t kCreaseSamplesPerSpp = 16384;

struct Crease {
  std::vector<V3<float>> a, b;
  std::vector<float> len;
  std::vector<int> ta, tb;
  std::vector<double> w, pre;
  // Segment where triangles A and B cross (double arithmetic, vertices on a plane count as
  // on its positive side).
  static bool segment(const V3<double>* A, const V3<double>* B, V3<double>& s0, V3<double>& s1) {
    auto cut = [](const V3<double>* T, const V3<double>& n, double d, V3<double>& p, V3<double>& q) {
      double sd[3];
      for (int k = 0; k < 3; ++k) sd[k] = dot(n, T[k]) + d;
      const bool p0 = sd[0] >= 0, p1 = sd[1] >= 0, p2 = sd[2] >= 0;
      if (p0 == p1 && p1 == p2) return false;
      const int k = (p0 != p1 && p0 != p2) ? 0 : (p1 != p0 && p1 != p2) ? 1 : 2;
      const int i = (k + 1) % 3, j = (k + 2) % 3;
      p = T[k] + (T[i] - T[k]) * (sd[k] / (sd[k] - sd[i]));
      q = T[k] + (T[j] - T[k]) * (sd[k] / (sd[k] - sd[j]));
      return true;
    };
    const V3<double> na = cross(A[1] - A[0], A[2] - A[0]), nb = cross(B[1] - B[0], B[2] - B[0]);
    const V3<double> D = cross(na, nb);
    if (!(dot(D, D) > 1e-30 * dot(na, na) * dot(nb, nb))) return false;
    V3<double> pa, qa, pb, qb;
    if (!cut(A, nb, -dot(nb, B[0]), pa, qa) || !cut(B, na, -dot(na, A[0]), pb, qb)) return false;
    double ta0 = dot(pa, D), ta1 = dot(qa, D), tb0 = dot(pb, D), tb1 = dot(qb, D);
    if (ta0 > ta1) { std::swap(ta0, ta1); std::swap(pa, qa); }
    if (tb0 > tb1) { std::swap(tb0, tb1); std::swap(pb, qb); }
    if (!(std::max(ta0, tb0) < std::min(ta1, tb1))) return false;
    s0 = ta0 >= tb0 ? pa : pb;
    s1 = ta1 <= tb1 ? qa : qb;
    return true;
  }
  void build(const Scene<float>& sf) {
    const int nt = (int)sf.tris.size();
    auto box = [&](int t, V3<float>& lo, V3<float>& hi) {
      const Tri<float>& T = sf.tris[t];
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(T.p0[k], std::min(T.p1[k], T.p2[k]));
        hi[k] = std::max(T.p0[k], std::max(T.p1[k], T.p2[k]));
      }
    };
    auto dv = [](const V3<float>& p) { return V3<double>(p.x, p.y, p.z); };
    const int nmesh = sf.n_obj - (int)sf.light_kind.size();  // objects are meshes, then light meshes
    for (int t = 0; t < nt; ++t) {
      const int ot = sf.tris[t].obj;
      if (ot >= nmesh) continue;
      V3<float> lo, hi;
      box(t, lo, hi);
      for (int u = 0; u < nt; ++u) {
        const int ou = sf.tris[u].obj;
        if (ou <= ot || ou >= nmesh) continue;
        V3<float> l2, h2;
        box(u, l2, h2);
        if (l2.x > hi.x || h2.x < lo.x || l2.y > hi.y || h2.y < lo.y || l2.z > hi.z || h2.z < lo.z) continue;
        const V3<double> A[3] = {dv(sf.tris[t].p0), dv(sf.tris[t].p1), dv(sf.tris[t].p2)};
        const V3<double> B[3] = {dv(sf.tris[u].p0), dv(sf.tris[u].p1), dv(sf.tris[u].p2)};
        V3<double> s0, s1;
        if (!segment(A, B, s0, s1)) continue;
        const double L = norm(s1 - s0);
        if (!(L > 0)) continue;
        a.push_back(V3<float>(float(s0.x), float(s0.y), float(s0.z)));
        b.push_back(V3<float>(float(s1.x), float(s1.y), float(s1.z)));
        len.push_back(float(L));
        ta.push_back(t);
        tb.push_back(u);
      }
    }
    double acc = 0;
    for (float l : len) { w.push_back(double(l)); acc += double(l); pre.push_back(acc); }
  }
  long long locate(long long i, long long N, float xi, float& t, double& pmf) const {
    const double tot = pre.back();
    const double tt = (double(i) + double(xi)) / double(N) * tot;
    long long q = (long long)(std::upper_bound(pre.begin(), pre.end(), tt) - pre.begin());
    if (q >= (long long)pre.size()) q = (long long)pre.size() - 1;
    const double base = q > 0 ? pre[q - 1] : 0.0;
    double r = (tt - base) / w[q];
    t = std::min(float(r < 0 ? 0.0 : r), 0.99999994f);
    pmf = w[q] / tot;
    return q;
  }
};

// Barycentric weights (of p1, p2) of point x in triangle T.
inline void bary_in(const Tri<float>& T, const V3<float>& x, double& b1, double& b2) {
  const V3<double> p0(T.p0.x, T.p0.y, T.p0.z), e1 = V3<double>(T.p1.x, T.p1.y, T.p1.z) - p0,
      e2 = V3<double>(T.p2.x, T.p2.y, T.p2.z) - p0, q = V3<double>(x.x, x.y, x.z) - p0;
  const double d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2), q1 = dot(q, e1), q2 = dot(q, e2);
  const double den = d11 * d22 - d12 * d12;
  b1 = (d22 * q1 - d12 * q2) / den;
  b2 = (d11 * q2 - d12 * q1) / den;
}

template <class S, bool AD>
inline void crease_sample(const Ctx<S, AD>& c, const Crease& K, uint64_t i, uint64_t N, const double* dLdI,
                          double* dphi) {
  if constexpr (AD) {
    constexpr int KD = sizeof(S) / sizeof(double) - 1;
    const uint64_t so = c.cfg.seed * 2654435761ull;
    const Scene<float>& sf = *c.scf;
    const Camera<float>& cam = c.camf;
    Pcg32 rng = make_sampler(kCreaseStream + i + so);
    const float xi = rng.next_float();
    float t;
    double pmf;
    const long long q = K.locate((long long)i, (long long)N, xi, t, pmf);
    if (!(pmf > 0)) return;
    const V3<float> s0 = K.a[q], s1 = K.b[q];
    const V3<float> x = s0 + (s1 - s0) * t;
    const V3<float> tang = (s1 - s0) * (1.f / K.len[q]);
    const double wgt = K.w[q] / (pmf * double(N));
    const V3<float> pc = Camera<float>::xpos(cam.w2c, x), pr = Camera<float>::xpos(cam.c2r, pc);
    if (!(pc.z < 0 && pr.x > 0 && pr.x < cam.W && pr.y > 0 && pr.y < cam.H)) return;
    // raster Jacobian rows at x (gradients of u_x, u_y w.r.t. the world point)
    V3<float> g[2];
    {
      const float wden = cam.c2r[3][0] * pc.x + cam.c2r[3][1] * pc.y + cam.c2r[3][2] * pc.z + cam.c2r[3][3];
      for (int r = 0; r < 2; ++r) {
        const float u = (cam.c2r[r][0] * pc.x + cam.c2r[r][1] * pc.y + cam.c2r[r][2] * pc.z + cam.c2r[r][3]) / wden;
        const V3<float> gp((cam.c2r[r][0] - u * cam.c2r[3][0]) / wden, (cam.c2r[r][1] - u * cam.c2r[3][1]) / wden,
                           (cam.c2r[r][2] - u * cam.c2r[3][2]) / wden);
        for (int k = 0; k < 3; ++k)
          g[r][k] = cam.w2c[0][k] * gp.x + cam.w2c[1][k] * gp.y + cam.w2c[2][k] * gp.z;
      }
    }
    const float mx = dot(g[0], tang), my = dot(g[1], tang);
    const float rlen = std::sqrt(mx * mx + my * my);
    if (!(rlen > 0)) return;
    const float nx = -my / rlen, ny = mx / rlen;
    const int oa = sf.tris[K.ta[q]].obj, ob = sf.tris[K.tb[q]].obj;
    const float off = 5.f * 1e-3f;  // 5 ray epsilons (tmin) in world units, scaled to pixels below
    const float tol = 10.f * off;
    Its<float> hs[2];
    int objs[2];
    for (int side = 0; side < 2; ++side) {
      const float sg = (side ? off : -off) * rlen;
      const V3<float> pcam = Camera<float>::xpos(cam.r2c, V3<float>(pr.x + sg * nx, pr.y + sg * ny, 1.f));
      const V3<float> d = normalize(Camera<float>::xdir(cam.c2w, pcam));
      hs[side] = scene_hit<float, false>(sf, c.posf, d, true);
      objs[side] = hs[side].valid && norm(hs[side].p - x) < tol ? hs[side].obj : -1;
    }
    if (!(objs[0] >= 0 && objs[1] >= 0 && objs[0] != objs[1] && (objs[0] == oa || objs[0] == ob) &&
          (objs[1] == oa || objs[1] == ob)))
      return;
    V3<float> Ls[2];
    for (int side = 0; side < 2; ++side) {
      Pcg32 rs = make_sampler(kCreaseStream + 0x10000000ull + 2 * i + (uint64_t)side + so);
      Ls[side] = trace2light<float, false>(sf, rs, hs[side], true, c.cfg.mis_light_samples, c.cfg.mis_bsdf_samples,
                                           c.cfg.max_bounce, c.cfg.enable_light_visable != 0);
    }
    const int px = std::min(cam.W - 1, (int)std::floor(pr.x)), py = std::min(cam.H - 1, (int)std::floor(pr.y));
    const double* gp = dLdI + 3 * ((size_t)py * cam.W + px);
    double G[2];
    for (int side = 0; side < 2; ++side)
      G[side] = gp[0] * double(Ls[side].x) + gp[1] * double(Ls[side].y) + gp[2] * double(Ls[side].z);
    if (!std::isfinite(G[0]) || !std::isfinite(G[1])) return;
    const int t1 = objs[0] == oa ? K.ta[q] : K.tb[q], t2 = objs[0] == oa ? K.tb[q] : K.ta[q];
    const V3<double> n1 = normalize(V3<double>(sf.tris[t1].n.x, sf.tris[t1].n.y, sf.tris[t1].n.z));
    const V3<double> n2 = normalize(V3<double>(sf.tris[t2].n.x, sf.tris[t2].n.y, sf.tris[t2].n.z));
    const V3<double> wv = V3<double>(g[0].x, g[0].y, g[0].z) * double(nx) + V3<double>(g[1].x, g[1].y, g[1].z) * double(ny);
    const double cc = dot(n1, n2), sn2 = 1 - cc * cc;
    if (!(sn2 > 1e-6)) return;
    const double A1 = (dot(wv, n1) - cc * dot(wv, n2)) / sn2, A2 = (dot(wv, n2) - cc * dot(wv, n1)) / sn2;
    double b1, b2, c1, c2;
    bary_in(sf.tris[t1], x, b1, b2);
    bary_in(sf.tris[t2], x, c1, c2);
    const Tri<S>& T1 = c.sc.tris[t1];
    const Tri<S>& T2 = c.sc.tris[t2];
    const V3<S> X1 = T1.p0 + (T1.p1 - T1.p0) * S(b1) + (T1.p2 - T1.p0) * S(b2) - c.cam_pos;
    const V3<S> X2 = T2.p0 + (T2.p1 - T2.p0) * S(c1) + (T2.p2 - T2.p0) * S(c2) - c.cam_pos;
    auto dotc = [](const V3<double>& a, const V3<S>& b) { return b.x * S(a.x) + b.y * S(a.y) + b.z * S(a.z); };
    const S f = (dotc(n1, X1) * S(A1) + dotc(n2, X2) * S(A2)) * S(G[0] - G[1]) - dotc(wv, X1) * S(G[0]) +
                dotc(wv, X2) * S(G[1]);
    const double k = wgt * double(rlen);
    for (int qd = 0; qd < KD; ++qd) dphi[qd] += k * f.d[qd];
  }
}

// Film::add (camera.h:75-87): per pixel sum of the samples, divided by spp.
template <class S, bool AD>
static void render_camera(const Ctx<S, AD>& c, int which, double* img, const double* dLdI, double* dphi,
                          double* per_sample, const Ctx<typename Traits<S>::R, false>* cv,
                          const Ctx<float, false>* cf) {
  using R = typename Traits<S>::R;
  const int H = c.cam.H, W = c.cam.W;
  const size_t npix = (size_t)H * W;
  constexpr int KD = std::is_same<S, R>::value ? 0 : sizeof(S) / sizeof(double) - 1;
  const bool unb = c.cfg.mode == 1;
  // ---- interior
  if (which & 1) {
    const int spp = c.cfg.spp_interior;
    const uint64_t N = (uint64_t)npix * spp;
    std::vector<R> samp(N * 3, R(0));
    std::vector<double> phi_s(KD ? N * KD : 0, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      if constexpr (KD > 0) {
        // derivatives only: a sample of a pixel with zero weight adds nothing to dphi (the
        // image buffer is not an output of the derivative queries)
        const int64_t p = i / spp;
        if (!per_sample && dLdI[3 * p] == 0.0 && dLdI[3 * p + 1] == 0.0 && dLdI[3 * p + 2] == 0.0) continue;
      }
      int pix;
      bool valid;
      V3<S> L = interior_sample<S, AD>(c, (uint64_t)i, pix, valid);
      if (!valid) L = V3<S>();
      for (int k = 0; k < 3; ++k) samp[3 * i + k] = R(val(L[k]));
      if constexpr (KD > 0) {
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < KD; ++j) phi_s[i * KD + j] += dLdI[3 * pix + k] * L[k].d[j] / spp;
      }
      if (per_sample) for (int k = 0; k < 3; ++k) per_sample[3 * i + k] = double(val(L[k]));
    }
    for (size_t p = 0; p < npix; ++p)
      for (int k = 0; k < 3; ++k) {
        R acc = R(0);
        for (int s = 0; s < spp; ++s) acc += samp[3 * (p * spp + s) + k];
        img[3 * p + k] += double(acc / R(spp));
      }
    if constexpr (KD > 0) for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
  }
  // ---- primary boundary (renderD only; zero-valued, gradient only)
  if (which & 2) {
    HyperCube<float> hc = preprocess_primary<float>(*cf);
    const int spp = c.cfg.spp_primary_edge;
    const uint64_t N = (uint64_t)npix * spp;
    std::vector<double> phi_s(KD ? N * KD : 0, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      Pcg32 rng = make_sampler((uint64_t)i + c.cfg.seed * 2654435761ull);
      float s1 = rng.next_float();
      const double hp = unb ? hc.sample_unb(&s1, rng) : double(hc.sample_reuse(&s1));
      int rx, ry;
      bool valid;
      V3<S> v = unb ? eval_primary_unb<S, AD>(c, rng, s1, rx, ry, valid) : eval_primary<S, AD>(c, rng, s1, rx, ry, valid);
      if (!valid) continue;
      const double dens = double(hp) * (unb ? double(hc.cells) : 1.0);
      if constexpr (KD > 0) {
        size_t pix = (size_t)ry * W + rx;
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < KD; ++j) phi_s[i * KD + j] += dLdI[3 * pix + k] * v[k].d[j] / dens / spp;
      }
    }
    if constexpr (KD > 0) for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
  }
  // ---- direct boundary
  if (which & 4) {
    HyperCube<R> hc = preprocess_direct<R>(*cv);
    const int spp = c.cfg.spp_secondary_edge;
    const uint64_t N = (uint64_t)npix * spp;
    std::vector<double> phi_s(KD ? N * KD : 0, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      Pcg32 rng = make_sampler((uint64_t)i + c.cfg.seed * 2654435761ull);
      R s3[3];
      for (int k = 0; k < 3; ++k) s3[k] = rng.next_float();
      const double hp = unb ? hc.sample_unb(s3, rng) : double(hc.sample_reuse(s3));
      if (unb) {
        if constexpr (KD > 0) {
          DirectOut o;
          const S dn = eval_direct_unb<S, AD>(c, s3, rng, o);
          const double dens = hp * double(hc.cells) * spp;
          for (int q = 0; q < o.n; ++q) {
            double wg = 0;
            for (int k = 0; k < 3; ++k) wg += dLdI[3 * o.pix[q] + k] * o.w[q][k];
            if (!std::isfinite(wg)) continue;
            for (int j = 0; j < KD; ++j) phi_s[i * KD + j] += wg * dn.d[j] / dens;
          }
        }
        continue;
      }
      int rx, ry;
      bool valid;
      V3<S> v = eval_direct<S, AD>(c, s3, rx, ry, valid);
      if (!valid) continue;
      const double dens = double(hp);
      if constexpr (KD > 0) {
        size_t pix = (size_t)ry * W + rx;
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < KD; ++j) phi_s[i * KD + j] += dLdI[3 * pix + k] * v[k].d[j] / dens / spp;
      }
    }
    if constexpr (KD > 0) for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
  }
  // ---- pixel borders (unbiased estimator only)
  if ((which & 8) && unb && c.cfg.spp_pixel_boundary > 0) {
    if constexpr (KD > 0) {
      Border B;
      B.build(H, W, dLdI);
      if (B.pre[B.S - 1] > 0) {
        const uint64_t N = (uint64_t)B.S * c.cfg.spp_pixel_boundary;
        std::vector<double> phi_s(N * KD, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)N; ++i) pixel_border_sample<S, AD>(c, B, (uint64_t)i, N, dLdI, &phi_s[i * KD]);
        for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
      }
    }
  }
  // ---- indirect shadow boundaries (unbiased estimator only, perspective cameras, D >= 2)
  if ((which & 64) && unb && !c.cam.ortho && c.cfg.max_bounce >= 2) {
    if constexpr (KD > 0) {
      HyperCube<R> hc = preprocess_indirect<R>(*cv);
      const uint64_t N = std::max<uint64_t>(1, (uint64_t)npix * c.cfg.spp_secondary_edge / kIndirectSampleDiv);
      const uint64_t so = c.cfg.seed * 2654435761ull;
      std::vector<double> phi_s(N * KD, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t i = 0; i < (int64_t)N; ++i) {
        Pcg32 rng = make_sampler(kIndirectStream + (uint64_t)i + so);
        R s3[3];
        for (int k = 0; k < 3; ++k) s3[k] = rng.next_float();
        const double hp = hc.sample_unb(s3, rng);
        IndirectOut o;
        const S dn = eval_indirect_unb<S, AD>(c, s3, o);
        if (!o.ok) continue;
        // the radiance leaving y toward x_b: a path of max_bounce - 1 bounces from y
        Pcg32 ry = make_sampler(kIndirectStream + 0x10000000ull + (uint64_t)i + so);
        Its<float> iy = its_at(*c.scf, o.ytri, o.yb1, o.yb2, o.xb);
        V3<float> Lo = trace2light<float, false>(*c.scf, ry, iy, true, c.cfg.mis_light_samples,
                                                 c.cfg.mis_bsdf_samples, c.cfg.max_bounce - 1, false);
        double wg = 0;
        for (int k = 0; k < 3; ++k) wg += dLdI[3 * o.pix + k] * o.w[k] * double(Lo[k]);
        if (!std::isfinite(wg)) continue;
        const double dens = hp * double(hc.cells) * (double(N) / double(npix));
        for (int j = 0; j < KD; ++j) phi_s[i * KD + j] += wg * dn.d[j] / dens;
      }
      for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
    }
  }
  // ---- interpenetration creases (unbiased estimator only, perspective cameras)
  if ((which & 32) && unb && !c.cam.ortho) {
    if constexpr (KD > 0) {
      Crease K;
      K.build(*c.scf);
      if (!K.pre.empty() && K.pre.back() > 0) {
        const uint64_t N = (uint64_t)c.cfg.spp_primary_edge * kCreaseSamplesPerSpp;
        std::vector<double> phi_s(N * KD, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)N; ++i) crease_sample<S, AD>(c, K, (uint64_t)i, N, dLdI, &phi_s[i * KD]);
        for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
      }
    }
  }
  // ---- BSDF jumps of DiffuseBsdfMaterial (unbiased estimator only)
  if ((which & 16) && unb &&
      std::find(c.sc.obj_mat.begin(), c.sc.obj_mat.end(), 1) != c.sc.obj_mat.end()) {
    if constexpr (KD > 0) {
      const uint64_t N = (uint64_t)npix * c.cfg.spp_interior;
      std::vector<double> phi_s(N * KD, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t i = 0; i < (int64_t)N; ++i) bsdf_jump_sample<S, AD>(c, (uint64_t)i, dLdI, &phi_s[i * KD]);
      for (uint64_t i = 0; i < N; ++i) for (int j = 0; j < KD; ++j) dphi[j] += phi_s[i * KD + j];
    }
  }
}

template <class S>
static Scene<S> mk_scene(const OrcMesh* m, int nm, const OrcLight* l, int nl, const Seeds<S>& seeds) {
  return build_scene<S>(m, nm, l, nl, seeds);
}

template <class S, bool AD>
static int render_impl(const OrcMesh* m, int nm, const OrcLight* l, int nl, const OrcCamera* cams, int nc,
                       const OrcConfig* cfg, int which, double* images, const double* dLdI, double* dphi,
                       double* per_sample, const Seeds<S>& seeds) {

  using R = typename Traits<S>::R;
  Scene<S> sc = mk_scene<S>(m, nm, l, nl, seeds);
  Seeds<R> none;
  Scene<R> scv_own;
  const Scene<R>* scv;
  if constexpr (std::is_same<S, R>::value) scv = &sc;
  else { scv_own = mk_scene<R>(m, nm, l, nl, none); scv = &scv_own; }
  Scene<float> scf_own;
  const Scene<float>* scf = nullptr;
  if (which & (2 | 32 | 64)) {
    if constexpr (std::is_same<S, float>::value) scf = &sc;
    else { scf_own = mk_scene<float>(m, nm, l, nl, Seeds<float>{}); scf = &scf_own; }
  }
  size_t off = 0;
  for (int ci = 0; ci < nc; ++ci) {
    Ctx<S, AD> c{sc, *scv, {}, {}, *cfg};
    c.cam.setup(cams[ci]);
    Ctx<R, false> cv{*scv, *scv, {}, {}, *cfg};
    cv.cam = c.cam;
    Camera<float> camf;
    camf.setup(cams[ci]);
    V3<float> posf(cams[ci].look_from[0], cams[ci].look_from[1], cams[ci].look_from[2]);
    c.scf = scf; c.camf = camf; c.posf = posf;
    cv.scf = scf; cv.camf = camf; cv.posf = posf;
    std::unique_ptr<Ctx<float, false>> cf;
    if (scf) {
      cf.reset(new Ctx<float, false>{*scf, *scf, camf, posf, *cfg});
      cf->scf = scf; cf->camf = camf; cf->posf = posf;
    }
    for (int k = 0; k < 3; ++k) {
      c.cam_pos[k] = Seeder<S>::make(cams[ci].look_from[k], seeds.campos, 3 * ci + k);
      cv.cam_pos[k] = R(cams[ci].look_from[k]);
    }
    size_t npix = (size_t)c.cam.H * c.cam.W;
    std::vector<double> img(3 * npix, 0.0);
    for (int pass = 0; pass < std::max(1, cfg->n_pass); ++pass)
      render_camera<S, AD>(c, which, img.data(), dLdI ? dLdI + off : nullptr, dphi, per_sample, &cv, cf.get());
    if (images) for (size_t i = 0; i < 3 * npix; ++i) images[off + i] = img[i] / std::max(1, cfg->n_pass);
    off += 3 * npix;
    if (per_sample) per_sample += 3 * npix * cfg->spp_interior;
  }
  return 0;
}

extern "C" {

int orc_num_threads() { return omp_get_max_threads(); }

// Raw PCG32 outputs for (initstate, initseq) (pins the restatement to the published
// pcg-basic demo vector).
void orc_pcg32(uint64_t initstate, uint64_t initseq, int n, uint32_t* out) {
  Pcg32 p;
  p.seed(initstate, initseq);
  for (int i = 0; i < n; ++i) out[i] = p.next();
}
// First n floats of sampler stream i (sampler.h:11-17 seeding).
void orc_sampler_floats(uint64_t i, int n, float* out) {
  Pcg32 p = make_sampler(i);
  for (int k = 0; k < n; ++k) out[k] = p.next_float();
}
void orc_set_threads(int n) { omp_set_num_threads(n); }

// sampler.h:86-117 DiscreteSampler over the weights w[0..n) (float instance): for each of
// the m uniforms u, the sampled index, the rescaled uniform and the index's pmf.
int orc_discrete_sample(const double* w, int n, const float* u, int m, int* idx, float* u_out, float* pmf) {
  Discrete<float> d;
  d.build(std::vector<double>(w, w + n));
  for (int i = 0; i < m; ++i) {
    float s = u[i], p;
    idx[i] = d.sample_reuse(s, p);
    u_out[i] = s;
    pmf[i] = p;
  }
  return 0;
}

// Image render (interior term). precision 0 = float, 1 = double.
int orc_render(const OrcMesh* m, int nm, const OrcLight* l, int nl, const OrcCamera* cams, int nc,
               const OrcConfig* cfg, int precision, double* images, double* per_sample) {
  if (precision == 0) return render_impl<float, false>(m, nm, l, nl, cams, nc, cfg, 1, images, nullptr, nullptr, per_sample, Seeds<float>{});
  return render_impl<double, false>(m, nm, l, nl, cams, nc, cfg, 1, images, nullptr, nullptr, per_sample, Seeds<double>{});
}

// Directional derivatives dPhi/dtheta . seed_k (k < 8) of Phi = sum dLdI * image, with the
// reference's renderD semantics. which: bit0 interior, bit1 primary edges, bit2 direct edges,
// bit3 pixel-border segments, bit4 DiffuseBsdfMaterial jumps (both unbiased estimator only).
int orc_grad_dir(const OrcMesh* m, int nm, const OrcLight* l, int nl, const OrcCamera* cams, int nc,
                 const OrcConfig* cfg, int which, const double* dLdI, const double* seed_verts,
                 const double* seed_tex, const double* seed_emit, const double* seed_cam, double* dphi_out) {
  using D = Dual<8>;
  Seeds<D> s;
  s.verts = seed_verts; s.tex = seed_tex; s.emit = seed_emit; s.campos = seed_cam;
  double dphi[8] = {0};
  int rc = render_impl<D, true>(m, nm, l, nl, cams, nc, cfg, which, nullptr, dLdI, dphi, nullptr, s);
  for (int k = 0; k < 8; ++k) dphi_out[k] = dphi[k];
  return rc;
}

// Closest-hit queries in float (bit-exact KAT reference). rays: n x 6 (o, d).
int orc_intersect(const OrcMesh* m, int nm, const OrcLight* l, int nl, const float* rays, int n, int use_bvh,
                  int* tri, float* bary, float* tout) {
  Seeds<float> none;
  Scene<float> sc = build_scene<float>(m, nm, l, nl, none);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    Hit<float> h = intersect(sc, rays + 6 * i, rays + 6 * i + 3, use_bvh != 0);
    tri[i] = h.tri;
    bary[2 * i] = h.tri >= 0 ? h.b1 : -1.f;
    bary[2 * i + 1] = h.tri >= 0 ? h.b2 : -1.f;
    if (tout) tout[i] = h.tri >= 0 ? h.t : -1.f;
  }
  return 0;
}

// Edge list (float instance): v0, v1 global vertex ids; geo: 16 floats per edge
// (p0, p1, out, n_left, n_right, length).
int orc_edges(const OrcMesh* m, int nm, const OrcLight* l, int nl, int cap, int* v01, float* geo) {
  Seeds<float> none;
  Scene<float> sc = build_scene<float>(m, nm, l, nl, none);
  int ne = (int)sc.edges.size();
  for (int i = 0; i < ne && i < cap; ++i) {
    const auto& e = sc.edges[i];
    v01[2 * i] = e.v0; v01[2 * i + 1] = e.v1;
    const V3<float>* vs[5] = {&e.p0, &e.p1, &e.out, &e.nl, &e.nr};
    for (int q = 0; q < 5; ++q) for (int k = 0; k < 3; ++k) geo[16 * i + 3 * q + k] = (*vs[q])[k];
    geo[16 * i + 15] = e.len;
  }
  return ne;
}

}  // extern "C"
