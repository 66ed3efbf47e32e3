// capi.cu -- the extern "C" entry points declared in include/psdr.h.
#include <algorithm>
#include <climits>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "render.h"

namespace psdr {

thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }

void scene_build_geometry(psdr_scene* s, cudaStream_t st);
void psdr_scene_alloc(psdr_scene* s);

namespace {

__global__ void k_intersect(DevScene sc, const float* __restrict__ rays, long long n, int* __restrict__ tri,
                            float* __restrict__ bary, float* __restrict__ tout, int brute) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float* r = rays + 8 * i;
    const float3 o = f3(r[0], r[1], r[2]), d = f3(r[4], r[5], r[6]);
    const float tmin = r[3], tmax = r[7];
    HitRec h;
    if (brute == 0) {
      h = trace_closest(sc, o, d, tmin, tmax);
    } else if (brute == 2) {
      // the resumable traversal of the wavefront closest-hit kernel (trace_step)
      struct Stk {
        int a[kStack];
        __device__ void push(int i, int v) { a[i] = v; }
        __device__ int pop(int i) const { return a[i]; }
      } stk;
      TraceState s;
      trace_begin(s, o, d, tmin, tmax, -INFINITY, sc.root);
      if (sc.ntri > 0)
        while (!trace_step(sc, s, stk)) {
        }
      h = s.h;
    } else {
      h.tri = -1; h.t = tmax; h.b1 = h.b2 = 0.f;
      const RayPre rp = ray_pre(o, d);
      for (int t = 0; t < sc.ntri; ++t) {
        const float4* q = sc.tri + 6 * (size_t)t;
        float tt, b1, b2;
        if (tri_test(rp, xyz(q[0]), xyz(q[1]), xyz(q[2]), tmin, h.t, tt, b1, b2))
          if (tt < h.t || h.tri < 0 || t < h.tri) { h.t = tt; h.tri = t; h.b1 = b1; h.b2 = b2; }
      }
    }
    tri[i] = h.tri;
    if (bary) { bary[2 * i] = h.tri >= 0 ? h.b1 : -1.f; bary[2 * i + 1] = h.tri >= 0 ? h.b2 : -1.f; }
    if (tout) tout[i] = h.tri >= 0 ? h.t : -1.f;
  }
}

__global__ void k_edges_out(const float4* __restrict__ e, const int2* __restrict__ ev, int n, int* __restrict__ v01,
                            float* __restrict__ geo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = e[4 * i], b = e[4 * i + 1], c = e[4 * i + 2], d = e[4 * i + 3];
  const float g[16] = {a.x, a.y, a.z, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w, a.w};
  for (int k = 0; k < 16; ++k) geo[16 * i + k] = g[k];
  v01[2 * i] = ev[i].x;
  v01[2 * i + 1] = ev[i].y;
}

void check_tex(const psdr_texture_desc& t, const char* what, bool allow_none) {
  if (t.kind == PSDR_TEX_NONE && allow_none) return;
  PSDR_CHECK(t.kind == PSDR_TEX_CONSTANT || t.kind == PSDR_TEX_UV, std::string(what) + ": bad texture kind");
  PSDR_CHECK(t.channels == 1 || t.channels == 3, std::string(what) + ": channels must be 1 or 3");
  PSDR_CHECK(t.data != nullptr, std::string(what) + ": null texture data");
  if (t.kind == PSDR_TEX_UV) PSDR_CHECK(t.height > 0 && t.width > 0, std::string(what) + ": empty texture");
}

void check_cfg(const psdr_config* c) {
  PSDR_CHECK(c != nullptr, "null config");
  PSDR_CHECK(c->n_pass > 0, "n_pass must be > 0");
  PSDR_CHECK(c->spp_interior > 0, "spp_interior must be > 0");
  PSDR_CHECK(c->spp_primary_edge > 0, "spp_primary_edge must be > 0");
  PSDR_CHECK(c->spp_secondary_edge > 0, "spp_secondary_edge must be > 0");
  PSDR_CHECK(c->max_bounce > 0 && c->max_bounce <= kMaxDepth, "max_bounce must be in [1, 16]");
  PSDR_CHECK(c->mis_light_samples >= 0 && c->mis_bsdf_samples >= 0, "mis sample counts must be >= 0");
  PSDR_CHECK(c->mis_light_samples + std::max(c->mis_bsdf_samples, 1) + 1 <= kMaxRays, "too many mis samples");
  PSDR_CHECK(c->primary_edge_preprocess_rounds > 0 && c->secondary_edge_preprocess_rounds > 0,
             "preprocess rounds must be > 0");
  PSDR_CHECK(c->primary_edge_hypercube_resolution > 0, "primary hypercube resolution must be > 0");
  for (int k = 0; k < 3; ++k)
    PSDR_CHECK(c->secondary_edge_hypercube_resolution[k] > 0, "secondary hypercube resolution must be > 0");
  PSDR_CHECK(c->estimator == PSDR_EST_REFERENCE || c->estimator == PSDR_EST_UNBIASED, "bad estimator");
  PSDR_CHECK(c->tile_paths >= 0, "tile_paths must be >= 0");
  PSDR_CHECK(c->spp_pixel_boundary >= 0, "spp_pixel_boundary must be >= 0");
  PSDR_CHECK(c->trace_queue >= 0 && c->trace_queue <= 8, "trace_queue must be in [0, 8]");
  PSDR_CHECK(c->batch_lanes >= 0 && c->batch_lanes <= 8, "batch_lanes must be in [0, 8]");
  PSDR_CHECK(c->batch_records >= -1 && c->batch_records <= 1, "batch_records must be -1, 0 or 1");
}

void check_cams(const psdr_camera_desc* cams, int n) {
  PSDR_CHECK(cams != nullptr && n > 0, "no cameras");
  for (int i = 0; i < n; ++i) {
    PSDR_CHECK(cams[i].type == PSDR_CAM_PERSPECTIVE || cams[i].type == PSDR_CAM_ORTHOGRAPHIC, "bad camera type");
    PSDR_CHECK(cams[i].height > 0 && cams[i].width > 0, "camera height and width must be > 0");
    PSDR_CHECK(cams[i].fov > 0.f, "camera fov / view width must be > 0");
  }
}

DevScene* dev_scene(psdr_scene* s) { return s->d_dev.as<DevScene>(); }

}  // namespace

SceneGradInfo grad_info(const psdr_scene* s) {
  SceneGradInfo gi;
  gi.bsdf = s->has_bsdf || s->env_light >= 0 ? 1 : 0;
  gi.jump = s->has_bsdf ? 1 : 0;
  const int nm = (int)s->meshes.size();
  if (s->nlight == 1) {
    gi.emit_hot = 1;
    if (s->obj_nvert[nm] <= kMaxLightVerts) {
      gi.hot_lv0 = s->obj_vert_off[nm];
      gi.hot_nlv = s->obj_nvert[nm];
    }
  }
  return gi;
}

void check_config(const psdr_config* c) { check_cfg(c); }
void check_cameras(const psdr_camera_desc* cams, int n) { check_cams(cams, n); }

// Elements of an environment light's parameter gradient (cube map or SH coefficients).
long long light_param_count(const psdr_scene* s, int l) {
  const DevLight& L = s->h_lights[l];
  if (L.kind == PSDR_LIGHT_ENV) return (long long)L.tex.h * L.tex.w * 3;
  return L.kind == PSDR_LIGHT_SH9 ? 27 : 0;
}


// Min and max of n indices into out[0] / out[1] (initialised to INT_MAX / INT_MIN):
// grid-stride loads, warp reduction, one atomic pair per warp.
__global__ void k_index_range(const int* __restrict__ idx, long long n, int* __restrict__ out) {
  int lo = INT_MAX, hi = INT_MIN;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int v = __ldg(idx + i);
    lo = min(lo, v);
    hi = max(hi, v);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, lo);
    atomicMax(out + 1, hi);
  }
}

}  // namespace psdr

using namespace psdr;

#define API_BEGIN try {
#define API_END                                                          \
  }                                                                      \
  catch (const psdr::Error& e) {                                         \
    psdr::set_error(e.msg);                                              \
    return e.code;                                                       \
  }                                                                      \
  catch (const std::bad_alloc&) {                                        \
    psdr::set_error("host allocation failed");                          \
    return PSDR_ERR_OOM;                                                 \
  }                                                                      \
  catch (const std::exception& e) {                                      \
    psdr::set_error(e.what());                                           \
    return PSDR_ERR_CUDA;                                                \
  }                                                                      \
  return PSDR_OK;

// Every face index of a mesh or area light in [0, num_vertices), every uv index in
// [0, num_uvs): one min/max reduction per index buffer and one host read. Throws
// PSDR_ERR_INVALID_ARG naming the first buffer out of range.
static void check_index_ranges(const psdr_scene_desc* desc, void* stream) {
  PSDR_CHECK(desc != nullptr, "null argument");
  PSDR_CHECK(desc->num_meshes >= 0 && desc->num_lights >= 0, "negative counts");
  PSDR_CHECK(desc->num_meshes == 0 || desc->meshes != nullptr, "null mesh array");
  PSDR_CHECK(desc->num_lights == 0 || desc->lights != nullptr, "null light array");
  // (index buffer, entries, bound, what) of every mesh's faces and uv indices and every
  // area light's faces; environment lights have no caller index buffers
  struct Job { const int* p; long long n; int bound; std::string what; };
  std::vector<Job> jobs;
  for (int i = 0; i < desc->num_meshes; ++i) {
    const psdr_mesh_desc& m = desc->meshes[i];
    PSDR_CHECK(m.num_faces >= 0 && m.num_vertices >= 0 && m.num_uvs >= 0, "negative counts");
    PSDR_CHECK(m.num_faces == 0 || m.faces != nullptr, "null face buffer");
    jobs.push_back({m.faces, 3LL * m.num_faces, m.num_vertices, "mesh " + std::to_string(i) + " face"});
    if (m.uvs != nullptr && m.uv_indices != nullptr)
      jobs.push_back({m.uv_indices, 3LL * m.num_faces, m.num_uvs, "mesh " + std::to_string(i) + " uv"});
  }
  for (int l = 0; l < desc->num_lights; ++l) {
    const psdr_area_light_desc& L = desc->lights[l];
    if (L.type != PSDR_LIGHT_AREA) continue;
    PSDR_CHECK(L.num_faces >= 0 && L.num_vertices >= 0, "negative counts");
    PSDR_CHECK(L.num_faces == 0 || L.faces != nullptr, "null face buffer");
    jobs.push_back({L.faces, 3LL * L.num_faces, L.num_vertices, "light " + std::to_string(l) + " face"});
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int k = (int)jobs.size();
  if (k == 0) return;
  DBuf range;
  range.alloc(sizeof(int) * 2 * k, st);
  std::vector<int> h(2 * k);
  for (int j = 0; j < k; ++j) { h[2 * j] = INT_MAX; h[2 * j + 1] = INT_MIN; }
  PSDR_CUDA(cudaMemcpyAsync(range.p, h.data(), sizeof(int) * 2 * k, cudaMemcpyHostToDevice, st));
  for (int j = 0; j < k; ++j) {
    if (jobs[j].n == 0) continue;
    const int blocks = (int)std::min<long long>((jobs[j].n + 255) / 256, 148LL * 8);
    k_index_range<<<blocks, 256, 0, st>>>(jobs[j].p, jobs[j].n, range.as<int>() + 2 * j);
  }
  PSDR_CUDA(cudaGetLastError());
  PSDR_CUDA(cudaMemcpyAsync(h.data(), range.p, sizeof(int) * 2 * k, cudaMemcpyDeviceToHost, st));
  PSDR_CUDA(cudaStreamSynchronize(st));
  for (int j = 0; j < k; ++j) {
    if (jobs[j].n == 0) continue;
    PSDR_CHECK(h[2 * j] >= 0 && h[2 * j + 1] < jobs[j].bound,
               jobs[j].what + " indices must lie in [0, " + std::to_string(jobs[j].bound) + "): found [" +
                   std::to_string(h[2 * j]) + ", " + std::to_string(h[2 * j + 1]) + "]");
  }
}

extern "C" {

const char* psdr_last_error(void) { return psdr::g_err.c_str(); }
const char* psdr_version(void) { return "torch_psdr_b200 0.1.0 (sm_100a)"; }
int32_t psdr_abi_version(void) { return 6; }

// emitter.cc:103-119: the environment lights' bounding-box mesh. Vertex v has x = max if
// bit 2, y = max if bit 1, z = max if bit 0; the faces and the cube-map uvs (a 4 x 3 cross)
// are the reference's tables.
const int kEnvFaces[36] = {0, 1, 2, 3, 2, 1, 4, 5, 6, 7, 6, 5, 0, 4, 1, 5, 1, 4,
                           2, 6, 3, 7, 3, 6, 4, 0, 6, 2, 6, 0, 5, 1, 7, 3, 7, 1};
const float kEnvUvs[28] = {0.25f, 0.f, 0.5f, 0.f, 0.f, 1.f / 3, 0.25f, 1.f / 3, 0.5f, 1.f / 3,
                           0.75f, 1.f / 3, 1.f, 1.f / 3, 0.f, 2.f / 3, 0.25f, 2.f / 3, 0.5f, 2.f / 3,
                           0.75f, 2.f / 3, 1.f, 2.f / 3, 0.25f, 1.f, 0.5f, 1.f};
const int kEnvUvIndices[36] = {2, 3, 7, 8, 7, 3, 5, 4, 10, 9, 10, 4, 0, 1, 3, 4, 3, 1,
                               12, 13, 8, 9, 8, 13, 5, 6, 10, 11, 10, 6, 4, 3, 9, 8, 9, 3};

psdr_status psdr_scene_create(const psdr_scene_desc* desc, void* stream, psdr_scene** out) {
  API_BEGIN
  PSDR_CHECK(desc != nullptr && out != nullptr, "null argument");
  PSDR_CHECK(desc->num_meshes >= 0 && desc->num_lights >= 0, "negative counts");
  PSDR_CHECK(desc->num_meshes + desc->num_lights > 0, "scene has no geometry");
  PSDR_CHECK(desc->num_meshes == 0 || desc->meshes != nullptr, "null mesh array");
  PSDR_CHECK(desc->num_lights == 0 || desc->lights != nullptr, "null light array");
  *out = nullptr;
  psdr_scene* s = new psdr_scene();
  s->stream = (cudaStream_t)stream;
  try {
    // the device that will hold the scene (argument errors below are reported first on a
    // machine without one; its first allocation reports a missing device)
    if (cudaGetDevice(&s->device) != cudaSuccess) {
      s->device = -1;
      cudaGetLastError();
    }
    const int nm = desc->num_meshes, nl = desc->num_lights;
    s->meshes.assign(desc->meshes, desc->meshes + nm);
    s->lights.assign(desc->lights, desc->lights + nl);
    s->nobj = nm + nl;
    s->nlight = nl;
    // environment light (scene.cc:15-53): at most one, appended after the other lights
    for (int l = 0; l < nl; ++l) {
      const psdr_area_light_desc& L = s->lights[l];
      PSDR_CHECK(L.type == PSDR_LIGHT_AREA || L.type == PSDR_LIGHT_ENV || L.type == PSDR_LIGHT_SH9, "bad light type");
      if (L.type == PSDR_LIGHT_AREA) continue;
      PSDR_CHECK(l == nl - 1, "the environment light (EnvLight / SH9Light) must be the last light, and only one");
      PSDR_CHECK(nm > 0, "an environment light needs a mesh in the scene");
      for (int k = 0; k < 3; ++k) PSDR_CHECK(L.box_max[k] > L.box_min[k], "empty environment light box");
      if (L.type == PSDR_LIGHT_ENV) {
        check_tex(L.cube_map, "cube_map", false);
        PSDR_CHECK(L.cube_map.kind == PSDR_TEX_UV && L.cube_map.channels == 3, "cube map must be a UV3f texture");
      }
      s->env_light = l;
      cudaStream_t st = s->stream;
      for (int v = 0; v < 8; ++v) {
        s->env_host_v[3 * v] = (v & 4) ? L.box_max[0] : L.box_min[0];
        s->env_host_v[3 * v + 1] = (v & 2) ? L.box_max[1] : L.box_min[1];
        s->env_host_v[3 * v + 2] = (v & 1) ? L.box_max[2] : L.box_min[2];
      }
      s->env_v.alloc(sizeof(float) * 24, st);
      s->env_f.alloc(sizeof(int) * 36, st);
      s->env_uv.alloc(sizeof(float) * 28, st);
      s->env_uvi.alloc(sizeof(int) * 36, st);
      PSDR_CUDA(cudaMemcpyAsync(s->env_v.p, s->env_host_v, sizeof(float) * 24, cudaMemcpyHostToDevice, st));
      PSDR_CUDA(cudaMemcpyAsync(s->env_f.p, kEnvFaces, sizeof(int) * 36, cudaMemcpyHostToDevice, st));
      PSDR_CUDA(cudaMemcpyAsync(s->env_uv.p, kEnvUvs, sizeof(float) * 28, cudaMemcpyHostToDevice, st));
      PSDR_CUDA(cudaMemcpyAsync(s->env_uvi.p, kEnvUvIndices, sizeof(int) * 36, cudaMemcpyHostToDevice, st));
      PSDR_CUDA(cudaStreamSynchronize(st));
      s->lights[l].vertices = s->env_v.as<float>();
      s->lights[l].num_vertices = 8;
      s->lights[l].faces = s->env_f.as<int>();
      s->lights[l].num_faces = 12;
    }
    int voff = 0, toff = 0;
    size_t texoff = 0;
    for (int o = 0; o < s->nobj; ++o) {
      const bool is_mesh = o < nm;
      const float* V = is_mesh ? s->meshes[o].vertices : s->lights[o - nm].vertices;
      const int* F = is_mesh ? s->meshes[o].faces : s->lights[o - nm].faces;
      const int nV = is_mesh ? s->meshes[o].num_vertices : s->lights[o - nm].num_vertices;
      const int nF = is_mesh ? s->meshes[o].num_faces : s->lights[o - nm].num_faces;
      PSDR_CHECK(V != nullptr && F != nullptr, "null vertex or face buffer");
      PSDR_CHECK(nV > 0 && nF > 0, "empty mesh");
      s->obj_vert_off.push_back(voff);
      s->obj_tri_off.push_back(toff);
      s->obj_nvert.push_back(nV);
      s->obj_ntri.push_back(nF);
      DevObj ob{};
      ob.mat = 0;
      ob.light = is_mesh ? -1 : o - nm;
      ob.color.kind = -1;
      ob.rough.kind = -1;
      ob.normal.kind = -1;
      if (is_mesh) {
        const psdr_mesh_desc& m = s->meshes[o];
        PSDR_CHECK(m.material == PSDR_MAT_DIFFUSE || m.material == PSDR_MAT_DIFFUSE_BSDF, "bad material");
        check_tex(m.color, "color", false);
        PSDR_CHECK(m.color.channels == 3, "color texture must have 3 channels");
        PSDR_CHECK((m.uvs == nullptr) == (m.uv_indices == nullptr) || m.uvs == nullptr || m.uv_indices == nullptr,
                   "uvs / uv_indices mismatch");
        ob.mat = m.material;
        ob.color = DevTex{m.color.kind, m.color.channels, m.color.kind == PSDR_TEX_UV ? m.color.height : 1,
                          m.color.kind == PSDR_TEX_UV ? m.color.width : 1, m.color.data, nullptr};
        const size_t cnt = (size_t)ob.color.h * ob.color.w * ob.color.ch;
        s->tex_grad_off.push_back(texoff);
        texoff += cnt;
      } else {
        s->tex_grad_off.push_back(SIZE_MAX);
      }
      s->h_objs.push_back(ob);
      voff += nV;
      toff += nF;
    }
    // DiffuseBsdfMaterial: roughness (1 channel) and optional normal map (3 channels);
    // their accumulators follow every color texture, roughness then normal per mesh
    auto tex_of = [](const psdr_texture_desc& t) {
      return DevTex{t.kind, t.channels, t.kind == PSDR_TEX_UV ? t.height : 1, t.kind == PSDR_TEX_UV ? t.width : 1,
                    t.data, nullptr};
    };
    for (int o = 0; o < nm; ++o) {
      const psdr_mesh_desc& m = s->meshes[o];
      DevObj& ob = s->h_objs[o];
      size_t ro = SIZE_MAX, no = SIZE_MAX;
      if (m.material == PSDR_MAT_DIFFUSE_BSDF) {
        s->has_bsdf = true;
        check_tex(m.roughness, "roughness", false);
        PSDR_CHECK(m.roughness.channels == 1, "roughness texture must have 1 channel");
        check_tex(m.normal, "normal", true);
        PSDR_CHECK(m.normal.kind == PSDR_TEX_NONE || m.normal.channels == 3, "normal texture must have 3 channels");
        ob.rough = tex_of(m.roughness);
        ro = texoff;
        texoff += (size_t)ob.rough.h * ob.rough.w;
        if (m.normal.kind != PSDR_TEX_NONE) {
          ob.normal = tex_of(m.normal);
          no = texoff;
          texoff += (size_t)ob.normal.h * ob.normal.w * 3;
        }
      }
      s->rough_grad_off.push_back(ro);
      s->nrm_grad_off.push_back(no);
    }
    s->nvert = voff;
    s->ntri = toff;
    for (int l = 0; l < nl; ++l) {
      const psdr_area_light_desc& D = s->lights[l];
      DevLight L{};
      L.tri0 = s->obj_tri_off[nm + l];
      L.ntri = s->obj_ntri[nm + l];
      for (int k = 0; k < 3; ++k) L.emit[k] = D.emit[k];
      L.kind = D.type;
      L.tex.kind = -1;
      size_t go = SIZE_MAX;
      if (D.type == PSDR_LIGHT_ENV) {
        L.tex = DevTex{PSDR_TEX_UV, 3, D.cube_map.height, D.cube_map.width, D.cube_map.data, nullptr};
        go = texoff;
        texoff += (size_t)D.cube_map.height * D.cube_map.width * 3;
      } else if (D.type == PSDR_LIGHT_SH9) {
        for (int k = 0; k < 27; ++k) L.sh[k] = D.sh9[k];
        go = texoff;
        texoff += 27;
      }
      s->light_grad_off.push_back(go);
      s->h_lights.push_back(L);
    }
    s->dev.ltri_base = nl > 0 ? s->obj_tri_off[nm] : 0;
    // the build gathers vertices and uvs through the index buffers: check them first
    check_index_ranges(desc, stream);
    psdr_scene_alloc(s);
    // fp64 gradient accumulators live with the scene
    cudaStream_t st = s->stream;
    s->g_verts.alloc(sizeof(GradAcc) * 3 * s->nvert, st);
    s->g_tex.alloc(sizeof(GradAcc) * std::max<size_t>(1, texoff), st);
    s->g_emit.alloc(sizeof(GradAcc) * 3 * std::max(1, nl), st);
    s->dev.grad_verts = s->g_verts.as<GradAcc>();
    s->vmask.alloc(std::max<size_t>(1, s->nvert), st);
    PSDR_CUDA(cudaMemsetAsync(s->vmask.p, 1, std::max<size_t>(1, s->nvert), st));
    s->dev.vmask = s->vmask.as<unsigned char>();
    for (int o = 0; o < nm; ++o) {
      s->h_objs[o].color.grad = s->g_tex.as<GradAcc>() + s->tex_grad_off[o];
      if (s->rough_grad_off[o] != SIZE_MAX) s->h_objs[o].rough.grad = s->g_tex.as<GradAcc>() + s->rough_grad_off[o];
      if (s->nrm_grad_off[o] != SIZE_MAX) s->h_objs[o].normal.grad = s->g_tex.as<GradAcc>() + s->nrm_grad_off[o];
    }
    for (int l = 0; l < nl; ++l) {
      s->h_lights[l].grad_emit = s->g_emit.as<GradAcc>() + 3 * l;
      if (s->light_grad_off[l] == SIZE_MAX) continue;
      GradAcc* g = s->g_tex.as<GradAcc>() + s->light_grad_off[l];
      if (s->h_lights[l].kind == PSDR_LIGHT_ENV) s->h_lights[l].tex.grad = g;
      else s->h_lights[l].grad_sh = g;
    }
    s->upload_tables();
    scene_build_geometry(s, s->stream);
  } catch (...) {
    delete s;
    throw;
  }
  *out = s;
  API_END
}

psdr_status psdr_scene_validate(const psdr_scene_desc* desc, void* stream) {
  API_BEGIN
  check_index_ranges(desc, stream);
  API_END
}

psdr_status psdr_scene_destroy(psdr_scene* scene) {
  API_BEGIN
  delete scene;
  API_END
}

psdr_status psdr_scene_update(psdr_scene* scene, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene != nullptr, "null scene");
  scene_build_geometry(scene, stream ? (cudaStream_t)stream : scene->stream);
  API_END
}

psdr_status psdr_scene_refit(psdr_scene* scene, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene != nullptr, "null scene");
  scene_refit_geometry(scene, stream ? (cudaStream_t)stream : scene->stream);
  API_END
}

psdr_status psdr_scene_set_leaf_size(psdr_scene* scene, int32_t leaf_size, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene != nullptr, "null scene");
  PSDR_CHECK(leaf_size >= 1 && leaf_size <= 8, "leaf_size must be in [1, 8]");
  scene->leaf_size = leaf_size;
  scene_build_geometry(scene, stream ? (cudaStream_t)stream : scene->stream);
  API_END
}

psdr_status psdr_scene_info(psdr_scene* scene, int64_t* info) {
  API_BEGIN
  PSDR_CHECK(scene != nullptr && info != nullptr, "null argument");
  int ne = 0;
  PSDR_CUDA(cudaMemcpyAsync(&ne, scene->n_edges.p, sizeof(int), cudaMemcpyDeviceToHost, scene->stream));
  PSDR_CUDA(cudaStreamSynchronize(scene->stream));
  info[0] = scene->ntri;
  info[1] = scene->nvert;
  info[2] = ne;
  info[3] = std::max(0, scene->ntri - 1);
  info[4] = scene->nlight;
  info[5] = scene->nobj;
  API_END
}

psdr_status psdr_scene_edges(psdr_scene* scene, int32_t* v01, float* geo, int64_t cap, int64_t* n_out, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene && v01 && geo && n_out, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int ne = 0;
  PSDR_CUDA(cudaStreamSynchronize(scene->stream));
  PSDR_CUDA(cudaMemcpy(&ne, scene->n_edges.p, sizeof(int), cudaMemcpyDeviceToHost));
  *n_out = ne;
  const int n = (int)std::min<int64_t>(ne, cap);
  if (n > 0)
    k_edges_out<<<(n + 255) / 256, 256, 0, st>>>(scene->edge.as<float4>(), scene->edge_v.as<int2>(), n, v01, geo);
  PSDR_CUDA(cudaGetLastError());
  PSDR_CUDA(cudaStreamSynchronize(st));
  API_END
}

psdr_status psdr_intersect(psdr_scene* scene, const float* rays, int64_t n, int32_t* tri, float* bary, float* t,
                           int32_t brute_force, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene && (rays || n == 0) && (tri || n == 0), "null argument");
  PSDR_CHECK(n >= 0, "negative ray count");
  if (n == 0) return PSDR_OK;
  const int blocks = (int)std::min<int64_t>((n + 127) / 128, (int64_t)num_sms() * 16);
  k_intersect<<<blocks, 128, 0, (cudaStream_t)stream>>>(scene->dev, rays, n, tri, bary, t, brute_force);
  PSDR_CUDA(cudaGetLastError());
  API_END
}

psdr_status psdr_workspace_create(psdr_workspace** out) {
  API_BEGIN
  PSDR_CHECK(out != nullptr, "null argument");
  *out = new psdr_workspace();
  API_END
}

psdr_status psdr_workspace_destroy(psdr_workspace* ws) {
  API_BEGIN
  delete ws;
  API_END
}

psdr_status psdr_render_fwd(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cams, int32_t n_cams,
                            const psdr_config* cfg, float** images, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene && ws && images, "null argument");
  check_cfg(cfg);
  check_cams(cams, n_cams);
  ws->bsdf = scene->has_bsdf || scene->env_light >= 0 ? 1 : 0;  // extended kernel instances
  PSDR_CHECK(scene->nlight > 0 || cfg->mis_light_samples == 0, "scene has no light to sample");
  std::vector<DevView> views(n_cams);
  for (int i = 0; i < n_cams; ++i) {
    PSDR_CHECK(images[i] != nullptr, "null image buffer");
    make_view(cams[i], cfg->spp_interior, views[i]);
    views[i].image = images[i];
  }
  render_forward_impl(dev_scene(scene), views, *cfg, ws, (cudaStream_t)stream, nullptr);
  API_END
}

psdr_status psdr_render_samples(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cam,
                                const psdr_config* cfg, float* samples, void* stream) {
  API_BEGIN
  PSDR_CHECK(scene && ws && samples, "null argument");
  check_cfg(cfg);
  check_cams(cam, 1);
  ws->bsdf = scene->has_bsdf || scene->env_light >= 0 ? 1 : 0;  // extended kernel instances
  PSDR_CHECK(scene->nlight > 0 || cfg->mis_light_samples == 0, "scene has no light to sample");
  std::vector<DevView> views(1);
  make_view(*cam, cfg->spp_interior, views[0]);
  render_forward_impl(dev_scene(scene), views, *cfg, ws, (cudaStream_t)stream, samples);
  API_END
}

psdr_status psdr_autotune(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cams, int32_t n_cams,
                          psdr_config* cfg, int32_t* best_leaf, float* best_ms, void* stream) {
  struct Ev {
    cudaEvent_t e = nullptr;
    ~Ev() { if (e) cudaEventDestroy(e); }
  };
  API_BEGIN
  PSDR_CHECK(scene && ws && cfg, "null argument");
  check_cfg(cfg);
  check_cams(cams, n_cams);
  ws->bsdf = scene->has_bsdf || scene->env_light >= 0 ? 1 : 0;  // extended kernel instances
  PSDR_CHECK(scene->nlight > 0 || cfg->mis_light_samples == 0, "scene has no light to sample");
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<DevView> views(n_cams);
  size_t floats = 0;
  for (int i = 0; i < n_cams; ++i) floats += 3 * (size_t)cams[i].height * cams[i].width;
  DBuf img;
  img.alloc(sizeof(float) * floats, st);
  size_t off = 0;
  for (int i = 0; i < n_cams; ++i) {
    make_view(cams[i], cfg->spp_interior, views[i]);
    views[i].image = img.as<float>() + off;
    off += 3 * (size_t)cams[i].height * cams[i].width;
  }
  Ev ev0, ev1;
  PSDR_CUDA(cudaEventCreate(&ev0.e));
  PSDR_CUDA(cudaEventCreate(&ev1.e));
  cudaEvent_t e0 = ev0.e, e1 = ev1.e;
  const int leaves[3] = {1, 2, 4};
  const int tiles[4] = {1 << 18, 1 << 19, 1 << 20, 1 << 21};
  const int queues[3] = {4, 6, 8};
  float best = INFINITY;
  int bl = scene->leaf_size, bt = cfg->tile_paths, bq = cfg->trace_queue;
  for (int leaf : leaves) {
    scene->leaf_size = leaf;
    scene_build_geometry(scene, st);
    for (int trial = 0; trial < 12; ++trial) {
      const int tile = tiles[trial % 4], queue = queues[trial / 4];
      psdr_config c = *cfg;
      c.tile_paths = tile;
      c.trace_queue = queue;
      std::vector<DevView> v = views;
      render_forward_impl(dev_scene(scene), v, c, ws, st, nullptr);  // warm-up, sizes the workspace
      PSDR_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < 2; ++r) render_forward_impl(dev_scene(scene), v, c, ws, st, nullptr);
      PSDR_CUDA(cudaEventRecord(e1, st));
      PSDR_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      PSDR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      ms *= 0.5f;
      if (ms < best) { best = ms; bl = leaf; bt = tile; bq = queue; }
    }
  }
  scene->leaf_size = bl;
  scene_build_geometry(scene, st);
  PSDR_CUDA(cudaStreamSynchronize(st));
  cfg->tile_paths = bt;
  cfg->trace_queue = bq;
  if (best_leaf) *best_leaf = bl;
  if (best_ms) *best_ms = best;
  API_END
}

psdr_status psdr_camera_lens_jacobian(const psdr_camera_desc* cam, double* m9, double* p90) {
  API_BEGIN
  PSDR_CHECK(cam != nullptr, "null argument");
  check_cams(cam, 1);
  PSDR_CHECK(cam->type == PSDR_CAM_PERSPECTIVE, "the lens map is defined for perspective cameras");
  LensChain ch;
  double m[9];
  lens_chain(*cam, ch, m);
  if (m9) std::copy(m, m + 9, m9);
  if (p90) std::copy(&ch.P[0][0], &ch.P[0][0] + 90, p90);
  API_END
}

psdr_status psdr_render_bwd(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cams, int32_t n_cams,
                            const psdr_config* cfg, const float** d_images, const psdr_grad_targets* grads,
                            void* stream) {
  API_BEGIN
  PSDR_CHECK(scene && ws && d_images && grads, "null argument");
  check_cfg(cfg);
  check_cams(cams, n_cams);
  ws->bsdf = scene->has_bsdf || scene->env_light >= 0 ? 1 : 0;  // extended kernel instances
  PSDR_CHECK(scene->nlight > 0, "scene has no light");
  const bool unb = cfg->estimator == PSDR_EST_UNBIASED;
  std::vector<LensChain> chains(n_cams);
  for (int i = 0; grads->camera_lens && i < n_cams; ++i) {
    if (!grads->camera_lens[i]) continue;
    if (cams[i].type != PSDR_CAM_PERSPECTIVE)
      throw Error{PSDR_ERR_UNSUPPORTED, "camera_lens gradients are implemented for perspective cameras only"};
    if (unb) lens_chain(cams[i], chains[i]);
  }
  cudaStream_t st = (cudaStream_t)stream;
  // only the vertices whose gradient the caller asked for are accumulated
  {
    std::vector<unsigned char> m(std::max(1, scene->nvert), 0);
    for (int o = 0; o < scene->nobj; ++o)
      if (grads->vertices && grads->vertices[o])
        std::fill(m.begin() + scene->obj_vert_off[o], m.begin() + scene->obj_vert_off[o] + scene->obj_nvert[o], 1);
    PSDR_CUDA(cudaMemcpyAsync(scene->vmask.p, m.data(), m.size(), cudaMemcpyHostToDevice, st));
    // and only the textures asked for: their accumulators stay in the object table
    std::vector<DevObj> objs = scene->h_objs;
    for (int o = 0; o < (int)scene->meshes.size(); ++o) {
      if (!(grads->textures && grads->textures[o])) objs[o].color.grad = nullptr;
      if (!(grads->roughness && grads->roughness[o])) objs[o].rough.grad = nullptr;
      if (!(grads->normal && grads->normal[o])) objs[o].normal.grad = nullptr;
    }
    PSDR_CUDA(cudaMemcpyAsync(scene->objs.p, objs.data(), sizeof(DevObj) * std::max<size_t>(1, objs.size()),
                              cudaMemcpyHostToDevice, st));
  }
  PSDR_CUDA(cudaMemsetAsync(scene->g_verts.p, 0, scene->g_verts.bytes, st));
  PSDR_CUDA(cudaMemsetAsync(scene->g_tex.p, 0, scene->g_tex.bytes, st));
  PSDR_CUDA(cudaMemsetAsync(scene->g_emit.p, 0, scene->g_emit.bytes, st));
  ws->campos_acc.alloc(sizeof(GradAcc) * 3 * n_cams, st);
  PSDR_CUDA(cudaMemsetAsync(ws->campos_acc.p, 0, sizeof(GradAcc) * 3 * n_cams, st));
  ws->lens_acc.alloc(sizeof(GradAcc) * kLensAcc * n_cams, st);
  PSDR_CUDA(cudaMemsetAsync(ws->lens_acc.p, 0, sizeof(GradAcc) * kLensAcc * n_cams, st));
  std::vector<DevView> views(n_cams);
  for (int i = 0; i < n_cams; ++i) {
    PSDR_CHECK(d_images[i] != nullptr, "null image gradient");
    make_view(cams[i], cfg->spp_interior, views[i]);
    views[i].dimage = d_images[i];
    views[i].grad_pos = ws->campos_acc.as<GradAcc>() + 3 * i;
    if (grads->camera_lens && grads->camera_lens[i] && unb) views[i].grad_lens = ws->lens_acc.as<GradAcc>() + kLensAcc * i;
  }
  {
    const psdr_scene* sl[1] = {scene};
    set_scene_ntri(views, sl);
  }
  render_backward_impl(dev_scene(scene), views, *cfg, ws, grad_info(scene), st);
  const int nm = (int)scene->meshes.size();
  for (int o = 0; o < scene->nobj; ++o) {
    if (grads->vertices && grads->vertices[o])
      grad_out(scene->g_verts.as<GradAcc>() + 3 * (size_t)scene->obj_vert_off[o], grads->vertices[o],
               3 * (long long)scene->obj_nvert[o], grads->accumulate, st);
    if (o < nm && grads->textures && grads->textures[o]) {
      const DevObj& ob = scene->h_objs[o];
      grad_out(scene->g_tex.as<GradAcc>() + scene->tex_grad_off[o], grads->textures[o],
               (long long)ob.color.h * ob.color.w * ob.color.ch, grads->accumulate, st);
    }
    if (o < nm && grads->roughness && grads->roughness[o] && scene->rough_grad_off[o] != SIZE_MAX) {
      const DevObj& ob = scene->h_objs[o];
      grad_out(scene->g_tex.as<GradAcc>() + scene->rough_grad_off[o], grads->roughness[o],
               (long long)ob.rough.h * ob.rough.w, grads->accumulate, st);
    }
    if (o < nm && grads->normal && grads->normal[o] && scene->nrm_grad_off[o] != SIZE_MAX) {
      const DevObj& ob = scene->h_objs[o];
      grad_out(scene->g_tex.as<GradAcc>() + scene->nrm_grad_off[o], grads->normal[o],
               (long long)ob.normal.h * ob.normal.w * 3, grads->accumulate, st);
    }
  }
  for (int l = 0; l < scene->nlight; ++l) {
    if (grads->emit && grads->emit[l]) grad_out(scene->g_emit.as<GradAcc>() + 3 * l, grads->emit[l], 3, grads->accumulate, st);
    if (grads->light_params && grads->light_params[l] && scene->light_grad_off[l] != SIZE_MAX)
      grad_out(scene->g_tex.as<GradAcc>() + scene->light_grad_off[l], grads->light_params[l],
               light_param_count(scene, l), grads->accumulate, st);
  }
  for (int i = 0; i < n_cams; ++i) {
    if (grads->camera_origin && grads->camera_origin[i])
      grad_out(ws->campos_acc.as<GradAcc>() + 3 * i, grads->camera_origin[i], 3, grads->accumulate, st);
    if (grads->camera_lens && grads->camera_lens[i]) {
      if (unb) lens_out(ws->lens_acc.as<GradAcc>() + kLensAcc * i, chains[i], grads->camera_lens[i], grads->accumulate, st);
      else if (!grads->accumulate) PSDR_CUDA(cudaMemsetAsync(grads->camera_lens[i], 0, sizeof(float) * 10, st));
    }
  }
  PSDR_CUDA(cudaGetLastError());
  API_END
}



}  // extern "C"
