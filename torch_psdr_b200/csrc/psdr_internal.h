// psdr_internal.h -- host-side objects behind the C ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "psdr.h"
#include "psdr_common.cuh"

namespace psdr {

void set_error(const std::string& msg);
struct Error {
  psdr_status code;
  std::string msg;
};

#define PSDR_CUDA(call)                                                                       \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      throw ::psdr::Error{e_ == cudaErrorMemoryAllocation ? PSDR_ERR_OOM : PSDR_ERR_CUDA,     \
                          std::string(#call) + ": " + cudaGetErrorString(e_)};                \
  } while (0)
#define PSDR_CHECK(cond, msg) \
  do { if (!(cond)) throw ::psdr::Error{PSDR_ERR_INVALID_ARG, msg}; } while (0)

// Device allocation owned by the library (stream-ordered allocator).
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
  }
  void alloc(size_t n, cudaStream_t s) {
    if (n <= bytes && p) return;
    release();
    st = s;
    size_t nb = n ? n : 16;
    PSDR_CUDA(cudaMallocAsync(&p, nb, s));
    bytes = nb;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

int num_sms();
void count_launches(int n);  // profiler launch counter (psdr_profile_read)

// Scan / sort primitives (sort.cu).
void exclusive_scan_int(const int* in, int* out, int n, int* tmp_blocks, cudaStream_t st);
size_t scan_tmp_ints(int n);
void inclusive_scan_double(const double* in, double* out, int n, double* tmp_blocks, cudaStream_t st);
size_t scan_tmp_doubles(int n);
struct SortTmp {
  DBuf keys2, vals2, hist;
};
// Stable LSD radix sort of (key, value) pairs over the low `bits` bits of the keys.
void radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int bits, SortTmp& tmp, cudaStream_t st);

}  // namespace psdr

struct psdr_scene {
  cudaStream_t stream = nullptr;
  int device = 0;  // the CUDA device current at psdr_scene_create (holds every buffer below)
  std::vector<psdr_mesh_desc> meshes;
  std::vector<psdr_area_light_desc> lights;
  int ntri = 0, nvert = 0, nobj = 0, nlight = 0, nnode = 0, leaf_size = 1;
  std::vector<int> obj_vert_off, obj_tri_off, obj_nvert, obj_ntri;
  std::vector<psdr::DevObj> h_objs;
  std::vector<psdr::DevLight> h_lights;
  // device storage
  psdr::DBuf verts, tri, tri_v, objs, lights_buf, light_pmf, light_cmf, ltri_pmf, ltri_cmf;
  psdr::DBuf n_edges, edge, edge_v, edge_f, edge_pmf, edge_cmf;
  psdr::DBuf nodes, leaf, err;
  // tree topology of the last full build, kept for psdr_scene_refit: binary child links,
  // leaf triangle order, 4-wide node flags and indices (the build's scratch is reused)
  psdr::DBuf bvh_child, bvh_order, bvh_f4;
  psdr::DBuf bvh_slots;  // per 4-wide node (by binary node id): its four children, -1 for none
  // build scratch
  psdr::DBuf keys, vals, aux_i, aux_i2, aux_d, aux_d2, aabb, parent, range, flags, cbox;
  psdr::SortTmp sort_tmp;
  // fp64 gradient accumulators (allocated on first backward)
  psdr::DBuf g_verts, g_tex, g_emit;
  psdr::DBuf vmask;  // per-vertex gradient mask (set from the gradient targets of a backward)
  std::vector<size_t> tex_grad_off;  // per object offset into g_tex (doubles), SIZE_MAX if none
  // DiffuseBsdfMaterial roughness / normal-map accumulators (after every color texture)
  std::vector<size_t> rough_grad_off, nrm_grad_off;
  bool has_bsdf = false;
  // environment light (EnvLight / SH9Light): its index (the last light) or -1, the box
  // mesh the library builds for it, and each light's parameter accumulator offset in g_tex
  int env_light = -1;
  float env_host_v[24];
  psdr::DBuf env_v, env_f, env_uv, env_uvi;
  std::vector<size_t> light_grad_off;
  bool grads_ready = false;
  psdr::DevScene dev{};
  psdr::DBuf d_dev;  // device copy of `dev`
  void upload_tables();
};
