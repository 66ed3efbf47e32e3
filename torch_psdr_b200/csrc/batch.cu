// batch.cu -- many views over one or more scenes as one work list, replayed from CUDA
// graphs (psdr_batch_*). The reference renders cameras one after another with a
// device synchronisation per ray query (path_integrator.cc:381-406,
// scene_optix.cc:240-277); here all views share the wavefront tiles (small views
// are packed together), and the whole forward (optionally preceded by the scenes'
// geometry rebuild) and the whole backward are each recorded once into a graph and
// replayed with a single launch. Inside each graph the independent parts of the job run
// on concurrent lanes (forked streams, one wavefront workspace each): the forward's
// tiles, and the backward's interior tiles and every boundary term of every view, spread
// by their ray counts. Each part is a chain of short dependent kernels (a wavefront depth
// loop, guide preprocessing, prefix sums); running several chains at once fills the SMs
// that one chain leaves idle between and at the tails of its launches.
#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "render.h"

struct psdr_batch {
  std::vector<psdr_scene*> scenes;
  std::vector<psdr::DevView> views;
  psdr_config cfg{};
  psdr_workspace ws;
  psdr::DBuf scenes_dev;  // DevScene array, one entry per scene
  psdr::DBuf campos;      // fp64 camera-origin accumulators, 3 per view
  psdr::DBuf lens;        // fp64 camera-lens accumulators, kLensAcc per view
  int cap = 0;
  bool backward = false;
  bool rebuild = true;
  psdr::SceneGradInfo gi;
  // gradient targets, deep-copied pointer arrays per scene
  std::vector<std::vector<float*>> gv, gt, ge, gr, gn, gl;
  std::vector<float*> gc, glens;
  std::vector<psdr::LensChain> lens_chain;
  std::vector<int> gacc;
  std::vector<std::unique_ptr<psdr::DBuf>> vmasks;  // per-scene vertex-gradient masks of this batch's targets
  std::vector<std::unique_ptr<psdr::DBuf>> objs;    // per-scene object tables (texture accumulators asked for)
  // concurrent lanes: lane 0 is the caller's stream with `ws`, lane k >= 1 has its own
  // stream and workspace; fork/join events of the graph captures
  int nlanes = 1;
  // replay records of every interior path, written by the forward (cfg.batch_records)
  bool kept = false;
  psdr::DBuf keep_rec, keep_view, keep_pix;
  psdr::KeptRecords keep;
  std::vector<std::unique_ptr<psdr_workspace>> lane_ws;
  std::vector<cudaStream_t> lane_st;
  std::vector<cudaEvent_t> lane_ev;
  cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;
  long long fwd_launches = 0, bwd_launches = 0;
  std::vector<psdr::Profiler::EvPair> fwd_ev, bwd_ev;  // trace timing events recorded in the graphs
  ~psdr_batch() {
    if (fwd_exec) cudaGraphExecDestroy(fwd_exec);
    if (bwd_exec) cudaGraphExecDestroy(bwd_exec);
    for (cudaStream_t s : lane_st) cudaStreamDestroy(s);
    for (cudaEvent_t e : lane_ev) cudaEventDestroy(e);
    auto& reps = psdr::profiler().replays;
    for (size_t i = reps.size(); i-- > 0;)
      if (reps[i].first == &fwd_ev || reps[i].first == &bwd_ev) reps.erase(reps.begin() + i);
    for (auto* v : {&fwd_ev, &bwd_ev})
      for (auto& e : *v) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  }
};

namespace psdr {
namespace {

// Records `body` on `st` into a graph and instantiates it. With profiling on, the
// trace kernels' timing events are recorded into the graph (list `gev`).
template <class F>
cudaGraphExec_t capture(cudaStream_t st, F body, long long& launches, std::vector<Profiler::EvPair>* gev) {
  Profiler& pf = profiler();
  pf.capture_ev = gev;
  const long long l0 = pf.launches;
  PSDR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    body();
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    pf.capture_ev = nullptr;
    throw;
  }
  cudaGraph_t graph = nullptr;
  pf.capture_ev = nullptr;
  PSDR_CUDA(cudaStreamEndCapture(st, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  PSDR_CUDA(e);
  launches = pf.launches - l0;
  pf.launches = l0;
  return exec;
}

// Runs body(k, stream_k, workspace_k) for every lane k of the batch: lanes k >= 1 are
// forked from st and joined back into it (inside a capture this forms parallel branches
// of the graph).
template <class F>
void over_lanes(psdr_batch* b, cudaStream_t st, F body) {
  const int K = b->nlanes;
  if (K > 1) {
    PSDR_CUDA(cudaEventRecord(b->lane_ev[0], st));
    for (int k = 1; k < K; ++k) PSDR_CUDA(cudaStreamWaitEvent(b->lane_st[k - 1], b->lane_ev[0], 0));
  }
  for (int k = 0; k < K; ++k) body(k, k == 0 ? st : b->lane_st[k - 1], k == 0 ? &b->ws : b->lane_ws[k - 1].get());
  for (int k = 1; k < K; ++k) {
    PSDR_CUDA(cudaEventRecord(b->lane_ev[k], b->lane_st[k - 1]));
    PSDR_CUDA(cudaStreamWaitEvent(st, b->lane_ev[k], 0));
  }
}

}  // namespace
}  // namespace psdr

using namespace psdr;

extern "C" {

PSDR_API psdr_status psdr_batch_create(psdr_scene* const* scenes, int32_t n_scenes, const psdr_camera_desc* cams,
                                       const int32_t* cam_scene, int32_t n_cams, const psdr_config* cfg,
                                       float** images, const float** d_images, const psdr_grad_targets* grads,
                                       psdr_batch** out) {
  psdr_batch* b = nullptr;
  try {
    PSDR_CHECK(out != nullptr && scenes != nullptr && n_scenes > 0 && cam_scene != nullptr && images != nullptr,
               "null argument");
    *out = nullptr;
    check_config(cfg);
    check_cameras(cams, n_cams);
    for (int i = 0; i < n_scenes; ++i) {
      PSDR_CHECK(scenes[i] != nullptr, "null scene");
      PSDR_CHECK(scenes[i]->nlight > 0 || cfg->mis_light_samples == 0, "a scene has no light to sample");
    }
    b = new psdr_batch();
    b->scenes.assign(scenes, scenes + n_scenes);
    b->cfg = *cfg;
    b->backward = d_images != nullptr;
    if (b->backward) {
      PSDR_CHECK(grads != nullptr, "d_images given without gradient targets");
    }
    cudaStream_t st = nullptr;
    const bool unb = cfg->estimator == PSDR_EST_UNBIASED;
    b->lens_chain.resize(n_cams);
    b->glens.assign(n_cams, nullptr);
    for (int i = 0; b->backward && i < n_cams; ++i) {
      PSDR_CHECK(cam_scene[i] >= 0 && cam_scene[i] < n_scenes, "camera scene index out of range");
      const psdr_grad_targets& g = grads[cam_scene[i]];
      if (!(g.camera_lens && g.camera_lens[i])) continue;
      if (cams[i].type != PSDR_CAM_PERSPECTIVE)
        throw Error{PSDR_ERR_UNSUPPORTED, "camera_lens gradients are implemented for perspective cameras only"};
      b->glens[i] = g.camera_lens[i];
      if (unb) lens_chain(cams[i], b->lens_chain[i]);
    }
    b->campos.alloc(sizeof(GradAcc) * 3 * n_cams, st);
    b->lens.alloc(sizeof(GradAcc) * kLensAcc * n_cams, st);
    b->views.resize(n_cams);
    for (int i = 0; i < n_cams; ++i) {
      PSDR_CHECK(cam_scene[i] >= 0 && cam_scene[i] < n_scenes, "camera scene index out of range");
      PSDR_CHECK(images[i] != nullptr, "null image buffer");
      make_view(cams[i], cfg->spp_interior, b->views[i]);
      b->views[i].scene = cam_scene[i];
      b->views[i].image = images[i];
      b->views[i].dimage = b->backward ? d_images[i] : nullptr;
      b->views[i].grad_pos = b->campos.as<GradAcc>() + 3 * i;
      if (b->glens[i] && unb) b->views[i].grad_lens = b->lens.as<GradAcc>() + kLensAcc * i;
      if (b->backward) PSDR_CHECK(d_images[i] != nullptr, "null image gradient");
    }
    assign_offsets(b->views);
    set_scene_ntri(b->views, scenes);
    b->cap = choose_cap(*cfg, b->views, true);
    const int Rmax = cfg->mis_light_samples + std::max(cfg->mis_bsdf_samples, 1) + 1;
    if (b->backward && cfg->batch_records >= 0) {
      long long paths = 0;
      for (const DevView& v : b->views) paths += (long long)v.H * v.W * v.spp;
      const int R = cfg->mis_light_samples + cfg->mis_bsdf_samples + 1;
      const size_t stride = 1 + (size_t)cfg->max_bounce * R + 2 * (size_t)cfg->max_bounce;
      const size_t bytes = (size_t)paths * (16 * stride + 8);
      size_t free_b = 0, total_b = 0;
      PSDR_CUDA(cudaMemGetInfo(&free_b, &total_b));
      b->kept = cfg->batch_records == 1 || bytes <= free_b / 4;
      if (b->kept) {
        b->keep_rec.alloc(16 * stride * (size_t)paths, st);
        b->keep_view.alloc(4 * (size_t)paths, st);
        b->keep_pix.alloc(4 * (size_t)paths, st);
        b->keep.rec = b->keep_rec.as<float4>();
        b->keep.view = b->keep_view.as<int>();
        b->keep.pix = b->keep_pix.as<int>();
      }
    }
    const int rec_needed = b->backward && !b->kept ? 1 : 0;
    b->ws.ensure(b->cap, Rmax, cfg->max_bounce, n_cams, rec_needed, st);
    if (b->backward) ensure_border(&b->ws, *cfg, b->views, st);
    upload_views(&b->ws, b->views, st);
    // lanes: no more than the job has independent parts
    {
      SceneGradInfo any;
      any.bsdf = any.jump = 1;
      const size_t parts = std::max(plan_tiles(b->views, b->cap).size(),
                                    b->backward ? backward_units(b->views, *cfg, b->cap, any).size() : (size_t)1);
      b->nlanes = (int)std::min<size_t>(cfg->batch_lanes > 0 ? cfg->batch_lanes : 4, parts);
    }
    for (int k = 1; k < b->nlanes; ++k) {
      b->lane_ws.emplace_back(new psdr_workspace());
      psdr_workspace* lw = b->lane_ws.back().get();
      lw->ensure(b->cap, Rmax, cfg->max_bounce, 1, rec_needed, st);
      if (b->backward) ensure_border(lw, *cfg, b->views, st);
      cudaStream_t ls = nullptr;
      PSDR_CUDA(cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking));
      b->lane_st.push_back(ls);
    }
    for (int k = 0; k < b->nlanes; ++k) {
      cudaEvent_t e = nullptr;
      PSDR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->lane_ev.push_back(e);
    }
    std::vector<DevScene> ds(n_scenes);
    for (int i = 0; i < n_scenes; ++i) ds[i] = scenes[i]->dev;
    if (b->backward) {
      // only the vertices whose gradient the caller bound are accumulated
      b->vmasks.resize(n_scenes);
      b->objs.resize(n_scenes);
      for (int i = 0; i < n_scenes; ++i) {
        const psdr_scene* s = scenes[i];
        std::vector<unsigned char> m(std::max(1, s->nvert), 0);
        for (int o = 0; o < s->nobj; ++o)
          if (grads[i].vertices && grads[i].vertices[o])
            std::fill(m.begin() + s->obj_vert_off[o], m.begin() + s->obj_vert_off[o] + s->obj_nvert[o], 1);
        b->vmasks[i].reset(new psdr::DBuf());
        b->vmasks[i]->alloc(m.size(), st);
        PSDR_CUDA(cudaMemcpyAsync(b->vmasks[i]->p, m.data(), m.size(), cudaMemcpyHostToDevice, st));
        PSDR_CUDA(cudaStreamSynchronize(st));
        ds[i].vmask = b->vmasks[i]->as<unsigned char>();
        std::vector<DevObj> ob = s->h_objs;
        for (int o = 0; o < (int)s->meshes.size(); ++o) {
          if (!(grads[i].textures && grads[i].textures[o])) ob[o].color.grad = nullptr;
          if (!(grads[i].roughness && grads[i].roughness[o])) ob[o].rough.grad = nullptr;
          if (!(grads[i].normal && grads[i].normal[o])) ob[o].normal.grad = nullptr;
        }
        b->objs[i].reset(new psdr::DBuf());
        b->objs[i]->alloc(sizeof(DevObj) * std::max<size_t>(1, ob.size()), st);
        PSDR_CUDA(cudaMemcpyAsync(b->objs[i]->p, ob.data(), sizeof(DevObj) * std::max<size_t>(1, ob.size()),
                                  cudaMemcpyHostToDevice, st));
        PSDR_CUDA(cudaStreamSynchronize(st));
        ds[i].objs = b->objs[i]->as<DevObj>();
      }
    }
    b->scenes_dev.alloc(sizeof(DevScene) * n_scenes, st);
    PSDR_CUDA(cudaMemcpyAsync(b->scenes_dev.p, ds.data(), sizeof(DevScene) * n_scenes, cudaMemcpyHostToDevice, st));
    if (n_scenes == 1) b->gi = grad_info(scenes[0]);
    b->ws.bsdf = 0;
    for (int i = 0; i < n_scenes; ++i) {
      if (scenes[i]->has_bsdf || scenes[i]->env_light >= 0) b->gi.bsdf = b->ws.bsdf = 1;
      if (scenes[i]->has_bsdf) b->gi.jump = 1;
    }
    for (auto& lw : b->lane_ws) lw->bsdf = b->ws.bsdf;
    if (b->backward) {
      b->gv.resize(n_scenes);
      b->gt.resize(n_scenes);
      b->gr.resize(n_scenes);
      b->gn.resize(n_scenes);
      b->gl.resize(n_scenes);
      b->ge.resize(n_scenes);
      b->gacc.resize(n_scenes);
      for (int i = 0; i < n_scenes; ++i) {
        const psdr_scene* s = scenes[i];
        const psdr_grad_targets& g = grads[i];
        const int nm = (int)s->meshes.size();
        for (int o = 0; o < s->nobj; ++o) b->gv[i].push_back(g.vertices ? g.vertices[o] : nullptr);
        for (int m = 0; m < nm; ++m) {
          b->gt[i].push_back(g.textures ? g.textures[m] : nullptr);
          b->gr[i].push_back(g.roughness && s->rough_grad_off[m] != SIZE_MAX ? g.roughness[m] : nullptr);
          b->gn[i].push_back(g.normal && s->nrm_grad_off[m] != SIZE_MAX ? g.normal[m] : nullptr);
        }
        for (int l = 0; l < s->nlight; ++l) {
          b->ge[i].push_back(g.emit ? g.emit[l] : nullptr);
          b->gl[i].push_back(g.light_params && s->light_grad_off[l] != SIZE_MAX ? g.light_params[l] : nullptr);
        }
        b->gacc[i] = g.accumulate;
      }
      for (int c = 0; c < n_cams; ++c) {
        const psdr_grad_targets& g = grads[cam_scene[c]];
        b->gc.push_back(g.camera_origin ? g.camera_origin[c] : nullptr);
      }
    }
    PSDR_CUDA(cudaStreamSynchronize(st));
    *out = b;
  } catch (const psdr::Error& e) {
    delete b;
    psdr::set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    delete b;
    psdr::set_error(e.what());
    return PSDR_ERR_CUDA;
  }
  return PSDR_OK;
}

// Forward of every view: geometry rebuild of each scene from its vertex buffers (the
// caller may have changed them in place), then the interior render into the images.
PSDR_API psdr_status psdr_batch_forward(psdr_batch* b, void* stream) {
  try {
    PSDR_CHECK(b != nullptr, "null batch");
    cudaStream_t st = (cudaStream_t)stream;
    PSDR_CHECK(st != nullptr, "batches need a non-default stream (graph capture)");
    if (!b->fwd_exec) {
      b->fwd_exec = capture(st, [&] {
        if (b->rebuild)
          for (psdr_scene* s : b->scenes) scene_build_geometry(s, st);
        const DevView* vd = b->ws.views.as<DevView>();
        const auto plan = schedule_tiles(plan_tiles(b->views, b->cap), b->nlanes);
        over_lanes(b, st, [&](int k, cudaStream_t ls, psdr_workspace* lw) {
          for (const Tile& t : plan[k])
            forward_tile(b->scenes_dev.as<DevScene>(), b->views, vd, t, b->cfg, lw, ls, nullptr,
                         b->kept ? &b->keep : nullptr);
        });
      }, b->fwd_launches, &b->fwd_ev);
    }
    PSDR_CUDA(cudaGraphLaunch(b->fwd_exec, st));
    profiler().launches += b->fwd_launches;
    profiler().replayed(&b->fwd_ev, (long long)b->fwd_ev.size());
  } catch (const psdr::Error& e) {
    psdr::set_error(e.msg);
    return e.code;
  }
  return PSDR_OK;
}

// Backward of every view (interior replay + adjoint, both edge terms), fp64
// accumulation, then the fp32 gradient outputs bound at creation.
PSDR_API psdr_status psdr_batch_backward(psdr_batch* b, void* stream) {
  try {
    PSDR_CHECK(b != nullptr, "null batch");
    PSDR_CHECK(b->backward, "the batch was created without image gradients");
    cudaStream_t st = (cudaStream_t)stream;
    PSDR_CHECK(st != nullptr, "batches need a non-default stream (graph capture)");
    if (!b->bwd_exec) {
      b->bwd_exec = capture(st, [&] {
        for (psdr_scene* s : b->scenes) {
          PSDR_CUDA(cudaMemsetAsync(s->g_verts.p, 0, s->g_verts.bytes, st));
          PSDR_CUDA(cudaMemsetAsync(s->g_tex.p, 0, s->g_tex.bytes, st));
          PSDR_CUDA(cudaMemsetAsync(s->g_emit.p, 0, s->g_emit.bytes, st));
        }
        PSDR_CUDA(cudaMemsetAsync(b->campos.p, 0, sizeof(GradAcc) * 3 * b->views.size(), st));
        PSDR_CUDA(cudaMemsetAsync(b->lens.p, 0, sizeof(GradAcc) * kLensAcc * b->views.size(), st));
        const DevView* vd = b->ws.views.as<DevView>();
        const auto plan = schedule_units(backward_units(b->views, b->cfg, b->cap, b->gi), b->nlanes);
        over_lanes(b, st, [&](int k, cudaStream_t ls, psdr_workspace* lw) {
          for (const BwdUnit& u : plan[k])
            backward_unit(b->scenes_dev.as<DevScene>(), b->views, vd, u, b->cfg, b->cap, lw, b->gi, ls,
                          b->kept ? &b->keep : nullptr);
        });
        for (size_t i = 0; i < b->scenes.size(); ++i) {
          psdr_scene* s = b->scenes[i];
          const int nm = (int)s->meshes.size();
          for (int o = 0; o < s->nobj; ++o)
            grad_out(s->g_verts.as<GradAcc>() + 3 * (size_t)s->obj_vert_off[o], b->gv[i][o],
                     3 * (long long)s->obj_nvert[o], b->gacc[i], st);
          for (int m = 0; m < nm; ++m) {
            const DevObj& ob = s->h_objs[m];
            grad_out(s->g_tex.as<GradAcc>() + s->tex_grad_off[m], b->gt[i][m],
                     (long long)ob.color.h * ob.color.w * ob.color.ch, b->gacc[i], st);
            if (b->gr[i][m])
              grad_out(s->g_tex.as<GradAcc>() + s->rough_grad_off[m], b->gr[i][m], (long long)ob.rough.h * ob.rough.w,
                       b->gacc[i], st);
            if (b->gn[i][m])
              grad_out(s->g_tex.as<GradAcc>() + s->nrm_grad_off[m], b->gn[i][m],
                       (long long)ob.normal.h * ob.normal.w * 3, b->gacc[i], st);
          }
          for (int l = 0; l < s->nlight; ++l) {
            grad_out(s->g_emit.as<GradAcc>() + 3 * l, b->ge[i][l], 3, b->gacc[i], st);
            if (b->gl[i][l])
              grad_out(s->g_tex.as<GradAcc>() + s->light_grad_off[l], b->gl[i][l], light_param_count(s, l), b->gacc[i],
                       st);
          }
        }
        for (size_t c = 0; c < b->views.size(); ++c) {
          grad_out(b->campos.as<GradAcc>() + 3 * c, b->gc[c], 3, b->gacc[b->views[c].scene], st);
          if (!b->glens[c]) continue;
          if (b->views[c].grad_lens)
            lens_out(b->views[c].grad_lens, b->lens_chain[c], b->glens[c], b->gacc[b->views[c].scene], st);
          else if (!b->gacc[b->views[c].scene])
            PSDR_CUDA(cudaMemsetAsync(b->glens[c], 0, sizeof(float) * 10, st));
        }
      }, b->bwd_launches, &b->bwd_ev);
    }
    PSDR_CUDA(cudaGraphLaunch(b->bwd_exec, st));
    profiler().launches += b->bwd_launches;
    profiler().replayed(&b->bwd_ev, (long long)b->bwd_ev.size());
  } catch (const psdr::Error& e) {
    psdr::set_error(e.msg);
    return e.code;
  }
  return PSDR_OK;
}

PSDR_API psdr_status psdr_batch_destroy(psdr_batch* b) {
  delete b;
  return PSDR_OK;
}

}  // extern "C"
