// render.h -- wavefront state shared by the render kernels and the host orchestration.
#pragma once

#include <vector>

#include "psdr_internal.h"

namespace psdr {

constexpr int kMaxDepth = 16;
constexpr int kMaxRays = 18;          // rays per path per depth: light + bsdf + indirect
constexpr int kMaxLightVerts = 8;     // light vertices accumulated in registers by the adjoint

// One camera view of a job. Matrices are row-major 4x4 (camera.h:108-124).
struct DevView {
  float r2c[16], c2w[16], w2c[16], c2r[16];
  float3 pos;
  int H, W, spp, scene;
  int ortho;             // orthographic camera (camera.h:279-353)
  long long sample_off;  // first sample of this view in the job's sample space
  long long pix_off;     // first pixel of this view in the job's pixel space
  float* image;          // (H,W,3) or null
  const float* dimage;   // (H,W,3) or null
  GradAcc* grad_pos;     // 3 accumulators or null
  GradAcc* grad_lens;    // 12 accumulators or null: the camera-lens sums (k_lens_interior, k_lens_border)
  int scene_ntri;        // host side (backward): triangles of the view's scene
};

// Path states and ray queues of one tile (structure of arrays, capacity `cap`).
struct WF {
  int cap, R, D, nL, nB, light_vis, nviews, spp_pass;
  unsigned long long seed;
  unsigned long long* rs;
  unsigned long long* ri;
  int* view;
  int* pix;
  float4* T;
  float4* L;
  float4* cur;   // current vertex: tri(bits), b1, b2, -
  float4* org;   // origin of the ray that reached it
  int* q0;
  int* q1;
  int* qs;
  int* cnt;      // per depth: [2d] live paths, [2d+1] shaded paths
  float4* ro;    // ray origin + tmax
  float4* rd;    // ray direction + aux (light index bits)
  float4* ra;    // aux: NEE target point + pdf / bsdf cos(theta)
  float4* hit;   // tri(bits), b1, b2, t
  float4* rec;   // replay records: 1 + D*R per path
  int rec_stride;
  int bsdf;      // host side: launch the extended kernel instances (DiffuseBsdfMaterial, environment light)
  int ortho;     // host side: an orthographic view is in the job (camera kernel instance)
  int trace_bps; // host side: blocks of 128 rays per SM of the closest-hit kernel (queue depth)
};

struct Tile {
  long long begin;  // first sample (job sample space)
  int n;            // samples in the tile
  long long pix_begin;
  int npix;
};

// Side buffers of the primary-edge term (one entry per edge sample of a tile).
struct EdgeBuf {
  float4* a;     // edge id(bits), s, pdf_e, hc_pdf
  float4* n;     // edge normal, pixel(bits)
  float4* hb;    // hit of the +eps ray: tri(bits), b1, b2, valid(bits)
  float4* La;    // radiance of the -eps path
  unsigned long long* rng_keep;  // preprocess: sampler state across rounds
};

// MODE_FWD accumulates the image; MODE_REPLAY re-traces a tile's paths for the backward
// and writes their replay records; MODE_KEEP does both in one pass (the batch's forward
// when it keeps the records of every tile for its backward).
enum Mode { MODE_FWD = 0, MODE_REPLAY = 1, MODE_KEEP = 2 };

// Replay records of every interior path of a job kept from its forward (psdr_batch): path
// s of the job's sample space has its record at rec + s * rec_stride and its view and
// pixel at view[s], pix[s].
struct KeptRecords {
  float4* rec = nullptr;
  int* view = nullptr;
  int* pix = nullptr;
};

struct psdr_ws_impl;

}  // namespace psdr

struct psdr_workspace {
  int cap = 0, R = 0, D = 0, nviews_cap = 0;
  psdr::DBuf rs, ri, view, pix, T, L, cur, org, q0, q1, qs, cnt, ro, rd, ra, hit, rec;
  psdr::DBuf views, eb_a, eb_n, eb_hb, eb_La, eb_rng, mass, mass_d, mass_pre, hc_pmf, hc_cmf, scan_tmp, ncells;
  psdr::DBuf campos_acc, lens_acc;
  psdr::DBuf crease;  // interpenetration segments (unbiased estimator): kCreaseCap records + count
  long long mass_cap = 0;
  // a DiffuseBsdfMaterial mesh or an environment light is in the scenes of the current job
  // (each entry point sets it; the extended kernel instances also handle the plain
  // scenes, so 1 is always safe)
  int bsdf = 1;
  cudaStream_t stream = nullptr;
  std::vector<psdr::DevView> h_views;
  psdr::WF wf{};
  void ensure(int cap, int R, int D, int nviews, int rec_needed, cudaStream_t st);
  void ensure_mass(long long n, cudaStream_t st);
};

namespace psdr {
// In-library profiler (psdr_profile_*): launch counts and trace-kernel event timing.
struct Profiler {
  using EvPair = std::pair<cudaEvent_t, cudaEvent_t>;
  bool on = false;
  long long launches = 0, trace_launches = 0;
  std::vector<EvPair> ev;  // events of directly launched trace kernels
  size_t used = 0;
  // While a graph is being recorded, trace events go to the graph's own list; every
  // replay re-records them, and psdr_profile_read weights the last replay's times by
  // the number of replays since the last reset.
  std::vector<EvPair>* capture_ev = nullptr;
  std::vector<std::pair<std::vector<EvPair>*, long long>> replays;
  unsigned long long* d_rays = nullptr;
  void begin_trace(cudaStream_t st);
  void end_trace(cudaStream_t st);
  void replayed(std::vector<EvPair>* graph_ev, long long n_trace);
};
Profiler& profiler();
struct SceneGradInfo;
void make_view(const psdr_camera_desc& c, int spp, DevView& v);
void render_forward_impl(const DevScene* scenes_dev, std::vector<DevView>& views, const psdr_config& cfg,
                         psdr_workspace* ws, cudaStream_t st, float* samples_out);
struct SceneGradInfo {
  int hot_lv0 = 0, hot_nlv = 0, emit_hot = 0;
  int bsdf = 0;  // a DiffuseBsdfMaterial mesh or an environment light (extended adjoint kernel)
  int jump = 0;  // a DiffuseBsdfMaterial mesh: the unbiased default terms include its BRDF jumps
};
void render_backward_impl(const DevScene* scenes_dev, std::vector<DevView>& views, const psdr_config& cfg,
                          psdr_workspace* ws, const SceneGradInfo& gi, cudaStream_t st);
void grad_out(const GradAcc* acc, float* out, long long n, int accumulate, cudaStream_t st);
void assign_offsets(std::vector<DevView>& views);
int choose_cap(const psdr_config& cfg, const std::vector<DevView>& views, bool backward);
void upload_views(psdr_workspace* ws, const std::vector<DevView>& views, cudaStream_t st);
void forward_launch(const DevScene* scenes_dev, const std::vector<DevView>& views, const psdr_config& cfg, int cap,
                    psdr_workspace* ws, cudaStream_t st, float* samples_out);
void backward_launch(const DevScene* scenes_dev, const std::vector<DevView>& views, const psdr_config& cfg,
                     int cap, psdr_workspace* ws, const SceneGradInfo& gi, cudaStream_t st);
// One forward tile (camera paths, depth loop, film) on workspace ws; views at vd.
// With `keep`, the tile's replay records, views and pixels go to its place in `keep`.
void forward_tile(const DevScene* scenes_dev, const std::vector<DevView>& views, const DevView* vd, const Tile& t,
                  const psdr_config& cfg, psdr_workspace* ws, cudaStream_t st, float* samples_out,
                  const KeptRecords* keep = nullptr);
// The backward of a job as independent units: the interior replay + adjoint of each
// wavefront tile (term 1) and each boundary term (bits 2..64 of psdr_config.terms) of
// each view. A unit writes only its own workspace and the integer gradient accumulators,
// whose sums do not depend on the order of the additions, so units may run in any order,
// or concurrently on separate workspaces, with bitwise the same gradients.
struct BwdUnit {
  int term;      // 1 interior tile, else the boundary term's bit
  int view;      // boundary terms: the view
  Tile tile;     // interior: the tile
  double cost;   // relative device work (rays traced), for scheduling
};
std::vector<BwdUnit> backward_units(const std::vector<DevView>& views, const psdr_config& cfg, int cap,
                                    const SceneGradInfo& gi);
// With `keep` (records kept by the forward), an interior unit runs only the adjoint.
void backward_unit(const DevScene* scenes_dev, const std::vector<DevView>& views, const DevView* vd,
                   const BwdUnit& u, const psdr_config& cfg, int cap, psdr_workspace* ws, const SceneGradInfo& gi,
                   cudaStream_t st, const KeptRecords* keep = nullptr);
// Units split over `lanes` lists by longest-processing-time-first scheduling on `cost`
// (each list keeps the units' original order).
std::vector<std::vector<BwdUnit>> schedule_units(const std::vector<BwdUnit>& units, int lanes);
// Forward tiles split over `lanes` lists the same way (cost = paths).
std::vector<std::vector<Tile>> schedule_tiles(const std::vector<Tile>& tiles, int lanes);
SceneGradInfo grad_info(const psdr_scene* s);
void check_config(const psdr_config* c);
void check_cameras(const psdr_camera_desc* cams, int n);
long long light_param_count(const psdr_scene* s, int l);
void scene_build_geometry(psdr_scene* s, cudaStream_t st);
void scene_refit_geometry(psdr_scene* s, cudaStream_t st);
std::vector<Tile> plan_tiles(const std::vector<DevView>& views, int cap);
// Camera-lens gradient (unbiased estimator, perspective cameras): P[j] = M^-1 dM/dtheta_j
// for the raster-to-direction map M of camera c and its parameters theta = (look_from,
// look_at, up, fov) as they enter the camera's basis and projection (row-major 3x3 each).
struct LensChain {
  double P[10][9];
};
void lens_chain(const psdr_camera_desc& c, LensChain& out, double* m9 = nullptr);
constexpr int kLensAcc = 12;  // accumulators per view: S0, Sx, Sy, B (3x3)
// out[10] (fp32, overwritten or accumulated) from a view's accumulators.
void lens_out(const GradAcc* acc, const LensChain& ch, float* out, int accumulate, cudaStream_t st);
long long border_segments(const DevView& V);
void ensure_border(psdr_workspace* ws, const psdr_config& cfg, const std::vector<DevView>& views, cudaStream_t st);
// Views of a backward job: their scene triangle counts (DevView::scene_ntri), before ensure_border.
void set_scene_ntri(std::vector<DevView>& views, const psdr_scene* const* scenes);
}  // namespace psdr
