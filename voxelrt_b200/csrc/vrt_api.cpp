// vrt_api.cpp -- host side of the C ABI (include/vrt.h).
//
// Owns contexts (device + stream + HBM admission budget), device-resident
// scenes and per-view sessions, and drives the reference's pass order
// (main.js:680-772): pathtrace -> temporal -> a-trous x3 -> present, with
// G-buffer and history ping-ponged by frame parity (main.js:429-431) and the
// a-trous chain accum -> dA -> dB -> dA (main.js:503-507).
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <mutex>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <unordered_map>
#include "vrt_internal.h"

using namespace vrt;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int vrt::set_error(int code, const char* msg) { return fail(code, "%s", msg); }

#define CUDA_TRY(expr)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (expr);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      return fail(e_ == cudaErrorMemoryAllocation ? VRT_ERR_OOM : VRT_ERR_CUDA, "%s: %s (%s:%d)", \
                  #expr, cudaGetErrorString(e_), __FILE__, __LINE__);                            \
    }                                                                                            \
  } while (0)

// ---------------------------------------------------------------------------
// objects
// ---------------------------------------------------------------------------
struct VrtCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;   // 0 = unlimited
  uint64_t used = 0;
  float* present_lut = nullptr;   // kPresentLut floats, built on the stream at creation
};

struct VrtScene {
  VrtCtx* ctx = nullptr;
  SceneDev dev;
  uint64_t bytes = 0;
  // emissive-face light list, alias table, light grid (vrt_scene_build_lights)
  uint32_t* light_words = nullptr;   // 2 per light
  double* light_w = nullptr;         // weight per light
  float* light_alias = nullptr;      // 4 per light
  uint32_t* light_grid = nullptr;    // 34 per brick cell
  uint32_t* light_tmp = nullptr;     // block offsets + count
  size_t light_cap = 0;              // lights the word/weight buffers hold
  size_t light_alias_bytes = 0;
  uint32_t light_count = 0;
  bool lights_built = false;
};

struct VrtSession {
  VrtCtx* ctx = nullptr;
  VrtScene* scene = nullptr;
  int W = 0, H = 0;
  float fclamp = 48.0f;
  bool acc_f32 = false;
  bool keep_f32 = false;
  uint64_t bytes = 0;
  // render targets (main.js:82-90 equivalents)
  void* rad16 = nullptr;
  void* rad32 = nullptr;
  uint32_t* alb8 = nullptr;
  void* gbuf[2] = {nullptr, nullptr};
  void* accum[2] = {nullptr, nullptr};
  void* den[2] = {nullptr, nullptr};
  uint32_t* ldr = nullptr;
  unsigned long long* stats = nullptr;
  // wavefront scratch
  int path_kernel = VRT_PATH_WAVEFRONT;
  void* wf_mem = nullptr;
  size_t wf_bytes = 0;
  WavefrontBufs wf;
  WavefrontTuning tune;
  // frame state
  uint64_t frame_counter = 0;     // host frame index (parity source)
  bool last_denoise = false;
  bool have_frame = false;
  int last_parity = 0;
  // timing
  bool timing = false;
  cudaEvent_t ev[6] = {};
  static constexpr int kTimedWaves = 16;
  cudaEvent_t tev[2 * kTimedWaves] = {};   // brackets of each wave's trace kernel
  int timed_waves = 0;
  uint32_t launches = 0;
  // radiance cache
  VrtCacheConfig cache_cfg{};
  bool cache_on = false;
  VrtMlp* mlp = nullptr;
  void* cache_mem = nullptr;
  size_t cache_bytes = 0;
  CacheDev cache{};
  float* pred = nullptr;
  cudaEvent_t cev[2] = {};
  bool cache_timed = false;
  uint64_t cache_version = 0;     // changes with every vrt_session_set_cache
  // HDR reference pipeline (FP64 sums, reference image, error partials)
  double* hdr_acc = nullptr;
  float* hdr_ref = nullptr;
  double* hdr_part = nullptr;
  uint32_t hdr_count = 0;
  // ReSTIR reservoirs A and B (32 B per pixel each) + pass-through radiance
  // (8 B per pixel), allocated by the first frame with reservoir flags
  void* restir_mem = nullptr;
  size_t restir_bytes = 0;
  uint32_t* pairing = nullptr;    // pairing textures (RF_PAIRED), built on first use
  double pairing_built[3] = {0.0, 0.0, 0.0};   // their sigmas
  double pairing_sigma = 16.0;    // base sigma (main.js:73 `sigma`)
  bool restir_timed = false;      // ev[5] marks the end of the initial pass
  uint64_t events_frame = ~0ull;  // frame whose pass events vrt_frame recorded
};

constexpr int kMaxWaves = 72;   // wave counters allocated per wavefront scratch

static int set_dev(VrtCtx* ctx) {
  CUDA_TRY(cudaSetDevice(ctx->device));
  return VRT_OK;
}

static int dev_alloc(VrtCtx* ctx, void** p, size_t bytes, uint64_t* acct) {
  if (ctx->budget && ctx->used + bytes > ctx->budget)
    return fail(VRT_ERR_BUDGET, "HBM budget exceeded: in use %llu + request %zu > budget %llu",
                (unsigned long long)ctx->used, bytes, (unsigned long long)ctx->budget);
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(VRT_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  ctx->used += bytes;
  *acct += bytes;
  return VRT_OK;
}

static void dev_free(VrtCtx* ctx, void* p, size_t bytes, uint64_t* acct) {
  if (!p) return;
  cudaFree(p);
  ctx->used -= bytes;
  *acct -= bytes;
}

extern "C" {

int vrt_abi_version(void) { return VRT_ABI_VERSION; }
const char* vrt_last_error_string(void) { return g_err.c_str(); }

int vrt_create(const VrtDeviceConfig* cfg, VrtCtx** out) {
  if (!out) return fail(VRT_ERR_INVALID, "vrt_create: out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(VRT_ERR_NO_DEVICE, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "count 0");
  VrtCtx* c = new VrtCtx();
  c->device = cfg ? cfg->device : 0;
  c->budget = cfg ? cfg->hbm_budget_bytes : 0;
  if (c->device < 0 || c->device >= n) {
    delete c;
    return fail(VRT_ERR_INVALID, "device %d out of range (%d devices)", cfg ? cfg->device : 0, n);
  }
  e = cudaSetDevice(c->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&c->present_lut, kPresentLut * sizeof(float));
  if (e == cudaSuccess) e = launch_present_lut(c->present_lut, c->stream);
  if (e != cudaSuccess) {
    if (c->present_lut) cudaFree(c->present_lut);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return fail(VRT_ERR_CUDA, "context init: %s", cudaGetErrorString(e));
  }
  *out = c;
  return VRT_OK;
}

int vrt_destroy(VrtCtx* ctx) {
  if (!ctx) return VRT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  if (ctx->present_lut) cudaFree(ctx->present_lut);
  delete ctx;
  return VRT_OK;
}

int vrt_ctx_synchronize(VrtCtx* ctx) {
  if (!ctx) return fail(VRT_ERR_INVALID, "ctx is NULL");
  if (int r = set_dev(ctx)) return r;
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return VRT_OK;
}

uint64_t vrt_ctx_bytes_in_use(const VrtCtx* ctx) { return ctx ? ctx->used : 0; }

int vrt_selftest_present(VrtCtx* ctx, uint64_t* mismatches, uint32_t* first_bits) {
  if (!ctx || !mismatches || !first_bits) return fail(VRT_ERR_INVALID, "vrt_selftest_present: NULL argument");
  if (int r = set_dev(ctx)) return r;
  void* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, 16));
  unsigned long long* bad = (unsigned long long*)d;
  unsigned int* first = (unsigned int*)((char*)d + 8);
  cudaError_t e = cudaMemsetAsync(bad, 0, 8, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(first, 0xff, 4, ctx->stream);
  if (e == cudaSuccess) e = launch_present_check(ctx->present_lut, bad, first, ctx->stream);
  unsigned long long hb = 0;
  unsigned int hf = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, bad, 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hf, first, 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(VRT_ERR_CUDA, "vrt_selftest_present: %s", cudaGetErrorString(e));
  *mismatches = hb;
  *first_bits = hf;
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// scenes
// ---------------------------------------------------------------------------
static int scene_alloc(VrtCtx* ctx, int N, VrtScene** out) {
  if (!ctx || !out) return fail(VRT_ERR_INVALID, "NULL argument");
  if (N < 8 || N % 8 != 0 || N > 2048) return fail(VRT_ERR_INVALID, "grid size %d must be a multiple of 8 in [8, 2048]", N);
  if (int r = set_dev(ctx)) return r;
  VrtScene* s = new VrtScene();
  s->ctx = ctx;
  s->dev.N = N;
  s->dev.BG = N / 8;
  const size_t nv = (size_t)N * N * N, nb = (size_t)s->dev.BG * s->dev.BG * s->dev.BG;
  int r = dev_alloc(ctx, (void**)&s->dev.vox, nv * 4, &s->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&s->dev.bricks, nb * 4, &s->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&s->dev.masks, nb * 64, &s->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&s->dev.bits, occ_words(s->dev.BG) * 4 + 128, &s->bytes);
  if (r) {
    std::string keep = g_err;
    vrt_scene_destroy(s);
    g_err = keep;
    return r;
  }
  *out = s;
  return VRT_OK;
}

int vrt_scene_upload(VrtCtx* ctx, const uint32_t* voxels, int N, VrtScene** out) {
  if (!voxels) return fail(VRT_ERR_INVALID, "voxels is NULL");
  VrtScene* s = nullptr;
  if (int r = scene_alloc(ctx, N, &s)) return r;
  const size_t nv = (size_t)N * N * N;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(s->dev.vox, voxels, nv * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_build_bricks(s->dev, 0, 0, 0, s->dev.BG - 1, s->dev.BG - 1, s->dev.BG - 1, st);
  if (e == cudaSuccess) e = launch_build_bits(s->dev, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    vrt_scene_destroy(s);
    return fail(VRT_ERR_CUDA, "scene upload: %s", cudaGetErrorString(e));
  }
  *out = s;
  return VRT_OK;
}

int vrt_scene_upload_prebuilt(VrtCtx* ctx, const uint32_t* voxels, const uint32_t* bricks,
                              const uint32_t* brick_masks, int N, VrtScene** out) {
  if (!voxels || !bricks || !brick_masks) return fail(VRT_ERR_INVALID, "NULL buffer");
  VrtScene* s = nullptr;
  if (int r = scene_alloc(ctx, N, &s)) return r;
  const size_t nv = (size_t)N * N * N, nb = (size_t)s->dev.BG * s->dev.BG * s->dev.BG;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(s->dev.vox, voxels, nv * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->dev.bricks, bricks, nb * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->dev.masks, brick_masks, nb * 64, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_build_bits(s->dev, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    vrt_scene_destroy(s);
    return fail(VRT_ERR_CUDA, "scene upload: %s", cudaGetErrorString(e));
  }
  *out = s;
  return VRT_OK;
}

int vrt_scene_edit_box(VrtScene* s, int x0, int y0, int z0, int x1, int y1, int z1, uint32_t value) {
  if (!s) return fail(VRT_ERR_INVALID, "scene is NULL");
  const int N = s->dev.N;
  if (x0 > x1) std::swap(x0, x1);
  if (y0 > y1) std::swap(y0, y1);
  if (z0 > z1) std::swap(z0, z1);
  x0 = std::max(x0, 0); y0 = std::max(y0, 0); z0 = std::max(z0, 0);
  x1 = std::min(x1, N - 1); y1 = std::min(y1, N - 1); z1 = std::min(z1, N - 1);
  if (x0 > x1 || y0 > y1 || z0 > z1) return VRT_OK;   // box fully outside: nothing to do
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  CUDA_TRY(launch_fill_box(s->dev, x0, y0, z0, x1, y1, z1, value, st));
  CUDA_TRY(launch_build_bricks(s->dev, x0 / 8, y0 / 8, z0 / 8, x1 / 8, y1 / 8, z1 / 8, st));
  CUDA_TRY(launch_build_bits(s->dev, st));
  return VRT_OK;
}

int vrt_scene_read(VrtScene* s, uint32_t* voxels, uint32_t* bricks, uint32_t* masks) {
  if (!s) return fail(VRT_ERR_INVALID, "scene is NULL");
  if (int r = set_dev(s->ctx)) return r;
  const size_t N = s->dev.N, nb = (size_t)s->dev.BG * s->dev.BG * s->dev.BG;
  cudaStream_t st = s->ctx->stream;
  if (voxels) CUDA_TRY(cudaMemcpyAsync(voxels, s->dev.vox, N * N * N * 4, cudaMemcpyDeviceToHost, st));
  if (bricks) CUDA_TRY(cudaMemcpyAsync(bricks, s->dev.bricks, nb * 4, cudaMemcpyDeviceToHost, st));
  if (masks) CUDA_TRY(cudaMemcpyAsync(masks, s->dev.masks, nb * 64, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return VRT_OK;
}

int vrt_scene_destroy(VrtScene* s) {
  if (!s) return VRT_OK;
  VrtCtx* c = s->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  const size_t N = s->dev.N, nb = (size_t)s->dev.BG * s->dev.BG * s->dev.BG;
  dev_free(c, s->dev.vox, N * N * N * 4, &s->bytes);
  dev_free(c, s->dev.bricks, nb * 4, &s->bytes);
  dev_free(c, s->dev.masks, nb * 64, &s->bytes);
  dev_free(c, s->dev.bits, occ_words(s->dev.BG) * 4 + 128, &s->bytes);
  const size_t cap = s->light_cap;
  dev_free(c, s->light_words, cap * 8, &s->bytes);
  dev_free(c, s->light_w, cap * 8, &s->bytes);
  dev_free(c, s->light_alias, s->light_alias_bytes, &s->bytes);
  dev_free(c, s->light_grid, nb * 34 * 4, &s->bytes);
  dev_free(c, s->light_tmp, ((size_t)light_blocks((int)N) + 1) * 4, &s->bytes);
  delete s;
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// DDA parity entry
// ---------------------------------------------------------------------------
int vrt_trace_rays_device(VrtScene* s, const float* o, const float* d, const float* tmax, int n, VrtHit* out) {
  if (!s || n < 0) return fail(VRT_ERR_INVALID, "bad argument");
  if (n == 0) return VRT_OK;
  if (!o || !d || !tmax || !out) return fail(VRT_ERR_INVALID, "NULL buffer");
  if (int r = set_dev(s->ctx)) return r;
  CUDA_TRY(launch_trace_rays(s->dev, o, d, tmax, n, out, s->ctx->stream));
  return VRT_OK;
}

int vrt_trace_rays(VrtScene* s, const float* o, const float* d, const float* tmax, int n, VrtHit* out) {
  if (!s || n < 0) return fail(VRT_ERR_INVALID, "bad argument");
  if (n == 0) return VRT_OK;
  if (!o || !d || !tmax || !out) return fail(VRT_ERR_INVALID, "NULL buffer");
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  char* buf = nullptr;
  const size_t bo = (size_t)n * 12, bt = (size_t)n * 4, bh = (size_t)n * sizeof(VrtHit);
  CUDA_TRY(cudaMalloc(&buf, 2 * bo + bt + bh));
  float* dO = (float*)buf;
  float* dD = (float*)(buf + bo);
  float* dT = (float*)(buf + 2 * bo);
  VrtHit* dH = (VrtHit*)(buf + 2 * bo + bt);
  cudaError_t e = cudaMemcpyAsync(dO, o, bo, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dD, d, bo, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, tmax, bt, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_trace_rays(s->dev, dO, dD, dT, n, dH, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dH, bh, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(VRT_ERR_CUDA, "trace_rays: %s", cudaGetErrorString(e));
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// sessions
// ---------------------------------------------------------------------------
static size_t px(const VrtSession* s) { return (size_t)s->W * s->H; }
static size_t acc_bpp(const VrtSession* s) { return s->acc_f32 ? 16 : 8; }

int vrt_session_destroy(VrtSession* s) {
  if (!s) return VRT_OK;
  VrtCtx* c = s->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  const size_t P = px(s);
  dev_free(c, s->rad16, P * 8, &s->bytes);
  dev_free(c, s->rad32, P * 16, &s->bytes);
  dev_free(c, s->alb8, P * 4, &s->bytes);
  for (int i = 0; i < 2; i++) {
    dev_free(c, s->gbuf[i], P * 16, &s->bytes);
    dev_free(c, s->accum[i], P * acc_bpp(s), &s->bytes);
    dev_free(c, s->den[i], P * 8, &s->bytes);
  }
  dev_free(c, s->ldr, P * 4, &s->bytes);
  dev_free(c, s->stats, kStatCount * 8, &s->bytes);
  dev_free(c, s->wf_mem, s->wf_bytes, &s->bytes);
  dev_free(c, s->cache_mem, s->cache_bytes, &s->bytes);
  dev_free(c, s->hdr_acc, P * 24, &s->bytes);
  dev_free(c, s->hdr_ref, P * 12, &s->bytes);
  dev_free(c, s->hdr_part, (size_t)hdr_blocks((int)P) * 8, &s->bytes);
  dev_free(c, s->restir_mem, s->restir_bytes, &s->bytes);
  dev_free(c, s->pairing, (size_t)kPairingWords * 4, &s->bytes);
  if (s->mlp) vrt_mlp_destroy(s->mlp);
  for (auto& e : s->cev)
    if (e) cudaEventDestroy(e);
  for (auto& e : s->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : s->tev)
    if (e) cudaEventDestroy(e);
  delete s;
  return VRT_OK;
}

int vrt_session_reset(VrtSession* s) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = set_dev(s->ctx)) return r;
  const size_t P = px(s);
  cudaStream_t st = s->ctx->stream;
  for (int i = 0; i < 2; i++) {
    CUDA_TRY(cudaMemsetAsync(s->gbuf[i], 0, P * 16, st));
    CUDA_TRY(cudaMemsetAsync(s->accum[i], 0, P * acc_bpp(s), st));
    CUDA_TRY(cudaMemsetAsync(s->den[i], 0, P * 8, st));
  }
  CUDA_TRY(cudaMemsetAsync(s->rad16, 0, P * 8, st));
  if (s->rad32) CUDA_TRY(cudaMemsetAsync(s->rad32, 0, P * 16, st));
  CUDA_TRY(cudaMemsetAsync(s->alb8, 0, P * 4, st));
  CUDA_TRY(cudaMemsetAsync(s->ldr, 0, P * 4, st));
  CUDA_TRY(cudaMemsetAsync(s->stats, 0, kStatCount * 8, st));
  // a fresh history reservoir B decodes as "no sample" (main.js:350-352)
  if (s->restir_mem) CUDA_TRY(cudaMemsetAsync(s->restir_mem, 0, s->restir_bytes, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  s->frame_counter = 0;
  s->events_frame = ~0ull;
  s->have_frame = false;
  s->last_parity = 0;
  return VRT_OK;
}

int vrt_session_create(VrtCtx* ctx, VrtScene* scene, const VrtSessionConfig* cfg, VrtSession** out) {
  if (!ctx || !scene || !cfg || !out) return fail(VRT_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (cfg->width < 1 || cfg->height < 1 || cfg->width > 16384 || cfg->height > 16384)
    return fail(VRT_ERR_INVALID, "render size %dx%d out of range", cfg->width, cfg->height);
  if (scene->ctx != ctx) return fail(VRT_ERR_INVALID, "scene belongs to another context");
  if (int r = set_dev(ctx)) return r;
  VrtSession* s = new VrtSession();
  s->ctx = ctx;
  s->scene = scene;
  s->W = cfg->width;
  s->H = cfg->height;
  s->fclamp = cfg->firefly_clamp;
  s->acc_f32 = cfg->accum_f32 != 0;
  s->keep_f32 = cfg->keep_radiance_f32 != 0;
  const size_t P = px(s);
  int r = dev_alloc(ctx, &s->rad16, P * 8, &s->bytes);
  if (!r && s->keep_f32) r = dev_alloc(ctx, &s->rad32, P * 16, &s->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&s->alb8, P * 4, &s->bytes);
  for (int i = 0; i < 2 && !r; i++) {
    r = dev_alloc(ctx, &s->gbuf[i], P * 16, &s->bytes);
    if (!r) r = dev_alloc(ctx, &s->accum[i], P * acc_bpp(s), &s->bytes);
    if (!r) r = dev_alloc(ctx, &s->den[i], P * 8, &s->bytes);
  }
  if (!r) r = dev_alloc(ctx, (void**)&s->ldr, P * 4, &s->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&s->stats, kStatCount * 8, &s->bytes);
  s->path_kernel = (cfg->path_kernel == VRT_PATH_MEGAKERNEL || cfg->path_kernel == VRT_PATH_BATCH_ONLY)
                       ? cfg->path_kernel : VRT_PATH_WAVEFRONT;
  if (!r && s->path_kernel == VRT_PATH_WAVEFRONT) {
    const int max_waves = kMaxWaves;
    s->wf_bytes = wavefront_bytes(s->W, s->H, max_waves, 4);
    r = dev_alloc(ctx, &s->wf_mem, s->wf_bytes, &s->bytes);
    if (!r) carve_wavefront(s->wf_mem, P, max_waves, s->wf, 4);
  }
  if (!r) {
    for (auto& e : s->ev) {
      if (cudaEventCreate(&e) != cudaSuccess) { r = fail(VRT_ERR_CUDA, "cudaEventCreate failed"); break; }
    }
    for (auto& e : s->tev) {
      if (r) break;
      if (cudaEventCreate(&e) != cudaSuccess) { r = fail(VRT_ERR_CUDA, "cudaEventCreate failed"); break; }
    }
  }
  if (!r) r = vrt_session_reset(s);
  if (r) {
    std::string keep = g_err;
    vrt_session_destroy(s);
    g_err = keep;
    return r;
  }
  *out = s;
  return VRT_OK;
}

int vrt_session_set_scene(VrtSession* s, VrtScene* scene) {
  if (!s || !scene || scene->ctx != s->ctx) return fail(VRT_ERR_INVALID, "bad scene");
  s->scene = scene;
  return VRT_OK;
}

int vrt_session_get_tuning(VrtSession* s, VrtTuning* t) {
  if (!s || !t) return fail(VRT_ERR_INVALID, "NULL argument");
  t->refill_min = s->tune.refill_min;
  t->trace_blocks_per_sm = s->tune.trace_blocks_per_sm;
  t->shade_blocks_per_sm = s->tune.shade_blocks_per_sm;
  t->trace_variant = s->tune.trace_variant;
  t->atrous_tile_rows = s->tune.atrous_rows;
  t->tail_wave = s->tune.tail_wave;
  return VRT_OK;
}

int vrt_session_set_tuning(VrtSession* s, const VrtTuning* t) {
  if (!s || !t) return fail(VRT_ERR_INVALID, "NULL argument");
  if (t->refill_min < 0 || t->refill_min > 32 || t->trace_blocks_per_sm < 0 || t->trace_blocks_per_sm > 32 ||
      t->shade_blocks_per_sm < 0 || t->shade_blocks_per_sm > 64 || t->trace_variant < 0 || t->trace_variant > 8 ||
      (t->atrous_tile_rows != 0 && t->atrous_tile_rows != 8 && t->atrous_tile_rows != 16) || t->tail_wave < -1 ||
      t->tail_wave > 64)
    return fail(VRT_ERR_INVALID, "tuning out of range");
  s->tune.refill_min = t->refill_min ? t->refill_min : 8;
  s->tune.trace_blocks_per_sm = t->trace_blocks_per_sm;
  s->tune.shade_blocks_per_sm = t->shade_blocks_per_sm ? t->shade_blocks_per_sm : 32;
  s->tune.trace_variant = t->trace_variant;
  s->tune.atrous_rows = t->atrous_tile_rows;
  s->tune.tail_wave = t->tail_wave;
  return VRT_OK;
}

static int check_uniforms(const VrtSession* s, const VrtUniforms* u);
static bool restir_on(const VrtUniforms* u) { return (u->params2[0] & kRfRestir) != 0u; }

// Autotuner: renders `frames` path-trace passes of `u` per candidate launch
// shape (refill threshold x occupancy variant x shading grid) and keeps the
// candidate with the smallest median pass time.  The session's history is
// reset afterwards (the candidate frames are not part of any sequence).
int vrt_session_autotune(VrtSession* s, const VrtUniforms* u, int frames, VrtTuning* best, float* best_ms) {
  if (!s || !u || frames < 1) return fail(VRT_ERR_INVALID, "bad argument");
  if (s->path_kernel != VRT_PATH_WAVEFRONT) return fail(VRT_ERR_STATE, "autotune needs the wavefront path kernel");
  if (int r = check_uniforms(s, u)) return r;
  if (restir_on(u)) return fail(VRT_ERR_INVALID, "autotune tunes the plain path's tracer (restir flags set)");
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  static const int refills[] = {4, 8, 12, 16, 24};
  static const int variants[] = {0, 1, 2};
  static const int shades[] = {8, 16, 32};
  const WavefrontTuning keep = s->tune;
  WavefrontTuning win = keep;
  float win_ms = 1e30f;
  std::vector<float> ms((size_t)frames);
  for (int rf : refills)
    for (int va : variants)
      for (int sh : shades) {
        s->tune.refill_min = rf;
        s->tune.trace_variant = va;
        s->tune.shade_blocks_per_sm = sh;
        s->tune.trace_blocks_per_sm = 0;
        if (int r = vrt_pass_pathtrace(s, u)) { s->tune = keep; return r; }   // warm-up
        for (int f = 0; f < frames; f++) {
          CUDA_TRY(cudaEventRecord(s->ev[0], st));
          if (int r = vrt_pass_pathtrace(s, u)) { s->tune = keep; return r; }
          CUDA_TRY(cudaEventRecord(s->ev[1], st));
          CUDA_TRY(cudaEventSynchronize(s->ev[1]));
          CUDA_TRY(cudaEventElapsedTime(&ms[(size_t)f], s->ev[0], s->ev[1]));
        }
        std::sort(ms.begin(), ms.end());
        const float med = ms[(size_t)frames / 2];
        if (med < win_ms) { win_ms = med; win = s->tune; }
      }
  s->tune = win;
  // where the remaining paths finish one thread each: automatic, never, or
  // from wave 2 / 3 (frames of more than one bounce)
  {
    const int nb = s->cache_on ? s->cache_cfg.train_bounces : (int)u->params0[1];
    float best_tail = 1e30f;
    int best_wave = win.tail_wave;
    for (int tw : {-1, 0, 2, 3}) {
      if (tw > 0 && tw >= nb + 2) continue;
      s->tune.tail_wave = tw;
      if (int r = vrt_pass_pathtrace(s, u)) { s->tune = keep; return r; }   // warm-up
      for (int f = 0; f < frames; f++) {
        CUDA_TRY(cudaEventRecord(s->ev[0], st));
        if (int r = vrt_pass_pathtrace(s, u)) { s->tune = keep; return r; }
        CUDA_TRY(cudaEventRecord(s->ev[1], st));
        CUDA_TRY(cudaEventSynchronize(s->ev[1]));
        CUDA_TRY(cudaEventElapsedTime(&ms[(size_t)f], s->ev[0], s->ev[1]));
      }
      std::sort(ms.begin(), ms.end());
      if (ms[(size_t)frames / 2] < best_tail) { best_tail = ms[(size_t)frames / 2]; best_wave = tw; }
    }
    s->tune.tail_wave = best_wave;
    win = s->tune;
    win_ms = best_tail;
  }
  // the a-trous tile shape: the three iterations of a frame timed per shape
  if (u->params0[2] & 2u) {
    if (int r = vrt_pass_temporal(s, u)) { s->tune = keep; return r; }
    float best_atrous = 1e30f;
    int best_rows = win.atrous_rows;
    for (int rows : {0, 16}) {
      s->tune.atrous_rows = rows;
      for (int it = 0; it < 3; it++)
        if (int r = vrt_pass_atrous(s, u, it)) { s->tune = keep; return r; }   // warm-up
      for (int f = 0; f < frames; f++) {
        CUDA_TRY(cudaEventRecord(s->ev[0], st));
        for (int it = 0; it < 3; it++)
          if (int r = vrt_pass_atrous(s, u, it)) { s->tune = keep; return r; }
        CUDA_TRY(cudaEventRecord(s->ev[1], st));
        CUDA_TRY(cudaEventSynchronize(s->ev[1]));
        CUDA_TRY(cudaEventElapsedTime(&ms[(size_t)f], s->ev[0], s->ev[1]));
      }
      std::sort(ms.begin(), ms.end());
      if (ms[(size_t)frames / 2] < best_atrous) { best_atrous = ms[(size_t)frames / 2]; best_rows = rows; }
    }
    s->tune.atrous_rows = best_rows;
    win = s->tune;
  }
  if (best) {
    best->refill_min = win.refill_min;
    best->trace_blocks_per_sm = win.trace_blocks_per_sm;
    best->shade_blocks_per_sm = win.shade_blocks_per_sm;
    best->trace_variant = win.trace_variant;
    best->atrous_tile_rows = win.atrous_rows;
    best->tail_wave = win.tail_wave;
  }
  if (best_ms) *best_ms = win_ms;
  return vrt_session_reset(s);
}

int vrt_session_set_timing(VrtSession* s, int enable) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  s->timing = enable != 0;
  return VRT_OK;
}

static int check_uniforms(const VrtSession* s, const VrtUniforms* u) {
  if (!u) return fail(VRT_ERR_INVALID, "uniforms is NULL");
  if ((int)u->params1[0] != s->W || (int)u->params1[1] != s->H)
    return fail(VRT_ERR_INVALID, "uniform render size %gx%g does not match session %dx%d", u->params1[0],
                u->params1[1], s->W, s->H);
  const uint32_t f = u->params2[0];
  if (f & ~kRestirFlagsImplemented)
    return fail(VRT_ERR_INVALID,
                "restir flags 0x%x: only RF_RESTIR|RF_TEMPORAL|RF_SPATIAL (preset=gi) and 0 (preset=base) are "
                "implemented", f);
  if (f != 0u && !(f & kRfRestir))
    return fail(VRT_ERR_INVALID, "restir flags 0x%x set without RF_RESTIR", f);
  return VRT_OK;
}


// Reservoir buffers of the session, allocated (zeroed) on first use.
static int ensure_restir(VrtSession* s) {
  if (s->restir_mem) return VRT_OK;
  const size_t bytes = px(s) * (32 + 32 + 80 + 8 + 4);
  if (int r = dev_alloc(s->ctx, &s->restir_mem, bytes, &s->bytes)) return r;
  s->restir_bytes = bytes;
  CUDA_TRY(cudaMemsetAsync(s->restir_mem, 0, bytes, s->ctx->stream));
  return VRT_OK;
}

static RestirBufs restir_bufs(const VrtSession* s, int parity) {
  RestirBufs rb;
  char* m = (char*)s->restir_mem;
  rb.resA = m;
  rb.resB = m + px(s) * 32;
  rb.scratch = m + px(s) * 64;   // 16-byte records before the 8- and 4-byte ones:
  rb.direct = m + px(s) * 144;   // every region starts on its own alignment for any P
  rb.dup = (float*)(m + px(s) * 152);
  rb.gbuf_prev = s->gbuf[1 - parity];
  rb.pairing = s->pairing;
  const VrtScene* sc = s->scene;
  rb.light_words = sc->light_words;
  rb.light_alias = sc->light_alias;
  rb.light_grid = sc->light_grid;
  return rb;
}

// Pairing textures for the frame's sigmas (main.js:252-263): texture 0 takes
// the wide sigma (params5.x) under RF_MIXSIGMA, the others the base sigma.
static int ensure_pairing(VrtSession* s, const VrtUniforms* u) {
  if (!(u->params2[0] & kRfPaired)) return VRT_OK;
  const double base = std::max(0.8, s->pairing_sigma);
  const double wide = (u->params2[0] & kRfMixSigma) ? std::max(0.8, (double)u->params5[0]) : base;
  const double want[3] = {wide, base, base};
  if (s->pairing && std::equal(want, want + 3, s->pairing_built)) return VRT_OK;
  if (!s->pairing)
    if (int r = dev_alloc(s->ctx, (void**)&s->pairing, (size_t)kPairingWords * 4, &s->bytes)) return r;
  std::vector<uint32_t> host(kPairingWords);
  make_pairing_buffer(want, host.data());
  CUDA_TRY(cudaMemcpyAsync(s->pairing, host.data(), host.size() * 4, cudaMemcpyHostToDevice, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  std::copy(want, want + 3, s->pairing_built);
  return VRT_OK;
}

// Unified NEE reads the scene's light list (built on first use; an edited
// scene's lights are rebuilt by vrt_scene_build_lights).
static int ensure_lights(VrtSession* s, const VrtUniforms* u) {
  if (!(u->params2[0] & kRfUnified) || u->params2[1] == 0u) return VRT_OK;
  if (!s->scene->lights_built)
    if (int r = vrt_scene_build_lights(s->scene, nullptr)) return r;
  if (u->params2[1] > s->scene->light_count)
    return fail(VRT_ERR_INVALID, "params2.y = %u lights, the scene has %u", u->params2[1], s->scene->light_count);
  if ((u->params2[0] & kRfLightGrid) && !s->scene->light_grid)
    return fail(VRT_ERR_STATE, "light grid not built");
  return VRT_OK;
}

static int parity_of(const VrtSession* s) { return (int)(s->frame_counter & 1u); }
static int cache_frame(VrtSession* s, const VrtUniforms* u, const PathOut& o);
static CacheLaunch cache_launch_of(VrtSession* s, uint32_t frame);

int vrt_pass_pathtrace(VrtSession* s, const VrtUniforms* u) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (int r = set_dev(s->ctx)) return r;
  PathOut o;
  o.rad16 = s->rad16; o.rad32 = s->rad32; o.alb8 = s->alb8; o.gbuf = s->gbuf[parity_of(s)]; o.stats = s->stats;
  if (s->path_kernel == VRT_PATH_BATCH_ONLY)
    return fail(VRT_ERR_STATE, "session was created for batches only (VRT_PATH_BATCH_ONLY)");
  if (restir_on(u)) {
    if (s->cache_on) return fail(VRT_ERR_STATE, "the radiance cache serves the plain path only (restir flags set)");
    if (int r = ensure_restir(s)) return r;
    if (int r = ensure_lights(s, u)) return r;
    const RestirBufs rb = restir_bufs(s, parity_of(s));
    if (s->path_kernel == VRT_PATH_WAVEFRONT && (u->params2[0] & kRfUnified) && s->wf.slots >= 2 &&
        (int)u->params0[1] + 5 <= s->wf.max_waves) {
      CUDA_TRY(launch_restir_unified_wavefront(s->scene->dev, *u, s->fclamp, s->W, s->H, o, rb, s->wf, s->tune,
                                               s->ctx->stream, &s->launches, s->timing ? s->tev : nullptr,
                                               VrtSession::kTimedWaves, &s->timed_waves));
    } else if (s->path_kernel == VRT_PATH_WAVEFRONT && !(u->params2[0] & kRfUnified) &&
               (int)u->params0[1] + 3 <= s->wf.max_waves) {
      CUDA_TRY(launch_restir_initial_wavefront(s->scene->dev, *u, s->fclamp, s->W, s->H, o, rb, s->wf, s->tune,
                                               s->ctx->stream, &s->launches, s->timing ? s->tev : nullptr,
                                               VrtSession::kTimedWaves, &s->timed_waves));
    } else {
      CUDA_TRY(launch_restir_initial(s->scene->dev, *u, s->fclamp, s->W, s->H, o, rb, s->ctx->stream));
      s->launches++;
    }
    return VRT_OK;
  }
  if (s->cache_on) return cache_frame(s, u, o);
  if (s->path_kernel == VRT_PATH_WAVEFRONT && (int)u->params0[1] + 3 <= s->wf.max_waves) {
    CUDA_TRY(launch_wavefront(s->scene->dev, *u, s->fclamp, s->W, s->H, o, s->wf, s->tune, s->ctx->stream,
                              &s->launches, s->timing ? s->tev : nullptr, VrtSession::kTimedWaves,
                              &s->timed_waves));
  } else {
    CUDA_TRY(launch_pathtrace(s->scene->dev, *u, s->fclamp, s->W, s->H, o, s->ctx->stream));
    s->launches++;
  }
  return VRT_OK;
}

static int restir_pass(VrtSession* s, const VrtUniforms* u, bool spatial) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (!restir_on(u)) return fail(VRT_ERR_STATE, "reservoir reuse needs RF_RESTIR in params2.x");
  if (!s->restir_mem) return fail(VRT_ERR_STATE, "reservoir reuse before the initial pass of a ReSTIR frame");
  if (int r = set_dev(s->ctx)) return r;
  const int p = parity_of(s);
  PathOut o;
  o.rad16 = s->rad16; o.rad32 = s->rad32; o.alb8 = s->alb8; o.gbuf = s->gbuf[p]; o.stats = s->stats;
  if (spatial)
    if (int r = ensure_pairing(s, u)) return r;
  // visibility rays (up to four per pixel with vector weights) on the wavefront tracer
  if (spatial && s->path_kernel == VRT_PATH_WAVEFRONT && s->wf.slots >= 4) {
    CUDA_TRY(launch_restir_spatial_wavefront(s->scene->dev, *u, s->W, s->H, o, restir_bufs(s, p), s->wf, s->tune,
                                             s->ctx->stream, &s->launches));
    return VRT_OK;
  }
  if (spatial) {
    CUDA_TRY(launch_restir_spatial(s->scene->dev, *u, s->W, s->H, o, restir_bufs(s, p), s->ctx->stream));
  } else {
    if (!(u->params2[0] & kRfTemporal)) return VRT_OK;   // reuse_temporal.wgsl:144
    CUDA_TRY(launch_restir_temporal(s->scene->dev, *u, s->W, s->H, o, restir_bufs(s, p), s->ctx->stream));
  }
  s->launches++;
  return VRT_OK;
}

int vrt_pass_reuse_temporal(VrtSession* s, const VrtUniforms* u) { return restir_pass(s, u, false); }
int vrt_pass_reuse_spatial(VrtSession* s, const VrtUniforms* u) { return restir_pass(s, u, true); }

int vrt_pass_dupmap(VrtSession* s, const VrtUniforms* u) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (!restir_on(u) || !(u->params2[0] & (kRfDupmap | kRfMutate))) return VRT_OK;   // main.js:741
  if (!s->restir_mem) return fail(VRT_ERR_STATE, "duplication map before the initial pass of a ReSTIR frame");
  if (int r = set_dev(s->ctx)) return r;
  CUDA_TRY(launch_restir_dupmap(*u, s->W, s->H, restir_bufs(s, parity_of(s)), s->ctx->stream));
  s->launches++;
  return VRT_OK;
}

int vrt_session_set_pairing_sigma(VrtSession* s, float sigma) {
  if (!s || !(sigma > 0.0f)) return fail(VRT_ERR_INVALID, "bad argument");
  s->pairing_sigma = (double)sigma;
  return VRT_OK;
}

int vrt_pass_temporal(VrtSession* s, const VrtUniforms* u) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (int r = set_dev(s->ctx)) return r;
  const int p = parity_of(s);
  CUDA_TRY(launch_temporal(*u, s->W, s->H, s->rad16, s->gbuf[p], s->accum[1 - p], s->gbuf[1 - p], s->accum[p],
                           s->acc_f32, s->ctx->stream));
  s->launches++;
  return VRT_OK;
}

int vrt_pass_atrous(VrtSession* s, const VrtUniforms* u, int it) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (it < 0 || it > 2) return fail(VRT_ERR_INVALID, "a-trous iteration %d not in 0..2", it);
  if (int r = set_dev(s->ctx)) return r;
  const int p = parity_of(s);
  // chain accum -> dA (1) -> dB (2) -> dA (4)   (main.js:503-507)
  const void* src = it == 0 ? s->accum[p] : (it == 1 ? s->den[0] : s->den[1]);
  const bool src_f32 = it == 0 && s->acc_f32;
  void* dst = it == 1 ? s->den[1] : s->den[0];
  CUDA_TRY(launch_atrous_staged(s->W, s->H, src, src_f32, s->gbuf[p], dst, 1 << it, s->stats + kStatError,
                                s->ctx->stream, s->tune.atrous_rows));
  s->launches++;
  return VRT_OK;
}

static const void* final_buf(const VrtSession* s, int parity, bool denoise, bool* f32) {
  *f32 = !denoise && s->acc_f32;
  return denoise ? s->den[0] : s->accum[parity];
}

int vrt_pass_present(VrtSession* s, const VrtUniforms* u) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (int r = set_dev(s->ctx)) return r;
  const bool denoise = (u->params0[2] & 2u) != 0u;
  bool f32;
  const void* fin = final_buf(s, parity_of(s), denoise, &f32);
  CUDA_TRY(launch_present(*u, s->W, s->H, fin, f32, s->alb8, s->ldr, s->ctx->present_lut, s->ctx->stream));
  s->launches++;
  s->last_denoise = denoise;
  return VRT_OK;
}

int vrt_end_frame(VrtSession* s) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  s->last_parity = parity_of(s);
  s->have_frame = true;
  s->frame_counter++;
  return VRT_OK;
}

int vrt_frame(VrtSession* s, const VrtUniforms* u) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = check_uniforms(s, u)) return r;
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  s->launches = 0;
  s->timed_waves = 0;
  CUDA_TRY(cudaMemsetAsync(s->stats, 0, kStatCount * 8, st));
  if (s->timing) CUDA_TRY(cudaEventRecord(s->ev[0], st));
  if (int r = vrt_pass_pathtrace(s, u)) return r;
  s->restir_timed = restir_on(u) && s->timing;
  if (restir_on(u)) {   // main.js:737-739
    if (s->timing) CUDA_TRY(cudaEventRecord(s->ev[5], st));
    if (u->params2[0] & kRfTemporal)
      if (int r = vrt_pass_reuse_temporal(s, u)) return r;
    if (int r = vrt_pass_reuse_spatial(s, u)) return r;
    if (int r = vrt_pass_dupmap(s, u)) return r;
  }
  if (s->timing) CUDA_TRY(cudaEventRecord(s->ev[1], st));
  if (int r = vrt_pass_temporal(s, u)) return r;
  if (s->timing) CUDA_TRY(cudaEventRecord(s->ev[2], st));
  const bool denoise = (u->params0[2] & 2u) != 0u;
  if (denoise)
    for (int it = 0; it < 3; it++)
      if (int r = vrt_pass_atrous(s, u, it)) return r;
  if (s->timing) CUDA_TRY(cudaEventRecord(s->ev[3], st));
  if (int r = vrt_pass_present(s, u)) return r;
  if (s->timing) {
    CUDA_TRY(cudaEventRecord(s->ev[4], st));
    s->events_frame = s->frame_counter;
  }
  return vrt_end_frame(s);
}

int vrt_session_last_stats(VrtSession* s, VrtFrameStats* out) {
  if (!s || !out) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(s->ctx)) return r;
  std::memset(out, 0, sizeof(*out));
  unsigned long long h[kStatCount];
  CUDA_TRY(cudaMemcpyAsync(h, s->stats, sizeof h, cudaMemcpyDeviceToHost, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  out->rays = h[kStatRays];
  out->dda_outer = h[kStatOuter];
  out->dda_inner = h[kStatInner];
  out->voxel_reads = h[kStatVReads];
  out->pixels = h[kStatPixels];
  out->trace_step_slots = h[kStatTraceSlots];
  out->launches = s->launches;
  if (h[kStatError]) return fail(VRT_ERR_TIMEOUT, "a bounded wait for staged image tiles ran out");
  out->cache_on = s->cache_on ? 1u : 0u;
  out->cache_queries = h[kStatCacheQueries];
  out->cache_samples = h[kStatCacheSamples];
  if (s->cache_on && s->mlp) {
    if (int r = vrt_mlp_check(s->mlp)) return r;
  }
  if (s->timing && s->have_frame && s->cache_timed) CUDA_TRY(cudaEventElapsedTime(&out->ms_cache, s->cev[0], s->cev[1]));
  // pass timings exist only for a frame rendered by vrt_frame with timing on
  if (s->timing && s->have_frame && s->events_frame + 1 == s->frame_counter) {
    float a = 0, b = 0, c = 0, d = 0;
    CUDA_TRY(cudaEventElapsedTime(&a, s->ev[0], s->ev[1]));
    CUDA_TRY(cudaEventElapsedTime(&b, s->ev[1], s->ev[2]));
    CUDA_TRY(cudaEventElapsedTime(&c, s->ev[2], s->ev[3]));
    CUDA_TRY(cudaEventElapsedTime(&d, s->ev[3], s->ev[4]));
    out->ms_pathtrace = a; out->ms_temporal = b; out->ms_atrous = c; out->ms_present = d;
    out->ms_total = a + b + c + d;
    float tr = 0.0f;
    for (int w = 0; w < s->timed_waves; w++) {
      float x = 0.0f;
      CUDA_TRY(cudaEventElapsedTime(&x, s->tev[2 * w], s->tev[2 * w + 1]));
      tr += x;
    }
    out->ms_trace = tr;
    out->trace_launches = (uint32_t)s->timed_waves;
    if (s->restir_timed) CUDA_TRY(cudaEventElapsedTime(&out->ms_reuse, s->ev[5], s->ev[1]));
  }
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// readbacks
// ---------------------------------------------------------------------------
static int read_buf(VrtSession* s, const void* dev, size_t need, void* host, size_t bytes) {
  if (!s || !host) return fail(VRT_ERR_INVALID, "NULL argument");
  if (!dev) return fail(VRT_ERR_STATE, "buffer not allocated for this session");
  if (bytes < need) return fail(VRT_ERR_INVALID, "host buffer %zu bytes < %zu needed", bytes, need);
  if (int r = set_dev(s->ctx)) return r;
  CUDA_TRY(cudaMemcpyAsync(host, dev, need, cudaMemcpyDeviceToHost, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  return VRT_OK;
}

static int done_parity(const VrtSession* s) { return s->have_frame ? s->last_parity : parity_of(s); }

int vrt_read_radiance(VrtSession* s, void* h, size_t b) { return read_buf(s, s ? s->rad16 : nullptr, s ? px(s) * 8 : 0, h, b); }
int vrt_read_radiance_f32(VrtSession* s, void* h, size_t b) { return read_buf(s, s ? s->rad32 : nullptr, s ? px(s) * 16 : 0, h, b); }
int vrt_read_albedo(VrtSession* s, void* h, size_t b) { return read_buf(s, s ? s->alb8 : nullptr, s ? px(s) * 4 : 0, h, b); }
int vrt_read_gbuffer(VrtSession* s, void* h, size_t b) {
  return read_buf(s, s ? s->gbuf[done_parity(s)] : nullptr, s ? px(s) * 16 : 0, h, b);
}
int vrt_read_accum(VrtSession* s, void* h, size_t b) {
  return read_buf(s, s ? s->accum[done_parity(s)] : nullptr, s ? px(s) * acc_bpp(s) : 0, h, b);
}
int vrt_read_denoise(VrtSession* s, int i, void* h, size_t b) {
  if (i < 0 || i > 1) return fail(VRT_ERR_INVALID, "denoise index %d", i);
  return read_buf(s, s ? s->den[i] : nullptr, s ? px(s) * 8 : 0, h, b);
}
int vrt_read_final(VrtSession* s, void* h, size_t b) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  bool f32;
  const void* fin = final_buf(s, done_parity(s), s->last_denoise, &f32);
  return read_buf(s, fin, px(s) * (f32 ? 16 : 8), h, b);
}
int vrt_read_ldr(VrtSession* s, void* h, size_t b) { return read_buf(s, s ? s->ldr : nullptr, s ? px(s) * 4 : 0, h, b); }
int vrt_read_reservoirs(VrtSession* s, int which, void* h, size_t b) {
  if (which < 0 || which > 1) return fail(VRT_ERR_INVALID, "reservoir set %d (0 = A, 1 = B)", which);
  if (s && !s->restir_mem) return fail(VRT_ERR_STATE, "no ReSTIR frame rendered by this session");
  return read_buf(s, s ? (const char*)s->restir_mem + (size_t)which * px(s) * 32 : nullptr, s ? px(s) * 32 : 0, h,
                  b);
}
int vrt_read_dupmap(VrtSession* s, void* h, size_t b) {
  if (s && !s->restir_mem) return fail(VRT_ERR_STATE, "no ReSTIR frame rendered by this session");
  return read_buf(s, s ? (const char*)s->restir_mem + px(s) * 152 : nullptr, s ? px(s) * 4 : 0, h, b);
}
int vrt_read_direct(VrtSession* s, void* h, size_t b) {
  if (s && !s->restir_mem) return fail(VRT_ERR_STATE, "no ReSTIR frame rendered by this session");
  return read_buf(s, s ? (const char*)s->restir_mem + px(s) * 144 : nullptr, s ? px(s) * 8 : 0, h, b);
}

static float half_to_float(uint16_t hbits) {
  const uint32_t sign = (uint32_t)(hbits & 0x8000u) << 16;
  const uint32_t e = (hbits >> 10) & 0x1fu, m = hbits & 0x3ffu;
  uint32_t out;
  if (e == 0) {
    float v = (float)m * 5.96046448e-08f;
    return sign ? -v : v;
  }
  if (e == 31) out = sign | 0x7f800000u | (m << 13);
  else out = sign | ((e + 112u) << 23) | (m << 13);
  float f;
  std::memcpy(&f, &out, 4);
  return f;
}

// HDR capture of main.js:628-659: illum * (a/255)^2 in double, stored f32.
int vrt_read_hdr(VrtSession* s, float* rgb, size_t bytes) {
  if (!s || !rgb) return fail(VRT_ERR_INVALID, "NULL argument");
  const size_t P = px(s);
  if (bytes < P * 12) return fail(VRT_ERR_INVALID, "host buffer %zu bytes < %zu needed", bytes, P * 12);
  bool f32;
  final_buf(s, done_parity(s), s->last_denoise, &f32);
  std::vector<uint8_t> fin(P * (f32 ? 16 : 8));
  std::vector<uint8_t> alb(P * 4);
  if (int r = vrt_read_final(s, fin.data(), fin.size())) return r;
  if (int r = vrt_read_albedo(s, alb.data(), alb.size())) return r;
  for (size_t p = 0; p < P; p++) {
    for (int c = 0; c < 3; c++) {
      double il;
      if (f32) {
        float v;
        std::memcpy(&v, fin.data() + p * 16 + c * 4, 4);
        il = v;
      } else {
        uint16_t hb;
        std::memcpy(&hb, fin.data() + p * 8 + c * 2, 2);
        il = half_to_float(hb);
      }
      const double a = (double)alb[p * 4 + c] / 255.0;
      rgb[p * 3 + c] = (float)((il * a) * a);
    }
  }
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
}  // extern "C"

struct VrtBatch {
  VrtCtx* ctx = nullptr;
  std::vector<VrtSession*> sessions;   // job slots (a server's free slots are NULL)
  uint32_t P = 0;                      // pixel capacity of the scratch pool
  uint64_t bytes = 0;
  JobHost* h_jobs = nullptr;          // pinned staging of the job table
  uint32_t* h_firsts = nullptr;       // pinned staging of the jobs' first pixels
  void* d_jobs = nullptr;
  uint32_t* d_firsts = nullptr;
  void* wf_mem = nullptr;
  size_t wf_bytes = 0;
  WavefrontBufs wf;
  WavefrontTuning tune;
  unsigned long long* stats = nullptr;
  bool use_graph = true;
  cudaGraphExec_t gexec = nullptr;
  int graph_waves = -1;
  WavefrontTuning graph_tune;
  uint64_t graph_cache_sig = 0;
  uint32_t graph_launches = 0;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr, ev_upload = nullptr;
  bool uploaded = false;
  uint32_t launches = 0;
  bool have_frame = false;
};

static void batch_drop_graph(VrtBatch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->graph_waves = -1;
}

extern "C" {

int vrt_batch_destroy(VrtBatch* b) {
  if (!b) return VRT_OK;
  VrtCtx* c = b->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  batch_drop_graph(b);
  dev_free(c, b->d_jobs, b->sessions.size() * sizeof(JobHost), &b->bytes);
  dev_free(c, b->d_firsts, (3 * b->sessions.size() + 2) * 4, &b->bytes);
  dev_free(c, b->wf_mem, b->wf_bytes, &b->bytes);
  dev_free(c, b->stats, kStatCount * 8, &b->bytes);
  if (b->h_jobs) cudaFreeHost(b->h_jobs);
  if (b->h_firsts) cudaFreeHost(b->h_firsts);
  for (cudaEvent_t e : {b->ev_start, b->ev_end, b->ev_upload})
    if (e) cudaEventDestroy(e);
  delete b;
  return VRT_OK;
}

}  // extern "C"

// A batch with n job slots and a scratch pool for P pixels per launch; the
// slots are filled from `sessions` (NULL: all slots free).
static int batch_create_capacity(VrtCtx* ctx, VrtSession* const* sessions, int n, uint64_t P, VrtBatch** out) {
  if (P >= (1ull << 31)) return fail(VRT_ERR_INVALID, "batch of %llu pixels exceeds 2^31", (unsigned long long)P);
  if (P < 1 || n < 1) return fail(VRT_ERR_INVALID, "empty batch");
  if (int r = set_dev(ctx)) return r;
  VrtBatch* b = new VrtBatch();
  b->ctx = ctx;
  // batch default launch shape: the tracer variant that holds its walk in registers for the batch's
  // job lookups (6 steps per pass, 4 blocks per SM; the 8 x 5 shape spills there), refill at 16 idle lanes
  b->tune.trace_variant = 2;
  b->tune.refill_min = 16;
  if (sessions) b->sessions.assign(sessions, sessions + n);
  else b->sessions.assign((size_t)n, nullptr);
  b->P = (uint32_t)P;
  const int max_waves = 72;
  b->wf_bytes = wavefront_bytes((int)b->P, 1, max_waves);
  int r = dev_alloc(ctx, &b->wf_mem, b->wf_bytes, &b->bytes);
  if (!r) r = dev_alloc(ctx, &b->d_jobs, (size_t)n * sizeof(JobHost), &b->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&b->d_firsts, (size_t)(3 * n + 2) * 4, &b->bytes);   // firsts, tile tables
  if (!r) r = dev_alloc(ctx, (void**)&b->stats, kStatCount * 8, &b->bytes);
  if (!r && (cudaMallocHost((void**)&b->h_jobs, (size_t)n * sizeof(JobHost)) != cudaSuccess ||
             cudaMallocHost((void**)&b->h_firsts, (size_t)(3 * n + 2) * 4) != cudaSuccess))
    r = fail(VRT_ERR_OOM, "pinned job table");
  if (!r && (cudaEventCreate(&b->ev_start) != cudaSuccess || cudaEventCreate(&b->ev_end) != cudaSuccess ||
             cudaEventCreateWithFlags(&b->ev_upload, cudaEventDisableTiming) != cudaSuccess))
    r = fail(VRT_ERR_CUDA, "cudaEventCreate failed");
  if (r) {
    std::string keep = g_err;
    vrt_batch_destroy(b);
    g_err = keep;
    return r;
  }
  carve_wavefront(b->wf_mem, b->P, max_waves, b->wf);
  *out = b;
  return VRT_OK;
}

extern "C" {

int vrt_batch_create(VrtCtx* ctx, VrtSession* const* sessions, int n, VrtBatch** out) {
  if (!ctx || !sessions || n < 1 || !out) return fail(VRT_ERR_INVALID, "bad argument");
  *out = nullptr;
  uint64_t P = 0;
  for (int i = 0; i < n; i++) {
    if (!sessions[i] || sessions[i]->ctx != ctx) return fail(VRT_ERR_INVALID, "session %d is NULL or of another context", i);
    for (int k = 0; k < i; k++)
      if (sessions[k] == sessions[i]) return fail(VRT_ERR_INVALID, "session %d appears twice", i);
    P += (uint64_t)sessions[i]->W * sessions[i]->H;
  }
  return batch_create_capacity(ctx, sessions, n, P, out);
}

int vrt_batch_set_graph(VrtBatch* b, int enable) {
  if (!b) return fail(VRT_ERR_INVALID, "batch is NULL");
  b->use_graph = enable != 0;
  if (!b->use_graph) batch_drop_graph(b);
  return VRT_OK;
}

int vrt_batch_set_tuning(VrtBatch* b, const VrtTuning* t) {
  if (!b || !t) return fail(VRT_ERR_INVALID, "NULL argument");
  if (t->refill_min < 0 || t->refill_min > 32 || t->trace_blocks_per_sm < 0 || t->trace_blocks_per_sm > 32 ||
      t->shade_blocks_per_sm < 0 || t->shade_blocks_per_sm > 64 || t->trace_variant < 0 || t->trace_variant > 8 ||
      (t->atrous_tile_rows != 0 && t->atrous_tile_rows != 8 && t->atrous_tile_rows != 16) || t->tail_wave < -1 ||
      t->tail_wave > 64)
    return fail(VRT_ERR_INVALID, "tuning out of range");
  b->tune.refill_min = t->refill_min ? t->refill_min : 8;
  b->tune.atrous_rows = t->atrous_tile_rows;
  b->tune.trace_blocks_per_sm = t->trace_blocks_per_sm;
  b->tune.shade_blocks_per_sm = t->shade_blocks_per_sm ? t->shade_blocks_per_sm : 32;
  b->tune.trace_variant = t->trace_variant;
  b->tune.tail_wave = t->tail_wave;
  return VRT_OK;
}

static bool same_tuning(const WavefrontTuning& a, const WavefrontTuning& c) {
  return a.refill_min == c.refill_min && a.trace_blocks_per_sm == c.trace_blocks_per_sm &&
         a.shade_blocks_per_sm == c.shade_blocks_per_sm && a.trace_variant == c.trace_variant &&
         a.tail_wave == c.tail_wave && a.atrous_rows == c.atrous_rows;
}

}  // extern "C"

// One frame for sessions idx[0..m) of the batch (all of them when idx is
// NULL), uniforms u[0..m).  The CUDA graph is used only for the full set in
// creation order.
static int batch_frame_impl(VrtBatch* b, const int* idx, int m, const VrtUniforms* u) {
  const int n = (int)b->sessions.size();
  if (m < 1 || m > n) return fail(VRT_ERR_INVALID, "job count %d not in 1..%d", m, n);
  bool full = idx == nullptr && m == n;
  std::vector<VrtSession*> ss((size_t)m);
  for (int i = 0; i < m; i++) {
    const int k = idx ? idx[i] : i;
    if (k < 0 || k >= n) return fail(VRT_ERR_INVALID, "job index %d out of range", k);
    ss[(size_t)i] = b->sessions[(size_t)k];
    if (!ss[(size_t)i]) return fail(VRT_ERR_INVALID, "job slot %d holds no session", k);
    for (int q = 0; q < i; q++)
      if (ss[(size_t)q] == ss[(size_t)i]) return fail(VRT_ERR_INVALID, "session %d listed twice", k);
  }
  int maxB = 0;
  uint64_t cache_sig = 0x9e3779b97f4a7c15ull;
  for (int i = 0; i < m; i++) {
    VrtSession* s = ss[(size_t)i];
    if (int r = check_uniforms(s, &u[i])) return r;
    if (restir_on(&u[i])) return fail(VRT_ERR_INVALID, "batched frames render the plain path (restir flags set)");
    maxB = std::max(maxB, s->cache_on ? s->cache_cfg.train_bounces : (int)u[i].params0[1]);
    if (s->cache_on && !s->mlp) return fail(VRT_ERR_STATE, "cache session without a network");
    // the captured graph bakes each cache job's buffers and sizes in
    const uint64_t v = s->cache_on ? (s->cache_version * 0x100000001b3ull) ^ (uint64_t)s->scene->dev.N : 0ull;
    cache_sig = (cache_sig ^ (v + (uint64_t)i)) * 0x100000001b3ull;
  }
  const int waves = maxB + 2;
  if (waves + 1 > b->wf.max_waves) return fail(VRT_ERR_INVALID, "bounce count %d too large for a batch", maxB);
  if (int r = set_dev(b->ctx)) return r;
  cudaStream_t st = b->ctx->stream;
  // the staging tables may still be read by the previous frame's upload
  if (b->uploaded) CUDA_TRY(cudaEventSynchronize(b->ev_upload));
  uint32_t first = 0;
  std::vector<CacheLaunch> cls;
  const bool graph = b->use_graph && full;
  for (int i = 0; i < m; i++) {
    VrtSession* s = ss[(size_t)i];
    JobHost& j = b->h_jobs[i];
    std::memset(&j, 0, sizeof j);
    const int p = parity_of(s);
    j.u = u[i];
    j.vox = s->scene->dev.vox; j.masks = s->scene->dev.masks; j.bits = s->scene->dev.bits;
    j.N = s->scene->dev.N; j.BG = s->scene->dev.BG;
    j.rad16 = s->rad16; j.rad32 = s->rad32; j.alb8 = s->alb8; j.gbuf = s->gbuf[p];
    j.W = s->W; j.H = s->H; j.first = first; j.fclamp = s->fclamp;
    j.acc_prev = s->accum[1 - p]; j.acc_cur = s->accum[p]; j.gbuf_prev = s->gbuf[1 - p];
    j.den0 = s->den[0]; j.den1 = s->den[1]; j.ldr = s->ldr; j.acc_f32 = s->acc_f32 ? 1 : 0;
    if (s->cache_on) {
      cls.push_back(cache_launch_of(s, u[i].params0[0]));
      j.cache = cls.back().cd;
    }
    b->h_firsts[i] = first;
    first += (uint32_t)(s->W * s->H);
  }
  const uint32_t P = first;
  if (P > b->P) return fail(VRT_ERR_INVALID, "batch frame of %u pixels exceeds the pool's %u", P, b->P);
  // a-trous tile tables: prefix counts of each job's 32 x 16 and 32 x 8 tiles
  uint32_t* t16 = b->h_firsts + n;
  uint32_t* t8 = t16 + n + 1;
  t16[0] = t8[0] = 0u;
  for (int i = 0; i < m; i++) {
    const VrtSession* s = ss[(size_t)i];
    const uint32_t tw = (uint32_t)(s->W + 31) / 32u;
    t16[i + 1] = t16[i] + tw * (uint32_t)((s->H + 15) / 16);
    t8[i + 1] = t8[i] + tw * (uint32_t)((s->H + 7) / 8);
  }
  const AtrousTiles at{b->d_firsts + n, b->d_firsts + 2 * n + 1, t16[m], t8[m]};
  CUDA_TRY(cudaMemcpyAsync(b->d_jobs, b->h_jobs, (size_t)m * sizeof(JobHost), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(b->d_firsts, b->h_firsts, (size_t)(3 * n + 2) * 4, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaEventRecord(b->ev_upload, st));
  b->uploaded = true;
  CUDA_TRY(cudaMemsetAsync(b->stats, 0, kStatCount * 8, st));
  CUDA_TRY(cudaEventRecord(b->ev_start, st));
  b->launches = 0;
  if (graph) {
    if (!b->gexec || b->graph_waves != waves || !same_tuning(b->graph_tune, b->tune) ||
        b->graph_cache_sig != cache_sig) {
      batch_drop_graph(b);
      cudaGraph_t graph = nullptr;
      CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      uint32_t nl = 0;
      cudaError_t e = launch_batch_frame(b->d_jobs, b->d_firsts, m, P, waves, b->wf, b->tune, b->stats, st, &nl,
                                         b->ctx->present_lut, cls.data(), (int)cls.size(), &at);
      cudaError_t e2 = cudaStreamEndCapture(st, &graph);
      if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(VRT_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
      }
      e = cudaGraphInstantiate(&b->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        b->gexec = nullptr;
        return fail(VRT_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
      }
      b->graph_waves = waves;
      b->graph_tune = b->tune;
      b->graph_cache_sig = cache_sig;
      b->graph_launches = nl;
    }
    b->launches = b->graph_launches;
    CUDA_TRY(cudaGraphLaunch(b->gexec, st));
  } else {
    CUDA_TRY(launch_batch_frame(b->d_jobs, b->d_firsts, m, P, waves, b->wf, b->tune, b->stats, st, &b->launches,
                                b->ctx->present_lut, cls.data(), (int)cls.size(), &at));
  }
  CUDA_TRY(cudaEventRecord(b->ev_end, st));
  for (int i = 0; i < m; i++) {
    VrtSession* s = ss[(size_t)i];
    s->last_denoise = (u[i].params0[2] & 2u) != 0u;
    s->launches = 0;
    vrt_end_frame(s);
  }
  b->have_frame = true;
  return VRT_OK;
}

extern "C" {

int vrt_batch_frame(VrtBatch* b, const VrtUniforms* u) {
  if (!b || !u) return fail(VRT_ERR_INVALID, "NULL argument");
  return batch_frame_impl(b, nullptr, (int)b->sessions.size(), u);
}

int vrt_batch_frame_subset(VrtBatch* b, const int* idx, int m, const VrtUniforms* u) {
  if (!b || !idx || !u) return fail(VRT_ERR_INVALID, "NULL argument");
  return batch_frame_impl(b, idx, m, u);
}

int vrt_batch_last_stats(VrtBatch* b, VrtFrameStats* out) {
  if (!b || !out) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(b->ctx)) return r;
  std::memset(out, 0, sizeof(*out));
  unsigned long long h[kStatCount];
  CUDA_TRY(cudaMemcpyAsync(h, b->stats, sizeof h, cudaMemcpyDeviceToHost, b->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(b->ctx->stream));
  out->rays = h[kStatRays];
  out->dda_outer = h[kStatOuter];
  out->dda_inner = h[kStatInner];
  out->voxel_reads = h[kStatVReads];
  out->pixels = h[kStatPixels];
  out->trace_step_slots = h[kStatTraceSlots];
  out->launches = b->launches;
  out->cache_queries = h[kStatCacheQueries];
  out->cache_samples = h[kStatCacheSamples];
  for (VrtSession* s : b->sessions)
    if (s && s->cache_on) {
      out->cache_on = 1u;
      if (int r = vrt_mlp_check(s->mlp)) return r;
    }
  if (b->have_frame) {
    float ms = 0.0f;
    CUDA_TRY(cudaEventElapsedTime(&ms, b->ev_start, b->ev_end));
    out->ms_total = ms;
  }
  return VRT_OK;
}

int vrt_batch_autotune(VrtBatch* b, const VrtUniforms* u, int frames, VrtTuning* best, float* best_ms) {
  if (!b || !u || frames < 1) return fail(VRT_ERR_INVALID, "bad argument");
  static const int refills[] = {4, 8, 12, 16, 24};
  static const int variants[] = {0, 1, 2};
  static const int shades[] = {8, 16, 32};
  const WavefrontTuning keep = b->tune;
  const bool keep_graph = b->use_graph;
  WavefrontTuning win = keep;
  float win_ms = 1e30f;
  std::vector<float> ms((size_t)frames);
  b->use_graph = false;
  for (int rf : refills)
    for (int va : variants)
      for (int sh : shades) {
        b->tune.refill_min = rf;
        b->tune.trace_variant = va;
        b->tune.shade_blocks_per_sm = sh;
        b->tune.trace_blocks_per_sm = 0;
        int r = vrt_batch_frame(b, u);
        for (int f = 0; f < frames && !r; f++) {
          r = vrt_batch_frame(b, u);
          VrtFrameStats st;
          if (!r) r = vrt_batch_last_stats(b, &st);
          ms[(size_t)f] = st.ms_total;
        }
        if (r) { b->tune = keep; b->use_graph = keep_graph; return r; }
        std::sort(ms.begin(), ms.end());
        if (ms[(size_t)frames / 2] < win_ms) { win_ms = ms[(size_t)frames / 2]; win = b->tune; }
      }
  // where the remaining paths of the batch finish one thread each (0: never)
  for (int tw : {2, 3, 4}) {
    b->tune = win;
    b->tune.tail_wave = tw;
    int r = vrt_batch_frame(b, u);
    for (int f = 0; f < frames && !r; f++) {
      r = vrt_batch_frame(b, u);
      VrtFrameStats st;
      if (!r) r = vrt_batch_last_stats(b, &st);
      ms[(size_t)f] = st.ms_total;
    }
    if (r) { b->tune = keep; b->use_graph = keep_graph; return r; }
    std::sort(ms.begin(), ms.end());
    if (ms[(size_t)frames / 2] < win_ms) { win_ms = ms[(size_t)frames / 2]; win = b->tune; }
  }
  // the a-trous tile rows (8 at every step, or 16 at steps 1-2)
  {
    b->tune = win;
    b->tune.atrous_rows = win.atrous_rows == 16 ? 0 : 16;
    int r = vrt_batch_frame(b, u);
    for (int f = 0; f < frames && !r; f++) {
      r = vrt_batch_frame(b, u);
      VrtFrameStats st;
      if (!r) r = vrt_batch_last_stats(b, &st);
      ms[(size_t)f] = st.ms_total;
    }
    if (r) { b->tune = keep; b->use_graph = keep_graph; return r; }
    std::sort(ms.begin(), ms.end());
    if (ms[(size_t)frames / 2] < win_ms) { win_ms = ms[(size_t)frames / 2]; win = b->tune; }
  }
  b->tune = win;
  b->use_graph = keep_graph;
  batch_drop_graph(b);
  if (best) {
    best->refill_min = win.refill_min;
    best->trace_blocks_per_sm = win.trace_blocks_per_sm;
    best->shade_blocks_per_sm = win.shade_blocks_per_sm;
    best->trace_variant = win.trace_variant;
    best->atrous_tile_rows = win.atrous_rows;
    best->tail_wave = win.tail_wave;
  }
  if (best_ms) *best_ms = win_ms;
  for (VrtSession* s : b->sessions)
    if (int r = vrt_session_reset(s)) return r;
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// serving: continuous batching over device-resident sessions
// ---------------------------------------------------------------------------
}  // extern "C"

struct VrtServer {
  struct Req {
    uint64_t ticket = 0;
    int session = 0;
    VrtUniforms u;
    std::vector<VrtEditBox> edits;
    double t_arrival = 0.0;
    void* ldr_out = nullptr;
  };
  struct Flight {
    cudaEvent_t done = nullptr;
    std::vector<Req> reqs;
  };
  // a session waiting for admission: created once the HBM budget has room
  struct Open {
    uint64_t ticket = 0;
    VrtScene* scene = nullptr;
    VrtSessionConfig cfg;
  };
  VrtCtx* ctx = nullptr;
  VrtBatch* batch = nullptr;     // batch->sessions is the slot table (NULL = free slot)
  int n = 0;                     // slots
  int max_in_flight = 2;
  bool sequential = false;       // one request per launch through the session's own frame path
  uint64_t solo_pixels = 0;      // batched mode: sessions this large (with their own path scratch) render alone
  int min_batch = 1;             // batched mode: fewer sessions with pending requests launch one request alone
  std::deque<Req> pending;
  std::deque<Flight> flights;
  std::vector<int> busy;         // requests of the slot in flight
  std::vector<int> queued;       // requests of the slot pending
  std::vector<char> owned;       // session created by the server (destroyed when closed)
  std::vector<char> closing;     // close requested: destroyed once idle
  std::deque<Open> opens;        // admission queue, FIFO
  std::unordered_map<uint64_t, int> open_result;   // ticket -> slot (>= 0) or -error code
  std::vector<cudaEvent_t> spare_events;
  uint64_t next_ticket = 1;
  std::chrono::steady_clock::time_point t0;
  cudaEvent_t ref = nullptr;     // device time origin
  double ref_host = 0.0;         // host time (s) at which `ref` had completed
  uint64_t completed = 0;
  uint64_t launched_frames = 0;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  VrtSession* at(int k) const { return batch->sessions[(size_t)k]; }
};

// Destroys closed sessions that went idle, then admits queued sessions in
// arrival order while the budget has room (the first that does not fit
// waits, so later, smaller ones cannot overtake it).
static int server_admit(VrtServer* sv) {
  for (int k = 0; k < sv->n; k++) {
    if (sv->closing[(size_t)k] && !sv->busy[(size_t)k] && !sv->queued[(size_t)k]) {
      VrtSession* s = sv->at(k);
      if (sv->owned[(size_t)k] && s) vrt_session_destroy(s);
      sv->batch->sessions[(size_t)k] = nullptr;
      sv->closing[(size_t)k] = 0;
      sv->owned[(size_t)k] = 0;
    }
  }
  while (!sv->opens.empty()) {
    VrtServer::Open& o = sv->opens.front();
    int slot = -1;
    for (int k = 0; k < sv->n && slot < 0; k++)
      if (!sv->at(k)) slot = k;
    if (slot < 0) break;                              // every slot in use: wait for a close
    if ((uint64_t)o.cfg.width * (uint64_t)o.cfg.height > sv->batch->P && !sv->sequential) {
      sv->open_result[o.ticket] = -VRT_ERR_INVALID;   // larger than the launch pool: never admissible
      sv->opens.pop_front();
      continue;
    }
    VrtSession* s = nullptr;
    const std::string keep = g_err;
    const int r = vrt_session_create(sv->ctx, o.scene, &o.cfg, &s);
    if (r == VRT_ERR_BUDGET) { g_err = keep; break; }   // wait until memory frees
    if (r) {
      sv->open_result[o.ticket] = -r;
    } else {
      sv->batch->sessions[(size_t)slot] = s;
      sv->owned[(size_t)slot] = 1;
      sv->open_result[o.ticket] = slot;
    }
    sv->opens.pop_front();
  }
  return VRT_OK;
}

static int server_launch(VrtServer* sv) {
  std::vector<VrtServer::Req> take;
  if (sv->sequential) {
    // the plain form: the oldest request alone, through its session's frame path
    if (sv->pending.empty()) return VRT_OK;
    take.push_back(std::move(sv->pending.front()));
    sv->pending.pop_front();
  } else {
    auto solo = [&](const VrtSession* s) {
      return sv->solo_pixels > 0 && s->path_kernel == VRT_PATH_WAVEFRONT && (uint64_t)s->W * s->H >= sv->solo_pixels;
    };
    // the oldest request decides the launch: a large session renders alone
    // through its own frame path; otherwise the oldest request of every small
    // session joins one batch frame.  A session's next frame may be launched
    // while its previous one is in flight: its frames run in stream order on
    // the context's stream (history, edits and read-backs included), so the
    // device always has the next launch queued
    if (!sv->pending.empty() && solo(sv->at(sv->pending.front().session))) {
      take.push_back(std::move(sv->pending.front()));
      sv->pending.pop_front();
    }
  }
  if (!sv->sequential && take.empty() && sv->min_batch > 1) {
    // too few sessions to batch: the oldest request of a session with its
    // own path scratch renders alone
    std::vector<char> seen((size_t)sv->n, 0);
    int distinct = 0;
    for (const auto& r : sv->pending) {
      if (seen[(size_t)r.session]) continue;
      seen[(size_t)r.session] = 1;
      if (++distinct >= sv->min_batch) break;
    }
    if (distinct < sv->min_batch) {
      for (auto it = sv->pending.begin(); it != sv->pending.end(); ++it) {
        if (sv->at(it->session)->path_kernel != VRT_PATH_WAVEFRONT) continue;
        take.push_back(std::move(*it));
        sv->pending.erase(it);
        break;
      }
    }
  }
  const bool alone = sv->sequential || !take.empty();
  if (!alone) {
    // oldest pending request of every session, in arrival order, while their
    // pixels fit the pool
    std::vector<char> picked((size_t)sv->n, 0);
    uint64_t pix = 0;
    for (auto it = sv->pending.begin(); it != sv->pending.end();) {
      const int k = it->session;
      VrtSession* s = sv->at(k);
      const uint64_t p = (uint64_t)s->W * s->H;
      const bool large = sv->solo_pixels > 0 && s->path_kernel == VRT_PATH_WAVEFRONT && p >= sv->solo_pixels;
      if (!large && !picked[(size_t)k] && pix + p <= sv->batch->P) {
        picked[(size_t)k] = 1;
        pix += p;
        take.push_back(std::move(*it));
        it = sv->pending.erase(it);
      } else {
        ++it;
      }
    }
  }
  if (take.empty()) return VRT_OK;
  cudaStream_t st = sv->ctx->stream;
  std::vector<int> idx;
  std::vector<VrtUniforms> us;
  for (auto& r : take) {
    VrtSession* s = sv->at(r.session);
    sv->queued[(size_t)r.session]--;
    for (const VrtEditBox& e : r.edits)
      if (int rc = vrt_scene_edit_box(s->scene, e.x0, e.y0, e.z0, e.x1, e.y1, e.z1, e.value)) return rc;
    idx.push_back(r.session);
    us.push_back(r.u);
  }
  if (alone) {
    if (int rc = vrt_frame(sv->at(idx[0]), &us[0])) return rc;
  } else {
    if (int rc = batch_frame_impl(sv->batch, idx.data(), (int)idx.size(), us.data())) return rc;
  }
  for (auto& r : take) {
    VrtSession* s = sv->at(r.session);
    if (r.ldr_out)
      CUDA_TRY(cudaMemcpyAsync(r.ldr_out, s->ldr, px(s) * 4, cudaMemcpyDeviceToHost, st));
    sv->busy[(size_t)r.session]++;
  }
  VrtServer::Flight f;
  if (!sv->spare_events.empty()) {
    f.done = sv->spare_events.back();
    sv->spare_events.pop_back();
  } else {
    CUDA_TRY(cudaEventCreate(&f.done));
  }
  CUDA_TRY(cudaEventRecord(f.done, st));
  f.reqs = std::move(take);
  sv->flights.push_back(std::move(f));
  sv->launched_frames++;
  return VRT_OK;
}

// Retires finished flights into out[]; returns the number written.
static int server_retire(VrtServer* sv, VrtCompletion* out, int max_out, bool block, int* err) {
  int k = 0;
  *err = VRT_OK;
  while (!sv->flights.empty()) {
    VrtServer::Flight& f = sv->flights.front();
    if ((int)f.reqs.size() > max_out - k) break;
    cudaError_t q = block ? cudaEventSynchronize(f.done) : cudaEventQuery(f.done);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) { *err = fail(VRT_ERR_CUDA, "server: %s", cudaGetErrorString(q)); break; }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, sv->ref, f.done);
    const double t_done = sv->ref_host + ms / 1e3;
    for (auto& r : f.reqs) {
      out[k].ticket = r.ticket;
      out[k].session = r.session;
      out[k].pad = 0;
      out[k].t_arrival = r.t_arrival;
      out[k].t_done = t_done;
      k++;
      sv->busy[(size_t)r.session]--;
      sv->completed++;
    }
    sv->spare_events.push_back(f.done);
    sv->flights.pop_front();
  }
  return k;
}

static int server_new(VrtCtx* ctx, int max_in_flight, VrtServer** out) {
  VrtServer* sv = new VrtServer();
  sv->ctx = ctx;
  sv->max_in_flight = max_in_flight;
  sv->t0 = std::chrono::steady_clock::now();
  *out = sv;
  return VRT_OK;
}

static int server_setup(VrtServer* sv) {
  sv->n = (int)sv->batch->sessions.size();
  sv->busy.assign((size_t)sv->n, 0);
  sv->queued.assign((size_t)sv->n, 0);
  sv->owned.assign((size_t)sv->n, 0);
  sv->closing.assign((size_t)sv->n, 0);
  sv->batch->use_graph = false;
  cudaError_t e = cudaEventCreate(&sv->ref);
  if (e == cudaSuccess) e = cudaEventRecord(sv->ref, sv->ctx->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(sv->ref);
  if (e != cudaSuccess) return fail(VRT_ERR_CUDA, "server setup: %s", cudaGetErrorString(e));
  sv->ref_host = sv->now();
  return VRT_OK;
}

extern "C" {

int vrt_server_create(VrtCtx* ctx, VrtSession* const* sessions, int n, int max_in_flight, VrtServer** out) {
  if (!ctx || !sessions || n < 1 || !out || max_in_flight < 1 || max_in_flight > 8)
    return fail(VRT_ERR_INVALID, "bad argument");
  *out = nullptr;
  VrtServer* sv = nullptr;
  server_new(ctx, max_in_flight, &sv);
  int r = vrt_batch_create(ctx, sessions, n, &sv->batch);
  if (!r) r = server_setup(sv);
  if (r) {
    if (sv->batch) vrt_batch_destroy(sv->batch);
    delete sv;
    return r;
  }
  *out = sv;
  return VRT_OK;
}

int vrt_server_create_dynamic(VrtCtx* ctx, int max_sessions, long long max_pixels, int max_in_flight,
                              VrtServer** out) {
  if (!ctx || !out || max_sessions < 1 || max_sessions > 4096 || max_pixels < 1 || max_in_flight < 1 ||
      max_in_flight > 8)
    return fail(VRT_ERR_INVALID, "bad argument");
  *out = nullptr;
  VrtServer* sv = nullptr;
  server_new(ctx, max_in_flight, &sv);
  int r = batch_create_capacity(ctx, nullptr, max_sessions, (uint64_t)max_pixels, &sv->batch);
  if (!r) r = server_setup(sv);
  if (r) {
    if (sv->batch) vrt_batch_destroy(sv->batch);
    delete sv;
    return r;
  }
  *out = sv;
  return VRT_OK;
}

int vrt_server_destroy(VrtServer* sv) {
  if (!sv) return VRT_OK;
  cudaSetDevice(sv->ctx->device);
  cudaStreamSynchronize(sv->ctx->stream);
  for (auto& f : sv->flights) cudaEventDestroy(f.done);
  for (cudaEvent_t e : sv->spare_events) cudaEventDestroy(e);
  if (sv->ref) cudaEventDestroy(sv->ref);
  for (int k = 0; k < sv->n; k++)
    if (sv->owned[(size_t)k] && sv->at(k)) vrt_session_destroy(sv->at(k));
  vrt_batch_destroy(sv->batch);
  delete sv;
  return VRT_OK;
}

double vrt_server_now(VrtServer* sv) { return sv ? sv->now() : 0.0; }

int vrt_server_set_sequential(VrtServer* sv, int on) {
  if (!sv) return fail(VRT_ERR_INVALID, "server is NULL");
  if (!sv->pending.empty() || !sv->flights.empty()) return fail(VRT_ERR_STATE, "server has requests in progress");
  if (on)
    for (int k = 0; k < sv->n; k++)
      if (sv->at(k) && sv->at(k)->path_kernel == VRT_PATH_BATCH_ONLY)
        return fail(VRT_ERR_STATE, "session %d has no path scratch of its own (VRT_PATH_BATCH_ONLY)", k);
  sv->sequential = on != 0;
  return VRT_OK;
}

int vrt_server_set_solo_pixels(VrtServer* sv, long long pixels) {
  if (!sv || pixels < 0) return fail(VRT_ERR_INVALID, "bad argument");
  sv->solo_pixels = (uint64_t)pixels;
  return VRT_OK;
}

int vrt_server_set_min_batch(VrtServer* sv, int sessions) {
  if (!sv || sessions < 1 || sessions > 4096) return fail(VRT_ERR_INVALID, "bad argument");
  sv->min_batch = sessions;
  return VRT_OK;
}

int vrt_server_open_session(VrtServer* sv, VrtScene* scene, const VrtSessionConfig* cfg, uint64_t* ticket) {
  if (!sv || !scene || !cfg || !ticket) return fail(VRT_ERR_INVALID, "NULL argument");
  if (scene->ctx != sv->ctx) return fail(VRT_ERR_INVALID, "scene belongs to another context");
  if (sv->sequential && cfg->path_kernel == VRT_PATH_BATCH_ONLY)
    return fail(VRT_ERR_INVALID, "a sequential server's sessions need their own path scratch");
  VrtServer::Open o;
  o.ticket = sv->next_ticket++;
  o.scene = scene;
  o.cfg = *cfg;
  sv->opens.push_back(o);
  *ticket = o.ticket;
  if (int r = set_dev(sv->ctx)) return r;
  return server_admit(sv);
}

int vrt_server_session_of(VrtServer* sv, uint64_t ticket, int* slot) {
  if (!sv || !slot) return fail(VRT_ERR_INVALID, "NULL argument");
  auto it = sv->open_result.find(ticket);
  if (it == sv->open_result.end()) {
    for (const auto& o : sv->opens)
      if (o.ticket == ticket) return fail(VRT_ERR_STATE, "session of ticket %llu is waiting for admission",
                                          (unsigned long long)ticket);
    return fail(VRT_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  }
  if (it->second < 0) return fail(-it->second, "opening the session of ticket %llu failed",
                                  (unsigned long long)ticket);
  *slot = it->second;
  return VRT_OK;
}

int vrt_server_close_session(VrtServer* sv, int slot) {
  if (!sv || slot < 0 || slot >= sv->n || !sv->at(slot)) return fail(VRT_ERR_INVALID, "no session in slot %d", slot);
  sv->closing[(size_t)slot] = 1;
  if (int r = set_dev(sv->ctx)) return r;
  return server_admit(sv);
}

int vrt_server_sessions(VrtServer* sv, int* open, int* waiting) {
  if (!sv) return fail(VRT_ERR_INVALID, "server is NULL");
  int k = 0;
  for (int i = 0; i < sv->n; i++) k += sv->at(i) && !sv->closing[(size_t)i] ? 1 : 0;
  if (open) *open = k;
  if (waiting) *waiting = (int)sv->opens.size();
  return VRT_OK;
}

int vrt_server_submit(VrtServer* sv, int session, const VrtUniforms* u, const VrtEditBox* edits, int n_edits,
                      double t_arrival, void* ldr_out, uint64_t* ticket) {
  if (!sv || !u || session < 0 || session >= sv->n || n_edits < 0 || (n_edits && !edits))
    return fail(VRT_ERR_INVALID, "bad argument");
  if (!sv->at(session) || sv->closing[(size_t)session])
    return fail(VRT_ERR_INVALID, "slot %d holds no open session", session);
  if (int r = check_uniforms(sv->at(session), u)) return r;
  if (restir_on(u)) return fail(VRT_ERR_INVALID, "served frames render the plain path (restir flags set)");
  VrtServer::Req r;
  r.ticket = sv->next_ticket++;
  r.session = session;
  r.u = *u;
  r.edits.assign(edits, edits + n_edits);
  r.t_arrival = t_arrival >= 0.0 ? t_arrival : sv->now();
  r.ldr_out = ldr_out;
  sv->pending.push_back(std::move(r));
  sv->queued[(size_t)session]++;
  if (ticket) *ticket = sv->pending.back().ticket;
  return VRT_OK;
}

int vrt_server_poll(VrtServer* sv, VrtCompletion* out, int max_out, int* n_out) {
  if (!sv || (max_out > 0 && !out) || !n_out) return fail(VRT_ERR_INVALID, "bad argument");
  *n_out = 0;
  if (int r = set_dev(sv->ctx)) return r;
  int err = VRT_OK;
  *n_out = server_retire(sv, out, max_out, false, &err);
  if (err) return err;
  if (int r = server_admit(sv)) return r;
  while ((int)sv->flights.size() < sv->max_in_flight && !sv->pending.empty()) {
    const size_t before = sv->flights.size();
    if (int r = server_launch(sv)) return r;
    if (sv->flights.size() == before) break;   // nothing could be launched
  }
  return VRT_OK;
}

int vrt_server_drain(VrtServer* sv, VrtCompletion* out, int max_out, int* n_out) {
  if (!sv || (max_out > 0 && !out) || !n_out) return fail(VRT_ERR_INVALID, "bad argument");
  *n_out = 0;
  if (int r = set_dev(sv->ctx)) return r;
  while (!sv->pending.empty() || !sv->flights.empty()) {
    int k = 0;
    if (int r = vrt_server_poll(sv, out + *n_out, max_out - *n_out, &k)) return r;
    *n_out += k;
    if (sv->flights.empty()) continue;
    if ((int)sv->flights.front().reqs.size() > max_out - *n_out) break;   // caller's buffer is full
    int err = VRT_OK;
    const int got = server_retire(sv, out + *n_out, max_out - *n_out, true, &err);
    if (err) return err;
    *n_out += got;
  }
  return server_admit(sv);
}

int vrt_server_pending(VrtServer* sv, int* queued, int* in_flight) {
  if (!sv) return fail(VRT_ERR_INVALID, "server is NULL");
  if (queued) *queued = (int)sv->pending.size();
  if (in_flight) *in_flight = (int)sv->flights.size();
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// radiance-cache MLP
// ---------------------------------------------------------------------------
}  // extern "C"

struct VrtMlp {
  VrtCtx* ctx = nullptr;
  uint64_t bytes = 0;
  float* wm = nullptr;      // fp32 masters
  float* m = nullptr;       // Adam first moment
  float* v = nullptr;       // Adam second moment
  float* grad = nullptr;
  uint16_t* wb = nullptr;   // bf16 copy read by the kernels
  float* partial = nullptr; // per-CTA gradient partials
  float* loss = nullptr;    // per-CTA loss sums
  int* err = nullptr;        // [0]: a tensor-core wait ran out; [1]: Adam step counter
  int P = 0, ctas = 0;
  int* step() const { return err + 1; }
};

// He-normal initial weights from a PCG-hash stream (Box-Muller).
static void mlp_init_host(std::vector<float>& w, uint32_t seed) {
  const int P = mlp_num_params();
  w.assign((size_t)P, 0.0f);
  auto h = [](uint32_t v) {
    v = v * 747796405u + 2891336453u;
    uint32_t x = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
    return (x >> 22u) ^ x;
  };
  const int kin[4] = {80, 64, 64, 64}, nout[4] = {64, 64, 64, 16};
  int off = 0;
  uint32_t s = h(seed ^ 0x5eed1234u);
  for (int l = 0; l < 4; l++) {
    const double std_ = std::sqrt(2.0 / kin[l]);
    for (int k = 0; k < kin[l]; k++)
      for (int n = 0; n < nout[l]; n++) {
        s = h(s);
        const double u1 = ((double)s + 1.0) / 4294967297.0;
        s = h(s);
        const double u2 = (double)s / 4294967296.0;
        double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2) * std_;
        if (l == 3) z = n < 3 ? z * 0.1 : 0.0;
        w[(size_t)off + (size_t)k * nout[l] + n] = (float)z;
      }
    off += kin[l] * nout[l];
  }
}

extern "C" {

int vrt_mlp_num_params(void) { return mlp_num_params(); }

int vrt_mlp_destroy(VrtMlp* m) {
  if (!m) return VRT_OK;
  VrtCtx* c = m->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  const size_t P = (size_t)m->P;
  dev_free(c, m->wm, P * 4, &m->bytes);
  dev_free(c, m->m, P * 4, &m->bytes);
  dev_free(c, m->v, P * 4, &m->bytes);
  dev_free(c, m->grad, P * 4, &m->bytes);
  dev_free(c, m->wb, P * 2, &m->bytes);
  dev_free(c, m->partial, P * 4 * (size_t)m->ctas, &m->bytes);
  dev_free(c, m->loss, (size_t)m->ctas * 4, &m->bytes);
  dev_free(c, m->err, 16, &m->bytes);
  delete m;
  return VRT_OK;
}

int vrt_mlp_set_params(VrtMlp* m, const float* host) {
  if (!m || !host) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(m->ctx)) return r;
  cudaStream_t st = m->ctx->stream;
  const size_t P = (size_t)m->P;
  CUDA_TRY(cudaMemcpyAsync(m->wm, host, P * 4, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(m->m, 0, P * 4, st));
  CUDA_TRY(cudaMemsetAsync(m->v, 0, P * 4, st));
  CUDA_TRY(mlp_to_bf16(m->wm, m->wb, st));
  CUDA_TRY(cudaMemsetAsync(m->step(), 0, 4, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return VRT_OK;
}

int vrt_mlp_get_params(VrtMlp* m, float* host) {
  if (!m || !host) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(m->ctx)) return r;
  CUDA_TRY(cudaMemcpyAsync(host, m->wm, (size_t)m->P * 4, cudaMemcpyDeviceToHost, m->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  return VRT_OK;
}

int vrt_mlp_create(VrtCtx* ctx, uint32_t seed, VrtMlp** out) {
  if (!ctx || !out) return fail(VRT_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (int r = set_dev(ctx)) return r;
  VrtMlp* m = new VrtMlp();
  m->ctx = ctx;
  m->P = mlp_num_params();
  m->ctas = mlp_max_ctas();
  const size_t P = (size_t)m->P;
  int r = dev_alloc(ctx, (void**)&m->wm, P * 4, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->m, P * 4, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->v, P * 4, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->grad, P * 4, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->wb, P * 2, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->partial, P * 4 * (size_t)m->ctas, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->loss, (size_t)m->ctas * 4, &m->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&m->err, 16, &m->bytes);
  if (!r && cudaMemset(m->err, 0, 16) != cudaSuccess) r = fail(VRT_ERR_CUDA, "memset");
  if (!r) {
    std::vector<float> w;
    mlp_init_host(w, seed);
    r = vrt_mlp_set_params(m, w.data());
  }
  if (r) {
    std::string keep = g_err;
    vrt_mlp_destroy(m);
    g_err = keep;
    return r;
  }
  *out = m;
  return VRT_OK;
}

static int mlp_check_err(VrtMlp* m) {
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, m->err, 4, cudaMemcpyDeviceToHost, m->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  if (h) {
    cudaMemsetAsync(m->err, 0, 4, m->ctx->stream);
    return fail(VRT_ERR_TIMEOUT, "radiance cache: a tensor-core completion wait ran out");
  }
  return VRT_OK;
}

int vrt_mlp_encode_device(VrtMlp* m, const float* d_q9, int n, float extent, uint16_t* d_feat) {
  if (!m || n < 0 || (n && (!d_q9 || !d_feat)) || !(extent > 0.0f)) return fail(VRT_ERR_INVALID, "bad argument");
  if (int r = set_dev(m->ctx)) return r;
  CUDA_TRY(mlp_encode(d_q9, n, extent, d_feat, m->ctx->stream));
  return VRT_OK;
}

int vrt_mlp_infer_device(VrtMlp* m, const float* d_q9, int n, float extent, float* d_out3) {
  if (!m || n < 0 || (n && (!d_q9 || !d_out3)) || !(extent > 0.0f)) return fail(VRT_ERR_INVALID, "bad argument");
  if (int r = set_dev(m->ctx)) return r;
  MlpTaskSet ts;
  std::memset(&ts, 0, sizeof ts);
  ts.n = 1;
  MlpTask& t = ts.t[0];
  t.wb = m->wb; t.q9 = d_q9; t.out3 = d_out3; t.n_max = n; t.extent = extent; t.err = m->err;
  CUDA_TRY(mlp_infer_tasks(ts, m->ctx->stream));
  return VRT_OK;
}

// advance: the reduction advances the Adam step counter (a training step follows).
static int mlp_grad_impl(VrtMlp* m, const float* d_q9, const float* d_y3, int n, float extent, float* loss_out,
                         bool advance) {
  int ctas = 0;
  MlpTaskSet ts;
  std::memset(&ts, 0, sizeof ts);
  ts.n = 1;
  MlpTask& t = ts.t[0];
  t.wb = m->wb; t.q9 = d_q9; t.y3 = d_y3; t.n_max = n; t.extent = extent; t.err = m->err;
  t.step = advance ? m->step() : nullptr;
  t.partial = m->partial; t.loss = m->loss; t.grad = m->grad;
  CUDA_TRY(mlp_gradient_tasks(ts, m->ctx->stream));
  ctas = ts.t[0].ctas;
  if (loss_out) {
    std::vector<float> l((size_t)ctas);
    CUDA_TRY(cudaMemcpyAsync(l.data(), m->loss, (size_t)ctas * 4, cudaMemcpyDeviceToHost, m->ctx->stream));
    if (int r = mlp_check_err(m)) return r;
    double s = 0.0;
    for (float x : l) s += x;
    *loss_out = (float)(s / (double)n);
  }
  return VRT_OK;
}

int vrt_mlp_gradient_device(VrtMlp* m, const float* d_q9, const float* d_y3, int n, float extent, float* d_grad,
                            float* loss_out) {
  if (!m || n < 1 || !d_q9 || !d_y3 || !(extent > 0.0f)) return fail(VRT_ERR_INVALID, "bad argument");
  if (int r = set_dev(m->ctx)) return r;
  if (int r = mlp_grad_impl(m, d_q9, d_y3, n, extent, loss_out, false)) return r;
  if (d_grad)
    CUDA_TRY(cudaMemcpyAsync(d_grad, m->grad, (size_t)m->P * 4, cudaMemcpyDeviceToDevice, m->ctx->stream));
  return mlp_check_err(m);
}

int vrt_mlp_train_device(VrtMlp* m, const float* d_q9, const float* d_y3, int n, float extent, float lr, int steps,
                         float* loss_out) {
  if (!m || n < 1 || !d_q9 || !d_y3 || !(extent > 0.0f) || steps < 1 || !(lr > 0.0f))
    return fail(VRT_ERR_INVALID, "bad argument");
  if (int r = set_dev(m->ctx)) return r;
  for (int i = 0; i < steps; i++) {
    if (int r = mlp_grad_impl(m, d_q9, d_y3, n, extent, (loss_out && i == 0) ? loss_out : nullptr, true)) return r;
    MlpTaskSet ts;
    std::memset(&ts, 0, sizeof ts);
    ts.n = 1;
    MlpTask& t = ts.t[0];
    t.step = m->step(); t.grad = m->grad; t.wm = m->wm; t.m = m->m; t.v = m->v; t.wbw = m->wb; t.lr = lr;
    CUDA_TRY(mlp_adam_tasks(ts, m->ctx->stream));
  }
  return VRT_OK;
}

int vrt_mlp_check(VrtMlp* m) {
  if (!m) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(m->ctx)) return r;
  return mlp_check_err(m);
}

// ---------------------------------------------------------------------------
// cache-assisted sessions
// ---------------------------------------------------------------------------
int vrt_session_cache_mlp(VrtSession* s, VrtMlp** out) {
  if (!s || !out) return fail(VRT_ERR_INVALID, "NULL argument");
  *out = s->mlp;
  return VRT_OK;
}

int vrt_session_set_cache(VrtSession* s, const VrtCacheConfig* cfg_in) {
  if (!s || !cfg_in) return fail(VRT_ERR_INVALID, "NULL argument");
  VrtCacheConfig cfg = *cfg_in;
  s->cache_version++;
  if (!cfg.enabled) {
    s->cache_on = false;
    return VRT_OK;
  }
  if (s->path_kernel == VRT_PATH_MEGAKERNEL) return fail(VRT_ERR_STATE, "the cache needs the wavefront path kernel");
  if (cfg.train_bounces == 0) cfg.train_bounces = 6;
  if (cfg.train_vertices == 0) cfg.train_vertices = 3;
  if (cfg.train_batch == 0) cfg.train_batch = 65536;
  if (cfg.train_steps == 0) cfg.train_steps = 1;
  if (cfg.learning_rate == 0.0f) cfg.learning_rate = 1e-2f;
  if (cfg.train_bounces < 1 || cfg.train_bounces + 3 > kMaxWaves || cfg.train_vertices < 1 ||
      cfg.train_vertices > kCacheMaxRec || cfg.train_batch < 1 || cfg.train_batch > (1 << 22) ||
      cfg.train_steps < 0 || cfg.train_steps > 64 || !(cfg.learning_rate > 0.0f))
    return fail(VRT_ERR_INVALID, "cache configuration out of range");
  if (int r = set_dev(s->ctx)) return r;
  VrtCtx* c = s->ctx;
  const size_t P = px(s);
  const int TW = (s->W + 3) / 4, TH = (s->H + 3) / 4;
  const size_t T = (size_t)TW * TH;
  const size_t cap = T * (size_t)cfg.train_vertices;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t b_rec = al(T * kCacheMaxRec * 64), b_recn = al(T * 4), b_q = al(P * 36), b_qpix = al(P * 4),
               b_ctr = 256, b_cq = al(cap * 36), b_cy = al(cap * 12), b_pred = al(P * 12);
  const size_t need = b_rec + b_recn + b_q + b_qpix + b_ctr + b_cq + b_cy + b_pred;
  if (need != s->cache_bytes) {
    cudaStreamSynchronize(c->stream);
    dev_free(c, s->cache_mem, s->cache_bytes, &s->bytes);
    s->cache_bytes = 0;
    if (int r = dev_alloc(c, &s->cache_mem, need, &s->bytes)) return r;
    s->cache_bytes = need;
  }
  char* m = (char*)s->cache_mem;
  CacheDev& d = s->cache;
  std::memset(&d, 0, sizeof d);
  d.rec = (float4*)m; m += b_rec;
  d.rec_n = (int*)m; m += b_recn;
  d.qbuf = (float*)m; m += b_q;
  d.qpix = (uint32_t*)m; m += b_qpix;
  d.qcount = (int*)m;
  d.cand_count = (int*)m + 1;
  m += b_ctr;
  d.cand_q9 = (float*)m; m += b_cq;
  d.cand_y3 = (float*)m; m += b_cy;
  s->pred = (float*)m;
  d.cand_cap = (int)cap;
  d.TW = TW;
  d.train_bounces = (uint32_t)cfg.train_bounces;
  d.rec_vertices = cfg.train_vertices;
  d.tclamp = s->fclamp;
  if (!s->mlp) {
    if (int r = vrt_mlp_create(c, cfg.seed, &s->mlp)) return r;
  }
  if (!s->cev[0]) {
    for (auto& e : s->cev)
      if (cudaEventCreate(&e) != cudaSuccess) return fail(VRT_ERR_CUDA, "cudaEventCreate failed");
  }
  s->cache_cfg = cfg;
  s->cache_on = true;
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// Session checkpoint: everything the next frames depend on -- the scene's
// voxels (bricks, masks and the occupancy bitmap are rebuilt from them), both
// history / G-buffer parities and the frame parity, the radiance cache's
// network (fp32 masters, Adam moments, step), the ReSTIR history (reservoirs
// and duplication map) and the HDR reference accumulation.  A session
// restored into a fresh session of the same size renders the same frames
// bit for bit.  The layout is a header followed by the sections in order.
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {
struct CkptHeader {
  char magic[8];              // "VRTCKPT1"
  uint32_t version, flags;    // flags: 1 cache network, 2 ReSTIR history, 4 HDR accumulation
  int32_t W, H, N, acc_f32;
  uint64_t frame_counter;
  int32_t last_parity, have_frame, last_denoise, hdr_count;
  VrtCacheConfig cache_cfg;
  uint64_t restir_bytes, total_bytes;
};
constexpr uint32_t kCkptCache = 1u, kCkptRestir = 2u, kCkptHdr = 4u;

uint64_t ckpt_size(const VrtSession* s, uint32_t flags) {
  const uint64_t P = px(s), N = (uint64_t)s->scene->dev.N;
  uint64_t b = sizeof(CkptHeader) + N * N * N * 4 + 2 * P * acc_bpp(s) + 2 * P * 16;
  if (flags & kCkptCache) b += 3ull * (uint64_t)s->mlp->P * 4 + 4;
  if (flags & kCkptRestir) b += s->restir_bytes;
  if (flags & kCkptHdr) b += P * 3 * 8;
  return b;
}

uint32_t ckpt_flags(const VrtSession* s) {
  return (s->mlp ? kCkptCache : 0u) | (s->restir_mem ? kCkptRestir : 0u) | (s->hdr_acc ? kCkptHdr : 0u);
}
}  // namespace

extern "C" {

int vrt_session_checkpoint_size(VrtSession* s, uint64_t* bytes) {
  if (!s || !bytes) return fail(VRT_ERR_INVALID, "NULL argument");
  *bytes = ckpt_size(s, ckpt_flags(s));
  return VRT_OK;
}

int vrt_session_checkpoint(VrtSession* s, void* host, uint64_t bytes) {
  if (!s || !host) return fail(VRT_ERR_INVALID, "NULL argument");
  const uint32_t flags = ckpt_flags(s);
  const uint64_t need = ckpt_size(s, flags);
  if (bytes < need) return fail(VRT_ERR_INVALID, "checkpoint buffer %llu bytes < %llu needed",
                                (unsigned long long)bytes, (unsigned long long)need);
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  CkptHeader h;
  std::memset(&h, 0, sizeof h);
  std::memcpy(h.magic, "VRTCKPT1", 8);
  h.version = 1;
  h.flags = flags;
  h.W = s->W; h.H = s->H; h.N = s->scene->dev.N; h.acc_f32 = s->acc_f32 ? 1 : 0;
  h.frame_counter = s->frame_counter;
  h.last_parity = s->last_parity; h.have_frame = s->have_frame ? 1 : 0; h.last_denoise = s->last_denoise ? 1 : 0;
  h.hdr_count = (int32_t)s->hdr_count;
  h.cache_cfg = s->cache_cfg;
  h.cache_cfg.enabled = s->cache_on ? 1 : 0;
  h.restir_bytes = (flags & kCkptRestir) ? s->restir_bytes : 0;
  h.total_bytes = need;
  char* o = (char*)host;
  std::memcpy(o, &h, sizeof h);
  o += sizeof h;
  const uint64_t P = px(s), N = (uint64_t)h.N;
  auto d2h = [&](const void* src, uint64_t n) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(o, src, n, cudaMemcpyDeviceToHost, st);
    o += n;
    return e;
  };
  CUDA_TRY(d2h(s->scene->dev.vox, N * N * N * 4));
  for (int i = 0; i < 2; i++) CUDA_TRY(d2h(s->accum[i], P * acc_bpp(s)));
  for (int i = 0; i < 2; i++) CUDA_TRY(d2h(s->gbuf[i], P * 16));
  if (flags & kCkptCache) {
    const uint64_t np = (uint64_t)s->mlp->P * 4;
    CUDA_TRY(d2h(s->mlp->wm, np));
    CUDA_TRY(d2h(s->mlp->m, np));
    CUDA_TRY(d2h(s->mlp->v, np));
    CUDA_TRY(d2h(s->mlp->step(), 4));
  }
  if (flags & kCkptRestir) CUDA_TRY(d2h(s->restir_mem, s->restir_bytes));
  if (flags & kCkptHdr) CUDA_TRY(d2h(s->hdr_acc, P * 3 * 8));
  CUDA_TRY(cudaStreamSynchronize(st));
  return VRT_OK;
}

int vrt_session_restore(VrtSession* s, const void* host, uint64_t bytes) {
  if (!s || !host) return fail(VRT_ERR_INVALID, "NULL argument");
  if (bytes < sizeof(CkptHeader)) return fail(VRT_ERR_INVALID, "checkpoint shorter than its header");
  CkptHeader h;
  std::memcpy(&h, host, sizeof h);
  if (std::memcmp(h.magic, "VRTCKPT1", 8) != 0 || h.version != 1)
    return fail(VRT_ERR_INVALID, "not a session checkpoint (bad magic or version)");
  if (h.W != s->W || h.H != s->H || h.N != s->scene->dev.N || h.acc_f32 != (s->acc_f32 ? 1 : 0))
    return fail(VRT_ERR_INVALID, "checkpoint of a %dx%d session on a %d^3 scene (history %s) does not fit this "
                "session", h.W, h.H, h.N, h.acc_f32 ? "rgba32f" : "rgba16f");
  if (h.total_bytes != bytes) return fail(VRT_ERR_INVALID, "checkpoint size %llu != its header's %llu",
                                         (unsigned long long)bytes, (unsigned long long)h.total_bytes);
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  // state the sections need on this side before anything is copied
  if ((h.flags & kCkptCache) && !s->mlp) {
    VrtCacheConfig cfg = h.cache_cfg;
    cfg.enabled = 1;
    if (int r = vrt_session_set_cache(s, &cfg)) return r;
  }
  if ((h.flags & kCkptRestir) && (!s->restir_mem || s->restir_bytes != h.restir_bytes))
    return fail(VRT_ERR_STATE, "restore the ReSTIR history into a session that rendered a ReSTIR frame");
  if ((h.flags & kCkptHdr) && !s->hdr_acc) {
    if (int r = vrt_hdr_accum_reset(s)) return r;
  }
  if (ckpt_size(s, h.flags) != bytes) return fail(VRT_ERR_INVALID, "checkpoint sections do not match this session");
  const char* o = (const char*)host + sizeof h;
  const uint64_t P = px(s), N = (uint64_t)h.N;
  auto h2d = [&](void* dst, uint64_t n) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(dst, o, n, cudaMemcpyHostToDevice, st);
    o += n;
    return e;
  };
  CUDA_TRY(h2d(s->scene->dev.vox, N * N * N * 4));
  const int BG = s->scene->dev.BG;
  CUDA_TRY(launch_build_bricks(s->scene->dev, 0, 0, 0, BG - 1, BG - 1, BG - 1, st));
  CUDA_TRY(launch_build_bits(s->scene->dev, st));
  s->scene->lights_built = false;
  for (int i = 0; i < 2; i++) CUDA_TRY(h2d(s->accum[i], P * acc_bpp(s)));
  for (int i = 0; i < 2; i++) CUDA_TRY(h2d(s->gbuf[i], P * 16));
  if (h.flags & kCkptCache) {
    VrtMlp* m = s->mlp;
    const uint64_t np = (uint64_t)m->P * 4;
    CUDA_TRY(h2d(m->wm, np));
    CUDA_TRY(h2d(m->m, np));
    CUDA_TRY(h2d(m->v, np));
    CUDA_TRY(h2d(m->step(), 4));
    CUDA_TRY(mlp_to_bf16(m->wm, m->wb, st));
    s->cache_cfg = h.cache_cfg;
    s->cache_cfg.enabled = 1;
    s->cache_on = h.cache_cfg.enabled != 0;
    s->cache_version++;
  }
  if (h.flags & kCkptRestir) CUDA_TRY(h2d(s->restir_mem, s->restir_bytes));
  if (h.flags & kCkptHdr) CUDA_TRY(h2d(s->hdr_acc, P * 3 * 8));
  CUDA_TRY(cudaStreamSynchronize(st));
  s->frame_counter = h.frame_counter;
  s->last_parity = h.last_parity;
  s->have_frame = h.have_frame != 0;
  s->last_denoise = h.last_denoise != 0;
  s->hdr_count = (uint32_t)h.hdr_count;
  return VRT_OK;
}

int vrt_session_read_cache_samples(VrtSession* s, float* q9, float* y3, int cap, int* count) {
  if (!s || !count || cap < 0 || (cap > 0 && (!q9 || !y3))) return fail(VRT_ERR_INVALID, "bad argument");
  if (!s->cache_mem) return fail(VRT_ERR_STATE, "the cache was never enabled on this session");
  if (int r = set_dev(s->ctx)) return r;
  cudaStream_t st = s->ctx->stream;
  int n = 0;
  CUDA_TRY(cudaMemcpyAsync(&n, s->cache.cand_count, 4, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  *count = n;
  const int k = std::min(std::min(n, s->cache.cand_cap), cap);
  if (k > 0) {
    CUDA_TRY(cudaMemcpyAsync(q9, s->cache.cand_q9, (size_t)k * 36, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(y3, s->cache.cand_y3, (size_t)k * 12, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
  }
  return VRT_OK;
}

// The post-wave work description of a cache session for frame `frame`.
static CacheLaunch cache_launch_of(VrtSession* s, uint32_t frame) {
  VrtMlp* m = s->mlp;
  CacheLaunch cl;
  cl.cd = s->cache;
  cl.cd.on = 1;
  cl.cd.phase = (frame * 7u) & 15u;   // 7 is odd: all 16 positions within 16 frames
  cl.wb = m->wb; cl.wm = m->wm; cl.m = m->m; cl.v = m->v; cl.grad = m->grad;
  cl.partial = m->partial; cl.loss = m->loss; cl.err = m->err; cl.step = m->step();
  cl.pred = s->pred;
  cl.P = s->W * s->H;
  cl.extent = (float)s->scene->dev.N * 0.0625f;
  cl.train_batch = s->cache_cfg.train_batch;
  cl.train_steps = s->cache_cfg.train_steps;
  cl.lr = s->cache_cfg.learning_rate;
  return cl;
}

// One cache-assisted path-trace pass: waves (training + query paths),
// inference over the queries, resolve, then the frame's training steps.
static int cache_frame(VrtSession* s, const VrtUniforms* u, const PathOut& o) {
  const CacheLaunch cl = cache_launch_of(s, u->params0[0]);
  s->cache_timed = s->timing;
  CUDA_TRY(launch_wavefront(s->scene->dev, *u, s->fclamp, s->W, s->H, o, s->wf, s->tune, s->ctx->stream,
                            &s->launches, s->timing ? s->tev : nullptr, VrtSession::kTimedWaves, &s->timed_waves,
                            &cl, s->timing ? s->cev : nullptr));
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// scene lights (scene.js:58-200, 435-461)
// ---------------------------------------------------------------------------
}  // extern "C"

// Power alias table of the light weights (makeAliasTable, scene.js:67-104):
// doubles throughout, float32 where the reference stores into a Float32Array.
static void alias_table(const std::vector<double>& wts, std::vector<float>& table) {
  const size_t n = wts.size();
  if (n == 0) { table = {1.0f, 0.0f, 1.0f, 0.0f}; return; }
  double total = 0.0;
  for (double w : wts) total += std::max(0.0, w);
  std::vector<double> prob(n), scaled(n);
  for (size_t i = 0; i < n; i++) {
    prob[i] = total > 0.0 ? std::max(0.0, wts[i]) / total : 1.0 / (double)n;
    scaled[i] = prob[i] * (double)n;
  }
  std::vector<uint32_t> alias(n, 0u);
  std::vector<float> q(n, 0.0f);
  std::vector<size_t> small, large;
  for (size_t i = 0; i < n; i++) (scaled[i] < 1.0 ? small : large).push_back(i);
  while (!small.empty() && !large.empty()) {
    const size_t a = small.back(), b = large.back();
    small.pop_back();
    large.pop_back();
    q[a] = (float)scaled[a];
    alias[a] = (uint32_t)b;
    scaled[b] = (scaled[b] + scaled[a]) - 1.0;
    (scaled[b] < 1.0 ? small : large).push_back(b);
  }
  for (size_t i : large) { q[i] = 1.0f; alias[i] = (uint32_t)i; }
  for (size_t i : small) { q[i] = 1.0f; alias[i] = (uint32_t)i; }
  table.assign(n * 4, 0.0f);
  for (size_t i = 0; i < n; i++) {
    table[4 * i] = q[i];
    table[4 * i + 1] = (float)alias[i];
    table[4 * i + 2] = (float)(prob[i] > 0.0 ? prob[i] : 1.0 / (double)n);
  }
}

extern "C" {

int vrt_scene_build_lights(VrtScene* sc, VrtLightStats* st) {
  if (!sc) return fail(VRT_ERR_INVALID, "scene is NULL");
  const int N = sc->dev.N, BG = sc->dev.BG;
  if (N > 512) return fail(VRT_ERR_INVALID, "the light word packing holds grids up to 512^3 (scene.js:437)");
  if (int r = set_dev(sc->ctx)) return r;
  VrtCtx* c = sc->ctx;
  cudaStream_t s = c->stream;
  const size_t nb = (size_t)light_blocks(N), cells = (size_t)BG * BG * BG;
  cudaEvent_t ev[4];
  for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
  struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int i = 0; i < 4; i++) cudaEventDestroy(e[i]); } } guard{ev};
  if (!sc->light_tmp)
    if (int r = dev_alloc(c, (void**)&sc->light_tmp, (nb + 1) * 4, &sc->bytes)) return r;
  if (!sc->light_grid)
    if (int r = dev_alloc(c, (void**)&sc->light_grid, cells * 34 * 4, &sc->bytes)) return r;
  CUDA_TRY(cudaEventRecord(ev[0], s));
  CUDA_TRY(launch_light_count(sc->dev.vox, N, sc->light_tmp, sc->light_tmp + nb, s));
  uint32_t n = 0;
  CUDA_TRY(cudaMemcpyAsync(&n, sc->light_tmp + nb, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (n > sc->light_cap) {
    const size_t cap = sc->light_cap;
    dev_free(c, sc->light_words, cap * 8, &sc->bytes);
    dev_free(c, sc->light_w, cap * 8, &sc->bytes);
    sc->light_words = nullptr; sc->light_w = nullptr;
    sc->light_cap = 0;
    const size_t ncap = std::max<size_t>(n, 1);
    int r = dev_alloc(c, (void**)&sc->light_words, ncap * 8, &sc->bytes);
    if (!r) r = dev_alloc(c, (void**)&sc->light_w, ncap * 8, &sc->bytes);
    if (r) return r;
    sc->light_cap = ncap;
  }
  if (n > 0) CUDA_TRY(launch_light_write(sc->dev.vox, N, sc->light_tmp, sc->light_words, sc->light_w, s));
  CUDA_TRY(cudaEventRecord(ev[1], s));
  // alias table on the host (a sequential O(n) pass), then uploaded
  std::vector<double> w(n);
  if (n > 0) CUDA_TRY(cudaMemcpyAsync(w.data(), sc->light_w, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<float> table;
  alias_table(w, table);
  const double alias_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (sc->light_alias_bytes < table.size() * 4) {
    dev_free(c, sc->light_alias, sc->light_alias_bytes, &sc->bytes);
    sc->light_alias = nullptr;
    sc->light_alias_bytes = 0;
    if (int r = dev_alloc(c, (void**)&sc->light_alias, table.size() * 4, &sc->bytes)) return r;
    sc->light_alias_bytes = table.size() * 4;
  }
  CUDA_TRY(cudaMemcpyAsync(sc->light_alias, table.data(), table.size() * 4, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaEventRecord(ev[2], s));
  CUDA_TRY(launch_light_grid(N, sc->light_words, sc->light_w, (int)n, sc->light_grid, s));
  CUDA_TRY(cudaEventRecord(ev[3], s));
  CUDA_TRY(cudaStreamSynchronize(s));
  sc->light_count = n;
  sc->lights_built = true;
  if (st) {
    std::memset(st, 0, sizeof *st);
    st->count = n;
    double tot = 0.0;
    for (double x : w) tot += std::max(0.0, x);
    st->total_weight = tot;
    float a = 0, g = 0;
    CUDA_TRY(cudaEventElapsedTime(&a, ev[0], ev[1]));
    CUDA_TRY(cudaEventElapsedTime(&g, ev[2], ev[3]));
    st->ms_list = a;
    st->ms_alias = (float)alias_ms;
    st->ms_grid = g;
  }
  return VRT_OK;
}

int vrt_scene_read_lights(VrtScene* sc, uint32_t* words, size_t words_bytes, float* alias, size_t alias_bytes,
                          uint32_t* grid, size_t grid_bytes) {
  if (!sc) return fail(VRT_ERR_INVALID, "scene is NULL");
  if (!sc->lights_built) return fail(VRT_ERR_STATE, "lights not built (vrt_scene_build_lights)");
  if (int r = set_dev(sc->ctx)) return r;
  cudaStream_t s = sc->ctx->stream;
  const size_t n = sc->light_count, cells = (size_t)sc->dev.BG * sc->dev.BG * sc->dev.BG;
  const size_t alias_need = std::max<size_t>(n, 1) * 16;
  if (words) {
    if (words_bytes < n * 8) return fail(VRT_ERR_INVALID, "words buffer too small");
    if (n) CUDA_TRY(cudaMemcpyAsync(words, sc->light_words, n * 8, cudaMemcpyDeviceToHost, s));
  }
  if (alias) {
    if (alias_bytes < alias_need) return fail(VRT_ERR_INVALID, "alias buffer too small");
    CUDA_TRY(cudaMemcpyAsync(alias, sc->light_alias, alias_need, cudaMemcpyDeviceToHost, s));
  }
  if (grid) {
    if (grid_bytes < cells * 136) return fail(VRT_ERR_INVALID, "grid buffer too small");
    CUDA_TRY(cudaMemcpyAsync(grid, sc->light_grid, cells * 136, cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  return VRT_OK;
}

// ---------------------------------------------------------------------------
// HDR reference pipeline
// ---------------------------------------------------------------------------
static int hdr_alloc(VrtSession* s) {
  const size_t P = px(s);
  if (!s->hdr_acc) {
    if (int r = dev_alloc(s->ctx, (void**)&s->hdr_acc, P * 24, &s->bytes)) return r;
    CUDA_TRY(cudaMemsetAsync(s->hdr_acc, 0, P * 24, s->ctx->stream));
    s->hdr_count = 0;
  }
  if (!s->hdr_part) {
    if (int r = dev_alloc(s->ctx, (void**)&s->hdr_part, (size_t)hdr_blocks((int)P) * 8, &s->bytes)) return r;
  }
  return VRT_OK;
}

int vrt_hdr_accum_reset(VrtSession* s) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = set_dev(s->ctx)) return r;
  if (int r = hdr_alloc(s)) return r;
  CUDA_TRY(cudaMemsetAsync(s->hdr_acc, 0, px(s) * 24, s->ctx->stream));
  s->hdr_count = 0;
  return VRT_OK;
}

int vrt_hdr_accum_add(VrtSession* s) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (!s->rad32) return fail(VRT_ERR_STATE, "the session keeps no fp32 radiance (keep_radiance_f32)");
  if (int r = set_dev(s->ctx)) return r;
  if (int r = hdr_alloc(s)) return r;
  CUDA_TRY(launch_hdr_add((int)px(s), s->rad32, s->alb8, s->hdr_acc, s->ctx->stream));
  s->hdr_count++;
  return VRT_OK;
}

int vrt_hdr_accumulate(VrtSession* s, const VrtUniforms* u, uint32_t frame0, int spp) {
  if (!s || !u || spp < 1) return fail(VRT_ERR_INVALID, "bad argument");
  // independent path-trace passes: the reference convention (preset=base);
  // a reservoir chain is accumulated frame by frame with vrt_hdr_accum_add
  if (restir_on(u)) return fail(VRT_ERR_INVALID, "reference accumulation renders the plain path (restir flags set)");
  VrtUniforms v = *u;
  for (int k = 0; k < spp; k++) {
    v.params0[0] = frame0 + (uint32_t)k;
    if (int r = vrt_pass_pathtrace(s, &v)) return r;
    if (int r = vrt_hdr_accum_add(s)) return r;
  }
  return VRT_OK;
}

int vrt_hdr_accum_read(VrtSession* s, double* rgb, size_t bytes, uint32_t* count) {
  if (!s || !rgb) return fail(VRT_ERR_INVALID, "NULL argument");
  if (!s->hdr_acc) return fail(VRT_ERR_STATE, "nothing accumulated");
  const size_t P = px(s);
  if (bytes < P * 24) return fail(VRT_ERR_INVALID, "host buffer %zu bytes < %zu needed", bytes, P * 24);
  if (int r = set_dev(s->ctx)) return r;
  CUDA_TRY(cudaMemcpyAsync(rgb, s->hdr_acc, P * 24, cudaMemcpyDeviceToHost, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  if (count) *count = s->hdr_count;
  return VRT_OK;
}

int vrt_hdr_set_reference(VrtSession* s, const float* rgb, size_t bytes) {
  if (!s || !rgb) return fail(VRT_ERR_INVALID, "NULL argument");
  const size_t P = px(s);
  if (bytes < P * 12) return fail(VRT_ERR_INVALID, "reference %zu bytes < %zu needed", bytes, P * 12);
  if (int r = set_dev(s->ctx)) return r;
  if (!s->hdr_ref)
    if (int r = dev_alloc(s->ctx, (void**)&s->hdr_ref, P * 12, &s->bytes)) return r;
  if (int r = hdr_alloc(s)) return r;
  CUDA_TRY(cudaMemcpyAsync(s->hdr_ref, rgb, P * 12, cudaMemcpyHostToDevice, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  return VRT_OK;
}

static int hdr_error(VrtSession* s, int mode, double* sum_sq) {
  if (!s || !sum_sq) return fail(VRT_ERR_INVALID, "NULL argument");
  if (!s->hdr_ref) return fail(VRT_ERR_STATE, "no reference image (vrt_hdr_set_reference)");
  if (mode == 0 && !s->rad32) return fail(VRT_ERR_STATE, "the session keeps no fp32 radiance (keep_radiance_f32)");
  if (mode == 1 && s->hdr_count == 0) return fail(VRT_ERR_STATE, "nothing accumulated");
  if (int r = set_dev(s->ctx)) return r;
  const int P = (int)px(s), nb = hdr_blocks(P);
  CUDA_TRY(launch_hdr_sq_err(P, mode, s->rad32, s->alb8, s->hdr_acc, mode == 1 ? 1.0 / (double)s->hdr_count : 0.0,
                             s->hdr_ref, s->hdr_part, s->ctx->stream));
  std::vector<double> part((size_t)nb);
  CUDA_TRY(cudaMemcpyAsync(part.data(), s->hdr_part, (size_t)nb * 8, cudaMemcpyDeviceToHost, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  double acc = 0.0;
  for (double x : part) acc += x;     // fixed order
  *sum_sq = acc;
  return VRT_OK;
}

int vrt_hdr_frame_error(VrtSession* s, double* sum_sq) { return hdr_error(s, 0, sum_sq); }
int vrt_hdr_accum_error(VrtSession* s, double* sum_sq) { return hdr_error(s, 1, sum_sq); }

int vrt_write_history(VrtSession* s, const void* accum_prev, const float* gbuf_prev) {
  if (!s) return fail(VRT_ERR_INVALID, "session is NULL");
  if (int r = set_dev(s->ctx)) return r;
  const int prev = 1 - parity_of(s);
  cudaStream_t st = s->ctx->stream;
  if (accum_prev) CUDA_TRY(cudaMemcpyAsync(s->accum[prev], accum_prev, px(s) * acc_bpp(s), cudaMemcpyHostToDevice, st));
  if (gbuf_prev) CUDA_TRY(cudaMemcpyAsync(s->gbuf[prev], gbuf_prev, px(s) * 16, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return VRT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// VoxelBench technique adapter (VoxelBench/pipeline/technique.h:8-14): the
// harness's grid, palette, emitters and sky on the device, its G-buffer per
// frame, and its baseline estimator (techniques/pt.h) on this library's DDA.
// ---------------------------------------------------------------------------
struct VrtVb {
  VrtCtx* ctx = nullptr;
  int W = 0, H = 0;
  VrtScene* scene = nullptr;     // the harness's grid embedded in an N^3 packed grid
  int nx = 0, ny = 0, nz = 0;
  uint64_t bytes = 0;
  void* px = nullptr;            // 48 B per pixel (VrtVbPixel)
  void* hist = nullptr;          // float4 per pixel
  void* out = nullptr;           // float4 per pixel
  int* emitters = nullptr;       // int4 per emissive face
  size_t em_cap = 0;
  int n_em = 0;
  unsigned long long* rays = nullptr;
  float albedo[16][3] = {}, emission[16][3] = {};
  int sky = 0;
  float sun_dir[3] = {}, sun_e[3] = {}, zenith[3] = {}, horizon[3] = {};
  uint32_t fcount = 0;
  bool have_world = false, have_gbuf = false;
};

static_assert(sizeof(VrtVbPixel) == 48, "VrtVbPixel is 3 float4");

extern "C" {

int vrt_vb_create(VrtCtx* ctx, int width, int height, VrtVb** out) {
  if (!ctx || !out || width < 1 || height < 1 || (long long)width * height > (1ll << 26))
    return fail(VRT_ERR_INVALID, "bad argument");
  *out = nullptr;
  if (int r = set_dev(ctx)) return r;
  VrtVb* v = new VrtVb();
  v->ctx = ctx;
  v->W = width;
  v->H = height;
  const size_t P = (size_t)width * height;
  int r = dev_alloc(ctx, &v->px, P * 48, &v->bytes);
  if (!r) r = dev_alloc(ctx, &v->hist, P * 16, &v->bytes);
  if (!r) r = dev_alloc(ctx, &v->out, P * 16, &v->bytes);
  if (!r) r = dev_alloc(ctx, (void**)&v->rays, 8, &v->bytes);
  if (!r) r = vrt_vb_reset(v);
  if (r) {
    std::string keep = g_err;
    vrt_vb_destroy(v);
    g_err = keep;
    return r;
  }
  *out = v;
  return VRT_OK;
}

int vrt_vb_destroy(VrtVb* v) {
  if (!v) return VRT_OK;
  VrtCtx* c = v->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  const size_t P = (size_t)v->W * v->H;
  dev_free(c, v->px, P * 48, &v->bytes);
  dev_free(c, v->hist, P * 16, &v->bytes);
  dev_free(c, v->out, P * 16, &v->bytes);
  dev_free(c, v->rays, 8, &v->bytes);
  dev_free(c, v->emitters, v->em_cap * 16, &v->bytes);
  if (v->scene) vrt_scene_destroy(v->scene);
  delete v;
  return VRT_OK;
}

int vrt_vb_reset(VrtVb* v) {
  if (!v) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(v->ctx)) return r;
  CUDA_TRY(cudaMemsetAsync(v->hist, 0, (size_t)v->W * v->H * 16, v->ctx->stream));
  CUDA_TRY(cudaMemsetAsync(v->out, 0, (size_t)v->W * v->H * 16, v->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(v->ctx->stream));
  v->fcount = 0;
  return VRT_OK;
}

int vrt_vb_set_world(VrtVb* v, const VrtVbWorld* w) {
  if (!v || !w || !w->grid || w->nx < 1 || w->ny < 1 || w->nz < 1 || w->n_emitters < 0 ||
      (w->n_emitters > 0 && !w->emitters))
    return fail(VRT_ERR_INVALID, "bad world");
  const int N = ((std::max(w->nx, std::max(w->ny, w->nz)) + 7) / 8) * 8;
  if (N > 1024) return fail(VRT_ERR_INVALID, "grid %dx%dx%d larger than 1024", w->nx, w->ny, w->nz);
  for (size_t i = 0; i < (size_t)w->nx * w->ny * w->nz; i++)
    if (w->grid[i] >= 16) return fail(VRT_ERR_INVALID, "material id %u >= 16", (unsigned)w->grid[i]);
  if (int r = set_dev(v->ctx)) return r;
  // the harness's grid (index (z*ny + y)*nx + x) at the origin of an N^3 grid
  std::vector<uint32_t> vox((size_t)N * N * N, 0u);
  for (int z = 0; z < w->nz; z++)
    for (int y = 0; y < w->ny; y++)
      for (int x = 0; x < w->nx; x++)
        vox[(size_t)x + (size_t)y * N + (size_t)z * N * N] = w->grid[((size_t)z * w->ny + y) * w->nx + x];
  if (v->scene) {
    vrt_scene_destroy(v->scene);
    v->scene = nullptr;
  }
  if (int r = vrt_scene_upload(v->ctx, vox.data(), N, &v->scene)) return r;
  if ((size_t)w->n_emitters > v->em_cap) {
    dev_free(v->ctx, v->emitters, v->em_cap * 16, &v->bytes);
    v->emitters = nullptr;
    v->em_cap = 0;
    if (int r = dev_alloc(v->ctx, (void**)&v->emitters, (size_t)w->n_emitters * 16, &v->bytes)) return r;
    v->em_cap = (size_t)w->n_emitters;
  }
  std::vector<int> em((size_t)w->n_emitters * 4);
  for (int i = 0; i < w->n_emitters; i++) {
    const int32_t* e = w->emitters + 5 * (size_t)i;
    if (e[3] < 0 || e[3] > 5 || e[4] < 0 || e[4] >= 16) return fail(VRT_ERR_INVALID, "bad emitter %d", i);
    em[4 * (size_t)i] = e[0];
    em[4 * (size_t)i + 1] = e[1];
    em[4 * (size_t)i + 2] = e[2];
    em[4 * (size_t)i + 3] = e[3] | (e[4] << 8);
  }
  if (!em.empty())
    CUDA_TRY(cudaMemcpyAsync(v->emitters, em.data(), em.size() * 4, cudaMemcpyHostToDevice, v->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(v->ctx->stream));
  v->n_em = w->n_emitters;
  v->nx = w->nx; v->ny = w->ny; v->nz = w->nz;
  std::memcpy(v->albedo, w->albedo, sizeof v->albedo);
  std::memcpy(v->emission, w->emission, sizeof v->emission);
  v->sky = w->sky_enabled;
  std::memcpy(v->sun_dir, w->sun_dir, 12);
  std::memcpy(v->sun_e, w->sun_e, 12);
  std::memcpy(v->zenith, w->zenith, 12);
  std::memcpy(v->horizon, w->horizon, 12);
  v->have_world = true;
  return VRT_OK;
}

int vrt_vb_set_gbuffer(VrtVb* v, const VrtVbPixel* pixels) {
  if (!v || !pixels) return fail(VRT_ERR_INVALID, "NULL argument");
  if (int r = set_dev(v->ctx)) return r;
  CUDA_TRY(cudaMemcpyAsync(v->px, pixels, (size_t)v->W * v->H * 48, cudaMemcpyHostToDevice, v->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(v->ctx->stream));
  v->have_gbuf = true;
  return VRT_OK;
}

int vrt_vb_frame(VrtVb* v, long long budget, float* out_rgb, uint64_t* rays) {
  if (!v || budget < 0) return fail(VRT_ERR_INVALID, "bad argument");
  if (!v->have_world || !v->have_gbuf) return fail(VRT_ERR_STATE, "set the world and the G-buffer first");
  if (int r = set_dev(v->ctx)) return r;
  cudaStream_t st = v->ctx->stream;
  // paths per pixel from the ray budget (techniques/pt.h:25-28): 5 rays a path
  const double ppp = (double)budget / ((double)v->W * v->H * 5.0);
  VbLaunch L;
  L.scene = v->scene->dev;
  L.nx = v->nx; L.ny = v->ny; L.nz = v->nz;
  L.W = v->W; L.H = v->H;
  L.px = v->px; L.hist = v->hist; L.out = v->out;
  L.emitters = v->emitters;
  L.n_emitters = v->n_em;
  std::memcpy(L.albedo, v->albedo, sizeof L.albedo);
  std::memcpy(L.emission, v->emission, sizeof L.emission);
  L.sky = v->sky;
  std::memcpy(L.sun_dir, v->sun_dir, 12);
  std::memcpy(L.sun_e, v->sun_e, 12);
  std::memcpy(L.zenith, v->zenith, 12);
  std::memcpy(L.horizon, v->horizon, 12);
  L.rays = v->rays;
  L.fcount = v->fcount;
  L.base_paths = (int)std::max(1.0, std::floor(ppp));
  L.frac_p = ppp > 1.0 ? ppp - std::floor(ppp) : 0.0;
  L.stride = ppp < 1.0 ? (int)std::lround(1.0 / std::max(ppp, 1e-9)) : 1;
  CUDA_TRY(cudaMemsetAsync(v->rays, 0, 8, st));
  CUDA_TRY(launch_vb_frame(L, st));
  v->fcount++;
  unsigned long long n = 0;
  CUDA_TRY(cudaMemcpyAsync(&n, v->rays, 8, cudaMemcpyDeviceToHost, st));
  std::vector<float> o4;
  if (out_rgb) {
    o4.resize((size_t)v->W * v->H * 4);
    CUDA_TRY(cudaMemcpyAsync(o4.data(), v->out, o4.size() * 4, cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  if (out_rgb)
    for (size_t i = 0; i < (size_t)v->W * v->H; i++) {
      out_rgb[3 * i] = o4[4 * i];
      out_rgb[3 * i + 1] = o4[4 * i + 1];
      out_rgb[3 * i + 2] = o4[4 * i + 2];
    }
  if (rays) *rays = n;
  return VRT_OK;
}

}  // extern "C"
