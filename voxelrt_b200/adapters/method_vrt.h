// method_vrt.h -- VoxelBench Technique backed by libvrt (VoxelBench/pipeline/technique.h:8-14).
//
// Drop-in for the VoxelBench harness: place this header where the harness can
// include it (e.g. VoxelBench/pipeline/techniques/), add the include path of
// include/vrt.h, link -lvrt, and register it in makeTech (harness.cpp:39-199):
//
//     if (m == "VRT") return new MethodVRT();
//
// The technique reads the harness's globals -- grid and size, MAT palette,
// emFaces, SKY, gbuf -- uploads them to the GPU, and estimates the indirect
// radiance of every pixel with the harness's baseline estimator
// (techniques/pt.h) on libvrt's two-level DDA, within the harness's ray
// budget.  The harness's metrics (psnrTM, ssimTM, gradPsnrTM, flickerTM) then
// score the GPU output like any other technique.
#pragma once
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>
#include "technique.h"
#include "vrt.h"

struct MethodVRT : Technique {
  VrtCtx* ctx = nullptr;
  VrtVb* vb = nullptr;
  std::vector<VrtVbPixel> px;
  std::vector<float> rgb;
  int device = 0;

  explicit MethodVRT(int cuda_device = 0) : device(cuda_device) {}

  static void check(int code, const char* what) {
    if (code != VRT_OK) throw std::runtime_error(std::string(what) + ": " + vrt_last_error_string());
  }

  const char* name() override { return "VRT"; }

  // The harness's world as the library wants it (core.h:60-116).
  void upload_world() {
    VrtVbWorld w{};
    w.nx = NX; w.ny = NY; w.nz = NZ;
    w.grid = grid.data();
    for (int m = 0; m < MAXMAT && m < 16; m++) {
      w.albedo[m][0] = MAT[m].alb.x; w.albedo[m][1] = MAT[m].alb.y; w.albedo[m][2] = MAT[m].alb.z;
      w.emission[m][0] = MAT[m].emi.x; w.emission[m][1] = MAT[m].emi.y; w.emission[m][2] = MAT[m].emi.z;
    }
    std::vector<int32_t> em;
    em.reserve(emFaces.size() * 5);
    for (const EmFace& e : emFaces) {
      em.push_back(e.x); em.push_back(e.y); em.push_back(e.z); em.push_back(e.f); em.push_back(e.m);
    }
    w.emitters = em.data();
    w.n_emitters = (int)emFaces.size();
    w.sky_enabled = SKY.enabled ? 1 : 0;
    const V3* v[4] = {&SKY.sunDir, &SKY.sunE, &SKY.zenith, &SKY.horizon};
    float* dst[4] = {w.sun_dir, w.sun_e, w.zenith, w.horizon};
    for (int k = 0; k < 4; k++) { dst[k][0] = v[k]->x; dst[k][1] = v[k]->y; dst[k][2] = v[k]->z; }
    check(vrt_vb_set_world(vb, &w), "vrt_vb_set_world");
  }

  void upload_gbuffer() {
    px.resize((size_t)W * H);
    for (int i = 0; i < W * H; i++) {
      const GPix& g = gbuf[(size_t)i];
      VrtVbPixel& p = px[(size_t)i];
      p.pos[0] = g.pos.x; p.pos[1] = g.pos.y; p.pos[2] = g.pos.z;
      p.depth = g.depth;
      p.n[0] = g.n.x; p.n[1] = g.n.y; p.n[2] = g.n.z;
      p.flags = (g.hit ? 1u : 0u) | (g.hit && emissive(g.m) ? 2u : 0u);
      p.albedo[0] = g.alb.x; p.albedo[1] = g.alb.y; p.albedo[2] = g.alb.z;
      p.pad = 0u;
    }
    check(vrt_vb_set_gbuffer(vb, px.data()), "vrt_vb_set_gbuffer");
  }

  void init() override {
    if (!vb) {
      VrtDeviceConfig cfg{device, 0};
      check(vrt_create(&cfg, &ctx), "vrt_create");
      check(vrt_vb_create(ctx, W, H, &vb), "vrt_vb_create");
    }
    check(vrt_vb_reset(vb), "vrt_vb_reset");
    upload_world();
    upload_gbuffer();
    out.assign((size_t)W * H, V3{});
    rgb.assign((size_t)W * H * 3, 0.0f);
  }

  // Geometry or lighting changed: the world and the G-buffer are re-read; the
  // history is kept, as the baseline technique does (techniques/pt.h:16-20).
  void onEvent(const SceneEvent& e) override {
    (void)e;
    upload_world();
    upload_gbuffer();
  }

  long frame(long budget) override {
    uint64_t rays = 0;
    check(vrt_vb_frame(vb, budget, rgb.data(), &rays), "vrt_vb_frame");
    for (int i = 0; i < W * H; i++) out[(size_t)i] = V3(rgb[3 * (size_t)i], rgb[3 * (size_t)i + 1], rgb[3 * (size_t)i + 2]);
    return (long)rays;
  }

  ~MethodVRT() override {
    if (vb) vrt_vb_destroy(vb);
    if (ctx) vrt_destroy(ctx);
  }
};
