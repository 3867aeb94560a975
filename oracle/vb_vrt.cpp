// vb_vrt.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The VoxelBench harness's `run` protocol (VoxelBench/pipeline/harness.cpp:
// 280-330) for two techniques side by side: the reference's own baseline
// MethodPT (techniques/pt.h, CPU) and MethodVRT (voxelrt_b200/adapters/
// method_vrt.h, the library on the GPU), at the same ray budget, on one of
// the reference's scenes, scored with the reference's metrics (metrics.h)
// against a path-traced reference rendered here with the reference's own
// renderReference (core.cpp:238-253) -- the frozen results/raw references are
// not part of this repository.
//
// Built by oracle/Makefile (target vbvrt) from the reference sources into
// oracle/_ref/vb_vrt, linked against voxelrt_b200/libvrt.so.
//
// usage: vb_vrt <scene> <mult> <frames> <ref_spp> [threads] [event_frame]
// threads: OpenMP threads of the techniques (the harness uses 2,
// harness.cpp:201); the references use every host thread.  Prints one JSON
// line per technique and frame, then a summary line each.
#include "core.h"
#include "scenes.h"
#include "technique.h"
#include "metrics.h"
#include "techniques/pt.h"
#include "method_vrt.h"
#include <chrono>
#include <memory>
#include <omp.h>

static void prep_state(Scene* s, bool post) {   // harness.cpp:32-39
  s->build();
  if (post) s->applyEvent();
  collectEmitters();
  s->camera();
  buildGBuffer();
  buildDirect(128);
}

static double mean_luma(const std::vector<V3>& img) {
  double acc = 0.0;
  long n = 0;
  for (int i = 0; i < W * H; i++)
    if (gbuf[(size_t)i].hit) { acc += luma(img[(size_t)i]); n++; }
  return n ? acc / (double)n : 0.0;
}

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: vb_vrt <scene> <mult> <frames> <ref_spp> [threads] [event_frame]\n");
    return 2;
  }
  const std::string sc = argv[1];
  const float mult = (float)atof(argv[2]);
  const int frames = atoi(argv[3]), ref_spp = atoi(argv[4]);
  const int all_threads = omp_get_max_threads();
  const int threads = argc > 5 && atoi(argv[5]) > 0 ? atoi(argv[5]) : all_threads;
  const int event_frame = argc > 6 ? atoi(argv[6]) : -1;
  std::unique_ptr<Scene> s(makeScene(sc));
  if (!s) { fprintf(stderr, "unknown scene %s\n", sc.c_str()); return 2; }
  const long budget = (long)(4L * W * H * mult);

  // references of the pre- and post-event states
  std::vector<V3> refPre((size_t)W * H), refPost((size_t)W * H);
  prep_state(s.get(), true);
  renderReference(refPost, ref_spp, 7919u * 1u + 13u);
  s.reset(makeScene(sc));
  prep_state(s.get(), false);
  auto t0 = std::chrono::high_resolution_clock::now();
  renderReference(refPre, ref_spp, 7919u * 1u);
  const double ref_s = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  printf("{\"reference\": \"%s\", \"spp\": %d, \"seconds\": %.3f, \"mean_luma\": %.6f, \"threads\": %d}\n",
         sc.c_str(), ref_spp, ref_s, mean_luma(refPre), all_threads);
  omp_set_num_threads(threads);

  for (int which = 0; which < 2; which++) {
    s.reset(makeScene(sc));
    prep_state(s.get(), false);
    std::unique_ptr<Technique> m(which == 0 ? (Technique*)new MethodPT() : (Technique*)new MethodVRT());
    m->init();
    std::vector<V3> prev;
    double ms_sum = 0.0, last_psnr = 0.0, last_ssim = 0.0, last_gpsnr = 0.0;
    long rays_sum = 0;
    for (int f = 0; f < frames; f++) {
      if (f == event_frame) {   // harness.cpp:301-306
        if (s->event.geomEdit) { s->applyEvent(); collectEmitters(); buildGBuffer(); }
        else s->applyEvent();
        buildDirect(128);
        m->onEvent(s->event);
      }
      const auto a = std::chrono::high_resolution_clock::now();
      const long rays = m->frame(budget);
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - a).count();
      const auto& ref = (event_frame >= 0 && f >= event_frame) ? refPost : refPre;
      const double psnr = psnrTM(m->out, ref), ssim = ssimTM(m->out, ref), gpsnr = gradPsnrTM(m->out, ref);
      const double flick = prev.empty() ? 0.0 : flickerTM(m->out, prev);
      prev = m->out;
      ms_sum += ms;
      rays_sum += rays;
      last_psnr = psnr; last_ssim = ssim; last_gpsnr = gpsnr;
      printf("{\"method\": \"%s\", \"frame\": %d, \"psnr\": %.4f, \"ssim\": %.5f, \"gpsnr\": %.4f, \"flicker\": %.6f, "
             "\"rays\": %ld, \"ms\": %.3f}\n", m->name(), f, psnr, ssim, gpsnr, flick, rays, ms);
    }
    printf("{\"summary\": \"%s\", \"scene\": \"%s\", \"mult\": %.2f, \"budget\": %ld, \"frames\": %d, "
           "\"mean_ms\": %.4f, \"rays_per_frame\": %.1f, \"psnr\": %.4f, \"ssim\": %.5f, \"gpsnr\": %.4f, "
           "\"mean_luma\": %.6f, \"threads\": %d}\n",
           m->name(), sc.c_str(), mult, budget, frames, ms_sum / frames, (double)rays_sum / frames, last_psnr,
           last_ssim, last_gpsnr, mean_luma(m->out), threads);
    fflush(stdout);
  }
  return 0;
}
