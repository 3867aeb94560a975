// vb_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C entry layer compiled together with the reference's own VoxelBench CPU
// sources (VoxelBench/pipeline/core.cpp, scenes_town.cpp, scenes_city.cpp;
// scenes.h for the scene factory) into oracle/_ref/libvbref.so.  It exposes:
//   * the reference's scenes (scenes.h:183-190 makeScene) as voxel grids,
//   * its per-voxel traversal traceNaive (core.cpp:23-50) and its brickmap
//     traversal trace (core.cpp:52-130),
// so that tests can pin the oracle's DDA to the reference's traversal and
// bench.py's reference arm can time the reference's own CPU traversal.
#include "core.h"
#include "scenes.h"
#include <memory>
#include <omp.h>

extern "C" {

// Build a named VoxelBench scene (pre-event or post-event state).
// dims[0..2] receive NX, NY, NZ.  Returns 0 on success.
int vb_build_scene(const char* name, int post, int* dims) {
  std::unique_ptr<Scene> s(makeScene(name));
  if (!s) return -1;
  s->build();
  if (post) s->applyEvent();
  dims[0] = NX; dims[1] = NY; dims[2] = NZ;
  return 0;
}

// Copy the current grid (material ids, index (z*NY+y)*NX+x) to out.
long vb_copy_grid(uint8_t* out) {
  std::memcpy(out, grid.data(), grid.size());
  return (long)grid.size();
}

// Replace the grid (dims multiples of 4) and rebuild the 4^3 brick masks.
int vb_set_grid(int nx, int ny, int nz, const uint8_t* g) {
  if (nx % 4 || ny % 4 || nz % 4) return -1;
  setDims(nx, ny, nz);
  std::memcpy(grid.data(), g, grid.size());
  rebuildAllBricks();
  return 0;
}

// Rays in voxel units.  hit[i] = 0/1, vox[3i..] = hit voxel, face[i], t[i].
static void run_batch(bool naive, const float* o, const float* d, const float* tmax, int n,
                      int* hit, int* vox, int* face, float* t, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    Hit h{};
    V3 oo(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
    V3 dd(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
    bool r = naive ? traceNaive(oo, dd, tmax[i], h) : trace(oo, dd, tmax[i], h);
    if (hit) hit[i] = r ? 1 : 0;
    if (vox) { vox[3 * i] = r ? h.vx : -1; vox[3 * i + 1] = r ? h.vy : -1; vox[3 * i + 2] = r ? h.vz : -1; }
    if (face) face[i] = r ? h.face : -1;
    if (t) t[i] = r ? h.t : -1.0f;
  }
}

void vb_trace_naive_batch(const float* o, const float* d, const float* tmax, int n,
                          int* hit, int* vox, int* face, float* t) {
  run_batch(true, o, d, tmax, n, hit, vox, face, t, 0);
}

void vb_trace_batch(const float* o, const float* d, const float* tmax, int n,
                    int* hit, int* vox, int* face, float* t, int threads) {
  run_batch(false, o, d, tmax, n, hit, vox, face, t, threads);
}

// Wall-clock seconds for tracing n rays with the brickmap traversal on
// `threads` OpenMP threads (results discarded).
double vb_time_trace(const float* o, const float* d, const float* tmax, int n, int threads) {
  std::vector<int> hit(n);
  auto t0 = std::chrono::high_resolution_clock::now();
  run_batch(false, o, d, tmax, n, hit.data(), nullptr, nullptr, nullptr, threads);
  auto t1 = std::chrono::high_resolution_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
