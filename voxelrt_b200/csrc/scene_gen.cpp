// scene_gen.cpp -- host-only helpers of the C ABI (no GPU needed):
//   * vrt_camera_matrices / vrt_make_uniforms: camera.js:47-57, math.js:3-74
//     and main.js writeUniforms (399-426), evaluated in double like the
//     JavaScript host and stored as f32;
//   * vrt_camera_spline: the benchmark camera path (0.05 m and 0.5 deg of yaw
//     per frame);
//   * vrt_scene_generate: the reference's procedural world (scene.js:223-405,
//     'default' variant) and the seeded benchmark worlds built from the same
//     pieces (value-noise terrain, Cornell room, trees, lanterns).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include "../../include/vrt.h"

extern "C" int vrt_camera_spline(const VrtCameraPose* spawn, int frame, VrtCameraPose* out);

namespace {

// ---------------------------------------------------------------------------
// camera (math.js / camera.js)
// ---------------------------------------------------------------------------
void mat4_mul_js(const float* a, const float* b, float* out) {
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += (double)a[k * 4 + r] * (double)b[c * 4 + k];
      out[c * 4 + r] = (float)s;
    }
}

void camera_mats(const VrtCameraPose& p, double aspect, float* viewProj, float* invViewProj) {
  const double f = 1.0 / std::tan(p.fov_y / 2.0);
  float proj[16] = {0}, iproj[16] = {0};
  proj[0] = (float)(f / aspect);
  proj[5] = (float)f;
  proj[10] = (float)(p.far_z / (p.near_z - p.far_z));
  proj[11] = -1.0f;
  proj[14] = (float)((p.near_z * p.far_z) / (p.near_z - p.far_z));
  iproj[0] = (float)(aspect / f);
  iproj[5] = (float)(1.0 / f);
  iproj[11] = (float)((p.near_z - p.far_z) / (p.near_z * p.far_z));
  iproj[14] = -1.0f;
  iproj[15] = (float)(1.0 / p.near_z);
  const double cp = std::cos(p.pitch), sp = std::sin(p.pitch), cy = std::cos(p.yaw), sy = std::sin(p.yaw);
  const double fw[3] = {sy * cp, sp, cy * cp};
  const double rt[3] = {-cy, 0.0, sy};
  const double up[3] = {rt[1] * fw[2] - rt[2] * fw[1], rt[2] * fw[0] - rt[0] * fw[2], rt[0] * fw[1] - rt[1] * fw[0]};
  const double z[3] = {-fw[0], -fw[1], -fw[2]};
  const float c2w[16] = {(float)rt[0], (float)rt[1], (float)rt[2], 0.0f,
                         (float)up[0], (float)up[1], (float)up[2], 0.0f,
                         (float)-fw[0], (float)-fw[1], (float)-fw[2], 0.0f,
                         (float)p.pos[0], (float)p.pos[1], (float)p.pos[2], 1.0f};
  auto d3 = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  const float w2c[16] = {(float)rt[0], (float)up[0], (float)z[0], 0.0f,
                         (float)rt[1], (float)up[1], (float)z[1], 0.0f,
                         (float)rt[2], (float)up[2], (float)z[2], 0.0f,
                         (float)-d3(rt, p.pos), (float)-d3(up, p.pos), (float)-d3(z, p.pos), 1.0f};
  mat4_mul_js(proj, w2c, viewProj);
  mat4_mul_js(c2w, iproj, invViewProj);
}

// ---------------------------------------------------------------------------
// world building blocks (scene.js)
// ---------------------------------------------------------------------------
constexpr double kVS = 1.0 / 16.0;
inline uint32_t M(int r, int g, int b, int e = 0) {
  return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16) | ((uint32_t)e << 24);
}
inline int V(double metres) { return (int)std::floor(metres / kVS + 0.5); }   // Math.round for x >= 0
inline int ifl(double x) { return (int)std::floor(x); }

struct Grid {
  int N;
  uint32_t* v;
  size_t idx(int x, int y, int z) const { return (size_t)x + (size_t)y * N + (size_t)z * N * N; }
  bool inb(int x, int y, int z) const { return x >= 0 && y >= 0 && z >= 0 && x < N && y < N && z < N; }
  void set(int x, int y, int z, uint32_t m) { if (inb(x, y, z)) v[idx(x, y, z)] = m; }
  template <typename F>
  void boxf(int x0, int y0, int z0, int x1, int y1, int z1, F f) {
    for (int z = z0; z <= z1; z++)
      for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++) set(x, y, z, f(x, y, z));
  }
  void box(int x0, int y0, int z0, int x1, int y1, int z1, uint32_t m) {
    boxf(x0, y0, z0, x1, y1, z1, [m](int, int, int) { return m; });
  }
};

// Value noise of scene.js:203-222 with the seed as a parameter.
struct Noise {
  int64_t seed;
  double hash(int64_t x, int64_t y) const {
    uint32_t h = (uint32_t)(uint64_t)(x * 374761393LL + y * 668265263LL + seed * 1442695041LL);
    h = (h ^ (h >> 13)) * 1274126177u;
    return (double)(h ^ (h >> 16)) / 4294967296.0;
  }
  static double smooth(double t) { return t * t * (3 - 2 * t); }
  double noise2(double x, double y) const {
    const double xi = std::floor(x), yi = std::floor(y);
    const double xf = smooth(x - xi), yf = smooth(y - yi);
    const int64_t X = (int64_t)xi, Y = (int64_t)yi;
    const double a = hash(X, Y), b = hash(X + 1, Y), c = hash(X, Y + 1), d = hash(X + 1, Y + 1);
    return a + (b - a) * xf + (c - a) * yf + (a - b - c + d) * xf * yf;
  }
  double operator()(double x, double y) const {
    double v = 0, amp = 0.5, f = 1;
    for (int o = 0; o < 4; o++) { v += noise2(x * f, y * f) * amp; amp *= 0.5; f *= 2; }
    return v;
  }
};

// Small counter-based generator for seeded placements (PCG hash chain).
struct Pcg {
  uint32_t s;
  static uint32_t h(uint32_t v) {
    v = v * 747796405u + 2891336453u;
    uint32_t w = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
    return (w >> 22u) ^ w;
  }
  uint32_t u32() { s = h(s); return s; }
  double uni() { return (double)u32() / 4294967296.0; }
};

namespace mat {
uint32_t grass(int v) { return M(88 + v, 130 + v, 60); }
uint32_t dirt(int v) { return M(110 + v, 82 + v, 58); }
uint32_t rock(int v) { return M(120 + v, 120 + v, 125 + v); }
const uint32_t white = M(225, 222, 215), red = M(200, 45, 40), green = M(55, 175, 60);
const uint32_t floorA = M(180, 150, 110), floorB = M(150, 118, 84);
const uint32_t boxTall = M(200, 200, 210), boxShort = M(210, 170, 90), trunk = M(95, 68, 42);
uint32_t leaf(int v) { return M(50 + v, 120 + v, 45); }
const uint32_t lampPost = M(60, 60, 65), lampWarm = M(255, 190, 110, 255), lampCyan = M(90, 220, 255, 255);
const uint32_t lampMagenta = M(255, 90, 200, 255), ceilLight = M(255, 240, 220, 210);
// the 'lamps' variant's emitters and occluders (scene.js:38-56)
const uint32_t lampHot = M(255, 214, 150, 255);
const uint32_t panelOrange = M(255, 140, 40, 200), panelTeal = M(40, 220, 200, 165);
const uint32_t panelViolet = M(190, 80, 255, 245), panelLime = M(150, 255, 60, 125);
const uint32_t dimStrip = M(140, 180, 255, 45), pillar = M(118, 116, 126), shelf = M(140, 105, 70);
const uint32_t lampWarmDim = M(255, 190, 110, 64), lampCyanDim = M(90, 220, 255, 64);
const uint32_t lampMagentaDim = M(255, 90, 200, 64);
}  // namespace mat

// Emissive byte for a radiance intensity I: Le = alb^2 (E/255) 24.
int emissive_byte(double I) { return std::min(255, std::max(1, (int)std::floor(I * 255.0 / 24.0 + 0.5))); }

struct Room { int cx, cz, x0, x1, z0, z1, floorY, y1, roomW, roomH; };

struct World {
  Grid g;
  std::vector<int> heights;
  int groundAt(int x, int z) const {
    const int N = g.N;
    return heights[std::max(0, std::min(N - 1, x)) + std::max(0, std::min(N - 1, z)) * N];
  }
};

// scene.js:248-264 terrain.
void terrain_voxelrt(World& w, const Noise& noise) {
  const int N = w.g.N;
  const int baseH = ifl(N * 0.16);
  w.heights.assign((size_t)N * N, 0);
  for (int z = 0; z < N; z++)
    for (int x = 0; x < N; x++) {
      const int h = baseH + ifl(noise(x * 0.02, z * 0.02) * N * 0.10);
      w.heights[x + z * N] = h;
      for (int y = 0; y <= h && y < N; y++) {
        const int v = (x * 7 + y * 13 + z * 5) % 9;
        uint32_t m;
        if (y == h) m = mat::grass(v);
        else if (y > h - 4) m = mat::dirt(v);
        else m = mat::rock(v);
        w.g.v[w.g.idx(x, y, z)] = m;
      }
    }
}

// The 'lamps' variant's interior lighting in place of the ceiling strip
// (scene.js:303-360): dim cool strips, four coloured wall panels, two pillars
// and a shelf as occluders, and small very bright lamps (ceiling pendants,
// standing lamps, two wall lamps), all placed by room-coordinate arithmetic.
void lamps_interior(Grid& g, const Room& r) {
  const int cx = r.cx, cz = r.cz, x0 = r.x0, x1 = r.x1, z0 = r.z0, z1 = r.z1, floorY = r.floorY, y1 = r.y1;
  const int roomW = r.roomW, roomH = r.roomH;
  const int stripLen = ifl(roomW * 0.5);
  const int sx0 = cx - (stripLen >> 1), sx1 = sx0 + stripLen - 1;
  const int stripDz = ifl(roomW * 0.22);
  for (const int dz : {-stripDz, 0, stripDz}) g.box(sx0, y1, cz + dz - 1, sx1, y1, cz + dz + 1, mat::dimStrip);
  g.box(sx0, y1 - 4, z1, sx1, y1 - 3, z1, mat::dimStrip);
  const int pW = 5, pH = 3;
  const int pMidY = floorY + ifl(roomH * 0.35);
  g.box(x0, pMidY, cz - 9, x0, pMidY + pH, cz - 9 + pW, mat::panelOrange);
  const int tealY = floorY + ifl(roomH * 0.2);
  g.box(x1, tealY, cz - 22, x1, tealY + pH, cz - 22 + pW, mat::panelTeal);
  const int violetY = floorY + ifl(roomH * 0.5);
  g.box(cx + 10, violetY, z1, cx + 10 + pW, violetY + pH, z1, mat::panelViolet);
  const int limeY = floorY + ifl(roomH * 0.4);
  g.box(x0 + 6, limeY, z0, x0 + 6 + pW, limeY + pH, z0, mat::panelLime);
  const int pAx = cx - ifl(roomW * 0.12), pAz = cz + ifl(roomW * 0.15);
  g.box(pAx - 1, floorY + 1, pAz - 1, pAx + 2, y1, pAz + 2, mat::pillar);
  const int pBx = cx + ifl(roomW * 0.22), pBz = cz - ifl(roomW * 0.12);
  g.box(pBx - 1, floorY + 1, pBz - 1, pBx + 2, floorY + ifl(roomH * 0.75), pBz + 2, mat::pillar);
  const int shelfY = floorY + ifl(roomH * 0.3);
  g.box(x1 - 10, shelfY, cz + 10, x1 - 1, shelfY + 1, cz + 26, mat::shelf);
  auto pendant = [&](int lx, int lz) {
    for (int y = y1 - 2; y <= y1; y++) g.set(lx, y, lz, mat::lampPost);
    g.box(lx, y1 - 4, lz, lx, y1 - 3, lz, mat::lampHot);
  };
  pendant(cx + ifl(roomW * 0.19), cz - ifl(roomW * 0.16));
  pendant(cx - ifl(roomW * 0.3), cz + ifl(roomW * 0.3));
  auto standing = [&](int lx, int lz) {
    g.set(lx, floorY + 1, lz, mat::lampPost);
    g.box(lx, floorY + 2, lz, lx, floorY + 3, lz, mat::lampHot);
  };
  standing(x1 - 5, cz + 18);
  standing(pAx - 4, z1 - 4);
  standing(pBx + 4, pBz - 4);
  standing(x0 + 3, z1 - 3);
  g.box(cx - 24, y1 - 6, z0, cx - 24, y1 - 5, z0, mat::lampHot);
  g.box(cx - 6, floorY + 8, z1, cx - 6, floorY + 9, z1, mat::lampHot);
}

// scene.js:267-301 room + 363-366 ceiling strip (or the 'lamps' interior,
// 303-360) + 368-374 boxes.
Room room_voxelrt(World& w, bool lamps = false) {
  const int N = w.g.N;
  Grid& g = w.g;
  Room r;
  r.roomW = std::min(V(5), ifl(N * 0.45));
  r.roomH = std::min(V(3.2), ifl(N * 0.3));
  r.cx = ifl(N * 0.5);
  r.cz = ifl(N * 0.55);
  r.x0 = r.cx - (r.roomW >> 1); r.x1 = r.cx + (r.roomW >> 1);
  r.z0 = r.cz - (r.roomW >> 1); r.z1 = r.cz + (r.roomW >> 1);
  r.floorY = w.groundAt(r.cx, r.cz) + 1;
  r.y1 = r.floorY + r.roomH;
  const int T = 2, x0 = r.x0, x1 = r.x1, z0 = r.z0, z1 = r.z1, floorY = r.floorY, y1 = r.y1, cx = r.cx, cz = r.cz;
  const int roomW = r.roomW, roomH = r.roomH;
  g.boxf(x0 - T, floorY, z0 - T, x1 + T, floorY, z1 + T, [](int x, int, int z) { return mat::dirt((x + z) % 9); });
  g.box(x0 - T, floorY + 1, z0 - T, x1 + T, y1 + T + 4, z1 + T, 0);
  g.boxf(x0 - T, floorY, z0 - T, x1 + T, floorY, z1 + T,
         [](int x, int, int z) { return (((x >> 3) + (z >> 3)) % 2) ? mat::floorA : mat::floorB; });
  g.box(x0 - T, floorY + 1, z1 + 1, x1 + T, y1, z1 + T, mat::white);
  g.box(x0 - T, floorY + 1, z0 - T, x1 + T, y1, z0 - 1, mat::white);
  g.box(x0 - T, floorY + 1, z0 - T, x0 - 1, y1, z1 + T, mat::red);
  g.box(x1 + 1, floorY + 1, z0 - T, x1 + T, y1, z1 + T, mat::green);
  g.box(x0 - T, y1 + 1, z0 - T, x1 + T, y1 + T, z1 + T, mat::white);
  const int doorHalf = ifl(roomW * 0.28);
  g.box(cx - doorHalf, floorY + 1, z0 - T, cx + doorHalf, y1 - 2, z0 - 1, 0);
  const int winY0 = floorY + ifl(roomH * 0.45), winY1 = floorY + ifl(roomH * 0.8);
  g.box(x1 + 1, winY0, cz - ifl(roomW * 0.3), x1 + T, winY1, cz + ifl(roomW * 0.3), 0);
  if (lamps) {
    lamps_interior(g, r);
  } else {
    const int lHalf = ifl(roomW * 0.18);
    g.box(cx - lHalf, y1, cz - lHalf, cx + lHalf, y1, cz + lHalf, mat::ceilLight);
  }
  const int tallW = ifl(roomW * 0.16), tallH = ifl(roomH * 0.55);
  g.box(cx - ifl(roomW * 0.28) - tallW, floorY + 1, cz + ifl(roomW * 0.05), cx - ifl(roomW * 0.28), floorY + tallH,
        cz + ifl(roomW * 0.05) + tallW, mat::boxTall);
  const int shortW = ifl(roomW * 0.18), shortH = ifl(roomH * 0.28);
  g.box(cx + ifl(roomW * 0.10), floorY + 1, cz - ifl(roomW * 0.25), cx + ifl(roomW * 0.10) + shortW,
        floorY + shortH, cz - ifl(roomW * 0.25) + shortW, mat::boxShort);
  return r;
}

// scene.js:376-391 tree.
void tree(World& w, int tx, int tz) {
  Grid& g = w.g;
  const int gr = w.groundAt(tx, tz);
  const int trunkH = V(1.4) + ((tx * 31 + tz * 17) % V(0.8));
  for (int y = gr + 1; y <= gr + trunkH; y++) { g.set(tx, y, tz, mat::trunk); g.set(tx + 1, y, tz, mat::trunk); }
  const int cy = gr + trunkH + V(0.35);
  const int r = V(0.7) + ((tx + tz) % 3);
  for (int dz = -r; dz <= r; dz++)
    for (int dy = -r; dy <= r; dy++)
      for (int dx = -r; dx <= r; dx++) {
        const double d2 = dx * dx + dy * dy * 1.6 + dz * dz;
        if (d2 <= r * r && ((dx * 13 + dy * 7 + dz * 11) % 5 != 0 || d2 < r * r * 0.5)) {
          g.set(tx + dx, cy + dy, tz + dz, mat::leaf((dx * 3 + dy * 5 + dz * 7) % 12 + ((dx + dy + dz) % 2) * 6));
        }
      }
}

// scene.js:395-401 lantern post.
void lantern(World& w, int lx, int lz, uint32_t m) {
  const int gr = w.groundAt(lx, lz);
  const int h = V(1.1);
  for (int y = gr + 1; y <= gr + h; y++) w.g.set(lx, y, lz, mat::lampPost);
  w.g.box(lx - 1, gr + h + 1, lz - 1, lx + 1, gr + h + 3, lz + 1, m);
}

// scene.js generateScene(N, variant): 'default' or 'lamps' (dimmed exterior
// lanterns, no corner lamp: scene.js:402-409).
void gen_voxelrt(Grid g, uint32_t seed, VrtCameraPose* spawn, bool lamps = false) {
  World w{g, {}};
  const int N = g.N;
  Noise noise{(int64_t)seed};
  terrain_voxelrt(w, noise);
  Room r = room_voxelrt(w, lamps);
  const double spots[6][2] = {{0.15, 0.2}, {0.82, 0.25}, {0.2, 0.8}, {0.86, 0.78}, {0.12, 0.55}, {0.65, 0.12}};
  for (auto& s : spots) tree(w, ifl(N * s[0]), ifl(N * s[1]));
  lantern(w, ifl(N * 0.35), ifl(N * 0.25), lamps ? mat::lampWarmDim : mat::lampWarm);
  lantern(w, ifl(N * 0.68), ifl(N * 0.30), lamps ? mat::lampCyanDim : mat::lampCyan);
  lantern(w, ifl(N * 0.25), ifl(N * 0.65), lamps ? mat::lampMagentaDim : mat::lampMagenta);
  if (!lamps) w.g.box(r.x0 + 2, r.floorY + 1, r.z1 - 4, r.x0 + 4, r.floorY + 3, r.z1 - 2, mat::lampWarm);
  if (spawn) {
    spawn->pos[0] = r.cx * kVS;
    spawn->pos[1] = (w.groundAt(r.cx, r.z0 - V(3)) + 1) * kVS + 1.65;
    spawn->pos[2] = (r.z0 - V(3.5)) * kVS;
    spawn->yaw = 0.0;
    spawn->pitch = -0.05;
    spawn->fov_y = 70.0 * M_PI / 180.0;
    spawn->near_z = 0.05;
    spawn->far_z = 400.0;
  }
}

// Benchmark world (256^3 class): the reference world with the noise seed,
// 40 seeded trees, and red/green/blue lanterns of intensity 15.  The default
// camera path starts outside the room doorway and walks in.
void gen_full(Grid g, uint32_t seed, VrtCameraPose* spawn) {
  World w{g, {}};
  const int N = g.N;
  Noise noise{(int64_t)seed};
  terrain_voxelrt(w, noise);
  Room r = room_voxelrt(w);
  // camera corridor (kept free of trees): x in [cx-24, cx+24], z < room
  const int corX0 = r.cx - 24, corX1 = r.cx + 24;
  Pcg rng{Pcg::h(seed * 2654435761u + 17u)};
  int placed = 0;
  for (int attempt = 0; attempt < 4000 && placed < 40; attempt++) {
    const int tx = ifl(N * (0.05 + 0.90 * rng.uni()));
    const int tz = ifl(N * (0.05 + 0.90 * rng.uni()));
    const int margin = V(0.7) + 3;
    const bool inRoom = tx >= r.x0 - 2 - margin && tx <= r.x1 + 2 + margin && tz >= r.z0 - 2 - margin &&
                        tz <= r.z1 + 2 + margin;
    const bool inCorridor = tx >= corX0 - margin && tx <= corX1 + margin && tz < r.z0;
    if (inRoom || inCorridor) continue;
    tree(w, tx, tz);
    placed++;
  }
  const int E = emissive_byte(15.0);
  lantern(w, ifl(N * 0.35), ifl(N * 0.25), M(255, 40, 40, E));
  lantern(w, ifl(N * 0.68), ifl(N * 0.30), M(40, 255, 40, E));
  lantern(w, ifl(N * 0.25), ifl(N * 0.65), M(40, 40, 255, E));
  w.g.box(r.x0 + 2, r.floorY + 1, r.z1 - 4, r.x0 + 4, r.floorY + 3, r.z1 - 2, mat::lampWarm);
  if (spawn) {
    const int zStart = std::max(2, r.z0 - 60);
    int gmax = r.floorY - 1;
    for (int z = zStart; z <= r.z0; z++)
      for (int x = r.cx - 16; x <= r.cx + 16; x++) gmax = std::max(gmax, w.groundAt(x, z));
    spawn->pos[0] = r.cx * kVS;
    spawn->pos[1] = (gmax + 1) * kVS + 1.65;
    spawn->pos[2] = zStart * kVS;
    spawn->yaw = -30.0 * M_PI / 180.0;
    spawn->pitch = -0.05;
    spawn->fov_y = 60.0 * M_PI / 180.0;
    spawn->near_z = 0.05;
    spawn->far_z = 400.0;
  }
}

// Small world (64^3): value-noise heightfield of height 8-20 voxels in green
// with +-10% albedo jitter, and a 24^3 Cornell box (white floor/ceiling/back,
// red left, green right, open front) holding two white boxes under a
// one-voxel 6x6 emissive ceiling panel of intensity 10.
void gen_small(Grid g, uint32_t seed, VrtCameraPose* spawn) {
  const int N = g.N;
  Noise noise{(int64_t)seed};
  const double sc = 64.0 / N;
  auto S = [&](int v) { return (int)std::floor(v / sc + 1e-9); };
  for (int z = 0; z < N; z++)
    for (int x = 0; x < N; x++) {
      int h = S(8) + ifl(noise(x * 0.06 * sc, z * 0.06 * sc) * (S(20) - S(8) + 1));
      h = std::min(std::max(h, S(8)), S(20));
      for (int y = 0; y <= h; y++) {
        const uint32_t hv = Pcg::h((uint32_t)(x + y * N + z * N * N) ^ (seed * 0x9e3779b9u));
        const double j = 0.9 + 0.2 * (double)hv / 4294967296.0;
        const int r = std::min(255, (int)std::floor(90 * j + 0.5));
        const int gg = std::min(255, (int)std::floor(150 * j + 0.5));
        const int b = std::min(255, (int)std::floor(60 * j + 0.5));
        g.v[g.idx(x, y, z)] = M(r, gg, b);
      }
    }
  const int bx0 = S(20), bx1 = S(44) - 1, by0 = S(21), by1 = S(45) - 1, bz0 = S(30), bz1 = S(54) - 1;
  g.box(bx0 + 1, by0 + 1, bz0, bx1 - 1, by1 - 1, bz1 - 1, 0);   // interior air (open front)
  g.box(bx0, by0, bz0, bx1, by0, bz1, mat::white);              // floor
  g.box(bx0, by1, bz0, bx1, by1, bz1, mat::white);              // ceiling
  g.box(bx0, by0, bz1, bx1, by1, bz1, mat::white);              // back
  g.box(bx0, by0, bz0, bx0, by1, bz1, mat::red);                // left (-x)
  g.box(bx1, by0, bz0, bx1, by1, bz1, mat::green);              // right (+x)
  const int E = emissive_byte(10.0);
  const int pc = (bx0 + bx1) / 2, pz = (bz0 + bz1) / 2 + S(2);
  g.box(pc - S(3) + 1, by1, pz - S(3) + 1, pc + S(3), by1, pz + S(3), M(255, 255, 255, E));
  g.box(S(24), by0 + 1, S(42), S(30) - 1, by0 + S(12), S(48) - 1, mat::white);   // tall box
  g.box(S(34), by0 + 1, S(34), S(40) - 1, by0 + S(6), S(40) - 1, mat::white);     // short box
  if (spawn) {
    spawn->pos[0] = 2.0 * N / 64.0;
    spawn->pos[1] = 2.125 * N / 64.0;
    spawn->pos[2] = 0.5 * N / 64.0;
    spawn->yaw = 0.0;
    spawn->pitch = -0.12;
    spawn->fov_y = 60.0 * M_PI / 180.0;
    spawn->near_z = 0.05;
    spawn->far_z = 400.0;
  }
}

// Random world: terrain, N/8 seeded boxes, 0.1% of solid voxels emissive with
// intensity U(1,20); camera at a seeded pose above the terrain.
void gen_random(Grid g, uint32_t seed, VrtCameraPose* spawn) {
  const int N = g.N;
  Noise noise{(int64_t)seed + 7};
  Pcg rng{Pcg::h(seed ^ 0xa511e9b3u)};
  std::vector<int> heights((size_t)N * N);
  const int base = ifl(N * 0.1), amp = ifl(N * 0.15) + 1;
  for (int z = 0; z < N; z++)
    for (int x = 0; x < N; x++) {
      const int h = base + ifl(noise(x * 0.03 * 64.0 / N, z * 0.03 * 64.0 / N) * amp);
      heights[x + (size_t)z * N] = h;
      for (int y = 0; y <= h; y++) {
        const int v = (x * 7 + y * 13 + z * 5) % 9;
        g.v[g.idx(x, y, z)] = y == h ? mat::grass(v) : (y > h - 4 ? mat::dirt(v) : mat::rock(v));
      }
    }
  const int nboxes = std::max(4, N / 8);
  for (int i = 0; i < nboxes; i++) {
    const int sx = 2 + (int)(rng.uni() * N * 0.08), sy = 2 + (int)(rng.uni() * N * 0.15), sz = 2 + (int)(rng.uni() * N * 0.08);
    const int x0 = (int)(rng.uni() * (N - sx)), z0 = (int)(rng.uni() * (N - sz));
    const int y0 = heights[x0 + (size_t)z0 * N];
    const uint32_t m = M(60 + (int)(rng.uni() * 190), 60 + (int)(rng.uni() * 190), 60 + (int)(rng.uni() * 190));
    g.box(x0, y0, z0, x0 + sx - 1, std::min(N - 1, y0 + sy - 1), z0 + sz - 1, m);
  }
  // 0.1% emissive voxels: each solid voxel independently with p = 0.001
  for (size_t i = 0; i < (size_t)N * N * N; i++) {
    if (g.v[i] == 0u) continue;
    const uint32_t hv = Pcg::h((uint32_t)i * 2654435761u ^ seed);
    if (hv % 1000u != 0u) continue;
    const double I = 1.0 + 19.0 * (double)Pcg::h(hv) / 4294967296.0;
    g.v[i] = (g.v[i] & 0x00ffffffu) | ((uint32_t)emissive_byte(I) << 24);
  }
  if (spawn) {
    const int cx = (int)(N * (0.25 + 0.5 * rng.uni())), cz = (int)(N * (0.25 + 0.5 * rng.uni()));
    int gmax = 0;
    for (int z = std::max(0, cz - 4); z <= std::min(N - 1, cz + 4); z++)
      for (int x = std::max(0, cx - 4); x <= std::min(N - 1, cx + 4); x++) {
        for (int y = N - 1; y >= 0; y--)
          if (g.v[g.idx(x, y, z)]) { gmax = std::max(gmax, y); break; }
      }
    spawn->pos[0] = (cx + 0.5) * kVS;
    spawn->pos[1] = std::min(N - 2.0, gmax + 2.0 + 0.2 * N * rng.uni()) * kVS;
    spawn->pos[2] = (cz + 0.5) * kVS;
    spawn->yaw = rng.uni() * 2.0 * M_PI;
    spawn->pitch = -0.35 * rng.uni();
    spawn->fov_y = 60.0 * M_PI / 180.0;
    spawn->near_z = 0.05;
    spawn->far_z = 400.0;
  }
}

}  // namespace

extern "C" {

int vrt_camera_matrices(const VrtCameraPose* pose, double aspect, float* view_proj, float* inv_view_proj) {
  if (!pose || !view_proj || !inv_view_proj || !(aspect > 0.0)) return VRT_ERR_INVALID;
  camera_mats(*pose, aspect, view_proj, inv_view_proj);
  return VRT_OK;
}

int vrt_make_uniforms(const VrtCameraPose* cur, const VrtCameraPose* prev, const VrtLighting* light,
                      uint32_t frame, uint32_t bounces, uint32_t flags, int width, int height, float exposure,
                      float max_history, VrtUniforms* out) {
  if (!cur || !light || !out || width < 1 || height < 1) return VRT_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  const double aspect = (double)width / (double)height;
  float vp[16], ivp[16];
  camera_mats(*cur, aspect, vp, ivp);
  std::memcpy(out->invViewProj, ivp, sizeof ivp);
  if (prev) {
    float pvp[16], pivp[16];
    camera_mats(*prev, aspect, pvp, pivp);
    std::memcpy(out->prevViewProj, pvp, sizeof pvp);
  } else {
    std::memcpy(out->prevViewProj, vp, sizeof vp);   // first frame: prev = current (main.js:401)
  }
  const VrtCameraPose* pp = prev ? prev : cur;
  for (int i = 0; i < 3; i++) {
    out->camPos[i] = (float)cur->pos[i];
    out->prevCamPos[i] = (float)pp->pos[i];
  }
  double sd[3] = {light->sun_dir[0], light->sun_dir[1], light->sun_dir[2]};
  double l = std::sqrt(sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]);
  if (!(l > 0.0)) l = 1.0;
  for (int i = 0; i < 3; i++) out->sunDir[i] = (float)(sd[i] / l);
  out->sunDir[3] = light->sun_cos_radius;
  for (int i = 0; i < 3; i++) out->sunRadiance[i] = light->sun_irradiance[i];
  out->sunRadiance[3] = light->sky_intensity;
  out->params0[0] = frame;
  out->params0[1] = bounces;
  out->params0[2] = flags;
  out->params1[0] = (float)width;
  out->params1[1] = (float)height;
  out->params1[2] = exposure;
  // reference defaults of the ReSTIR tuning slots (main.js:71-89); params2.x
  // (the preset flags) stays 0 = preset=base
  out->params2[0] = 0u;
  out->params2[2] = 3u;
  out->params3[0] = 20.0f; out->params3[1] = 1.0f; out->params3[2] = 0.1f; out->params3[3] = 0.0008f;
  out->params4[0] = 30.0f; out->params4[1] = max_history; out->params4[2] = 24.0f;
  out->params5[0] = 48.0f; out->params5[1] = 1.0f; out->params5[2] = 1.0f; out->params5[3] = 0.5f;
  out->params6[0] = 8.0f;
  return VRT_OK;
}

// Camera path of the benchmark: yaw advances 0.5 degree per frame and the
// camera moves 0.05 m per frame along its horizontal heading.
int vrt_camera_spline(const VrtCameraPose* spawn, int frame, VrtCameraPose* out) {
  if (!spawn || !out || frame < 0) return VRT_ERR_INVALID;
  VrtCameraPose p = *spawn;
  const double dyaw = 0.5 * M_PI / 180.0;
  for (int f = 0; f < frame; f++) {
    const double yaw = spawn->yaw + f * dyaw;
    p.pos[0] += 0.05 * std::sin(yaw);
    p.pos[2] += 0.05 * std::cos(yaw);
  }
  p.yaw = spawn->yaw + frame * dyaw;
  *out = p;
  return VRT_OK;
}

int vrt_scene_generate(int kind, int N, uint32_t seed, uint32_t* out_voxels, VrtCameraPose* spawn) {
  if (!out_voxels || N < 8 || N % 8 != 0 || N > 2048) return VRT_ERR_INVALID;
  if (kind < VRT_SCENE_VOXELRT || kind > VRT_SCENE_VOXELRT_LAMPS) return VRT_ERR_INVALID;
  std::memset(out_voxels, 0, (size_t)N * N * N * sizeof(uint32_t));
  Grid g{N, out_voxels};
  switch (kind) {
    case VRT_SCENE_VOXELRT: gen_voxelrt(g, seed, spawn); break;
    case VRT_SCENE_SMALL: gen_small(g, seed, spawn); break;
    case VRT_SCENE_FULL: gen_full(g, seed, spawn); break;
    case VRT_SCENE_RANDOM: gen_random(g, seed, spawn); break;
    case VRT_SCENE_VOXELRT_LAMPS: gen_voxelrt(g, seed, spawn, true); break;
    default: return VRT_ERR_INVALID;
  }
  return VRT_OK;
}

}  // extern "C"
