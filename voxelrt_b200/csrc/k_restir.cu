// k_restir.cu -- the reference's ReSTIR GI preset (`preset=gi`, main.js:44:
// flags RF_RESTIR | RF_TEMPORAL | RF_SPATIAL): reservoirs for indirect light
// only, temporal reuse with a confidence cap, random-disk spatial reuse and
// shading of the selected sample.  Three passes, as the reference dispatches
// them (main.js:736-739):
//
//   initial  (pathtrace.wgsl:248-284, 332-457, RF_UNIFIED off): primary hit,
//            G-buffer and albedo, pass-through radiance `direct` = emission +
//            sun-cone NEE, one BSDF bounce candidate whose reconnection vertex
//            x2 carries Lo(x2) estimated by continuing the path (estimateLo,
//            pathtrace.wgsl:205-246) -> reservoirs A, direct -> rgba16f
//   temporal (reuse_temporal.wgsl:140-279, no dupmap / rescue / world cache /
//            mutation): confidence-weighted merge with the reprojected history
//            reservoir of B -> A
//   spatial  (reuse_spatial.wgsl:128-354, random disk, generic neighbour test,
//            scalar shading weight): balance-heuristic merge over the canonical
//            and up to three neighbour domains, one visibility ray for a
//            neighbour's sample, radiance (demodulated) = direct + f W -> rgba16f,
//            post-reuse reservoir -> B (next frame's history)
//
// Reservoirs keep the reference's 32-byte record (restir.wgsl:14-31, 61-84):
// posW = (position or direction, W); data = (radiance RG as f16 x 2, radiance
// B f16 | kind << 16 | confidence u8 << 18, octahedral normal as snorm16 x 2,
// seed), stored as two 16-byte words per pixel (array-of-structures: the
// spatial pass gathers whole records of random neighbours, one 32-byte sector
// each).  One thread per pixel; 16 x 16 blocks whose warps cover 8 x 4 tiles;
// the brick occupancy bitmap is staged in shared memory.  The arithmetic
// follows the WGSL expression by expression (no contraction), so the CPU
// restatement reproduces every word bit for bit.
#include "trace_kernel.cuh"
#include "wavefront_core.cuh"

namespace vrt {

enum : uint32_t { kSkNone = 0u, kSkPoint = 1u, kSkDir = 2u };   // restir.wgsl:29-31

// Decoded reservoir sample (restir.wgsl:33-41).
struct RSample {
  uint32_t kind;
  F3 pos, n, rad;
  float W, c;
  uint32_t seed;
};

VRT_DI RSample null_sample(float c) {
  RSample s;
  s.kind = kSkNone;
  s.pos = s.n = s.rad = f3(0.0f, 0.0f, 0.0f);
  s.W = 0.0f;
  s.c = c;
  s.seed = 0u;
  return s;
}

// WGSL f32 -> i32 conversion: toward zero, saturating, NaN -> 0.
VRT_DI int itrunc_(float x) { return __float2int_rz(x); }

// pack2x16snorm / unpack2x16snorm, one component.
VRT_DI uint32_t snorm16(float v) {
  const float c = fmin_(1.0f, fmax_(-1.0f, v));
  return (uint32_t)(uint16_t)(int16_t)(int)floorf(0.5f + 32767.0f * c);
}
VRT_DI float unsnorm16(uint32_t b) { return fmax_((float)(int16_t)(uint16_t)b / 32767.0f, -1.0f); }

VRT_DI float sgn_ge0(float x) { return x >= 0.0f ? 1.0f : -1.0f; }

// octEncode / octDecode (restir.wgsl:43-59).
VRT_DI void oct_encode(F3 nIn, float& ex, float& ey) {
  const float s = (fabsf(nIn.x) + fabsf(nIn.y)) + fabsf(nIn.z);
  const F3 n = f3(nIn.x / s, nIn.y / s, nIn.z / s);
  ex = n.x;
  ey = n.y;
  if (n.z < 0.0f) {
    ex = (1.0f - fabsf(n.y)) * sgn_ge0(n.x);
    ey = (1.0f - fabsf(n.x)) * sgn_ge0(n.y);
  }
}

VRT_DI F3 oct_decode(float ex, float ey) {
  F3 n = f3(ex, ey, (1.0f - fabsf(ex)) - fabsf(ey));
  if (n.z < 0.0f) n = f3((1.0f - fabsf(n.y)) * sgn_ge0(n.x), (1.0f - fabsf(n.x)) * sgn_ge0(n.y), n.z);
  return normalize3(n);
}

// packReservoir (restir.wgsl:61-71) into the two 16-byte words of pixel p.
VRT_DI void store_res(uint4* res, size_t p, const RSample& s) {
  const uint32_t cq = min((uint32_t)__float2uint_rz(s.c + 0.5f), 255u);
  const F3 nn = s.kind != kSkPoint ? f3(0.0f, 1.0f, 0.0f) : s.n;
  float ex, ey;
  oct_encode(nn, ex, ey);
  res[2 * p] = make_uint4(__float_as_uint(s.pos.x), __float_as_uint(s.pos.y), __float_as_uint(s.pos.z),
                          __float_as_uint(s.W));
  res[2 * p + 1] = make_uint4(h2bits(s.rad.x) | (h2bits(s.rad.y) << 16),
                              (h2bits(s.rad.z) & 0xffffu) | (s.kind << 16) | (cq << 18),
                              snorm16(ex) | (snorm16(ey) << 16), s.seed);
}

// unpackReservoir (restir.wgsl:73-84).
VRT_DI RSample load_res(const uint4* res, size_t p) {
  const uint4 a = res[2 * p], d = res[2 * p + 1];
  RSample s;
  s.pos = f3(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
  s.W = __uint_as_float(a.w);
  s.rad = f3(bits2f(d.x & 0xffffu), bits2f(d.x >> 16), bits2f(d.y & 0xffffu));
  s.kind = (d.y >> 16) & 3u;
  s.c = (float)((d.y >> 18) & 0xffu);
  s.n = oct_decode(unsnorm16(d.z & 0xffffu), unsnorm16(d.z >> 16));
  s.seed = d.w;
  return s;
}

VRT_DI float rlum(F3 c) { return (c.x * 0.2126f + c.y * 0.7152f) + c.z * 0.0722f; }   // restir.wgsl:90-92

// evalF (restir.wgsl:143-159): demodulated integrand without visibility;
// inverseSqrt(r2) is 1 / sqrt(r2).
VRT_DI F3 eval_f(const RSample& s, F3 x1, F3 n1) {
  if (s.kind == kSkPoint) {
    const F3 d = s.pos - x1;
    const float r2 = fmax_(dot3(d, d), 1e-4f);
    const F3 dir = d * (1.0f / __fsqrt_rn(r2));
    const float cos1 = dot3(n1, dir);
    const float cos2 = dot3(s.n, f3(-dir.x, -dir.y, -dir.z));
    if (cos1 <= 0.0f || cos2 <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    return s.rad * (((kInvPi * cos1) * cos2) / r2);
  }
  if (s.kind == kSkDir) {
    const float cos1 = dot3(n1, s.pos);
    if (cos1 <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    return s.rad * (kInvPi * cos1);
  }
  return f3(0.0f, 0.0f, 0.0f);
}
VRT_DI float eval_target(const RSample& s, F3 x1, F3 n1) { return rlum(eval_f(s, x1, n1)); }

// receiverPoint (restir.wgsl:127-137): the reconstruction ray meets the voxel
// face plane recovered by rounding (half to even) the dominant coordinate.
VRT_DI F3 receiver_point(F3 ro, F3 rd, float t, F3 n1) {
  const F3 approx = ro + rd * t;
  const int ax = fabsf(n1.x) > 0.5f ? 0 : (fabsf(n1.y) > 0.5f ? 1 : 2);
  const float ac = ax == 0 ? approx.x : (ax == 1 ? approx.y : approx.z);
  const float roA = ax == 0 ? ro.x : (ax == 1 ? ro.y : ro.z);
  const float rdA = ax == 0 ? rd.x : (ax == 1 ? rd.y : rd.z);
  if (fabsf(rdA) < 1e-4f) return approx;
  const float d = rintf(ac * kInvVoxel) * kVoxelSize;
  const float tp = (d - roA) / rdA;
  return tp > 0.0f ? ro + rd * tp : approx;
}

// surfaceAt (reuse_spatial.wgsl:111-114) / the temporal pass's x1.
VRT_DI F3 surface_at(const Uni& u, int qx, int qy, int W, int H, float4 g) {
  return receiver_point(f3(u.camPos[0], u.camPos[1], u.camPos[2]),
                        camera_ray(u, ((float)qx + 0.5f) / (float)W, ((float)qy + 0.5f) / (float)H), g.w,
                        f3(g.x, g.y, g.z));
}

struct RestirDev {
  DScene S;
  Uni u;
  int W, H;
  float fclamp;
  uint4* resA;              // working reservoirs (initial, then temporal merge)
  uint4* resB;              // post-spatial reservoirs = next frame's history
  uint2* direct;            // rgba16f pass-through radiance
  uint2* rad16;             // rgba16f radiance (demodulated)
  float4* rad32;            // optional fp32 copy of the radiance
  uint32_t* alb8;
  float4* gbuf;             // current G-buffer (n, t)
  const float4* gprev;      // previous frame's G-buffer
  unsigned long long* stats;
  float* dup;               // duplication score (dupmap.wgsl), read at the reprojected pixel
  const uint32_t* pairing;  // pairing textures (RF_PAIRED)
  const uint2* lights;      // emissive faces: x|y<<9|z<<18|face<<27, material (RF_UNIFIED)
  const float4* lightAlias; // acceptance, alias index, selection pdf, 0
  const uint32_t* lightGrid;// 34 words per brick cell (RF_LIGHTGRID)
};

VRT_DI bool rflag(const Uni& u, uint32_t f) { return (u.params2[0] & f) != 0u; }

// WGSL f32 -> u32 conversion: toward zero, saturating, NaN -> 0.
VRT_DI uint32_t utrunc_(float x) { return __float2uint_rz(x); }

VRT_DI bool occluded(const RestirDev& R, const uint32_t* occ, F3 o, F3 d, float maxT, DCount& cnt) {
  return trace<true>(R.S, occ, o, d, maxT, cnt).t >= 0.0f;
}

VRT_DI F3 fclamp3(const RestirDev& R, F3 v) {
  return R.fclamp <= 0.0f ? v : min3(v, f3(R.fclamp, R.fclamp, R.fclamp));
}

// ---------------------------------------------------------------------------
// emissive-face sampling for unified NEE (pathtrace.wgsl:37-199)
// ---------------------------------------------------------------------------
constexpr uint32_t kLgK = 16u, kLgStride = 2u + 2u * kLgK;
constexpr float kLgPCell = 0.75f;

struct LightPoint {
  F3 pos, n, Le;
  float pdfA;
};

// sampleGlobalLightIndex / globalLightPdf (pathtrace.wgsl:49-65)
VRT_DI uint32_t global_light_index(const RestirDev& R, uint32_t& rng) {
  const uint32_t count = R.u.params2[1];
  if (rflag(R.u, kRfLightPower)) {
    const float uLight = rand_(rng) * (float)count;
    const uint32_t base = min(utrunc_(uLight), count - 1u);
    const float frac = uLight - (float)base;
    const float4 rec = R.lightAlias[base];
    const uint32_t aliasLi = min(utrunc_(rec.y + 0.5f), count - 1u);
    return frac >= rec.x ? aliasLi : base;
  }
  return min(utrunc_(rand_(rng) * (float)count), count - 1u);
}
VRT_DI float global_light_pdf(const RestirDev& R, uint32_t li) {
  if (rflag(R.u, kRfLightPower)) return fmax_(R.lightAlias[li].z, 1e-8f);
  return 1.0f / (float)R.u.params2[1];
}

// pickLightIndex (pathtrace.wgsl:80-121): global distribution, or with
// RF_LIGHTGRID the 0.75 / 0.25 mixture of the receiver cell's top-K table and
// the global distribution, with its exact mixture pdf.
VRT_DI uint32_t pick_light(const RestirDev& R, F3 pos, uint32_t& rng, float& pdf) {
  if (!rflag(R.u, kRfLightGrid)) {
    const uint32_t li = global_light_index(R, rng);
    pdf = global_light_pdf(R, li);
    return li;
  }
  const int BG = R.S.BG;
  const float sc = kInvVoxel / (float)kBrick;
  const int bx = iclamp_(ifloor_(pos.x * sc), 0, BG - 1), by = iclamp_(ifloor_(pos.y * sc), 0, BG - 1),
            bz = iclamp_(ifloor_(pos.z * sc), 0, BG - 1);
  const uint32_t base = (uint32_t)(bx + by * BG + bz * BG * BG) * kLgStride;
  const uint32_t n = min(R.lightGrid[base], kLgK);
  const float wSum = __uint_as_float(R.lightGrid[base + 1u]);
  if (n == 0u || wSum <= 0.0f) {
    const uint32_t li = global_light_index(R, rng);
    pdf = global_light_pdf(R, li);
    return li;
  }
  uint32_t li;
  if (rand_(rng) < kLgPCell) {   // by cumulative weight over the cell's entries
    float r = rand_(rng) * wSum;
    li = R.lightGrid[base + 2u];
    for (uint32_t k = 0u; k < n; k++) {
      li = R.lightGrid[base + 2u + 2u * k];
      r = r - __uint_as_float(R.lightGrid[base + 3u + 2u * k]);
      if (r <= 0.0f) break;
    }
  } else {
    li = global_light_index(R, rng);
  }
  float pCell = 0.0f;
  for (uint32_t k = 0u; k < n; k++) {
    if (R.lightGrid[base + 2u + 2u * k] == li) {
      pCell = __uint_as_float(R.lightGrid[base + 3u + 2u * k]) / wSum;
      break;
    }
  }
  pdf = kLgPCell * pCell + (1.0f - kLgPCell) * global_light_pdf(R, li);
  return li;
}

// sampleLightFace (pathtrace.wgsl:123-144): a uniform point on the face.
VRT_DI LightPoint sample_light_face(const RestirDev& R, F3 shadePos, uint32_t& rng) {
  float pdfSelect;
  const uint32_t li = pick_light(R, shadePos, rng, pdfSelect);
  const uint2 l = R.lights[li];
  const F3 v = f3((float)(l.x & 0x1ffu), (float)((l.x >> 9) & 0x1ffu), (float)((l.x >> 18) & 0x1ffu));
  const uint32_t face = (l.x >> 27) & 7u, axis = face >> 1;
  const float side = (face & 1u) == 0u ? 1.0f : 0.0f;   // +side faces sit at v+1
  const float j0 = rand_(rng);
  const float j1 = rand_(rng);
  const float j2 = rand_(rng);
  F3 q = v + f3(j0, j1, j2);
  F3 n = f3(0.0f, 0.0f, 0.0f);
  const float sg = side > 0.5f ? 1.0f : -1.0f;
  if (axis == 0u) { q.x = v.x + side; n.x = sg; }
  else if (axis == 1u) { q.y = v.y + side; n.y = sg; }
  else { q.z = v.z + side; n.z = sg; }
  const Mat mat = unpack_material(l.y);
  LightPoint lp;
  lp.pos = q * kVoxelSize;
  lp.n = n;
  lp.Le = mat.albedo * (mat.emissive * kEmissiveScale);
  lp.pdfA = pdfSelect / (kVoxelSize * kVoxelSize);
  return lp;
}

// emissiveCandCount (pathtrace.wgsl:155-159)
VRT_DI uint32_t emissive_cand_count(const Uni& u, uint32_t bounce) {
  if (!rflag(u, kRfAdaptCand)) return bounce == 0u ? 4u : 1u;
  const float n0 =
      clamp_(rintf((u.params5[1] * 4.0f) * (1.0f + log2_(1.0f + (float)u.params2[1] / 256.0f))), 1.0f, 16.0f);
  return max(utrunc_(n0) >> min(bounce, 31u), 1u);
}

// emissiveNEE (pathtrace.wgsl:167-199): RIS over nCand light-face samples,
// one shadow ray on the survivor; the first valid candidate is taken
// without a draw.
VRT_DI F3 emissive_nee(const RestirDev& R, const uint32_t* occ, F3 pos, F3 n, F3 albedo, uint32_t nCand,
                       uint32_t& rng, DCount& cnt) {
  if (R.u.params2[1] == 0u) return f3(0.0f, 0.0f, 0.0f);
  const F3 surf = pos + n * 1e-3f;
  const float invM = 1.0f / (float)nCand;
  float wSum = 0.0f, selLum = 0.0f, selR2 = 0.0f;
  F3 sel = f3(0.0f, 0.0f, 0.0f), selDir = sel;
  for (uint32_t k = 0u; k < nCand; k++) {
    const LightPoint lp = sample_light_face(R, pos, rng);
    const F3 d = lp.pos - surf;
    const float r2 = fmax_(dot3(d, d), 1e-6f);
    const F3 dir = d * (1.0f / __fsqrt_rn(r2));
    const float cos1 = dot3(n, dir);
    const float cos2 = dot3(lp.n, f3(-dir.x, -dir.y, -dir.z));
    if (cos1 <= 0.0f || cos2 <= 0.0f) continue;
    const F3 a = ((albedo * kInvPi) * cos1) * cos2;
    const F3 v = f3((a.x / r2) * lp.Le.x / lp.pdfA, (a.y / r2) * lp.Le.y / lp.pdfA, (a.z / r2) * lp.Le.z / lp.pdfA);
    const float w = rlum(v) * invM;
    if (w <= 0.0f) continue;
    const bool first = wSum == 0.0f;
    wSum = wSum + w;
    if (first || rand_(rng) * wSum < w) {
      sel = v;
      selLum = rlum(v);
      selDir = dir;
      selR2 = r2;
    }
  }
  if (wSum <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
  const float r = __fsqrt_rn(selR2);
  if (occluded(R, occ, surf, selDir, r - 2e-3f, cnt)) return f3(0.0f, 0.0f, 0.0f);
  return sel * (wSum / selLum);
}

// estimateLo (pathtrace.wgsl:205-246): sun-cone NEE at every vertex,
// Russian roulette from vertex 2; emission rides on hits (unification off)
// or comes from light-list NEE at every vertex (RF_UNIFIED).
VRT_DI F3 estimate_lo(const RestirDev& R, const uint32_t* occ, F3 x2, F3 n2, Mat mat2, uint32_t& rng,
                      DCount& cnt) {
  const bool unified = rflag(R.u, kRfUnified);
  const Uni& u = R.u;
  F3 Lo = f3(0.0f, 0.0f, 0.0f), tp = f3(1.0f, 1.0f, 1.0f);
  F3 pos = x2, n = n2;
  Mat mat = mat2;
  const uint32_t nB = u.params0[1];
  const F3 sunRad = f3(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
  for (uint32_t v = 1u; v <= nB; v++) {
    if (!unified && mat.emissive > 0.0f && v > 1u) Lo = Lo + (tp * mat.albedo) * (mat.emissive * kEmissiveScale);
    const F3 surf = pos + n * 1e-3f;
    const F3 l = sample_sun_dir(u, rng);
    const float ndl = dot3(n, l);
    if (ndl > 0.0f && l.y > 0.0f && !occluded(R, occ, surf, l, 1e4f, cnt))
      Lo = Lo + (((tp * mat.albedo) * kInvPi) * ndl) * sunRad;
    if (unified) Lo = Lo + tp * emissive_nee(R, occ, pos, n, mat.albedo, emissive_cand_count(u, v), rng, cnt);
    if (v == nB) break;
    const F3 rd = cosine_hemisphere(n, rng);
    tp = tp * mat.albedo;
    if (v >= 2u) {
      const float p = clamp_(fmax_(tp.x, fmax_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rand_(rng) > p) break;
      tp = f3(tp.x / p, tp.y / p, tp.z / p);
    }
    const DHit h = trace<true>(R.S, occ, surf, rd, 1e4f, cnt);
    if (h.t < 0.0f) {
      Lo = Lo + tp * sky_color(u, rd, false);
      break;
    }
    pos = surf + rd * h.t;
    n = h.n;
    mat = unpack_material(h.mat);
  }
  return fclamp3(R, Lo);
}

// ---------------------------------------------------------------------------
// initial candidates (pathtrace.wgsl:248-284, 332-457)
// ---------------------------------------------------------------------------
// The bounce candidate when its ray escapes: a sky direction, W = 1/pdf_omega.
VRT_DI void cand_dir(const Uni& u, F3 n1, F3 brd, RSample& s, float& Wc) {
  s = null_sample(0.0f);
  s.kind = kSkDir;
  s.pos = brd;
  s.rad = sky_color(u, brd, false);
  Wc = kPi / fmax_(dot3(n1, brd), 1e-4f);
}

// The bounce candidate at reconnection vertex x2 carrying Lo (already
// clamped), W = 1/pdf in area measure.
VRT_DI void cand_point(F3 x1, F3 n1, F3 x2, F3 n2, F3 Lo, RSample& s, float& Wc) {
  s = null_sample(0.0f);
  s.kind = kSkPoint;
  s.pos = x2;
  s.n = n2;
  s.rad = Lo;
  const F3 d = x2 - x1;
  const float r2 = fmax_(dot3(d, d), 1e-6f);
  const F3 dn = normalize3(d);
  const float cos1 = fmax_(dot3(n1, dn), 1e-4f);
  const float cos2 = fmax_(dot3(n2, f3(-dn.x, -dn.y, -dn.z)), 1e-4f);
  Wc = ((kPi / cos1) * r2) / cos2;
}

// Streaming RIS of the initial candidates (pathtrace.wgsl:340-440).
struct Ris {
  float wSum = 0.0f, selP = 0.0f;
  RSample sel;
  VRT_DI void add(const RSample& s, float p, float w, uint32_t& rng) {
    if (w > 0.0f) {
      wSum = wSum + w;
      if (rand_(rng) * wSum < w) { sel = s; selP = p; }
    }
  }
};

// The reservoir record of pixel p after the initial RIS (pathtrace.wgsl:442-455).
VRT_DI void store_ris(uint4* resA, size_t p, const Uni& u, int W, int H, const Ris& ris) {
  RSample out = null_sample(0.0f);
  if (ris.sel.kind != kSkNone && ris.selP > 0.0f) {
    out = ris.sel;
    out.W = ris.wSum / ris.selP;
  }
  out.c = 1.0f;   // a failed candidate is a zero-valued outcome, confidence 1
  out.seed = pcg_hash((uint32_t)p + u.params0[0] * ((uint32_t)W * (uint32_t)H + 1u));
  store_res(resA, p, out);
}

// Initial RIS over the (at most one) bounce candidate (unification off).
VRT_DI void store_initial(uint4* resA, size_t p, const Uni& u, int W, int H, bool has, const RSample& s, float Wc,
                          F3 x1, F3 n1, uint32_t& rng) {
  Ris ris;
  ris.sel = null_sample(0.0f);
  if (has) {
    const float pt = eval_target(s, x1, n1);
    ris.add(s, pt, pt * Wc, rng);
  }
  store_ris(resA, p, u, W, H, ris);
}

VRT_DI void initial_pixel(const RestirDev& R, const uint32_t* occ, int gx, int gy, DCount& cnt) {
  const Uni& u = R.u;
  const size_t p = (size_t)gy * R.W + gx;
  uint32_t rng = init_rng((uint32_t)gx, (uint32_t)gy, u.params0[0]);
  const float jx = rand_(rng) - 0.5f;
  const float jy = rand_(rng) - 0.5f;
  const F3 ro = f3(u.camPos[0], u.camPos[1], u.camPos[2]);
  const F3 rd = camera_ray(u, (((float)gx + 0.5f) + jx) / (float)R.W, (((float)gy + 0.5f) + jy) / (float)R.H);
  const DHit h0 = trace<true>(R.S, occ, ro, rd, 1e4f, cnt);
  if (h0.t < 0.0f) {
    const F3 sky = sky_color(u, rd, true);
    const uint2 sk = pack_h4(sky.x, sky.y, sky.z, 1.0f);
    R.rad16[p] = sk;
    if (R.rad32) R.rad32[p] = make_float4(sky.x, sky.y, sky.z, 1.0f);
    R.direct[p] = sk;
    R.alb8[p] = 0xffffffffu;
    R.gbuf[p] = make_float4(-rd.x, -rd.y, -rd.z, -1.0f);
    R.resA[2 * p] = make_uint4(0u, 0u, 0u, 0u);
    R.resA[2 * p + 1] = make_uint4(0u, 0u, 0u, 0u);
    return;
  }
  const Mat mat1 = unpack_material(h0.mat);
  const F3 x1 = ro + rd * h0.t;
  const F3 n1 = h0.n;
  const F3 surf1 = x1 + n1 * fmax_(1e-3f, h0.t * 1e-4f);
  R.alb8[p] = unorm8_(__fsqrt_rn(mat1.albedo.x)) | (unorm8_(__fsqrt_rn(mat1.albedo.y)) << 8) |
              (unorm8_(__fsqrt_rn(mat1.albedo.z)) << 16) | (255u << 24);
  R.gbuf[p] = make_float4(n1.x, n1.y, n1.z, h0.t);

  const bool unified = rflag(u, kRfUnified);
  const float em = mat1.emissive * kEmissiveScale;
  F3 direct = f3(em, em, em);   // radiance that bypasses the reservoir
  Ris ris;
  ris.sel = null_sample(0.0f);
  {   // sun-cone NEE at x1: a direction candidate (unified) or pass-through radiance
    const F3 l = sample_sun_dir(u, rng);
    const float ndl = dot3(n1, l);
    if (ndl > 0.0f && l.y > 0.0f && !occluded(R, occ, surf1, l, 1e4f, cnt)) {
      if (unified) {
        const float coneSA = kTwoPi * (1.0f - u.sunDir[3]);
        RSample s = null_sample(0.0f);
        s.kind = kSkDir;
        s.pos = l;
        const float den = fmax_(coneSA, 1e-5f);
        s.rad = f3(u.sunRadiance[0] / den, u.sunRadiance[1] / den, u.sunRadiance[2] / den);
        const float pt = eval_target(s, x1, n1);
        ris.add(s, pt, pt * coneSA, rng);   // W = 1/pdf = cone solid angle
      } else {
        direct = direct + f3(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]) * (kInvPi * ndl);
      }
    }
  }
  if (unified && u.params2[1] > 0u) {   // light-list NEE at x1: RIS over emissive faces
    const uint32_t nCand = emissive_cand_count(u, 0u);
    float eSum = 0.0f, eSelP = 0.0f;
    RSample eSel = null_sample(0.0f);
    for (uint32_t k = 0u; k < nCand; k++) {
      const LightPoint lp = sample_light_face(R, x1, rng);
      RSample s = null_sample(0.0f);
      s.kind = kSkPoint;
      s.pos = lp.pos;
      s.n = lp.n;
      s.rad = lp.Le;
      const float pt = eval_target(s, x1, n1);
      const float w = pt / ((float)nCand * lp.pdfA);
      if (w > 0.0f) {
        eSum = eSum + w;
        if (rand_(rng) * eSum < w) { eSel = s; eSelP = pt; }
      }
    }
    if (eSel.kind != kSkNone && eSelP > 0.0f) {
      const F3 d = eSel.pos - surf1;
      const float r = __fsqrt_rn(dot3(d, d));
      if (!occluded(R, occ, surf1, f3(d.x / r, d.y / r, d.z / r), r - 2e-3f, cnt)) {
        const float We = eSum / eSelP;
        ris.add(eSel, eSelP, eSelP * We, rng);
      }
    }
  }
  if (u.params0[1] > 0u) {   // BSDF bounce candidate: reconnection vertex x2 carries Lo
    const F3 brd = cosine_hemisphere(n1, rng);
    const DHit h = trace<true>(R.S, occ, surf1, brd, 1e4f, cnt);
    RSample s;
    float Wc;
    if (h.t < 0.0f) {
      cand_dir(u, n1, brd, s, Wc);
    } else {
      const F3 x2 = surf1 + brd * h.t;
      const Mat mat2 = unpack_material(h.mat);
      F3 Lo = estimate_lo(R, occ, x2, h.n, mat2, rng, cnt);
      if (!unified && mat2.emissive > 0.0f) Lo = Lo + mat2.albedo * (mat2.emissive * kEmissiveScale);
      cand_point(x1, n1, x2, h.n, fclamp3(R, Lo), s, Wc);
    }
    const float pt = eval_target(s, x1, n1);
    ris.add(s, pt, pt * Wc, rng);
  }
  store_ris(R.resA, p, u, R.W, R.H, ris);
  R.direct[p] = pack_h4(direct.x, direct.y, direct.z, 1.0f);
}

template <bool kSmem>
__global__ void __launch_bounds__(256) k_restir_initial(const __grid_constant__ RestirDev R) {
  extern __shared__ uint32_t s_occ[];
  const uint32_t* occ = stage_occupancy<kSmem>(R.S, s_occ);
  int gx, gy;
  block_pixel_16x16(gx, gy);
  DCount cnt{0u, 0u, 0u, 0u};
  uint32_t pix = 0u;
  if (gx < R.W && gy < R.H) {
    initial_pixel(R, occ, gx, gy, cnt);
    pix = 1u;
  }
  if (R.stats) block_flush_stats(R.stats, cnt, pix);
}

// ---------------------------------------------------------------------------
// temporal reuse (reuse_temporal.wgsl:38-46, 140-279)
// ---------------------------------------------------------------------------
VRT_DI bool valid_prev(const RestirDev& R, int px, int py, F3 wp, F3 n1) {
  if (px < 0 || py < 0 || px >= R.W || py >= R.H) return false;
  const float4 pg = R.gprev[(size_t)py * R.W + px];
  if (pg.w <= 0.0f) return false;
  const F3 dv = wp - f3(R.u.prevCamPos[0], R.u.prevCamPos[1], R.u.prevCamPos[2]);
  const float expectedT = __fsqrt_rn(dot3(dv, dv));
  const bool depthOk = fabsf(pg.w - expectedT) < 0.08f * expectedT + 0.02f;
  const bool normalOk = dot3(f3(pg.x, pg.y, pg.z), n1) > 0.9f;
  return depthOk && normalOk;
}

// Five blocks per SM (48 registers) for the per-pixel reuse and wave kernels below:
// they wait on scattered reservoir, G-buffer and path-state reads (gi 2.87 -> 2.77 ms).
__global__ void __launch_bounds__(256, 5) k_restir_temporal(const __grid_constant__ RestirDev R) {
  int gx, gy;
  block_pixel_16x16(gx, gy);
  if (gx >= R.W || gy >= R.H) return;
  const Uni& u = R.u;
  const size_t p = (size_t)gy * R.W + gx;
  const float4 g = R.gbuf[p];
  if (g.w <= 0.0f) return;
  uint32_t rng = init_rng((uint32_t)gx, (uint32_t)gy, u.params0[0] ^ 0x5f356495u);
  const F3 n1 = f3(g.x, g.y, g.z);
  const F3 x1 = surface_at(u, gx, gy, R.W, R.H, g);
  float pc[4];
  matvec4(u.prevViewProj, x1.x, x1.y, x1.z, 1.0f, pc);
  if (pc[3] <= 0.0f) return;
  const float ndx = pc[0] / pc[3], ndy = pc[1] / pc[3];
  int ppx = itrunc_((ndx * 0.5f + 0.5f) * (float)R.W);
  int ppy = itrunc_(((-ndy) * 0.5f + 0.5f) * (float)R.H);
  bool found = valid_prev(R, ppx, ppy, x1, n1);
  if (!found && rflag(u, kRfRescue)) {   // disocclusion rescue: first validating 3x3 neighbour
    for (int dy = -1; dy <= 1 && !found; dy++)
      for (int dx = -1; dx <= 1 && !found; dx++)
        if ((dx != 0 || dy != 0) && valid_prev(R, ppx + dx, ppy + dy, x1, n1)) {
          ppx += dx;
          ppy += dy;
          found = true;
        }
  }
  if (!found) return;   // disocclusion: keep the fresh reservoir
  const RSample st = load_res(R.resB, (size_t)ppy * R.W + ppx);
  float cap = u.params3[0];
  if (rflag(u, kRfDupmap)) {   // duplication-adaptive confidence cap (Lin 2026 section 5)
    const float dupScore = clamp_(R.dup[(size_t)ppy * R.W + ppx], 0.0f, 1.0f);
    cap = mix_(u.params3[0], u.params3[1], pow_(dupScore, u.params3[2]));
  }
  const float cT = fmin_(st.c, cap);
  const RSample sc = load_res(R.resA, p);
  const float cC = fmax_(sc.c, 0.0f);
  const float pC = eval_target(sc, x1, n1), pT = eval_target(st, x1, n1);
  const float mDen = fmax_(cC + cT, 1e-3f);
  const float wC = ((cC / mDen) * pC) * fmax_(sc.W, 0.0f);
  const float wT = ((cT / mDen) * pT) * fmax_(st.W, 0.0f);
  const float wSum = wC + wT;
  if (wSum <= 0.0f) {   // pooled null keeps the merged confidence
    store_res(R.resA, p, null_sample(cC + cT));
    return;
  }
  RSample sel = sc;
  float selP = pC;
  if (rand_(rng) * wSum >= wC) { sel = st; selP = pT; }
  if (selP <= 0.0f) return;
  sel.W = wSum / selP;
  sel.c = cC + cT;
  store_res(R.resA, p, sel);
}

// ---------------------------------------------------------------------------
// spatial reuse + shading (reuse_spatial.wgsl:116-126, 128-354)
//
// Domains and candidates sit in fixed slots -- 0 the canonical pixel, k the
// k-th tap -- with validity flags instead of the reference's compacted
// arrays; every loop runs over the slots in increasing order and skips the
// invalid ones, so sums and RNG draws happen in the reference's order, and
// the arrays stay in registers.  A candidate's position in the compacted
// list (`rank`) decides whether its visibility is tested (rank > 0).  Each
// target evaluation serves the denominator, the MIS numerator (its own
// domain's term) and p-hat at the receiver (the canonical domain's term).
// ---------------------------------------------------------------------------
struct SpatialPick {
  bool ok;          // a sample was selected (else: pooled null)
  bool vis_test;    // its visibility must be tested (a neighbour's sample, or RF_FULLV)
  RSample sel;      // the selected sample with W and pooled confidence
  float cTotal;
  F3 vcontrib;      // RF_VECTOR: the summed per-candidate contributions (deferred: those without a ray)
  int nrays;        // RF_VECTOR, deferred: visibility rays left pending
};

// Deferred RF_VECTOR terms of path g: term j (candidate slot j) in
// T[j][g] = (contribution, code): code 0 no term, 1 visible without a ray,
// 2 + k visible iff ray slot k (path g + k P) is unoccluded.
struct VecSink {
  float4* T[4];     // S0, S1, S2, R1 of the wavefront scratch
  float4* R0;
  float4* R2;
  uint32_t g, P;
};

// pairSize / pairOff / wrapMod / pairedPartner (reuse_spatial.wgsl:65-109):
// the mutual partner of pixel (px, py) in pairing texture ti, varied per
// frame by a hashed offset, mirror and swap; the pixel itself when the
// partner falls off the image (rejected by the caller's bounds test).
VRT_DI int wrap_mod(int v, int sz) { return ((v % sz) + sz) % sz; }

// Texture ti of size kSz at word offset kOff; the sizes are compile-time
// constants so that the modulos reduce to multiplies.
template <int kSz, uint32_t kOff>
VRT_DI void paired_partner_sz(const RestirDev& R, int px, int py, uint32_t ti, int& qx, int& qy) {
  const uint32_t h = pcg_hash(R.u.params0[0] * 2654435761u + ti * 0x68bc21ebu + 0x9e3779b9u);
  const uint32_t h2 = pcg_hash(h);
  const int ox = (int)(h % (uint32_t)kSz), oy = (int)(h2 % (uint32_t)kSz);
  const bool mx = (h & 0x40000000u) != 0u, my = (h & 0x20000000u) != 0u, sw = (h & 0x10000000u) != 0u;
  int ax = wrap_mod(px + ox, kSz), ay = wrap_mod(py + oy, kSz);
  if (sw) { const int t = ax; ax = ay; ay = t; }
  if (mx) ax = kSz - 1 - ax;
  if (my) ay = kSz - 1 - ay;
  const uint32_t word = R.pairing[kOff + (uint32_t)(ay * kSz + ax)];
  const int dtx = (int)(word << 16) >> 16, dty = (int)word >> 16;
  int bx = wrap_mod(ax + dtx, kSz), by = wrap_mod(ay + dty, kSz);
  if (mx) bx = kSz - 1 - bx;
  if (my) by = kSz - 1 - by;
  if (sw) { const int t = bx; bx = by; by = t; }
  int dx = wrap_mod(bx - ox - px, kSz), dy = wrap_mod(by - oy - py, kSz);
  if (dx > kSz / 2) dx -= kSz;
  if (dy > kSz / 2) dy -= kSz;
  qx = px + dx;
  qy = py + dy;
}

// The texture index is the same for every pixel of a pass (it depends on
// the tap and the flags only), so the branch is uniform.
VRT_DI void paired_partner(const RestirDev& R, int px, int py, uint32_t ti, int& qx, int& qy) {
  if (ti == 0u) paired_partner_sz<254, 0u>(R, px, py, ti, qx, qy);
  else if (ti == 1u) paired_partner_sz<230, 64516u>(R, px, py, ti, qx, qy);
  else paired_partner_sz<210, 117416u>(R, px, py, ti, qx, qy);
}

// footprintOK (restir.wgsl:172-180)
VRT_DI bool footprint_ok(const Uni& u, const RSample& s, F3 x1, F3 n1, float tPrim, float cosView) {
  if (s.kind != kSkPoint) return true;
  const F3 d = s.pos - x1;
  const float r2 = dot3(d, d);
  const F3 dir = d * (1.0f / __fsqrt_rn(fmax_(r2, 1e-8f)));
  const float cos1 = fmax_(dot3(n1, dir), 0.0f);
  const float cos2 = fmax_(dot3(s.n, f3(-dir.x, -dir.y, -dir.z)), 0.0f);
  return r2 >= ((((u.params3[3] * tPrim) * tPrim) * cos1) * cos2) / fmax_(cosView, 0.05f);
}

// The shadow ray of sampleVisible (reuse_spatial.wgsl:117-126); false when
// the sample is closer than 2 mm (visible without a ray).
VRT_DI bool visibility_ray(const RSample& s, F3 x1, F3 n1, F3& o, F3& d, float& maxT) {
  o = x1 + n1 * 1e-3f;
  if (s.kind == kSkDir) {
    d = s.pos;
    maxT = 1e4f;
    return true;
  }
  const F3 v = s.pos - o;
  const float r = __fsqrt_rn(dot3(v, v));
  if (r < 2e-3f) return false;
  d = f3(v.x / r, v.y / r, v.z / r);
  maxT = r - 2e-3f;
  return true;
}

VRT_DI bool sample_visible(const RestirDev& R, const uint32_t* occ, const RSample& s, F3 x1, F3 n1, DCount& cnt) {
  F3 o, d;
  float maxT;
  if (!visibility_ray(s, x1, n1, o, d, maxT)) return true;
  return !occluded(R, occ, o, d, maxT, cnt);
}

// Neighbour selection, confidence-weighted balance-heuristic resampling and
// (RF_VECTOR, kTraceHere only) the vector-valued shading sum of pixel (gx, gy).
template <bool kTraceHere, bool kVector>
VRT_DI SpatialPick spatial_pick(const RestirDev& R, const uint32_t* occ, DCount& cnt, int gx, int gy, float4 g, F3 x1,
                                F3 n1, const VecSink* sink) {
  const Uni& u = R.u;
  const size_t p = (size_t)gy * R.W + gx;
  uint32_t rng = init_rng((uint32_t)gx, (uint32_t)gy, u.params0[0] ^ 0x2c1b3c6du);
  const float tPrim = g.w;
  const bool footprint = rflag(u, kRfFootprint);
  float cosView = 0.0f;
  if (footprint) cosView = fmax_(dot3(n1, normalize3(f3(u.camPos[0], u.camPos[1], u.camPos[2]) - x1)), 0.0f);
  F3 dx[4], dn[4];
  float dc[4];
  uint32_t qi[4];
  bool dok[4], cok[4];
  dx[0] = x1;
  dn[0] = n1;
  qi[0] = (uint32_t)p;
  {
    const uint4 d0 = R.resA[2 * p + 1];
    dc[0] = (float)((d0.y >> 18) & 0xffu);
    dok[0] = true;
    cok[0] = ((d0.y >> 16) & 3u) != kSkNone;
  }
  const uint32_t taps = rflag(u, kRfSpatial) ? min(u.params2[2], 3u) : 0u;
  const bool paired = rflag(u, kRfPaired), plane = rflag(u, kRfPlane);
#pragma unroll
  for (int k = 1; k < 4; k++) {
    dok[k] = cok[k] = false;
    dc[k] = 0.0f;
    qi[k] = 0u;
    dx[k] = dn[k] = f3(0.0f, 0.0f, 0.0f);
    const uint32_t ti = (uint32_t)k - 1u;
    if (ti >= taps) continue;
    int qx, qy;
    if (paired) {
      // RF_MIXSIGMA: the last tap reads the wide-sigma texture 0, the others shift up
      uint32_t tex = ti;
      if (rflag(u, kRfMixSigma)) tex = ti + 1u == taps ? 0u : ti + 1u;
      paired_partner(R, gx, gy, tex, qx, qy);
    } else {   // classic random neighbour in a uniform disk of radius params4.x
      const float r = u.params4[0] * __fsqrt_rn(rand_(rng));
      const float a = kTwoPi * rand_(rng);
      float sa, ca;
      sincos_(a, sa, ca);
      qx = gx + itrunc_(ca * r);
      qy = gy + itrunc_(sa * r);
    }
    if ((qx == gx && qy == gy) || qx < 0 || qy < 0 || qx >= R.W || qy >= R.H) continue;
    const size_t q = (size_t)qy * R.W + qx;
    const float4 gq = R.gbuf[q];
    if (gq.w <= 0.0f) continue;
    const F3 nq = f3(gq.x, gq.y, gq.z);
    const float nDot = dot3(n1, nq);
    const bool genericOk = nDot > 0.9f && fabsf(gq.w - g.w) < 0.1f * g.w + 0.02f;
    F3 x1q = f3(0.0f, 0.0f, 0.0f);
    bool ok = genericOk;
    if (plane) {   // same voxel face plane, regardless of depth
      x1q = surface_at(u, qx, qy, R.W, R.H, gq);
      ok = genericOk || (nDot > 0.99f && fabsf(dot3(n1, x1q - x1)) < 0.02f);
    }
    if (!ok) continue;
    const uint4 dq = R.resA[2 * q + 1];
    const bool nonnull = ((dq.y >> 16) & 3u) != kSkNone;
    if (footprint && nonnull && !footprint_ok(u, load_res(R.resA, q), x1, n1, tPrim, cosView)) continue;
    dx[k] = plane ? x1q : surface_at(u, qx, qy, R.W, R.H, gq);
    dn[k] = nq;
    dc[k] = (float)((dq.y >> 18) & 0xffu);
    qi[k] = (uint32_t)q;
    dok[k] = true;
    cok[k] = nonnull;
  }
  SpatialPick pk;
  pk.cTotal = 0.0f;
  pk.vcontrib = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int l = 0; l < 4; l++)
    if (dok[l]) pk.cTotal = pk.cTotal + dc[l];
  const bool vector = kVector;
  const bool fullV = rflag(u, kRfFullV);
  float wSum = 0.0f, selP = 0.0f;
  int rank = 0, selRank = 0;
  pk.sel = null_sample(0.0f);
  pk.nrays = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    F3 vterm = f3(0.0f, 0.0f, 0.0f);
    uint32_t vcode = 0u;
    if (cok[j]) {
      const RSample s = load_res(R.resA, qi[j]);
      float denom = 0.0f, num = 0.0f, pMe = 0.0f;   // balance heuristic over all domains
#pragma unroll
      for (int l = 0; l < 4; l++) {
        if (!dok[l]) continue;
        const float e = eval_target(s, dx[l], dn[l]);
        const float term = dc[l] * e;
        denom = denom + term;
        if (l == j) num = term;
        if (l == 0) pMe = e;
      }
      if (denom > 0.0f) {
        const float m = num / denom;
        const float w = (m * pMe) * fmax_(s.W, 0.0f);
        if (w > 0.0f) {
          wSum = wSum + w;
          if (rand_(rng) * wSum < w) { pk.sel = s; selP = pMe; selRank = rank; }
        }
        if (vector && w > 0.0f) {   // vector-valued shading weight with per-candidate visibility
          const bool test = rank > 0 || fullV;
          if (kTraceHere) {
            if (!test || sample_visible(R, occ, s, x1, n1, cnt))
              pk.vcontrib = pk.vcontrib + eval_f(s, x1, n1) * (m * fmax_(s.W, 0.0f));
          } else {
            vterm = eval_f(s, x1, n1) * (m * fmax_(s.W, 0.0f));
            vcode = 1u;
            F3 o, d;
            float mt;
            if (test && visibility_ray(s, x1, n1, o, d, mt)) {
              const uint32_t gk = sink->g + (uint32_t)pk.nrays * sink->P;
              sink->R0[gk] = make_float4(o.x, o.y, o.z, 0.0f);
              sink->R2[gk] = make_float4(d.x, d.y, d.z, mt);
              vcode = 2u + (uint32_t)pk.nrays;
              pk.nrays++;
            } else {
              pk.vcontrib = pk.vcontrib + vterm;
            }
          }
        }
      }
      rank++;
    }
    if (!kTraceHere && vector) sink->T[j][sink->g] = make_float4(vterm.x, vterm.y, vterm.z, __uint_as_float(vcode));
  }
  pk.ok = pk.sel.kind != kSkNone && selP > 0.0f && wSum > 0.0f;
  pk.vis_test = selRank > 0 || fullV;
  if (pk.ok) {
    pk.sel.W = wSum / selP;
    pk.sel.c = fmin_(pk.cTotal, 255.0f);
  }
  return pk;
}

VRT_DI void out_radiance(const RestirDev& R, size_t p, F3 v) {
  R.rad16[p] = pack_h4(v.x, v.y, v.z, 1.0f);
  if (R.rad32) R.rad32[p] = make_float4(v.x, v.y, v.z, 1.0f);
}

VRT_DI F3 load_direct(const RestirDev& R, size_t p) {
  const float4 dr = unpack_h4(R.direct[p]);
  return f3(dr.x, dr.y, dr.z);
}

// RF_CLAMP: luminance clamp of the reservoir contribution (params4.z).
VRT_DI F3 clamp_contrib(const Uni& u, F3 c) {
  if (!rflag(u, kRfClamp)) return c;
  const float l = rlum(c);
  return l > u.params4[2] ? c * (u.params4[2] / l) : c;
}

// Next frame's history record: the post-spatial sample, or with
// RF_HISTISOLATE the pre-spatial (temporal) reservoir.
VRT_DI void store_history(const RestirDev& R, size_t p, const RSample& s) {
  if (rflag(R.u, kRfHistIsolate)) {
    R.resB[2 * p] = R.resA[2 * p];
    R.resB[2 * p + 1] = R.resA[2 * p + 1];
  } else {
    store_res(R.resB, p, s);
  }
}

// Selection, record and (unless visibility rays are left pending) radiance
// of pixel (gx, gy).  kTraceHere: every visibility ray is traced in place.
// Otherwise returns the number of pending rays: the scalar weight's single ray
// in o / d / maxT gating contrib (clamped after the test), or RF_VECTOR's
// rays and terms written through `sink`.
template <bool kTraceHere, bool kVector>
VRT_DI int spatial_pixel(const RestirDev& R, const uint32_t* occ, DCount& cnt, int gx, int gy, F3& o, F3& d,
                         float& maxT, F3& contrib, const VecSink* sink) {
  const size_t p = (size_t)gy * R.W + gx;
  const F3 direct = load_direct(R, p);
  const float4 g = R.gbuf[p];
  if (g.w <= 0.0f) {   // sky: direct carries the analytic sky radiance
    out_radiance(R, p, direct);
    R.resB[2 * p] = make_uint4(0u, 0u, 0u, 0u);
    R.resB[2 * p + 1] = make_uint4(0u, 0u, 0u, 0u);
    return 0;
  }
  const F3 x1 = surface_at(R.u, gx, gy, R.W, R.H, g);
  const F3 n1 = f3(g.x, g.y, g.z);
  const SpatialPick pk = spatial_pick<kTraceHere, kVector>(R, occ, cnt, gx, gy, g, x1, n1, sink);
  if (!pk.ok) {   // pooled null
    out_radiance(R, p, direct);
    store_history(R, p, null_sample(fmin_(pk.cTotal, 255.0f)));
    return 0;
  }
  store_history(R, p, pk.sel);
  if (kVector) {
    if (!kTraceHere && pk.nrays > 0) return pk.nrays;
    out_radiance(R, p, direct + clamp_contrib(R.u, pk.vcontrib));
    return 0;
  }
  contrib = eval_f(pk.sel, x1, n1) * pk.sel.W;
  if (pk.vis_test && visibility_ray(pk.sel, x1, n1, o, d, maxT)) {
    if (!kTraceHere) return 1;
    if (occluded(R, occ, o, d, maxT, cnt)) contrib = f3(0.0f, 0.0f, 0.0f);
  }
  out_radiance(R, p, direct + clamp_contrib(R.u, contrib));
  return 0;
}

// Fused form (megakernel sessions): rays traced in place.
template <bool kSmem>
__global__ void __launch_bounds__(256) k_restir_spatial(const __grid_constant__ RestirDev R) {
  extern __shared__ uint32_t s_occ[];
  const uint32_t* occ = stage_occupancy<kSmem>(R.S, s_occ);
  int gx, gy;
  block_pixel_16x16(gx, gy);
  DCount cnt{0u, 0u, 0u, 0u};
  if (gx < R.W && gy < R.H) {
    F3 o, d, contrib;
    float maxT;
    if (rflag(R.u, kRfVector)) spatial_pixel<true, true>(R, occ, cnt, gx, gy, o, d, maxT, contrib, nullptr);
    else spatial_pixel<true, false>(R, occ, cnt, gx, gy, o, d, maxT, contrib, nullptr);
  }
  if (R.stats) block_flush_stats(R.stats, cnt, 0u);
}

// Split form (wavefront sessions): selection here; the pending visibility
// rays (ray k of pixel g traced as path g + k P: origin R0, direction and
// maxT R2) go to the persistent tracer's queue, the pixels with rays to the
// active list; k_restir_spatial_resolve then sums the terms whose rays were
// unoccluded.  Terms: the scalar weight's gated contribution in S1 (code 2),
// RF_VECTOR's per-candidate terms in S0, S1, S2, R1 (VecSink codes).
// Three blocks per SM (80 registers): the neighbour reads are scattered and the
// kernel waits on them; ours 5.20 -> 5.12 ms per frame against 2 blocks at 101
// registers (4 blocks at 64 registers: the same time, more spilling).
template <bool kVector>
__global__ void __launch_bounds__(256, 3) k_restir_spatial_select(const __grid_constant__ RestirDev R, WfDev b,
                                                               int wave) {
  int gx, gy;
  block_pixel_16x16(gx, gy);
  const uint32_t P = (uint32_t)R.W * (uint32_t)R.H;
  const bool in = gx < R.W && gy < R.H;
  const uint32_t g = in ? (uint32_t)gy * (uint32_t)R.W + (uint32_t)gx : 0u;
  const VecSink sink{{b.S0, b.S1, b.S2, b.R1}, b.R0, b.R2, g, P};
  F3 o, d, contrib;
  float maxT;
  DCount cnt{0u, 0u, 0u, 0u};
  const int nr = in ? spatial_pixel<false, kVector>(R, nullptr, cnt, gx, gy, o, d, maxT, contrib, &sink) : 0;
  if (nr > 0 && !kVector) {   // the scalar weight's ray, slot 0
    b.R0[g] = make_float4(o.x, o.y, o.z, 0.0f);
    b.R2[g] = make_float4(d.x, d.y, d.z, maxT);
    b.S1[g] = make_float4(contrib.x, contrib.y, contrib.z, __uint_as_float(2u));
  }
  uint32_t fs, bs, as;
  int* c = b.ctr + 4 * wave;
  block_append(c, c + 3, c + 2, nr, 0, nr > 0, fs, bs, as);
  uint32_t* q = queue_of(b, wave);
  for (int k = 0; k < nr; k++) q[fs + (uint32_t)k] = (g + (uint32_t)k * P) | kShadowBit;
  if (nr > 0) active_of(b, wave)[as] = g;
}

__global__ void __launch_bounds__(256) k_restir_spatial_resolve(const __grid_constant__ RestirDev R, WfDev b,
                                                                int wave) {
  const int n = b.ctr[4 * wave + 2];
  const uint32_t* list = active_of(b, wave);
  const uint32_t P = (uint32_t)R.W * (uint32_t)R.H;
  const bool vector = rflag(R.u, kRfVector);
  const float4* T[4] = {b.S0, b.S1, b.S2, b.R1};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t g = list[i];
    F3 contrib = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (!vector && j != 1) continue;   // the scalar weight keeps its single term in S1
      const float4 t = T[j][g];
      const uint32_t code = __float_as_uint(t.w);
      if (code == 1u || (code >= 2u && b.hit[g + (code - 2u) * P].w == 0u)) contrib = contrib + f3(t.x, t.y, t.z);
    }
    out_radiance(R, g, load_direct(R, g) + clamp_contrib(R.u, contrib));
  }
}

// dupmap.wgsl: share of the 9x9 window (centre excluded) whose reservoirs B
// carry the same initial candidate (seed) as this pixel's.  The block's
// 16 x 16 tile and its 4-pixel halo are staged in shared memory as (seed,
// non-null) pairs; the count is an integer, so the window order is free.
__global__ void __launch_bounds__(256) k_restir_dupmap(const __grid_constant__ RestirDev R) {
  constexpr int kHalo = 4, kT = 16 + 2 * kHalo;
  __shared__ uint32_t s_seed[kT * kT];
  __shared__ uint8_t s_live[kT * kT];
  const int x0 = blockIdx.x * 16 - kHalo, y0 = blockIdx.y * 16 - kHalo;
  for (int i = threadIdx.x; i < kT * kT; i += blockDim.x) {
    const int qx = x0 + i % kT, qy = y0 + i / kT;
    uint32_t seed = 0u, live = 0u;
    if (qx >= 0 && qy >= 0 && qx < R.W && qy < R.H) {
      const uint4 d = R.resB[2 * ((size_t)qy * R.W + qx) + 1];
      seed = d.w;
      live = ((d.y >> 16) & 3u) != kSkNone ? 1u : 0u;
    }
    s_seed[i] = seed;
    s_live[i] = (uint8_t)live;
  }
  __syncthreads();
  int gx, gy;
  block_pixel_16x16(gx, gy);
  if (gx >= R.W || gy >= R.H) return;
  const int c = (gy - y0) * kT + (gx - x0);
  float score = 0.0f;
  if (s_live[c]) {
    const uint32_t mine = s_seed[c];
    int count = 0;
    for (int dy = -kHalo; dy <= kHalo; dy++)
      for (int dx = -kHalo; dx <= kHalo; dx++) {
        const int k = c + dy * kT + dx;
        count += ((dx | dy) != 0 && s_live[k] && s_seed[k] == mine) ? 1 : 0;
      }
    score = (float)count / 80.0f;
  }
  R.dup[(size_t)gy * R.W + gx] = score;
}

// ---------------------------------------------------------------------------
// wavefront form of the initial pass.  The candidate path has the plain
// path's ray structure -- primary hit x1, sun shadow + bounce at x1, then
// estimateLo's vertices x2, x3, ... with a sun shadow each -- so it runs on
// the wavefront tracer's waves with its own shading kernels:
//   shade(0): G-buffer, albedo, x1's sun sample (pass-through radiance) and
//             bounce direction;
//   shade(1): x1's shadow resolves the pass-through radiance (stored); the
//             bounce hit is x2 (stored with its normal) or the sky (a
//             direction candidate, finished here); x2 is shaded as
//             estimateLo's vertex 1 (no emission pickup there);
//   shade(k): estimateLo's vertex k (shade_vertex: emission, sun sample,
//             Russian roulette from vertex 2, bounce);
// and a finished path builds its candidate and writes reservoir A.  Per-path
// state lives in the tracer's buffers (Lo in the radiance slot, throughput,
// RNG); x1 is rebuilt from the G-buffer and the primary ray (recomputed from
// the pixel's RNG stream).  Every draw and sum is the megakernel's, in the
// same order, so the records are bit-identical to it.
// ---------------------------------------------------------------------------
struct RestirWf {
  uint4* resA;
  uint2* direct;
  float4* x2;     // per path: reconnection vertex x2 (xyz), code of its normal (w bits; unified: + state bits)
  int W, H;
  // unified (RF_UNIFIED) path state: the initial RIS at x1 across its waves
  float4* selPW;  // selected candidate's position / direction, RIS weight sum
  float4* selRP;  // its radiance, its target p-hat
  float4* aux;    // light-list candidate's position and weight sum (x1), or the pending NEE term (x2...)
  float4* aux2;   // light-list candidate's radiance and p-hat
};

// Exact code of a DDA normal (components +-0 or +-1): sign and magnitude
// bits per component, so that signed zeros survive the round trip.
VRT_DI uint32_t normal_code(F3 n) {
  const float c[3] = {n.x, n.y, n.z};
  uint32_t code = 0u;
#pragma unroll
  for (int i = 0; i < 3; i++)
    code |= ((__float_as_uint(c[i]) >> 31) | ((c[i] != 0.0f ? 1u : 0u) << 1)) << (2 * i);
  return code;
}
VRT_DI F3 normal_decode(uint32_t code) {
  float c[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const uint32_t b = (code >> (2 * i)) & 3u;
    c[i] = __uint_as_float(((b & 1u) << 31) | ((b & 2u) ? 0x3f800000u : 0u));
  }
  return f3(c[0], c[1], c[2]);
}

// Primary ray direction of pixel (gx, gy): the first two draws of its stream
// are the sub-pixel jitter (pathtrace.wgsl:255-262).
VRT_DI F3 primary_dir(const Uni& u, uint32_t gx, uint32_t gy, int W, int H) {
  uint32_t rng = init_rng(gx, gy, u.params0[0]);
  const float jx = rand_(rng) - 0.5f;
  const float jy = rand_(rng) - 0.5f;
  return camera_ray(u, (((float)gx + 0.5f) + jx) / (float)W, (((float)gy + 0.5f) + jy) / (float)H);
}

// Candidate at the end of estimateLo: Lo (unclamped), x2's material; x1
// from the G-buffer.
VRT_DI void finish_point(const SingleJob& job, const RestirWf& r, uint32_t g, F3 Lo, uint32_t mat2bits, F3 x2, F3 n2,
                         uint32_t& rng) {
  const Uni& u = job.u;
  const float fc = job.fclamp;
  auto clampf3 = [&](F3 v) { return fc <= 0.0f ? v : min3(v, f3(fc, fc, fc)); };
  Lo = clampf3(Lo);
  const Mat mat2 = unpack_material(mat2bits);
  if (mat2.emissive > 0.0f) Lo = Lo + mat2.albedo * (mat2.emissive * kEmissiveScale);
  const float4 gb = job.out.gbuf[g];
  const F3 n1 = f3(gb.x, gb.y, gb.z);
  const uint32_t gx = g % (uint32_t)r.W, gy = g / (uint32_t)r.W;
  const F3 x1 = f3(u.camPos[0], u.camPos[1], u.camPos[2]) + primary_dir(u, gx, gy, r.W, r.H) * gb.w;
  RSample s;
  float Wc;
  cand_point(x1, n1, x2, n2, clampf3(Lo), s, Wc);
  store_initial(r.resA, g, u, r.W, r.H, true, s, Wc, x1, n1, rng);
}

__global__ void __launch_bounds__(256) k_wf_restir_primary(const __grid_constant__ SingleJob job, RestirWf r,
                                                           uint32_t P, WfDev b, unsigned long long* stats) {
  const uint32_t stride = gridDim.x * blockDim.x;
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats + kStatPixels, (unsigned long long)P);
  const Uni& u = job.u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < P; base += stride) {
    const uint32_t g = base + threadIdx.x;
    bool shadow = false, bounce = false, keep = false;
    if (g < P) {
      const uint4 h = b.hit[g];
      const F3 rd = xyz(b.R1[g]);
      const float t = __uint_as_float(h.x);
      if (t < 0.0f) {
        const F3 sky = sky_color(u, rd, true);
        const uint2 sk = pack_h4(sky.x, sky.y, sky.z, 1.0f);
        job.out.rad16[g] = sk;
        if (job.out.rad32) job.out.rad32[g] = make_float4(sky.x, sky.y, sky.z, 1.0f);
        r.direct[g] = sk;
        job.out.alb8[g] = 0xffffffffu;
        job.out.gbuf[g] = make_float4(-rd.x, -rd.y, -rd.z, -1.0f);
        r.resA[2 * (size_t)g] = make_uint4(0u, 0u, 0u, 0u);
        r.resA[2 * (size_t)g + 1] = make_uint4(0u, 0u, 0u, 0u);
      } else {
        const Mat mat1 = unpack_material(h.y);
        const F3 x1 = f3(u.camPos[0], u.camPos[1], u.camPos[2]) + rd * t;
        const F3 n1 = hit_normal((int)h.z, rd);
        job.out.alb8[g] = unorm8_(__fsqrt_rn(mat1.albedo.x)) | (unorm8_(__fsqrt_rn(mat1.albedo.y)) << 8) |
                          (unorm8_(__fsqrt_rn(mat1.albedo.z)) << 16) | (255u << 24);
        job.out.gbuf[g] = make_float4(n1.x, n1.y, n1.z, t);
        uint32_t rng = __float_as_uint(b.S0[g].w);
        const F3 surf1 = x1 + n1 * fmax_(1e-3f, t * 1e-4f);
        const F3 l = sample_sun_dir(u, rng);
        const float ndl = dot3(n1, l);
        shadow = ndl > 0.0f && l.y > 0.0f;
        F3 sunc = f3(0.0f, 0.0f, 0.0f);
        uint32_t flags = 0u;
        if (shadow) {
          sunc = f3(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]) * (kInvPi * ndl);
          flags |= kFlagShadow;
          b.R2[g] = make_float4(l.x, l.y, l.z, 1e4f);
        }
        bounce = u.params0[1] > 0u;
        if (bounce) {
          const F3 brd = cosine_hemisphere(n1, rng);
          b.R1[g] = make_float4(brd.x, brd.y, brd.z, 0.0f);
        } else {
          flags |= kFlagTerminal;
        }
        keep = shadow || bounce;
        if (keep) {
          b.R0[g] = make_float4(surf1.x, surf1.y, surf1.z, 0.0f);
          b.S0[g] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng));
          b.S1[g] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(h.y));
          b.S2[g] = make_float4(sunc.x, sunc.y, sunc.z, __uint_as_float(flags));
        } else {   // no sun sample, no bounce: emission only, null reservoir
          const float em = mat1.emissive * kEmissiveScale;
          r.direct[g] = pack_h4(em, em, em, 1.0f);
          store_initial(r.resA, g, u, r.W, r.H, false, null_sample(0.0f), 0.0f, x1, n1, rng);
        }
      }
    }
    emit_block(b, 1, g, shadow, bounce, keep);
  }
}

__global__ void __launch_bounds__(256, 5) k_wf_restir_wave(const __grid_constant__ SingleJob job, RestirWf r, WfDev b,
                                                        int wave) {
  const int n = b.ctr[4 * wave + 2];
  const uint32_t* list = active_of(b, wave);
  const Uni& u = job.u;
  const uint32_t nB = u.params0[1];
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int i = base + threadIdx.x;
    bool shadow = false, bounce = false, keep = false;
    uint32_t g = 0u;
    if (i < n) {
      g = list[i];
      const float4 s0 = b.S0[g];
      const float4 s1 = b.S1[g];
      const float4 s2 = b.S2[g];
      const uint4 h = b.hit[g];
      F3 Lo = xyz(s0), tp = xyz(s1);
      uint32_t rng = __float_as_uint(s0.w);
      const uint32_t flags = __float_as_uint(s2.w);
      const bool lit = (flags & kFlagShadow) && h.w == 0u;
      const bool terminal = (flags & kFlagTerminal) != 0u;
      if (wave == 1) {
        // x1's sun shadow resolved: the pass-through radiance is complete
        const float em = unpack_material(__float_as_uint(s1.w)).emissive * kEmissiveScale;
        F3 direct = f3(em, em, em);
        if (lit) direct = direct + xyz(s2);
        r.direct[g] = pack_h4(direct.x, direct.y, direct.z, 1.0f);
        const float4 gb = job.out.gbuf[g];
        const F3 n1 = f3(gb.x, gb.y, gb.z);
        if (terminal) {   // no bounce candidate (0 bounces)
          store_initial(r.resA, g, u, r.W, r.H, false, null_sample(0.0f), 0.0f, f3(0.0f, 0.0f, 0.0f), n1, rng);
        } else {
          const F3 brd = xyz(b.R1[g]);
          const float t = __uint_as_float(h.x);
          if (t < 0.0f) {   // escaped: a sky direction candidate (x1 unused by its target)
            RSample s;
            float Wc;
            cand_dir(u, n1, brd, s, Wc);
            store_initial(r.resA, g, u, r.W, r.H, true, s, Wc, f3(0.0f, 0.0f, 0.0f), n1, rng);
          } else {
            const F3 x2 = xyz(b.R0[g]) + brd * t;
            const F3 n2 = hit_normal((int)h.z, brd);
            r.x2[g] = make_float4(x2.x, x2.y, x2.z, __uint_as_float(normal_code(n2)));
            Mat m2 = unpack_material(h.y);
            m2.emissive = 0.0f;   // estimateLo picks up emission from vertex 2 on
            Lo = f3(0.0f, 0.0f, 0.0f);
            tp = f3(1.0f, 1.0f, 1.0f);
            keep = shade_vertex(u, b, g, 1u, x2, n2, m2, Lo, tp, rng, h.y, shadow, bounce, nB, nullptr);
            if (!keep) finish_point(job, r, g, Lo, h.y, x2, n2, rng);
          }
        }
      } else {
        if (lit) Lo = Lo + xyz(s2);
        bool done = terminal;
        if (!done) {
          const F3 rd = xyz(b.R1[g]);
          const float t = __uint_as_float(h.x);
          if (t < 0.0f) {
            Lo = Lo + tp * sky_color(u, rd, false);
            done = true;
          } else {
            const F3 pos = xyz(b.R0[g]) + rd * t;
            keep = shade_vertex(u, b, g, (uint32_t)wave, pos, hit_normal((int)h.z, rd), unpack_material(h.y), Lo,
                                tp, rng, __float_as_uint(s1.w), shadow, bounce, nB, nullptr);
            done = !keep;
          }
        }
        if (done) {
          const float4 x2c = r.x2[g];
          finish_point(job, r, g, Lo, __float_as_uint(s1.w), xyz(x2c), normal_decode(__float_as_uint(x2c.w)), rng);
        }
      }
    }
    emit_block(b, wave + 1, g, shadow, bounce, keep);
  }
}

// ---------------------------------------------------------------------------
// wavefront form of the unified initial pass (RF_UNIFIED).  At x1 the RNG
// stream depends on each visibility result (a candidate that survives its
// shadow ray draws its RIS number), so x1's rays run one per wave:
//   kStSun    sun-cone shadow ray -> sun direction candidate
//   kStLight  light-list RIS over emissive faces -> its shadow ray -> candidate
//   kStBounce bounce ray -> x2 (or a sky direction candidate)
// then every estimateLo vertex issues its sun shadow ray, its light-list NEE
// shadow ray (the tracer's second shadow slot) and its bounce ray in one wave
// (kStLo): no draw depends on their results.  The RIS state at x1 (weight
// sum, selected candidate, p-hat) is kept per path between waves.
// ---------------------------------------------------------------------------
enum : uint32_t { kStSun = 0u, kStLight = 1u, kStBounce = 2u, kStLo = 3u };

// State bits (x2.w): x2's normal code 0-5, selected kind 6-7, its normal
// code 8-13, stage 14-15, light candidate's normal code 16-21, estimateLo
// vertex index 22-29 (paths reach x2 in different waves).
VRT_DI uint32_t bits_get(uint32_t b, int at, int n) { return (b >> at) & ((1u << n) - 1u); }
VRT_DI uint32_t bits_set(uint32_t b, int at, int n, uint32_t v) {
  const uint32_t m = ((1u << n) - 1u) << at;
  return (b & ~m) | ((v << at) & m);
}

VRT_DI void ris_save(const RestirWf& r, uint32_t g, const Ris& q, uint32_t& bits) {
  r.selPW[g] = make_float4(q.sel.pos.x, q.sel.pos.y, q.sel.pos.z, q.wSum);
  r.selRP[g] = make_float4(q.sel.rad.x, q.sel.rad.y, q.sel.rad.z, q.selP);
  bits = bits_set(bits, 6, 2, q.sel.kind);
  bits = bits_set(bits, 8, 6, normal_code(q.sel.n));
}

VRT_DI Ris ris_load(const RestirWf& r, uint32_t g, uint32_t bits) {
  const float4 a = r.selPW[g], c = r.selRP[g];
  Ris q;
  q.sel = null_sample(0.0f);
  q.sel.kind = bits_get(bits, 6, 2);
  q.sel.pos = f3(a.x, a.y, a.z);
  q.sel.n = normal_decode(bits_get(bits, 8, 6));
  q.sel.rad = f3(c.x, c.y, c.z);
  q.wSum = a.w;
  q.selP = c.w;
  return q;
}

// x1 and n1 of path g from the G-buffer and the recomputed primary ray.
VRT_DI void x1_of(const RestirDev& R, uint32_t g, F3& x1, F3& n1, F3& surf1) {
  const float4 gb = R.gbuf[g];
  n1 = f3(gb.x, gb.y, gb.z);
  const uint32_t gx = g % (uint32_t)R.W, gy = g / (uint32_t)R.W;
  x1 = f3(R.u.camPos[0], R.u.camPos[1], R.u.camPos[2]) + primary_dir(R.u, gx, gy, R.W, R.H) * gb.w;
  surf1 = x1 + n1 * fmax_(1e-3f, gb.w * 1e-4f);
}

struct URays {
  bool shadow = false, shadow2 = false, bounce = false;
};

// The path's candidate is final: reservoir A.
VRT_DI void unified_finish(const RestirDev& R, uint32_t g, const Ris& ris) { store_ris(R.resA, g, R.u, R.W, R.H, ris); }

// Runs x1's stages from the start of stage `st` (earlier stages resolved)
// until a ray is pending (returned in rays, state saved) or the candidate
// path ends.
VRT_DI void x1_run(const RestirDev& R, const RestirWf& r, const WfDev& b, uint32_t g, uint32_t st, Ris& ris,
                   uint32_t& bits, uint32_t& rng, F3 x1, F3 n1, F3 surf1, URays& rays) {
  const Uni& u = R.u;
  if (st == kStLight) {   // light-list NEE at x1: RIS over emissive faces
    if (u.params2[1] > 0u) {
      const uint32_t nCand = emissive_cand_count(u, 0u);
      float eSum = 0.0f, eSelP = 0.0f;
      RSample eSel = null_sample(0.0f);
      for (uint32_t k = 0u; k < nCand; k++) {
        const LightPoint lp = sample_light_face(R, x1, rng);
        RSample s = null_sample(0.0f);
        s.kind = kSkPoint;
        s.pos = lp.pos;
        s.n = lp.n;
        s.rad = lp.Le;
        const float pt = eval_target(s, x1, n1);
        const float w = pt / ((float)nCand * lp.pdfA);
        if (w > 0.0f) {
          eSum = eSum + w;
          if (rand_(rng) * eSum < w) { eSel = s; eSelP = pt; }
        }
      }
      if (eSel.kind != kSkNone && eSelP > 0.0f) {
        const F3 d = eSel.pos - surf1;
        const float rr = __fsqrt_rn(dot3(d, d));
        b.R0[g] = make_float4(surf1.x, surf1.y, surf1.z, 0.0f);
        b.R2[g] = make_float4(d.x / rr, d.y / rr, d.z / rr, rr - 2e-3f);
        r.aux[g] = make_float4(eSel.pos.x, eSel.pos.y, eSel.pos.z, eSum);
        r.aux2[g] = make_float4(eSel.rad.x, eSel.rad.y, eSel.rad.z, eSelP);
        bits = bits_set(bits, 16, 6, normal_code(eSel.n));
        bits = bits_set(bits, 14, 2, kStLight);
        rays.shadow = true;
      }
    }
    if (!rays.shadow) st = kStBounce;
  }
  if (st == kStBounce) {
    if (u.params0[1] > 0u) {
      const F3 brd = cosine_hemisphere(n1, rng);
      b.R0[g] = make_float4(surf1.x, surf1.y, surf1.z, 0.0f);
      b.R1[g] = make_float4(brd.x, brd.y, brd.z, 1e4f);
      bits = bits_set(bits, 14, 2, kStBounce);
      rays.bounce = true;
    } else {
      unified_finish(R, g, ris);
      return;
    }
  }
  ris_save(r, g, ris, bits);
  b.S0[g] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng));
  r.x2[g] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(bits));
}

// estimateLo's vertex v with unification (pathtrace.wgsl:213-244): sun shadow,
// light-list NEE shadow and bounce rays issued together.  Returns whether the
// path stays active.
VRT_DI bool lo_vertex(const RestirDev& R, const WfDev& b, const RestirWf& r, uint32_t g, uint32_t v, F3 pos, F3 n,
                      Mat mat, F3 Lo, F3 tp, uint32_t& rng, URays& rays) {
  const Uni& u = R.u;
  const uint32_t nB = u.params0[1];
  const F3 surf = pos + n * 1e-3f;
  uint32_t flags = 0u;
  const F3 l = sample_sun_dir(u, rng);
  const float ndl = dot3(n, l);
  F3 sunc = f3(0.0f, 0.0f, 0.0f);
  if (ndl > 0.0f && l.y > 0.0f) {
    sunc = (((tp * mat.albedo) * kInvPi) * ndl) * f3(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
    b.R2[g] = make_float4(l.x, l.y, l.z, 1e4f);
    flags |= kFlagShadow;
    rays.shadow = true;
  }
  // light-list NEE: the candidate RIS of emissiveNEE; its shadow ray pending
  F3 neeC = f3(0.0f, 0.0f, 0.0f);
  if (u.params2[1] > 0u) {
    const uint32_t nCand = emissive_cand_count(u, v);
    const float invM = 1.0f / (float)nCand;
    float wSum = 0.0f, selLum = 0.0f, selR2 = 0.0f;
    F3 sel = f3(0.0f, 0.0f, 0.0f), selDir = sel;
    for (uint32_t k = 0u; k < nCand; k++) {
      const LightPoint lp = sample_light_face(R, pos, rng);
      const F3 d = lp.pos - surf;
      const float r2 = fmax_(dot3(d, d), 1e-6f);
      const F3 dir = d * (1.0f / __fsqrt_rn(r2));
      const float cos1 = dot3(n, dir);
      const float cos2 = dot3(lp.n, f3(-dir.x, -dir.y, -dir.z));
      if (cos1 <= 0.0f || cos2 <= 0.0f) continue;
      const F3 a = ((mat.albedo * kInvPi) * cos1) * cos2;
      const F3 vv =
          f3((a.x / r2) * lp.Le.x / lp.pdfA, (a.y / r2) * lp.Le.y / lp.pdfA, (a.z / r2) * lp.Le.z / lp.pdfA);
      const float w = rlum(vv) * invM;
      if (w <= 0.0f) continue;
      const bool first = wSum == 0.0f;
      wSum = wSum + w;
      if (first || rand_(rng) * wSum < w) {
        sel = vv;
        selLum = rlum(vv);
        selDir = dir;
        selR2 = r2;
      }
    }
    if (wSum > 0.0f) {
      neeC = tp * (sel * (wSum / selLum));
      const uint32_t g2 = g + (uint32_t)r.W * (uint32_t)r.H;   // the second shadow ray's path index
      b.R0[g2] = make_float4(surf.x, surf.y, surf.z, 0.0f);
      b.R2[g2] = make_float4(selDir.x, selDir.y, selDir.z, __fsqrt_rn(selR2) - 2e-3f);
      flags |= kFlagShadow2;
      rays.shadow2 = true;
    }
  }
  if (v == nB) {
    flags |= kFlagTerminal;
  } else {
    const F3 rd = cosine_hemisphere(n, rng);
    tp = tp * mat.albedo;
    bool alive = true;
    if (v >= 2u) {
      const float p = clamp_(fmax_(tp.x, fmax_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rand_(rng) > p) alive = false;
      else tp = f3(tp.x / p, tp.y / p, tp.z / p);
    }
    if (alive) {
      b.R1[g] = make_float4(rd.x, rd.y, rd.z, 1e4f);
      rays.bounce = true;
    } else {
      flags |= kFlagTerminal;
    }
  }
  b.R0[g] = make_float4(surf.x, surf.y, surf.z, 0.0f);
  b.S0[g] = make_float4(Lo.x, Lo.y, Lo.z, __uint_as_float(rng));
  b.S1[g] = make_float4(tp.x, tp.y, tp.z, 0.0f);
  b.S2[g] = make_float4(sunc.x, sunc.y, sunc.z, __uint_as_float(flags));
  r.aux[g] = make_float4(neeC.x, neeC.y, neeC.z, 0.0f);
  return rays.shadow || rays.shadow2 || rays.bounce;
}

// The end of estimateLo: the bounce candidate at x2, then the final RIS.
VRT_DI void lo_finish(const RestirDev& R, const RestirWf& r, uint32_t g, F3 Lo, uint32_t bits, uint32_t& rng) {
  F3 x1, n1, surf1;
  x1_of(R, g, x1, n1, surf1);
  const float4 x2c = r.x2[g];
  RSample s;
  float Wc;
  cand_point(x1, n1, xyz(x2c), normal_decode(bits_get(bits, 0, 6)), fclamp3(R, fclamp3(R, Lo)), s, Wc);
  Ris ris = ris_load(r, g, bits);
  const float pt = eval_target(s, x1, n1);
  ris.add(s, pt, pt * Wc, rng);
  unified_finish(R, g, ris);
}

__global__ void __launch_bounds__(256, 5) k_wf_unified_primary(const __grid_constant__ RestirDev R, RestirWf r,
                                                            uint32_t P, WfDev b) {
  const uint32_t stride = gridDim.x * blockDim.x;
  if (R.stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(R.stats + kStatPixels, (unsigned long long)P);
  const Uni& u = R.u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < P; base += stride) {
    const uint32_t g = base + threadIdx.x;
    URays rays;
    if (g < P) {
      const uint4 h = b.hit[g];
      const F3 rd = xyz(b.R1[g]);
      const float t = __uint_as_float(h.x);
      if (t < 0.0f) {
        const F3 sky = sky_color(u, rd, true);
        const uint2 sk = pack_h4(sky.x, sky.y, sky.z, 1.0f);
        R.rad16[g] = sk;
        if (R.rad32) R.rad32[g] = make_float4(sky.x, sky.y, sky.z, 1.0f);
        R.direct[g] = sk;
        R.alb8[g] = 0xffffffffu;
        R.gbuf[g] = make_float4(-rd.x, -rd.y, -rd.z, -1.0f);
        R.resA[2 * (size_t)g] = make_uint4(0u, 0u, 0u, 0u);
        R.resA[2 * (size_t)g + 1] = make_uint4(0u, 0u, 0u, 0u);
      } else {
        const Mat mat1 = unpack_material(h.y);
        const F3 x1 = f3(u.camPos[0], u.camPos[1], u.camPos[2]) + rd * t;
        const F3 n1 = hit_normal((int)h.z, rd);
        R.alb8[g] = unorm8_(__fsqrt_rn(mat1.albedo.x)) | (unorm8_(__fsqrt_rn(mat1.albedo.y)) << 8) |
                    (unorm8_(__fsqrt_rn(mat1.albedo.z)) << 16) | (255u << 24);
        R.gbuf[g] = make_float4(n1.x, n1.y, n1.z, t);
        const float em = mat1.emissive * kEmissiveScale;   // unified: the sun goes through the reservoir
        R.direct[g] = pack_h4(em, em, em, 1.0f);
        uint32_t rng = __float_as_uint(b.S0[g].w);
        const F3 surf1 = x1 + n1 * fmax_(1e-3f, t * 1e-4f);
        Ris ris;
        ris.sel = null_sample(0.0f);
        uint32_t bits = 0u;
        const F3 l = sample_sun_dir(u, rng);
        const float ndl = dot3(n1, l);
        if (ndl > 0.0f && l.y > 0.0f) {   // sun-cone shadow ray first
          b.R0[g] = make_float4(surf1.x, surf1.y, surf1.z, 0.0f);
          b.R2[g] = make_float4(l.x, l.y, l.z, 1e4f);
          ris_save(r, g, ris, bits);
          b.S0[g] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng));
          r.x2[g] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(bits_set(bits, 14, 2, kStSun)));
          rays.shadow = true;
        } else {
          x1_run(R, r, b, g, kStLight, ris, bits, rng, x1, n1, surf1, rays);
        }
      }
    }
    const bool keep = rays.shadow || rays.shadow2 || rays.bounce;
    emit2_block(b, 1, g, P, rays.shadow, rays.shadow2, rays.bounce, keep);
  }
}

// Four blocks per SM (64 registers): the wave gathers scattered path state and
// waits on it; ours 5.11 -> 5.05 ms per frame against three blocks at 80
// registers (five at 48 registers spill ~1 KB and run slower).
__global__ void __launch_bounds__(256, 4) k_wf_unified_wave(const __grid_constant__ RestirDev R, RestirWf r, WfDev b,
                                                         int wave) {
  const int n = b.ctr[4 * wave + 2];
  const uint32_t* list = active_of(b, wave);
  const Uni& u = R.u;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int i = base + threadIdx.x;
    URays rays;
    uint32_t g = 0u;
    if (i < n) {
      g = list[i];
      const float4 s0 = b.S0[g];
      uint32_t rng = __float_as_uint(s0.w);
      uint32_t bits = __float_as_uint(r.x2[g].w);
      const uint32_t st = bits_get(bits, 14, 2);
      const uint4 h = b.hit[g];
      if (st != kStLo) {
        F3 x1, n1, surf1;
        x1_of(R, g, x1, n1, surf1);
        Ris ris = ris_load(r, g, bits);
        if (st == kStSun) {   // the sun-cone shadow ray resolved
          if (h.w == 0u) {
            const float4 l = b.R2[g];
            const float coneSA = kTwoPi * (1.0f - u.sunDir[3]);
            RSample s = null_sample(0.0f);
            s.kind = kSkDir;
            s.pos = f3(l.x, l.y, l.z);
            const float den = fmax_(coneSA, 1e-5f);
            s.rad = f3(u.sunRadiance[0] / den, u.sunRadiance[1] / den, u.sunRadiance[2] / den);
            const float pt = eval_target(s, x1, n1);
            ris.add(s, pt, pt * coneSA, rng);
          }
          x1_run(R, r, b, g, kStLight, ris, bits, rng, x1, n1, surf1, rays);
        } else if (st == kStLight) {   // the light-list candidate's shadow ray resolved
          if (h.w == 0u) {
            const float4 a = r.aux[g], a2 = r.aux2[g];
            RSample eSel = null_sample(0.0f);
            eSel.kind = kSkPoint;
            eSel.pos = f3(a.x, a.y, a.z);
            eSel.n = normal_decode(bits_get(bits, 16, 6));
            eSel.rad = f3(a2.x, a2.y, a2.z);
            const float We = a.w / a2.w;
            ris.add(eSel, a2.w, a2.w * We, rng);
          }
          x1_run(R, r, b, g, kStBounce, ris, bits, rng, x1, n1, surf1, rays);
        } else {   // the bounce ray resolved: x2, or a sky direction candidate
          const F3 brd = xyz(b.R1[g]);
          const float t = __uint_as_float(h.x);
          if (t < 0.0f) {
            RSample s;
            float Wc;
            cand_dir(u, n1, brd, s, Wc);
            const float pt = eval_target(s, x1, n1);
            ris.add(s, pt, pt * Wc, rng);
            unified_finish(R, g, ris);
          } else {
            const F3 x2 = surf1 + brd * t;
            const F3 n2 = hit_normal((int)h.z, brd);
            bits = bits_set(bits, 0, 6, normal_code(n2));
            bits = bits_set(bits, 14, 2, kStLo);
            bits = bits_set(bits, 22, 8, 1u);
            ris_save(r, g, ris, bits);
            r.x2[g] = make_float4(x2.x, x2.y, x2.z, __uint_as_float(bits));
            if (!lo_vertex(R, b, r, g, 1u, x2, n2, unpack_material(h.y), f3(0.0f, 0.0f, 0.0f),
                           f3(1.0f, 1.0f, 1.0f), rng, rays))
              lo_finish(R, r, g, f3(0.0f, 0.0f, 0.0f), bits, rng);
          }
        }
      } else {   // estimateLo vertex (wave - 3) resolved: shadows, then the bounce hit
        const float4 s1 = b.S1[g], s2 = b.S2[g];
        const uint32_t flags = __float_as_uint(s2.w);
        F3 Lo = xyz(s0), tp = xyz(s1);
        if ((flags & kFlagShadow) && h.w == 0u) Lo = Lo + xyz(s2);
        if ((flags & kFlagShadow2) && b.hit[g + (uint32_t)r.W * (uint32_t)r.H].w == 0u) Lo = Lo + xyz(r.aux[g]);
        bool done = (flags & kFlagTerminal) != 0u;
        if (!done) {
          const F3 rd = xyz(b.R1[g]);
          const float t = __uint_as_float(h.x);
          if (t < 0.0f) {
            Lo = Lo + tp * sky_color(u, rd, false);
            done = true;
          } else {
            const uint32_t v = bits_get(bits, 22, 8) + 1u;
            bits = bits_set(bits, 22, 8, v);
            const float4 x2c = r.x2[g];
            r.x2[g] = make_float4(x2c.x, x2c.y, x2c.z, __uint_as_float(bits));
            const F3 pos = xyz(b.R0[g]) + rd * t;
            done = !lo_vertex(R, b, r, g, v, pos, hit_normal((int)h.z, rd), unpack_material(h.y), Lo, tp, rng, rays);
          }
        }
        if (done) lo_finish(R, r, g, Lo, bits, rng);
      }
    }
    const bool keep = rays.shadow || rays.shadow2 || rays.bounce;
    emit2_block(b, wave + 1, g, (uint32_t)r.W * (uint32_t)r.H, rays.shadow, rays.shadow2, rays.bounce, keep);
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
static RestirDev restir_dev(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H, const PathOut& out,
                            const RestirBufs& rb) {
  RestirDev R;
  R.S = to_dscene(s);
  R.u = to_uni(u);
  R.W = W;
  R.H = H;
  R.fclamp = fclamp;
  R.resA = (uint4*)rb.resA;
  R.resB = (uint4*)rb.resB;
  R.direct = (uint2*)rb.direct;
  R.rad16 = (uint2*)out.rad16;
  R.rad32 = (float4*)out.rad32;
  R.alb8 = out.alb8;
  R.gbuf = (float4*)out.gbuf;
  R.gprev = (const float4*)rb.gbuf_prev;
  R.stats = out.stats;
  R.dup = rb.dup;
  R.pairing = rb.pairing;
  R.lights = (const uint2*)rb.light_words;
  R.lightAlias = (const float4*)rb.light_alias;
  R.lightGrid = rb.light_grid;
  return R;
}

template <typename K>
static cudaError_t launch_occ_kernel(K kern_smem, K kern_glob, const SceneDev& s, int W, int H, const RestirDev& R,
                                     cudaStream_t st) {
  const size_t smem = occ_words(s.BG) * sizeof(uint32_t);
  const dim3 grid((W + 15) / 16, (H + 15) / 16);
  if (smem <= kMaxSmemOccBytes) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(kern_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    kern_smem<<<grid, 256, smem, st>>>(R);
  } else {
    kern_glob<<<grid, 256, 0, st>>>(R);
  }
  return cudaGetLastError();
}

cudaError_t launch_restir_initial(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                                  const PathOut& out, const RestirBufs& rb, cudaStream_t st) {
  const RestirDev R = restir_dev(s, u, fclamp, W, H, out, rb);
  return launch_occ_kernel(k_restir_initial<true>, k_restir_initial<false>, s, W, H, R, st);
}

static SingleJob restir_job(const SceneDev& s, const VrtUniforms& uu, float fclamp, int W, int H, const PathOut& out) {
  SingleJob job;
  std::memset(&job, 0, sizeof job);
  job.u = to_uni(uu);
  job.S = to_dscene(s);
  job.out.rad16 = (uint2*)out.rad16;
  job.out.rad32 = (float4*)out.rad32;
  job.out.alb8 = out.alb8;
  job.out.gbuf = (float4*)out.gbuf;
  job.fclamp = fclamp;
  job.W = W;
  job.H = H;
  return job;
}

static int occ_smem(const SceneDev& s) {
  const int smem_occ = (int)(occ_words(s.BG) * sizeof(uint32_t));
  return smem_occ <= (int)kMaxSmemOccBytes ? smem_occ : 0;
}

cudaError_t launch_restir_initial_wavefront(const SceneDev& s, const VrtUniforms& uu, float fclamp, int W, int H,
                                            const PathOut& out, const RestirBufs& rb, const WavefrontBufs& wb,
                                            const WavefrontTuning& tune, cudaStream_t st, uint32_t* launches,
                                            cudaEvent_t* trace_ev, int max_timed_waves, int* timed_waves) {
  const SingleJob job = restir_job(s, uu, fclamp, W, H, out);
  const RestirWf r{(uint4*)rb.resA, (uint2*)rb.direct, (float4*)rb.scratch, W, H, nullptr, nullptr, nullptr, nullptr};
  const uint32_t P = (uint32_t)W * (uint32_t)H;
  const int smem = occ_smem(s);
  unsigned long long* stats = out.stats;
  return wf_run_waves(job, P, (int)job.u.params0[1] + 2, smem, wb, tune, stats, st, launches, trace_ev,
                      max_timed_waves, timed_waves, [&](const WfDev& b, int w, int sblocks) {
                        if (w == 0) k_wf_restir_primary<<<sblocks, 256, 0, st>>>(job, r, P, b, stats);
                        else k_wf_restir_wave<<<sblocks, 256, 0, st>>>(job, r, b, w);
                        return cudaGetLastError();
                      });
}

cudaError_t launch_restir_unified_wavefront(const SceneDev& s, const VrtUniforms& uu, float fclamp, int W, int H,
                                            const PathOut& out, const RestirBufs& rb, const WavefrontBufs& wb,
                                            const WavefrontTuning& tune, cudaStream_t st, uint32_t* launches,
                                            cudaEvent_t* trace_ev, int max_timed_waves, int* timed_waves) {
  const SingleJob job = restir_job(s, uu, fclamp, W, H, out);
  const RestirDev R = restir_dev(s, uu, fclamp, W, H, out, rb);
  const uint32_t P = (uint32_t)W * (uint32_t)H;
  float4* sc = (float4*)rb.scratch;
  const RestirWf r{(uint4*)rb.resA, (uint2*)rb.direct, sc, W, H, sc + P, sc + 2 * (size_t)P, sc + 3 * (size_t)P,
                   sc + 4 * (size_t)P};
  const int smem = occ_smem(s);
  // x1's three sequential rays, then one wave per estimateLo vertex
  auto shade = [&](const WfDev& b, int w, int sblocks) {
    if (w == 0) k_wf_unified_primary<<<sblocks, 256, 0, st>>>(R, r, P, b);
    else k_wf_unified_wave<<<sblocks, 256, 0, st>>>(R, r, b, w);
    return cudaGetLastError();
  };
  return wf_run_waves<SingleJob, decltype(shade), true>(job, P, (int)job.u.params0[1] + 4, smem, wb, tune, out.stats,
                                                        st, launches, trace_ev, max_timed_waves, timed_waves, shade);
}

cudaError_t launch_restir_temporal(const SceneDev& s, const VrtUniforms& u, int W, int H, const PathOut& out,
                                   const RestirBufs& rb, cudaStream_t st) {
  const RestirDev R = restir_dev(s, u, 0.0f, W, H, out, rb);
  k_restir_temporal<<<dim3((W + 15) / 16, (H + 15) / 16), 256, 0, st>>>(R);
  return cudaGetLastError();
}

cudaError_t launch_restir_spatial(const SceneDev& s, const VrtUniforms& u, int W, int H, const PathOut& out,
                                  const RestirBufs& rb, cudaStream_t st) {
  const RestirDev R = restir_dev(s, u, 0.0f, W, H, out, rb);
  return launch_occ_kernel(k_restir_spatial<true>, k_restir_spatial<false>, s, W, H, R, st);
}

cudaError_t launch_restir_dupmap(const VrtUniforms& u, int W, int H, const RestirBufs& rb, cudaStream_t st) {
  SceneDev none;
  PathOut out;
  const RestirDev R = restir_dev(none, u, 0.0f, W, H, out, rb);
  k_restir_dupmap<<<dim3((W + 15) / 16, (H + 15) / 16), 256, 0, st>>>(R);
  return cudaGetLastError();
}

cudaError_t launch_restir_spatial_wavefront(const SceneDev& s, const VrtUniforms& u, int W, int H, const PathOut& out,
                                            const RestirBufs& rb, const WavefrontBufs& wb,
                                            const WavefrontTuning& tune, cudaStream_t st, uint32_t* launches) {
  const RestirDev R = restir_dev(s, u, 0.0f, W, H, out, rb);
  const SingleJob job = restir_job(s, u, 0.0f, W, H, out);
  const WfDev b = wf_view(wb);
  const int wave = 0;   // the initial pass's waves are complete: reuse slot 0
  cudaError_t e = cudaMemsetAsync(wb.ctr, 0, 16, st);
  if (e != cudaSuccess) return e;
  const dim3 grid((W + 15) / 16, (H + 15) / 16);
  if (u.params2[0] & kRfVector) k_restir_spatial_select<true><<<grid, 256, 0, st>>>(R, b, wave);
  else k_restir_spatial_select<false><<<grid, 256, 0, st>>>(R, b, wave);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int sms = wf_sm_count();
  const int smem = occ_smem(s);
  const int refill = tune.refill_min > 0 ? tune.refill_min : 8;
  if (smem > 0)
    e = wf_dispatch_trace<SingleJob, true, true>(tune.trace_variant, job, smem, tune.trace_blocks_per_sm, sms, b, wave,
                                                 0, refill, out.stats, st);
  else
    e = wf_dispatch_trace<SingleJob, false, true>(tune.trace_variant, job, 0, tune.trace_blocks_per_sm, sms, b, wave,
                                                  0, refill, out.stats, st);
  if (e != cudaSuccess) return e;
  k_restir_spatial_resolve<<<sms * 8, 256, 0, st>>>(R, b, wave);
  if (launches) *launches += 3;
  return cudaGetLastError();
}

}  // namespace vrt
