// pairing.cpp -- the self-inverting Gaussian pairing textures of paired
// spatial reuse (pairing.js:1-89, Lin 2026 section 3), built on the host.
//
// Pixels of an S x S texture are filled with link indices so every index
// appears exactly twice side by side, then shuffled by n(sigma) passes of
// 2 x 2 Fisher-Yates permutations over a tiling (every other pass offset
// diagonally by one, wrapping); the two pixels sharing an index become mutual
// partners, stored as wrapped coordinate deltas (two i16 per u32).  The
// generator is the reference's deterministic mulberry32 stream with its
// seeds (0xc0ffee + 7919 i), and JavaScript's number semantics are kept: the
// PRNG works on 32-bit integers, the random index is floor(rand * (i + 1))
// of a double, the repeat count is a double expression.
#include <cmath>
#include <cstdint>
#include <vector>
#include "vrt_internal.h"

namespace vrt {

namespace {

struct Mulberry32 {
  uint32_t a;
  double next() {
    a = a + 0x6d2b79f5u;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
};

// shuffleCount (pairing.js:20-24): repeat count for a target sigma.
int shuffle_count(double sigma) {
  const double v = (sigma * sigma) / 2.0 + 1.46 / sigma + 1.76 / (sigma * sigma) + 0.656 / std::pow(sigma, 3.0) + 0.5;
  const double f = std::floor(v);
  return f < 1.0 ? 1 : (int)f;
}

void make_texture(int S, double sigma, uint32_t seed, uint32_t* out) {
  Mulberry32 rng{seed};
  std::vector<int32_t> link((size_t)S * S);
  for (int y = 0; y < S; y++)
    for (int x = 0; x < S; x++) link[(size_t)y * S + x] = (x >> 1) + (S >> 1) * y;
  const int n = shuffle_count(sigma);
  for (int it = 0; it < n; it++) {
    const int o = it & 1;
    for (int by = 0; by < S; by += 2)
      for (int bx = 0; bx < S; bx += 2) {
        const int x0 = (bx + o) % S, x1 = (bx + o + 1) % S, y0 = (by + o) % S, y1 = (by + o + 1) % S;
        const size_t cell[4] = {(size_t)y0 * S + x0, (size_t)y0 * S + x1, (size_t)y1 * S + x0, (size_t)y1 * S + x1};
        for (int i = 3; i > 0; i--) {
          const int j = (int)(rng.next() * (double)(i + 1));
          const int32_t t = link[cell[i]];
          link[cell[i]] = link[cell[j]];
          link[cell[j]] = t;
        }
      }
  }
  std::vector<int32_t> first(((size_t)S * S) >> 1, -1);
  auto wrap = [S](int d) {
    int w = d % S;
    if (w > S / 2) w -= S;
    if (w < -S / 2) w += S;
    return w;
  };
  for (int i = 0; i < S * S; i++) {
    const int32_t l = link[(size_t)i];
    if (first[(size_t)l] < 0) {
      first[(size_t)l] = i;
      continue;
    }
    const int a = first[(size_t)l], b = i;
    const int dx = wrap((b % S) - (a % S));
    const int dy = wrap(b / S - a / S);
    out[a] = ((uint32_t)(dy & 0xffff) << 16) | (uint32_t)(dx & 0xffff);
    out[b] = ((uint32_t)(-dy & 0xffff) << 16) | (uint32_t)(-dx & 0xffff);
  }
}

}  // namespace

void make_pairing_buffer(const double sigmas[3], uint32_t* out) {
  size_t off = 0;
  for (int i = 0; i < 3; i++) {
    const int S = kPairSizes[i];
    make_texture(S, sigmas[i], 0xc0ffeeu + (uint32_t)i * 7919u, out + off);
    off += (size_t)S * S;
  }
}

}  // namespace vrt

extern "C" int vrt_make_pairing(const double* sigmas, uint32_t* out, size_t words) {
  if (!sigmas || !out || words < vrt::kPairingWords) return VRT_ERR_INVALID;
  for (int i = 0; i < 3; i++)
    if (!(sigmas[i] > 0.0)) return VRT_ERR_INVALID;
  vrt::make_pairing_buffer(sigmas, out);
  return VRT_OK;
}
