// Host side of the hash families: the xoshiro256** stream and the draw of
// hash-function parameters.  Parameters must match the reference bit for
// bit, so the draw order is the reference's:
//   rng                 rng.hpp:26-33 (splitmix64 seeding), 59-72 (step)
//   multiply_shift      hashing.hpp:69-87   odd `a` by rejection
//   multiply_add_shift  hashing.hpp:145-160 `a` then `b`
//   tabulation<8|16>    hashing.hpp:277-295 table words, u32-truncated,
//                       T[c][v] row-major, functions back to back
//   matmul_sketch       matmul_sketch.hpp:15-18 h1/h2/s1/s2 <- seed+0..3
#include <chrono>

#include "cmm_internal.h"

namespace cmm {

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

Xoshiro256ss::Xoshiro256ss(uint64_t x) {
  for (int i = 0; i < 4; ++i) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    s[i] = z ^ (z >> 31);
  }
}

uint64_t Xoshiro256ss::operator()() {
  const uint64_t result = rotl64(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return result;
}

uint64_t time_millis() {
  using namespace std::chrono;
  return (uint64_t)duration_cast<milliseconds>(system_clock::now().time_since_epoch()).count();
}

uint64_t time_seed() {
  Xoshiro256ss r(time_millis());
  return r();
}

size_t hash_param_bytes(int kind) {
  switch (kind) {
    case MS: return 8;
    case MAS: return 16;
    case TAB8: return 4u * 256u * 4u;
    case TAB16: return 2u * 65536u * 4u;
  }
  throw invalid_argument("unknown hash kind");
}

std::vector<uint8_t> draw_hash_params(int kind, int n, uint64_t seed) {
  const size_t fb = hash_param_bytes(kind);
  std::vector<uint8_t> out(fb * (size_t)n);
  Xoshiro256ss rng(seed);
  if (kind == MS) {
    uint64_t* a = reinterpret_cast<uint64_t*>(out.data());
    for (int f = 0; f < n; ++f) {
      uint64_t v;
      do { v = rng(); } while ((v & 1) == 0);
      a[f] = v;
    }
  } else if (kind == MAS) {
    uint64_t* ab = reinterpret_cast<uint64_t*>(out.data());
    for (int f = 0; f < n; ++f) {
      ab[2 * f] = rng();
      ab[2 * f + 1] = rng();
    }
  } else {
    uint32_t* T = reinterpret_cast<uint32_t*>(out.data());
    const size_t words = fb / 4 * (size_t)n;
    for (size_t w = 0; w < words; ++w) T[w] = (uint32_t)rng();
  }
  return out;
}

SketchParams make_sketch_params(int kind, int d, int b, uint64_t seed) {
  SketchParams P;
  P.kind = kind;
  P.d = d;
  P.b = b;
  P.log2b = 0;
  while ((1 << P.log2b) < b) ++P.log2b;
  P.seed = seed;
  P.fn_bytes = hash_param_bytes(kind);
  const size_t set = P.fn_bytes * (size_t)d;
  P.blob.resize(4 * set);
  for (int f = 0; f < 4; ++f) {
    std::vector<uint8_t> one = draw_hash_params(kind, d, seed + (uint64_t)f);
    std::copy(one.begin(), one.end(), P.blob.begin() + f * set);
  }
  return P;
}

}  // namespace cmm
