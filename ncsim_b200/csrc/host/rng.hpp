// The caller's random generator: rand 0.8's StdRng (ChaCha with 12 rounds),
// seeded by rand_core 0.6's `seed_from_u64` (PCG32 output words form the
// 256-bit key), read through a 64-word block buffer (four 16-word blocks per
// refill), as the reference's measurement and noise draws consume it
// (src/state/mod.rs:128, src/circuit.rs:138, src/state/vector.rs:505).
#pragma once

#include <cstdint>
#include <stdexcept>

struct ncsim_rng {
  uint32_t key[8];
  uint64_t next_block = 0;
  uint32_t buf[64];
  unsigned pos = 64;

  explicit ncsim_rng(uint64_t seed) {
    // PCG32 (XSH-RR) steps: advance, then output
    uint64_t st = seed;
    for (int w = 0; w < 8; ++w) {
      st = st * 6364136223846793005ull + 11634580027462260723ull;
      uint32_t xs = uint32_t(((st >> 18) ^ st) >> 27);
      uint32_t r = uint32_t(st >> 59);
      key[w] = r ? (xs >> r) | (xs << (32 - r)) : xs;
    }
  }

  static inline uint32_t rl(uint32_t v, int s) { return (v << s) | (v >> (32 - s)); }

  void refill() {
    for (int b = 0; b < 4; ++b) {
      const uint64_t ctr = next_block + uint64_t(b);
      uint32_t in[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                         key[4],      key[5],      key[6],      key[7],      uint32_t(ctr), uint32_t(ctr >> 32), 0u, 0u};
      uint32_t s[16];
      for (int i = 0; i < 16; ++i) s[i] = in[i];
#define NCSIM_QR(a, b, c, d)                     \
  s[a] += s[b], s[d] = rl(s[d] ^ s[a], 16);      \
  s[c] += s[d], s[b] = rl(s[b] ^ s[c], 12);      \
  s[a] += s[b], s[d] = rl(s[d] ^ s[a], 8);       \
  s[c] += s[d], s[b] = rl(s[b] ^ s[c], 7)
      for (int dr = 0; dr < 6; ++dr) {  // 12 rounds = 6 column + diagonal pairs
        NCSIM_QR(0, 4, 8, 12);
        NCSIM_QR(1, 5, 9, 13);
        NCSIM_QR(2, 6, 10, 14);
        NCSIM_QR(3, 7, 11, 15);
        NCSIM_QR(0, 5, 10, 15);
        NCSIM_QR(1, 6, 11, 12);
        NCSIM_QR(2, 7, 8, 13);
        NCSIM_QR(3, 4, 9, 14);
      }
#undef NCSIM_QR
      for (int i = 0; i < 16; ++i) buf[16 * b + i] = s[i] + in[i];
    }
    next_block += 4;
  }

  uint32_t u32() {
    if (pos >= 64) {
      refill();
      pos = 0;
    }
    return buf[pos++];
  }

  uint64_t u64() {
    if (pos + 1 < 64) {
      uint64_t v = uint64_t(buf[pos]) | (uint64_t(buf[pos + 1]) << 32);
      pos += 2;
      return v;
    }
    if (pos == 63) {  // one word left: it is the low half
      uint64_t lo = buf[63];
      refill();
      pos = 1;
      return lo | (uint64_t(buf[0]) << 32);
    }
    refill();
    pos = 2;
    return uint64_t(buf[0]) | (uint64_t(buf[1]) << 32);
  }

  // Standard f64: 53 high bits times 2^-53
  double f64() { return double(u64() >> 11) * 0x1.0p-53; }

  // Index of the next u32 word in the key stream.  The buffer holds four
  // consecutive blocks and a u64 draw that straddles a refill takes the last
  // word of one buffer and the first of the next, so every draw reads the
  // stream's next words in order: skipping draws is moving this index.
  uint64_t position() const { return next_block * 16 + pos - 64; }
  void seek(uint64_t p) {
    next_block = (p / 64) * 4;
    pos = 64;
    if (p % 64) {
      refill();
      pos = unsigned(p % 64);
    }
  }

  // UniformInt sample_single over [lo, hi) with u64 words
  uint64_t range64(uint64_t lo, uint64_t hi) {
    if (hi <= lo) throw std::invalid_argument("empty range");
    const uint64_t span = hi - lo;
    const uint64_t zone = (span << __builtin_clzll(span)) - 1;
    for (;;) {
      const unsigned __int128 prod = (unsigned __int128)u64() * span;
      if (uint64_t(prod) <= zone) return lo + uint64_t(prod >> 64);
    }
  }

  // the same over u32 words (what slice shuffles use for bounds below 2^32)
  uint32_t range32(uint32_t lo, uint32_t hi) {
    if (hi <= lo) throw std::invalid_argument("empty range");
    const uint32_t span = hi - lo;
    const uint32_t zone = (span << __builtin_clz(span)) - 1;
    for (;;) {
      const uint64_t prod = uint64_t(u32()) * span;
      if (uint32_t(prod) <= zone) return lo + uint32_t(prod >> 32);
    }
  }
};
