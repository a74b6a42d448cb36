// Host-side exact scalars of the engine: the phasor values that gate tables
// and phase polynomials evaluate to (src/scalar.rs:101-154, 211-295).
#pragma once

#include <cmath>
#include <cstdint>

namespace ncsim {

struct Cd {
  double re, im;
};

inline int64_t emod(int64_t a, int64_t m) {
  int64_t r = a % m;
  return r < 0 ? r + m : r;
}

// exp(2 pi i k / 2^bits), exact on quarter and eighth turns (scalar.rs:112-132)
inline Cd root_value(int64_t k, uint32_t bits) {
  const int64_t m = int64_t(1) << bits;
  k = emod(k, m);
  if ((4 * k) % m == 0) {
    static const Cd q[4] = {{1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}, {0.0, -1.0}};
    return q[(4 * k / m) & 3];
  }
  if ((8 * k) % m == 0) {
    const double h = 0.70710678118654752440;
    switch (8 * k / m) {
      case 1: return {h, h};
      case 3: return {-h, h};
      case 5: return {-h, -h};
      default: return {h, -h};
    }
  }
  const double t = 2.0 * 3.14159265358979323846 * double(k) / double(m);
  return {std::cos(t), std::sin(t)};
}

// sqrt(2)^k (scalar.rs:133-140)
inline double sqrt2_power(int64_t k) {
  int64_t half = k >= 0 ? k / 2 : -((-k + 1) / 2);
  double v = std::ldexp(1.0, int(half));
  if (emod(k, 2) == 1) v *= 1.41421356237309504880;
  return v;
}

// A normalized phasor sqrt2^s2 * exp(2 pi i phase / 2^bits) (scalar.rs:234-248).
struct Phase {
  int32_t s2 = 0;
  uint64_t phase = 0;
  uint32_t bits = 0;
  static Phase make(int32_t s2, int64_t ph, uint32_t bits) {
    Phase p;
    const uint64_t m = uint64_t(1) << bits;
    uint64_t v = uint64_t(emod(ph, int64_t(m)));
    while (bits > 0 && (v & 1) == 0) {
      v >>= 1;
      --bits;
    }
    p.s2 = s2;
    p.phase = v;
    p.bits = bits;
    return p;
  }
  Phase times(const Phase& o) const {
    uint32_t b = bits > o.bits ? bits : o.bits;
    uint64_t f = (phase << (b - bits)) + (o.phase << (b - o.bits));
    return make(s2 + o.s2, int64_t(f), b);
  }
  bool is_one() const { return s2 == 0 && phase == 0; }
  // the complex value: root times the real sqrt2 power (scalar.rs:39-52)
  Cd value() const {
    Cd r = root_value(int64_t(phase), bits);
    double s = sqrt2_power(s2);
    return {r.re * s - r.im * 0.0, r.re * 0.0 + r.im * s};
  }
};

}  // namespace ncsim
