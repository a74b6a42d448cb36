// CPU ORACLE — test infrastructure only (see ncsim_ref.hpp).
//
// Seeded synthetic workloads.  The reference publishes no generator for these
// families, so the definitions are this project's own; the product library
// carries an independent implementation and the tests check that both emit
// the same circuit text for the same seed.
//
//  random layer family (n, depth, seed):
//    rng = StdRng::seed_from_u64(seed)
//    per layer: for q in 0..n: g = gen_range(0..5) -> H, S, T, SQRT_X, RZ(gen_f64() * TAU)
//               perm = (0..n) shuffled (rand 0.8 SliceRandom::shuffle)
//               CZ(perm[2i], perm[2i+1]) for i < n/2, each optionally followed by
//               DEPOLARIZE2(p) on the same pair
//  reversible family (n, gates, seed):
//    H on qubits 0..min(16,n); then per gate g = gen_range(0..5):
//      CX (2 qubits), CCX (3), CCZ (3), DIAG over the whole register
//      (bits 3, 40 monomials of degree 1..3, coefficients 1..7),
//      MONOMIAL on 8 qubits (random invertible GF(2) 8x8 by rejection,
//      random shift, bits-3 phase polynomial of 8 monomials, scalar 1).
//    Distinct qubits are drawn by rejection with gen_range(0..n).
#pragma once

#include "ncsim_ref.hpp"

#include <sstream>

namespace ref {

constexpr double TAU = 6.28318530717958647692;

inline void layer_family(std::ostringstream& os, size_t n, size_t depth, StdRng& rng, double noise_p) {
  static const char* names[] = {"H", "S", "T", "SQRT_X"};
  for (size_t layer = 0; layer < depth; ++layer) {
    for (size_t q = 0; q < n; ++q) {
      uint64_t g = rng.gen_range_u64(0, 5);
      if (g < 4) os << names[g] << ' ' << q << '\n';
      else os << "RZ(" << fmt_double(rng.gen_f64() * TAU) << ") " << q << '\n';
    }
    std::vector<size_t> perm(n);
    for (size_t i = 0; i < n; ++i) perm[i] = i;
    rng.shuffle(perm);
    for (size_t i = 0; i + 1 < n; i += 2) {
      os << "CZ " << perm[i] << ' ' << perm[i + 1] << '\n';
      if (noise_p > 0.0) os << "DEPOLARIZE2(" << fmt_double(noise_p) << ") " << perm[i] << ' ' << perm[i + 1] << '\n';
    }
  }
}

// The random layer family; measures Z on qubits [m_lo, m_hi) at the end.
inline std::string random_circuit_text(size_t n, size_t depth, StdRng& rng, double noise_p, size_t m_lo, size_t m_hi) {
  std::ostringstream os;
  os << "QUBITS " << n << '\n';
  layer_family(os, n, depth, rng, noise_p);
  for (size_t q = m_lo; q < m_hi && q < n; ++q) os << "M " << q << '\n';
  return os.str();
}

inline std::vector<size_t> distinct_qubits(StdRng& rng, size_t n, size_t k) {
  std::vector<size_t> qs;
  while (qs.size() < k) {
    size_t q = size_t(rng.gen_range_u64(0, n));
    if (std::find(qs.begin(), qs.end(), q) == qs.end()) qs.push_back(q);
  }
  return qs;
}

inline std::string poly_terms_text(size_t nv, size_t nterms, StdRng& rng) {
  std::ostringstream os;
  for (size_t t = 0; t < nterms; ++t) {
    size_t d = 1 + size_t(rng.gen_range_u64(0, 3));
    auto vars = distinct_qubits(rng, nv, std::min(d, nv));
    uint64_t c = 1 + rng.gen_range_u64(0, 7);
    os << ';' << c << ':';
    for (size_t i = 0; i < vars.size(); ++i) os << (i ? "," : "") << (1ull << vars[i]);
  }
  return os.str();
}

inline std::string reversible_circuit_text(size_t n, size_t gates, StdRng& rng) {
  std::ostringstream os;
  os << "QUBITS " << n << '\n';
  for (size_t q = 0; q < std::min<size_t>(16, n); ++q) os << "H " << q << '\n';
  for (size_t i = 0; i < gates; ++i) {
    uint64_t g = rng.gen_range_u64(0, 5);
    if (g == 0 || g == 1 || g == 2) {
      size_t k = g == 0 ? 2 : 3;
      auto qs = distinct_qubits(rng, n, k);
      os << (g == 0 ? "CX" : g == 1 ? "CCX" : "CCZ");
      for (size_t q : qs) os << ' ' << q;
      os << '\n';
    } else if (g == 3) {
      os << "DIAG(3;0" << poly_terms_text(n, 40, rng) << ")";
      for (size_t q = 0; q < n; ++q) os << ' ' << q;
      os << '\n';
    } else {
      const size_t k = 8;
      auto qs = distinct_qubits(rng, n, k);
      std::vector<uint64_t> rows(k);
      for (;;) {
        for (size_t r = 0; r < k; ++r) rows[r] = rng.gen_range_u64(0, 256);
        if (gf2_rank(rows, k) == k) break;
      }
      uint64_t shift = rng.gen_range_u64(0, 256);
      os << "MONOMIAL(";
      for (size_t r = 0; r < k; ++r) os << (r ? "," : "") << rows[r];
      os << ';' << shift << ";3;0" << poly_terms_text(k, 8, rng) << ";0,0,0)";
      for (size_t q : qs) os << ' ' << q;
      os << '\n';
    }
  }
  return os.str();
}


// The frame-sampler benchmark of the reference (examples/bench.rs:264-294)
inline std::string frames_circuit_text(size_t n, size_t rounds, size_t meas, double p, StdRng& rng) {
  std::ostringstream os;
  os << "QUBITS " << n << '\n';
  for (size_t q = 0; q < n / 2; ++q) os << "H " << q << '\n';
  for (size_t r = 0; r < rounds; ++r) {
    for (size_t q = 0; q < n; q += 2) {
      const size_t b = (q + 1 + rng.gen_range_u64(0, n - 1)) % n;
      os << "CX " << q << ' ' << b << '\n' << "DEPOLARIZE2(" << fmt_double(p) << ") " << q << ' ' << b << '\n';
    }
    for (size_t k = 0; k < meas; ++k) os << "M " << rng.gen_range_u64(0, n) << '\n';
  }
  return os.str();
}
}  // namespace ref
