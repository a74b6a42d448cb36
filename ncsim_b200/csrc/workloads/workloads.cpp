// Seeded synthetic workloads of the benchmark and the tests (libncsim_workloads.so,
// declared in include/ncsim_workloads.h): the random layer family, the
// permutation/diagonal (reversible) family and a batch of the noisy random
// layer family.  They are not part of the drop-in interface of
// include/ncsim_cuda.h; every choice is drawn from StdRng::seed_from_u64(seed)
// (or the caller's generator), in the same order as the CPU oracle's
// generators, and the tests compare the two texts byte for byte.
#include <algorithm>
#include <cstring>

#include "../../../include/ncsim_workloads.h"
#include "../batch_plan.hpp"
#include "../host/ir.hpp"

namespace ncsim {
namespace {

// rank over GF(2) of rows given as bit masks
size_t gf2_rank(std::vector<uint64_t> r) {
  size_t rank = 0;
  for (int b = 63; b >= 0; --b) {
    size_t piv = rank;
    while (piv < r.size() && !((r[piv] >> b) & 1)) ++piv;
    if (piv == r.size()) continue;
    std::swap(r[rank], r[piv]);
    for (size_t i = 0; i < r.size(); ++i)
      if (i != rank && ((r[i] >> b) & 1)) r[i] ^= r[rank];
    ++rank;
  }
  return rank;
}

std::string random_layer_text(uint32_t n, uint32_t depth, ncsim_rng& rng, double noise_p, uint32_t m_lo, uint32_t m_hi) {
  std::string s = "QUBITS " + std::to_string(n) + "\n";
  static const char* one[] = {"H", "S", "T", "SQRT_X"};
  const double tau = 6.28318530717958647692;
  std::vector<uint32_t> perm(n);
  for (uint32_t layer = 0; layer < depth; ++layer) {
    for (uint32_t q = 0; q < n; ++q) {
      uint64_t g = rng.range64(0, 5);
      if (g < 4) s += std::string(one[g]) + " " + std::to_string(q) + "\n";
      else s += "RZ(" + fmt_f64(rng.f64() * tau) + ") " + std::to_string(q) + "\n";
    }
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    for (uint32_t i = n; i-- > 1;) std::swap(perm[i], perm[rng.range32(0, i + 1)]);
    for (uint32_t i = 0; i + 1 < n; i += 2) {
      const std::string pair = std::to_string(perm[i]) + " " + std::to_string(perm[i + 1]);
      s += "CZ " + pair + "\n";
      if (noise_p > 0.0) s += "DEPOLARIZE2(" + fmt_f64(noise_p) + ") " + pair + "\n";
    }
  }
  for (uint32_t q = m_lo; q < m_hi && q < n; ++q) s += "M " + std::to_string(q) + "\n";
  return s;
}

// The frame-sampler benchmark of the reference (examples/bench.rs:264-294):
// H on qubits 0..n/2, then `rounds` rounds of CX(q, b) + DEPOLARIZE2(p) for
// every even q with b = (q + 1 + gen_range(0..n-1)) mod n, followed by
// `meas` Z measurements of gen_range(0..n) qubits.
std::string frames_text(uint32_t n, uint32_t rounds, uint32_t meas, double p, ncsim_rng& rng) {
  std::string s = "QUBITS " + std::to_string(n) + "\n";
  for (uint32_t q = 0; q < n / 2; ++q) s += "H " + std::to_string(q) + "\n";
  const std::string noise = "DEPOLARIZE2(" + fmt_f64(p) + ") ";
  for (uint32_t r = 0; r < rounds; ++r) {
    for (uint32_t q = 0; q < n; q += 2) {
      const uint64_t b = (q + 1 + rng.range64(0, n - 1)) % n;
      const std::string pair = std::to_string(q) + " " + std::to_string(b);
      s += "CX " + pair + "\n" + noise + pair + "\n";
    }
    for (uint32_t k = 0; k < meas; ++k) s += "M " + std::to_string(rng.range64(0, n)) + "\n";
  }
  return s;
}

std::vector<uint32_t> pick_distinct(ncsim_rng& rng, uint32_t n, uint32_t k) {
  std::vector<uint32_t> v;
  while (v.size() < k) {
    uint32_t q = uint32_t(rng.range64(0, n));
    if (std::find(v.begin(), v.end(), q) == v.end()) v.push_back(q);
  }
  return v;
}

std::string random_terms(ncsim_rng& rng, uint32_t nv, uint32_t count) {
  std::string s;
  for (uint32_t t = 0; t < count; ++t) {
    uint32_t deg = 1 + uint32_t(rng.range64(0, 3));
    auto vars = pick_distinct(rng, nv, std::min(deg, nv));
    uint64_t c = 1 + rng.range64(0, 7);
    s += ";" + std::to_string(c) + ":";
    for (size_t i = 0; i < vars.size(); ++i) s += (i ? "," : "") + std::to_string(uint64_t(1) << vars[i]);
  }
  return s;
}

std::string reversible_text(uint32_t n, uint32_t gates, ncsim_rng& rng) {
  std::string s = "QUBITS " + std::to_string(n) + "\n";
  for (uint32_t q = 0; q < std::min<uint32_t>(16, n); ++q) s += "H " + std::to_string(q) + "\n";
  for (uint32_t i = 0; i < gates; ++i) {
    uint64_t g = rng.range64(0, 5);
    if (g <= 2) {
      auto qs = pick_distinct(rng, n, g == 0 ? 2 : 3);
      s += g == 0 ? "CX" : g == 1 ? "CCX" : "CCZ";
      for (uint32_t q : qs) s += " " + std::to_string(q);
      s += "\n";
    } else if (g == 3) {
      s += "DIAG(3;0" + random_terms(rng, n, 40) + ")";
      for (uint32_t q = 0; q < n; ++q) s += " " + std::to_string(q);
      s += "\n";
    } else {
      auto qs = pick_distinct(rng, n, 8);
      std::vector<uint64_t> rows(8);
      do {
        for (auto& r : rows) r = rng.range64(0, 256);
      } while (gf2_rank(rows) != 8);
      uint64_t shift = rng.range64(0, 256);
      s += "MONOMIAL(";
      for (int r = 0; r < 8; ++r) s += (r ? "," : "") + std::to_string(rows[r]);
      s += ";" + std::to_string(shift) + ";3;0" + random_terms(rng, 8, 8) + ";0,0,0)";
      for (uint32_t q : qs) s += " " + std::to_string(q);
      s += "\n";
    }
  }
  return s;
}


void need(const void* p, const char* what) {
  if (!p) throw Error(NCSIM_ERR_INVALID, std::string(what) + " is null");
}

}  // namespace
}  // namespace ncsim

using namespace ncsim;

extern "C" {

ncsim_status ncsim_workload_random_circuit(uint32_t n, uint32_t depth, uint64_t seed, double noise_p, uint32_t m_lo,
                                           uint32_t m_hi, ncsim_circuit** out) {
  return guarded([&] {
    need(out, "out");
    *out = nullptr;
    if (n < 1 || n > 64) throw Error(NCSIM_ERR_INVALID, "workload register must have 1..64 qubits");
    ncsim_rng rng(seed);
    *out = new ncsim_circuit(parse_circuit(random_layer_text(n, depth, rng, noise_p, m_lo, m_hi)));
  });
}
ncsim_status ncsim_workload_random_circuit_rng(ncsim_rng* rng, uint32_t n, uint32_t depth, double noise_p, uint32_t m_lo,
                                               uint32_t m_hi, ncsim_circuit** out) {
  return guarded([&] {
    need(rng, "rng");
    need(out, "out");
    *out = nullptr;
    if (n < 1 || n > 64) throw Error(NCSIM_ERR_INVALID, "workload register must have 1..64 qubits");
    *out = new ncsim_circuit(parse_circuit(random_layer_text(n, depth, *rng, noise_p, m_lo, m_hi)));
  });
}
ncsim_status ncsim_workload_frames_circuit(uint32_t n, uint32_t rounds, uint32_t meas, double p, uint64_t seed,
                                           ncsim_circuit** out) {
  return guarded([&] {
    need(out, "out");
    *out = nullptr;
    if (n < 2 || n > MAX_CIRCUIT_QUBITS) throw Error(NCSIM_ERR_INVALID, "frame workload needs 2..2^24 qubits");
    ncsim_rng rng(seed);
    *out = new ncsim_circuit(parse_circuit(frames_text(n, rounds, meas, p, rng)));
  });
}
ncsim_status ncsim_workload_reversible_circuit(uint32_t n, uint32_t gates, uint64_t seed, ncsim_circuit** out) {
  return guarded([&] {
    need(out, "out");
    *out = nullptr;
    if (n < 8 || n > 64) throw Error(NCSIM_ERR_INVALID, "reversible workload needs 8..64 qubits");
    ncsim_rng rng(seed);
    *out = new ncsim_circuit(parse_circuit(reversible_text(n, gates, rng)));
  });
}


ncsim_status ncsim_batch_random_layers(uint32_t count, uint64_t seed0, uint32_t n_lo, uint32_t n_span, uint32_t depth,
                                       double p, ncsim_batch** out) {
  return guarded([&] {
    need(out, "out");
    *out = nullptr;
    *out = batch::batch_random_layers(count, seed0, n_lo, n_span, depth, p);
  });
}

}  // extern "C"
