// Test infrastructure (the oracle): a CPU restatement of ncsim's
// SparseVector<C64> (src/state/sparse.rs) on registers of any width, with keys
// as Bits (src/bits.rs: Vec<u64>, nwords(n) words, qubit q = bit q % 64 of
// word q / 64).  It keeps the reference's entry-order rules: monomial gates,
// permutation matrices and Paulis move entries in place (sparse.rs:131-231),
// dense gates and projections expand and normalise (sort by key, add
// duplicates, drop exact zeros, sparse.rs:114-128), sampling walks the
// cumulative weights in entry order (sparse.rs:407-424).  Only the tests load
// it; nothing in the product links it.
#pragma once

#include "frames_ref.hpp"
#include "ncsim_ref.hpp"

#include <memory>

namespace ref {

using Bits = std::vector<uint64_t>;

// nwords (bits.rs:14-17) comes with the frame restatement
inline bool bget(const Bits& b, size_t i) { return (b[i / 64] >> (i % 64)) & 1; }
inline void bset(Bits& b, size_t i, bool v) {
  if (v) b[i / 64] |= 1ull << (i % 64);
  else b[i / 64] &= ~(1ull << (i % 64));
}
inline void bxor(Bits& a, const Bits& b) {
  for (size_t i = 0; i < a.size() && i < b.size(); ++i) a[i] ^= b[i];
}
inline uint32_t bdot_count(const Bits& a, const Bits& b) {
  uint32_t c = 0;
  for (size_t i = 0; i < a.size() && i < b.size(); ++i) c += uint32_t(__builtin_popcountll(a[i] & b[i]));
  return c;
}

struct WideSparse {
  size_t n = 0;
  std::vector<std::pair<Bits, C64>> ent;
  bool sorted = true;
  double cutoff = 0.0;

  static WideSparse zero_state(size_t n) {  // sparse.rs:37-52
    WideSparse s;
    s.n = n;
    s.ent.push_back({Bits(nwords(n), 0), C64(1.0, 0.0)});
    return s;
  }
  static size_t local(const Bits& b, const std::vector<size_t>& qs) {  // sparse.rs:244-251
    size_t x = 0;
    for (size_t j = 0; j < qs.size(); ++j) x |= size_t(bget(b, qs[j])) << j;
    return x;
  }
  static void set_local(Bits& b, const std::vector<size_t>& qs, size_t y) {  // sparse.rs:253-258
    for (size_t j = 0; j < qs.size(); ++j) bset(b, qs[j], (y >> j) & 1);
  }
  void normalize_entries() {  // sparse.rs:114-128
    std::sort(ent.begin(), ent.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<std::pair<Bits, C64>> out;
    for (auto& e : ent) {
      if (!out.empty() && out.back().first == e.first) out.back().second = cadd(out.back().second, e.second);
      else out.push_back(e);
    }
    const double cut = cutoff * cutoff;
    std::vector<std::pair<Bits, C64>> kept;
    for (auto& e : out)
      if (!is_exactly_zero(e.second) && (cut == 0.0 || norm_sqr(e.second) >= cut)) kept.push_back(e);
    ent.swap(kept);
    sorted = true;
  }
  std::vector<std::pair<Bits, C64>> sorted_view() const {
    auto v = ent;
    if (!sorted) std::sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    return v;
  }
  static const C64* find_in(const std::vector<std::pair<Bits, C64>>& v, const Bits& x) {
    auto it = std::lower_bound(v.begin(), v.end(), x, [](const auto& e, const Bits& k) { return e.first < k; });
    return it != v.end() && it->first == x ? &it->second : nullptr;
  }
  void apply_monomial(const MonomialGate& g, const std::vector<size_t>& qs) {  // sparse.rs:131-159
    const size_t gd = size_t(1) << qs.size();
    std::vector<std::pair<C64, size_t>> img(gd);
    bool permutes = false;
    for (size_t x = 0; x < gd; ++x) {
      auto [s, y] = g.apply_to_basis(x);
      img[x] = {from_phasor(s), size_t(y)};
      permutes |= y != x;
    }
    for (auto& e : ent) {
      const size_t x = local(e.first, qs);
      e.second = cmul(e.second, img[x].first);
      if (img[x].second != x) set_local(e.first, qs, img[x].second);
    }
    if (permutes) sorted = false;
  }
  void apply_matrix(const std::vector<C64>& m, const std::vector<size_t>& qs) {  // sparse.rs:161-214
    const size_t gd = size_t(1) << qs.size();
    std::vector<std::vector<std::pair<size_t, C64>>> cols(gd);
    for (size_t b = 0; b < gd; ++b)
      for (size_t a = 0; a < gd; ++a)
        if (!is_exactly_zero(m[a * gd + b])) cols[b].push_back({a, m[a * gd + b]});
    std::vector<size_t> targets;
    bool single = true;
    for (auto& c : cols) {
      if (c.size() == 1) targets.push_back(c[0].first);
      single &= c.size() == 1;
    }
    std::sort(targets.begin(), targets.end());
    targets.erase(std::unique(targets.begin(), targets.end()), targets.end());
    if (single && targets.size() == gd) {
      bool moved = false;
      for (size_t b = 0; b < gd; ++b) moved |= cols[b][0].first != b;
      for (auto& e : ent) {
        const size_t b = local(e.first, qs);
        e.second = cmul(cols[b][0].second, e.second);
        if (cols[b][0].first != b) set_local(e.first, qs, cols[b][0].first);
      }
      if (moved) sorted = false;
      return;
    }
    std::vector<std::pair<Bits, C64>> out;
    for (auto& e : ent) {
      const size_t b = local(e.first, qs);
      for (auto& [a, c] : cols[b]) {
        Bits k2 = e.first;
        set_local(k2, qs, a);
        out.push_back({k2, cmul(c, e.second)});
      }
    }
    ent.swap(out);
    normalize_entries();
  }
  void apply_pauli(const Bits& x, const Bits& z, uint32_t phase) {  // sparse.rs:216-231
    bool moves = false;
    for (uint64_t w : x) moves |= w != 0;
    for (auto& e : ent) {
      const uint32_t k = (phase + 2 * bdot_count(z, e.first)) & 3u;
      e.second = cmul(e.second, i_pow(k));
      bxor(e.first, x);
    }
    if (moves) sorted = false;
  }
  // sparse.rs:266-297
  void apply_gate(const Gate& gate, const std::vector<size_t>& qs) {
    check_qubits(qs, n);
    if (qs.size() != gate.arity()) throw SimError(ErrKind::Arity, "arity");
    if (gate.g == G::PauliG) {  // Pauli::embed
      Bits x(nwords(n), 0), z(nwords(n), 0);
      for (size_t j = 0; j < qs.size(); ++j) {
        if ((gate.pauli.x >> j) & 1) bset(x, qs[j], true);
        if ((gate.pauli.z >> j) & 1) bset(z, qs[j], true);
      }
      return apply_pauli(x, z, gate.pauli.phase);
    }
    if (auto m = gate.monomial()) return apply_monomial(*m, qs);
    if (auto m = gate.matrix()) return apply_matrix(*m, qs);
    throw SimError(ErrKind::NotRepresentable, "gate");
  }
  C64 norm_sq() const {  // sparse.rs:298-301
    std::vector<C64> t;
    for (auto& e : ent) t.push_back(abs_sq(e.second));
    return pairwise_sum(t.data(), t.size());
  }
  C64 amplitude(const Bits& idx) const {  // sparse.rs:303-313
    if (sorted) {
      const C64* p = find_in(ent, idx);
      return p ? *p : C64();
    }
    for (auto& e : ent)
      if (e.first == idx) return e.second;
    return C64();
  }
  C64 expectation(const Bits& x, const Bits& z, uint32_t phase) const {  // sparse.rs:315-335
    const auto view = sorted_view();
    std::vector<C64> terms;
    for (auto& [c, a] : view) {
      Bits d = c;
      bxor(d, x);
      const C64* b = find_in(view, d);
      if (!b) continue;
      const uint32_t k = (phase + 2 * bdot_count(z, c)) & 3u;
      terms.push_back(cmul(cconj(*b), cmul(i_pow(k), a)));
    }
    return pairwise_sum(terms.data(), terms.size());
  }
  C64 project(const Bits& x, const Bits& z, uint32_t phase, bool outcome) {  // sparse.rs:351-380
    const C64 half(0.5, 0.0);
    std::vector<std::pair<Bits, C64>> out;
    for (auto& [c, a] : ent) {
      Bits d = c;
      bxor(d, x);
      const uint32_t k = (phase + 2 * bdot_count(z, c)) & 3u;
      C64 f = cmul(i_pow(k), half);
      if (outcome) f = cneg(f);
      out.push_back({c, cmul(a, half)});
      out.push_back({d, cmul(f, a)});
    }
    ent.swap(out);
    normalize_entries();
    return norm_sq();
  }
  bool measure(const Bits& x, const Bits& z, uint32_t phase, StdRng& rng) {  // mod.rs:113-131
    if (((phase & 1) == 1) != bool(bdot_count(x, z) & 1))
      throw SimError(ErrKind::Invalid, "measured operator is not Hermitian");
    const double e = expectation(x, z, phase).re;
    const double nn = norm_sq().re;
    double p_plus = (1.0 + e / nn) / 2.0;
    if (!std::isnan(p_plus)) p_plus = std::min(1.0, std::max(0.0, p_plus));
    bool outcome;
    if (p_plus > 1.0 - 1e-12) outcome = false;
    else if (p_plus < 1e-12) outcome = true;
    else outcome = rng.gen_f64() >= p_plus;
    project(x, z, phase, outcome);
    return outcome;
  }
  std::vector<Bits> sample(StdRng& rng, size_t shots) const {  // sparse.rs:407-424
    std::vector<double> cum;
    double acc = 0.0;
    for (auto& e : ent) {
      acc += norm_sqr(e.second);
      cum.push_back(acc);
    }
    if (acc <= 0.0) throw SimError(ErrKind::ZeroState, "sample");
    std::vector<Bits> out;
    for (size_t s = 0; s < shots; ++s) {
      const double u = rng.gen_f64() * acc;
      size_t i = size_t(std::upper_bound(cum.begin(), cum.end(), u) - cum.begin());
      out.push_back(ent[std::min(i, cum.size() - 1)].first);
    }
    return out;
  }
  // the words of a measured Pauli's sites (Y = i X Z adds one to the phase)
  void sites_words(const WidePauli& w, Bits& x, Bits& z, uint32_t& phase) const {
    x.assign(nwords(n), 0);
    z.assign(nwords(n), 0);
    uint32_t ys = 0;
    for (auto& [q, l] : w.sites) {
      if (l & 1) bset(x, q, true);
      if (l & 2) bset(z, q, true);
      ys += l == 3;
    }
    phase = (w.phase + ys) & 3u;
  }
  // mod.rs:134-183
  std::vector<uint8_t> run(const Circuit& c, StdRng& rng) {
    if (c.n != n) throw SimError(ErrKind::Invalid, "circuit on a different register");
    std::vector<uint8_t> rec;
    Bits x, z;
    uint32_t ph = 0;
    for (auto& op : c.ops) {
      switch (op.kind) {
        case OpKind::GateOp: apply_gate(op.gate, op.qubits); break;
        case OpKind::Measure:
          sites_words(op.wide, x, z, ph);
          rec.push_back(measure(x, z, ph, rng) ? 1 : 0);
          break;
        case OpKind::Reset:
          x.assign(nwords(n), 0);
          z.assign(nwords(n), 0);
          bset(z, op.qubit, true);
          if (measure(x, z, 0, rng)) {
            Bits fx(nwords(n), 0);
            bset(fx, op.qubit, true);
            apply_pauli(fx, Bits(nwords(n), 0), 0);
          }
          break;
        case OpKind::NoiseOp: {
          auto e = op.noise.sample(rng);
          if (e) {
            x.assign(nwords(n), 0);
            z.assign(nwords(n), 0);
            for (size_t j = 0; j < op.qubits.size(); ++j) {
              if ((e->first >> j) & 1) bset(x, op.qubits[j], true);
              if ((e->second >> j) & 1) bset(z, op.qubits[j], true);
            }
            apply_pauli(x, z, 0);
          }
          break;
        }
        default: break;
      }
    }
    return rec;
  }
};

}  // namespace ref
