// CPU ORACLE — test infrastructure only (see ncsim_ref.hpp).  Nothing in the
// product path includes, links or runs this file.
//
// A restatement of the reference's Pauli-frame sampler, src/frame.rs:34-300,
// with the pieces it stands on:
// - Gate::tableau / is_clifford (gate.rs:568-665) and MonomialGate::to_tableau
//   (gate.rs:244-294): the images of X_j and Z_j under a Clifford gate;
// - the noiseless reference run of FrameSampler::new on a stabilizer tableau
//   (frame.rs:41-60): an Aaronson-Gottesman tableau stored by rows, with
//   Stabilizer::collapse's draw rule (stabilizer.rs:571-591: a random outcome
//   is `rng.gen::<bool>()`, drawn only when the outcome is not determined) and
//   the trait's reset (state/mod.rs:141-147);
// - run_batch / hits / inject / sample_packed / sample / sample_detectors /
//   parity (frame.rs:69-307), frames kept by columns (pauli/columns.rs).
#pragma once

#include "ncsim_ref.hpp"

namespace ref {

// i^phase X^x Z^z on a gate's k qubits (pauli/mod.rs convention)
struct LocalPauli {
  uint64_t x = 0, z = 0;
  uint8_t phase = 0;
};

inline Phasor phasor_inverse(const Phasor& p) { return Phasor::make(-p.sqrt2_power, -int64_t(p.phase), p.bits); }

// phasepoly.rs:680-695 on the canonical terms the oracle's PhasePoly keeps
inline bool poly_is_clifford(const PhasePoly& p) {
  for (auto& kv : p.terms) {
    const uint32_t s = uint32_t(kv.first.size()) + p.bits;
    const uint32_t sub = uint32_t(__builtin_ctzll(kv.second)) + 1;
    if ((s > sub ? s - sub : 0) > 2) return false;
  }
  return true;
}

// rows of M^{-1} (bits::inverse)
inline std::vector<uint64_t> gf2_inverse_rows(const std::vector<uint64_t>& rows, size_t k) {
  std::vector<uint64_t> a = rows, inv(k);
  for (size_t i = 0; i < k; ++i) inv[i] = 1ull << i;
  for (size_t c = 0; c < k; ++c) {
    size_t p = c;
    while (p < k && !((a[p] >> c) & 1)) ++p;
    if (p == k) throw SimError(ErrKind::Invalid, "singular");
    std::swap(a[p], a[c]);
    std::swap(inv[p], inv[c]);
    for (size_t r = 0; r < k; ++r)
      if (r != c && ((a[r] >> c) & 1)) a[r] ^= a[c], inv[r] ^= inv[c];
  }
  return inv;
}

// MonomialGate::to_tableau (gate.rs:244-294): U G U† on |0> and |e_j>
inline std::optional<std::vector<LocalPauli>> monomial_images(const MonomialGate& m) {
  if (!poly_is_clifford(m.phase)) return std::nullopt;
  const size_t k = m.k;
  const std::vector<uint64_t> inv = gf2_inverse_rows(m.rows, k);
  // MonomialGate::inverse applied to |x>: s^-1 zeta^-f(y) |y>, y = M^-1 (x ^ shift)
  auto inv_apply = [&](uint64_t x) {
    uint64_t y = 0;
    for (size_t i = 0; i < k; ++i)
      if (dot(inv[i], x ^ m.shift)) y |= 1ull << i;
    Phasor s = phasor_inverse(m.scalar).mul(Phasor::root(-int64_t(m.phase.eval(y)), m.phase.bits));
    return std::make_pair(s, y);
  };
  std::vector<LocalPauli> out;
  for (size_t t = 0; t < 2 * k; ++t) {
    const uint64_t gx = t < k ? 1ull << t : 0, gz = t < k ? 0 : 1ull << (t - k);
    auto conj = [&](uint64_t x) {
      auto [s1, y] = inv_apply(x);
      const int64_t ph = 2 * int64_t(dot(gz, y));  // Pauli::apply_to_basis: X^gx Z^gz
      auto [s2, o] = m.apply_to_basis(y ^ gx);
      return std::make_pair(s1.mul(Phasor::ipow(ph)).mul(s2), o);
    };
    auto [s0, a] = conj(0);
    if (s0.sqrt2_power != 0 || s0.bits > 2) return std::nullopt;
    LocalPauli q;
    q.x = a;
    q.phase = uint8_t(s0.bits == 0 ? 0 : (s0.phase << (2 - s0.bits)) & 3);
    for (size_t j = 0; j < k; ++j) {
      auto [sj, o] = conj(1ull << j);
      Phasor ratio = sj.mul(phasor_inverse(s0));
      if (o != (a ^ (1ull << j)) || ratio.sqrt2_power != 0 || ratio.bits > 1) return std::nullopt;
      if (ratio.bits == 1) q.z |= 1ull << j;
    }
    out.push_back(q);
  }
  return out;
}

inline LocalPauli local_of(const Pauli& p) { return LocalPauli{p.x, p.z, p.phase}; }

// Gate::tableau (gate.rs:587-634): X_j images, then Z_j images
inline std::optional<std::vector<LocalPauli>> clifford_images(const Gate& g) {
  auto tab = [](std::initializer_list<const char*> xs, std::initializer_list<const char*> zs, size_t k) {
    std::vector<LocalPauli> v;
    for (auto* s : xs) v.push_back(local_of(Pauli::from_string(k, s)));
    for (auto* s : zs) v.push_back(local_of(Pauli::from_string(k, s)));
    return v;
  };
  switch (g.g) {
    case G::I: return tab({"X0"}, {"Z0"}, 1);
    case G::X: return tab({"X0"}, {"-Z0"}, 1);
    case G::Y: return tab({"-X0"}, {"-Z0"}, 1);
    case G::Z: return tab({"-X0"}, {"Z0"}, 1);
    case G::H: return tab({"Z0"}, {"X0"}, 1);
    case G::S: return tab({"Y0"}, {"Z0"}, 1);
    case G::Sdg: return tab({"-Y0"}, {"Z0"}, 1);
    case G::SqrtX: return tab({"X0"}, {"-Y0"}, 1);
    case G::SqrtXdg: return tab({"X0"}, {"Y0"}, 1);
    case G::SqrtY: return tab({"-Z0"}, {"X0"}, 1);
    case G::SqrtYdg: return tab({"Z0"}, {"-X0"}, 1);
    case G::Cx: return tab({"X0*X1", "X1"}, {"Z0", "Z0*Z1"}, 2);
    case G::Cy: return tab({"X0*Y1", "Z0*X1"}, {"Z0", "Z0*Z1"}, 2);
    case G::Cz: return tab({"X0*Z1", "Z0*X1"}, {"Z0", "Z1"}, 2);
    case G::Swap: return tab({"X1", "X0"}, {"Z1", "Z0"}, 2);
    case G::PauliG: {
      const Pauli& p = g.pauli;
      std::vector<LocalPauli> v;
      for (size_t q = 0; q < p.n; ++q) {
        Pauli xq = Pauli::xq(p.n, q);
        v.push_back(local_of(((p.z >> q) & 1) ? xq.negated() : xq));
      }
      for (size_t q = 0; q < p.n; ++q) {
        Pauli zq = Pauli::zq(p.n, q);
        v.push_back(local_of(((p.x >> q) & 1) ? zq.negated() : zq));
      }
      return v;
    }
    case G::T: case G::Tdg: case G::Cs: case G::Csdg: case G::Ccz: case G::Ccx: case G::Rx: case G::Ry:
    case G::Rz: case G::Unitary:
      return std::nullopt;
    default: {
      auto m = g.monomial();
      if (!m) return std::nullopt;
      return monomial_images(*m);
    }
  }
}

// ---------------------------------------------------------------------------
// Stabilizer tableau by rows (Aaronson & Gottesman, "Improved simulation of
// stabilizer circuits", 2004), rows i^phase X^x Z^z
// ---------------------------------------------------------------------------
struct RowTableau {
  size_t n, nw;
  std::vector<std::vector<uint64_t>> x, z;  // 2n rows
  std::vector<uint8_t> ph;
  explicit RowTableau(size_t nq) : n(nq), nw((nq + 63) / 64), x(2 * nq, std::vector<uint64_t>(nw)),
                                   z(2 * nq, std::vector<uint64_t>(nw)), ph(2 * nq, 0) {
    for (size_t q = 0; q < n; ++q) {
      x[q][q / 64] |= 1ull << (q % 64);
      z[n + q][q / 64] |= 1ull << (q % 64);
    }
  }
  static bool get(const std::vector<uint64_t>& v, size_t q) { return (v[q / 64] >> (q % 64)) & 1; }
  static void set(std::vector<uint64_t>& v, size_t q, bool b) {
    if (b) v[q / 64] |= 1ull << (q % 64);
    else v[q / 64] &= ~(1ull << (q % 64));
  }
  // row h <- row h * row p
  void mul_row(size_t h, size_t p) {
    uint32_t c = 0;
    for (size_t w = 0; w < nw; ++w) c += popc(z[h][w] & x[p][w]);
    ph[h] = uint8_t((ph[h] + ph[p] + 2 * (c & 1)) & 3);
    for (size_t w = 0; w < nw; ++w) {
      x[h][w] ^= x[p][w];
      z[h][w] ^= z[p][w];
    }
  }
  void conjugate(const std::vector<LocalPauli>& img, const std::vector<size_t>& qs) {
    const size_t k = qs.size();
    for (size_t r = 0; r < 2 * n; ++r) {
      LocalPauli acc;
      for (size_t t = 0; t < 2 * k; ++t) {
        const bool b = t < k ? get(x[r], qs[t]) : get(z[r], qs[t - k]);
        if (!b) continue;
        const LocalPauli& m = img[t];
        acc.phase = uint8_t((acc.phase + m.phase + 2 * (popc(acc.z & m.x) & 1)) & 3);
        acc.x ^= m.x;
        acc.z ^= m.z;
      }
      ph[r] = uint8_t((ph[r] + acc.phase) & 3);
      for (size_t j = 0; j < k; ++j) {
        set(x[r], qs[j], (acc.x >> j) & 1);
        set(z[r], qs[j], (acc.z >> j) & 1);
      }
    }
  }
  bool anticommutes(size_t r, const std::vector<uint64_t>& px, const std::vector<uint64_t>& pz) const {
    uint32_t c = 0;
    for (size_t w = 0; w < nw; ++w) c += popc(x[r][w] & pz[w]) + popc(z[r][w] & px[w]);
    return c & 1;
  }
  bool measure(const WidePauli& P, StdRng& rng) {
    std::vector<uint64_t> px(nw), pz(nw);
    uint8_t pphase = P.phase;
    for (auto& s : P.sites) {
      if (s.second & 1) set(px, s.first, true);
      if (s.second & 2) set(pz, s.first, true);
      if (s.second == 3) pphase = uint8_t((pphase + 1) & 3);
    }
    size_t p = 2 * n;
    for (size_t r = n; r < 2 * n; ++r)
      if (anticommutes(r, px, pz)) {
        p = r;
        break;
      }
    if (p == 2 * n) {  // determined: +-P is the product of the stabilizers paired with anticommuting destabilizers
      std::vector<uint64_t> sx(nw), sz(nw);
      uint8_t sp = 0;
      for (size_t i = 0; i < n; ++i) {
        if (!anticommutes(i, px, pz)) continue;
        uint32_t c = 0;
        for (size_t w = 0; w < nw; ++w) c += popc(sz[w] & x[n + i][w]);
        sp = uint8_t((sp + ph[n + i] + 2 * (c & 1)) & 3);
        for (size_t w = 0; w < nw; ++w) sx[w] ^= x[n + i][w], sz[w] ^= z[n + i][w];
      }
      return ((sp + 4 - pphase) & 3) == 2;
    }
    const bool outcome = rng.gen_bool();
    for (size_t r = 0; r < 2 * n; ++r)
      if (r != p && anticommutes(r, px, pz)) mul_row(r, p);
    x[p - n] = x[p];
    z[p - n] = z[p];
    ph[p - n] = ph[p];
    x[p] = px;
    z[p] = pz;
    ph[p] = uint8_t((pphase + (outcome ? 2 : 0)) & 3);
    return outcome;
  }
};

// FrameSampler::new's reference record (frame.rs:41-60)
inline std::vector<bool> frame_reference(const Circuit& c, uint64_t seed) {
  for (auto& op : c.ops)
    if (op.kind == OpKind::GateOp && !clifford_images(op.gate))
      throw SimError(ErrKind::Unsupported, "FrameSampler: non-Clifford gate " + op.gate.name());
  RowTableau t(c.n);
  StdRng rng = StdRng::seed_from_u64(seed);
  std::vector<bool> rec;
  const auto ximg = *clifford_images(Gate::named(G::X));
  for (auto& op : c.ops) {
    switch (op.kind) {
      case OpKind::GateOp: t.conjugate(*clifford_images(op.gate), op.qubits); break;
      case OpKind::Measure: rec.push_back(t.measure(op.wide, rng)); break;
      case OpKind::Reset: {
        WidePauli zq;
        zq.n = c.n;
        zq.sites = {{op.qubit, 2}};
        if (t.measure(zq, rng)) t.conjugate(ximg, {op.qubit});
        break;
      }
      default: break;  // without_noise(): noise is dropped
    }
  }
  return rec;
}

// ---------------------------------------------------------------------------
// frame.rs
// ---------------------------------------------------------------------------
constexpr size_t FRAME_BATCH = size_t(1) << 14;  // frame.rs:31

inline size_t nwords(size_t bits) { return (bits + 63) / 64; }
inline void mask_to(std::vector<uint64_t>& b, size_t len) {  // bits::mask_to
  for (size_t w = 0; w < b.size(); ++w) {
    if (w * 64 >= len) b[w] = 0;
    else if (len - w * 64 < 64) b[w] &= (1ull << (len - w * 64)) - 1;
  }
}

// frame.rs:241-266
inline std::vector<size_t> frame_hits(size_t shots, double p, StdRng& rng) {
  std::vector<size_t> out;
  if (p <= 0.0) return out;
  if (p >= 0.25) {
    for (size_t s = 0; s < shots; ++s)
      if (rng.gen_f64() < p) out.push_back(s);
    return out;
  }
  const double l = std::log(1.0 - p);
  size_t s = 0;
  for (;;) {
    const double u = rng.gen_f64();
    const double gap = std::floor(std::log(1.0 - u) / l);
    if (!std::isfinite(gap) || gap >= double(shots - s)) break;
    s += size_t(gap);
    out.push_back(s);
    s += 1;
    if (s >= shots) break;
  }
  return out;
}

struct FrameSamplerRef {
  Circuit circuit;
  std::vector<bool> reference;
  std::vector<std::vector<LocalPauli>> images;  // per op (gates)

  FrameSamplerRef(const Circuit& c, std::vector<bool> ref) : circuit(c), reference(std::move(ref)) {
    if (reference.size() != c.num_measurements()) throw SimError(ErrKind::Invalid, "reference record length");
    for (auto& op : c.ops) {
      if (op.kind == OpKind::GateOp) {
        auto im = clifford_images(op.gate);
        if (!im) throw SimError(ErrKind::Unsupported, "FrameSampler: non-Clifford gate " + op.gate.name());
        images.push_back(*im);
      } else {
        images.emplace_back();
      }
    }
  }

  // frame.rs:104-153: the records of one batch, one packed vector per measurement
  std::vector<std::vector<uint64_t>> run_batch(size_t shots, uint64_t seed) const {
    const size_t n = circuit.n, W = nwords(shots);
    StdRng rng = StdRng::seed_from_u64(seed);
    std::vector<std::vector<uint64_t>> x(n, std::vector<uint64_t>(W)), z(n, std::vector<uint64_t>(W));
    auto random_mask = [&]() {
      std::vector<uint64_t> b(W);
      for (auto& w : b) w = rng.next_u64();
      mask_to(b, shots);
      return b;
    };
    for (size_t q = 0; q < n; ++q) z[q] = random_mask();
    std::vector<std::vector<uint64_t>> out;
    size_t k = 0;
    for (size_t oi = 0; oi < circuit.ops.size(); ++oi) {
      const Op& op = circuit.ops[oi];
      switch (op.kind) {
        case OpKind::GateOp: {  // frames conjugate; signs do not matter
          const auto& img = images[oi];
          const size_t kq = op.qubits.size();
          for (size_t w = 0; w < W; ++w) {
            std::vector<uint64_t> nx(kq, 0), nz(kq, 0);
            for (size_t t = 0; t < 2 * kq; ++t) {
              const uint64_t v = t < kq ? x[op.qubits[t]][w] : z[op.qubits[t - kq]][w];
              for (size_t i = 0; i < kq; ++i) {
                if ((img[t].x >> i) & 1) nx[i] ^= v;
                if ((img[t].z >> i) & 1) nz[i] ^= v;
              }
            }
            for (size_t i = 0; i < kq; ++i) x[op.qubits[i]][w] = nx[i], z[op.qubits[i]][w] = nz[i];
          }
          break;
        }
        case OpKind::Measure: {
          std::vector<uint64_t> rec(W, 0);  // anticommute_mask
          for (auto& s : op.wide.sites)
            for (size_t w = 0; w < W; ++w) {
              if (s.second & 1) rec[w] ^= z[s.first][w];
              if (s.second & 2) rec[w] ^= x[s.first][w];
            }
          mask_to(rec, shots);
          if (reference[k]) {
            for (auto& w : rec) w = ~w;
            mask_to(rec, shots);
          }
          out.push_back(rec);
          ++k;
          auto r = random_mask();  // xor_pauli_masked
          for (auto& s : op.wide.sites)
            for (size_t w = 0; w < W; ++w) {
              if (s.second & 1) x[s.first][w] ^= r[w];
              if (s.second & 2) z[s.first][w] ^= r[w];
            }
          break;
        }
        case OpKind::Reset: {
          auto r = random_mask();
          std::fill(x[op.qubit].begin(), x[op.qubit].end(), 0);
          z[op.qubit] = r;
          break;
        }
        case OpKind::NoiseOp: {  // inject (frame.rs:269-293)
          const auto errors = op.noise.errors();
          double total = 0.0;
          for (auto& e : errors) total += e.p;
          for (size_t s : frame_hits(shots, total, rng)) {
            double u = rng.gen_f64() * total;
            size_t pick = errors.size() - 1;
            for (size_t i = 0; i < errors.size(); ++i) {
              if (u < errors[i].p) {
                pick = i;
                break;
              }
              u -= errors[i].p;
            }
            const size_t w = s / 64;
            const uint64_t m = 1ull << (s % 64);
            for (size_t j = 0; j < op.qubits.size(); ++j) {
              if ((errors[pick].x >> j) & 1) x[op.qubits[j]][w] ^= m;
              if ((errors[pick].z >> j) & 1) z[op.qubits[j]][w] ^= m;
            }
          }
          break;
        }
        default: break;
      }
    }
    return out;
  }

  std::vector<uint64_t> batch_seeds(size_t shots, StdRng& rng) const {
    std::vector<uint64_t> s((shots + FRAME_BATCH - 1) / FRAME_BATCH);  // one draw per batch (frame.rs:72-74)
    for (auto& v : s) v = rng.next_u64();
    return s;
  }

  // frame.rs:69-89 with the batch seeds given; batches over `threads` threads
  std::vector<std::vector<uint64_t>> sample_packed_seeds(size_t shots, const std::vector<uint64_t>& seeds,
                                                         int threads = 1) const {
    const size_t m = reference.size(), nb = seeds.size();
    std::vector<std::vector<std::vector<uint64_t>>> parts(nb);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (long b = 0; b < long(nb); ++b)
      parts[b] = run_batch(std::min(FRAME_BATCH, shots - size_t(b) * FRAME_BATCH), seeds[b]);
    std::vector<std::vector<uint64_t>> out(m, std::vector<uint64_t>(nwords(shots), 0));
    for (size_t b = 0; b < nb; ++b)
      for (size_t k = 0; k < m; ++k)
        for (size_t w = 0; w < parts[b][k].size(); ++w) out[k][b * (FRAME_BATCH / 64) + w] |= parts[b][k][w];
    return out;
  }

  // frame.rs:155-205
  void sample_detectors_seeds(size_t shots, const std::vector<uint64_t>& seeds, std::vector<std::vector<uint64_t>>& det,
                              std::vector<std::vector<uint64_t>>& obs) const {
    std::vector<std::vector<size_t>> dets, obss;
    size_t m = 0;
    for (auto& op : circuit.ops) {
      if (op.kind == OpKind::Measure) ++m;
      if (op.kind == OpKind::Detector) {
        std::vector<size_t> d;
        for (size_t k : op.lookback) d.push_back(m - k);
        dets.push_back(d);
      }
      if (op.kind == OpKind::Observable) {
        if (obss.size() <= op.index) obss.resize(op.index + 1);
        for (size_t k : op.lookback) obss[op.index].push_back(m - k);
      }
    }
    auto form = [&](const std::vector<std::vector<size_t>>& idx, const std::vector<std::vector<uint64_t>>& rec,
                    size_t size) {
      std::vector<std::vector<uint64_t>> v;
      for (auto& d : idx) {
        std::vector<uint64_t> b(nwords(size), 0);
        bool f = false;
        for (size_t k : d) {
          f ^= bool(reference[k]);
          for (size_t w = 0; w < b.size(); ++w) b[w] ^= rec[k][w];
        }
        if (f)
          for (auto& w : b) w = ~w;
        mask_to(b, size);
        v.push_back(b);
      }
      return v;
    };
    det.assign(dets.size(), std::vector<uint64_t>(nwords(shots), 0));
    obs.assign(obss.size(), std::vector<uint64_t>(nwords(shots), 0));
    for (size_t b = 0; b < seeds.size(); ++b) {
      const size_t size = std::min(FRAME_BATCH, shots - b * FRAME_BATCH);
      auto rec = run_batch(size, seeds[b]);
      auto pd = form(dets, rec, size), po = form(obss, rec, size);
      for (size_t k = 0; k < pd.size(); ++k)
        for (size_t w = 0; w < pd[k].size(); ++w) det[k][b * (FRAME_BATCH / 64) + w] |= pd[k][w];
      for (size_t k = 0; k < po.size(); ++k)
        for (size_t w = 0; w < po[k].size(); ++w) obs[k][b * (FRAME_BATCH / 64) + w] |= po[k][w];
    }
  }
};

}  // namespace ref
