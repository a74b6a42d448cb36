// Host side of the Pauli-frame sampler: Clifford actions, the reference run
// on a bit-sliced tableau, the layered device program and the random-stream
// scan of each batch.
#include "frames_plan.hpp"

#include <algorithm>
#include <cmath>
#include <map>

namespace ncsim {
namespace frames {

namespace {

inline uint32_t popc(uint64_t v) { return uint32_t(__builtin_popcountll(v)); }
inline uint64_t low_mask(uint32_t n) { return n >= 64 ? ~uint64_t(0) : ((uint64_t(1) << n) - 1); }

// a Pauli written with letters: phase counts the Y letters (Y = i X Z) and the sign
LocalPauli lp(uint64_t x, uint64_t z, bool negative = false) {
  return LocalPauli{x, z, (popc(x & z) + (negative ? 2u : 0u)) & 3u};
}

// Images of the named Cliffords, as their tableaux list them (gate.rs:590-604):
// X_j images first, then Z_j.
bool named_action(GateKind kind, CliffordAction& a) {
  switch (kind) {
    case GateKind::I: a.k = 1; a.img = {lp(1, 0), lp(0, 1)}; return true;
    case GateKind::X: a.k = 1; a.img = {lp(1, 0), lp(0, 1, true)}; return true;
    case GateKind::Y: a.k = 1; a.img = {lp(1, 0, true), lp(0, 1, true)}; return true;
    case GateKind::Z: a.k = 1; a.img = {lp(1, 0, true), lp(0, 1)}; return true;
    case GateKind::H: a.k = 1; a.img = {lp(0, 1), lp(1, 0)}; return true;
    case GateKind::S: a.k = 1; a.img = {lp(1, 1), lp(0, 1)}; return true;
    case GateKind::Sdg: a.k = 1; a.img = {lp(1, 1, true), lp(0, 1)}; return true;
    case GateKind::SqrtX: a.k = 1; a.img = {lp(1, 0), lp(1, 1, true)}; return true;
    case GateKind::SqrtXdg: a.k = 1; a.img = {lp(1, 0), lp(1, 1)}; return true;
    case GateKind::SqrtY: a.k = 1; a.img = {lp(0, 1, true), lp(1, 0)}; return true;
    case GateKind::SqrtYdg: a.k = 1; a.img = {lp(0, 1), lp(1, 0, true)}; return true;
    // two qubits: bit 0 is the first listed (the control)
    case GateKind::Cx: a.k = 2; a.img = {lp(3, 0), lp(2, 0), lp(0, 1), lp(0, 3)}; return true;
    case GateKind::Cy: a.k = 2; a.img = {lp(3, 2), lp(2, 1), lp(0, 1), lp(0, 3)}; return true;
    case GateKind::Cz: a.k = 2; a.img = {lp(1, 2), lp(2, 1), lp(0, 1), lp(0, 2)}; return true;
    case GateKind::Swap: a.k = 2; a.img = {lp(2, 0), lp(1, 0), lp(0, 2), lp(0, 1)}; return true;
    default: return false;
  }
}

// PhasePoly::max_level <= 2 on the canonical terms (phasepoly.rs:594-628,
// 680-695): parities masked to the variables, a zero parity drops the term,
// repeats collapse, equal parity sets add mod 2^bits.
bool poly_is_clifford(const PhasePolyIR& p) {
  const uint64_t mod = uint64_t(1) << p.bits;
  std::map<std::vector<uint64_t>, uint64_t> terms;
  for (size_t t = 0; t < p.coeffs.size(); ++t) {
    const uint64_t c = p.coeffs[t] % mod;
    if (c == 0) continue;
    std::vector<uint64_t> key;
    bool vanish = false;
    for (uint64_t l : p.parities[t]) {
      const uint64_t g = l & low_mask(p.nvars);
      if (g == 0) {
        vanish = true;
        break;
      }
      key.push_back(g);
    }
    if (vanish) continue;
    std::sort(key.begin(), key.end());
    key.erase(std::unique(key.begin(), key.end()), key.end());
    if (key.empty()) continue;  // a constant
    uint64_t& v = terms[key];
    v = (v + c) % mod;
    if (v == 0) terms.erase(key);
  }
  for (auto& kv : terms) {
    const uint32_t level_num = uint32_t(kv.first.size()) + p.bits;
    const uint32_t sub = uint32_t(__builtin_ctzll(kv.second)) + 1;
    const uint32_t level = level_num > sub ? level_num - sub : 0;
    if (level > 2) return false;
  }
  return true;
}

// rows of M^{-1} over GF(2) (k <= 64; rows[i] = the inputs feeding output i)
std::vector<uint64_t> gf2_inverse(const std::vector<uint64_t>& rows, uint32_t k) {
  std::vector<uint64_t> a(rows), inv(k);
  for (uint32_t i = 0; i < k; ++i) inv[i] = uint64_t(1) << i;
  for (uint32_t col = 0; col < k; ++col) {
    uint32_t piv = col;
    while (piv < k && !((a[piv] >> col) & 1)) ++piv;
    if (piv == k) throw Error(NCSIM_ERR_INVALID, "monomial gate: singular affine map");
    std::swap(a[piv], a[col]);
    std::swap(inv[piv], inv[col]);
    for (uint32_t r = 0; r < k; ++r)
      if (r != col && ((a[r] >> col) & 1)) {
        a[r] ^= a[col];
        inv[r] ^= inv[col];
      }
  }
  return inv;
}

inline uint64_t apply_rows(const std::vector<uint64_t>& rows, uint64_t x) {
  uint64_t y = 0;
  for (size_t i = 0; i < rows.size(); ++i) y |= uint64_t(popc(rows[i] & x) & 1) << i;
  return y;
}

// MonomialGate::to_tableau (gate.rs:244-294): U G U† evaluated on |0> and
// |e_j>, in units of 2^-B turns (B = max(bits, 2)); false when an image
// leaves the Pauli group.
bool monomial_action(const MonomialIR& m, CliffordAction& a) {
  const uint32_t k = m.k;
  if (k == 0 || k > 64) return false;
  const uint32_t B = std::max<uint32_t>(m.phase.bits, 2);
  const uint64_t modB = uint64_t(1) << B;
  const uint32_t up = B - m.phase.bits;
  const std::vector<uint64_t> inv = gf2_inverse(m.rows, k);
  auto conj_exp = [&](uint64_t gx, uint64_t gz, uint64_t y) {
    const uint64_t x = apply_rows(inv, y ^ m.shift);
    const uint64_t f1 = m.phase.eval(x ^ gx), f0 = m.phase.eval(x);
    uint64_t e = ((f1 + (uint64_t(1) << m.phase.bits) - f0) << up) % modB;
    if (popc(gz & x) & 1) e = (e + (modB >> 1)) % modB;
    return e;
  };
  a.k = k;
  a.img.assign(2 * size_t(k), LocalPauli{});
  for (uint32_t t = 0; t < 2 * k; ++t) {
    const uint64_t gx = t < k ? uint64_t(1) << t : 0;
    const uint64_t gz = t < k ? 0 : uint64_t(1) << (t - k);
    const uint64_t e0 = conj_exp(gx, gz, 0);
    if (e0 % (modB >> 2)) return false;  // not a power of i
    LocalPauli q;
    q.x = apply_rows(m.rows, gx);
    q.phase = uint32_t(e0 / (modB >> 2)) & 3u;
    for (uint32_t j = 0; j < k; ++j) {
      const uint64_t ej = conj_exp(gx, gz, uint64_t(1) << j);
      const uint64_t ratio = (ej + modB - e0) % modB;
      if (ratio == modB >> 1) q.z |= uint64_t(1) << j;
      else if (ratio != 0) return false;  // not +-1
    }
    a.img[t] = q;
  }
  return true;
}

// i^p1 X^x1 Z^z1 * i^p2 X^x2 Z^z2 = i^(p1+p2+2 z1.x2) X^(x1^x2) Z^(z1^z2)
inline void mul_into(LocalPauli& acc, const LocalPauli& b) {
  acc.phase = (acc.phase + b.phase + 2 * (popc(acc.z & b.x) & 1)) & 3;
  acc.x ^= b.x;
  acc.z ^= b.z;
}

}  // namespace

bool clifford_action(const GateIR& g, CliffordAction& out) {
  out = CliffordAction{};
  switch (g.kind) {
    case GateKind::T: case GateKind::Tdg: case GateKind::Cs: case GateKind::Csdg: case GateKind::Ccz:
    case GateKind::Ccx: case GateKind::Rx: case GateKind::Ry: case GateKind::Rz: case GateKind::Unitary:
      return false;
    case GateKind::Pauli: {  // X_j -> -X_j where P has Z_j; Z_j -> -Z_j where P has X_j
      const uint32_t k = g.pauli.n;
      out.k = k;
      out.img.resize(2 * size_t(k));
      for (uint32_t j = 0; j < k; ++j) {
        out.img[j] = lp(uint64_t(1) << j, 0, (g.pauli.z >> j) & 1);
        out.img[k + j] = lp(0, uint64_t(1) << j, (g.pauli.x >> j) & 1);
      }
      return true;
    }
    case GateKind::Phase: case GateKind::CPhase: case GateKind::Diagonal: case GateKind::Monomial: {
      MonomialIR m;
      if (!monomial_view(g, m) || !poly_is_clifford(m.phase)) return false;
      return monomial_action(m, out);
    }
    default: return named_action(g.kind, out);
  }
}

// ---------------------------------------------------------------------------
// Reference run: a stabilizer tableau stored by columns (for each qubit the x
// and z bits of all 2n rows, rows 0..n-1 destabilizers, n..2n-1 stabilizers,
// row i = i^phase X^x Z^z with the phase in two bit planes), so a gate is a
// few word operations per row word and a measurement O(n) of them.
// ---------------------------------------------------------------------------
namespace {

struct Tableau {
  uint32_t n, rw;
  std::vector<uint64_t> x, z;  // [q * rw + w]
  std::vector<uint64_t> p0, p1;

  explicit Tableau(uint32_t nq) : n(nq), rw((2 * nq + 63) / 64), x(size_t(nq) * rw), z(size_t(nq) * rw), p0(rw), p1(rw) {
    for (uint32_t q = 0; q < n; ++q) {
      x[size_t(q) * rw + q / 64] |= uint64_t(1) << (q % 64);
      const uint32_t r = n + q;
      z[size_t(q) * rw + r / 64] |= uint64_t(1) << (r % 64);
    }
  }
  uint64_t* X(uint32_t q) { return &x[size_t(q) * rw]; }
  uint64_t* Z(uint32_t q) { return &z[size_t(q) * rw]; }
  static bool bit(const uint64_t* v, uint32_t r) { return (v[r / 64] >> (r % 64)) & 1; }
  static void put(uint64_t* v, uint32_t r, bool b) {
    const uint64_t m = uint64_t(1) << (r % 64);
    v[r / 64] = b ? (v[r / 64] | m) : (v[r / 64] & ~m);
  }
  // phase += c on the rows of plane m (word w)
  void add_phase(uint32_t w, uint64_t m, uint32_t c) {
    if (c & 1) {
      const uint64_t carry = p0[w] & m;
      p0[w] ^= m;
      p1[w] ^= carry;
    }
    if (c & 2) p1[w] ^= m;
  }
  uint32_t phase_of(uint32_t r) const { return uint32_t(bit(p0.data(), r)) | (uint32_t(bit(p1.data(), r)) << 1); }

  // conjugate every row by a Clifford on qubits qs
  void apply(const CliffordAction& a, const std::vector<uint32_t>& qs) {
    const uint32_t k = a.k;
    std::vector<uint32_t> q2(2 * k);
    for (uint32_t t = 0; t < 2 * k; ++t) q2[t] = qs[t % k];
    // cross terms of the ordered product: img[s].z . img[t].x for s < t
    std::vector<std::pair<uint32_t, uint32_t>> cross;
    for (uint32_t s = 0; s < 2 * k; ++s)
      for (uint32_t t = s + 1; t < 2 * k; ++t)
        if (popc(a.img[s].z & a.img[t].x) & 1) cross.push_back({s, t});
    std::vector<uint64_t> v(2 * k), nx(k), nz(k);
    for (uint32_t w = 0; w < rw; ++w) {
      for (uint32_t j = 0; j < k; ++j) {
        v[j] = X(qs[j])[w];
        v[k + j] = Z(qs[j])[w];
      }
      for (uint32_t i = 0; i < k; ++i) nx[i] = nz[i] = 0;
      for (uint32_t t = 0; t < 2 * k; ++t) {
        if (!v[t]) continue;
        for (uint32_t i = 0; i < k; ++i) {
          if ((a.img[t].x >> i) & 1) nx[i] ^= v[t];
          if ((a.img[t].z >> i) & 1) nz[i] ^= v[t];
        }
        add_phase(w, v[t], a.img[t].phase);
      }
      for (auto& st : cross) p1[w] ^= v[st.first] & v[st.second];
      for (uint32_t i = 0; i < k; ++i) {
        X(qs[i])[w] = nx[i];
        Z(qs[i])[w] = nz[i];
      }
    }
  }

  // rows anticommuting with the Pauli (sites with letter bits 1 = X, 2 = Z)
  std::vector<uint64_t> anticommuting(const std::vector<std::pair<uint32_t, uint8_t>>& sites) {
    std::vector<uint64_t> m(rw, 0);
    for (auto& s : sites) {
      if (s.second & 1) for (uint32_t w = 0; w < rw; ++w) m[w] ^= Z(s.first)[w];
      if (s.second & 2) for (uint32_t w = 0; w < rw; ++w) m[w] ^= X(s.first)[w];
    }
    return m;
  }

  // measure P = i^pphase X^px Z^pz (PauliOp convention); `draw` gives the random outcome
  template <class Draw>
  bool measure(const PauliSites& P, Draw&& draw) {
    const std::vector<uint64_t> anti = anticommuting(P.sites);
    uint32_t pphase = P.phase;
    for (auto& s : P.sites) pphase += s.second == 3;
    pphase &= 3;
    // a stabilizer row anticommuting with P?
    uint32_t p = UINT32_MAX;
    for (uint32_t r = n; r < 2 * n; ++r)
      if (bit(anti.data(), r)) {
        p = r;
        break;
      }
    if (p == UINT32_MAX) {
      // deterministic: the product of the stabilizers n+i over the
      // destabilizers i that anticommute with P is +-P
      std::vector<uint64_t> sel(rw, 0);
      for (uint32_t i = 0; i < n; ++i)
        if (bit(anti.data(), i)) put(sel.data(), n + i, true);
      uint32_t ph = 0;
      for (uint32_t w = 0; w < rw; ++w) {
        ph += 1 * (popc(p0[w] & sel[w]) & 3) + 2 * (popc(p1[w] & sel[w]) & 1);
      }
      // ordered product: + 2 per pair s < t (both selected) with z_s[q] x_t[q]
      uint32_t pairs = 0;
      for (uint32_t q = 0; q < n; ++q) {
        const uint64_t* xq = X(q);
        const uint64_t* zq = Z(q);
        uint32_t carry = 0;  // parity of the selected z bits in earlier words
        for (uint32_t w = 0; w < rw; ++w) {
          const uint64_t zs = zq[w] & sel[w];
          uint64_t pre = zs ^ (zs << 1);  // inclusive prefix parity ...
          pre ^= pre << 2;
          pre ^= pre << 4;
          pre ^= pre << 8;
          pre ^= pre << 16;
          pre ^= pre << 32;
          pre ^= zs;                       // ... made exclusive
          if (carry) pre = ~pre;
          pairs += popc(pre & xq[w] & sel[w]);
          carry ^= popc(zs) & 1;
        }
      }
      ph = (ph + 2 * (pairs & 1)) & 3;
      return ((ph + 4 - pphase) & 3) == 2;
    }
    const bool outcome = draw();
    // every other row anticommuting with P: row_h <- row_h * row_p
    std::vector<uint64_t> m(anti);
    put(m.data(), p, false);
    const uint32_t php = phase_of(p);
    std::vector<uint64_t> par(rw, 0);  // z_h . x_p per row, before the update
    for (uint32_t q = 0; q < n; ++q)
      if (bit(X(q), p))
        for (uint32_t w = 0; w < rw; ++w) par[w] ^= Z(q)[w];
    for (uint32_t w = 0; w < rw; ++w) {
      add_phase(w, m[w], php);
      p1[w] ^= par[w] & m[w];
    }
    for (uint32_t q = 0; q < n; ++q) {
      const bool bx = bit(X(q), p), bz = bit(Z(q), p);
      if (bx) for (uint32_t w = 0; w < rw; ++w) X(q)[w] ^= m[w];
      if (bz) for (uint32_t w = 0; w < rw; ++w) Z(q)[w] ^= m[w];
    }
    // destabilizer p - n <- old stabilizer p; stabilizer p <- (-1)^outcome P
    const uint32_t d = p - n;
    for (uint32_t q = 0; q < n; ++q) {
      put(X(q), d, bit(X(q), p));
      put(Z(q), d, bit(Z(q), p));
      put(X(q), p, false);
      put(Z(q), p, false);
    }
    put(p0.data(), d, php & 1);
    put(p1.data(), d, (php >> 1) & 1);
    for (auto& s : P.sites) {
      if (s.second & 1) put(X(s.first), p, true);
      if (s.second & 2) put(Z(s.first), p, true);
    }
    const uint32_t np = (pphase + (outcome ? 2 : 0)) & 3;
    put(p0.data(), p, np & 1);
    put(p1.data(), p, (np >> 1) & 1);
    return outcome;
  }
};

}  // namespace

std::vector<uint8_t> reference_record(const ncsim_circuit& c, uint64_t seed) {
  Tableau t(c.n);
  ncsim_rng rng(seed);
  auto draw = [&] { return int32_t(rng.u32()) < 0; };  // rand 0.8: Standard bool
  std::vector<uint8_t> rec;
  rec.reserve(c.num_measurements());
  CliffordAction xgate;
  named_action(GateKind::X, xgate);
  for (const auto& op : c.ops) {
    switch (op.kind) {
      case OpKind::Gate: {
        CliffordAction a;
        if (!clifford_action(op.gate, a))
          throw Error(NCSIM_ERR_UNSUPPORTED, "FrameSampler: non-Clifford gate " + op.gate.text());
        t.apply(a, op.qubits);
        break;
      }
      case OpKind::Measure: rec.push_back(t.measure(op.sites, draw) ? 1 : 0); break;
      case OpKind::Reset: {
        PauliSites zq;
        zq.n = c.n;
        zq.sites = {{op.qubits[0], uint8_t(2)}};
        if (t.measure(zq, draw)) t.apply(xgate, op.qubits);
        break;
      }
      default: break;  // noise is left out; detectors and ticks do nothing
    }
  }
  return rec;
}

// ---------------------------------------------------------------------------
// the device program
// ---------------------------------------------------------------------------
namespace {

NoiseChannel channel_of(const NoiseIR& nz) {  // Noise::errors (circuit.rs:119-128)
  NoiseChannel ch;
  auto add = [&](double p, uint8_t x, uint8_t z) {
    ch.p.push_back(p);
    ch.x.push_back(x);
    ch.z.push_back(z);
  };
  switch (nz.kind) {
    case NoiseKind::XError: add(nz.p[0], 1, 0); break;
    case NoiseKind::YError: add(nz.p[0], 1, 1); break;
    case NoiseKind::ZError: add(nz.p[0], 0, 1); break;
    case NoiseKind::PauliChannel1: add(nz.p[0], 1, 0); add(nz.p[1], 1, 1); add(nz.p[2], 0, 1); break;
    case NoiseKind::Depolarize1:
      add(nz.p[0] / 3.0, 1, 0); add(nz.p[0] / 3.0, 1, 1); add(nz.p[0] / 3.0, 0, 1);
      break;
    case NoiseKind::Depolarize2:
      for (uint8_t k = 1; k < 16; ++k) add(nz.p[0] / 15.0, k & 3, k >> 2);
      break;
  }
  double t = 0.0;
  for (double p : ch.p) t += p;
  ch.total = t;
  return ch;
}

constexpr uint64_t K_END = uint64_t(1) << 53;  // draws are k 2^-53 with k < 2^53

// the reference's expressions, as functions of the draw's 53 bits
inline double skip_of(uint64_t k, double l) {
  const double u = double(k) * 0x1.0p-53;
  return std::floor(std::log(1.0 - u) / l);
}
inline uint32_t pick_of(uint64_t k, const NoiseChannel& ch) {
  double u = double(k) * 0x1.0p-53 * ch.total;
  for (uint32_t i = 0; i < ch.p.size(); ++i) {
    if (u < ch.p[i]) return i;
    u -= ch.p[i];
  }
  return uint32_t(ch.p.size() - 1);
}

// least k in [lo, K_END] with pred(k) (pred monotone: false ... false true ... true)
template <class Pred>
uint64_t least_true(uint64_t lo, uint64_t guess, Pred pred) {
  guess = std::min(std::max(guess, lo), K_END - 1);
  uint64_t a, b;  // pred(a) false (or a = lo - 1), pred(b) true (or b = K_END)
  if (pred(guess)) {
    b = guess;
    uint64_t step = 1;
    for (;;) {
      if (b - lo < step) {
        a = lo;
        if (pred(a)) return a;
        break;
      }
      const uint64_t c = b - step;
      if (!pred(c)) {
        a = c;
        break;
      }
      b = c;
      step *= 2;
    }
  } else {
    a = guess;
    uint64_t step = 1;
    for (;;) {
      if (K_END - 1 - a < step) {
        b = K_END - 1;
        if (!pred(b)) return K_END;
        break;
      }
      const uint64_t c = a + step;
      if (pred(c)) {
        b = c;
        break;
      }
      a = c;
      step *= 2;
    }
  }
  while (b - a > 1) {
    const uint64_t m = a + (b - a) / 2;
    if (pred(m)) b = m;
    else a = m;
  }
  return b;
}

constexpr uint64_t CHECK_SIDE = 3;  // k checked on each side of every step

std::shared_ptr<const SkipTable> build_skip(double p) {
  auto t = std::make_shared<SkipTable>();
  t->l = std::log(1.0 - p);
  const double l = t->l;
  t->thr.assign(BATCH + 1, K_END);
  t->thr[0] = 0;
  for (uint32_t g = 1; g <= BATCH; ++g) {
    const uint64_t lo = t->thr[g - 1];
    if (lo >= K_END) break;
    const double approx = -std::expm1(double(g) * l) * 0x1.0p53;
    const uint64_t guess = approx >= 0x1.0p53 ? K_END - 1 : uint64_t(approx);
    const uint64_t k = least_true(lo, guess, [&](uint64_t x) { return skip_of(x, l) >= double(g); });
    t->thr[g] = k;
    if (k >= K_END) break;
    for (uint64_t j = 1; j <= CHECK_SIDE; ++j) {
      if (k >= j && k - j >= lo && skip_of(k - j, l) >= double(g)) return nullptr;
      if (k + j - 1 < K_END && skip_of(k + j - 1, l) < double(g)) return nullptr;
    }
  }
  t->bucket.resize(size_t(1) << 16);
  uint32_t g = 0;
  for (uint64_t b = 0; b < t->bucket.size(); ++b) {
    const uint64_t k = b << 37;
    while (g < BATCH && t->thr[g + 1] <= k) ++g;
    t->bucket[b] = uint16_t(g);
  }
  return t;
}

std::shared_ptr<const PickTable> build_pick(const NoiseChannel& ch) {
  auto t = std::make_shared<PickTable>();
  uint64_t lo = 0;
  for (uint32_t i = 0; i + 1 < ch.p.size(); ++i) {
    const uint64_t k = least_true(lo, lo, [&](uint64_t x) { return pick_of(x, ch) > i; });
    for (uint64_t j = 1; j <= CHECK_SIDE; ++j) {
      if (k >= j && k - j >= lo && pick_of(k - j, ch) > i) return nullptr;
      if (k + j - 1 < K_END && pick_of(k + j - 1, ch) <= i) return nullptr;
    }
    t->thr.push_back(k);
    lo = std::min(k, K_END - 1);
  }
  return t;
}

// tables for the channels used often enough to repay them (one per distinct
// probability list, shared by the channel's ops)
void attach_tables(std::vector<NoiseChannel>& noise) {
  std::map<std::vector<double>, std::pair<size_t, std::vector<size_t>>> uses;
  for (size_t i = 0; i < noise.size(); ++i) {
    auto& u = uses[noise[i].p];
    u.second.push_back(i);
  }
  for (auto& kv : uses) {
    const auto& idx = kv.second.second;
    if (idx.size() < 64) continue;
    const NoiseChannel& ch = noise[idx[0]];
    if (!(ch.total > 0.0)) continue;
    std::shared_ptr<const SkipTable> skip = ch.total < 0.25 ? build_skip(ch.total) : nullptr;
    std::shared_ptr<const PickTable> pick = build_pick(ch);
    for (size_t i : idx) {
      noise[i].skip = skip;
      noise[i].pick = pick;
    }
  }
}

}  // namespace

Program compile(const ncsim_circuit& c, const std::vector<uint8_t>& reference) {
  Program P;
  P.n = c.n;
  P.num_measurements = c.num_measurements();
  if (reference.size() != P.num_measurements)
    throw Error(NCSIM_ERR_INVALID, "reference record of " + std::to_string(reference.size()) + " bits for " +
                                       std::to_string(P.num_measurements) + " measurements");
  P.reference = reference;
  for (uint32_t q = 0; q < c.n; ++q) P.draws.push_back({0, q});
  uint32_t mask = c.n;
  uint64_t k = 0;
  struct Pending {
    FrameOp op;
    std::vector<uint32_t> qubits;  // for the layering
  };
  std::vector<Pending> pend;
  for (const auto& op : c.ops) {
    switch (op.kind) {
      case OpKind::Gate: {
        CliffordAction a;
        if (!clifford_action(op.gate, a))
          throw Error(NCSIM_ERR_UNSUPPORTED, "FrameSampler: non-Clifford gate " + op.gate.text());
        // the frame action: images with signs dropped
        bool identity = true;
        for (uint32_t j = 0; j < a.k; ++j)
          identity = identity && a.img[j].x == (uint64_t(1) << j) && a.img[j].z == 0 && a.img[a.k + j].x == 0 &&
                     a.img[a.k + j].z == (uint64_t(1) << j);
        if (identity) break;
        Pending pd;
        pd.qubits = op.qubits;
        const auto& q = op.qubits;
        switch (op.gate.kind) {
          case GateKind::H: case GateKind::SqrtY: case GateKind::SqrtYdg: pd.op = {FOP_H, q[0], 0, 0}; break;
          case GateKind::S: case GateKind::Sdg: pd.op = {FOP_S, q[0], 0, 0}; break;
          case GateKind::SqrtX: case GateKind::SqrtXdg: pd.op = {FOP_SQRTX, q[0], 0, 0}; break;
          case GateKind::Cx: pd.op = {FOP_CX, q[0], q[1], 0}; break;
          case GateKind::Cz: pd.op = {FOP_CZ, q[0], q[1], 0}; break;
          case GateKind::Swap: pd.op = {FOP_SWAP, q[0], q[1], 0}; break;
          default: {
            if (a.k > MAX_LINEAR_K)
              throw Error(NCSIM_ERR_UNSUPPORTED, "FrameSampler: Clifford gates on more than " +
                                                     std::to_string(MAX_LINEAR_K) + " qubits");
            // output bit i (x_i at 2i, z_i at 2i+1) over input bits (x_j at 2j, z_j at 2j+1)
            pd.op = {FOP_LINEAR | (a.k << 8), 0, 0, uint32_t(P.pool.size())};
            for (uint32_t j = 0; j < a.k; ++j) P.pool.push_back(q[j]);
            for (uint32_t i = 0; i < a.k; ++i)
              for (int zo = 0; zo < 2; ++zo) {
                uint64_t row = 0;
                for (uint32_t j = 0; j < a.k; ++j) {
                  const LocalPauli& ix = a.img[j];
                  const LocalPauli& iz = a.img[a.k + j];
                  if (((zo ? ix.z : ix.x) >> i) & 1) row |= uint64_t(1) << (2 * j);
                  if (((zo ? iz.z : iz.x) >> i) & 1) row |= uint64_t(1) << (2 * j + 1);
                }
                P.pool.push_back(uint32_t(row));
                P.pool.push_back(uint32_t(row >> 32));
              }
          }
        }
        pend.push_back(std::move(pd));
        break;
      }
      case OpKind::Measure: {
        Pending pd;
        const uint32_t flip = reference[k] ? 1u : 0u;
        pd.op = {FOP_MEASURE | (uint32_t(op.sites.sites.size()) << 8) | (flip << 31), uint32_t(k), mask,
                 uint32_t(P.pool.size())};
        for (auto& s : op.sites.sites) {
          P.pool.push_back(s.first | (uint32_t(s.second) << 24));
          pd.qubits.push_back(s.first);
        }
        if (op.sites.sites.size() >= (1u << 23))
          throw Error(NCSIM_ERR_UNSUPPORTED, "FrameSampler: a measured Pauli on 2^23 qubits or more");
        P.draws.push_back({0, mask});
        ++mask;
        ++k;
        pend.push_back(std::move(pd));
        break;
      }
      case OpKind::Reset: {
        Pending pd;
        pd.op = {FOP_RESET, op.qubits[0], mask, 0};
        pd.qubits = op.qubits;
        P.draws.push_back({0, mask});
        ++mask;
        pend.push_back(std::move(pd));
        break;
      }
      case OpKind::Noise: {
        const uint32_t i = uint32_t(P.noise.size());
        P.noise.push_back(channel_of(op.noise));
        P.draws.push_back({1, i});
        if (!(P.noise.back().total > 0.0)) break;  // never hits: no frame operation
        Pending pd;
        pd.op = {FOP_NOISE | (uint32_t(op.qubits.size()) << 8), i, 0, uint32_t(P.pool.size())};
        for (uint32_t q : op.qubits) P.pool.push_back(q);
        pd.qubits = op.qubits;
        pend.push_back(std::move(pd));
        break;
      }
      case OpKind::Detector: case OpKind::Observable: {
        std::vector<uint64_t> idx;
        for (uint64_t lb : op.lookback) idx.push_back(k - lb);
        if (op.kind == OpKind::Detector) {
          P.detectors.push_back(idx);
        } else {
          if (P.observables.size() <= op.index) P.observables.resize(op.index + 1);
          P.observables[op.index].insert(P.observables[op.index].end(), idx.begin(), idx.end());
        }
        break;
      }
      case OpKind::Tick: break;
    }
  }
  P.num_masks = mask;
  attach_tables(P.noise);
  auto flip_of = [&](const std::vector<uint64_t>& idx) {
    uint32_t f = 0;
    for (uint64_t j : idx) f ^= reference[j];
    return uint8_t(f & 1);
  };
  for (auto& d : P.detectors) P.det_flip.push_back(flip_of(d));
  for (auto& o : P.observables) P.obs_flip.push_back(flip_of(o));
  // dependency layers: an operation goes one layer after the last one on any of its qubits
  std::vector<uint32_t> last(c.n, 0), layer(pend.size());
  uint32_t nlayers = 0;
  for (size_t i = 0; i < pend.size(); ++i) {
    uint32_t l = 0;
    for (uint32_t q : pend[i].qubits) l = std::max(l, last[q]);
    layer[i] = l;
    for (uint32_t q : pend[i].qubits) last[q] = l + 1;
    nlayers = std::max(nlayers, l + 1);
  }
  P.layer_off.assign(nlayers + 1, 0);
  for (size_t i = 0; i < pend.size(); ++i) ++P.layer_off[layer[i] + 1];
  for (uint32_t l = 0; l < nlayers; ++l) P.layer_off[l + 1] += P.layer_off[l];
  P.ops.resize(pend.size());
  std::vector<uint32_t> fill(P.layer_off.begin(), P.layer_off.end() - 1);
  for (size_t i = 0; i < pend.size(); ++i) P.ops[fill[layer[i]]++] = pend[i].op;
  return P;
}

// ---------------------------------------------------------------------------
// the random stream of one batch
// ---------------------------------------------------------------------------
void key_of_seed(uint64_t seed, uint32_t key[8]) {
  ncsim_rng r(seed);
  for (int i = 0; i < 8; ++i) key[i] = r.key[i];
}

namespace {

// Random access into a StdRng key stream: ChaCha12 blocks (the same block
// function as the host generator, host/rng.hpp) computed four at a time in
// the lanes of 128-bit vectors, starting at the block a read needs.  A noise
// channel's draws sit between masks the scan skips, so the stream is read in
// short runs at scattered positions.
struct KeyStream {
  typedef uint32_t v4 __attribute__((vector_size(16)));
  uint32_t key[8];
  uint64_t first = ~uint64_t(0) - 3;  // block index of buf[0..15] (none loaded yet: above every index)
  uint32_t buf[64];
  uint64_t pos = 0;                // u32 index of the next draw

  static inline v4 rl(v4 v, int s) { return (v << s) | (v >> (32 - s)); }
  void load(uint64_t b) {
    v4 x[16], in[16];
    const uint32_t c[4] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
    for (int i = 0; i < 4; ++i) in[i] = v4{c[i], c[i], c[i], c[i]};
    for (int i = 0; i < 8; ++i) in[4 + i] = v4{key[i], key[i], key[i], key[i]};
    for (int l = 0; l < 4; ++l) {
      in[12][l] = uint32_t(b + l);
      in[13][l] = uint32_t((b + l) >> 32);
      in[14][l] = 0;
      in[15][l] = 0;
    }
    for (int i = 0; i < 16; ++i) x[i] = in[i];
#define NCSIM_VQR(a, b, c, d)                  \
  x[a] += x[b], x[d] = rl(x[d] ^ x[a], 16);    \
  x[c] += x[d], x[b] = rl(x[b] ^ x[c], 12);    \
  x[a] += x[b], x[d] = rl(x[d] ^ x[a], 8);     \
  x[c] += x[d], x[b] = rl(x[b] ^ x[c], 7)
    for (int dr = 0; dr < 6; ++dr) {
      NCSIM_VQR(0, 4, 8, 12);
      NCSIM_VQR(1, 5, 9, 13);
      NCSIM_VQR(2, 6, 10, 14);
      NCSIM_VQR(3, 7, 11, 15);
      NCSIM_VQR(0, 5, 10, 15);
      NCSIM_VQR(1, 6, 11, 12);
      NCSIM_VQR(2, 7, 8, 13);
      NCSIM_VQR(3, 4, 9, 14);
    }
#undef NCSIM_VQR
    for (int i = 0; i < 16; ++i) {
      const v4 o = x[i] + in[i];
      for (int l = 0; l < 4; ++l) buf[16 * l + i] = o[l];
    }
    first = b;
  }
  // next_u64 and gen::<f64>() at the current position: a u64 draw reads two
  // consecutive words, and every draw of a frame batch is a u64 (masks and
  // gen::<f64>()), so positions stay even and a draw never straddles a block
  inline uint64_t u64() {
    const uint64_t b = pos >> 4;
    if (b < first || b >= first + 4) load(b);
    const uint32_t* w = buf + 16 * (b - first) + (pos & 15);
    pos += 2;
    return uint64_t(w[0]) | (uint64_t(w[1]) << 32);
  }
  inline double f64() { return double(u64() >> 11) * 0x1.0p-53; }
};

}  // namespace

void scan_batch(const Program& p, uint64_t seed, uint32_t shots, BatchScan& out) {
  const uint64_t words = (uint64_t(shots) + 63) / 64;
  KeyStream rng;
  key_of_seed(seed, rng.key);
  uint64_t& pos = rng.pos;  // u32 position of the next draw
  out.mask_pos.assign(p.num_masks, 0);
  out.ev_off.assign(p.noise.size() + 1, 0);
  out.events.clear();
  std::vector<uint32_t> hits;
  for (const auto& d : p.draws) {
    if (d.first == 0) {  // random_mask: `words` u64 draws (frame.rs:107-111)
      out.mask_pos[d.second] = pos;
      pos += 2 * words;
      continue;
    }
    const NoiseChannel& ch = p.noise[d.second];
    const double total = ch.total;
    // hits (frame.rs:241-266)
    hits.clear();
    if (total > 0.0) {
      if (total >= 0.25) {
        for (uint32_t s = 0; s < shots; ++s)
          if (rng.f64() < total) hits.push_back(s);
      } else if (ch.skip) {
        const SkipTable& t = *ch.skip;
        uint32_t s = 0;
        for (;;) {
          const uint32_t gap = t.at(rng.u64() >> 11);
          if (gap >= shots - s) break;
          s += gap;
          hits.push_back(s);
          s += 1;
          if (s >= shots) break;
        }
      } else {
        const double l = std::log(1.0 - total);
        uint64_t s = 0;
        for (;;) {
          const double u = rng.f64();
          const double gap = std::floor(std::log(1.0 - u) / l);
          if (!std::isfinite(gap) || gap >= double(shots - s)) break;
          s += uint64_t(gap);
          hits.push_back(uint32_t(s));
          s += 1;
          if (s >= shots) break;
        }
      }
      // which error, given that one happened (frame.rs:270-280)
      for (uint32_t s : hits) {
        const uint64_t k = rng.u64() >> 11;
        const uint32_t pick = ch.pick ? ch.pick->at(k) : pick_of(k, ch);
        out.events.push_back(s | (uint32_t(ch.x[pick]) << 16) | (uint32_t(ch.z[pick]) << 20));
      }
    }
    out.ev_off[d.second + 1] = uint32_t(out.events.size());
  }
  // noise ops are numbered in draw order: the offsets are already cumulative
  for (size_t i = 1; i < out.ev_off.size(); ++i) out.ev_off[i] = std::max(out.ev_off[i], out.ev_off[i - 1]);
}

}  // namespace frames
}  // namespace ncsim
