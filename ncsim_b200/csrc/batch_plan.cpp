// Batching form, host side: trajectory generation, per-qubit folding, the
// pass/stage planner and the FP64 emulator of the device program.
#include "batch_plan.hpp"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>

namespace ncsim::batch {

namespace {

using M2 = std::array<Cd, 4>;

Cd cmul(Cd a, Cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
Cd cadd(Cd a, Cd b) { return {a.re + b.re, a.im + b.im}; }

// g applied after p
M2 mat_mul(const M2& g, const M2& p) {
  M2 r;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) r[2 * i + j] = cadd(cmul(g[2 * i], p[j]), cmul(g[2 * i + 1], p[2 + j]));
  return r;
}
bool is_zero(Cd c) { return c.re == 0.0 && c.im == 0.0; }
bool is_one(Cd c) { return c.re == 1.0 && c.im == 0.0; }

// X^x Z^z on one qubit: the raw bits a sampled error sets (Pauli::set_raw_bits,
// src/pauli/mod.rs:281-308, stored phase 0), applied as apply_pauli does
M2 pauli_matrix(unsigned x, unsigned z) {
  const Cd o{1, 0}, m{-1, 0}, zr{0, 0};
  if (x && z) return {zr, m, o, zr};
  if (x) return {zr, o, o, zr};
  if (z) return {o, zr, zr, m};
  return {o, zr, zr, o};
}

// Per-qubit folding state: the product of one-qubit ops since the qubit's
// last emitted gate; diagonal products commute with the two-qubit diagonals
// and are carried across them.
struct Folder {
  uint32_t n;
  std::vector<M2> pend;
  std::vector<char> nondiag;
  std::vector<QOp>& out;
  Folder(uint32_t n_, std::vector<QOp>& o) : n(n_), pend(n_), nondiag(n_, 0), out(o) {
    for (auto& m : pend) m = pauli_matrix(0, 0);
  }
  void one(uint32_t q, const M2& g) {
    pend[q] = mat_mul(g, pend[q]);
    if (!is_zero(g[1]) || !is_zero(g[2])) nondiag[q] = 1;
  }
  // A balanced unitary (every entry of modulus 1/sqrt2) is diag(l0, l1) B(w)
  // with B(w) = s [[1, w], [1, -w]]: B goes to the device, the diagonal stays
  // pending on the qubit (it commutes with the two-qubit diagonals) and is
  // multiplied into the qubit's next gate.
  void emit_gate(uint32_t q) {
    const M2 u = pend[q];
    const double s = 0.70710678118654752440;
    auto mod = [](Cd c) { return std::sqrt(c.re * c.re + c.im * c.im); };
    bool balanced = true;
    for (int i = 0; i < 4; ++i) balanced = balanced && std::fabs(mod(u[i]) - s) < 1e-12;
    QOp o;
    o.a = q;
    if (balanced) {
      const Cd l0{u[0].re / s, u[0].im / s}, l1{u[2].re / s, u[2].im / s};
      // w = u01 / u00 (|u00| = s)
      const double n0 = u[0].re * u[0].re + u[0].im * u[0].im;
      const Cd w{(u[1].re * u[0].re + u[1].im * u[0].im) / n0, (u[1].im * u[0].re - u[1].re * u[0].im) / n0};
      // unitarity makes u11 = -l1 s w; anything else is not this form
      const Cd u11 = cmul(l1, Cd{-s * w.re, -s * w.im});
      if (std::fabs(u11.re - u[3].re) < 1e-12 && std::fabs(u11.im - u[3].im) < 1e-12) {
        o.code = OP_BGATE;
        o.m[0] = Cd{s * w.re, s * w.im};
        o.m[1] = Cd{s, 0.0};
        out.push_back(o);
        pend[q] = {l0, Cd{0, 0}, Cd{0, 0}, l1};
        nondiag[q] = 0;
        return;
      }
    }
    o.code = OP_GATE;
    for (int i = 0; i < 4; ++i) o.m[i] = u[i];
    out.push_back(o);
    pend[q] = pauli_matrix(0, 0);
    nondiag[q] = 0;
  }
  void two_diag(uint32_t a, uint32_t b, Cd phase) {
    if (nondiag[a]) emit_gate(a);
    if (nondiag[b]) emit_gate(b);
    QOp o;
    o.a = a;
    o.b = b;
    if (phase.re == -1.0 && phase.im == 0.0) {
      o.code = OP_CZ;
    } else {
      o.code = OP_CPHASE;
      o.m[0] = phase;
    }
    out.push_back(o);
  }
  void finish() {
    for (uint32_t q = 0; q < n; ++q) {
      if (nondiag[q]) {
        emit_gate(q);
      } else if (!is_one(pend[q][0]) || !is_one(pend[q][3])) {
        QOp o;
        o.code = OP_DIAG;
        o.a = q;
        o.m[0] = pend[q][0];
        o.m[1] = pend[q][3];
        out.push_back(o);
      }
    }
  }
};

M2 named_matrix(GateKind k, double theta = 0.0) {
  GateIR g;
  g.kind = k;
  g.theta = theta;
  auto v = gate_matrix(g);
  return {Cd{v[0].re, v[0].im}, Cd{v[1].re, v[1].im}, Cd{v[2].re, v[2].im}, Cd{v[3].re, v[3].im}};
}

void sample_noise(const NoiseIR& nz, const std::vector<uint32_t>& qubits, ncsim_rng& rng, Folder& f, Trajectory& t) {
  const int e = nz.sample(rng);  // always one draw
  if (e < 0) return;
  ++t.noise_events;
  const unsigned x = unsigned(e) & 0xff, z = unsigned(e) >> 8;
  for (size_t j = 0; j < qubits.size(); ++j) {
    const unsigned xj = (x >> j) & 1u, zj = (z >> j) & 1u;
    if (xj || zj) f.one(qubits[j], pauli_matrix(xj, zj));
  }
}

}  // namespace

Trajectory make_random_layers(uint64_t seed, uint32_t n_lo, uint32_t n_span, uint32_t depth, double p) {
  if (n_span < 1) throw Error(NCSIM_ERR_INVALID, "trajectory register span must be at least 1");
  ncsim_rng rng(seed);
  Trajectory t;
  t.n = n_lo + uint32_t(rng.range64(0, n_span));
  if (t.n < MIN_QUBITS || t.n > MAX_QUBITS)
    throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories need 13..26 qubits");
  const uint32_t n = t.n;
  // the circuit first, with the draws of the random-layer text generator
  struct G1 {
    uint32_t q;
    uint8_t kind;  // 0 H, 1 S, 2 T, 3 SqrtX, 4 Rz
    double theta;
  };
  std::vector<G1> ones;
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  ones.reserve(size_t(depth) * n);
  pairs.reserve(size_t(depth) * (n / 2));
  std::vector<uint32_t> perm(n);
  for (uint32_t layer = 0; layer < depth; ++layer) {
    for (uint32_t q = 0; q < n; ++q) {
      const uint64_t g = rng.range64(0, 5);
      G1 o{q, uint8_t(g), 0.0};
      if (g == 4) o.theta = rng.f64() * 6.28318530717958647692;
      ones.push_back(o);
    }
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    for (uint32_t i = n; i-- > 1;) std::swap(perm[i], perm[rng.range32(0, i + 1)]);
    for (uint32_t i = 0; i + 1 < n; i += 2) pairs.emplace_back(perm[i], perm[i + 1]);
  }
  // then the run: gates, one noise draw per DEPOLARIZE2, the measurements
  const M2 mh = named_matrix(GateKind::H), ms = named_matrix(GateKind::S), mt = named_matrix(GateKind::T),
           msx = named_matrix(GateKind::SqrtX);
  NoiseIR nz;
  nz.kind = NoiseKind::Depolarize2;
  nz.p[0] = p;
  Folder f(n, t.ops);
  const uint32_t per = n / 2;
  for (uint32_t layer = 0; layer < depth; ++layer) {
    for (uint32_t q = 0; q < n; ++q) {
      const G1& o = ones[size_t(layer) * n + q];
      switch (o.kind) {
        case 0: f.one(q, mh); break;
        case 1: f.one(q, ms); break;
        case 2: f.one(q, mt); break;
        case 3: f.one(q, msx); break;
        default: f.one(q, named_matrix(GateKind::Rz, o.theta)); break;
      }
    }
    for (uint32_t i = 0; i < per; ++i) {
      const auto& pr = pairs[size_t(layer) * per + i];
      f.two_diag(pr.first, pr.second, Cd{-1.0, 0.0});
      if (p > 0.0) sample_noise(nz, {pr.first, pr.second}, rng, f, t);
    }
  }
  f.finish();
  t.source_gates = uint64_t(depth) * (n + per);
  t.nmeas = n;
  t.draws.resize(n);
  for (auto& d : t.draws) d = rng.f64();
  return t;
}

Trajectory make_from_circuit(const ncsim_circuit& c, uint64_t seed) {
  if (c.n < MIN_QUBITS || c.n > MAX_QUBITS) throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories need 13..26 qubits");
  ncsim_rng rng(seed);
  Trajectory t;
  t.n = c.n;
  Folder f(c.n, t.ops);
  bool measuring = false;
  for (const auto& op : c.ops) {
    switch (op.kind) {
      case OpKind::Gate: {
        if (measuring) throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: gates after the measurements");
        ++t.source_gates;
        const auto m = gate_matrix(op.gate);
        if (op.qubits.size() == 1) {
          f.one(op.qubits[0], {Cd{m[0].re, m[0].im}, Cd{m[1].re, m[1].im}, Cd{m[2].re, m[2].im}, Cd{m[3].re, m[3].im}});
        } else if (op.qubits.size() == 2) {
          for (int r = 0; r < 4; ++r)
            for (int k = 0; k < 4; ++k)
              if (r != k && (m[4 * r + k].re != 0.0 || m[4 * r + k].im != 0.0))
                throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: two-qubit gates must be diagonal");
          for (int r = 0; r < 3; ++r)
            if (m[5 * r].re != 1.0 || m[5 * r].im != 0.0)
              throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: two-qubit diagonals must be controlled phases");
          f.two_diag(op.qubits[0], op.qubits[1], Cd{m[15].re, m[15].im});
        } else {
          throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: gates on more than two qubits");
        }
        break;
      }
      case OpKind::Noise:
        if (measuring) throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: noise after the measurements");
        sample_noise(op.noise, op.qubits, rng, f, t);
        break;
      case OpKind::Measure: {
        const auto& p = op.pauli;
        if (p.x != 0 || p.phase != 0 || p.z != (uint64_t(1) << t.nmeas))
          throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: measurements must be M 0, M 1, ... in order");
        measuring = true;
        ++t.nmeas;
        break;
      }
      case OpKind::Reset: throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories: resets");
      default: break;  // TICK, DETECTOR, OBSERVABLE_INCLUDE: annotations
    }
  }
  f.finish();
  t.draws.resize(t.nmeas);
  for (auto& d : t.draws) d = rng.f64();
  return t;
}

namespace {

std::vector<std::vector<uint32_t>> windows_for(uint32_t n, uint32_t step) {
  std::vector<std::vector<uint32_t>> ws;
  step = std::max<uint32_t>(1, step);
  for (uint32_t g0 = LOW_BITS; g0 < n; g0 += step) {
    std::vector<uint32_t> w;
    for (uint32_t q = 0; q < LOW_BITS; ++q) w.push_back(q);
    for (uint32_t q = g0; q < std::min(n, g0 + TILE_BITS - LOW_BITS); ++q) w.push_back(q);
    for (uint32_t q = n; w.size() < TILE_BITS && q-- > 0;)
      if (std::find(w.begin(), w.end(), q) == w.end()) w.push_back(q);
    std::sort(w.begin(), w.end());
    if (std::find(ws.begin(), ws.end(), w) == ws.end()) ws.push_back(w);
    if (g0 + TILE_BITS - LOW_BITS >= n) break;  // the block reached the top qubit
  }
  return ws;
}

uint64_t qmask(const QOp& o) {
  uint64_t m = uint64_t(1) << o.a;
  if (o.code == OP_CZ || o.code == OP_CPHASE) m |= uint64_t(1) << o.b;
  return m;
}

bool is_gate(const QOp& o) { return o.code == OP_GATE || o.code == OP_BGATE; }

// List scheduling: ops in order.  A gate that cannot go holds back every later
// op on its qubit; a diagonal that cannot go holds back only later gates on
// its qubits (diagonals commute with one another).  Then a taken diagonal
// that no later taken gate on its qubits follows, while the program still has
// a gate on one of them (later[i]), is put back: it waits for the stage of
// that gate, which absorbs its signs.
// Once every qubit of the register (full) is blocked for every op, nothing later
// can be taken: the rest of the list is copied to `rest` at once.
template <class Ok>
void schedule(const std::vector<uint32_t>& pend, const std::vector<QOp>& ops, const std::vector<char>& later, Ok ok,
              uint64_t full, std::vector<uint32_t>& taken, std::vector<uint32_t>& rest) {
  taken.clear();
  rest.clear();
  uint64_t block_all = 0, block_gates = 0;
  for (size_t pi = 0; pi < pend.size(); ++pi) {
    if ((block_all & full) == full) {
      rest.insert(rest.end(), pend.begin() + long(pi), pend.end());
      break;
    }
    const uint32_t i = pend[pi];
    const QOp& o = ops[i];
    const uint64_t m = qmask(o);
    if (is_gate(o)) {
      if ((m & (block_all | block_gates)) || !ok(o)) {
        block_all |= m;
        rest.push_back(i);
      } else {
        taken.push_back(i);
      }
    } else if ((m & block_all) || !ok(o)) {
      block_gates |= m;
      rest.push_back(i);
    } else {
      taken.push_back(i);
    }
  }
  uint64_t gated = 0;
  bool deferred = false;
  for (size_t k = taken.size(); k-- > 0;) {
    const QOp& o = ops[taken[k]];
    const uint64_t m = qmask(o);
    if (is_gate(o)) {
      gated |= m;
    } else if (!(m & gated) && later[taken[k]]) {
      rest.push_back(taken[k]);
      taken[k] = UINT32_MAX;
      deferred = true;
    }
  }
  if (deferred) {
    taken.erase(std::remove(taken.begin(), taken.end(), UINT32_MAX), taken.end());
    std::sort(rest.begin(), rest.end());
  }
}

size_t gate_count(const std::vector<uint32_t>& idx, const std::vector<QOp>& ops) {
  size_t c = 0;
  for (uint32_t i : idx) c += is_gate(ops[i]);
  return c;
}

struct Local {
  std::vector<DevPass> pass;
  std::vector<DevStage> stage;
  std::vector<DevOp> op;
  uint64_t tile_passes = 0, tile_stages = 0;
  double bytes = 0;
};

float f32(double v) { return float(v); }

void compile_one(const Trajectory& t, const PlanKnobs& kn, Local& L) {
  const uint32_t n = t.n;
  const auto ws = windows_for(n, kn.window_step);
  std::vector<std::vector<int>> wpos(ws.size(), std::vector<int>(n, -1));
  for (size_t w = 0; w < ws.size(); ++w)
    for (uint32_t b = 0; b < TILE_BITS; ++b) wpos[w][ws[w][b]] = int(b);
  const uint64_t ntiles = uint64_t(1) << (n - TILE_BITS);
  const uint64_t full = n >= 64 ? ~uint64_t(0) : (uint64_t(1) << n) - 1;

  auto add_pass = [&](size_t w, uint8_t flags) -> DevPass& {
    DevPass p{};
    p.stage0 = uint32_t(L.stage.size());
    p.flags = flags;
    for (uint32_t b = 0; b < TILE_BITS; ++b) p.win[b] = uint8_t(ws[w][b]);
    uint8_t k = 0;
    for (uint32_t q = 0; q < n; ++q)
      if (wpos[w][q] < 0) p.non[k++] = uint8_t(q);
    p.nnon = k;
    L.pass.push_back(p);
    return L.pass.back();
  };

  std::vector<uint32_t> pend(t.ops.size()), taken, rest, staken, srest;
  for (uint32_t i = 0; i < pend.size(); ++i) pend[i] = i;
  // later[i]: a gate on one of op i's qubits comes after it
  std::vector<char> later(t.ops.size(), 0);
  {
    uint64_t seen = 0;
    for (size_t i = t.ops.size(); i-- > 0;) {
      const uint64_t m = qmask(t.ops[i]);
      later[i] = (seen & m) != 0;
      if (is_gate(t.ops[i])) seen |= m;
    }
  }
  size_t last_window = 0, turn = 0;
  bool any = false;
  while (!pend.empty()) {
    size_t best_w = 0;
    std::vector<uint32_t> best_t, best_r;
    for (size_t k = 0; k < ws.size(); ++k) {
      const size_t w = kn.greedy_windows ? k : (turn + k) % ws.size();
      schedule(pend, t.ops, later, [&](const QOp& o) { return !is_gate(o) || wpos[w][o.a] >= 0; }, full, taken, rest);
      if (taken.size() > best_t.size()) {
        best_w = w;
        best_t.swap(taken);  // (taken and rest are cleared by the next schedule)
        best_r.swap(rest);
        if (!kn.greedy_windows) break;
      }
    }
    if (best_t.empty()) throw Error(NCSIM_ERR_INVALID, "batch planner: no window takes the next op");
    if (best_t.size() > MAX_PASS_OPS) {
      // a prefix of a list schedule is itself one: the rest waits for a later pass
      best_r.insert(best_r.end(), best_t.begin() + MAX_PASS_OPS, best_t.end());
      best_t.resize(MAX_PASS_OPS);
      std::sort(best_r.begin(), best_r.end());
    }
    turn = best_w + 1;
    const size_t w = best_w;
    DevPass& ps = add_pass(w, any ? 0 : PASS_ZERO_INIT);
    L.bytes += double(any ? 16 : 8) * double(uint64_t(1) << n);
    any = true;
    last_window = w;
    // stages
    std::vector<uint32_t> sp = best_t;
    uint32_t cyc = 0;
    uint32_t nst = 0;
    while (!sp.empty()) {
      uint32_t best_r_sel = 0;
      std::vector<uint32_t> bt, br;
      size_t bg = 0;
      for (uint32_t k = 0; k < NSEL; ++k) {
        const uint32_t r = kn.greedy_stages ? k : (cyc + k) % NSEL;
        const int lo = int(RSHIFT[r]), hi = lo + int(REG_BITS);
        schedule(sp, t.ops, later,
                 [&](const QOp& o) { return !is_gate(o) || (wpos[w][o.a] >= lo && wpos[w][o.a] < hi); }, full,
                 staken, srest);
        const size_t g = gate_count(staken, t.ops);
        if (bt.empty() || g > bg || (g == bg && staken.size() > bt.size())) {
          best_r_sel = r;
          bt.swap(staken);
          br.swap(srest);
          bg = g;
          if (!kn.greedy_stages && !staken.empty()) break;
        }
      }
      if (bt.empty()) throw Error(NCSIM_ERR_INVALID, "batch planner: no stage takes the next op");
      cyc = best_r_sel + 1;
      const int lo = int(RSHIFT[best_r_sel]);
      auto loc = [&](uint32_t q) -> uint32_t {
        const int b = wpos[w][q];
        if (b >= lo && b < lo + int(REG_BITS)) return (LOC_REG << 5) | uint32_t(b - lo);
        if (b >= 0) return (LOC_FIXED << 5) | uint32_t(b);
        uint32_t k = 0;
        while (ps.non[k] != q) ++k;
        return (LOC_TILE << 5) | k;
      };
      DevStage st{};
      st.op0 = uint32_t(L.op.size());
      st.info = best_r_sel | (uint32_t(bt.size()) << 2);
      for (uint32_t i : bt) {
        const QOp& o = t.ops[i];
        DevOp d{};
        uint32_t la = loc(o.a), lb = 0;
        if (o.code == OP_CZ || o.code == OP_CPHASE) lb = loc(o.b);
        d.hdr = o.code | (la << 3) | (lb << 10);
        if (o.code == OP_CZ) {
          // the register operands' patterns, multiplied here; the device masks in the others' bits
          static const uint32_t pat[REG_BITS] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
          uint32_t m = 0xFFFFFFFFu;
          if ((la >> 5) == LOC_REG) m &= pat[la & 31u];
          if ((lb >> 5) == LOC_REG) m &= pat[lb & 31u];
          std::memcpy(&d.v[0], &m, 4);
        } else if (o.code == OP_GATE) {
          for (int k = 0; k < 4; ++k) {
            d.v[2 * k] = f32(o.m[k].re);
            d.v[2 * k + 1] = f32(o.m[k].im);
          }
        } else if (o.code == OP_BGATE) {
          d.v[0] = f32(o.m[0].re), d.v[1] = f32(o.m[0].im), d.v[2] = f32(o.m[1].re);
        } else if (o.code == OP_DIAG) {
          d.v[0] = f32(o.m[0].re), d.v[1] = f32(o.m[0].im), d.v[2] = f32(o.m[1].re), d.v[3] = f32(o.m[1].im);
        } else if (o.code == OP_CPHASE) {
          d.v[0] = f32(o.m[0].re), d.v[1] = f32(o.m[0].im);
        }
        L.op.push_back(d);
      }
      L.stage.push_back(st);
      ++nst;
      sp.swap(br);
    }
    ps.nstage = uint16_t(nst);
    L.tile_passes += ntiles;
    L.tile_stages += ntiles * nst;
    pend.swap(best_r);
  }
  // the measurement sums need the window of qubits 0..12 in the last pass
  if (!any) {
    add_pass(0, PASS_ZERO_INIT | PASS_ACCUM);
    L.bytes += 8.0 * double(uint64_t(1) << n);
    L.tile_passes += ntiles;
  } else if (last_window == 0) {
    L.pass.back().flags |= PASS_ACCUM;
  } else {
    add_pass(0, PASS_ACCUM | PASS_NO_WRITE);
    L.bytes += 8.0 * double(uint64_t(1) << n);
    L.tile_passes += ntiles;
  }
}

}  // namespace

Program compile(const std::vector<Trajectory>& ts, const PlanKnobs& knobs) {
  return compile(ts, std::vector<PlanKnobs>(MAX_QUBITS + 1, knobs));
}

Program compile(const std::vector<Trajectory>& ts, const std::vector<PlanKnobs>& knobs_by_n) {
  std::vector<Local> loc(ts.size());
  std::atomic<size_t> next{0};
  std::vector<std::string> errs(ts.size());
  auto work = [&] {
    for (size_t i; (i = next.fetch_add(1)) < ts.size();) {
      try {
        compile_one(ts[i], knobs_by_n.at(ts[i].n), loc[i]);
      } catch (const std::exception& e) {
        errs[i] = e.what();
      }
    }
  };
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const unsigned nth = unsigned(std::min<size_t>(hw, std::max<size_t>(1, ts.size() / 8)));
  std::vector<std::thread> th;
  for (unsigned k = 1; k < nth; ++k) th.emplace_back(work);
  work();
  for (auto& x : th) x.join();
  for (auto& e : errs)
    if (!e.empty()) throw Error(NCSIM_ERR_INVALID, e);

  // the trajectories' places in the program (prefix sums), then their parts copied
  // in parallel into the sized (uninitialised) arrays
  Program P;
  std::vector<size_t> p0(ts.size() + 1, 0), s0(ts.size() + 1, 0), o0(ts.size() + 1, 0), d0(ts.size() + 1, 0);
  for (size_t i = 0; i < ts.size(); ++i) {
    p0[i + 1] = p0[i] + loc[i].pass.size();
    s0[i + 1] = s0[i] + loc[i].stage.size();
    o0[i + 1] = o0[i] + loc[i].op.size();
    d0[i + 1] = d0[i] + ts[i].draws.size();
  }
  if (o0.back() > UINT32_MAX || s0.back() > UINT32_MAX || d0.back() > UINT32_MAX)
    throw Error(NCSIM_ERR_UNSUPPORTED, "batch program too large (more than 2^32 ops, stages or draws)");
  P.pass.resize(p0.back());
  P.stage.resize(s0.back());
  P.op.resize(o0.back());
  P.draws.resize(d0.back());
  P.traj.resize(ts.size());
  for (size_t i = 0; i < ts.size(); ++i) {
    const Trajectory& t = ts[i];
    const Local& L = loc[i];
    DevTraj& d = P.traj[i];
    d = DevTraj{};
    d.n = t.n;
    d.npass = uint32_t(L.pass.size());
    d.pass0 = uint32_t(p0[i]);
    d.draw0 = uint32_t(d0[i]);
    d.nmeas = t.nmeas;
    P.source_gates += t.source_gates;
    P.noise_events += t.noise_events;
    P.folded_ops += t.ops.size();
    P.tile_passes += L.tile_passes;
    P.tile_stages += L.tile_stages;
    P.state_bytes += L.bytes;
    P.max_n = std::max(P.max_n, t.n);
  }
  next = 0;
  auto copy = [&] {
    for (size_t i; (i = next.fetch_add(1)) < ts.size();) {
      const Local& L = loc[i];
      for (size_t k = 0; k < L.pass.size(); ++k) {
        DevPass p = L.pass[k];
        p.stage0 += uint32_t(s0[i]);
        P.pass[p0[i] + k] = p;
      }
      for (size_t k = 0; k < L.stage.size(); ++k) {
        DevStage s = L.stage[k];
        s.op0 += uint32_t(o0[i]);
        P.stage[s0[i] + k] = s;
      }
      if (!L.op.empty()) std::memcpy(&P.op[o0[i]], L.op.data(), L.op.size() * sizeof(DevOp));
      if (!ts[i].draws.empty()) std::memcpy(&P.draws[d0[i]], ts[i].draws.data(), ts[i].draws.size() * sizeof(double));
    }
  };
  th.clear();
  for (unsigned k = 1; k < nth; ++k) th.emplace_back(copy);
  copy();
  for (auto& x : th) x.join();
  return P;
}

// ---------------------------------------------------------------------------
// host emulation of the device program (FP64)
// ---------------------------------------------------------------------------
namespace {

uint32_t fixed_index(uint32_t r, uint32_t tid) {
  if (r == 0) return tid << 5;
  if (r == 1) return (tid & 31u) | ((tid >> 5) << 10);
  return tid;
}

uint32_t loc_mask(uint32_t loc, uint32_t fixed, uint64_t tile) {
  static const uint32_t pat[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
  const uint32_t type = loc >> 5, idx = loc & 31u;
  if (type == LOC_REG) return pat[idx];
  const uint64_t bit = type == LOC_FIXED ? (fixed >> idx) & 1u : (tile >> idx) & 1u;
  return bit ? 0xFFFFFFFFu : 0u;
}

// the device's measurement decision (src/state/mod.rs:113-131)
int decide(double e, double nn, const double* draws, uint32_t& used) {
  double p = (1.0 + e / nn) / 2.0;
  if (!std::isnan(p)) p = std::min(1.0, std::max(0.0, p));
  if (p > 1.0 - 1e-12) return 0;
  if (p < 1e-12) return 1;
  return draws[used++] >= p ? 1 : 0;
}

}  // namespace

EmuResult emulate(const Program& P, uint32_t ti) {
  const DevTraj& tr = P.traj.at(ti);
  const uint32_t n = tr.n;
  const uint64_t len = uint64_t(1) << n, ntiles = len >> TILE_BITS;
  std::vector<Cd> st(len, Cd{0, 0});
  std::vector<Cd> tb(TILE);
  std::vector<double> T(TILE, 0.0);
  for (uint32_t pi = 0; pi < tr.npass; ++pi) {
    const DevPass& ps = P.pass[tr.pass0 + pi];
    std::vector<uint64_t> off(TILE);
    for (uint32_t i = 0; i < TILE; ++i) {
      uint64_t o = 0;
      for (uint32_t b = 0; b < TILE_BITS; ++b)
        if ((i >> b) & 1u) o |= uint64_t(1) << ps.win[b];
      off[i] = o;
    }
    if (ps.flags & PASS_ACCUM) std::fill(T.begin(), T.end(), 0.0);
    for (uint64_t k = 0; k < ntiles; ++k) {
      uint64_t base = 0;
      for (uint32_t b = 0; b < ps.nnon; ++b)
        if ((k >> b) & 1u) base |= uint64_t(1) << ps.non[b];
      for (uint32_t i = 0; i < TILE; ++i)
        tb[i] = (ps.flags & PASS_ZERO_INIT) ? Cd{(k == 0 && i == 0) ? 1.0 : 0.0, 0.0} : st[base + off[i]];
      for (uint32_t si = 0; si < ps.nstage; ++si) {
        const DevStage& sg = P.stage[ps.stage0 + si];
        const uint32_t r = sg.info & 3u, nops = sg.info >> 2, sh = RSHIFT[r];
        for (uint32_t tid = 0; tid < THREADS; ++tid) {
          const uint32_t fixed = fixed_index(r, tid);
          Cd a[32];
          for (uint32_t j = 0; j < 32; ++j) a[j] = tb[fixed | (j << sh)];
          uint32_t neg = 0;
          auto flush = [&] {
            for (uint32_t j = 0; j < 32; ++j)
              if ((neg >> j) & 1u) a[j] = Cd{-a[j].re, -a[j].im};
            neg = 0;
          };
          for (uint32_t oi = 0; oi < nops; ++oi) {
            const DevOp& d = P.op[sg.op0 + oi];
            const uint32_t code = d.hdr & 7u, la = (d.hdr >> 3) & 127u, lb = (d.hdr >> 10) & 127u;
            if (code == OP_CZ) {
              neg ^= loc_mask(la, fixed, k) & loc_mask(lb, fixed, k);
              continue;
            }
            flush();
            if (code == OP_BGATE) {
              const uint32_t kb = la & 31u;
              const Cd w{d.v[0], d.v[1]};
              const double sc = d.v[2];
              for (uint32_t j = 0; j < 32; ++j) {
                if ((j >> kb) & 1u) continue;
                const Cd x = a[j], y = cmul(w, a[j | (1u << kb)]);
                a[j] = Cd{sc * x.re + y.re, sc * x.im + y.im};
                a[j | (1u << kb)] = Cd{sc * x.re - y.re, sc * x.im - y.im};
              }
            } else if (code == OP_GATE) {
              const uint32_t kb = la & 31u;
              const Cd u00{d.v[0], d.v[1]}, u01{d.v[2], d.v[3]}, u10{d.v[4], d.v[5]}, u11{d.v[6], d.v[7]};
              for (uint32_t j = 0; j < 32; ++j) {
                if ((j >> kb) & 1u) continue;
                const Cd x = a[j], y = a[j | (1u << kb)];
                a[j] = cadd(cmul(u00, x), cmul(u01, y));
                a[j | (1u << kb)] = cadd(cmul(u10, x), cmul(u11, y));
              }
            } else if (code == OP_DIAG) {
              const uint32_t m = loc_mask(la, fixed, k);
              const Cd d0{d.v[0], d.v[1]}, d1{d.v[2], d.v[3]};
              for (uint32_t j = 0; j < 32; ++j) a[j] = cmul(a[j], ((m >> j) & 1u) ? d1 : d0);
            } else {
              const uint32_t m = loc_mask(la, fixed, k) & loc_mask(lb, fixed, k);
              const Cd ph{d.v[0], d.v[1]};
              for (uint32_t j = 0; j < 32; ++j)
                if ((m >> j) & 1u) a[j] = cmul(a[j], ph);
            }
          }
          flush();
          for (uint32_t j = 0; j < 32; ++j) tb[fixed | (j << sh)] = a[j];
        }
      }
      if (!(ps.flags & PASS_NO_WRITE))
        for (uint32_t i = 0; i < TILE; ++i) st[base + off[i]] = tb[i];
      if (ps.flags & PASS_ACCUM)
        for (uint32_t i = 0; i < TILE; ++i) T[i] += tb[i].re * tb[i].re + tb[i].im * tb[i].im;
    }
  }
  // measurements: Z marginals over the low 13 qubits, then over the rest
  EmuResult res;
  const double* draws = P.draws.data() + tr.draw0;
  uint32_t used = 0;
  uint64_t o = 0;
  const uint32_t kl = std::min<uint32_t>(tr.nmeas, TILE_BITS);
  for (uint32_t k = 0; k < std::max<uint32_t>(kl, 1); ++k) {
    double s[2] = {0.0, 0.0};
    for (uint32_t rr = 0; rr < (TILE >> k); ++rr) s[rr & 1u] += T[o | (uint64_t(rr) << k)];
    const double e = s[0] - s[1], nn = s[0] + s[1];
    if (k == 0) {
      res.z0 = e / nn;
      res.norm = nn;
    }
    if (k < tr.nmeas) o |= uint64_t(decide(e, nn, draws, used)) << k;
  }
  if (tr.nmeas > TILE_BITS) {
    const uint64_t nh = len >> TILE_BITS;
    std::vector<double> G(nh);
    for (uint64_t h = 0; h < nh; ++h) {
      const Cd v = st[o | (h << TILE_BITS)];
      G[h] = v.re * v.re + v.im * v.im;
    }
    uint64_t oh = 0;
    for (uint32_t k = TILE_BITS; k < tr.nmeas; ++k) {
      const uint32_t kk = k - TILE_BITS;
      double s[2] = {0.0, 0.0};
      for (uint64_t rr = 0; rr < (nh >> kk); ++rr) s[rr & 1u] += G[oh | (rr << kk)];
      const double e = s[0] - s[1], nn = s[0] + s[1];
      oh |= uint64_t(decide(e, nn, draws, used)) << kk;
    }
    o |= oh << TILE_BITS;
  }
  res.record = o;
  return res;
}

}  // namespace ncsim::batch
