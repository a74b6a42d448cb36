// The trait's provided methods on the device state (src/state/mod.rs:93-234)
// and the C ABI of the host layer: RNG, circuits, gates, run/measure/sample.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>

#include "ir.hpp"

using namespace ncsim;

namespace ncsim {

PolyTerms build_poly_terms(const PhasePolyIR& p, const std::vector<uint32_t>& qubits, const Phase& scalar);

struct PlainPlan;
std::shared_ptr<PlainPlan> plan_plain_passes(uint32_t n, int precision, const std::vector<const LoweredOp*>& gates);
void run_plain_plan(ncsim_state* s, PlainPlan& P);
size_t plain_plan_passes(const PlainPlan& P);
size_t plain_plan_pass_gates(const PlainPlan& P);

void apply_lowered(ncsim_state* s, const LoweredOp& op) {
  switch (op.kind) {
    case LoweredKind::Nothing: return;
    case LoweredKind::Dense: launch_dense(s, op.qubits, op.matrix); return;
    case LoweredKind::Monomial: launch_perm_table(s, op.qubits, op.image, op.matrix); return;
    case LoweredKind::PhasePoly: launch_phasepoly(s, op.poly); return;
    case LoweredKind::Pauli: launch_pauli(s, op.x, op.z, op.phase); return;
  }
}

// QuantumState::measure (mod.rs:113-131); expectation and norm in one pass
bool measure_op(ncsim_state* s, const PauliOp& p, ncsim_rng& rng) {
  if (!p.hermitian()) throw Error(NCSIM_ERR_INVALID, "measured operator is not Hermitian");
  if (p.n != s->n) throw Error(NCSIM_ERR_INVALID, "expectation: operator on the wrong register");
  double e[2], nn;
  state_measure_stats(s, p.x, p.z, p.phase, e, &nn);
  double p_plus = (1.0 + e[0] / nn) / 2.0;
  if (!std::isnan(p_plus)) p_plus = std::min(1.0, std::max(0.0, p_plus));
  bool outcome;
  if (p_plus > 1.0 - 1e-12) outcome = false;
  else if (p_plus < 1e-12) outcome = true;
  else outcome = rng.f64() >= p_plus;
  state_project(s, p.x, p.z, p.phase, outcome);
  return outcome;
}

// QuantumState::apply_op (mod.rs:134-165); returns -1, 0 or 1
int apply_op(ncsim_state* s, const OpIR& op, ncsim_rng& rng) {
  switch (op.kind) {
    case OpKind::Gate: apply_lowered(s, op.lowered); return -1;
    case OpKind::Measure: return measure_op(s, op.pauli, rng) ? 1 : 0;
    case OpKind::Reset: {
      PauliOp z;
      z.n = s->n;
      z.z = uint64_t(1) << op.qubits[0];
      if (measure_op(s, z, rng)) launch_pauli(s, uint64_t(1) << op.qubits[0], 0, 0);
      return -1;
    }
    case OpKind::Noise: {
      int e = op.noise.sample(rng);
      if (e >= 0) {
        // raw X^x Z^z bits with phase 0 (mod.rs:148-162)
        uint64_t x = 0, z = 0;
        for (size_t j = 0; j < op.qubits.size(); ++j) {
          x |= uint64_t((e >> j) & 1) << op.qubits[j];
          z |= uint64_t((e >> (8 + j)) & 1) << op.qubits[j];
        }
        launch_pauli(s, x, z, 0);
      }
      return -1;
    }
    default: return -1;
  }
}

}  // namespace ncsim

namespace {
void need(const void* p, const char* what) {
  if (!p) throw Error(NCSIM_ERR_INVALID, std::string(what) + " is null");
}
}  // namespace

extern "C" {

// ---- rng ----
ncsim_status ncsim_rng_new(uint64_t seed, ncsim_rng** out) {
  return guarded([&] {
    need(out, "out");
    *out = new ncsim_rng(seed);
  });
}
ncsim_status ncsim_rng_free(ncsim_rng* r) {
  return guarded([&] { delete r; });
}
ncsim_status ncsim_rng_next_u64(ncsim_rng* r, uint64_t* out) {
  return guarded([&] {
    need(r, "rng");
    need(out, "out");
    *out = r->u64();
  });
}
ncsim_status ncsim_rng_next_u32(ncsim_rng* r, uint32_t* out) {
  return guarded([&] {
    need(r, "rng");
    need(out, "out");
    *out = r->u32();
  });
}
ncsim_status ncsim_rng_gen_f64(ncsim_rng* r, double* out) {
  return guarded([&] {
    need(r, "rng");
    need(out, "out");
    *out = r->f64();
  });
}
ncsim_status ncsim_rng_gen_range(ncsim_rng* r, uint64_t lo, uint64_t hi, uint64_t* out) {
  return guarded([&] {
    need(r, "rng");
    need(out, "out");
    if (hi <= lo) throw Error(NCSIM_ERR_INVALID, "gen_range: empty range");
    *out = r->range64(lo, hi);
  });
}

// ---- circuits ----
ncsim_status ncsim_circuit_parse(const char* text, ncsim_circuit** out) {
  return guarded([&] {
    need(text, "text");
    need(out, "out");
    *out = nullptr;
    *out = new ncsim_circuit(parse_circuit(text));
  });
}
ncsim_status ncsim_circuit_free(ncsim_circuit* c) {
  return guarded([&] { delete c; });
}
ncsim_status ncsim_circuit_info(const ncsim_circuit* c, uint32_t* nq, uint64_t* nops, uint64_t* ng, uint64_t* nm) {
  return guarded([&] {
    need(c, "circuit");
    if (nq) *nq = c->n;
    if (nops) *nops = c->ops.size();
    if (ng) *ng = c->num_gates();
    if (nm) *nm = c->num_measurements();
  });
}
ncsim_status ncsim_circuit_to_text(const ncsim_circuit* c, char* buf, size_t cap, size_t* len) {
  return guarded([&] {
    need(c, "circuit");
    std::string t = c->text();
    if (len) *len = t.size();
    if (buf && cap > t.size()) std::memcpy(buf, t.c_str(), t.size() + 1);
  });
}
// ---- gates ----
ncsim_status ncsim_gate_parse(const char* token, uint32_t arity_hint, ncsim_gate** out, uint32_t* arity) {
  return guarded([&] {
    need(token, "token");
    need(out, "out");
    *out = nullptr;
    auto* g = new ncsim_gate();
    try {
      g->g = parse_gate_token(token, arity_hint);
    } catch (...) {
      delete g;
      throw;
    }
    if (arity) *arity = g->g.arity();
    *out = g;
  });
}
ncsim_status ncsim_gate_unitary(uint32_t k, const double* m, ncsim_gate** out) {
  return guarded([&] {
    need(m, "matrix");
    need(out, "out");
    if (k < 1 || k > uint32_t(MAX_WIDE_DENSE_K))
      throw Error(NCSIM_ERR_UNSUPPORTED, "dense gates on 1.." + std::to_string(MAX_WIDE_DENSE_K) + " qubits");
    auto* g = new ncsim_gate();
    g->g.kind = GateKind::Unitary;
    g->g.uk = k;
    const size_t d = size_t(1) << k;
    g->g.umat.resize(d * d);
    for (size_t i = 0; i < d * d; ++i) g->g.umat[i] = {m[2 * i], m[2 * i + 1]};
    *out = g;
  });
}
ncsim_status ncsim_gate_pauli(uint32_t k, uint64_t x, uint64_t z, uint32_t phase, ncsim_gate** out) {
  return guarded([&] {
    need(out, "out");
    if (k > 64) throw Error(NCSIM_ERR_INVALID, "Pauli on more than 64 qubits");
    const uint64_t mask = k >= 64 ? ~uint64_t(0) : ((uint64_t(1) << k) - 1);
    auto* g = new ncsim_gate();
    g->g.kind = GateKind::Pauli;
    g->g.pauli.n = k;
    g->g.pauli.x = x & mask;
    g->g.pauli.z = z & mask;
    g->g.pauli.phase = phase & 3;
    *out = g;
  });
}
ncsim_status ncsim_gate_free(ncsim_gate* g) {
  return guarded([&] { delete g; });
}
ncsim_status ncsim_gate_lowered_matrix(const ncsim_gate* g, double* out, size_t cap, uint32_t* kout) {
  return guarded([&] {
    need(g, "gate");
    need(out, "out");
    const uint32_t k = g->g.arity();
    if (k < 1 || k > 8) throw Error(NCSIM_ERR_UNSUPPORTED, "lowered matrices of 1..8 qubits");
    const size_t d = size_t(1) << k;
    if (cap < 2 * d * d) throw Error(NCSIM_ERR_INVALID, "output buffer too small");
    std::vector<uint32_t> qs(k);
    for (uint32_t j = 0; j < k; ++j) qs[j] = j;
    LoweredOp op = lower_gate(g->g, qs, k);
    std::vector<CplxD> m(d * d, CplxD{0, 0});
    switch (op.kind) {
      case LoweredKind::Dense: m = op.matrix; break;
      case LoweredKind::Monomial:
        for (size_t x = 0; x < d; ++x) m[size_t(op.image[x]) * d + x] = op.matrix[x];
        break;
      case LoweredKind::PhasePoly:
        for (uint64_t x = 0; x < d; ++x) {
          uint64_t f = op.poly.constant;
          for (size_t t = 0; t + 1 < op.poly.term_start.size(); ++t) {
            bool all = true;
            for (uint32_t l = op.poly.term_start[t]; l < op.poly.term_start[t + 1]; ++l)
              all &= bool(__builtin_popcountll(op.poly.parities[l] & x) & 1);
            if (all) f += op.poly.coeffs[t];
          }
          f &= (uint64_t(1) << op.poly.bits) - 1;
          Cd r = root_value(int64_t(f), op.poly.bits);
          CplxD c = op.poly.root_table.empty()
                        ? CplxD{op.poly.scalar.re * r.re - op.poly.scalar.im * r.im, op.poly.scalar.re * r.im + op.poly.scalar.im * r.re}
                        : op.poly.root_table[f];
          m[x * d + x] = c;
        }
        break;
      case LoweredKind::Pauli:
        for (uint64_t x = 0; x < d; ++x) {
          int kk = int(op.phase + 2 * __builtin_popcountll(op.z & x)) & 3;
          static const CplxD ip[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
          m[(x ^ op.x) * d + x] = ip[kk];
        }
        break;
      case LoweredKind::Nothing:
        for (size_t x = 0; x < d; ++x) m[x * d + x] = {1, 0};
        break;
    }
    for (size_t i = 0; i < d * d; ++i) out[2 * i] = m[i].re, out[2 * i + 1] = m[i].im;
    if (kout) *kout = k;
  });
}
ncsim_status ncsim_pauli_parse(const char* text, uint32_t n, uint64_t* x, uint64_t* z, uint32_t* phase) {
  return guarded([&] {
    need(text, "text");
    PauliOp p = parse_pauli(text, int64_t(n));
    if (x) *x = p.x;
    if (z) *z = p.z;
    if (phase) *phase = p.phase;
  });
}

ncsim_status ncsim_pauli_parse_words(const char* text, uint32_t n, uint64_t* x, uint64_t* z, uint32_t words,
                                     uint32_t* phase) {
  return guarded([&] {
    need(text, "text");
    const PauliSites ps = parse_pauli_sites(text, int64_t(n));
    if (uint64_t(words) * 64 < ps.n) throw Error(NCSIM_ERR_INVALID, "too few words for the Pauli's register");
    uint32_t ys = 0;
    for (uint32_t w = 0; w < words; ++w) {
      if (x) x[w] = 0;
      if (z) z[w] = 0;
    }
    for (const auto& st : ps.sites) {  // Y = i X Z: a Y site adds one to the phase
      const uint32_t q = st.first;
      if ((st.second & 1) && x) x[q >> 6] |= uint64_t(1) << (q & 63);
      if ((st.second & 2) && z) z[q >> 6] |= uint64_t(1) << (q & 63);
      ys += st.second == 3;
    }
    if (phase) *phase = (ps.phase + ys) & 3u;
  });
}

// ---- trait methods on the device state ----
ncsim_status ncsim_sv_apply_gate(ncsim_state* s, const ncsim_gate* g, const uint32_t* qubits, uint32_t k) {
  return guarded([&] {
    need(s, "state");
    need(g, "gate");
    if (k) need(qubits, "qubits");
    LoweredOp op = lower_gate(g->g, std::vector<uint32_t>(qubits, qubits + k), s->n);
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    apply_lowered(s, op);
  });
}

ncsim_status ncsim_sv_measure(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, ncsim_rng* rng, int32_t* outcome) {
  return guarded([&] {
    need(s, "state");
    need(rng, "rng");
    need(outcome, "out");
    PauliOp p;
    p.n = s->n;
    p.x = x;
    p.z = z;
    p.phase = phase & 3;
    if ((x | z) >> s->n && s->n < 64) throw Error(NCSIM_ERR_INVALID, "Pauli acts outside the register");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    *outcome = measure_op(s, p, *rng) ? 1 : 0;
  });
}

}  // extern "C"

namespace {

// Runs of at least MIN_GRAPH_GATES consecutive gates (annotations between them
// allowed) are captured as CUDA graphs on the second run of a circuit on a
// state and replayed by every later run: one graph launch instead of a host
// lowering step and a kernel launch per gate.  A circuit run only once (a
// noisy trajectory drawn for one run) launches its kernels directly and pays
// no capture.  Measurements, resets and
// noise stay outside the graphs (their draws and decisions are made on the
// host).  A run's gates go through tiled passes (plain_pass.cu) unless the
// state turns them off or the environment sets NCSIM_NO_TILE_PASSES.  No graph
// is captured while the launch profiler records per-launch events; the
// environment variable NCSIM_NO_GATE_GRAPHS turns runs off altogether
// (kernel-by-kernel launches).
constexpr size_t MIN_GRAPH_GATES = 16;

struct GateGraphs {
  uint64_t state_uid = 0;
  int device = -1;
  std::vector<std::pair<size_t, size_t>> runs;  // [first op, end op) of each run
  std::vector<cudaGraphExec_t> exec;            // null until captured
  std::vector<char> seen;                       // the run has been launched directly once
  std::vector<char> failed;                     // capture did not succeed: launch directly
  std::vector<std::shared_ptr<PlainPlan>> plans;  // tiled passes of each run (null: gate by gate)
  std::vector<char> planned;
  std::vector<char> plan_on;                    // the state's pass setting the plan was made under
  ~GateGraphs() {
    for (auto e : exec)
      if (e) cudaGraphExecDestroy(e);
  }
};

std::mutex g_graph_mu;

bool annotation(OpKind k) { return k == OpKind::Tick || k == OpKind::Detector || k == OpKind::Observable; }

std::shared_ptr<GateGraphs> gate_graphs_for(const ncsim_circuit* c, const ncsim_state* s) {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  auto g = std::static_pointer_cast<GateGraphs>(c->gate_graphs);
  if (g && g->state_uid == s->uid && g->device == s->device) return g;
  g = std::make_shared<GateGraphs>();
  g->state_uid = s->uid;
  g->device = s->device;
  for (size_t i = 0; i < c->ops.size();) {
    if (c->ops[i].kind != OpKind::Gate) {
      ++i;
      continue;
    }
    size_t j = i, gates = 0;
    while (j < c->ops.size() && (c->ops[j].kind == OpKind::Gate || annotation(c->ops[j].kind))) {
      gates += c->ops[j].kind == OpKind::Gate;
      ++j;
    }
    if (gates >= MIN_GRAPH_GATES) g->runs.push_back({i, j});
    i = j;
  }
  g->exec.assign(g->runs.size(), nullptr);
  g->seen.assign(g->runs.size(), 0);
  g->failed.assign(g->runs.size(), 0);
  g->plans.assign(g->runs.size(), nullptr);
  g->planned.assign(g->runs.size(), 0);
  g->plan_on.assign(g->runs.size(), 0);
  c->gate_graphs = g;
  return g;
}

// the gates of run k: through its tiled passes when the state uses them
void launch_run(ncsim_state* s, const ncsim_circuit* c, GateGraphs& g, size_t k) {
  const auto [first, end] = g.runs[k];
  if (g.plans[k]) {
    run_plain_plan(s, *g.plans[k]);
    return;
  }
  for (size_t i = first; i < end; ++i)
    if (c->ops[i].kind == OpKind::Gate) apply_lowered(s, c->ops[i].lowered);
}

// Launches the gates of ops[first, end) on the state's stream, as a graph when it can.
void run_gates(ncsim_state* s, const ncsim_circuit* c, GateGraphs& g, size_t k) {
  const auto [first, end] = g.runs[k];
  static const bool passes_off = std::getenv("NCSIM_NO_TILE_PASSES") != nullptr;
  const bool want = s->tile_passes && !passes_off;
  if (!g.planned[k] || bool(g.plan_on[k]) != want) {
    // a new plan drops the graph captured under the other setting
    if (g.exec[k]) {
      cudaGraphExecDestroy(g.exec[k]);
      g.exec[k] = nullptr;
    }
    g.plans[k] = nullptr;
    if (want) {
      std::vector<const LoweredOp*> gates;
      for (size_t i = first; i < end; ++i)
        if (c->ops[i].kind == OpKind::Gate) gates.push_back(&c->ops[i].lowered);
      g.plans[k] = plan_plain_passes(s->n, s->precision, gates);
    }
    g.planned[k] = 1;
    g.plan_on[k] = want ? 1 : 0;
    g.seen[k] = 0;
    g.failed[k] = 0;
  }
  if (s->prof) {  // the launch profiler times every launch: no graph
    launch_run(s, c, g, k);
    return;
  }
  if (!g.exec[k] && !g.failed[k] && g.seen[k]) {
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      try {
        launch_run(s, c, g, k);
      } catch (...) {
        ok = false;
      }
      ok = cudaStreamEndCapture(s->stream, &graph) == cudaSuccess && ok;
      cudaGraphExec_t e = nullptr;
      if (ok) ok = cudaGraphInstantiate(&e, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
      if (ok) g.exec[k] = e;
    }
    if (!ok) {
      cudaGetLastError();  // a failed capture leaves only its own error behind
      g.failed[k] = 1;
    }
  }
  g.seen[k] = 1;
  if (g.exec[k]) {
    NCSIM_CUDA(cudaGraphLaunch(g.exec[k], s->stream));
  } else {
    launch_run(s, c, g, k);
  }
}

}  // namespace

extern "C" {

ncsim_status ncsim_sv_run(ncsim_state* s, const ncsim_circuit* c, ncsim_rng* rng, uint8_t* rec, size_t cap, size_t* len) {
  return guarded([&] {
    need(s, "state");
    need(c, "circuit");
    need(rng, "rng");
    if (c->n != s->n)
      throw Error(NCSIM_ERR_INVALID, "circuit on " + std::to_string(c->n) + " qubits, state on " + std::to_string(s->n));
    if (c->num_measurements() > cap) throw Error(NCSIM_ERR_INVALID, "record buffer too small");
    if (c->num_measurements()) need(rec, "record");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    static const bool graphs_off = std::getenv("NCSIM_NO_GATE_GRAPHS") != nullptr;
    std::shared_ptr<GateGraphs> g;
    if (!graphs_off) g = gate_graphs_for(c, s);
    size_t m = 0, k = 0;
    for (size_t i = 0; i < c->ops.size();) {
      if (g && k < g->runs.size() && g->runs[k].first == i) {
        run_gates(s, c, *g, k);
        i = g->runs[k++].second;
        continue;
      }
      int r = apply_op(s, c->ops[i], *rng);
      if (r >= 0) rec[m++] = uint8_t(r);
      ++i;
    }
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    if (len) *len = m;
  });
}

ncsim_status ncsim_sv_sample_rng(const ncsim_state* s, ncsim_rng* rng, uint64_t shots, uint64_t* out) {
  return guarded([&] {
    need(s, "state");
    need(rng, "rng");
    std::vector<double> u(shots);
    for (auto& v : u) v = rng->f64();  // drawn first, in shot order (vector.rs:505)
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_sample(s, u.data(), shots, out);
  });
}

ncsim_status ncsim_sv_normalize(ncsim_state* s) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    const double nn = state_norm_sq(s).re;
    if (!(nn > 0.0)) throw Error(NCSIM_ERR_ZERO_STATE, "state vanished: normalize");
    const double l = -std::log2(nn);
    double c;
    if (std::fabs(l - std::round(l)) < 1e-9) c = sqrt2_power(int64_t(std::round(l)));
    else c = 1.0 / std::sqrt(nn);
    launch_scale(s, {c, 0.0});
  });
}

ncsim_status ncsim_sv_probability(const ncsim_state* s, uint64_t index, double* out) {
  return guarded([&] {
    need(s, "state");
    need(out, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    double a[2];
    uint64_t i = s->n >= 64 ? index : (index & ((uint64_t(1) << s->n) - 1));
    state_gather(s, &i, 1, a);
    *out = (a[0] * a[0] + a[1] * a[1]) / state_norm_sq(s).re;
  });
}

ncsim_status ncsim_sv_expectation_sum(const ncsim_state* s, uint64_t count, const uint64_t* x, const uint64_t* z,
                                      const uint32_t* phase, const double* coeffs, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    if (count) {
      need(x, "x");
      need(z, "z");
      need(phase, "phase");
      need(coeffs, "coeffs");
    }
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    std::vector<CplxD> t(count);
    for (uint64_t k = 0; k < count; ++k) {
      CplxD e = state_expectation(s, x[k], z[k], phase[k] & 3);
      const double cr = coeffs[2 * k], ci = coeffs[2 * k + 1];
      t[k] = {cr * e.re - ci * e.im, cr * e.im + ci * e.re};
    }
    // Amplitude::sum (scalar.rs:80-94): pairwise, leaves of at most 8
    struct Rec {
      static CplxD sum(const CplxD* v, size_t n) {
        if (n <= 8) {
          CplxD a{0, 0};
          for (size_t i = 0; i < n; ++i) a = {a.re + v[i].re, a.im + v[i].im};
          return a;
        }
        CplxD l = sum(v, n / 2), r = sum(v + n / 2, n - n / 2);
        return {l.re + r.re, l.im + r.im};
      }
    };
    CplxD r = Rec::sum(t.data(), t.size());
    re_im[0] = r.re;
    re_im[1] = r.im;
  });
}

ncsim_status ncsim_sv_run_fused(ncsim_state* s, const ncsim_circuit* c, ncsim_rng* rng, uint32_t max_fuse, uint8_t* rec,
                                size_t cap, size_t* len, ncsim_fused_stats* stats);

}  // extern "C"
