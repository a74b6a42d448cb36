// CPU ORACLE — test infrastructure only (see ncsim_ref.hpp).
//
// A flat C interface to the restatement so that pytest (ctypes) and the CPU
// baseline leg of bench.py can drive it.  Errors return a negative status and
// leave a message in oracle_last_error().
#include "frames_ref.hpp"
#include "ncsim_ref.hpp"
#include "sparse_wide_ref.hpp"
#include "workloads_ref.hpp"

#include <chrono>
#include <cstdio>

using namespace ref;

namespace {
thread_local std::string g_err;

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (SimError& e) {
    g_err = e.what();
    return -int(e.kind);
  } catch (std::exception& e) {
    g_err = e.what();
    return -100;
  }
}

int copy_text(const std::string& s, char* buf, size_t cap) {
  if (buf && cap > s.size()) std::memcpy(buf, s.c_str(), s.size() + 1);
  return int(s.size());
}

std::vector<size_t> qlist(const uint32_t* q, uint32_t k) { return std::vector<size_t>(q, q + k); }
}  // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }
int oracle_num_threads() { return omp_get_max_threads(); }
void oracle_set_threads(int t) { omp_set_num_threads(t); }

// ---- StdRng ----
void* oracle_rng_new(uint64_t seed) { return new StdRng(StdRng::seed_from_u64(seed)); }
void oracle_rng_free(void* r) { delete (StdRng*)r; }
uint64_t oracle_rng_next_u64(void* r) { return ((StdRng*)r)->next_u64(); }
uint32_t oracle_rng_next_u32(void* r) { return ((StdRng*)r)->next_u32(); }
double oracle_rng_gen_f64(void* r) { return ((StdRng*)r)->gen_f64(); }
uint64_t oracle_rng_gen_range(void* r, uint64_t lo, uint64_t hi) { return ((StdRng*)r)->gen_range_u64(lo, hi); }
// One ChaCha block with `rounds` rounds over the given key and 64-bit counter.
void oracle_chacha_block(const uint32_t* key, uint64_t counter, int rounds, uint32_t* out) {
  StdRng r;
  std::memcpy(r.key, key, 32);
  r.block_at(counter, out, rounds);
}

// ---- workloads ----
int oracle_random_circuit_text(uint32_t n, uint32_t depth, uint64_t seed, double noise_p, uint32_t m_lo, uint32_t m_hi,
                               char* buf, size_t cap) {
  StdRng rng = StdRng::seed_from_u64(seed);
  return copy_text(random_circuit_text(n, depth, rng, noise_p, m_lo, m_hi), buf, cap);
}
int oracle_frames_circuit_text(uint32_t n, uint32_t rounds, uint32_t meas, double p, uint64_t seed, char* buf,
                               size_t cap) {
  StdRng rng = StdRng::seed_from_u64(seed);
  return copy_text(frames_circuit_text(n, rounds, meas, p, rng), buf, cap);
}
int oracle_reversible_circuit_text(uint32_t n, uint32_t gates, uint64_t seed, char* buf, size_t cap) {
  StdRng rng = StdRng::seed_from_u64(seed);
  return copy_text(reversible_circuit_text(n, gates, rng), buf, cap);
}

// ---- circuits ----
void* oracle_circuit_parse(const char* text) {
  Circuit* c = nullptr;
  int st = guard([&] { c = new Circuit(Circuit::parse(text)); });
  return st == 0 ? c : nullptr;
}
void oracle_circuit_free(void* c) { delete (Circuit*)c; }
uint32_t oracle_circuit_num_qubits(void* c) { return uint32_t(((Circuit*)c)->n); }
uint32_t oracle_circuit_num_gates(void* c) { return uint32_t(((Circuit*)c)->num_gates()); }
uint32_t oracle_circuit_num_measurements(void* c) { return uint32_t(((Circuit*)c)->num_measurements()); }

// Gate::matrix() of the gate on line 1 of `text` (a one-gate circuit), written
// as 2*4^k doubles; returns k, or a negative status.
int oracle_gate_matrix(const char* text, double* out, size_t cap_doubles) {
  int k = -1;
  int st = guard([&] {
    Circuit c = Circuit::parse(text);
    if (c.ops.empty() || c.ops[0].kind != OpKind::GateOp) throw SimError(ErrKind::Invalid, "no gate");
    auto m = c.ops[0].gate.matrix();
    if (!m) throw SimError(ErrKind::NotRepresentable, "no matrix");
    if (m->size() * 2 > cap_doubles) throw SimError(ErrKind::Invalid, "buffer too small");
    for (size_t i = 0; i < m->size(); ++i) out[2 * i] = (*m)[i].re, out[2 * i + 1] = (*m)[i].im;
    k = int(c.ops[0].gate.arity());
  });
  return st == 0 ? k : st;
}
// The same gate's dagger's matrix.
int oracle_gate_dagger_matrix(const char* text, double* out, size_t cap_doubles) {
  int k = -1;
  int st = guard([&] {
    Circuit c = Circuit::parse(text);
    auto m = c.ops.at(0).gate.dagger().matrix();
    if (!m || m->size() * 2 > cap_doubles) throw SimError(ErrKind::Invalid, "no matrix");
    for (size_t i = 0; i < m->size(); ++i) out[2 * i] = (*m)[i].re, out[2 * i + 1] = (*m)[i].im;
    k = int(c.ops[0].gate.arity());
  });
  return st == 0 ? k : st;
}

// ---- dense state ----
void* oracle_sv_new(uint32_t n) {
  StateVector* s = nullptr;
  int st = guard([&] { s = new StateVector(StateVector::zero_state(n)); });
  return st == 0 ? s : nullptr;
}
void* oracle_sv_plus(uint32_t n) { return new StateVector(StateVector::plus_state(n)); }
void* oracle_sv_clone(void* h) { return new StateVector(*(StateVector*)h); }
void oracle_sv_free(void* h) { delete (StateVector*)h; }
int oracle_sv_set_amplitudes(void* h, const double* a, uint64_t len) {
  return guard([&] {
    auto* s = (StateVector*)h;
    if (len != s->amp.size()) throw SimError(ErrKind::Invalid, "length");
    for (uint64_t i = 0; i < len; ++i) s->amp[i] = C64(a[2 * i], a[2 * i + 1]);
  });
}
// amplitudes [first, first + count) from interleaved host doubles
int oracle_sv_set_range(void* h, const double* a, uint64_t first, uint64_t count) {
  return guard([&] {
    auto* s = (StateVector*)h;
    if (first > s->amp.size() || count > s->amp.size() - first) throw SimError(ErrKind::Invalid, "range");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(count); ++i) s->amp[first + i] = C64(a[2 * i], a[2 * i + 1]);
  });
}
// max |amp[first + i] - a[i]| over the range
int oracle_sv_max_abs_diff(void* h, const double* a, uint64_t first, uint64_t count, double* out) {
  return guard([&] {
    auto* s = (StateVector*)h;
    if (first > s->amp.size() || count > s->amp.size() - first) throw SimError(ErrKind::Invalid, "range");
    double m = 0.0;
#pragma omp parallel for schedule(static) reduction(max : m)
    for (int64_t i = 0; i < int64_t(count); ++i) {
      const C64 v = s->amp[first + i];
      m = std::max(m, std::hypot(v.re - a[2 * i], v.im - a[2 * i + 1]));
    }
    *out = m;
  });
}

int oracle_sv_get_amplitudes(void* h, double* a, uint64_t len) {
  return guard([&] {
    auto* s = (StateVector*)h;
    if (len != s->amp.size()) throw SimError(ErrKind::Invalid, "length");
    for (uint64_t i = 0; i < len; ++i) a[2 * i] = s->amp[i].re, a[2 * i + 1] = s->amp[i].im;
  });
}
int oracle_sv_apply_gate_text(void* h, const char* text) {
  return guard([&] {
    auto* s = (StateVector*)h;
    std::string t = "QUBITS " + std::to_string(s->n) + "\n" + text;
    Circuit c = Circuit::parse(t);
    for (auto& op : c.ops)
      if (op.kind == OpKind::GateOp) s->apply_gate(op.gate, op.qubits);
  });
}
int oracle_sv_apply_matrix(void* h, const uint32_t* q, uint32_t k, const double* m) {
  return guard([&] {
    size_t gd = size_t(1) << k;
    std::vector<C64> mm(gd * gd);
    for (size_t i = 0; i < gd * gd; ++i) mm[i] = C64(m[2 * i], m[2 * i + 1]);
    ((StateVector*)h)->apply_matrix(mm, qlist(q, k));
  });
}
int oracle_sv_apply_pauli(void* h, const char* pauli) {
  return guard([&] {
    auto* s = (StateVector*)h;
    s->apply_pauli(Pauli::from_string(s->n, pauli));
  });
}
int oracle_sv_apply_pauli_raw(void* h, uint64_t x, uint64_t z, uint32_t phase) {
  return guard([&] {
    auto* s = (StateVector*)h;
    s->apply_pauli(Pauli::make(s->n, x, z, uint8_t(phase)));
  });
}
int oracle_sv_norm_sq(void* h, double* out) {
  return guard([&] {
    C64 v = ((StateVector*)h)->norm_sq();
    out[0] = v.re, out[1] = v.im;
  });
}
int oracle_sv_expectation(void* h, const char* pauli, double* out) {
  return guard([&] {
    auto* s = (StateVector*)h;
    C64 v = s->expectation(Pauli::from_string(s->n, pauli));
    out[0] = v.re, out[1] = v.im;
  });
}
int oracle_sv_expectation_raw(void* h, uint64_t x, uint64_t z, uint32_t phase, double* out) {
  return guard([&] {
    auto* s = (StateVector*)h;
    C64 v = s->expectation(Pauli::make(s->n, x, z, uint8_t(phase)));
    out[0] = v.re, out[1] = v.im;
  });
}
int oracle_sv_inner(void* h, void* o, double* out) {
  return guard([&] {
    C64 v = ((StateVector*)h)->inner(*(StateVector*)o);
    out[0] = v.re, out[1] = v.im;
  });
}
int oracle_sv_project_raw(void* h, uint64_t x, uint64_t z, uint32_t phase, int outcome, double* out) {
  return guard([&] {
    auto* s = (StateVector*)h;
    C64 v = s->project(Pauli::make(s->n, x, z, uint8_t(phase)), outcome != 0);
    out[0] = v.re, out[1] = v.im;
  });
}
int oracle_sv_scale(void* h, double re, double im) {
  return guard([&] { ((StateVector*)h)->scale(C64(re, im)); });
}
int oracle_sv_normalize(void* h) {
  return guard([&] { ((StateVector*)h)->normalize(); });
}
int oracle_sv_measure(void* h, const char* pauli, void* rng, int* outcome) {
  return guard([&] {
    auto* s = (StateVector*)h;
    *outcome = s->measure(Pauli::from_string(s->n, pauli), *(StdRng*)rng) ? 1 : 0;
  });
}
int oracle_sv_sample(void* h, void* rng, uint64_t shots, uint64_t* out) {
  return guard([&] {
    auto v = ((StateVector*)h)->sample(*(StdRng*)rng, shots);
    std::memcpy(out, v.data(), shots * sizeof(uint64_t));
  });
}
int oracle_sv_sample_uniforms(void* h, const double* u, uint64_t shots, uint64_t* out) {
  return guard([&] {
    auto v = ((StateVector*)h)->sample_from_uniforms(std::vector<double>(u, u + shots));
    std::memcpy(out, v.data(), shots * sizeof(uint64_t));
  });
}
void* oracle_sv_kron(void* a, void* b) {
  StateVector* s = nullptr;
  guard([&] { s = new StateVector(((StateVector*)a)->kron(*(StateVector*)b)); });
  return s;
}
// Runs a circuit; writes the record (0/1 bytes); returns its length or a negative status.
int oracle_sv_run(void* h, void* circuit, void* rng, uint8_t* rec, size_t cap) {
  int len = 0;
  int st = guard([&] {
    auto r = ((StateVector*)h)->run(*(Circuit*)circuit, *(StdRng*)rng);
    if (r.size() > cap) throw SimError(ErrKind::Invalid, "record buffer too small");
    std::memcpy(rec, r.data(), r.size());
    len = int(r.size());
  });
  return st == 0 ? len : st;
}
// Runs only the first `max_gates` gate operations of the circuit (no
// measurements), for bounded CPU-baseline samples; returns seconds taken.
double oracle_sv_run_gates_timed(void* h, void* circuit, uint64_t max_gates) {
  auto* s = (StateVector*)h;
  auto* c = (Circuit*)circuit;
  auto t0 = std::chrono::steady_clock::now();
  uint64_t done = 0;
  for (auto& op : c->ops) {
    if (done >= max_gates) break;
    if (op.kind != OpKind::GateOp) continue;
    s->apply_gate(op.gate, op.qubits);
    ++done;
  }
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// One noisy trajectory of the random layer family: seed 1+t style draws are
// the caller's (seed), n = n_lo + gen_range(0..n_span), the circuit of `depth`
// layers with DEPOLARIZE2(p) after every CZ, then Z measurements of every
// qubit.  Outputs: n, <Z0>/<psi|psi> before the measurements, the record.
int oracle_trajectory(uint64_t seed, uint32_t n_lo, uint32_t n_span, uint32_t depth, double p, uint32_t* n_out,
                      double* z0_out, uint8_t* rec, size_t cap) {
  int len = 0;
  int st = guard([&] {
    StdRng rng = StdRng::seed_from_u64(seed);
    size_t n = n_lo + size_t(rng.gen_range_u64(0, n_span));
    std::string text = random_circuit_text(n, depth, rng, p, 0, n);
    Circuit c = Circuit::parse(text);
    StateVector s = StateVector::zero_state(n);
    std::vector<uint8_t> r;
    bool z_done = false;
    for (auto& op : c.ops) {
      if (op.kind == OpKind::Measure && !z_done) {
        *z0_out = s.expectation(Pauli::zq(n, 0)).re / s.norm_sq().re;
        z_done = true;
      }
      int o = s.apply_op(op, rng);
      if (o >= 0) r.push_back(uint8_t(o));
    }
    if (r.size() > cap) throw SimError(ErrKind::Invalid, "record buffer too small");
    std::memcpy(rec, r.data(), r.size());
    *n_out = uint32_t(n);
    len = int(r.size());
  });
  return st == 0 ? len : st;
}

// ---- sparse restatement (permutation/diagonal registers) ----
void* oracle_sparse_run(const char* text) {
  SparseState* s = nullptr;
  int st = guard([&] {
    Circuit c = Circuit::parse(text);
    s = new SparseState(SparseState::zero_state(c.n));
    for (auto& op : c.ops) {
      if (op.kind != OpKind::GateOp) throw SimError(ErrKind::Unsupported, "sparse oracle: gates only");
      s->apply_gate(op.gate, op.qubits);
    }
  });
  return st == 0 ? s : nullptr;
}
uint64_t oracle_sparse_len(void* h) { return ((SparseState*)h)->ent.size(); }
void oracle_sparse_get(void* h, uint64_t* idx, double* amp) {
  auto* s = (SparseState*)h;
  for (size_t i = 0; i < s->ent.size(); ++i) {
    idx[i] = s->ent[i].first;
    amp[2 * i] = s->ent[i].second.re;
    amp[2 * i + 1] = s->ent[i].second.im;
  }
}
void oracle_sparse_free(void* h) { delete (SparseState*)h; }


// ---- sparse restatement on registers of any width (sparse.rs with Bits keys) ----
// Runs the circuit from |0...0> with StdRng::seed_from_u64(seed); rec gets the record.
void* oracle_wsparse_run(const char* text, uint64_t seed, uint8_t* rec, size_t cap, size_t* len) {
  WideSparse* s = nullptr;
  int st = guard([&] {
    Circuit c = Circuit::parse(text);
    auto w = std::make_unique<WideSparse>(WideSparse::zero_state(c.n));
    StdRng rng = StdRng::seed_from_u64(seed);
    auto r = w->run(c, rng);
    if (r.size() > cap) throw SimError(ErrKind::Invalid, "record buffer too small");
    for (size_t i = 0; i < r.size(); ++i) rec[i] = r[i];
    *len = r.size();
    s = w.release();
  });
  return st == 0 ? s : nullptr;
}
uint64_t oracle_wsparse_len(void* h) { return ((WideSparse*)h)->ent.size(); }
uint32_t oracle_wsparse_words(void* h) { return uint32_t(nwords(((WideSparse*)h)->n)); }
// entries in entry order: nwords(n) words per key
void oracle_wsparse_get(void* h, uint64_t* keys, double* amps) {
  auto* s = (WideSparse*)h;
  const size_t W = nwords(s->n);
  for (size_t i = 0; i < s->ent.size(); ++i) {
    std::memcpy(keys + i * W, s->ent[i].first.data(), W * 8);
    amps[2 * i] = s->ent[i].second.re;
    amps[2 * i + 1] = s->ent[i].second.im;
  }
}
int oracle_wsparse_expect(void* h, const char* pauli, double* re_im) {
  return guard([&] {
    auto* s = (WideSparse*)h;
    WidePauli w = WidePauli::parse_with(pauli, s->n);
    Bits x, z;
    uint32_t ph = 0;
    s->sites_words(w, x, z, ph);
    C64 e = s->expectation(x, z, ph);
    re_im[0] = e.re;
    re_im[1] = e.im;
  });
}
int oracle_wsparse_sample(void* h, uint64_t seed, uint64_t shots, uint64_t* out) {
  return guard([&] {
    auto* s = (WideSparse*)h;
    StdRng rng = StdRng::seed_from_u64(seed);
    auto v = s->sample(rng, shots);
    const size_t W = nwords(s->n);
    for (size_t i = 0; i < v.size(); ++i) std::memcpy(out + i * W, v[i].data(), W * 8);
  });
}
void oracle_wsparse_free(void* h) { delete (WideSparse*)h; }

// ---- frame sampler (frame.rs) ----
// The reference record of FrameSampler::new; returns the number of measurements.
int oracle_frames_reference(const char* text, uint64_t seed, uint8_t* out, size_t cap) {
  int m = 0;
  int st = guard([&] {
    auto r = frame_reference(Circuit::parse(text), seed);
    if (cap < r.size()) throw SimError(ErrKind::Invalid, "buffer too small");
    for (size_t i = 0; i < r.size(); ++i) out[i] = r[i];
    m = int(r.size());
  });
  return st == 0 ? m : st;
}
// sample_packed with the batch seeds given: out holds m rows of nwords(shots)
int oracle_frames_sample_packed(const char* text, const uint8_t* reference, size_t m, uint64_t shots,
                                const uint64_t* seeds, size_t nseeds, int threads, uint64_t* out) {
  return guard([&] {
    FrameSamplerRef f(Circuit::parse(text), std::vector<bool>(reference, reference + m));
    auto rec = f.sample_packed_seeds(shots, std::vector<uint64_t>(seeds, seeds + nseeds), threads);
    const size_t W = nwords(shots);
    for (size_t k = 0; k < rec.size(); ++k) std::memcpy(out + k * W, rec[k].data(), W * 8);
  });
}
// sample_detectors with the batch seeds given
int oracle_frames_sample_detectors(const char* text, const uint8_t* reference, size_t m, uint64_t shots,
                                   const uint64_t* seeds, size_t nseeds, uint64_t* det, size_t det_rows, uint64_t* obs,
                                   size_t obs_rows) {
  return guard([&] {
    FrameSamplerRef f(Circuit::parse(text), std::vector<bool>(reference, reference + m));
    std::vector<std::vector<uint64_t>> d, o;
    f.sample_detectors_seeds(shots, std::vector<uint64_t>(seeds, seeds + nseeds), d, o);
    if (d.size() != det_rows || o.size() != obs_rows) throw SimError(ErrKind::Invalid, "detector or observable count");
    const size_t W = nwords(shots);
    for (size_t k = 0; k < d.size(); ++k) std::memcpy(det + k * W, d[k].data(), W * 8);
    for (size_t k = 0; k < o.size(); ++k) std::memcpy(obs + k * W, o[k].data(), W * 8);
  });
}
}  // extern "C"
