// Host-side circuit IR of the engine: the reference's gates, Paulis, phase
// polynomials, noise channels and circuits (src/gate.rs, src/pauli/mod.rs,
// src/phasepoly.rs, src/circuit.rs), each gate lowered once, at parse time,
// to the kernel that applies it ("lowered op").
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../engine.cuh"
#include "../host_math.hpp"
#include "rng.hpp"

namespace ncsim {

// i^phase X^x Z^z on n <= 64 qubits (src/pauli/mod.rs:81-87)
struct PauliOp {
  uint32_t n = 0;
  uint64_t x = 0, z = 0;
  uint32_t phase = 0;
  bool hermitian() const { return ((phase & 1) == 1) == bool(__builtin_popcountll(x & z) & 1); }
};
// Circuits (and the Paulis they measure) may name up to this many qubits; the
// dense forms take registers of at most 64 (the sparse form 1024), the frame
// sampler any of these.
constexpr uint32_t MAX_CIRCUIT_QUBITS = 1u << 24;

// A Pauli on any number of qubits as its non-identity sites (qubit ascending;
// letter bits 1 = X, 2 = Z, 3 = Y) and the phase i^phase in front of the
// letters (so Y counts as a letter, not as i X Z).
struct PauliSites {
  uint32_t n = 0;
  std::vector<std::pair<uint32_t, uint8_t>> sites;
  uint32_t phase = 0;
  bool hermitian() const { return (phase & 1) == 0; }
};
// Pauli::from_string / Pauli::parse (src/pauli/mod.rs:344-414); n < 0 infers the size
PauliSites parse_pauli_sites(const std::string& text, int64_t n);
PauliOp pauli_from_sites(const PauliSites& s);  // registers of at most 64 qubits
PauliOp parse_pauli(const std::string& text, int64_t n);

// f(x) = constant + sum_t c_t prod_{l in t} [l . x] mod 2^bits over nvars
// local variables (src/phasepoly.rs:536-545); terms kept as given
struct PhasePolyIR {
  uint32_t nvars = 0;
  uint32_t bits = 1;
  uint64_t constant = 0;
  std::vector<std::vector<uint64_t>> parities;
  std::vector<uint64_t> coeffs;
  uint64_t eval(uint64_t x) const;
};

// U|x> = scalar zeta^{f(x)} |M x + shift> (src/gate.rs:24-37)
struct MonomialIR {
  uint32_t k = 0;
  std::vector<uint64_t> rows;
  uint64_t shift = 0;
  PhasePolyIR phase;
  Phase scalar;
  bool affine_identity() const;
};
struct GateIR;
// Gate::monomial (gate.rs:519-564); false when the gate has no monomial view
bool monomial_view(const GateIR& g, MonomialIR& out);

enum class GateKind : int {
  I, X, Y, Z, H, S, Sdg, SqrtX, SqrtXdg, SqrtY, SqrtYdg, T, Tdg, Cx, Cy, Cz, Swap, Cs, Csdg, Ccz, Ccx,
  Phase, CPhase, Rx, Ry, Rz, Diagonal, Monomial, Pauli, Unitary
};

struct GateIR {
  GateKind kind = GateKind::I;
  int64_t pk = 0;
  uint32_t pbits = 1;
  double theta = 0.0;
  PhasePolyIR poly;
  MonomialIR mono;
  PauliOp pauli;
  uint32_t uk = 0;
  std::vector<CplxD> umat;
  uint32_t arity() const;
  std::string text() const;  // the circuit-text token
};

// What one kernel launch needs to apply a gate on given qubits.
enum class LoweredKind : int { Nothing, Dense, Monomial, PhasePoly, Pauli };
struct LoweredOp {
  LoweredKind kind = LoweredKind::Nothing;
  std::vector<uint32_t> qubits;
  std::vector<CplxD> matrix;   // Dense (row-major) or the monomial phases
  std::vector<uint32_t> image; // Monomial
  PolyTerms poly;              // PhasePoly
  uint64_t x = 0, z = 0;       // Pauli
  uint32_t phase = 0;
};

// The gate's views in the reference's order (vector.rs:364-395): Pauli,
// monomial, matrix.  Throws Error on arity or qubit problems.
LoweredOp lower_gate(const GateIR& g, const std::vector<uint32_t>& qubits, uint32_t n);
// Gate::matrix (gate.rs:670-747) for gates with a dense view
std::vector<CplxD> gate_matrix(const GateIR& g);

enum class NoiseKind : int { XError, YError, ZError, PauliChannel1, Depolarize1, Depolarize2 };
struct NoiseIR {
  NoiseKind kind = NoiseKind::XError;
  double p[3] = {0, 0, 0};
  uint32_t arity() const { return kind == NoiseKind::Depolarize2 ? 2 : 1; }
  std::string text() const;
  bool valid() const;
  // Noise::sample (circuit.rs:136-146): always one draw; -1 for no error,
  // otherwise (x bits) | (z bits) << 8
  int sample(ncsim_rng& rng) const;
};

enum class OpKind : int { Gate, Measure, Reset, Noise, Detector, Observable, Tick };
struct OpIR {
  OpKind kind = OpKind::Tick;
  GateIR gate;
  std::vector<uint32_t> qubits;
  LoweredOp lowered;  // on the register's qubits (n <= 64); wider: on local qubits 0..k-1 (= qubits[j])
  PauliOp pauli;      // measured Pauli, registers of at most 64 qubits
  PauliSites sites;   // measured Pauli, any register
  NoiseIR noise;
  std::vector<uint64_t> lookback;
  uint64_t index = 0;
};

}  // namespace ncsim

struct ncsim_circuit {
  uint32_t n = 0;
  std::vector<ncsim::OpIR> ops;
  // the fused form's device plan, built on first use (freed with the circuit)
  mutable std::shared_ptr<void> fused_plan;
  mutable uint32_t fused_plan_fuse = 0;
  mutable int fused_plan_device = -1;
  // runs of gates captured as CUDA graphs for one state (built on first use)
  mutable std::shared_ptr<void> gate_graphs;
  uint64_t num_gates() const;
  uint64_t num_measurements() const;
  std::string text() const;
};

struct ncsim_gate {
  ncsim::GateIR g;
};

namespace ncsim {
ncsim_circuit parse_circuit(const std::string& text);
GateIR parse_gate_token(const std::string& tok, uint32_t nq_hint);
std::string fmt_f64(double v);
}  // namespace ncsim
