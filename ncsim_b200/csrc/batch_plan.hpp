// Batching form: many independent noisy trajectories of small registers
// (13..26 qubits, complex64), each run by one CTA of a persistent kernel.
//
// A trajectory is the reference's `QuantumState::run` (src/state/mod.rs:168-183)
// of a circuit with its own StdRng: gates, Pauli noise channels (one draw per
// channel application, src/circuit.rs:136-146) and a trailing block of Z
// measurements M 0, M 1, ..., M m-1 (a draw only when the outcome is
// uncertain, src/state/mod.rs:113-131).
//
// The host folds the circuit, per qubit, into 2x2 gates and two-qubit
// diagonals: noise is sampled in circuit order (its draws do not depend on the
// state), one-qubit diagonals and sampled Paulis are multiplied into the next
// non-diagonal one-qubit gate on the qubit, and the m measurement uniforms that
// follow the noise draws in the stream are drawn ahead for the device.  A
// gate whose entries all have modulus 1/sqrt2 (H or SQRT_X times phases and
// Paulis) is split into diag(l0, l1) s [[1, w], [1, -w]]: the device applies
// the second factor (a complex multiply and four FMAs per pair instead of
// sixteen FMAs) and the diagonal joins the qubit's next gate.  The
// folded ops are grouped into passes over a 13-qubit window (a tile of 8192
// amplitudes in shared memory) and, inside a pass, into stages: each stage
// holds 32 amplitudes per thread in registers, over five consecutive tile
// bits, and applies every op whose non-diagonal qubit is one of them.
#pragma once

#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "host/ir.hpp"

namespace ncsim::batch {

constexpr uint32_t TILE_BITS = 13;
constexpr uint32_t TILE = 1u << TILE_BITS;  // amplitudes per tile
constexpr uint32_t LOW_BITS = 4;            // qubits 0..3 lie in every window
constexpr uint32_t REG_BITS = 5;            // 32 amplitudes per thread
constexpr uint32_t THREADS = 256;
constexpr uint32_t MIN_QUBITS = TILE_BITS;
constexpr uint32_t MAX_QUBITS = 26;         // 2^(n-13) <= 8192 high amplitudes per measurement gather
constexpr uint32_t MAX_NON = MAX_QUBITS - TILE_BITS;
constexpr uint32_t MAX_PASS_OPS = 256;      // a pass's ops and stages fit the kernel's shared copy
constexpr uint32_t NSEL = 3;                // stage register-bit sets: tile bits [RSHIFT, RSHIFT+5)
constexpr uint32_t RSHIFT[NSEL] = {0, 5, 8};

// op codes and qubit locators of the device program
enum : uint32_t { OP_GATE = 0, OP_CZ = 1, OP_CPHASE = 2, OP_DIAG = 3, OP_BGATE = 4 };
enum : uint32_t { LOC_REG = 0, LOC_FIXED = 1, LOC_TILE = 2 };
enum : uint32_t { PASS_ZERO_INIT = 1, PASS_ACCUM = 2, PASS_NO_WRITE = 4 };

// One op of a stage.  hdr = code | locA << 3 | locB << 10 with loc = type << 5 | index:
// LOC_REG index = register bit (0..4), LOC_FIXED = bit of the thread's tile
// index, LOC_TILE = bit of the tile number.  v: GATE 2x2 row-major
// (re, im); BGATE (s w, s) for s [[1, w], [1, -w]], s = 1/sqrt2, |w| = 1;
// DIAG (d0, d1); CPHASE the phase applied where both bits are 1; CZ: v[0]'s
// bits are the product of the register operands' 32-amplitude patterns.
struct alignas(16) DevOp {
  float v[8];
  uint32_t hdr;
  uint32_t pad[3];
};
struct DevStage {
  uint32_t info;  // register-bit set | op count << 2
  uint32_t op0;
};
struct DevPass {
  uint32_t stage0;
  uint16_t nstage;
  uint8_t flags;
  uint8_t nnon;
  uint8_t win[TILE_BITS];  // tile bit b holds qubit win[b] (ascending, win[0..3] = 0..3)
  uint8_t non[MAX_NON];    // tile-number bit b holds qubit non[b]
  uint8_t pad[2];
};
struct DevTraj {
  uint32_t n, npass, pass0, draw0, nmeas, pad;
};
static_assert(sizeof(DevPass) % 4 == 0 && sizeof(DevPass) / 4 <= THREADS, "pass descriptor copied as words");
static_assert(sizeof(DevOp) == 48, "op descriptor: two float4 loads and a header");

// a qubit-level op after folding
struct QOp {
  uint32_t code = OP_GATE;
  uint32_t a = 0, b = 0;
  Cd m[4] = {};
};

struct Trajectory {
  uint32_t n = 0;
  uint32_t nmeas = 0;          // M 0 .. M nmeas-1 at the end
  uint64_t source_gates = 0;   // Op::Gate count of the circuit
  uint64_t noise_events = 0;   // sampled Pauli errors
  std::vector<QOp> ops;
  std::vector<double> draws;   // the nmeas uniforms after the noise draws
};

// tuning knobs of the host planner (chosen per register size by the autotuner)
struct PlanKnobs {
  bool greedy_windows = true;  // pick the window that takes most ops (else alternate)
  bool greedy_stages = true;   // pick the register set that takes most gates (else cycle)
  uint32_t window_step = TILE_BITS - LOW_BITS;  // candidate windows: qubits 0..3 and a block of 9
                                                // consecutive qubits starting every window_step
                                                // qubits (9: disjoint blocks; less: overlapping)
};
constexpr uint32_t NUM_KNOB_SETS = 4;
// the candidate knob sets the autotuner times (set 0 is the default)
inline PlanKnobs knob_set(uint32_t i) {
  PlanKnobs k;
  if (i == 1) k.window_step = 3;
  if (i == 2) k.window_step = 5;
  if (i == 3) k.greedy_stages = false;
  return k;
}

// an allocator whose resize leaves trivially constructible elements
// uninitialised (the program's arrays are filled in parallel after sizing)
template <class T>
struct UninitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = UninitAlloc<U>;
  };
  UninitAlloc() = default;
  template <class U>
  UninitAlloc(const UninitAlloc<U>&) noexcept {}
  template <class U>
  void construct(U*) noexcept {}
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using ProgVec = std::vector<T, UninitAlloc<T>>;

struct Program {
  std::vector<DevTraj> traj;
  ProgVec<DevPass> pass;
  ProgVec<DevStage> stage;
  ProgVec<DevOp> op;
  ProgVec<double> draws;
  uint64_t source_gates = 0, noise_events = 0, folded_ops = 0, tile_passes = 0, tile_stages = 0;
  uint32_t max_n = 0;
  // algorithmic HBM bytes of one run: per pass 2 * 8 * 2^n (one read of 8 * 2^n
  // for a read-only pass, one write for the first pass, which starts from |0>)
  double state_bytes = 0;
};

// trajectory t of the random-layer family: StdRng::seed_from_u64(seed),
// n = n_lo + gen_range(0..n_span), `depth` layers with DEPOLARIZE2(p) after
// every CZ, M on every qubit; the same generator then runs it
Trajectory make_random_layers(uint64_t seed, uint32_t n_lo, uint32_t n_span, uint32_t depth, double p);
// a parsed circuit run with StdRng::seed_from_u64(seed)
Trajectory make_from_circuit(const ncsim_circuit& c, uint64_t seed);
// a batch of the random-layer family (trajectory t from StdRng(seed0 + t)),
// generated and compiled on the host threads (batch.cu)
ncsim_batch* batch_random_layers(uint32_t count, uint64_t seed0, uint32_t n_lo, uint32_t n_span, uint32_t depth,
                                 double p);
// compiles trajectories (in parallel) into one program, in the given order
Program compile(const std::vector<Trajectory>& ts, const PlanKnobs& knobs);
// with the knobs of each trajectory's register size (indexed by n)
Program compile(const std::vector<Trajectory>& ts, const std::vector<PlanKnobs>& knobs_by_n);

// FP64 host run of trajectory t of the program in the device's pass, tile,
// stage and op order, with the device's measurement rule; returns the record
// bits, <Z0>/<psi|psi> before the measurements and <psi|psi>
struct EmuResult {
  uint64_t record = 0;
  double z0 = 0, norm = 0;
};
EmuResult emulate(const Program& prog, uint32_t t);

}  // namespace ncsim::batch
