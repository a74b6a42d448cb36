// Host side of the Pauli-frame sampler (the reference's FrameSampler,
// src/frame.rs:34-300): the Clifford action of each gate, the noiseless
// reference run on a host tableau, the device program (the circuit's frame
// operations in dependency layers) and the per-batch scan of the random
// stream (mask positions and noise hits).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "host/ir.hpp"

namespace ncsim {
namespace frames {

constexpr uint32_t BATCH = 1u << 14;           // shots per batch (frame.rs:31)
constexpr uint32_t BATCH_WORDS = BATCH / 64;   // 64-bit words per column of a full batch
constexpr uint32_t MAX_LINEAR_K = 32;          // qubits of one generic Clifford frame map

// i^phase X^x Z^z on a gate's k local qubits (the reference's Pauli
// convention, src/pauli/mod.rs:81-87)
struct LocalPauli {
  uint64_t x = 0, z = 0;
  uint32_t phase = 0;
};

// U X_j U† (img[j]) and U Z_j U† (img[k + j]) of a Clifford gate on k qubits
struct CliffordAction {
  uint32_t k = 0;
  std::vector<LocalPauli> img;
};

// Gate::is_clifford and Gate::tableau (gate.rs:568-665): the named Cliffords
// and Paulis by their tableaux, T, T†, CS, CS†, CCZ, CCX, rotations and dense
// unitaries never, the other monomial gates when their phase polynomial has
// no term above level 2 and conjugation keeps X_j and Z_j in the Pauli group
// (MonomialGate::to_tableau, gate.rs:244-294).  False: not Clifford.
bool clifford_action(const GateIR& g, CliffordAction& out);

// The noiseless reference record of FrameSampler::new (frame.rs:41-60): the
// circuit without its noise on |0...0>, random outcomes drawn as
// Stabilizer::collapse draws them (`rng.gen::<bool>()`, stabilizer.rs:591),
// resets as the trait's measure-then-X (state/mod.rs:141-147).
std::vector<uint8_t> reference_record(const ncsim_circuit& c, uint64_t seed);

// One frame operation of the device program.
enum FrameOpKind : uint32_t {
  FOP_H = 0,       // x <-> z                       (H, SQRT_Y, SQRT_Y_DAG)
  FOP_S = 1,       // z ^= x                        (S, S_DAG)
  FOP_SQRTX = 2,   // x ^= z                        (SQRT_X, SQRT_X_DAG)
  FOP_CX = 3,      // x_b ^= x_a, z_a ^= z_b
  FOP_CZ = 4,      // z_a ^= x_b, z_b ^= x_a
  FOP_SWAP = 5,
  FOP_LINEAR = 6,  // k qubits, 2k output rows over the 2k frame bits (pool)
  FOP_MEASURE = 7, // record k, mask j, sites (pool); flip bit = reference[k]
  FOP_RESET = 8,   // x = 0, z = mask j
  FOP_NOISE = 9,   // noise op i (its hits per batch), k qubits (pool)
};

struct FrameOp {
  uint32_t kind;  // FrameOpKind | count << 8 | flip << 31
  uint32_t a;     // qubit / record index / noise index
  uint32_t b;     // qubit / mask index
  uint32_t off;   // into the pool
};

// The two decisions a noise channel takes from a draw u = k 2^-53 (k the
// draw's top 53 bits) as step tables over k.  Each decision is a monotone
// function of k: the geometric skip floor(ln(1 - u) / ln(1 - p)) (frame.rs:252)
// and the error picked by subtracting the probabilities from u * total in
// order (frame.rs:273-282).  A table lists the least k at which the decision
// steps up, found with the same floating-point expressions the reference
// evaluates (so the same log), and checked for monotonicity a few k on each
// side of every step; a channel whose check fails keeps the direct evaluation.
struct SkipTable {
  double l = 0.0;                 // ln(1 - p)
  std::vector<uint64_t> thr;      // thr[g]: least k with skip >= g (g = 0..BATCH; 2^53 when none)
  std::vector<uint16_t> bucket;   // the skip at k = b << 37 for each of the 2^16 buckets b
  uint32_t at(uint64_t k) const {
    uint32_t g = bucket[k >> 37];
    while (g < BATCH && thr[g + 1] <= k) ++g;
    return g;
  }
};
struct PickTable {
  std::vector<uint64_t> thr;      // thr[i]: least k with pick > i
  // starts from the pick of equal probabilities and walks to the step that holds k
  uint32_t at(uint64_t k) const {
    const uint32_t e = uint32_t(thr.size());
    uint32_t i = uint32_t((unsigned __int128)k * (e + 1) >> 53);
    if (i > e) i = e;
    while (i > 0 && thr[i - 1] > k) --i;
    while (i < e && thr[i] <= k) ++i;
    return i;
  }
};

struct NoiseChannel {
  std::vector<double> p;       // errors(): probabilities in order (circuit.rs:119-128)
  std::vector<uint8_t> x, z;   // local error bits
  double total = 0.0;          // their sum, left to right
  std::shared_ptr<const SkipTable> skip;  // null: evaluate the skips directly
  std::shared_ptr<const PickTable> pick;  // null: evaluate the picks directly
};

struct Program {
  uint32_t n = 0;
  uint64_t num_measurements = 0;
  uint32_t num_masks = 0;      // n initial randomisations, then one per measurement and reset
  std::vector<FrameOp> ops;    // grouped by layer
  std::vector<uint32_t> layer_off;
  std::vector<uint32_t> pool;
  // the random stream's consumers in circuit order: kind 0 = mask, 1 = noise channel index
  std::vector<std::pair<uint8_t, uint32_t>> draws;
  std::vector<NoiseChannel> noise;  // one per noise op, in circuit order
  std::vector<std::vector<uint64_t>> detectors, observables;  // absolute measurement indices
  std::vector<uint8_t> det_flip, obs_flip;                     // parity of the reference bits
  std::vector<uint8_t> reference;
};

// Compile the circuit (all gates Clifford, else NCSIM_ERR_UNSUPPORTED) with
// its reference record.
Program compile(const ncsim_circuit& c, const std::vector<uint8_t>& reference);

// The random stream of one batch (StdRng::seed_from_u64(seed), frame.rs:104-153):
// the u32 position of each mask's first word, and the noise hits of each
// noise op as (shot | x << 16 | z << 20), counted per op.
struct BatchScan {
  std::vector<uint64_t> mask_pos;    // num_masks
  std::vector<uint32_t> ev_off;      // noise ops + 1, offsets into events
  std::vector<uint32_t> events;
};
void scan_batch(const Program& p, uint64_t seed, uint32_t shots, BatchScan& out);

// The 256-bit ChaCha key of StdRng::seed_from_u64 (rand_core 0.6 PCG32 expansion)
void key_of_seed(uint64_t seed, uint32_t key[8]);

}  // namespace frames
}  // namespace ncsim
