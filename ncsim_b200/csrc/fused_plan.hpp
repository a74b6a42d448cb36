// Precision form, host side: plan a circuit's gates into passes over the
// register and fuse each pass's gates into 5-qubit unitaries (FP64 products)
// and diagonal phase terms.
//
// A pass streams the register through shared memory in tiles of 2^12
// complex64 amplitudes whose indices vary in a 12-bit window: the lowest 4
// bits of the index (128-byte runs in HBM) plus 8 chosen qubits.  Inside a
// pass the tile goes through an ordered program of
//   - unitaries on 5 window qubits (applied as BF16x3 tensor-core GEMMs), and
//   - diagonal term groups: a term (mask, c) multiplies every amplitude whose
//     index has all bits of `mask` set by c.  Masks may hold any register bits
//     (bits outside the window are constant over a tile), so diagonal gates
//     never need their qubits in the window.
// One pass = one HBM read and one write of the register.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "host/ir.hpp"

namespace ncsim {
namespace fused {

constexpr int TILE_BITS = 12;       // 4096 amplitudes, 32 KB of complex64
constexpr int LOW_BITS = 4;         // index bits 0..3 always in the window
constexpr int GROUP_QUBITS = 5;     // unitaries are 32 x 32
constexpr int MAX_UNITARIES = 8;    // per pass: 16 KB of BF16 operands each in shared memory
constexpr int MAX_OPS = 64;
constexpr int MAX_TERMS = 256;

struct Term {
  uint64_t mask;
  CplxD c;
};

struct FusedOp {
  int kind = 0;                 // 0: unitary, 1: diagonal terms
  std::vector<uint32_t> qubits; // unitary: exactly 5 window qubits, local bit j = qubits[j]
  std::vector<CplxD> u;         // 32 x 32 row-major (unitary)
  std::vector<Term> terms;      // diagonal terms, applied in any order
};

struct Pass {
  std::vector<uint32_t> window;  // TILE_BITS qubits, ascending, the lowest LOW_BITS included
  std::vector<FusedOp> ops;
  int unitaries = 0;
};

// A run of the circuit: either passes or one operation for the plain path.
struct Segment {
  bool fused = false;
  std::vector<Pass> passes;
  size_t op = 0;  // index into the circuit's ops (plain segment)
};

struct Plan {
  uint32_t n = 0;
  std::vector<Segment> segments;
  uint64_t source_gates = 0, unitaries = 0, passes = 0, terms = 0;
};

// Plans the circuit for an n-qubit register (n >= TILE_BITS).  Gates that
// cannot be fused (monomials on more than 5 qubits, phase polynomials,
// Paulis) and every non-gate operation become plain segments.
Plan make_plan(const ncsim_circuit& c, uint32_t max_fuse);

// The bf16 split (round to nearest even), as the device computes it.
uint16_t bf16_bits(float x);
float bf16_value(uint16_t b);

// The shared-memory image of one unitary's B operand: the real form
// [[Ur, -Ui], [Ui, Ur]] (64 x 64) in K-major 128-byte-swizzled layout, as
// bf16 hi (8 KB) followed by the bf16 residual lo (8 KB).
void build_operand_image(const std::vector<CplxD>& u, uint8_t* out16k);

// Byte offset of (row, 16-byte chunk) in a K-major, 128-byte-swizzled operand
// with 64 bf16 per row (rows grouped by 8 in 1024-byte atoms).
inline uint32_t sw128_offset(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
}

// Applies the plan to complex128 amplitudes on the host, in FP64: the passes
// with the same op order, window tiles and term masks as the device, the
// plain segments by their lowered gates (for checking the planner; gates
// only).
void emulate(const Plan& p, const ncsim_circuit& c, std::vector<CplxD>& amps);

}  // namespace fused
}  // namespace ncsim
