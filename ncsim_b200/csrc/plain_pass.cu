// Tiled passes of the plain path: a run of consecutive gates applied to tiles
// of the register in shared memory, one read and one write of HBM for the run.
//
// A pass picks a window of T <= 12 qubits (the qubits the run's gates move,
// filled up with the lowest other qubits so that tiles load in runs of
// consecutive amplitudes) and streams the register's 2^(n-T) tiles through
// shared memory: a persistent CTA double-buffers its tiles (cp.async copies
// of the next tile land while the current one is worked on) and applies the
// pass's gates to each tile in circuit order, one __syncthreads between gates.
// Gates that only multiply amplitudes by phases (diagonals, phase polynomials)
// join any pass: their phases depend on index bits outside the window only
// through the tile's base index.
//
// Every gate is applied with the arithmetic of the kernel that the gate-by-gate
// path would launch for it (the same dispatch rules, the same cmul/cfma
// expressions on the same operands in the same order), so a run gives the same
// amplitudes either way.  Gates with no tile form (dense gates on more than 3
// qubits, permutation tables other than pair swaps, phase polynomials of more
// than 64 terms) run as their own kernels between passes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "engine.cuh"
#include "host/ir.hpp"

namespace ncsim {

namespace {

constexpr int PASS_THREADS = 512;
constexpr int MAX_TILE_BITS = 12;
constexpr int MAX_FIBER_K = 3;  // 4- and 5-qubit matrices run as their own kernels (registers)
constexpr int MAX_TABLE_K = 10;
// longer phase polynomials run as the bit-sliced kernel: evaluated per element
// in a tile they cost a popcount per parity per amplitude
constexpr int MAX_PASS_TERMS = 4;
constexpr int MAX_PASS_PARITIES = 8;
constexpr int MAX_PASS_OPS = 192;  // ops of one pass (chain heads included)

template <class R>
using V = typename VecOf<R>::T;

enum TileKind : uint32_t {
  TK_DENSE1,      // 1-qubit dense matrix (k_dense1)
  TK_DENSE2,      // 2-qubit dense matrix (k_dense2)
  TK_FIBER,       // 3-qubit dense matrix (k_dense_fiber)
  TK_DIAG_CONST,  // one phase on the indices with every fixed bit set (k_diag_const)
  TK_DIAG_1Q,     // two phases selected by one bit (k_diag_1q)
  TK_DIAG_TABLE,  // phase table over <= 10 qubits (k_diag)
  TK_PAIRSWAP,    // exchange of i and i ^ x on a fixed-bit sub-cube (k_pairswap)
  TK_PHASEPOLY,   // phase polynomial of the global index (k_phasepoly)
  TK_CHAIN,       // the next k ops, applied group by group to 8-element cubes held in registers
};

// One gate of a pass, encoded against the pass's window: "local" masks are
// over the tile's T bits, "global" masks over the bits outside the window.
struct TileOp {
  uint32_t kind;
  uint32_t k;        // qubits (fiber, table), terms (phase polynomial)
  uint32_t l0, l1;   // local bit positions (dense1: l0; dense2: l0 = qubit 0, l1 = qubit 1; diag 1q: l1 = global qubit outside)
  uint32_t lfix;     // local mask of fixed bits
  uint32_t lones;    // the fixed bits' values at i (pairswap), or lfix (diagonal kinds)
  uint32_t lx;       // local xor mask (pairswap)
  uint32_t flags;    // pairswap: unit_i | unit_j << 1; diag 1q: 1 = the qubit lies outside (value in gval)
  uint64_t gfix;     // fixed bits outside the window ...
  uint64_t gval;     // ... and the values the tile base must have there
  uint64_t gz;       // phase polynomial: offset of its parities
  uint32_t phase;
  uint32_t cp;       // complex pool offset
  uint32_t up;       // word pool offset
  uint32_t reg;      // in a chain: the op's bits among the cube's three, or its cube elements (see chainify)
  uint32_t gml, gvl; // in a chain: fixed local bits outside the cube, and their values
};

struct PassGeom {
  int T;                         // tile bits
  int w;                         // low index bits in the window (0..w-1)
  int nh;                        // window bits above them
  uint8_t hq[MAX_TILE_BITS];     // their global positions, ascending
};

// global offset of tile element e (bits 0..w-1 stay, bit w+i goes to hq[i])
__host__ __device__ __forceinline__ uint64_t deposit(uint32_t e, const PassGeom& g) {
  uint64_t off = e & ((1u << g.w) - 1);
  for (int i = 0; i < g.nh; ++i) off |= uint64_t((e >> (g.w + i)) & 1u) << g.hq[i];
  return off;
}
// base index of tile t: t spread over the bits outside the window
__host__ __device__ __forceinline__ uint64_t tile_base_of(uint64_t t, const PassGeom& g) {
  uint64_t v = t << g.w;
  for (int i = 0; i < g.nh; ++i) {
    const int b = g.hq[i];
    v = ((v >> b) << (b + 1)) | (v & ((uint64_t(1) << b) - 1));
  }
  return v;
}

// v with zero bits inserted at the ascending local positions pos[0..cnt)
__device__ __forceinline__ uint32_t insert_zeros32(uint32_t v, const uint8_t* pos, int cnt) {
  for (int i = 0; i < cnt; ++i) {
    const int b = pos[i];
    v = ((v >> b) << (b + 1)) | (v & ((1u << b) - 1));
  }
  return v;
}
__device__ __forceinline__ int parity64(uint64_t v) { return __popcll(v) & 1; }

// A tile in shared memory, element e stored at e ^ ((e >> 3) & 7): the XOR of
// the low three index bits with the next three spreads the 16-byte elements of
// a warp's access over the banks whichever tile bits an op pairs (a thread
// holding a cube of three low bits reads eight consecutive elements; without
// the swizzle every thread of the warp would hit the same four banks).
template <class R>
struct SwTile {
  V<R>* p;
  __device__ __forceinline__ V<R>& operator[](uint32_t e) const { return p[e ^ ((e >> 3) & 7u)]; }
};

// The pass's ops travel in the kernel parameters (constant bank): every thread
// reads the same op at the same time, a broadcast the constant cache serves.
template <class R>
struct PassParams {
  V<R>* amp;
  uint64_t ntiles;
  PassGeom g;
  uint32_t nops;
  const V<R>* cpool;
  const uint32_t* upool;
  const uint64_t* ppool;  // phase polynomial parities (global masks)
  TileOp ops[MAX_PASS_OPS];
};

// constant i of the pass's pool
template <class R>
__device__ __forceinline__ V<R> pconst(const PassParams<R>& P, uint32_t i) {
  return P.cpool[i];
}

// -------- the gates on a tile (all threads of the CTA; `t` in shared memory) --------
template <class R>
__device__ void tile_dense1(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp) {
  const V<R> m00 = cp[op.cp], m01 = cp[op.cp + 1], m10 = cp[op.cp + 2], m11 = cp[op.cp + 3];
  const uint32_t lo = (1u << op.l0) - 1;
  for (uint32_t p = threadIdx.x; p < (tsz >> 1); p += blockDim.x) {
    const uint32_t i0 = ((p & ~lo) << 1) | (p & lo), i1 = i0 | (lo + 1);
    const V<R> a0 = t[i0], a1 = t[i1];
    t[i0] = cfma(m01, a1, cmul(m00, a0));
    t[i1] = cfma(m11, a1, cmul(m10, a0));
  }
}

template <class R>
__device__ void tile_dense2(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp) {
  const uint32_t ba = 1u << op.l0, bb = 1u << op.l1;
  uint8_t pos[2] = {uint8_t(min(op.l0, op.l1)), uint8_t(max(op.l0, op.l1))};
  for (uint32_t p = threadIdx.x; p < (tsz >> 2); p += blockDim.x) {
    const uint32_t i = insert_zeros32(p, pos, 2);
    const uint32_t idx[4] = {i, i | ba, i | bb, i | ba | bb};
    V<R> v[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) v[b] = t[idx[b]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      V<R> acc = cmul(cp[op.cp + 4 * r], v[0]);
      acc = cfma(cp[op.cp + 4 * r + 1], v[1], acc);
      acc = cfma(cp[op.cp + 4 * r + 2], v[2], acc);
      acc = cfma(cp[op.cp + 4 * r + 3], v[3], acc);
      t[idx[r]] = acc;
    }
  }
}

template <class R, int K>
__device__ void tile_fiber(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp, const uint32_t* up) {
  constexpr int D = 1 << K;
  uint8_t pos[K];
#pragma unroll
  for (int j = 0; j < K; ++j) pos[j] = uint8_t(up[op.up + j]);
  uint32_t off[D];
#pragma unroll
  for (int b = 0; b < D; ++b) off[b] = up[op.up + K + b];
  const V<R>* m = cp + op.cp;
  for (uint32_t f = threadIdx.x; f < (tsz >> K); f += blockDim.x) {
    const uint32_t base = insert_zeros32(f, pos, K);
    V<R> v[D];
#pragma unroll
    for (int b = 0; b < D; ++b) v[b] = t[base | off[b]];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      V<R> acc = cmul(m[r * D], v[0]);
#pragma unroll
      for (int b = 1; b < D; ++b) acc = cfma(m[r * D + b], v[b], acc);
      t[base | off[r]] = acc;
    }
  }
}

// the elements with every local fixed bit set to its value: p with zeros inserted, ORed with the values
template <class R>
__device__ void tile_diag_const(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp, const uint32_t* up) {
  const int nf = __popc(op.lfix);
  uint8_t pos[MAX_TILE_BITS];
  for (int i = 0; i < nf; ++i) pos[i] = uint8_t(up[op.up + i]);
  const V<R> c = cp[op.cp];
  for (uint32_t p = threadIdx.x; p < (tsz >> nf); p += blockDim.x) {
    const uint32_t e = insert_zeros32(p, pos, nf) | op.lones;
    const V<R> u = t[e];
    if (!is_zero(u)) t[e] = cmul(c, u);
  }
}

template <class R>
__device__ void tile_diag_1q(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp, uint64_t base) {
  const V<R> c0 = cp[op.cp], c1 = cp[op.cp + 1];
  const bool outside = op.flags & 1;
  const bool obit = (base >> op.l1) & 1;  // the qubit's global position when it lies outside
  for (uint32_t e = threadIdx.x; e < tsz; e += blockDim.x) {
    const V<R> u = t[e];
    const bool bit = outside ? obit : ((e >> op.l0) & 1u);
    if (!is_zero(u)) t[e] = cmul(bit ? c1 : c0, u);
  }
}

template <class R>
__device__ void tile_diag_table(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp, const uint32_t* up,
                                uint64_t base) {
  // up: [k] local position of qubit j (or 255 + its global position when outside), then the
  // local fixed positions (ascending), then the unit flags as bytes
  const int k = int(op.k);
  const int nf = __popc(op.lfix);
  uint32_t xout = 0;
  uint8_t lpos[MAX_TABLE_K];
  for (int j = 0; j < k; ++j) {
    const uint32_t v = up[op.up + j];
    if (v >= 256) {
      xout |= uint32_t((base >> (v - 256)) & 1u) << j;
      lpos[j] = 255;
    } else {
      lpos[j] = uint8_t(v);
    }
  }
  uint8_t fpos[MAX_TILE_BITS];
  for (int i = 0; i < nf; ++i) fpos[i] = uint8_t(up[op.up + k + i]);
  const uint8_t* unit = reinterpret_cast<const uint8_t*>(up + op.up + k + nf);
  const V<R>* d = cp + op.cp;
  for (uint32_t p = threadIdx.x; p < (tsz >> nf); p += blockDim.x) {
    const uint32_t e = insert_zeros32(p, fpos, nf) | op.lones;
    uint32_t x = xout;
    for (int j = 0; j < k; ++j)
      if (lpos[j] != 255) x |= ((e >> lpos[j]) & 1u) << j;
    if (unit[x]) continue;
    const V<R> v = t[e];
    if (!is_zero(v)) t[e] = cmul(d[x], v);
  }
}

template <class R>
__device__ void tile_pairswap(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp, const uint32_t* up) {
  const int nf = __popc(op.lfix);
  uint8_t pos[MAX_TILE_BITS];
  for (int i = 0; i < nf; ++i) pos[i] = uint8_t(up[op.up + i]);
  const V<R> ci = cp[op.cp], cj = cp[op.cp + 1];
  const bool ui = op.flags & 1, uj = (op.flags >> 1) & 1;
  for (uint32_t p = threadIdx.x; p < (tsz >> nf); p += blockDim.x) {
    const uint32_t i = insert_zeros32(p, pos, nf) | op.lones;
    const uint32_t j = i ^ op.lx;
    const V<R> vi = t[i], vj = t[j];
    t[i] = ui ? vj : cmul(ci, vj);
    t[j] = uj ? vi : cmul(cj, vi);
  }
}

__device__ __forceinline__ double2 pass_root(uint64_t f, uint32_t bits) {
  // exp(2 pi i f / 2^bits) with exact quarter and eighth turns (as the gate-by-gate kernel)
  const uint64_t m = uint64_t(1) << bits;
  if (((4 * f) & (m - 1)) == 0) {
    switch ((4 * f / m) & 3) {
      case 0: return make_double2(1.0, 0.0);
      case 1: return make_double2(0.0, 1.0);
      case 2: return make_double2(-1.0, 0.0);
      default: return make_double2(0.0, -1.0);
    }
  }
  if (((8 * f) & (m - 1)) == 0) {
    const double h = 0.70710678118654752440;
    switch ((8 * f / m) & 7) {
      case 1: return make_double2(h, h);
      case 3: return make_double2(-h, h);
      case 5: return make_double2(-h, -h);
      default: return make_double2(h, -h);
    }
  }
  double s, c;
  sincospi(2.0 * double(f) / double(m), &s, &c);
  return make_double2(c, s);
}

// up: bits, use_table, scalar_is_one, constant lo, constant hi, start[k+1], coeff[k]; cp: scalar, table[2^bits]
template <class R>
__device__ void tile_phasepoly(SwTile<R> t, uint32_t tsz, const TileOp& op, const V<R>* cp, const uint32_t* up,
                               const uint64_t* pp, uint64_t base, uint64_t dthread, const uint64_t* dround) {
  const uint32_t* u = up + op.up;
  const uint32_t bits = u[0];
  const bool use_table = u[1], s_one = u[2];
  const uint64_t constant = uint64_t(u[3]) | (uint64_t(u[4]) << 32);
  const int nt = int(op.k);
  const uint32_t* start = u + 5;
  const uint32_t* coeff = start + nt + 1;
  const uint64_t modmask = (uint64_t(1) << bits) - 1;
  const V<R> scalar = cp[op.cp];
  const V<R>* table = cp + op.cp + 1;
  const uint32_t nr = tsz / blockDim.x;
  for (uint32_t r = 0; r < max(nr, 1u); ++r) {
    const uint32_t e = threadIdx.x + r * blockDim.x;
    if (e >= tsz) break;
    const uint64_t i = base | dthread | dround[r];
    const V<R> v = t[e];
    if (is_zero(v)) continue;
    uint64_t f = constant;
    for (int tt = 0; tt < nt; ++tt) {
      int all = 1;
      for (uint32_t l = start[tt]; l < start[tt + 1]; ++l) all &= __popcll(pp[op.gz + l] & i) & 1;
      if (all) f += coeff[tt];
    }
    f &= modmask;
    V<R> c;
    if (use_table) {
      c = table[f];
      if (is_one_v(c)) continue;
    } else {
      if (f == 0 && s_one) continue;
      const double2 rr = pass_root(f, bits);
      c.x = R(rr.x);
      c.y = R(rr.y);
      if (!s_one) c = cmul(scalar, c);
    }
    t[e] = cmul(c, v);
  }
}

// ---- chains: consecutive ops whose bits lie in one cube of three tile bits ----
// A thread holds the 8 elements of a cube (v[b]: cube pattern b) and applies
// the chain's ops in order to them, one shared-memory round trip for the
// chain.  The ops couple elements only inside a cube, and each element sees
// its ops in circuit order with each op's own arithmetic.  Register indices
// are compile-time: the op's cube bits (`reg`) select a template instance.
template <class R, int J>
__device__ __forceinline__ void chain_dense1(V<R> (&v)[8], const V<R> (&m)[4]) {
  const V<R> m00 = m[0], m01 = m[1], m10 = m[2], m11 = m[3];
#pragma unroll
  for (int b = 0; b < 8; ++b)
    if (!((b >> J) & 1)) {
      const V<R> a0 = v[b], a1 = v[b | (1 << J)];
      v[b] = cfma(m01, a1, cmul(m00, a0));
      v[b | (1 << J)] = cfma(m11, a1, cmul(m10, a0));
    }
}

template <class R, int JA, int JB>
__device__ __forceinline__ void chain_dense2(V<R> (&v)[8], const PassParams<R>& P, uint32_t c0) {
  V<R> m[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) m[i] = pconst(P, c0 + i);
#pragma unroll
  for (int b = 0; b < 8; ++b)
    if (!((b >> JA) & 1) && !((b >> JB) & 1)) {
      const int idx[4] = {b, b | (1 << JA), b | (1 << JB), b | (1 << JA) | (1 << JB)};
      V<R> x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = v[idx[q]];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        V<R> acc = cmul(m[4 * r], x[0]);
        acc = cfma(m[4 * r + 1], x[1], acc);
        acc = cfma(m[4 * r + 2], x[2], acc);
        acc = cfma(m[4 * r + 3], x[3], acc);
        v[idx[r]] = acc;
      }
    }
}

// a 3-qubit matrix whose qubit j sits on cube bit PJ (the permutation P0 P1 P2)
template <class R, int P0, int P1, int P2>
__device__ __forceinline__ void chain_fiber(V<R> (&v)[8], const PassParams<R>& P, uint32_t c0) {
  const V<R>* m = P.cpool + c0;
  auto mat = [&](int i) { return m[i]; };
  V<R> x[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) x[b] = v[((b & 1) << P0) | (((b >> 1) & 1) << P1) | (((b >> 2) & 1) << P2)];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    V<R> acc = cmul(mat(r * 8), x[0]);
#pragma unroll
    for (int b = 1; b < 8; ++b) acc = cfma(mat(r * 8 + b), x[b], acc);
    v[((r & 1) << P0) | (((r >> 1) & 1) << P1) | (((r >> 2) & 1) << P2)] = acc;
  }
}

template <class R, int X>
__device__ __forceinline__ void chain_pairswap(V<R> (&v)[8], uint32_t em, uint32_t flags, V<R> ci, V<R> cj) {
  const bool ui = flags & 1, uj = (flags >> 1) & 1;
#pragma unroll
  for (int b = 0; b < 8; ++b)
    if ((em >> b) & 1) {
      const V<R> vi = v[b], vj = v[b ^ X];
      v[b] = ui ? vj : cmul(ci, vj);
      v[b ^ X] = uj ? vi : cmul(cj, vi);
    }
}

template <class R>
__device__ __forceinline__ V<R> phasepoly_elem(V<R> v, uint64_t i, const TileOp& op, const V<R>* cp, const uint32_t* up,
                                               const uint64_t* pp, bool& changed) {
  changed = false;
  if (is_zero(v)) return v;
  const uint32_t* u = up + op.up;
  const uint32_t bits = u[0];
  const bool use_table = u[1], s_one = u[2];
  const uint64_t constant = uint64_t(u[3]) | (uint64_t(u[4]) << 32);
  const int nt = int(op.k);
  const uint32_t* start = u + 5;
  const uint32_t* coeff = start + nt + 1;
  uint64_t f = constant;
  for (int tt = 0; tt < nt; ++tt) {
    int all = 1;
    for (uint32_t l = start[tt]; l < start[tt + 1]; ++l) all &= __popcll(pp[op.gz + l] & i) & 1;
    if (all) f += coeff[tt];
  }
  f &= (uint64_t(1) << bits) - 1;
  V<R> c;
  if (use_table) {
    c = cp[op.cp + 1 + f];
    if (is_one_v(c)) return v;
  } else {
    if (f == 0 && s_one) return v;
    const double2 rr = pass_root(f, bits);
    c.x = R(rr.x);
    c.y = R(rr.y);
    if (!s_one) c = cmul(cp[op.cp], c);
  }
  changed = true;
  return cmul(c, v);
}

template <class R>
__device__ void tile_chain(SwTile<R> t, uint32_t tsz, const TileOp* ops, const PassParams<R>& P, uint64_t base) {
  const TileOp& head = ops[0];
  const uint32_t nsub = head.k;
  const uint8_t cpos[3] = {uint8_t(head.l0 & 0xff), uint8_t((head.l0 >> 8) & 0xff), uint8_t((head.l0 >> 16) & 0xff)};
  uint32_t loff[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) loff[b] = ((b & 1u) << cpos[0]) | (((b >> 1) & 1u) << cpos[1]) | (((b >> 2) & 1u) << cpos[2]);
  for (uint32_t grp = threadIdx.x; grp < (tsz >> 3); grp += blockDim.x) {
    const uint32_t gb = insert_zeros32(grp, cpos, 3);
    uint32_t e[8];
    V<R> v[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      e[b] = gb | loff[b];
      v[b] = t[e[b]];
    }
    for (uint32_t s = 0; s < nsub; ++s) {
      const TileOp& op = ops[1 + s];
      if ((base & op.gfix) != op.gval) continue;
      // the op's constants (at most 64 of them: a 3-qubit matrix)
      V<R> m[4];
      switch (op.kind) {
        case TK_DENSE1:
#pragma unroll
          for (int i = 0; i < 4; ++i) m[i] = pconst(P, op.cp + i);
          if (op.reg == 0) chain_dense1<R, 0>(v, m);
          else if (op.reg == 1) chain_dense1<R, 1>(v, m);
          else chain_dense1<R, 2>(v, m);
          break;
        case TK_DENSE2:
          switch (op.reg) {  // ja | jb << 4
            case 0x10: chain_dense2<R, 0, 1>(v, P, op.cp); break;
            case 0x20: chain_dense2<R, 0, 2>(v, P, op.cp); break;
            case 0x01: chain_dense2<R, 1, 0>(v, P, op.cp); break;
            case 0x21: chain_dense2<R, 1, 2>(v, P, op.cp); break;
            case 0x02: chain_dense2<R, 2, 0>(v, P, op.cp); break;
            default: chain_dense2<R, 2, 1>(v, P, op.cp); break;
          }
          break;
        case TK_FIBER:
          switch (op.reg) {  // p0 | p1 << 4 | p2 << 8
            case 0x210: chain_fiber<R, 0, 1, 2>(v, P, op.cp); break;
            case 0x120: chain_fiber<R, 0, 2, 1>(v, P, op.cp); break;
            case 0x201: chain_fiber<R, 1, 0, 2>(v, P, op.cp); break;
            case 0x021: chain_fiber<R, 1, 2, 0>(v, P, op.cp); break;
            case 0x102: chain_fiber<R, 2, 0, 1>(v, P, op.cp); break;
            default: chain_fiber<R, 2, 1, 0>(v, P, op.cp); break;
          }
          break;
        case TK_PAIRSWAP: {
          if ((gb & op.gml) != op.gvl) break;
          const V<R> ci = pconst(P, op.cp), cj = pconst(P, op.cp + 1);
          const uint32_t em = op.reg >> 8;
          switch (op.reg & 7) {
            case 1: chain_pairswap<R, 1>(v, em, op.flags, ci, cj); break;
            case 2: chain_pairswap<R, 2>(v, em, op.flags, ci, cj); break;
            case 3: chain_pairswap<R, 3>(v, em, op.flags, ci, cj); break;
            case 4: chain_pairswap<R, 4>(v, em, op.flags, ci, cj); break;
            case 5: chain_pairswap<R, 5>(v, em, op.flags, ci, cj); break;
            case 6: chain_pairswap<R, 6>(v, em, op.flags, ci, cj); break;
            default: chain_pairswap<R, 7>(v, em, op.flags, ci, cj); break;
          }
          break;
        }
        case TK_DIAG_CONST: {
          if ((gb & op.gml) != op.gvl) break;
          const V<R> c = pconst(P, op.cp);
          const uint32_t em = op.reg;  // the cube elements with the fixed pattern
#pragma unroll
          for (int b = 0; b < 8; ++b)
            if (((em >> b) & 1) && !is_zero(v[b])) v[b] = cmul(c, v[b]);
          break;
        }
        case TK_DIAG_1Q: {
          const V<R> c0 = pconst(P, op.cp), c1 = pconst(P, op.cp + 1);
          // the cube elements whose qubit bit is 1: from the cube, the group or the tile base
          const uint32_t ones = (op.flags & 4) ? op.reg
                              : (op.flags & 1) ? (((base >> op.l1) & 1) ? 0xffu : 0u)
                                               : (((gb >> op.l0) & 1) ? 0xffu : 0u);
#pragma unroll
          for (int b = 0; b < 8; ++b)
            if (!is_zero(v[b])) v[b] = cmul(((ones >> b) & 1) ? c1 : c0, v[b]);
          break;
        }
        case TK_DIAG_TABLE: {
          const int k = int(op.k);
          const int nf = __popc(op.lfix);
          const uint32_t* qp = P.upool + op.up;
          const uint8_t* unit = reinterpret_cast<const uint8_t*>(qp + k + nf);
          uint32_t xout = 0;
          for (int j = 0; j < k; ++j)
            if (qp[j] >= 256) xout |= uint32_t((base >> (qp[j] - 256)) & 1u) << j;
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            if ((e[b] & op.lfix) != op.lones) continue;
            uint32_t x = xout;
            for (int j = 0; j < k; ++j)
              if (qp[j] < 256) x |= ((e[b] >> qp[j]) & 1u) << j;
            if (unit[x]) continue;
            if (!is_zero(v[b])) v[b] = cmul(pconst(P, op.cp + x), v[b]);
          }
          break;
        }
        case TK_PHASEPOLY: {
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            bool ch;
            v[b] = phasepoly_elem<R>(v[b], base | deposit(e[b], P.g), op, P.cpool, P.upool, P.ppool, ch);
          }
          break;
        }
        default: break;
      }
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) t[e[b]] = v[b];
  }
}

template <class R>
__global__ void __launch_bounds__(PASS_THREADS) k_plain_pass(const __grid_constant__ PassParams<R> P) {
  extern __shared__ __align__(16) unsigned char pass_smem[];
  const PassGeom& g = P.g;
  const uint32_t tsz = 1u << g.T;
  V<R>* buf[2] = {reinterpret_cast<V<R>*>(pass_smem), reinterpret_cast<V<R>*>(pass_smem) + tsz};
  __shared__ uint64_t dround[MAX_TILE_BITS > 9 ? (1 << MAX_TILE_BITS) / 32 : 32];
  __shared__ TileOp s_ops[MAX_PASS_OPS];  // the ops, read from shared memory in the tile loop
  const uint32_t nr = (tsz + blockDim.x - 1) / blockDim.x;  // element rounds per thread
  for (uint32_t r = threadIdx.x; r < nr; r += blockDim.x) dround[r] = deposit(r * blockDim.x, g);
  {
    const uint32_t words = P.nops * uint32_t(sizeof(TileOp) / 4);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(P.ops);
    uint32_t* dst = reinterpret_cast<uint32_t*>(s_ops);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  const uint64_t dthread = deposit(threadIdx.x, g);
  __syncthreads();
  auto load = [&](uint64_t tile, V<R>* dst) {
    const V<R>* src = P.amp + (tile_base_of(tile, g) | dthread);
    for (uint32_t r = 0; r < nr; ++r) {
      const uint32_t e = threadIdx.x + r * blockDim.x;
      if (e >= tsz) break;
      const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(&SwTile<R>{dst}[e]));
      if constexpr (sizeof(V<R>) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + dround[r]) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src + dround[r]) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  uint64_t tile = blockIdx.x;
  if (tile < P.ntiles) load(tile, buf[0]);
  for (uint32_t it = 0; tile < P.ntiles; ++it, tile += gridDim.x) {
    const SwTile<R> t{buf[it & 1]};
    const uint64_t next = tile + gridDim.x;
    if (next < P.ntiles) {
      load(next, buf[(it & 1) ^ 1]);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    const uint64_t base = tile_base_of(tile, g);
    for (uint32_t o = 0; o < P.nops; ++o) {
      const TileOp& op = s_ops[o];
      if (op.kind == TK_CHAIN) {
        tile_chain<R>(t, tsz, s_ops + o, P, base);
        o += op.k;
        __syncthreads();
        continue;
      }
      if ((base & op.gfix) != op.gval) continue;  // uniform over the CTA
      switch (op.kind) {
        case TK_DENSE1: tile_dense1<R>(t, tsz, op, P.cpool); break;
        case TK_DENSE2: tile_dense2<R>(t, tsz, op, P.cpool); break;
        case TK_FIBER: tile_fiber<R, 3>(t, tsz, op, P.cpool, P.upool); break;
        case TK_DIAG_CONST: tile_diag_const<R>(t, tsz, op, P.cpool, P.upool); break;
        case TK_DIAG_1Q: tile_diag_1q<R>(t, tsz, op, P.cpool, base); break;
        case TK_DIAG_TABLE: tile_diag_table<R>(t, tsz, op, P.cpool, P.upool, base); break;
        case TK_PAIRSWAP: tile_pairswap<R>(t, tsz, op, P.cpool, P.upool); break;
        case TK_PHASEPOLY: tile_phasepoly<R>(t, tsz, op, P.cpool, P.upool, P.ppool, base, dthread, dround); break;
        default: break;
      }
      __syncthreads();
    }
    V<R>* dst = P.amp + (base | dthread);
    for (uint32_t r = 0; r < nr; ++r) {
      const uint32_t e = threadIdx.x + r * blockDim.x;
      if (e >= tsz) break;
      dst[dround[r]] = t[e];
    }
    __syncthreads();  // the buffer is refilled two tiles later
  }
}

// ---------------------------------------------------------------------------
// host: how the gate-by-gate path would apply a lowered gate (its dispatch
// rules, kernels_plain.cu launch_*), as a tile op over global qubits
// ---------------------------------------------------------------------------
bool one_c(const CplxD& c) { return c.re == 1.0 && c.im == 0.0; }
bool zero_c(const CplxD& c) { return c.re == 0.0 && c.im == 0.0; }

struct GateForm {
  uint32_t kind = 0;
  bool tileable = false;
  bool nothing = false;
  std::vector<uint32_t> qubits;   // gate qubits (local order)
  uint64_t moving = 0;            // qubits whose amplitudes the gate mixes or moves
  std::vector<CplxD> c;           // matrix / constants / table
  uint64_t fixmask = 0, ones = 0, xmask = 0;
  uint32_t flags = 0;
  std::vector<uint8_t> unit;
  const PolyTerms* poly = nullptr;
};

GateForm form_diag_table(const std::vector<uint32_t>& qubits, const std::vector<CplxD>& diag) {
  GateForm f;
  const int k = int(qubits.size());
  f.qubits = qubits;
  if (k > MAX_TABLE_K) return f;
  const int gd = 1 << k;
  uint32_t fixed = (1u << k) - 1;
  bool any = false;
  int nphased = 0;
  for (int x = 0; x < gd; ++x)
    if (!one_c(diag[x])) fixed &= uint32_t(x), any = true, ++nphased;
  if (!any) {
    f.nothing = true;
    return f;
  }
  f.tileable = true;
  if (nphased == 1 && fixed == uint32_t(gd - 1)) {
    f.kind = TK_DIAG_CONST;
    for (uint32_t q : qubits) f.fixmask |= uint64_t(1) << q;
    f.ones = f.fixmask;
    f.c = {diag[gd - 1]};
    return f;
  }
  if (k == 1) {
    f.kind = TK_DIAG_1Q;
    f.c = {diag[0], diag[1]};
    return f;
  }
  f.kind = TK_DIAG_TABLE;
  for (int j = 0; j < k; ++j)
    if ((fixed >> j) & 1) f.fixmask |= uint64_t(1) << qubits[j];
  f.ones = f.fixmask;
  f.c.assign(diag.begin(), diag.end());
  f.unit.resize(gd);
  for (int x = 0; x < gd; ++x) f.unit[x] = one_c(diag[x]) ? 1 : 0;
  return f;
}

// the share of the register the gate's own kernel reads and writes (its
// algorithmic bytes over a full pass: the sectors that hold an amplitude it changes)
double touched_share(const GateForm& f, int precision) {
  const uint64_t below = precision == NCSIM_C128 ? 1 : 3;  // index bits inside a 32-byte sector
  auto share = [&](uint64_t fixed) { return std::ldexp(1.0, -__builtin_popcountll(fixed & ~below)); };
  switch (f.kind) {
    case TK_DIAG_CONST: case TK_DIAG_TABLE: return share(f.fixmask);
    case TK_PAIRSWAP: {
      const uint64_t ctrl = f.fixmask & ~f.xmask;
      return std::min(1.0, share(ctrl) * 2.0 / double(uint64_t(1) << __builtin_popcountll(f.xmask)));
    }
    default: return 1.0;
  }
}

GateForm form_of(const LoweredOp& op) {
  GateForm f;
  f.qubits = op.qubits;
  switch (op.kind) {
    case LoweredKind::Nothing: f.nothing = true; return f;
    case LoweredKind::Dense: {
      const int k = int(op.qubits.size());
      const int gd = 1 << k;
      bool diag = true;
      for (int r = 0; r < gd && diag; ++r)
        for (int c = 0; c < gd; ++c)
          if (r != c && !zero_c(op.matrix[size_t(r) * gd + c])) {
            diag = false;
            break;
          }
      if (diag && k <= MAX_TABLE_K) {
        std::vector<CplxD> d(gd);
        for (int x = 0; x < gd; ++x) d[x] = op.matrix[size_t(x) * gd + x];
        return form_diag_table(op.qubits, d);
      }
      if (k > MAX_FIBER_K) return f;
      f.tileable = true;
      f.kind = k == 1 ? TK_DENSE1 : k == 2 ? TK_DENSE2 : TK_FIBER;
      for (uint32_t q : op.qubits) f.moving |= uint64_t(1) << q;
      f.c = op.matrix;
      return f;
    }
    case LoweredKind::Monomial: {
      const int k = int(op.qubits.size());
      const int gd = 1 << k;
      bool diagonal = true;
      for (int x = 0; x < gd; ++x) diagonal &= op.image[x] == uint32_t(x);
      if (diagonal && k <= MAX_TABLE_K) return form_diag_table(op.qubits, op.matrix);
      if (k > MAX_TABLE_K) return f;
      // the pair-swap shape of launch_perm_table; other tables run as their own kernels
      uint32_t d = 0;
      bool ok = true;
      std::vector<uint32_t> moved;
      for (int x = 0; x < gd; ++x)
        if (op.image[x] != uint32_t(x)) {
          moved.push_back(uint32_t(x));
          const uint32_t dx = op.image[x] ^ uint32_t(x);
          if (d == 0) d = dx;
          ok &= dx == d && op.image[op.image[x]] == uint32_t(x);
        } else {
          ok &= one_c(op.matrix[x]);
        }
      if (!ok || !d) return f;
      const uint32_t hbit = 1u << (31 - __builtin_clz(d));
      std::vector<uint32_t> leads;
      for (uint32_t x : moved)
        if (!(x & hbit)) leads.push_back(x);
      uint32_t ones = (1u << k) - 1, zeros = (1u << k) - 1;
      for (uint32_t x : leads) ones &= x, zeros &= ~x;
      const int nfixed = __builtin_popcount(ones) + __builtin_popcount(zeros);
      ok &= leads.size() == (size_t(1) << (k - nfixed)) && (zeros & hbit);
      if (!ok) return f;
      const CplxD c_j = op.matrix[leads[0]], c_i = op.matrix[leads[0] ^ d];
      for (uint32_t x : leads)
        ok &= op.matrix[x].re == c_j.re && op.matrix[x].im == c_j.im && op.matrix[x ^ d].re == c_i.re &&
              op.matrix[x ^ d].im == c_i.im;
      if (!ok) return f;
      f.tileable = true;
      f.kind = TK_PAIRSWAP;
      for (int j = 0; j < k; ++j) {
        if (((ones | zeros) >> j) & 1) f.fixmask |= uint64_t(1) << op.qubits[j];
        if ((ones >> j) & 1) f.ones |= uint64_t(1) << op.qubits[j];
        if ((d >> j) & 1) f.xmask |= uint64_t(1) << op.qubits[j];
      }
      f.moving = f.xmask;
      f.c = {c_i, c_j};
      f.flags = (one_c(c_i) ? 1u : 0u) | (one_c(c_j) ? 2u : 0u);
      return f;
    }
    case LoweredKind::PhasePoly: {
      const PolyTerms& t = op.poly;
      const int nt = int(t.coeffs.size());
      if (nt == 0 && t.scalar_is_one && (t.constant & ((t.bits >= 64 ? 0 : (uint64_t(1) << t.bits)) - 1)) == 0) {
        f.nothing = true;
        return f;
      }
      if (nt > MAX_PASS_TERMS || t.parities.size() > size_t(MAX_PASS_PARITIES) || t.bits > 32) return f;
      f.tileable = true;
      f.kind = TK_PHASEPOLY;
      f.poly = &op.poly;
      return f;
    }
    case LoweredKind::Pauli:  // Pauli gates come only from the API, not from circuit text: own kernel
      if (op.x == 0 && op.z == 0 && (op.phase & 3) == 0) f.nothing = true;
      return f;
  }
  return f;
}

template <class R>
V<R> cvt(const CplxD& c) {
  V<R> r;
  r.x = R(c.re);
  r.y = R(c.im);
  return r;
}

// the window's tile-local position of each global bit (-1: outside)
struct Window {
  PassGeom g{};
  int local[64];
  uint64_t mask = 0;
};

Window make_window(uint32_t n, int T, uint64_t moving) {
  Window W;
  uint64_t m = moving;
  for (uint32_t q = 0; q < n && __builtin_popcountll(m) < T; ++q) m |= uint64_t(1) << q;
  W.mask = m;
  int w = 0;
  while (w < int(n) && ((m >> w) & 1)) ++w;
  W.g.T = __builtin_popcountll(m);
  W.g.w = w;
  W.g.nh = 0;
  for (int i = 0; i < 64; ++i) W.local[i] = -1;
  for (int q = 0; q < w; ++q) W.local[q] = q;
  for (uint32_t q = uint32_t(w); q < n; ++q)
    if ((m >> q) & 1) {
      W.local[q] = w + W.g.nh;
      W.g.hq[W.g.nh++] = uint8_t(q);
    }
  return W;
}

uint32_t local_mask(const Window& W, uint64_t gm) {
  uint32_t l = 0;
  for (int q = 0; q < 64; ++q)
    if (((gm >> q) & 1) && W.local[q] >= 0) l |= 1u << W.local[q];
  return l;
}

}  // namespace

// A planned run of gates: passes and the gates that run as their own kernels.
struct PlainPlan {
  struct Item {
    bool pass = false;
    size_t gate = 0;              // direct: index into `gates`
    Window win;
    std::vector<TileOp> ops;
    uint32_t cbeg = 0, cend = 0;  // the pass's range of the constant pool
  };
  int precision = NCSIM_C128;
  std::vector<const LoweredOp*> gates;
  std::vector<Item> items;
  std::vector<double> cpool;      // complex values, interleaved
  std::vector<uint32_t> upool;
  std::vector<uint64_t> ppool;
  int device = -1;
  void* d_cpool = nullptr;
  uint32_t* d_upool = nullptr;
  uint64_t* d_ppool = nullptr;
  size_t passes = 0, pass_gates = 0;
  ~PlainPlan() {
    if (device >= 0) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(device);
      cudaFree(d_cpool);
      cudaFree(d_upool);
      cudaFree(d_ppool);
      cudaSetDevice(cur);
    }
  }
};

namespace {

int pass_tile_bits(uint32_t n) { return int(std::min<uint32_t>(n, MAX_TILE_BITS)); }

// encode a gate form against a window (appends pool data)
TileOp encode(const GateForm& f, const Window& W, PlainPlan& P) {
  TileOp op{};
  op.kind = f.kind;
  auto push_c = [&](const CplxD& c) {
    P.cpool.push_back(c.re);
    P.cpool.push_back(c.im);
  };
  op.cp = uint32_t(P.cpool.size() / 2);
  op.up = uint32_t(P.upool.size());
  const uint64_t out = ~W.mask;
  switch (f.kind) {
    case TK_DENSE1:
      op.l0 = uint32_t(W.local[f.qubits[0]]);
      for (auto& c : f.c) push_c(c);
      break;
    case TK_DENSE2:
      op.l0 = uint32_t(W.local[f.qubits[0]]);
      op.l1 = uint32_t(W.local[f.qubits[1]]);
      for (auto& c : f.c) push_c(c);
      break;
    case TK_FIBER: {
      const int k = int(f.qubits.size());
      op.k = uint32_t(k);
      std::vector<uint32_t> lp;
      for (uint32_t q : f.qubits) lp.push_back(uint32_t(W.local[q]));
      std::vector<uint32_t> sorted = lp;
      std::sort(sorted.begin(), sorted.end());
      for (uint32_t v : sorted) P.upool.push_back(v);
      for (int b = 0; b < (1 << k); ++b) {
        uint32_t o = 0;
        for (int j = 0; j < k; ++j)
          if ((b >> j) & 1) o |= 1u << lp[j];
        P.upool.push_back(o);
      }
      for (auto& c : f.c) push_c(c);
      break;
    }
    case TK_DIAG_CONST:
    case TK_PAIRSWAP: {
      op.lfix = local_mask(W, f.fixmask);
      op.lones = local_mask(W, f.ones);
      op.gfix = f.fixmask & out;
      op.gval = f.ones & out;
      op.lx = local_mask(W, f.xmask);
      op.flags = f.flags;
      for (int b = 0; b < MAX_TILE_BITS; ++b)
        if ((op.lfix >> b) & 1) P.upool.push_back(uint32_t(b));
      for (auto& c : f.c) push_c(c);
      break;
    }
    case TK_DIAG_1Q: {
      const uint32_t q = f.qubits[0];
      if (W.local[q] >= 0) {
        op.l0 = uint32_t(W.local[q]);
      } else {
        op.flags = 1;
        op.l1 = q;
      }
      for (auto& c : f.c) push_c(c);
      break;
    }
    case TK_DIAG_TABLE: {
      const int k = int(f.qubits.size());
      op.k = uint32_t(k);
      op.lfix = local_mask(W, f.fixmask);
      op.lones = op.lfix;
      op.gfix = f.fixmask & out;
      op.gval = f.fixmask & out;
      for (uint32_t q : f.qubits) P.upool.push_back(W.local[q] >= 0 ? uint32_t(W.local[q]) : 256u + q);
      for (int b = 0; b < MAX_TILE_BITS; ++b)
        if ((op.lfix >> b) & 1) P.upool.push_back(uint32_t(b));
      const size_t nb = f.unit.size();
      std::vector<uint32_t> words((nb + 3) / 4, 0);
      for (size_t x = 0; x < nb; ++x) words[x / 4] |= uint32_t(f.unit[x]) << (8 * (x % 4));
      P.upool.insert(P.upool.end(), words.begin(), words.end());
      for (auto& c : f.c) push_c(c);
      break;
    }
    case TK_PHASEPOLY: {
      const PolyTerms& t = *f.poly;
      const int nt = int(t.coeffs.size());
      op.k = uint32_t(nt);
      op.gz = uint32_t(P.ppool.size());  // parity offset
      P.upool.push_back(t.bits);
      P.upool.push_back(t.root_table.empty() ? 0u : 1u);
      P.upool.push_back(t.scalar_is_one ? 1u : 0u);
      P.upool.push_back(uint32_t(t.constant));
      P.upool.push_back(uint32_t(t.constant >> 32));
      for (int i = 0; i <= nt; ++i) P.upool.push_back(t.term_start[i]);
      for (int i = 0; i < nt; ++i) P.upool.push_back(uint32_t(t.coeffs[i]));
      P.ppool.insert(P.ppool.end(), t.parities.begin(), t.parities.end());
      push_c(t.scalar);
      for (auto& c : t.root_table) push_c(c);
      break;
    }
  }
  return op;
}

// tile bits an op couples (0 for the ops that act on each element alone)
uint32_t coupled_bits(const TileOp& op, const std::vector<uint32_t>& upool) {
  switch (op.kind) {
    case TK_DENSE1: return 1u << op.l0;
    case TK_DENSE2: return (1u << op.l0) | (1u << op.l1);
    case TK_FIBER: return (1u << upool[op.up]) | (1u << upool[op.up + 1]) | (1u << upool[op.up + 2]);
    case TK_PAIRSWAP: return op.lx;
    default: return 0;
  }
}

// Groups a pass's ops into chains: maximal runs of two or more consecutive ops
// whose coupled bits fit in one cube of three tile bits.
std::vector<TileOp> chainify(const std::vector<TileOp>& ops, const std::vector<uint32_t>& upool, int T) {
  std::vector<TileOp> out;
  size_t i = 0;
  while (i < ops.size()) {
    uint32_t C = 0;
    size_t j = i;
    while (j < ops.size()) {
      const uint32_t need = coupled_bits(ops[j], upool);
      if (__builtin_popcount(C | need) > 3) break;
      C |= need;
      ++j;
    }
    if (j - i < 2 || T < 3) {
      out.push_back(ops[i]);
      i = i + 1;
      continue;
    }
    for (int b = 0; b < T && __builtin_popcount(C) < 3; ++b) C |= 1u << b;
    int cpos[3], nc = 0;
    for (int b = 0; b < T; ++b)
      if ((C >> b) & 1) cpos[nc++] = b;
    auto cube = [&](uint32_t l) {
      for (int q = 0; q < 3; ++q)
        if (cpos[q] == int(l)) return uint32_t(q);
      return 0u;
    };
    const uint32_t cmask = (1u << cpos[0]) | (1u << cpos[1]) | (1u << cpos[2]);
    uint32_t loff[8];
    for (int b = 0; b < 8; ++b)
      loff[b] = ((b & 1u) << cpos[0]) | (((b >> 1) & 1u) << cpos[1]) | (((b >> 2) & 1u) << cpos[2]);
    // the cube elements b whose cube bits match the op's fixed pattern there
    auto elements = [&](uint32_t lfix, uint32_t lones) {
      uint32_t em = 0;
      for (int b = 0; b < 8; ++b)
        if ((loff[b] & lfix) == (lones & cmask)) em |= 1u << b;
      return em;
    };
    TileOp head{};
    head.kind = TK_CHAIN;
    head.k = uint32_t(j - i);
    head.l0 = uint32_t(cpos[0]) | (uint32_t(cpos[1]) << 8) | (uint32_t(cpos[2]) << 16);
    out.push_back(head);
    for (size_t o = i; o < j; ++o) {
      TileOp op = ops[o];
      switch (op.kind) {
        case TK_DENSE1: op.reg = cube(op.l0); break;
        case TK_DENSE2: op.reg = cube(op.l0) | (cube(op.l1) << 4); break;
        case TK_FIBER: {
          uint32_t r = 0;
          for (int q = 0; q < 3; ++q) r |= cube(uint32_t(__builtin_ctz(upool[op.up + 3 + (1u << q)]))) << (4 * q);
          op.reg = r;
          break;
        }
        case TK_PAIRSWAP: {
          uint32_t r = 0;
          for (int b = 0; b < T; ++b)
            if ((op.lx >> b) & 1) r |= 1u << cube(uint32_t(b));
          op.reg = r | (elements(op.lfix, op.lones) << 8);
          op.gml = op.lfix & ~cmask;
          op.gvl = op.lones & ~cmask;
          break;
        }
        case TK_DIAG_CONST:
          op.reg = elements(op.lfix, op.lones);
          op.gml = op.lfix & ~cmask;
          op.gvl = op.lones & ~cmask;
          break;
        case TK_DIAG_1Q:
          if (!(op.flags & 1) && ((cmask >> op.l0) & 1)) {
            op.flags |= 4;
            op.reg = elements(1u << op.l0, 1u << op.l0);
          }
          break;
        default: break;
      }
      out.push_back(op);
    }
    i = j;
  }
  return out;
}

}  // namespace

// Plans the gates of a run for one register.  Returns null when no pass would
// carry two or more gates (the gate-by-gate path then runs them as before).
std::shared_ptr<PlainPlan> plan_plain_passes(uint32_t n, int precision, const std::vector<const LoweredOp*>& gates) {
  if (n < 8) return nullptr;
  auto P = std::make_shared<PlainPlan>();
  P->precision = precision;
  P->gates = gates;
  const int T = pass_tile_bits(n);
  std::vector<GateForm> forms(gates.size());
  for (size_t i = 0; i < gates.size(); ++i) forms[i] = form_of(*gates[i]);
  std::vector<size_t> cur;
  uint64_t moving = 0;
  auto flush = [&] {
    if (cur.empty()) return;
    // a pass reads and writes the whole register once; gates whose own kernels
    // touch less than that between them stay gate by gate
    double shares = 0.0;
    for (size_t i : cur) shares += touched_share(forms[i], precision);
    if (cur.size() == 1 || shares < 1.25) {
      for (size_t i : cur) {
        PlainPlan::Item it;
        it.gate = i;
        P->items.push_back(it);
      }
    } else {
      PlainPlan::Item it;
      it.pass = true;
      it.win = make_window(n, T, moving);
      std::vector<TileOp> ops;
      it.cbeg = uint32_t(P->cpool.size() / 2);
      for (size_t i : cur) ops.push_back(encode(forms[i], it.win, *P));
      it.cend = uint32_t(P->cpool.size() / 2);
      it.ops = chainify(ops, P->upool, it.win.g.T);
      if (it.ops.size() > size_t(MAX_PASS_OPS)) throw Error(NCSIM_ERR_INVALID, "tiled pass: too many ops");
      P->passes += 1;
      P->pass_gates += cur.size();
      P->items.push_back(std::move(it));
    }
    cur.clear();
    moving = 0;
  };
  for (size_t i = 0; i < gates.size(); ++i) {
    const GateForm& f = forms[i];
    if (f.nothing) continue;
    if (!f.tileable) {
      flush();
      PlainPlan::Item it;
      it.gate = i;
      P->items.push_back(it);
      continue;
    }
    // chains add at most one head per op: a pass of MAX_PASS_OPS / 2 gates fits in shared memory
    if (__builtin_popcountll(moving | f.moving) > T || cur.size() >= size_t(MAX_PASS_OPS / 2)) flush();
    cur.push_back(i);
    moving |= f.moving;
  }
  flush();
  if (P->passes == 0) return nullptr;
  return P;
}

// passes, gates in passes, chains and ops in chains, and gates left to their own kernels
std::string plain_plan_summary(const PlainPlan& P) {
  size_t chains = 0, chained = 0, direct = 0;
  for (const auto& it : P.items) {
    if (!it.pass) {
      ++direct;
      continue;
    }
    for (const auto& op : it.ops)
      if (op.kind == TK_CHAIN) ++chains, chained += op.k;
  }
  return "passes " + std::to_string(P.passes) + ", gates in passes " + std::to_string(P.pass_gates) + ", chains " +
         std::to_string(chains) + " holding " + std::to_string(chained) + " ops, own kernels " + std::to_string(direct);
}

size_t plain_plan_passes(const PlainPlan& P) { return P.passes; }
size_t plain_plan_pass_gates(const PlainPlan& P) { return P.pass_gates; }

void apply_lowered(ncsim_state* s, const LoweredOp& op);

template <class R>
void launch_pass(ncsim_state* s, const PlainPlan& P, const PlainPlan::Item& it) {
  PassParams<R> pp{};
  pp.amp = reinterpret_cast<V<R>*>(s->amp);
  pp.g = it.win.g;
  pp.ntiles = s->len >> it.win.g.T;
  pp.nops = uint32_t(it.ops.size());
  std::copy(it.ops.begin(), it.ops.end(), pp.ops);

  pp.upool = P.d_upool;
  pp.ppool = P.d_ppool;
  // the complex pool as this precision's values
  pp.cpool = reinterpret_cast<const V<R>*>(P.d_cpool);
  const size_t smem = 2 * (size_t(1) << it.win.g.T) * sizeof(V<R>);
  {
    // the kernel's shared-memory limit, set once per device and precision (host threads may race here)
    static std::mutex mu;
    static bool done[64][2] = {};
    std::lock_guard<std::mutex> lk(mu);
    const int dev = s->device;
    if (dev < 0 || dev >= 64 || !done[dev][sizeof(R) == 8]) {
      NCSIM_CUDA(cudaFuncSetAttribute(k_plain_pass<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(2 * (size_t(1) << MAX_TILE_BITS) * sizeof(V<R>))));
      if (dev >= 0 && dev < 64) done[dev][sizeof(R) == 8] = true;
    }
  }
  const uint64_t grid = std::min<uint64_t>(pp.ntiles, uint64_t(sm_count()) * (sizeof(R) == 8 ? 1 : 2));
  ProfScope ps(s, K_PLAIN_PASS, 2.0 * double(s->len) * double(s->elem_bytes()));
  k_plain_pass<R><<<unsigned(grid), PASS_THREADS, smem, s->stream>>>(pp);
  NCSIM_LAUNCHED("k_plain_pass");
}

void run_plain_plan(ncsim_state* s, PlainPlan& P) {
  if (P.device < 0) {
    // The pools go up on the state's own stream and are waited for: a cudaMemcpy from pageable
    // memory runs on the legacy stream and may return before its DMA lands, and the pass
    // kernels run on a non-blocking stream that does not wait for the legacy one.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    NCSIM_CUDA(cudaStreamIsCapturing(s->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) throw Error(NCSIM_ERR_DEVICE, "a gate plan is uploaded outside stream capture");
    const bool dbl = s->precision == NCSIM_C128;
    const size_t nc = P.cpool.size() / 2;
    std::vector<float> f;
    if (!dbl) f.assign(P.cpool.begin(), P.cpool.end());
    NCSIM_CUDA(cudaMalloc(&P.d_cpool, std::max<size_t>(nc, 1) * (dbl ? sizeof(double2) : sizeof(float2))));
    NCSIM_CUDA(cudaMalloc(&P.d_upool, std::max<size_t>(P.upool.size(), 1) * sizeof(uint32_t)));
    NCSIM_CUDA(cudaMalloc(&P.d_ppool, std::max<size_t>(P.ppool.size(), 1) * sizeof(uint64_t)));
    P.device = s->device;  // the destructor frees the pools from here on
    if (nc)
      NCSIM_CUDA(cudaMemcpyAsync(P.d_cpool, dbl ? static_cast<const void*>(P.cpool.data()) : f.data(),
                                 nc * (dbl ? sizeof(double2) : sizeof(float2)), cudaMemcpyHostToDevice, s->stream));
    if (!P.upool.empty())
      NCSIM_CUDA(cudaMemcpyAsync(P.d_upool, P.upool.data(), P.upool.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                 s->stream));
    if (!P.ppool.empty())
      NCSIM_CUDA(cudaMemcpyAsync(P.d_ppool, P.ppool.data(), P.ppool.size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
                                 s->stream));
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  }
  if (P.device != s->device) throw Error(NCSIM_ERR_DEVICE, "a gate plan stays on the device it was built for");
  for (const auto& it : P.items) {
    if (!it.pass) {
      apply_lowered(s, *P.gates[it.gate]);
      continue;
    }
    if (s->precision == NCSIM_C128) launch_pass<double>(s, P, it);
    else launch_pass<float>(s, P, it);
  }
}

}  // namespace ncsim
