// Plain-path kernels: one kernel per gate over the whole register, FP64
// (complex128) or FP32 (complex64) amplitudes, FP64 reductions.
//
// Every kernel is HBM-bound; each one reads and writes only the 32-byte
// sectors that hold amplitudes the operation changes (diagonal and
// controlled gates enumerate exactly the affected index subset).  Index
// arithmetic is 64-bit (registers up to 34 qubits).
#include "engine.cuh"

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

namespace ncsim {

namespace {

constexpr int THREADS = 256;

template <class R>
using V = typename VecOf<R>::T;

template <class R>
__device__ __forceinline__ V<R> to_v(double2 c) {
  V<R> r;
  r.x = R(c.x);
  r.y = R(c.y);
  return r;
}

// ---------------------------------------------------------------------------
// 1-qubit dense gate: the pair (i0, i0 + 2^q) per thread, two pairs in flight
// ---------------------------------------------------------------------------
template <class R>
struct Mat1 {
  V<R> m00, m01, m10, m11;
};

template <class R>
__global__ void __launch_bounds__(THREADS) k_dense1(V<R>* __restrict__ a, uint64_t npairs, int q, Mat1<R> m) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t lo = (uint64_t(1) << q) - 1;
  uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; p + stride < npairs; p += 2 * stride) {
    uint64_t pa = p, pb = p + stride;
    uint64_t ia = ((pa & ~lo) << 1) | (pa & lo), ib = ((pb & ~lo) << 1) | (pb & lo);
    V<R> a0 = a[ia], a1 = a[ia | (lo + 1)], b0 = a[ib], b1 = a[ib | (lo + 1)];
    a[ia] = cfma(m.m01, a1, cmul(m.m00, a0));
    a[ia | (lo + 1)] = cfma(m.m11, a1, cmul(m.m10, a0));
    a[ib] = cfma(m.m01, b1, cmul(m.m00, b0));
    a[ib | (lo + 1)] = cfma(m.m11, b1, cmul(m.m10, b0));
  }
  if (p < npairs) {
    uint64_t ia = ((p & ~lo) << 1) | (p & lo);
    V<R> a0 = a[ia], a1 = a[ia | (lo + 1)];
    a[ia] = cfma(m.m01, a1, cmul(m.m00, a0));
    a[ia | (lo + 1)] = cfma(m.m11, a1, cmul(m.m10, a0));
  }
}

// ---------------------------------------------------------------------------
// 2-qubit dense gate: the quad over (q0, q1) per thread
// ---------------------------------------------------------------------------
template <class R>
struct Mat2 {
  V<R> m[16];
  int qa, qb;       // gate qubits 0 and 1 (local bits 0 and 1)
  uint8_t pos[2];   // ascending positions
};

template <class R>
__global__ void __launch_bounds__(THREADS) k_dense2(V<R>* __restrict__ a, uint64_t nquads, Mat2<R> g) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t ba = uint64_t(1) << g.qa, bb = uint64_t(1) << g.qb;
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nquads; p += stride) {
    uint64_t i = insert_zeros(p, g.pos, 2);
    uint64_t idx[4] = {i, i | ba, i | bb, i | ba | bb};
    V<R> v[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) v[b] = a[idx[b]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      V<R> acc = cmul(g.m[4 * r], v[0]);
      acc = cfma(g.m[4 * r + 1], v[1], acc);
      acc = cfma(g.m[4 * r + 2], v[2], acc);
      acc = cfma(g.m[4 * r + 3], v[3], acc);
      a[idx[r]] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// Tiles: 2^T amplitudes whose indices agree off the tile bits, where the tile
// bits are the gate qubits plus the lowest w bits of the index (so runs of
// 2^w consecutive amplitudes are loaded and stored).  The generic dense and
// permutation kernels stage a tile in shared memory and write each output
// amplitude straight back to global memory (coalesced).
// ---------------------------------------------------------------------------
constexpr int MAX_TILE_K = 10;

struct TileGeom {
  int T;                    // tile bits
  int w;                    // low contiguous bits
  int k;                    // gate qubits
  int nh;                   // gate qubits >= w
  uint8_t hq[MAX_TILE_K];   // those qubits, ascending (global positions)
  uint8_t pos[MAX_TILE_K];  // tile-local position of gate qubit j (local order)
};

__device__ __forceinline__ uint64_t tile_offset(uint32_t e, const TileGeom& g) {
  uint64_t off = e & ((1u << g.w) - 1);
  for (int i = 0; i < g.nh; ++i) off |= uint64_t((e >> (g.w + i)) & 1u) << g.hq[i];
  return off;
}
__device__ __forceinline__ uint32_t tile_local_x(uint32_t e, const TileGeom& g) {
  uint32_t x = 0;
  for (int j = 0; j < g.k; ++j) x |= ((e >> g.pos[j]) & 1u) << j;
  return x;
}

TileGeom make_geom(uint32_t n, const std::vector<uint32_t>& qubits, int T) {
  TileGeom g{};
  g.k = int(qubits.size());
  uint64_t gmask = 0;
  for (uint32_t q : qubits) gmask |= uint64_t(1) << q;
  int w = 0;
  while (__builtin_popcountll(gmask | ((uint64_t(1) << w) - 1)) < T && w < int(n)) ++w;
  g.w = w;
  g.T = __builtin_popcountll(gmask | ((uint64_t(1) << w) - 1));
  std::vector<uint32_t> hs;
  for (uint32_t q : qubits)
    if (int(q) >= w) hs.push_back(q);
  std::sort(hs.begin(), hs.end());
  g.nh = int(hs.size());
  for (int i = 0; i < g.nh; ++i) g.hq[i] = uint8_t(hs[i]);
  for (int j = 0; j < g.k; ++j) {
    uint32_t q = qubits[j];
    if (int(q) < w) g.pos[j] = uint8_t(q);
    else g.pos[j] = uint8_t(w + (std::find(hs.begin(), hs.end(), q) - hs.begin()));
  }
  return g;
}

// base index of tile t: t deposited into the bits outside the tile
__device__ __forceinline__ uint64_t tile_base(uint64_t t, const TileGeom& g) {
  uint64_t v = t << g.w;
  for (int i = 0; i < g.nh; ++i) {
    int b = g.hq[i];
    v = ((v >> b) << (b + 1)) | (v & ((uint64_t(1) << b) - 1));
  }
  return v;
}

// Tile staging for the shared-memory tile kernels.  Element e of a tile is
// threadIdx.x + r*blockDim.x; its global offset and gate pattern are ORs of a
// per-thread part and a per-round part (the bit deposit sends each bit of e
// to its own position), computed once per block.  The loads are cp.async
// copies straight into shared memory, all of a thread's rounds in flight at
// once (no register staging).
struct TileRounds {
  uint64_t toff;   // offset of threadIdx.x
  uint32_t tx;     // gate pattern of threadIdx.x
  uint32_t nr;     // rounds
};

__device__ __forceinline__ TileRounds tile_rounds(const TileGeom& g, uint64_t* roff, uint32_t* rx) {
  const uint32_t tsz = 1u << g.T;
  const uint32_t nr = (tsz + blockDim.x - 1) / blockDim.x;
  if (threadIdx.x < nr) {
    roff[threadIdx.x] = tile_offset(threadIdx.x * blockDim.x, g);
    rx[threadIdx.x] = tile_local_x(threadIdx.x * blockDim.x, g);
  }
  return TileRounds{tile_offset(threadIdx.x, g), tile_local_x(threadIdx.x, g), nr};
}

template <class R>
__device__ __forceinline__ void tile_load_async(V<R>* tile, const V<R>* src, const uint64_t* roff, uint32_t nr, uint32_t tsz) {
  for (uint32_t r = 0; r < nr; ++r) {
    const uint32_t e = threadIdx.x + r * blockDim.x;
    if (e >= tsz) break;
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(tile + e));
    if constexpr (sizeof(V<R>) == 16)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + roff[r]) : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src + roff[r]) : "memory");
  }
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

constexpr int MAX_DENSE_K = 5;  // matrices up to 32x32 travel in the kernel parameters (k_dense_fiber)

// k = 3..5 dense gate, one fiber per thread: the fiber's 2^K amplitudes are
// loaded into registers (all loads before any arithmetic), each output row is
// a sum over the matrix row, and the matrix stays in the kernel parameters,
// read with warp-uniform, compile-time addresses (the constant cache
// broadcasts them).  In place: a thread owns its fiber.
template <class R, int K>
struct FiberParams {
  uint8_t pos[K];            // gate qubits, ascending (for the zero insertion)
  uint64_t off[1 << K];      // global offset bits of local pattern b (bit j = qubits[j])
  V<R> m[1 << (2 * K)];      // row-major
};

template <class R, int K>
__global__ void __launch_bounds__(THREADS) k_dense_fiber(V<R>* __restrict__ a, uint64_t nfib,
                                                         const __grid_constant__ FiberParams<R, K> P) {
  constexpr int D = 1 << K;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t f = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; f < nfib; f += stride) {
    const uint64_t base = insert_zeros(f, P.pos, K);
    V<R> v[D];
#pragma unroll
    for (int b = 0; b < D; ++b) v[b] = a[base | P.off[b]];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      V<R> acc = cmul(P.m[r * D], v[0]);
#pragma unroll
      for (int b = 1; b < D; ++b) acc = cfma(P.m[r * D + b], v[b], acc);
      a[base | P.off[r]] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// diagonal table: amplitude i *= diag[x(i)], enumerating only the indices
// whose fixed bits are set (every phased pattern has them set)
// ---------------------------------------------------------------------------
constexpr int MAX_DIAG_K = 10;

template <class R, int KMAX>
struct DiagParams {
  int k;
  uint8_t q[MAX_DIAG_K];        // gate qubits, local order
  int nfix;
  uint8_t fixpos[MAX_DIAG_K];   // ascending global positions of the fixed-one bits
  uint64_t fixmask;
  V<R> d[1 << KMAX];
  uint8_t unit[1 << KMAX];
};

// One phase for every enumerated amplitude: the gate's only phased pattern
// has all its gate bits fixed (S, T, Z, PHASE, CZ, CS, CPHASE, CCZ).  Two
// amplitudes in flight per thread.
template <class R>
struct DiagConstParams {
  int nfix;
  uint8_t fixpos[MAX_DIAG_K];
  uint64_t fixmask;
  V<R> c;
};

template <class R>
__global__ void __launch_bounds__(THREADS) k_diag_const(V<R>* __restrict__ a, uint64_t count, const __grid_constant__ DiagConstParams<R> P) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const V<R> c = P.c;
  uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; p + stride < count; p += 2 * stride) {
    const uint64_t i = insert_zeros(p, P.fixpos, P.nfix) | P.fixmask;
    const uint64_t j = insert_zeros(p + stride, P.fixpos, P.nfix) | P.fixmask;
    V<R> u = a[i], v = a[j];
    if (!is_zero(u)) a[i] = cmul(c, u);
    if (!is_zero(v)) a[j] = cmul(c, v);
  }
  if (p < count) {
    const uint64_t i = insert_zeros(p, P.fixpos, P.nfix) | P.fixmask;
    V<R> u = a[i];
    if (!is_zero(u)) a[i] = cmul(c, u);
  }
}

// Two phases selected by one index bit (RZ and any diagonal 1-qubit matrix).
template <class R>
__global__ void __launch_bounds__(THREADS) k_diag_1q(V<R>* __restrict__ a, uint64_t len, int q, V<R> c0, V<R> c1) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; i + stride < len; i += 2 * stride) {
    const uint64_t j = i + stride;
    V<R> u = a[i], v = a[j];
    if (!is_zero(u)) a[i] = cmul(((i >> q) & 1) ? c1 : c0, u);
    if (!is_zero(v)) a[j] = cmul(((j >> q) & 1) ? c1 : c0, v);
  }
  if (i < len) {
    V<R> u = a[i];
    if (!is_zero(u)) a[i] = cmul(((i >> q) & 1) ? c1 : c0, u);
  }
}

template <class R, int KMAX>
__global__ void __launch_bounds__(THREADS) k_diag(V<R>* __restrict__ a, uint64_t count, const __grid_constant__ DiagParams<R, KMAX> P) {
  __shared__ V<R> d[1 << KMAX];
  __shared__ uint8_t unit[1 << KMAX];
  for (int i = threadIdx.x; i < (1 << P.k); i += blockDim.x) d[i] = P.d[i], unit[i] = P.unit[i];
  __syncthreads();
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < count; p += stride) {
    uint64_t i = insert_zeros(p, P.fixpos, P.nfix) | P.fixmask;
    uint32_t x = 0;
    for (int j = 0; j < P.k; ++j) x |= uint32_t((i >> P.q[j]) & 1u) << j;
    if (unit[x]) continue;
    V<R> v = a[i];
    if (!is_zero(v)) a[i] = cmul(d[x], v);
  }
}

// ---------------------------------------------------------------------------
// pair swap: indices i with the fixed pattern exchange with i ^ D, with
// constant phases (X, Y, CX, CY, CCX, SWAP, any monomial of that shape)
// ---------------------------------------------------------------------------
template <class R>
struct SwapParams {
  int nfix;
  uint8_t fixpos[16];   // ascending global positions of every fixed bit
  uint64_t ones;        // fixed bits that are 1 at i
  uint64_t xmask;       // partner j = i ^ xmask
  V<R> c_i;             // new a[i] = c_i * old a[j]
  V<R> c_j;             // new a[j] = c_j * old a[i]
  int unit_i, unit_j;
};

template <class R>
__global__ void __launch_bounds__(THREADS) k_pairswap(V<R>* __restrict__ a, uint64_t count, SwapParams<R> P) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < count; p += stride) {
    uint64_t i = insert_zeros(p, P.fixpos, P.nfix) | P.ones;
    uint64_t j = i ^ P.xmask;
    V<R> vi = a[i], vj = a[j];
    a[i] = P.unit_i ? vj : cmul(P.c_i, vj);
    a[j] = P.unit_j ? vi : cmul(P.c_j, vi);
  }
}

// ---------------------------------------------------------------------------
// generic monomial: out(y) = phase[x] * in(x) for y = image(x), via tiles
// ---------------------------------------------------------------------------
template <class R>
struct PermParams {
  TileGeom g;
  uint16_t pre[1 << MAX_TILE_K];   // preimage x of each output pattern y
  V<R> ph[1 << MAX_TILE_K];        // phase of the preimage
  uint8_t unit[1 << MAX_TILE_K];
};

template <class R>
__global__ void __launch_bounds__(THREADS) k_perm_tile(V<R>* __restrict__ a, uint64_t ntiles, const __grid_constant__ PermParams<R> PP) {
  const PermParams<R>* P = &PP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const TileGeom& g = P->g;
  const int gd = 1 << g.k;
  const uint32_t tsz = 1u << g.T;
  V<R>* tile = reinterpret_cast<V<R>*>(smem_raw);
  V<R>* ph = tile + tsz;
  uint32_t* src = reinterpret_cast<uint32_t*>(ph + gd);  // tile pattern of the preimage
  uint8_t* unit = reinterpret_cast<uint8_t*>(src + gd);
  for (int y = threadIdx.x; y < gd; y += blockDim.x) {
    uint32_t x = P->pre[y];
    uint32_t o = 0;
    for (int j = 0; j < g.k; ++j) o |= ((x >> j) & 1u) << g.pos[j];
    src[y] = o;
    ph[y] = P->ph[y];
    unit[y] = P->unit[y];
  }
  __shared__ uint64_t roff[32];
  __shared__ uint32_t rx[32];
  const TileRounds tr = tile_rounds(g, roff, rx);
  uint32_t gtile = 0;
  for (int j = 0; j < g.k; ++j) gtile |= 1u << g.pos[j];
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    V<R>* amp = a + (tile_base(t, g) | tr.toff);
    __syncthreads();
    tile_load_async<R>(tile, amp, roff, tr.nr, tsz);
    __syncthreads();
#pragma unroll 4
    for (uint32_t q = 0; q < tr.nr; ++q) {
      const uint32_t e = threadIdx.x + q * blockDim.x;
      if (e >= tsz) break;
      const uint32_t y = tr.tx | rx[q];
      const V<R> v = tile[(e & ~gtile) | src[y]];
      amp[roff[q]] = unit[y] ? v : cmul(ph[y], v);
    }
  }
}
// ---------------------------------------------------------------------------
// Diagonal(PhasePoly) evaluated from the basis index
// ---------------------------------------------------------------------------
constexpr int MAX_POLY_TERMS = 512;
constexpr int MAX_POLY_PARITIES = 2048;

template <class R>
struct PolyParams {
  uint32_t bits;
  uint64_t modmask;
  uint64_t constant;
  int nterms;
  int use_table;
  int scalar_is_one;
  V<R> scalar;
  uint16_t start[MAX_POLY_TERMS + 1];
  uint32_t coeff[MAX_POLY_TERMS];
  uint64_t par[MAX_POLY_PARITIES];
  V<R> table[256];
};

__device__ __forceinline__ double2 device_root(uint64_t f, uint32_t bits) {
  // exp(2 pi i f / 2^bits) with exact quarter and eighth turns, as
  // root_of_unity does for complex doubles (scalar.rs:112-132)
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

template <class R>
__global__ void __launch_bounds__(THREADS) k_phasepoly(V<R>* __restrict__ a, uint64_t len, const __grid_constant__ PolyParams<R> PP) {
  const PolyParams<R>* P = &PP;
  __shared__ uint16_t start[MAX_POLY_TERMS + 1];
  __shared__ uint32_t coeff[MAX_POLY_TERMS];
  __shared__ uint64_t par[MAX_POLY_PARITIES];
  __shared__ V<R> table[256];
  const int nt = P->nterms;
  for (int i = threadIdx.x; i <= nt; i += blockDim.x) start[i] = P->start[i];
  for (int i = threadIdx.x; i < nt; i += blockDim.x) coeff[i] = P->coeff[i];
  const int npar = P->start[nt];
  for (int i = threadIdx.x; i < npar; i += blockDim.x) par[i] = P->par[i];
  if (P->use_table)
    for (int i = threadIdx.x; i < 256; i += blockDim.x) table[i] = P->table[i];
  __syncthreads();
  const uint64_t modmask = P->modmask, constant = P->constant;
  const uint32_t bits = P->bits;
  const bool use_table = P->use_table, s_one = P->scalar_is_one;
  const V<R> scalar = P->scalar;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    V<R> v = a[i];
    if (is_zero(v)) continue;
    uint64_t f = constant;
    for (int t = 0; t < nt; ++t) {
      int all = 1;
      for (int l = start[t]; l < start[t + 1]; ++l) all &= __popcll(par[l] & i) & 1;
      if (all) f += coeff[t];
    }
    f &= modmask;
    V<R> c;
    if (use_table) {
      c = table[f];
      if (is_one_v(c)) continue;
    } else {
      if (f == 0 && s_one) continue;
      double2 r = device_root(f, bits);
      c = to_v<R>(r);
      if (!s_one) c = cmul(scalar, c);
    }
    a[i] = cmul(c, v);
  }
}

// Bit-sliced form for exponents of at most 8 bits (a phasor table).  A warp
// owns 1024 consecutive indices; lane l holds the 32 indices chunk|j<<5|l,
// j = 0..31, and evaluates each parity for all of them at once as a 32-bit
// mask over j: parity(p & i) = parity(p_rest & (chunk|l)) ^ parity(p_j & j),
// the second factor a fixed mask per parity.  Terms are ANDs of those masks,
// and f = constant + sum coeff*term is accumulated mod 2^B in B bit planes
// (a ripple-carry add of the warp-uniform coefficient under the term mask).
// The per-amplitude work is then an extraction of B bits, a table lookup and
// the multiply; the term evaluation costs about 1/32 of the scalar form.
template <int B>
__device__ __forceinline__ void sliced_add(uint32_t (&F)[B], uint32_t m, uint32_t c) {
  uint32_t carry = 0;  // always a subset of m
#pragma unroll
  for (int k = 0; k < B; ++k) {
    const uint32_t f = F[k];
    if ((c >> k) & 1u) {
      F[k] = f ^ m ^ carry;
      carry = m & (f | carry);
    } else {
      F[k] = f ^ carry;
      carry = f & carry;
    }
  }
}

__host__ __device__ __forceinline__ uint32_t sliced_pattern(uint32_t m5) {
  // bit j of the result = parity(m5 & j), j = 0..31
  const uint32_t pat[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
  uint32_t r = 0;
  for (int b = 0; b < 5; ++b)
    if ((m5 >> b) & 1u) r ^= pat[b];
  return r;
}

template <class R, int B>
__global__ void __launch_bounds__(THREADS) k_phasepoly_sliced(V<R>* __restrict__ a, uint64_t len, const __grid_constant__ PolyParams<R> PP) {
  const PolyParams<R>* P = &PP;
  __shared__ uint64_t prest[MAX_POLY_PARITIES];  // parity mask outside index bits 5..9
  __shared__ uint32_t pj[MAX_POLY_PARITIES];     // its values over j
  __shared__ uint16_t start[MAX_POLY_TERMS + 1];
  __shared__ uint32_t coeff[MAX_POLY_TERMS];
  __shared__ V<R> table[1 << B];
  const int nt = P->nterms;
  for (int i = threadIdx.x; i <= nt; i += blockDim.x) start[i] = P->start[i];
  for (int i = threadIdx.x; i < nt; i += blockDim.x) coeff[i] = P->coeff[i];
  const int npar = P->start[nt];
  for (int i = threadIdx.x; i < npar; i += blockDim.x) {
    const uint64_t p = P->par[i];
    prest[i] = p & ~uint64_t(0x3E0);
    pj[i] = sliced_pattern(uint32_t(p >> 5) & 31u);
  }
  for (int i = threadIdx.x; i < (1 << B); i += blockDim.x) table[i] = P->table[i];
  __syncthreads();
  const uint64_t constant = P->constant;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nchunks = len >> 10;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t ch = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; ch < nchunks; ch += nwarps) {
    const uint64_t idx = (ch << 10) | lane;
    uint32_t F[B];
#pragma unroll
    for (int k = 0; k < B; ++k) F[k] = 0u - uint32_t((constant >> k) & 1);
    for (int t = 0; t < nt; ++t) {
      uint32_t m = ~0u;
      const int l1 = start[t + 1];
      for (int l = start[t]; l < l1; ++l) m &= pj[l] ^ (0u - (uint32_t(__popcll(prest[l] & idx)) & 1u));
      sliced_add<B>(F, m, coeff[t]);
    }
    V<R>* p = a + idx;
#pragma unroll
    for (int jb = 0; jb < 32; jb += 8) {
      V<R> v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = p[(jb + u) << 5];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = jb + u;
        uint32_t f = 0;
#pragma unroll
        for (int k = 0; k < B; ++k) f |= ((F[k] >> j) & 1u) << k;
        if (is_zero(v[u])) continue;
        const V<R> c = table[f];
        if (is_one_v(c)) continue;
        p[j << 5] = cmul(c, v[u]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Pauli i^ph X^x Z^z (vector.rs:143-164)
// ---------------------------------------------------------------------------
// Four grid-stride steps per iteration, their loads issued together: the
// amplitudes whose phase is 1 are neither read nor written, so a thread has
// about half as many loads in flight as indices it visits.
template <class R>
__global__ void __launch_bounds__(THREADS) k_pauli_diag(V<R>* __restrict__ a, uint64_t len, uint64_t z, int ph) {
  constexpr int U = 4;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t c0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; c0 < len; c0 += U * stride) {
    V<R> v[U];
    int k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t c = c0 + u * stride;
      k[u] = c < len ? (ph + 2 * __popcll(z & c)) & 3 : 0;
      if (k[u]) v[u] = a[c];
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (k[u] && !is_zero(v[u])) a[c0 + u * stride] = ipow_mul(k[u], v[u]);
  }
}

template <class R>
__global__ void __launch_bounds__(THREADS) k_pauli_pair(V<R>* __restrict__ a, uint64_t npairs, int h, uint64_t x, uint64_t z, int ph) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t lo = (uint64_t(1) << h) - 1;
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < npairs; p += stride) {
    uint64_t c = ((p & ~lo) << 1) | (p & lo);
    uint64_t d = c ^ x;
    V<R> vc = a[c], vd = a[d];
    // (P psi)(c) = i^{k(c ^ x)} psi(c ^ x)
    a[c] = ipow_mul((ph + 2 * __popcll(z & d)) & 3, vd);
    a[d] = ipow_mul((ph + 2 * __popcll(z & c)) & 3, vc);
  }
}

// ---------------------------------------------------------------------------
// elementwise
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(THREADS) k_scale(V<R>* __restrict__ a, uint64_t len, double2 c) {
  const V<R> cc = to_v<R>(c);
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    V<R> v = a[i];
    if (!is_zero(v)) a[i] = cmul(v, cc);
  }
}

template <class R>
__global__ void __launch_bounds__(THREADS) k_fill(V<R>* __restrict__ a, uint64_t len, double re) {
  V<R> v;
  v.x = R(re);
  v.y = R(0);
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) a[i] = v;
}

__global__ void k_set_one_f(float2* a, uint64_t i) { a[i] = make_float2(1.f, 0.f); }
__global__ void k_set_one_d(double2* a, uint64_t i) { a[i] = make_double2(1.0, 0.0); }

__global__ void k_convert_in(float2* __restrict__ dst, const double2* __restrict__ src, uint64_t count) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
    dst[i] = make_float2(float(src[i].x), float(src[i].y));
}
__global__ void k_convert_out(double2* __restrict__ dst, const float2* __restrict__ src, uint64_t count) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
    dst[i] = make_double2(double(src[i].x), double(src[i].y));
}

template <class R>
__global__ void k_gather(const V<R>* __restrict__ a, const uint64_t* __restrict__ idx, double2* __restrict__ out,
                         uint64_t count, uint64_t len) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    uint64_t j = idx[i] & (len - 1);
    V<R> v = a[j];
    out[i] = make_double2(double(v.x), double(v.y));
  }
}

template <class R>
__global__ void __launch_bounds__(THREADS) k_kron(V<R>* __restrict__ out, const V<R>* __restrict__ a, const V<R>* __restrict__ b,
                                                  int na, uint64_t len) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t amask = (uint64_t(1) << na) - 1;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    V<R> x = a[i & amask], y = b[i >> na];
    V<R> r;
    r.x = 0;
    r.y = 0;
    if (!is_zero(x) && !is_zero(y)) r = cmul(x, y);
    out[i] = r;
  }
}

// ---------------------------------------------------------------------------
// FP64 reductions: per-thread sums, warp shuffles, one partial per block
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int SLOTS>
__device__ __forceinline__ void block_store(double (&acc)[SLOTS], double* partials) {
  __shared__ double red[SLOTS][REDUCE_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    double v = warp_sum(acc[s]);
    if (lane == 0) red[s][wid] = v;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      double v = lane < int(blockDim.x >> 5) ? red[s][lane] : 0.0;
      v = warp_sum(v);
      if (lane == 0) partials[blockIdx.x * PARTIAL_SLOTS + s] = v;
    }
  }
}

// The reductions keep several independent loads in flight per thread (UNROLL
// grid-stride steps per iteration, all loads before any arithmetic), so that
// the 2 x 512 threads of an SM hold enough bytes in flight to stream HBM.
constexpr int UNROLL = 4;

template <class R>
__device__ __forceinline__ V<R> load_or_zero(const V<R>* a, uint64_t i, uint64_t len) {
  V<R> v;
  v.x = v.y = R(0);
  if (i < len) v = a[i];
  return v;
}

template <class R>
__global__ void __launch_bounds__(REDUCE_THREADS) k_norm(const V<R>* __restrict__ a, uint64_t len, double* partials) {
  double acc[1] = {0.0};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i0 < len; i0 += UNROLL * stride) {
    V<R> v[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) v[u] = load_or_zero<R>(a, i0 + u * stride, len);
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) acc[0] += double(v[u].x) * double(v[u].x) + double(v[u].y) * double(v[u].y);
  }
  block_store<1>(acc, partials);
}

// <psi|P|psi> (and optionally <psi|psi>): slots re, im[, norm]
template <class R, bool NORM>
__global__ void __launch_bounds__(REDUCE_THREADS) k_expect_diag(const V<R>* __restrict__ a, uint64_t len, uint64_t z, int ph,
                                                                double* partials) {
  // sum_c i^{k(c)} |psi(c)|^2
  double acc[3] = {0.0, 0.0, 0.0};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t c0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; c0 < len; c0 += UNROLL * stride) {
    V<R> v[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) v[u] = load_or_zero<R>(a, c0 + u * stride, len);
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const uint64_t c = c0 + u * stride;
      const double w = double(v[u].x) * double(v[u].x) + double(v[u].y) * double(v[u].y);
      const int k = (ph + 2 * __popcll(z & c)) & 3;
      const double sw = (k & 2) ? -w : w;
      if (k & 1) acc[1] += sw;
      else acc[0] += sw;
      if (NORM) acc[2] += w;
    }
  }
  block_store<3>(acc, partials);
}

template <class R, bool NORM>
__global__ void __launch_bounds__(REDUCE_THREADS) k_expect_pair(const V<R>* __restrict__ a, uint64_t npairs, int h, uint64_t x,
                                                                uint64_t z, int ph, double* partials) {
  double acc[3] = {0.0, 0.0, 0.0};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t lo = (uint64_t(1) << h) - 1;
  for (uint64_t p0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p0 < npairs; p0 += UNROLL * stride) {
    V<R> vc[UNROLL], vd[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const uint64_t p = p0 + u * stride;
      const uint64_t c = ((p & ~lo) << 1) | (p & lo);
      vc[u].x = vc[u].y = vd[u].x = vd[u].y = R(0);  // past the end: zeros add nothing
      if (p < npairs) {
        vc[u] = a[c];
        vd[u] = a[c ^ x];
      }
    }
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const uint64_t p = p0 + u * stride;
      const uint64_t c = ((p & ~lo) << 1) | (p & lo);
      const uint64_t d = c ^ x;
      double2 C = make_double2(vc[u].x, vc[u].y), D = make_double2(vd[u].x, vd[u].y);
      // conj(psi(d)) i^{k(c)} psi(c) + conj(psi(c)) i^{k(d)} psi(d)
      double2 t1 = ipow_mul((ph + 2 * __popcll(z & c)) & 3, C);
      double2 t2 = ipow_mul((ph + 2 * __popcll(z & d)) & 3, D);
      acc[0] += D.x * t1.x + D.y * t1.y + C.x * t2.x + C.y * t2.y;
      acc[1] += D.x * t1.y - D.y * t1.x + C.x * t2.y - C.y * t2.x;
      if (NORM) acc[2] += C.x * C.x + C.y * C.y + D.x * D.x + D.y * D.y;
    }
  }
  block_store<3>(acc, partials);
}

template <class R>
__global__ void __launch_bounds__(REDUCE_THREADS) k_inner(const V<R>* __restrict__ a, const V<R>* __restrict__ b, uint64_t len,
                                                          double* partials) {
  double acc[2] = {0.0, 0.0};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i0 < len; i0 += UNROLL * stride) {
    V<R> u[UNROLL], v[UNROLL];
#pragma unroll
    for (int k = 0; k < UNROLL; ++k) {
      u[k] = load_or_zero<R>(a, i0 + k * stride, len);
      v[k] = load_or_zero<R>(b, i0 + k * stride, len);
    }
#pragma unroll
    for (int k = 0; k < UNROLL; ++k) {
      acc[0] += double(u[k].x) * double(v[k].x) + double(u[k].y) * double(v[k].y);
      acc[1] += double(u[k].x) * double(v[k].y) - double(u[k].y) * double(v[k].x);
    }
  }
  block_store<2>(acc, partials);
}

// <a|b>, <a|a>, <b|b> and max |a_i - b_i| over registers of any precisions
template <class RA, class RB>
__global__ void __launch_bounds__(REDUCE_THREADS) k_compare(const V<RA>* __restrict__ a, const V<RB>* __restrict__ b, uint64_t len,
                                                            double* partials, double* maxdiff) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double mx = 0.0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    V<RA> u = a[i];
    V<RB> v = b[i];
    const double ux = u.x, uy = u.y, vx = v.x, vy = v.y;
    acc[0] += ux * vx + uy * vy;
    acc[1] += ux * vy - uy * vx;
    acc[2] += ux * ux + uy * uy;
    acc[3] += vx * vx + vy * vy;
    mx = fmax(mx, hypot(ux - vx, uy - vy));
  }
  block_store<4>(acc, partials);
  __shared__ double red[REDUCE_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    maxdiff[blockIdx.x] = m;
  }
}

// projection (1 + s P)/2 fused with the norm of the result
template <class R>
__global__ void __launch_bounds__(REDUCE_THREADS) k_project_diag(V<R>* __restrict__ a, uint64_t len, uint64_t z, int ph, int outcome,
                                                                 double* partials) {
  double acc[1] = {0.0};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t c0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; c0 < len; c0 += UNROLL * stride) {
    V<R> v[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) v[u] = load_or_zero<R>(a, c0 + u * stride, len);
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const uint64_t c = c0 + u * stride;
      if (is_zero(v[u])) continue;  // (also every index past the end)
      const int k = (ph + 2 * __popcll(z & c) + (outcome ? 2 : 0)) & 3;
      V<R> nv = ipow_mul(k, v[u]);
      nv.x = (v[u].x + nv.x) * R(0.5);
      nv.y = (v[u].y + nv.y) * R(0.5);
      if (nv.x != v[u].x || nv.y != v[u].y) a[c] = nv;
      acc[0] += double(nv.x) * double(nv.x) + double(nv.y) * double(nv.y);
    }
  }
  block_store<1>(acc, partials);
}

template <class R>
__global__ void __launch_bounds__(REDUCE_THREADS) k_project_pair(V<R>* __restrict__ a, uint64_t npairs, int h, uint64_t x, uint64_t z,
                                                                 int ph, int outcome, double* partials) {
  double acc[1] = {0.0};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t lo = (uint64_t(1) << h) - 1;
  const int so = outcome ? 2 : 0;
  for (uint64_t p0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p0 < npairs; p0 += UNROLL * stride) {
    V<R> vc[UNROLL], vd[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const uint64_t p = p0 + u * stride;
      const uint64_t c = ((p & ~lo) << 1) | (p & lo);
      vc[u].x = vc[u].y = vd[u].x = vd[u].y = R(0);
      if (p < npairs) {
        vc[u] = a[c];
        vd[u] = a[c ^ x];
      }
    }
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const uint64_t p = p0 + u * stride;
      if (p >= npairs) break;
      const uint64_t c = ((p & ~lo) << 1) | (p & lo);
      const uint64_t d = c ^ x;
      V<R> tc = ipow_mul((ph + 2 * __popcll(z & d) + so) & 3, vd[u]);
      V<R> td = ipow_mul((ph + 2 * __popcll(z & c) + so) & 3, vc[u]);
      V<R> nc, nd;
      nc.x = (vc[u].x + tc.x) * R(0.5);
      nc.y = (vc[u].y + tc.y) * R(0.5);
      nd.x = (vd[u].x + td.x) * R(0.5);
      nd.y = (vd[u].y + td.y) * R(0.5);
      a[c] = nc;
      a[d] = nd;
      acc[0] += double(nc.x) * double(nc.x) + double(nc.y) * double(nc.y) + double(nd.x) * double(nd.x) +
                double(nd.y) * double(nd.y);
    }
  }
  block_store<1>(acc, partials);
}

// ---------------------------------------------------------------------------
// sampling: block weights, then one warp per shot walks its block
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(THREADS) k_block_weights(const V<R>* __restrict__ a, uint64_t nblocks, uint64_t block, double* w) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; b < nblocks; b += warps) {
    double s = 0.0;
    const V<R>* p = a + b * block;
    for (uint64_t i = lane; i < block; i += 32) {
      V<R> v = p[i];
      s += double(v.x) * double(v.x) + double(v.y) * double(v.y);
    }
    s = warp_sum(s);
    if (lane == 0) w[b] = s;
  }
}

template <class R>
__global__ void __launch_bounds__(THREADS) k_sample_walk(const V<R>* __restrict__ a, const double* __restrict__ u, const uint64_t* __restrict__ blk,
                                                         const double* __restrict__ acc0, uint64_t shots, uint64_t block, uint64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
  for (uint64_t k = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; k < shots; k += warps) {
    const uint64_t start = blk[k] * block, end = start + block;
    const double target = u[k];
    double run = acc0[k];
    uint64_t pick = end - 1;
    // first idx in [start, end-1) with run + sum_{start..idx} w > target
    for (uint64_t c = start; c < end - 1; c += 32) {
      uint64_t i = c + lane;
      double w = 0.0;
      if (i < end - 1) {
        V<R> v = a[i];
        w = double(v.x) * double(v.x) + double(v.y) * double(v.y);
      }
      double incl = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        double t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      unsigned hit = __ballot_sync(0xffffffffu, i < end - 1 && run + incl > target);
      if (hit) {
        pick = c + __ffs(hit) - 1;
        break;
      }
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
      // never an index of zero weight (vector.rs:528-532)
      while (pick > start && is_zero(a[pick])) --pick;
      out[k] = pick;
    }
  }
}

#define NCSIM_DISPATCH(s, ...)                          \
  do {                                                  \
    if ((s)->precision == NCSIM_C128) {                 \
      using R = double;                                 \
      __VA_ARGS__;                                      \
    } else {                                            \
      using R = float;                                  \
      __VA_ARGS__;                                      \
    }                                                   \
  } while (0)

template <class R>
V<R>* amp_of(const ncsim_state* s) {
  return reinterpret_cast<V<R>*>(s->amp);
}

template <class R>
V<R> cv(const CplxD& c) {
  V<R> r;
  r.x = R(c.re);
  r.y = R(c.im);
  return r;
}

// algorithmic bytes: read + write of every amplitude in a touched 32-byte sector
double full_bytes(const ncsim_state* s) { return 2.0 * double(s->len) * double(s->elem_bytes()); }
int sector_bits(const ncsim_state* s) { return s->precision == NCSIM_C128 ? 1 : 2; }
// amplitudes selected by fixing the bits of `fixed` (sector-granular)
double touched_bytes(const ncsim_state* s, uint64_t fixed, double members = 1.0) {
  const uint64_t below = fixed & ((uint64_t(1) << sector_bits(s)) - 1);
  const int f = __builtin_popcountll(fixed & ~below);
  double amps = double(s->len >> f) * members;
  return std::min(2.0 * amps * double(s->elem_bytes()), full_bytes(s));
}

bool is_one(const CplxD& c) { return c.re == 1.0 && c.im == 0.0; }
bool is_zero_c(const CplxD& c) { return c.re == 0.0 && c.im == 0.0; }

// The generic monomial path: tiles of 2^T amplitudes.
template <class R>
int tile_bits_for(uint32_t n, int k) {
  const int cap = sizeof(R) == 8 ? 12 : 13;  // 64 KB of shared memory per tile
  int T = std::max(k + 4, 10);
  T = std::min(T, cap);
  T = std::max(T, k);
  return std::min<int>(T, int(n));
}

}  // namespace

// ===========================================================================
// launchers
// ===========================================================================
void launch_dense(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& m) {
  const int k = int(qubits.size());
  const uint64_t len = s->len;
  // diagonal matrices go to the diagonal kernel (touches only changed amplitudes)
  const int gd = 1 << k;
  bool diag = true;
  for (int r = 0; r < gd && diag; ++r)
    for (int c = 0; c < gd; ++c)
      if (r != c && !is_zero_c(m[size_t(r) * gd + c])) {
        diag = false;
        break;
      }
  if (diag && k <= MAX_DIAG_K) {
    std::vector<CplxD> d(gd);
    for (int x = 0; x < gd; ++x) d[x] = m[size_t(x) * gd + x];
    launch_diag_table(s, qubits, d);
    return;
  }
  if (k == 1) {
    NCSIM_DISPATCH(s, {
      Mat1<R> mm{cv<R>(m[0]), cv<R>(m[1]), cv<R>(m[2]), cv<R>(m[3])};
      uint64_t npairs = len >> 1;
      ProfScope ps(s, K_DENSE1, full_bytes(s));
      k_dense1<R><<<grid_for(npairs, THREADS, 2), THREADS, 0, s->stream>>>(amp_of<R>(s), npairs, int(qubits[0]), mm);
    });
    NCSIM_LAUNCHED("dense1");
    return;
  }
  if (k == 2) {
    NCSIM_DISPATCH(s, {
      Mat2<R> g;
      for (int i = 0; i < 16; ++i) g.m[i] = cv<R>(m[i]);
      g.qa = int(qubits[0]);
      g.qb = int(qubits[1]);
      g.pos[0] = uint8_t(std::min(qubits[0], qubits[1]));
      g.pos[1] = uint8_t(std::max(qubits[0], qubits[1]));
      uint64_t nq = len >> 2;
      ProfScope ps(s, K_DENSE2, full_bytes(s));
      k_dense2<R><<<grid_for(nq, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), nq, g);
    });
    NCSIM_LAUNCHED("dense2");
    return;
  }
  if (k > MAX_DENSE_K) {
    launch_dense_wide(s, qubits, m);
    return;
  }
  auto fiber = [&](auto tagR, auto tagK) {
    using R = decltype(tagR);
    constexpr int K = decltype(tagK)::value;
    FiberParams<R, K> P{};
    std::vector<uint32_t> sq(qubits.begin(), qubits.end());
    std::sort(sq.begin(), sq.end());
    for (int j = 0; j < K; ++j) P.pos[j] = uint8_t(sq[j]);
    for (int b = 0; b < (1 << K); ++b) {
      uint64_t o = 0;
      for (int j = 0; j < K; ++j)
        if ((b >> j) & 1) o |= uint64_t(1) << qubits[j];
      P.off[b] = o;
    }
    for (int i = 0; i < (1 << (2 * K)); ++i) P.m[i] = cv<R>(m[i]);
    const uint64_t nfib = len >> K;
    ProfScope ps(s, K_DENSE_FIBER, full_bytes(s));
    k_dense_fiber<R, K><<<grid_for(nfib, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), nfib, P);
  };
  using K3 = std::integral_constant<int, 3>;
  using K4 = std::integral_constant<int, 4>;
  using K5 = std::integral_constant<int, 5>;
  if (s->precision == NCSIM_C128) {
    if (k == 3) fiber(double(), K3());
    else if (k == 4) fiber(double(), K4());
    else fiber(double(), K5());
  } else {
    if (k == 3) fiber(float(), K3());
    else if (k == 4) fiber(float(), K4());
    else fiber(float(), K5());
  }
  NCSIM_LAUNCHED("dense_fiber");
}

void launch_diag_table(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& diag) {
  const int k = int(qubits.size());
  if (k > MAX_DIAG_K) throw Error(NCSIM_ERR_UNSUPPORTED, "diagonal table on more than 10 qubits");
  const int gd = 1 << k;
  // fixed bits: set in every pattern whose phase is not 1
  uint32_t fixed = (1u << k) - 1;
  bool any = false;
  for (int x = 0; x < gd; ++x)
    if (!is_one(diag[x])) fixed &= uint32_t(x), any = true;
  if (!any) return;  // identity: no amplitude changes
  int nphased = 0;
  for (int x = 0; x < gd; ++x) nphased += !is_one(diag[x]);
  if (nphased == 1 && fixed == uint32_t(gd - 1)) {
    // one phased pattern with every gate bit fixed: a constant phase on it
    NCSIM_DISPATCH(s, {
      DiagConstParams<R> P{};
      std::vector<int> fp(qubits.begin(), qubits.end());
      std::sort(fp.begin(), fp.end());
      P.nfix = k;
      uint64_t fm = 0;
      for (int i = 0; i < k; ++i) P.fixpos[i] = uint8_t(fp[i]), fm |= uint64_t(1) << fp[i];
      P.fixmask = fm;
      P.c = cv<R>(diag[gd - 1]);
      uint64_t count = s->len >> k;
      ProfScope ps(s, K_DIAG, touched_bytes(s, fm));
      k_diag_const<R><<<grid_for(count, THREADS, 2), THREADS, 0, s->stream>>>(amp_of<R>(s), count, P);
    });
    NCSIM_LAUNCHED("diag_const");
    return;
  }
  if (k == 1) {  // both patterns phased
    NCSIM_DISPATCH(s, {
      ProfScope ps(s, K_DIAG, full_bytes(s));
      k_diag_1q<R><<<grid_for(s->len, THREADS, 2), THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, int(qubits[0]),
                                                                             cv<R>(diag[0]), cv<R>(diag[1]));
    });
    NCSIM_LAUNCHED("diag_1q");
    return;
  }
  auto body = [&](auto tagR, auto tagK) {
    using R = decltype(tagR);
    constexpr int KM = decltype(tagK)::value;
    DiagParams<R, KM> P{};
    P.k = k;
    for (int j = 0; j < k; ++j) P.q[j] = uint8_t(qubits[j]);
    std::vector<int> fp;
    uint64_t fm = 0;
    for (int j = 0; j < k; ++j)
      if ((fixed >> j) & 1) fp.push_back(int(qubits[j])), fm |= uint64_t(1) << qubits[j];
    std::sort(fp.begin(), fp.end());
    P.nfix = int(fp.size());
    for (int i = 0; i < P.nfix; ++i) P.fixpos[i] = uint8_t(fp[i]);
    P.fixmask = fm;
    for (int x = 0; x < gd; ++x) {
      P.d[x] = cv<R>(diag[x]);
      P.unit[x] = is_one(diag[x]) ? 1 : 0;
    }
    uint64_t count = s->len >> P.nfix;
    ProfScope ps(s, K_DIAG, touched_bytes(s, fm));
    k_diag<R, KM><<<grid_for(count, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), count, P);
  };
  using K3 = std::integral_constant<int, 3>;
  using K10 = std::integral_constant<int, MAX_DIAG_K>;
  if (s->precision == NCSIM_C128) {
    if (k <= 3) body(double(), K3()); else body(double(), K10());
  } else {
    if (k <= 3) body(float(), K3()); else body(float(), K10());
  }
  NCSIM_LAUNCHED("diag");
}

void launch_perm_table(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& image,
                       const std::vector<CplxD>& phase) {
  const int k = int(qubits.size());
  const int gd = 1 << k;
  bool diagonal = true;
  for (int x = 0; x < gd; ++x) diagonal &= image[x] == uint32_t(x);
  if (diagonal && k <= MAX_DIAG_K) {
    launch_diag_table(s, qubits, phase);
    return;
  }
  if (k > MAX_TILE_K) {
    launch_perm_wide(s, qubits, image, phase);
    return;
  }
  // pair-swap shape: moved patterns pair up under one xor d on a sub-cube,
  // constant phases, unmoved patterns unphased
  {
    uint32_t d = 0;
    bool ok = true;
    std::vector<uint32_t> moved;
    for (int x = 0; x < gd; ++x)
      if (image[x] != uint32_t(x)) {
        moved.push_back(uint32_t(x));
        uint32_t dx = image[x] ^ uint32_t(x);
        if (d == 0) d = dx;
        ok &= dx == d && image[image[x]] == uint32_t(x);
      } else {
        ok &= is_one(phase[x]);
      }
    if (ok && d) {
      const uint32_t hbit = 1u << (31 - __builtin_clz(d));
      std::vector<uint32_t> leads;
      for (uint32_t x : moved)
        if (!(x & hbit)) leads.push_back(x);
      uint32_t ones = (1u << k) - 1, zeros = (1u << k) - 1;
      for (uint32_t x : leads) ones &= x, zeros &= ~x;
      int nfixed = __builtin_popcount(ones) + __builtin_popcount(zeros);
      ok &= leads.size() == (size_t(1) << (k - nfixed)) && (zeros & hbit);
      CplxD c_j = phase[leads[0]], c_i = phase[leads[0] ^ d];
      for (uint32_t x : leads) ok &= phase[x].re == c_j.re && phase[x].im == c_j.im &&
                                     phase[x ^ d].re == c_i.re && phase[x ^ d].im == c_i.im;
      if (ok) {
        NCSIM_DISPATCH(s, {
          SwapParams<R> P{};
          std::vector<int> fp;
          uint64_t gones = 0, gx = 0;
          for (int j = 0; j < k; ++j) {
            if (((ones | zeros) >> j) & 1) fp.push_back(int(qubits[j]));
            if ((ones >> j) & 1) gones |= uint64_t(1) << qubits[j];
            if ((d >> j) & 1) gx |= uint64_t(1) << qubits[j];
          }
          std::sort(fp.begin(), fp.end());
          P.nfix = int(fp.size());
          for (int i = 0; i < P.nfix; ++i) P.fixpos[i] = uint8_t(fp[i]);
          P.ones = gones;
          P.xmask = gx;
          P.c_i = cv<R>(c_i);
          P.c_j = cv<R>(c_j);
          P.unit_i = is_one(c_i);
          P.unit_j = is_one(c_j);
          uint64_t count = s->len >> P.nfix;
          uint64_t ctrl = 0;
          for (int j = 0; j < k; ++j)
            if ((((ones | zeros) & ~d) >> j) & 1) ctrl |= uint64_t(1) << qubits[j];
          ProfScope ps(s, K_PAIRSWAP, touched_bytes(s, ctrl, 2.0 / double(uint64_t(1) << __builtin_popcount(d))));
          k_pairswap<R><<<grid_for(count, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), count, P);
        });
        NCSIM_LAUNCHED("pairswap");
        return;
      }
    }
  }
  NCSIM_DISPATCH(s, {
    auto* P = new PermParams<R>();
    P->g = make_geom(s->n, qubits, tile_bits_for<R>(s->n, k));
    for (int x = 0; x < gd; ++x) {
      uint32_t y = image[x];
      P->pre[y] = uint16_t(x);
      P->ph[y] = cv<R>(phase[x]);
      P->unit[y] = is_one(phase[x]);
    }
    uint64_t ntiles = s->len >> P->g.T;
    size_t smem = (size_t(1) << P->g.T) * sizeof(V<R>) + gd * (sizeof(V<R>) + sizeof(uint32_t) + 1);
    cudaFuncSetAttribute(k_perm_tile<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    ProfScope ps(s, K_PERM_TILE, full_bytes(s));
    k_perm_tile<R><<<grid_for(ntiles, 1, 1, 8), THREADS, smem, s->stream>>>(amp_of<R>(s), ntiles, *P);
    delete P;
    NCSIM_LAUNCHED("perm_tile");
  });
}

template <class R>
void launch_phasepoly_sliced(uint32_t bits, unsigned grid, cudaStream_t st, V<R>* a, uint64_t len, const PolyParams<R>& P) {
  switch (bits) {
    case 1: k_phasepoly_sliced<R, 1><<<grid, THREADS, 0, st>>>(a, len, P); break;
    case 2: k_phasepoly_sliced<R, 2><<<grid, THREADS, 0, st>>>(a, len, P); break;
    case 3: k_phasepoly_sliced<R, 3><<<grid, THREADS, 0, st>>>(a, len, P); break;
    case 4: k_phasepoly_sliced<R, 4><<<grid, THREADS, 0, st>>>(a, len, P); break;
    case 5: k_phasepoly_sliced<R, 5><<<grid, THREADS, 0, st>>>(a, len, P); break;
    case 6: k_phasepoly_sliced<R, 6><<<grid, THREADS, 0, st>>>(a, len, P); break;
    case 7: k_phasepoly_sliced<R, 7><<<grid, THREADS, 0, st>>>(a, len, P); break;
    default: k_phasepoly_sliced<R, 8><<<grid, THREADS, 0, st>>>(a, len, P); break;
  }
}

void launch_phasepoly(ncsim_state* s, const PolyTerms& t) {
  const int nt = int(t.coeffs.size());
  if (nt > MAX_POLY_TERMS || t.parities.size() > size_t(MAX_POLY_PARITIES))
    throw Error(NCSIM_ERR_UNSUPPORTED, "phase polynomial with more than 512 terms or 2048 parities");
  if (nt == 0 && t.scalar_is_one && (t.constant & ((t.bits >= 64 ? 0 : (uint64_t(1) << t.bits)) - 1)) == 0) return;
  NCSIM_DISPATCH(s, {
    auto* P = new PolyParams<R>();
    P->bits = t.bits;
    P->modmask = (uint64_t(1) << t.bits) - 1;
    P->constant = t.constant;
    P->nterms = nt;
    for (int i = 0; i <= nt; ++i) P->start[i] = uint16_t(t.term_start[i]);
    for (int i = 0; i < nt; ++i) P->coeff[i] = uint32_t(t.coeffs[i]);
    for (size_t i = 0; i < t.parities.size(); ++i) P->par[i] = t.parities[i];
    P->scalar_is_one = t.scalar_is_one;
    P->scalar = cv<R>(t.scalar);
    P->use_table = !t.root_table.empty();
    for (size_t i = 0; i < t.root_table.size() && i < 256; ++i) P->table[i] = cv<R>(t.root_table[i]);
    ProfScope ps(s, K_PHASEPOLY, full_bytes(s));
    const bool sliced = P->use_table && t.bits >= 1 && t.bits <= 8 && s->len >= 1024;
    if (sliced) {
      const unsigned grid = grid_for(s->len >> 5, THREADS);
      launch_phasepoly_sliced<R>(t.bits, grid, s->stream, amp_of<R>(s), s->len, *P);
    } else {
      k_phasepoly<R><<<grid_for(s->len, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, *P);
    }
    delete P;
    NCSIM_LAUNCHED("phasepoly");
  });
}

void launch_pauli(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase) {
  NCSIM_DISPATCH(s, {
    if (x == 0) {
      if (z == 0 && (phase & 3) == 0) return;
      ProfScope ps(s, K_PAULI, (phase & 3) ? full_bytes(s) : 0.5 * full_bytes(s));
      k_pauli_diag<R><<<grid_for(s->len, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, z, int(phase & 3));
    } else {
      int h = 63 - __builtin_clzll(x);
      uint64_t np = s->len >> 1;
      ProfScope ps(s, K_PAULI, full_bytes(s));
      k_pauli_pair<R><<<grid_for(np, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), np, h, x, z, int(phase & 3));
    }
  });
  NCSIM_LAUNCHED("pauli");
}

void launch_scale(ncsim_state* s, CplxD c) {
  ProfScope ps(s, K_SCALE, full_bytes(s));
  NCSIM_DISPATCH(s, {
    k_scale<R><<<grid_for(s->len, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, make_double2(c.re, c.im));
  });
  NCSIM_LAUNCHED("scale");
}

void launch_fill_plus(ncsim_state* s, double v) {
  NCSIM_DISPATCH(s, { k_fill<R><<<grid_for(s->len, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, v); });
  NCSIM_LAUNCHED("fill");
}

void launch_set_basis(ncsim_state* s, uint64_t index) {
  NCSIM_CUDA(cudaMemsetAsync(s->amp, 0, s->bytes(), s->stream));
  if (s->precision == NCSIM_C128) k_set_one_d<<<1, 1, 0, s->stream>>>(reinterpret_cast<double2*>(s->amp), index);
  else k_set_one_f<<<1, 1, 0, s->stream>>>(reinterpret_cast<float2*>(s->amp), index);
  NCSIM_LAUNCHED("set_basis");
}

void launch_convert_in(ncsim_state* s, const double2* src, uint64_t offset, uint64_t count) {
  k_convert_in<<<grid_for(count, THREADS), THREADS, 0, s->stream>>>(reinterpret_cast<float2*>(s->amp) + offset, src, count);
  NCSIM_LAUNCHED("convert_in");
}
void launch_convert_out(const ncsim_state* s, double2* dst, uint64_t offset, uint64_t count) {
  k_convert_out<<<grid_for(count, THREADS), THREADS, 0, s->stream>>>(dst, reinterpret_cast<const float2*>(s->amp) + offset, count);
  NCSIM_LAUNCHED("convert_out");
}
void launch_gather(const ncsim_state* s, const uint64_t* idx, double2* out, uint64_t count) {
  NCSIM_DISPATCH(s, {
    k_gather<R><<<grid_for(count, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), idx, out, count, s->len);
  });
  NCSIM_LAUNCHED("gather");
}
void launch_kron(const ncsim_state* a, const ncsim_state* b, ncsim_state* out) {
  NCSIM_DISPATCH(out, {
    k_kron<R><<<grid_for(out->len, THREADS), THREADS, 0, out->stream>>>(amp_of<R>(out), amp_of<R>(a), amp_of<R>(b),
                                                                        int(a->n), out->len);
  });
  NCSIM_LAUNCHED("kron");
}

static int reduce_grid(uint64_t items) {
  int g = int(grid_for(items, REDUCE_THREADS, 4, 2));
  return std::min(g, MAX_REDUCE_BLOCKS);
}

int launch_norm_partials(const ncsim_state* s) {
  int g = reduce_grid(s->len);
  ProfScope ps(s, K_NORM, 0.5 * full_bytes(s));
  NCSIM_DISPATCH(s, { k_norm<R><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, s->partials); });
  NCSIM_LAUNCHED("norm");
  return g;
}

int launch_expect_partials(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, bool with_norm) {
  int g;
  ProfScope ps(s, K_EXPECT, 0.5 * full_bytes(s));
  NCSIM_DISPATCH(s, {
    if (x == 0) {
      g = reduce_grid(s->len);
      if (with_norm) k_expect_diag<R, true><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, z, int(phase & 3), s->partials);
      else k_expect_diag<R, false><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, z, int(phase & 3), s->partials);
    } else {
      int h = 63 - __builtin_clzll(x);
      uint64_t np = s->len >> 1;
      g = reduce_grid(np);
      if (with_norm) k_expect_pair<R, true><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), np, h, x, z, int(phase & 3), s->partials);
      else k_expect_pair<R, false><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), np, h, x, z, int(phase & 3), s->partials);
    }
  });
  NCSIM_LAUNCHED("expectation");
  return g;
}

int launch_inner_partials(const ncsim_state* a, const ncsim_state* b) {
  int g = reduce_grid(a->len);
  ProfScope ps(a, K_INNER, full_bytes(a));
  NCSIM_DISPATCH(a, { k_inner<R><<<g, REDUCE_THREADS, 0, a->stream>>>(amp_of<R>(a), amp_of<R>(b), a->len, a->partials); });
  NCSIM_LAUNCHED("inner");
  return g;
}

int launch_compare_partials(const ncsim_state* a, const ncsim_state* b, double* maxdiff) {
  int g = reduce_grid(a->len);
  ProfScope ps(a, K_INNER, 0.5 * (full_bytes(a) + full_bytes(b)));
  double* p = a->partials;
  if (a->precision == NCSIM_C128 && b->precision == NCSIM_C128)
    k_compare<double, double><<<g, REDUCE_THREADS, 0, a->stream>>>(amp_of<double>(a), amp_of<double>(b), a->len, p, maxdiff);
  else if (a->precision == NCSIM_C128)
    k_compare<double, float><<<g, REDUCE_THREADS, 0, a->stream>>>(amp_of<double>(a), amp_of<float>(b), a->len, p, maxdiff);
  else if (b->precision == NCSIM_C128)
    k_compare<float, double><<<g, REDUCE_THREADS, 0, a->stream>>>(amp_of<float>(a), amp_of<double>(b), a->len, p, maxdiff);
  else
    k_compare<float, float><<<g, REDUCE_THREADS, 0, a->stream>>>(amp_of<float>(a), amp_of<float>(b), a->len, p, maxdiff);
  NCSIM_LAUNCHED("compare");
  return g;
}

int launch_project_partials(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, bool outcome) {
  int g;
  // a diagonal projection reads every amplitude and writes only the nonzero ones of the other outcome, a
  // share that depends on the state's support (half of a dense register, none of one already measured): the
  // profiler counts the reads alone, a lower bound on its traffic
  ProfScope ps(s, K_PROJECT, x ? full_bytes(s) : 0.5 * full_bytes(s));
  NCSIM_DISPATCH(s, {
    if (x == 0) {
      g = reduce_grid(s->len);
      k_project_diag<R><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), s->len, z, int(phase & 3), outcome, s->partials);
    } else {
      int h = 63 - __builtin_clzll(x);
      uint64_t np = s->len >> 1;
      g = reduce_grid(np);
      k_project_pair<R><<<g, REDUCE_THREADS, 0, s->stream>>>(amp_of<R>(s), np, h, x, z, int(phase & 3), outcome, s->partials);
    }
  });
  NCSIM_LAUNCHED("project");
  return g;
}

void launch_block_weights(const ncsim_state* s, double* w, uint64_t nblocks, uint64_t block) {
  ProfScope ps(s, K_SAMPLE, 0.5 * full_bytes(s));
  NCSIM_DISPATCH(s, {
    k_block_weights<R><<<grid_for(nblocks * 32, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), nblocks, block, w);
  });
  NCSIM_LAUNCHED("block_weights");
}

void launch_sample_walk(const ncsim_state* s, const double* u, const uint64_t* blk, const double* acc, uint64_t shots,
                        uint64_t block, uint64_t* out) {
  NCSIM_DISPATCH(s, {
    k_sample_walk<R><<<grid_for(shots * 32, THREADS), THREADS, 0, s->stream>>>(amp_of<R>(s), u, blk, acc, shots, block, out);
  });
  NCSIM_LAUNCHED("sample_walk");
}

void fetch_partials(const ncsim_state* s, int nb, int slots, double* out) {
  NCSIM_CUDA(cudaMemcpyAsync(s->host_partials, s->partials, size_t(nb) * PARTIAL_SLOTS * sizeof(double),
                             cudaMemcpyDeviceToHost, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  // pairwise over the blocks, in a fixed order
  std::vector<double> v(nb);
  for (int j = 0; j < slots; ++j) {
    for (int b = 0; b < nb; ++b) v[b] = s->host_partials[b * PARTIAL_SLOTS + j];
    int m = nb;
    while (m > 1) {
      int h = (m + 1) / 2;
      for (int i = 0; i + h < m; ++i) v[i] += v[i + h];
      m = h;
    }
    out[j] = nb ? v[0] : 0.0;
  }
}

}  // namespace ncsim

// ===========================================================================
// <P> and <psi|psi> over caller-owned device amplitudes, allocating nothing.
//
// Some callers cannot let a library call cudaMalloc: they keep the amplitudes
// in device memory they already own (a framework's memory pool, a buffer
// carved from a fixed device budget), and a device allocation or free there
// could synchronize the device, fragment the pool or break the budget they
// reserved.  This entry point reads their buffer in place and keeps its
// reduction scratch in the file-scope array below instead.
//
// The array: NOALLOC_BLOCKS per-block partials (PARTIAL_SLOTS doubles each)
// plus 8 result doubles, 32 KB + 64 B, held by every GPU that loads the
// library until the process exits.  Host code must not pass the array's name
// to a kernel (on the host it is only a stand-in, not a device address): the
// device address comes from cudaGetSymbolAddress, fetched once per device,
// with that device current, by the first call made on it.  That first call
// therefore does the set-up and should come before any stream capture.
//
// Every call shares the array and it keeps the last call's contents.  Each
// call writes every partial slot it later reads (one per launched block) and
// then the result slots, so nothing has to start at zero; calls that overlap
// on the GPU (two streams, two host threads) race on the array and must be
// serialized by the caller.
// ===========================================================================
namespace ncsim {
namespace {

constexpr int NOALLOC_BLOCKS = 1024;
constexpr int NOALLOC_RESULT = NOALLOC_BLOCKS * PARTIAL_SLOTS;
constexpr int NOALLOC_MAX_QUBITS = 34;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_RESULT + 8];

// slot j of the result = the sum over blocks of slot j, in block order
__global__ void k_noalloc_finish(double* scratch, int nblocks, int slots) {
  const int j = threadIdx.x;
  if (j >= slots) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += scratch[b * PARTIAL_SLOTS + j];
  scratch[NOALLOC_RESULT + j] = s;
}

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// the array's device address on the current device (set-up on first use)
double* noalloc_scratch(int dev) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) throw Error(NCSIM_ERR_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw Error(NCSIM_ERR_DEVICE, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
    }
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_ptr[dev];
}

// cuMemGetAddressRange through the runtime's driver entry point (the library
// links no driver library); null when the driver does not provide it
using MemRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
MemRangeFn mem_range_fn() {
  static MemRangeFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<MemRangeFn>(f);
  }();
  return fn;
}

// Host-side checks of a caller's buffer and stream, none of which allocates:
// the buffer is device (or managed) memory of the current device and holds
// `bytes` bytes from `p` inside one allocation, and a given stream belongs to
// the current device.  A mistake is reported before anything is launched.
void check_caller_buffer(const void* p, size_t bytes, int dev, cudaStream_t st) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    throw Error(NCSIM_ERR_INVALID, "amplitudes: not a pointer the CUDA runtime knows");
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
    throw Error(NCSIM_ERR_INVALID, "amplitudes must be device or managed memory (host memory was given)");
  if (at.type == cudaMemoryTypeDevice && at.device != dev)
    throw Error(NCSIM_ERR_INVALID, "amplitudes live on device " + std::to_string(at.device) +
                                       ", but device " + std::to_string(dev) + " is current");
  if (MemRangeFn fn = mem_range_fn()) {
    CUdeviceptr base = 0;
    size_t size = 0;
    if (fn(&base, &size, reinterpret_cast<CUdeviceptr>(p)) != CUDA_SUCCESS)
      throw Error(NCSIM_ERR_INVALID, "amplitudes: no device allocation contains the pointer");
    const uint64_t off = uint64_t(reinterpret_cast<uintptr_t>(p)) - uint64_t(base);
    if (off > size || size - off < bytes)
      throw Error(NCSIM_ERR_INVALID, "amplitude buffer too short: " + std::to_string(bytes) + " bytes needed, " +
                                         std::to_string(size - std::min<uint64_t>(off, size)) +
                                         " left in its allocation");
  }
  if (st) {
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
      cudaGetLastError();
      throw Error(NCSIM_ERR_INVALID, "stream: not a valid CUDA stream");
    }
    if (sdev != dev)
      throw Error(NCSIM_ERR_INVALID, "stream belongs to device " + std::to_string(sdev) + ", but device " +
                                         std::to_string(dev) + " is current");
  }
}

}  // namespace

}  // namespace ncsim

extern "C" ncsim_status ncsim_measure_stats_noalloc(const void* amps, uint32_t n, int32_t precision, uint64_t x,
                                                    uint64_t z, uint32_t phase, void* stream, double* expectation_re_im,
                                                    double* norm_sq) {
  using namespace ncsim;
  return guarded([&] {
    if (!amps) throw Error(NCSIM_ERR_INVALID, "amplitudes are null");
    if (!expectation_re_im || !norm_sq) throw Error(NCSIM_ERR_INVALID, "outputs are null");
    if (precision != NCSIM_C128 && precision != NCSIM_C64) throw Error(NCSIM_ERR_INVALID, "precision must be C128 or C64");
    if (n > uint32_t(NOALLOC_MAX_QUBITS))
      throw Error(NCSIM_ERR_INVALID, "register of " + std::to_string(n) + " qubits exceeds the " +
                                         std::to_string(NOALLOC_MAX_QUBITS) + "-qubit maximum of the no-allocation entry point");
    const uint64_t len = uint64_t(1) << n;
    if ((x | z) & ~(len - 1)) throw Error(NCSIM_ERR_INVALID, "Pauli acts outside the register");
    int dev = 0;
    NCSIM_CUDA(cudaGetDevice(&dev));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    check_caller_buffer(amps, size_t(len) * (precision == NCSIM_C128 ? 16 : 8), dev, st);
    double* scratch = noalloc_scratch(dev);
    const int ph = int(phase & 3);
    int g;
    auto launch = [&](auto tag) {
      using R = decltype(tag);
      const V<R>* a = static_cast<const V<R>*>(amps);
      if (x == 0) {
        g = std::min(reduce_grid(len), NOALLOC_BLOCKS);
        k_expect_diag<R, true><<<g, REDUCE_THREADS, 0, st>>>(a, len, z, ph, scratch);
      } else {
        const int h = 63 - __builtin_clzll(x);
        g = std::min(reduce_grid(len >> 1), NOALLOC_BLOCKS);
        k_expect_pair<R, true><<<g, REDUCE_THREADS, 0, st>>>(a, len >> 1, h, x, z, ph, scratch);
      }
    };
    if (precision == NCSIM_C128) launch(double());
    else launch(float());
    NCSIM_LAUNCHED("measure_stats_noalloc");
    k_noalloc_finish<<<1, 32, 0, st>>>(scratch, g, 3);
    NCSIM_LAUNCHED("measure_stats_noalloc finish");
    double res[3];
    NCSIM_CUDA(cudaMemcpyAsync(res, scratch + NOALLOC_RESULT, sizeof(res), cudaMemcpyDeviceToHost, st));
    NCSIM_CUDA(cudaStreamSynchronize(st));
    expectation_re_im[0] = res[0];
    expectation_re_im[1] = res[1];
    *norm_sq = res[2];
  });
}
