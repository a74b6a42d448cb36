// Precision form, device side: one kernel launch per pass.
//
// A persistent CTA per SM streams tiles of 2^12 complex64 amplitudes (32 KB)
// through shared memory: two producer warps copy 16-byte chunks with cp.async
// (completion on the tile's mbarrier through cp.async.mbarrier.arrive) into
// five rotating tile buffers.  The CTA takes its tiles in sets of four, and
// four warpgroups run the pass's program, one on each tile of a set, so that a
// group splits amplitudes while the others' MMAs and read-backs run; each group
// writes its finished tile back itself (16-byte stores), so the stores overlap
// the other groups' work and the producers only load.  The unitaries' B
// operands (16 KB bf16 images each) stream from L2 into three rotating slots
// (a third producer warp); each group's tcgen05.commit (or release) frees a
// slot.  Per group and tile:
//   unitary op: the tile as 32 rows (the unitary's 5 qubits) x 128 columns;
//     each thread owns a column, splits its 32 amplitudes into bf16 hi/lo
//     and writes them into its own TMEM lane (A = X^T, 128 x 64, K-major,
//     tcgen05.st); one thread issues 12 tcgen05.mma with A in TMEM (M=128,
//     N=64, K=16, bf16 in, f32 accumulate in the group's 64 TMEM columns):
//       D = Xhi.Rhi + Xlo.Rhi + Xhi.Rlo
//     with R the real form [[Ur, -Ui], [Ui, Ur]] of the fused unitary (bf16
//     hi/lo images made on the host, output columns ordered so that each
//     row's real and imaginary parts are adjacent); each thread reads its D
//     row back (tcgen05.ld) and writes the 32 new amplitudes into the tile;
//   diagonal op: reduced, where it can be, to a phase per column and a sign
//     mask over the rows of a neighbouring unitary and applied in that
//     unitary's split or read-back; otherwise the tile index splits into two
//     6-bit halves, the active terms fold into a 64-entry phase table per half
//     and a parity table for cross-half signs, and one sweep applies them.
// Every wait on an mbarrier is bounded in time: on timeout the CTA records an
// error code and every role stops at its next uniform decision point, waits
// for its own copies and frees its TMEM.
#include <cuda_bf16.h>

#include "engine.cuh"
#include "fused_plan.hpp"

#include <algorithm>
#include <memory>

namespace ncsim {
namespace fused {

namespace {

constexpr int GROUP_THREADS = 128;                       // one warpgroup runs the program on one tile
constexpr int GROUPS = 4;                                // four tiles in flight per CTA
constexpr int COMPUTE_THREADS = GROUPS * GROUP_THREADS;  // warps 0-15
constexpr int WARP_TILES = COMPUTE_THREADS / 32;         // warps 16-17: tile loads and stores
constexpr int TILE_THREADS = 64;
constexpr int WARP_OPS = WARP_TILES + 2;                 // warp 18: B operand images
constexpr int THREADS = COMPUTE_THREADS + TILE_THREADS + 32;
constexpr int TILE = 1 << TILE_BITS;
constexpr uint32_t TILE_BYTES = uint32_t(TILE) * 8u;
constexpr int OPERAND_BYTES = 16384;  // B: bf16 hi (8 KB) + lo (8 KB)
constexpr int NTILEBUF = GROUPS + 1;  // tile buffers rotating over the CTA's tiles (one loading ahead)
constexpr int NOPSLOT = 3;            // B operand slots rotating over the unitary uses
constexpr int SM_B = 0;
constexpr int SM_TILE0 = SM_B + NOPSLOT * OPERAND_BYTES;
constexpr int SM_TOTAL = SM_TILE0 + NTILEBUF * int(TILE_BYTES);
constexpr int SM_DYNAMIC = SM_TOTAL + 1008;  // the dynamic base is 16-byte aligned: slack to reach 1024
// per group 128 columns: the accumulator D (64), the A operand's bf16 hi (32) and lo (32)
constexpr uint32_t TMEM_COLS = 512;  // 128 per group, rounded up to a power of two
constexpr long long WAIT_CYCLES = 4000000000ll;  // about 2 s at 1.9 GHz
constexpr int HALF = TILE_BITS / 2;              // 6-bit halves of the tile index
constexpr int COL_BITS = TILE_BITS - GROUP_QUBITS;  // a unitary's column index: the tile bits outside its qubits
constexpr int MAX_CHUNKS = 48;                      // column-term chunks per pass
// Tile layout in shared memory: element e sits at e ^ L(e), where the linear map L folds
// tile bits 4..11 into element bits 1..3 (bit j contributes w[j - 4] below).  A unitary's
// thread owns a column whose 32 lanes step through its lowest non-gate bits; without
// the fold, gate qubits among tile bits 0..3 send those lanes to a few banks (up to
// 16-way conflicts).  The fold keeps bit 0, so 16-byte pairs stay contiguous, and it
// is linear: the address of (column | row) is the XOR of the two parts' addresses.
// The weights minimise the modelled conflicts over the window placements of the
// layered-circuit plans (3.2 -> 2.3 shared-memory wavefronts per warp access; 2 is the
// minimum for 8-byte elements).
__host__ __device__ inline uint32_t swz_fold(uint32_t e) {
  const uint8_t w[TILE_BITS - 4] = {14, 6, 12, 10, 14, 12, 8, 6};
  uint32_t l = 0;
#pragma unroll
  for (int j = 4; j < TILE_BITS; ++j)
    if ((e >> j) & 1u) l ^= w[j - 4];
  return l;
}

enum TermClass : uint8_t { T_LOW = 0, T_HIGH = 1, T_CROSS_SIGN = 2, T_GENERIC = 3 };

struct OpDesc {
  uint8_t kind;  // 0 unitary, 1 terms, 2 terms applied by the next unitary's split, 3 by the previous one's read-back
  uint8_t u;     // unitary index (operand slot)
  // terms [t0, t1) sorted by class: low half [t0,tl), high half [tl,th),
  // cross-half signs [th,tc), the rest [tc,t1)
  uint16_t t0, tl, th, tc, t1;
  uint8_t pc0, pc1;  // unitary: chunks of the preceding terms op, applied while splitting
  uint8_t qc0, qc1;  // unitary: chunks of the following terms op, applied while reading back
};

struct TermDesc {
  uint64_t cmask;  // bits outside the window (constant over a tile)
  uint32_t tmask;  // tile-local bits (for a split-applied term: the unitary's non-gate bits)
  float cr, ci;
  uint32_t rowpat;  // split-applied sign term: the rows (gate index) whose sign flips; 0: a phase on the column
};

// Up to 32 terms of a diagonal op applied by a unitary's split or read-back,
// as bit masks over the chunk's terms (bit t = term t0 + t).  A term is active
// on a column when its bits outside the tile are set in the tile's base (a
// per-tile ballot) and its column bits are set in the column index; active
// terms then flip row signs (row[j]: rows with gate bit j set), negate the
// column (neg) or multiply it by their phase (gen).
struct ColChunk {
  uint32_t need[COL_BITS];     // terms whose condition includes column bit j
  uint32_t row[GROUP_QUBITS];  // sign terms on the rows with gate bit j set
  uint32_t neg;                // -1 on the whole column
  uint32_t gen;                // other phases on the whole column
  uint16_t t0;
  uint16_t cnt;
};

struct PassParams {
  float2* amp;
  const uint4* rops;  // nu x 16 KB operand images
  int* err;
  uint64_t ntiles;
  int wl;                      // window bits 0..wl-1 are index bits 0..wl-1
  uint8_t win[TILE_BITS];      // window qubits, ascending (tile-local bit j = win[j])
  int nops, nu;
  uint8_t pos[MAX_UNITARIES][GROUP_QUBITS];  // tile-local positions of each unitary's qubits
  int nchunks;
  OpDesc ops[MAX_OPS];
  TermDesc terms[MAX_TERMS];
  ColChunk chunks[MAX_CHUNKS];
};

// ---- PTX wrappers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// try_wait with a suspend-time hint: the thread sleeps (up to about 1 ms) until
// the phase completes instead of spinning
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}
// bounded wait: false when the phase did not complete within WAIT_CYCLES
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > WAIT_CYCLES) return false;
  }
  return true;
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// arrives on the mbarrier once this thread's earlier cp.async copies have landed
__device__ __forceinline__ void cp_async_arrive(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
constexpr int BAR_TILES = 1 + GROUPS;  // named barriers: 1..GROUPS the groups, then the tile loaders
// A named barrier that also ORs a flag over its threads: every thread gets the
// same answer, so a stop decided from it is uniform across the barrier's threads.
__device__ __forceinline__ bool bar_any(int id, int count, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(uint32_t(v)), "r"(id), "r"(count)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, 128-byte swizzle, 8-row atoms 1024 bytes apart (sm100 descriptor version 1)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(1) << 16;            // leading byte offset (16 B; unused by swizzled K-major)
  d |= uint64_t(1024 >> 4) << 32;    // stride byte offset between 8-row atoms
  d |= uint64_t(1) << 46;            // descriptor version for sm100
  d |= uint64_t(2) << 61;            // SWIZZLE_128B
  return d;
}

// D (TMEM) += A (TMEM, K-major rows = lanes) x B (shared memory descriptor)
__device__ __forceinline__ void mma_bf16_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "r"(tmem_a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
// four 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t (&v)[4]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
               "r"(v[2]), "r"(v[3])
               : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

#define NCSIM_TMEM_LD16(taddr, r)                                                                                     \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];" \
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),        \
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])    \
               : "r"(taddr))

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&v);
}
// the two bf16 of a packed pair as floats (low half = first element)
__device__ __forceinline__ float lo_half(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float hi_half(uint32_t p) { return __uint_as_float(p & 0xffff0000u); }

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// index of tile-local element e of a tile whose base index is `base`
__device__ __forceinline__ uint64_t global_index(uint64_t base, uint32_t e, const PassParams& P) {
  uint64_t g = base | (e & ((1u << P.wl) - 1));
  for (int j = P.wl; j < TILE_BITS; ++j) g |= uint64_t((e >> j) & 1u) << P.win[j];
  return g;
}
// the tile's base: the tile number deposited into the bits outside the window
__device__ __forceinline__ uint64_t tile_base(uint64_t t, const PassParams& P) {
  uint64_t v = t;
  for (int j = 0; j < TILE_BITS; ++j) {
    const int b = P.win[j];
    v = ((v >> b) << (b + 1)) | (v & ((uint64_t(1) << b) - 1));
  }
  return v;
}

// The tile's phase tables of a terms op, built by one group's 128 threads: the
// low-half phase products and cross-half sign parities (threads 0-63) and the
// high-half phase products (64-127).
__device__ __forceinline__ void build_tables(const OpDesc& op, uint64_t base, int tg, const TermDesc* terms,
                                             float2* tab_lo, float2* tab_hi, uint8_t* tab_cross) {
  if (tg < 64) {
    const uint32_t x = uint32_t(tg);
    float2 c = make_float2(1.f, 0.f);
    for (int k = op.t0; k < op.tl; ++k) {
      const TermDesc tm = terms[k];
      if ((base & tm.cmask) == tm.cmask && (x & tm.tmask) == tm.tmask) c = cmulf(c, make_float2(tm.cr, tm.ci));
    }
    tab_lo[x] = c;
    uint32_t v = 0;
    for (int k = op.th; k < op.tc; ++k) {
      const TermDesc tm = terms[k];
      if ((base & tm.cmask) != tm.cmask) continue;
      if (x & (tm.tmask >> HALF)) v ^= tm.tmask & ((1u << HALF) - 1);
    }
    tab_cross[x] = uint8_t(v);
  } else {
    const uint32_t x = uint32_t(tg - 64);
    float2 c = make_float2(1.f, 0.f);
    for (int k = op.tl; k < op.th; ++k) {
      const TermDesc tm = terms[k];
      const uint32_t hm = tm.tmask >> HALF;
      if ((base & tm.cmask) == tm.cmask && (x & hm) == hm) c = cmulf(c, make_float2(tm.cr, tm.ci));
    }
    tab_hi[x] = c;
  }
}

// the phase of tile element e under a terms op (its tables built)
__device__ __forceinline__ float2 term_phase(uint32_t e, const OpDesc& op, uint64_t base, const TermDesc* terms,
                                             const float2* tab_lo, const float2* tab_hi, const uint8_t* tab_cross) {
  const uint32_t lo = e & ((1u << HALF) - 1), hi = e >> HALF;
  float2 c = cmulf(tab_lo[lo], tab_hi[hi]);
  if (__popc(lo & tab_cross[hi]) & 1) c = make_float2(-c.x, -c.y);
  for (int k = op.tc; k < op.t1; ++k) {
    const TermDesc tm = terms[k];
    if ((base & tm.cmask) == tm.cmask && (e & tm.tmask) == tm.tmask) c = cmulf(c, make_float2(tm.cr, tm.ci));
  }
  return c;
}

// The chunks [c0, c1) of a diagonal op applied by a unitary's split or read-back,
// for column tg of that unitary (act: the chunks' terms active on this tile):
// a sign mask over the 32 rows and a phase for the whole column.
__device__ __forceinline__ void column_chunks(const ColChunk* chunks, const uint32_t* act, int c0, int c1, uint32_t tg,
                                              const TermDesc* terms, uint32_t& smask, float2& cth, bool& scal) {
  const uint32_t rowpat[GROUP_QUBITS] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
  for (int c = c0; c < c1; ++c) {
    const ColChunk& ch = chunks[c];
    uint32_t a = act[c];
#pragma unroll
    for (int j = 0; j < COL_BITS; ++j) a &= ((tg >> j) & 1u) ? ~0u : ~ch.need[j];
#pragma unroll
    for (int j = 0; j < GROUP_QUBITS; ++j) smask ^= rowpat[j] & (0u - (uint32_t(__popc(a & ch.row[j])) & 1u));
    if (__popc(a & ch.neg) & 1) {
      cth = make_float2(-cth.x, -cth.y);
      scal = true;
    }
    for (uint32_t gb = a & ch.gen; gb; gb &= gb - 1) {
      const TermDesc& td = terms[ch.t0 + (__ffs(gb) - 1)];
      cth = cmulf(cth, make_float2(td.cr, td.ci));
      scal = true;
    }
  }
}

__device__ __forceinline__ void bar_group(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(GROUP_THREADS) : "memory");
}

__global__ void __launch_bounds__(THREADS, 1) k_fused_pass(const __grid_constant__ PassParams P) {
  extern __shared__ uint8_t smem_raw[];
  // 1024-byte aligned (the swizzled operand images); an offset into the shared array keeps the
  // pointers in the shared address space (32-bit addressing for every tile access)
  uint8_t* smem = smem_raw + ((0u - smem_u32(smem_raw)) & 1023u);
  // mbarriers: tile full[3], tile done[3], operand full[3], operand empty[3], mma[2]
  __shared__ __align__(8) uint64_t bars[2 * NTILEBUF + 2 * NOPSLOT + GROUPS];
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ uint16_t nbit[MAX_UNITARIES][COL_BITS];       // stored offset of each non-gate bit (column bits)
  __shared__ uint16_t gbit[MAX_UNITARIES][GROUP_QUBITS];   // and of each gate bit (row bits)
  __shared__ uint8_t swz[1 << (TILE_BITS - 4)];             // L(e) by e >> 4
  __shared__ float2 tab_lo[GROUPS][1 << HALF], tab_hi[GROUPS][1 << HALF];
  __shared__ uint8_t tab_cross[GROUPS][1 << HALF];
  __shared__ uint64_t run_off[TILE >> LOW_BITS];  // index bits of run r of a tile (the window bits above wl)
  __shared__ TermDesc s_terms[MAX_TERMS];         // the pass's program, read with runtime indices
  __shared__ OpDesc s_ops[MAX_OPS];
  __shared__ ColChunk s_chunks[MAX_CHUNKS];
  __shared__ uint32_t act_sh[GROUPS][MAX_CHUNKS];  // per tile: the chunks' terms active on it

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto bar_tfull = [&](int b) { return smem_u32(&bars[b]); };
  auto bar_tdone = [&](int b) { return smem_u32(&bars[NTILEBUF + b]); };
  auto bar_ofull = [&](int s) { return smem_u32(&bars[2 * NTILEBUF + s]); };
  auto bar_oempty = [&](int s) { return smem_u32(&bars[2 * NTILEBUF + NOPSLOT + s]); };
  auto bar_mma = [&](int g) { return smem_u32(&bars[2 * NTILEBUF + 2 * NOPSLOT + g]); };
  auto fail = [&](int code) {
    abort_sh = 1;
    atomicCAS(P.err, 0, code);
  };

  if (tid == 0) {
    for (int i = 0; i < NTILEBUF; ++i) {
      mbar_init(bar_tfull(i), TILE_THREADS);  // one cp.async arrival per tile thread
      mbar_init(bar_tdone(i), GROUP_THREADS);
    }
    for (int i = 0; i < NOPSLOT; ++i) {
      mbar_init(bar_ofull(i), 1);
      mbar_init(bar_oempty(i), GROUPS);  // one commit (or release) per group
    }
    for (int g = 0; g < GROUPS; ++g) mbar_init(bar_mma(g), 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (uint32_t r = uint32_t(tid); r < (uint32_t(TILE) >> P.wl); r += THREADS) run_off[r] = global_index(0, r << P.wl, P);
  for (uint32_t h = uint32_t(tid); h < (1u << (TILE_BITS - 4)); h += THREADS) swz[h] = uint8_t(swz_fold(h << 4));
  for (int i = tid; i < P.nops; i += THREADS) s_ops[i] = P.ops[i];
  for (int i = tid; i < P.nchunks; i += THREADS) s_chunks[i] = P.chunks[i];
  {
    int nterms = 0;
    for (int i = 0; i < P.nops; ++i) nterms = max(nterms, int(P.ops[i].t1));
    for (int i = tid; i < nterms; i += THREADS) s_terms[i] = P.terms[i];
  }
  for (int u = tid; u < P.nu; u += THREADS) {  // the non-gate tile bits of each unitary
    uint32_t gm = 0;
    for (int j = 0; j < GROUP_QUBITS; ++j) gm |= 1u << P.pos[u][j];
    int m = 0;
    for (int b = 0; b < TILE_BITS; ++b)
      if (!((gm >> b) & 1)) nbit[u][m++] = uint16_t((1u << b) ^ swz_fold(1u << b));
    for (int j = 0; j < GROUP_QUBITS; ++j) gbit[u][j] = uint16_t((1u << P.pos[u][j]) ^ swz_fold(1u << P.pos[u][j]));
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  // tiles go in groups of GROUPS, one per warpgroup: this CTA's it-th tile is tile_of(it),
  // in buffer it % NTILEBUF; only the register's last group of tiles can be short, and it
  // is the last one of the CTA that takes it
  const uint64_t nsets = (P.ntiles + GROUPS - 1) / GROUPS;
  const uint64_t my_sets = nsets > blockIdx.x ? (nsets - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t my_tiles = uint64_t(GROUPS) * my_sets;
  auto tile_of = [&](uint64_t it) {
    return uint64_t(GROUPS) * (uint64_t(blockIdx.x) + (it / GROUPS) * gridDim.x) + (it % GROUPS);
  };
  auto have = [&](uint64_t it) { return tile_of(it) < P.ntiles; };
  float2* tiles = reinterpret_cast<float2*>(smem + SM_TILE0);
  auto at = [&](uint32_t e) { return e ^ uint32_t(swz[e >> 4]); };  // stored position of tile element e
  const uint32_t cshift = uint32_t(P.wl) - 1u;  // 16-byte chunks of 2 amplitudes per run: 2^(wl-1)
  auto chunk_addr = [&](uint64_t base, uint32_t c) {
    return P.amp + (base | run_off[c >> cshift]) + 2u * (c & ((1u << cshift) - 1u));
  };

  if (warp == WARP_TILES || warp == WARP_TILES + 1) {
    // ---------------- tile loads (cp.async): 64 threads, 16-byte chunks ----------------
    const int pt = tid - COMPUTE_THREADS;
    auto load_tile = [&](uint64_t it) {
      const int b = int(it % NTILEBUF);
      const uint64_t base = tile_base(tile_of(it), P);
      const uint32_t dst = smem_u32(tiles + size_t(b) * TILE);
#pragma unroll 4
      for (uint32_t c = uint32_t(pt); c < uint32_t(TILE) / 2; c += TILE_THREADS) cp_async16(dst + 8u * at(2u * c), chunk_addr(base, c));
      cp_async_arrive(bar_tfull(b));
    };
    // wait (one thread) until the group has written tile j back; false (for all 64 threads alike) to stop
    auto wait_done = [&](uint64_t j) -> bool {
      if (pt == 0 && have(j) && !mbar_wait(bar_tdone(int(j % NTILEBUF)), uint32_t((j / NTILEBUF) & 1))) fail(3);
      return !bar_any(BAR_TILES, TILE_THREADS, abort_sh);
    };
    for (uint64_t it = 0; it < my_tiles; ++it) {
      if (it >= NTILEBUF && !wait_done(it - NTILEBUF)) break;  // the buffer is free once its tile is written back
      if (have(it)) load_tile(it);
    }
    // copies of this thread still in flight land before the CTA exits
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp == WARP_OPS) {
    // ---------------- B operand images: use k = set * nu + u, slot k % NOPSLOT ----------------
    const uint64_t nk = my_sets * uint64_t(P.nu);
    uint64_t k = 0;
    for (; k < nk; ++k) {
      const int sl = int(k % NOPSLOT);
      if (k >= NOPSLOT) {
        bool go = true;
        if (lane == 0) {
          go = mbar_wait(bar_oempty(sl), uint32_t(((k - NOPSLOT) / NOPSLOT) & 1));
          if (!go) fail(4);
          go = go && !abort_sh;
        }
        if (!__shfl_sync(0xffffffffu, go, 0)) break;  // lane 0 decides for the warp
      }
      if (lane == 0) {
        mbar_expect_tx(bar_ofull(sl), OPERAND_BYTES);
        bulk_load(smem_u32(smem + SM_B + sl * OPERAND_BYTES), P.rops + (k % uint64_t(P.nu)) * (OPERAND_BYTES / 16),
                  OPERAND_BYTES, bar_ofull(sl));
      }
      __syncwarp();
    }
    if (k < nk)  // an abort: let the loads already issued land
      for (uint64_t j = k >= NOPSLOT ? k - NOPSLOT : 0; j < k; ++j)
        if (lane == 0) mbar_wait(bar_ofull(int(j % NOPSLOT)), uint32_t((j / NOPSLOT) & 1));
  } else {
    // ---------------- tensor-core program: group g on its tile of each set ----------------
    const int g = warp / 4, tg = tid & (GROUP_THREADS - 1);
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
    const uint32_t d_tmem = tmem + uint32_t(128 * g);  // columns: D [0,64), A hi [64,96), A lo [96,128)
    const uint32_t a_tmem = d_tmem + 64u;
    const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
    const uint32_t taddr = d_tmem + lane_base;          // this warp's lanes of D
    const uint32_t taddr_a = a_tmem + lane_base;        // and of A
    uint32_t mma_phase = 0;
    for (uint64_t p = 0; p < my_sets; ++p) {
      const uint64_t it = uint64_t(GROUPS) * p + uint64_t(g);
      const bool mine = have(it);
      const int b = int(it % NTILEBUF);
      const uint64_t base = mine ? tile_base(tile_of(it), P) : 0;
      if (mine && tg < 32) {  // which column terms apply on this tile (their bits outside it)
        for (int c = 0; c < P.nchunks; ++c) {
          bool on = false;
          if (tg < int(s_chunks[c].cnt)) {
            const uint64_t cm = s_terms[s_chunks[c].t0 + tg].cmask;
            on = (base & cm) == cm;
          }
          const uint32_t m = __ballot_sync(0xffffffffu, on);
          if (tg == 0) act_sh[g][c] = m;
        }
      }
      if (mine && tg == 0 && !mbar_wait(bar_tfull(b), uint32_t((it / NTILEBUF) & 1))) fail(1);
      if (bar_any(1 + g, GROUP_THREADS, abort_sh)) break;
      float2* T = tiles + size_t(b) * TILE;
      for (int oi = 0; oi < P.nops; ++oi) {
        const OpDesc op = s_ops[oi];
        if (op.kind >= 2) continue;  // applied by a neighbouring unitary's split or read-back
        if (op.kind == 1) {
          if (!mine) continue;
          // ---- diagonal terms: per-tile tables, then one sweep of the tile ----
          build_tables(op, base, tg, s_terms, tab_lo[g], tab_hi[g], tab_cross[g]);
          bar_group(g);
          {
            // element e = tg + 128 i: its low 6 bits are the thread's, so the low-half
            // phase is one read; the high-half entries are the same across a warp
            const uint32_t lo = uint32_t(tg) & ((1u << HALF) - 1);
            const float2 L = tab_lo[g][lo];
            if (op.tc == op.t1) {
              // blocks of 8: every load before any store (the tile and the tables may alias as far
              // as the compiler knows, so a store would hold back the next loads)
              const float2* __restrict__ th = tab_hi[g];
              const uint8_t* __restrict__ tx = tab_cross[g];
#pragma unroll 1
              for (int i0 = 0; i0 < TILE / GROUP_THREADS; i0 += 8) {
                float2 v[8], h[8];
                uint32_t x[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                  const uint32_t e = uint32_t(tg + GROUP_THREADS * (i0 + j)), hi = e >> HALF;
                  v[j] = T[at(e)];
                  h[j] = th[hi];
                  x[j] = tx[hi];
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                  float2 c = cmulf(L, h[j]);
                  const uint32_t sg = uint32_t(__popc(lo & x[j]) & 1) << 31;
                  c = make_float2(__uint_as_float(__float_as_uint(c.x) ^ sg), __uint_as_float(__float_as_uint(c.y) ^ sg));
                  T[at(uint32_t(tg + GROUP_THREADS * (i0 + j)))] = cmulf(c, v[j]);
                }
              }
            } else {
#pragma unroll 4
              for (int i = 0; i < TILE / GROUP_THREADS; ++i) {
                const uint32_t e = uint32_t(tg + GROUP_THREADS * i);
                T[at(e)] = cmulf(term_phase(e, op, base, s_terms, tab_lo[g], tab_hi[g], tab_cross[g]), T[at(e)]);
              }
            }
          }
          bar_group(g);
          continue;
        }
        // ---- unitary op: this thread owns column tg (A row / TMEM lane) and its 32 rows ----
        const int u = op.u;
        const uint64_t k = p * uint64_t(P.nu) + uint64_t(u);
        const int sl = int(k % NOPSLOT);
        if (!mine) {
          // this group has no tile in the set: release the operand slot without using it
          if (abort_sh) break;
          if (tg == 0) {
            if (!mbar_wait(bar_ofull(sl), uint32_t((k / NOPSLOT) & 1))) fail(2);
            mbar_arrive(bar_oempty(sl));
          }
          continue;
        }
        // stored positions (the layout fold is linear: column and row parts combine by XOR)
        uint32_t cb = 0;
#pragma unroll
        for (int j = 0; j < COL_BITS; ++j) cb ^= ((tg >> j) & 1) ? uint32_t(nbit[u][j]) : 0u;
        const uint32_t p0 = gbit[u][0], p1 = gbit[u][1], p2 = gbit[u][2], p3 = gbit[u][3], p4 = gbit[u][4];
        uint32_t lo8[8];  // rows 0..7 (gate bits 0-2) of this column
#pragma unroll
        for (int i = 0; i < 8; ++i) lo8[i] = cb ^ ((i & 1) ? p0 : 0u) ^ ((i & 2) ? p1 : 0u) ^ ((i & 4) ? p2 : 0u);
        const uint32_t hi4[4] = {0u, p3, p4, p3 ^ p4};  // rows 8q..8q+7
        // a preceding diagonal op, reduced to this column: a phase and a sign mask over the 32 rows
        uint32_t smask = 0;
        float2 cth = make_float2(1.f, 0.f);
        bool scal = false;
        column_chunks(s_chunks, act_sh[g], op.pc0, op.pc1, uint32_t(tg), s_terms, smask, cth, scal);
        // warp-uniform decisions (a lane without a phase multiplies by exactly 1, one without
        // signs flips nothing), so the unrolled loops carry no divergent branches
        scal = __any_sync(0xffffffffu, scal);
        const bool flip = __any_sync(0xffffffffu, smask != 0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float2 xx[8];  // rows 8q..8q+7, loaded before any other work
#pragma unroll
          for (int i = 0; i < 8; ++i) xx[i] = T[lo8[i] ^ hi4[q]];
          if (scal) {
#pragma unroll
            for (int i = 0; i < 8; ++i) xx[i] = cmulf(cth, xx[i]);
          }
          if (flip) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const uint32_t sg = (smask << (31 - (8 * q + i))) & 0x80000000u;
              xx[i] = make_float2(__uint_as_float(__float_as_uint(xx[i].x) ^ sg),
                                  __uint_as_float(__float_as_uint(xx[i].y) ^ sg));
            }
          }
          // A row (this lane): K = row (real parts) and 32 + row (imaginary parts), two bf16 per
          // column, so rows 8q .. 8q+7 are columns 4q .. 4q+3 (re) and 16 + the same (im)
          uint32_t hr[4], lr[4], hm[4], lm[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 a = xx[2 * i], c = xx[2 * i + 1];
            hr[i] = pack_bf16(a.x, c.x);
            hm[i] = pack_bf16(a.y, c.y);
            lr[i] = pack_bf16(a.x - lo_half(hr[i]), c.x - hi_half(hr[i]));
            lm[i] = pack_bf16(a.y - lo_half(hm[i]), c.y - hi_half(hm[i]));
          }
          tmem_st4(taddr_a + uint32_t(4 * q), hr);
          tmem_st4(taddr_a + uint32_t(16 + 4 * q), hm);
          tmem_st4(taddr_a + uint32_t(32 + 4 * q), lr);
          tmem_st4(taddr_a + uint32_t(48 + 4 * q), lm);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        if (bar_any(1 + g, GROUP_THREADS, abort_sh)) break;
        if (tg == 0) {
          if (!mbar_wait(bar_ofull(sl), uint32_t((k / NOPSLOT) & 1))) fail(2);
          tc_fence_after();
          const uint32_t b_hi = smem_u32(smem + SM_B + sl * OPERAND_BYTES);
          const uint32_t b_lo = b_hi + OPERAND_BYTES / 2;
          const uint64_t dbh = sw128_desc(b_hi), dbl = sw128_desc(b_lo);
          // K = 16 per MMA: eight A columns, two 16-byte steps of B
#pragma unroll
          for (int s = 0; s < 4; ++s) mma_bf16_ta(d_tmem, a_tmem + 8u * s, dbh + 2 * s, idesc, s > 0);
#pragma unroll
          for (int s = 0; s < 4; ++s) mma_bf16_ta(d_tmem, a_tmem + 32u + 8u * s, dbh + 2 * s, idesc, 1);
#pragma unroll
          for (int s = 0; s < 4; ++s) mma_bf16_ta(d_tmem, a_tmem + 8u * s, dbl + 2 * s, idesc, 1);
          mma_commit(bar_mma(g));
          mma_commit(bar_oempty(sl));  // the slot is free once these MMAs have read it
        }
        // a following diagonal op, reduced to this column (computed while the MMAs run)
        uint32_t smask2 = 0;
        float2 cth2 = make_float2(1.f, 0.f);
        bool scal2 = false;
        column_chunks(s_chunks, act_sh[g], op.qc0, op.qc1, uint32_t(tg), s_terms, smask2, cth2, scal2);
        scal2 = __any_sync(0xffffffffu, scal2);
        const bool flip2 = __any_sync(0xffffffffu, smask2 != 0);
        // every thread waits for the accumulator itself (no group barrier: each warp reads its
        // lanes back as soon as the MMAs land).  A phase cannot be skipped: the next commit
        // needs every warp past the barrier after this read-back.  On a timeout the read-back
        // reads stale columns and the barrier below stops the group.
        if (!mbar_wait(bar_mma(g), mma_phase)) fail(2);
        mma_phase ^= 1u;
        tc_fence_after();
        // D columns 16h .. 16h+15 hold rows 8h .. 8h+7 as (real, imaginary) pairs
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          uint32_t v[16];
          NCSIM_TMEM_LD16(taddr + uint32_t(16 * h), v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (scal2) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const float2 c = cmulf(cth2, make_float2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1])));
              v[2 * i] = __float_as_uint(c.x);
              v[2 * i + 1] = __float_as_uint(c.y);
            }
          }
          if (flip2) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const uint32_t sg = (smask2 << (31 - (8 * h + i))) & 0x80000000u;
              v[2 * i] ^= sg;
              v[2 * i + 1] ^= sg;
            }
          }
#pragma unroll
          for (int i = 0; i < 8; ++i)
            T[lo8[i] ^ hi4[h]] = make_float2(__uint_as_float(v[2 * i]), __uint_as_float(v[2 * i + 1]));
        }
        tc_fence_before();
        if (bar_any(1 + g, GROUP_THREADS, abort_sh)) break;
      }
      if (bar_any(1 + g, GROUP_THREADS, abort_sh)) break;
      if (mine) {
        // the group writes its tile back; each thread's shared-memory reads are done once its
        // stores are issued, so the buffer is free for the next load after every thread arrives
        const float4* buf = reinterpret_cast<const float4*>(T);
#pragma unroll 4
        for (uint32_t c = uint32_t(tg); c < uint32_t(TILE) / 2; c += GROUP_THREADS)
          *reinterpret_cast<float4*>(chunk_addr(base, c)) = buf[at(2u * c) >> 1];
        mbar_arrive(bar_tdone(b));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// device copy of a plan: every pass's operand images in one buffer
struct DevicePlan {
  Plan plan;
  std::vector<PassParams> params;  // per pass, in segment order (amp/err filled per run)
  uint8_t* rops = nullptr;
  int device = -1;
  ~DevicePlan() {
    if (rops) cudaFree(rops);
  }
};

// which device table a term goes to (tile-local mask tm over the two 6-bit halves)
TermClass term_class(uint32_t tm, const CplxD& c) {
  const uint32_t lo = tm & ((1u << HALF) - 1), hi = tm >> HALF;
  if (hi == 0) return T_LOW;
  if (lo == 0) return T_HIGH;
  if (__builtin_popcount(lo) == 1 && __builtin_popcount(hi) == 1 && c.re == -1.0 && c.im == 0.0) return T_CROSS_SIGN;
  return T_GENERIC;
}

std::unique_ptr<DevicePlan> build_device_plan(const ncsim_circuit& c, uint32_t max_fuse, cudaStream_t stream) {
  auto dp = std::make_unique<DevicePlan>();
  dp->plan = make_plan(c, max_fuse);
  std::vector<uint8_t> images;
  std::vector<size_t> offsets;
  for (const Segment& s : dp->plan.segments) {
    if (!s.fused) continue;
    for (const Pass& ps : s.passes) {
      PassParams P{};
      P.ntiles = (uint64_t(1) << c.n) >> TILE_BITS;
      uint64_t wmask = 0;
      for (int j = 0; j < TILE_BITS; ++j) P.win[j] = uint8_t(ps.window[j]), wmask |= uint64_t(1) << ps.window[j];
      int wl = 0;
      while (wl < TILE_BITS && ps.window[wl] == uint32_t(wl)) ++wl;
      if (wl < LOW_BITS) throw Error(NCSIM_ERR_INVALID, "fused pass window lacks the low index bits");
      P.wl = wl;
      int nu = 0, nt = 0, no = 0;
      for (const FusedOp& op : ps.ops) {
        OpDesc d{};
        if (op.kind == 0) {
          if (nu >= MAX_UNITARIES) throw Error(NCSIM_ERR_INVALID, "fused pass has too many unitaries");
          d.kind = 0;
          d.u = uint8_t(nu);
          for (int j = 0; j < GROUP_QUBITS; ++j) {
            auto it = std::find(ps.window.begin(), ps.window.end(), op.qubits[j]);
            if (it == ps.window.end()) throw Error(NCSIM_ERR_INVALID, "fused unitary outside its window");
            P.pos[nu][j] = uint8_t(it - ps.window.begin());
          }
          const size_t at = images.size();
          images.resize(at + OPERAND_BYTES);
          build_operand_image(op.u, images.data() + at);
          offsets.push_back(at);
          ++nu;
        } else {
          d.kind = 1;
          if (nt + int(op.terms.size()) > MAX_TERMS) throw Error(NCSIM_ERR_INVALID, "fused pass has too many terms");
          std::vector<std::pair<int, TermDesc>> ts;
          for (const Term& t : op.terms) {
            TermDesc td{};
            uint32_t tm = 0;
            for (int j = 0; j < TILE_BITS; ++j)
              if ((t.mask >> ps.window[j]) & 1) tm |= 1u << j;
            td.tmask = tm;
            td.cmask = t.mask & ~wmask;
            td.cr = float(t.c.re);
            td.ci = float(t.c.im);
            ts.push_back({int(term_class(tm, t.c)), td});
          }
          std::stable_sort(ts.begin(), ts.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
          uint16_t bound[5];  // start of each class, then the end
          bound[0] = uint16_t(nt);
          int cls = 0;
          for (const auto& e : ts) {
            while (cls < e.first) bound[++cls] = uint16_t(nt);
            P.terms[nt++] = e.second;
          }
          while (cls < 4) bound[++cls] = uint16_t(nt);
          d.t0 = bound[0];
          d.tl = bound[1];
          d.th = bound[2];
          d.tc = bound[3];
          d.t1 = bound[4];
        }
        if (no >= MAX_OPS) throw Error(NCSIM_ERR_INVALID, "fused pass has too many ops");
        P.ops[no++] = d;
      }
      P.nops = no;
      P.nu = nu;
      // A terms op right before a unitary whose terms are, relative to that unitary's five
      // qubits, phases of the other bits or signs on one of its qubits is applied while the
      // unitary splits the tile (kind 2); one left after a unitary, by its read-back (kind 3).
      // Their terms go to the device as chunks of bit masks over 32 terms.
      static const uint32_t rowpat[GROUP_QUBITS] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
      int nch = 0;
      auto fold = [&](OpDesc& t, OpDesc& un, uint8_t kind) -> bool {
        uint32_t gm = 0;
        for (int j = 0; j < GROUP_QUBITS; ++j) gm |= 1u << P.pos[un.u][j];
        for (int k = t.t0; k < t.t1; ++k) {
          const TermDesc& td = P.terms[k];
          const uint32_t gpart = td.tmask & gm;
          if (!(gpart == 0 || (__builtin_popcount(gpart) == 1 && td.cr == -1.0f && td.ci == 0.0f))) return false;
        }
        const int need = (t.t1 - t.t0 + 31) / 32;
        if (nch + need > MAX_CHUNKS) return false;
        int colbit[TILE_BITS];  // tile bit -> column bit of this unitary (-1: a gate bit)
        for (int b = 0, m = 0; b < TILE_BITS; ++b) colbit[b] = ((gm >> b) & 1) ? -1 : m++;
        const uint8_t c0 = uint8_t(nch);
        for (int k0 = t.t0; k0 < t.t1; k0 += 32) {
          ColChunk ch{};
          ch.t0 = uint16_t(k0);
          ch.cnt = uint16_t(std::min(32, t.t1 - k0));
          for (int i = 0; i < ch.cnt; ++i) {
            TermDesc& td = P.terms[k0 + i];
            const uint32_t bit = 1u << i;
            const uint32_t gpart = td.tmask & gm;
            td.rowpat = 0;
            for (int j = 0; j < GROUP_QUBITS; ++j)
              if (gpart == (1u << P.pos[un.u][j])) td.rowpat = rowpat[j], ch.row[j] |= bit;
            td.tmask &= ~gm;
            for (int b = 0; b < TILE_BITS; ++b)
              if ((td.tmask >> b) & 1) ch.need[colbit[b]] |= bit;
            if (!td.rowpat) {
              if (td.cr == -1.0f && td.ci == 0.0f) ch.neg |= bit;
              else ch.gen |= bit;
            }
          }
          P.chunks[nch++] = ch;
        }
        t.kind = kind;
        if (kind == 2) un.pc0 = c0, un.pc1 = uint8_t(nch);
        else un.qc0 = c0, un.qc1 = uint8_t(nch);
        return true;
      };
      for (int i = 0; i + 1 < no; ++i)
        if (P.ops[i].kind == 1 && P.ops[i + 1].kind == 0) fold(P.ops[i], P.ops[i + 1], 2);
      for (int i = 1; i < no; ++i)
        if (P.ops[i].kind == 1 && P.ops[i - 1].kind == 0) fold(P.ops[i], P.ops[i - 1], 3);
      P.nchunks = nch;
      // the pass's first operand: an offset for now, a device pointer below
      P.rops = reinterpret_cast<const uint4*>(uintptr_t(nu ? offsets[offsets.size() - nu] : 0));
      dp->params.push_back(P);
    }
  }
  if (!images.empty()) {
    NCSIM_CUDA(cudaMalloc(&dp->rops, images.size()));
    // on the state's stream, waited for: a pageable cudaMemcpy may return before its DMA lands,
    // and the pass kernels' non-blocking stream does not wait for the legacy stream
    NCSIM_CUDA(cudaMemcpyAsync(dp->rops, images.data(), images.size(), cudaMemcpyHostToDevice, stream));
    NCSIM_CUDA(cudaStreamSynchronize(stream));
  }
  for (auto& P : dp->params) P.rops = reinterpret_cast<const uint4*>(dp->rops + uintptr_t(P.rops));
  NCSIM_CUDA(cudaGetDevice(&dp->device));
  return dp;
}

}  // namespace

}  // namespace fused

int apply_op(ncsim_state* s, const OpIR& op, ncsim_rng& rng);

}  // namespace ncsim

using namespace ncsim;

namespace {
std::mutex g_fused_mu;

// the circuit's device plan for this device and fusion width (built once)
std::shared_ptr<fused::DevicePlan> device_plan_for(const ncsim_circuit* c, uint32_t max_fuse, cudaStream_t stream) {
  std::lock_guard<std::mutex> lk(g_fused_mu);
  int dev = 0;
  NCSIM_CUDA(cudaGetDevice(&dev));
  if (c->fused_plan && c->fused_plan_fuse == max_fuse && c->fused_plan_device == dev)
    return std::static_pointer_cast<fused::DevicePlan>(c->fused_plan);
  std::shared_ptr<fused::DevicePlan> dp(fused::build_device_plan(*c, max_fuse, stream).release());
  c->fused_plan = dp;
  c->fused_plan_fuse = max_fuse;
  c->fused_plan_device = dev;
  return dp;
}
}  // namespace

extern "C" ncsim_status ncsim_sv_run_fused(ncsim_state* s, const ncsim_circuit* c, ncsim_rng* rng, uint32_t max_fuse,
                                           uint8_t* rec, size_t cap, size_t* len, ncsim_fused_stats* stats) {
  return guarded([&] {
    if (!s || !c || !rng) throw Error(NCSIM_ERR_INVALID, "null argument");
    if (s->precision != NCSIM_C64) throw Error(NCSIM_ERR_INVALID, "the fused form runs on complex64 states");
    if (c->n != s->n) throw Error(NCSIM_ERR_INVALID, "circuit on a different register");
    if (c->num_measurements() > cap) throw Error(NCSIM_ERR_INVALID, "record buffer too small");
    if (c->num_measurements()) {
      if (!rec) throw Error(NCSIM_ERR_INVALID, "record is null");
    }
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    std::shared_ptr<fused::DevicePlan> dp = device_plan_for(c, max_fuse ? max_fuse : 5, s->stream);
    int* d_err = s->dev_flag;  // the state's own word: no allocation per run
    NCSIM_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s->stream));
    NCSIM_CUDA(cudaFuncSetAttribute(fused::k_fused_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, fused::SM_DYNAMIC));
    const uint64_t sets = ((s->len >> fused::TILE_BITS) + fused::GROUPS - 1) / fused::GROUPS;  // a tile per warpgroup
    const unsigned grid = unsigned(std::min<uint64_t>(uint64_t(sm_count()), sets));
    size_t m = 0, pi = 0;
    uint64_t gemm = 0;
    for (const fused::Segment& seg : dp->plan.segments) {
      if (!seg.fused) {
        int r = apply_op(s, c->ops[seg.op], *rng);
        if (r >= 0) rec[m++] = uint8_t(r);
        continue;
      }
      for (size_t k = 0; k < seg.passes.size(); ++k, ++pi) {
        fused::PassParams P = dp->params[pi];
        P.amp = reinterpret_cast<float2*>(s->amp);
        P.err = d_err;
        ++gemm;  // one pass kernel launch
        ProfScope ps(s, K_FUSED_GEMM, 2.0 * double(s->bytes()));
        fused::k_fused_pass<<<grid, fused::THREADS, fused::SM_DYNAMIC, s->stream>>>(P);
        NCSIM_LAUNCHED("fused pass");
      }
    }
    int h_err = 0;
    NCSIM_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    if (h_err) throw Error(NCSIM_ERR_DEVICE, "fused pass stopped: a bounded wait timed out (code " + std::to_string(h_err) + ")");
    if (len) *len = m;
    if (stats) {
      stats->source_gates = dp->plan.source_gates;
      stats->fused_unitaries = dp->plan.unitaries;
      stats->passes = dp->plan.passes;
      stats->remap_passes = 0;
      stats->gemm_launches = gemm;
      stats->diagonal_terms = dp->plan.terms;
    }
  });
}

extern "C" ncsim_status ncsim_fused_emulate(const ncsim_circuit* c, uint32_t max_fuse, double* amps, uint64_t len,
                                            ncsim_fused_stats* stats) {
  return guarded([&] {
    if (!c) throw Error(NCSIM_ERR_INVALID, "null circuit");
    fused::Plan p = fused::make_plan(*c, max_fuse ? max_fuse : 5);
    if (amps) {  // without amplitudes: the plan's statistics only
      if (c->n > 22) throw Error(NCSIM_ERR_UNSUPPORTED, "emulation is for registers of at most 22 qubits");
      if (len != (uint64_t(1) << c->n)) throw Error(NCSIM_ERR_INVALID, "amplitude buffer length differs from 2^n");
      std::vector<CplxD> a(len);
      for (uint64_t i = 0; i < len; ++i) a[i] = {amps[2 * i], amps[2 * i + 1]};
      fused::emulate(p, *c, a);
      for (uint64_t i = 0; i < len; ++i) amps[2 * i] = a[i].re, amps[2 * i + 1] = a[i].im;
    }
    if (stats) {
      stats->source_gates = p.source_gates;
      stats->fused_unitaries = p.unitaries;
      stats->passes = p.passes;
      stats->remap_passes = 0;
      stats->gemm_launches = p.passes;
      stats->diagonal_terms = p.terms;
    }
  });
}
