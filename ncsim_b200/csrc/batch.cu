// Batching form, device side: the persistent trajectory kernel, the batch
// object (program upload, per-CTA state slots, CUDA graph replay) and its
// autotuner.
//
// Kernel: a persistent grid; each CTA takes the next trajectory from a work
// counter (largest registers first, by default) and runs all of its passes on
// its own state slot, then its measurements, so CTAs never wait on one another
// (no inter-CTA synchronisation at all).  A pass streams the state through
// shared memory in tiles of 8192 complex64 amplitudes (64 KB), loaded with
// cp.async (16-byte chunks, runs of 16 amplitudes = 128 B) and, in the
// double-buffered variant, prefetched one tile ahead; each stage moves the
// tile into registers (32 amplitudes per thread over five tile bits), applies
// its 2x2 gates, CZ sign masks and diagonals in FP32, and writes it back.
// The last pass (window = qubits 0..12) sums |a|^2 per tile index in FP64;
// the Z marginals of M 0 .. M m-1 come from those sums and from a gather of
// the 2^(n-13) amplitudes that match the low outcomes.
//
// Shared-memory layout of a tile: amplitude i at i ^ (((i >> 5) & 7) << 1),
// which keeps every 16-byte chunk whole and makes the three stage layouts,
// the chunk copies and the FP64 sums conflict-free.
#include <algorithm>
#include <array>
#include <mutex>
#include <atomic>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <cmath>
#include <map>
#include <numeric>
#include <thread>

#include <sys/stat.h>
#include <unistd.h>

#include "batch_plan.hpp"
#include "engine.cuh"

using namespace ncsim;
using namespace ncsim::batch;

namespace {

struct KParams {
  const DevTraj* traj;
  const DevPass* pass;
  const DevStage* stage;
  const DevOp* op;
  const double* draws;
  const uint32_t* order;
  uint32_t count;
  uint32_t max_n;
  float2* slots;
  uint64_t slot_elems;
  double* gscratch;  // TILE doubles per CTA (single-buffered variant)
  uint32_t* queue;
  uint64_t* out_rec;
  double* out_z0;
  double* out_norm;
  uint32_t* err;
};

__device__ __forceinline__ uint32_t spos(uint32_t i) { return i ^ (((i >> 5) & 7u) << 1); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = uint32_t(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int R>
__device__ __forceinline__ uint32_t fixed_index(uint32_t tid) {
  if (R == 0) return tid << 5;
  if (R == 1) return (tid & 31u) | ((tid >> 5) << 10);
  return tid;
}

// A thread's 32 amplitudes, interleaved (re, im), over the stage's five tile bits.
struct Regs {
  float2 a[32];
};

template <int R>
__device__ __forceinline__ void load_stage(const float2* buf, uint32_t tid, Regs& r) {
  if (R == 0) {
    const float4* b4 = reinterpret_cast<const float4*>(buf) + (tid << 4);
    const uint32_t x = tid & 7u;
#pragma unroll
    for (uint32_t m = 0; m < 16; ++m) {
      const float4 v = b4[m ^ x];
      r.a[2 * m] = make_float2(v.x, v.y);
      r.a[2 * m + 1] = make_float2(v.z, v.w);
    }
  } else if (R == 1) {
    const uint32_t f = fixed_index<1>(tid);
#pragma unroll
    for (uint32_t j = 0; j < 32; ++j) r.a[j] = buf[(f ^ ((j & 7u) << 1)) + (j << 5)];
  } else {
    const uint32_t f = tid ^ (((tid >> 5) & 7u) << 1);
#pragma unroll
    for (uint32_t j = 0; j < 32; ++j) r.a[j] = buf[f + (j << 8)];
  }
}

template <int R>
__device__ __forceinline__ void store_stage(float2* buf, uint32_t tid, const Regs& r) {
  if (R == 0) {
    float4* b4 = reinterpret_cast<float4*>(buf) + (tid << 4);
    const uint32_t x = tid & 7u;
#pragma unroll
    for (uint32_t m = 0; m < 16; ++m)
      b4[m ^ x] = make_float4(r.a[2 * m].x, r.a[2 * m].y, r.a[2 * m + 1].x, r.a[2 * m + 1].y);
  } else if (R == 1) {
    const uint32_t f = fixed_index<1>(tid);
#pragma unroll
    for (uint32_t j = 0; j < 32; ++j) buf[(f ^ ((j & 7u) << 1)) + (j << 5)] = r.a[j];
  } else {
    const uint32_t f = tid ^ (((tid >> 5) & 7u) << 1);
#pragma unroll
    for (uint32_t j = 0; j < 32; ++j) buf[f + (j << 8)] = r.a[j];
  }
}

// mask over j = 0..31 of the amplitudes whose register bit k is 1
__device__ __forceinline__ uint32_t reg_pattern(uint32_t k) {
  switch (k) {
    case 0: return 0xAAAAAAAAu;
    case 1: return 0xCCCCCCCCu;
    case 2: return 0xF0F0F0F0u;
    case 3: return 0xFF00FF00u;
    default: return 0xFFFF0000u;
  }
}

// 32-bit mask over the thread's amplitudes j whose bit of the located qubit is 1
__device__ __forceinline__ uint32_t loc_mask(uint32_t loc, uint32_t fixed, uint32_t tile) {
  const uint32_t type = loc >> 5, idx = loc & 31u;
  if (type == LOC_REG) return reg_pattern(idx);
  const uint32_t bit = ((type == LOC_FIXED ? fixed : tile) >> idx) & 1u;
  return 0u - bit;
}

// the sign bit (as a float bit mask) of bit j of m
__device__ __forceinline__ uint32_t sgn(uint32_t m, int j) { return (m << (31 - j)) & 0x80000000u; }
__device__ __forceinline__ float flip(float v, uint32_t s) { return __uint_as_float(__float_as_uint(v) ^ s); }

// The gate updates below are written so that every output's last operation
// consumes the last use of an input it replaces (cross products first, into
// temporaries): the outputs can take their inputs' registers, and the op
// loop, whose switch cases must all leave the 32 amplitudes in the same
// registers, needs no copies back.

// 2x2 gate on register bit K: u0 = (u00, u01), u1 = (u10, u11) as (re, im).
// REL: the second amplitude of pair j is negated first where bit j of rel is set.
template <int K, bool REL>
__device__ __forceinline__ void gate_k(Regs& r, const float4 u0, const float4 u1, uint32_t rel) {
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j & (1 << K)) continue;
    float xr = r.a[j].x, xi = r.a[j].y, yr = r.a[j + (1 << K)].x, yi = r.a[j + (1 << K)].y;
    if (REL) {
      const uint32_t sg = sgn(rel, j);
      yr = flip(yr, sg);
      yi = flip(yi, sg);
    }
    // u10 x (kept for the second row), then u00 x in place of x
    float ar = fmaf(u1.x, xr, -(u1.y * xi)), ai = fmaf(u1.x, xi, u1.y * xr);
    const float p = u0.y * xi, q = u0.y * xr;
    xr = fmaf(u0.x, xr, -p);
    xi = fmaf(u0.x, xi, q);
    // + u01 y (y still needed below)
    xr = fmaf(u0.z, yr, fmaf(-u0.w, yi, xr));
    xi = fmaf(u0.z, yi, fmaf(u0.w, yr, xi));
    // u10 x + u11 y in place of y
    ar = fmaf(-u1.w, yi, ar);
    ai = fmaf(u1.w, yr, ai);
    yr = fmaf(u1.z, yr, ar);
    yi = fmaf(u1.z, yi, ai);
    r.a[j] = make_float2(xr, xi);
    r.a[j + (1 << K)] = make_float2(yr, yi);
  }
}

// balanced gate s [[1, w], [1, -w]] on register bit K: c = (s w.re, s w.im, s)
// (the first output as 2 s x - (s x - s w y): one extra FP32 rounding)
template <int K, bool REL>
__device__ __forceinline__ void bgate_k(Regs& r, const float4 c, uint32_t rel) {
  const float c2 = 2.0f * c.z;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j & (1 << K)) continue;
    float xr = r.a[j].x, xi = r.a[j].y, yr = r.a[j + (1 << K)].x, yi = r.a[j + (1 << K)].y;
    const float p = c.y * yi, q = c.y * yr;
    yr = fmaf(c.x, yr, -p);  // s w y, in place of y
    yi = fmaf(c.x, yi, q);
    if (REL) {
      const uint32_t sg = sgn(rel, j);
      yr = flip(yr, sg);
      yi = flip(yi, sg);
    }
    yr = fmaf(c.z, xr, -yr);  // s x - s w y
    yi = fmaf(c.z, xi, -yi);
    xr = fmaf(c2, xr, -yr);   // s x + s w y
    xi = fmaf(c2, xi, -yi);
    r.a[j] = make_float2(xr, xi);
    r.a[j + (1 << K)] = make_float2(yr, yi);
  }
}

template <int K>
__device__ __forceinline__ void any_gate(Regs& r, bool bal, float4 u0, float4 u1, uint32_t rel) {
  // a relative sign on every pair is a sign on the gate's second column
  if (rel == ~reg_pattern(K)) {
    if (bal) {
      u0.x = -u0.x;
      u0.y = -u0.y;
    } else {
      u0.z = -u0.z;
      u0.w = -u0.w;
      u1.z = -u1.z;
      u1.w = -u1.w;
    }
    rel = 0;
  }
  if (bal) {
    if (rel) bgate_k<K, true>(r, u0, rel);
    else bgate_k<K, false>(r, u0, 0);
  } else {
    if (rel) gate_k<K, true>(r, u0, u1, rel);
    else gate_k<K, false>(r, u0, u1, 0);
  }
}

// negate the amplitudes j with bit j of neg set (the pending CZ signs)
__device__ __forceinline__ void flush_neg(Regs& r, uint32_t neg) {
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const uint32_t sg = sgn(neg, j);
    r.a[j] = make_float2(flip(r.a[j].x, sg), flip(r.a[j].y, sg));
  }
}

// amplitude j *= (bit j of m ? d1 : d0)
__device__ __forceinline__ void diag_mask(Regs& r, uint32_t m, float2 d0, float2 d1) {
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const bool b = (m >> j) & 1u;
    const float dr = b ? d1.x : d0.x, di = b ? d1.y : d0.y;
    const float2 v = r.a[j];
    const float p = v.y * di, q = v.x * di;
    r.a[j] = make_float2(fmaf(v.x, dr, -p), fmaf(v.y, dr, q));
  }
}

// The ops of one stage on the registers (shared by the three layouts).  CZ
// signs stay pending as a mask over the 32 amplitudes until a gate absorbs
// them: the sign common to both amplitudes of a pair stays pending, the
// relative one is applied inside the gate; diagonals commute with the mask.
__device__ __forceinline__ void apply_ops(Regs& r, uint32_t fixed, uint32_t tile, const DevOp* ops, uint32_t nops) {
  uint32_t neg = 0;
  for (uint32_t o = 0; o < nops; ++o) {
    const DevOp* op = ops + o;
    const uint32_t hdr = op->hdr;
    const uint32_t code = hdr & 7u, la = (hdr >> 3) & 127u, lb = (hdr >> 10) & 127u;
    if (code == OP_CZ) {
      // the register operands' patterns come multiplied; a fixed or tile operand's bit masks them
      uint32_t m = __float_as_uint(op->v[0]);
      if ((la >> 5) != LOC_REG) m &= 0u - ((((la >> 5) == LOC_FIXED ? fixed : tile) >> (la & 31u)) & 1u);
      if ((lb >> 5) != LOC_REG) m &= 0u - ((((lb >> 5) == LOC_FIXED ? fixed : tile) >> (lb & 31u)) & 1u);
      neg ^= m;
      continue;
    }
    const float4 u0 = reinterpret_cast<const float4*>(op->v)[0];
    const float4 u1 = reinterpret_cast<const float4*>(op->v)[1];
    if (code == OP_GATE || code == OP_BGATE) {
      const uint32_t k = la & 31u, sh = 1u << k, lo = ~reg_pattern(k);
      const uint32_t rel = (neg ^ (neg >> sh)) & lo;
      const uint32_t common = neg & lo;
      neg = common | (common << sh);
      const bool bal = code == OP_BGATE;
      switch (k) {
        case 0: any_gate<0>(r, bal, u0, u1, rel); break;
        case 1: any_gate<1>(r, bal, u0, u1, rel); break;
        case 2: any_gate<2>(r, bal, u0, u1, rel); break;
        case 3: any_gate<3>(r, bal, u0, u1, rel); break;
        default: any_gate<4>(r, bal, u0, u1, rel); break;
      }
    } else if (code == OP_DIAG) {
      diag_mask(r, loc_mask(la, fixed, tile), make_float2(u0.x, u0.y), make_float2(u0.z, u0.w));
    } else {
      diag_mask(r, loc_mask(la, fixed, tile) & loc_mask(lb, fixed, tile), make_float2(1.f, 0.f),
                make_float2(u0.x, u0.y));
    }
  }
  if (neg) flush_neg(r, neg);
}

__device__ __forceinline__ void load_tile(float2* buf, const float2* st, uint32_t base, const uint32_t* off_lo,
                                          const uint32_t* off_hi, uint32_t tid) {
#pragma unroll 4
  for (uint32_t r = 0; r < TILE / 2 / THREADS; ++r) {
    const uint32_t i = 2u * (tid + THREADS * r);
    cp_async16(buf + spos(i), st + (base + off_lo[i & 127u] + off_hi[i >> 7]));
  }
}

__device__ __forceinline__ void zero_tile(float2* buf, uint32_t tid, bool first) {
  float4* b4 = reinterpret_cast<float4*>(buf);
#pragma unroll 4
  for (uint32_t r = 0; r < TILE / 2 / THREADS; ++r) {
    const uint32_t i = 2u * (tid + THREADS * r);
    b4[spos(i) >> 1] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (first && tid == 0) buf[0] = make_float2(1.f, 0.f);  // chunk 0 is thread 0's
}

// block-wide FP64 sums of two values in a fixed order; thread 0 gets them
__device__ __forceinline__ void block_sum2(double& s0, double& s1, double (*red)[2], uint32_t tid) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, d);
    s1 += __shfl_xor_sync(0xffffffffu, s1, d);
  }
  if ((tid & 31u) == 0) {
    red[tid >> 5][0] = s0;
    red[tid >> 5][1] = s1;
  }
  __syncthreads();
  if (tid == 0) {
    s0 = red[0][0];
    s1 = red[0][1];
    for (uint32_t w = 1; w < THREADS / 32; ++w) {
      s0 += red[w][0];
      s1 += red[w][1];
    }
  }
}

// QuantumState::measure's decision (src/state/mod.rs:113-131)
__device__ __forceinline__ uint32_t decide(double e, double nn, const double* draws, uint32_t& used) {
  double p = (1.0 + e / nn) / 2.0;
  if (!isnan(p)) p = fmin(1.0, fmax(0.0, p));
  if (p > 1.0 - 1e-12) return 0;
  if (p < 1e-12) return 1;
  return draws[used++] >= p ? 1u : 0u;
}

template <int NBUF>
__global__ void __launch_bounds__(THREADS, NBUF == 2 ? 1 : 2) k_batch(const __grid_constant__ KParams P) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  __shared__ uint32_t off_lo[128], off_hi[64];
  __shared__ DevPass sp;
  __shared__ DevOp s_ops[MAX_PASS_OPS];
  __shared__ uint2 s_stage[MAX_PASS_OPS];
  __shared__ double red[THREADS / 32][2];
  __shared__ uint32_t s_job, s_bit;
  __shared__ DevTraj s_tr;  // the job's descriptor, read where needed (frees registers in the stage loop)
  float2* bufs = reinterpret_cast<float2*>(dsm);
  double* T = NBUF == 2 ? reinterpret_cast<double*>(bufs + 2 * TILE) : P.gscratch + size_t(blockIdx.x) * TILE;
  double* G = NBUF == 2 ? T : reinterpret_cast<double*>(bufs);
  const uint32_t tid = threadIdx.x;
  float2* st = P.slots + size_t(blockIdx.x) * P.slot_elems;

  for (;;) {
    if (tid == 0) s_job = atomicAdd(P.queue, 1u);
    __syncthreads();
    const uint32_t job = s_job;
    __syncthreads();
    if (job >= P.count) break;
    const uint32_t t = P.order[job];
    if (tid == 0) s_tr = P.traj[t];
    __syncthreads();
    const DevTraj& tr = s_tr;
    if (tr.n < MIN_QUBITS || tr.n > P.max_n || tr.nmeas > tr.n) {
      if (tid == 0) atomicOr(P.err, 1u);
      continue;
    }
    const uint32_t ntiles = 1u << (tr.n - TILE_BITS);
    for (uint32_t pi = 0; pi < tr.npass; ++pi) {
      if (tid < sizeof(DevPass) / 4)
        reinterpret_cast<uint32_t*>(&sp)[tid] = reinterpret_cast<const uint32_t*>(P.pass + tr.pass0 + pi)[tid];
      __syncthreads();
      if (tid < 128) {
        uint32_t v = 0;
        for (uint32_t b = 0; b < 7; ++b)
          if ((tid >> b) & 1u) v += 1u << sp.win[b];
        off_lo[tid] = v;
      } else if (tid < 192) {
        const uint32_t i = tid - 128;
        uint32_t v = 0;
        for (uint32_t b = 0; b < 6; ++b)
          if ((i >> b) & 1u) v += 1u << sp.win[7 + b];
        off_hi[i] = v;
      }
      const bool zero = sp.flags & PASS_ZERO_INIT, accum = sp.flags & PASS_ACCUM,
                 write = !(sp.flags & PASS_NO_WRITE);
      // the pass's stages and ops (contiguous, at most MAX_PASS_OPS) into shared memory
      const uint32_t nstage = min(uint32_t(sp.nstage), MAX_PASS_OPS);
      uint32_t op_first = 0, op_count = 0;
      if (nstage) {
        const DevStage first = P.stage[sp.stage0], last = P.stage[sp.stage0 + nstage - 1];
        op_first = first.op0;
        op_count = min(last.op0 + (last.info >> 2) - op_first, MAX_PASS_OPS);
      }
      for (uint32_t i = tid; i < nstage; i += THREADS) {
        const DevStage d = P.stage[sp.stage0 + i];
        s_stage[i] = make_uint2(d.info, d.op0 - op_first);
      }
      for (uint32_t i = tid; i < op_count * 3; i += THREADS)
        reinterpret_cast<uint4*>(s_ops)[i] = reinterpret_cast<const uint4*>(P.op + op_first)[i];
      if (accum) {
#pragma unroll 4
        for (uint32_t r = 0; r < TILE / 2 / THREADS; ++r) {
          const uint32_t i = 2u * (tid + THREADS * r);
          *reinterpret_cast<double2*>(T + spos(i)) = make_double2(0.0, 0.0);
        }
      }
      __syncthreads();
      auto base_of = [&](uint32_t k) {
        uint32_t b = 0;
        for (uint32_t i = 0; i < sp.nnon; ++i)
          if ((k >> i) & 1u) b += 1u << sp.non[i];
        return b;
      };
      if (NBUF == 2 && !zero) {
        load_tile(bufs, st, base_of(0), off_lo, off_hi, tid);
        cp_async_commit();
      }
      for (uint32_t k = 0; k < ntiles; ++k) {
        float2* cur = bufs + (NBUF == 2 ? (k & 1u) * TILE : 0u);
        const uint32_t base = base_of(k);
        if (zero) {
          zero_tile(cur, tid, k == 0);
        } else if (NBUF == 2) {
          if (k + 1 < ntiles) {
            load_tile(bufs + ((k + 1) & 1u) * TILE, st, base_of(k + 1), off_lo, off_hi, tid);
            cp_async_commit();
            cp_async_wait<1>();
          } else {
            cp_async_wait<0>();
          }
        } else {
          load_tile(cur, st, base, off_lo, off_hi, tid);
          cp_async_commit();
          cp_async_wait<0>();
        }
        __syncthreads();
        for (uint32_t s = 0; s < nstage; ++s) {
          const uint2 d = s_stage[s];
          const uint32_t r = d.x & 3u;
          const uint32_t nops = min(d.x >> 2, op_count - min(d.y, op_count));
          Regs regs;
          if (r == 0) load_stage<0>(cur, tid, regs);
          else if (r == 1) load_stage<1>(cur, tid, regs);
          else load_stage<2>(cur, tid, regs);
          const uint32_t fixed = r == 0 ? fixed_index<0>(tid) : r == 1 ? fixed_index<1>(tid) : fixed_index<2>(tid);
          apply_ops(regs, fixed, k, s_ops + d.y, nops);
          if (r == 0) store_stage<0>(cur, tid, regs);
          else if (r == 1) store_stage<1>(cur, tid, regs);
          else store_stage<2>(cur, tid, regs);
          __syncthreads();
        }
        if (!(sp.flags & PASS_NO_WRITE) || (sp.flags & PASS_ACCUM)) {
          const bool write = !(sp.flags & PASS_NO_WRITE), accum = sp.flags & PASS_ACCUM;
          const uint32_t base = base_of(k);
#pragma unroll 4
          for (uint32_t r = 0; r < TILE / 2 / THREADS; ++r) {
            const uint32_t i = 2u * (tid + THREADS * r);
            const float4 v = *reinterpret_cast<const float4*>(cur + spos(i));
            if (write) *reinterpret_cast<float4*>(st + (base + off_lo[i & 127u] + off_hi[i >> 7])) = v;
            if (accum) {
              double2* tp = reinterpret_cast<double2*>(T + spos(i));
              double2 tv = *tp;
              tv.x += double(v.x) * double(v.x) + double(v.y) * double(v.y);
              tv.y += double(v.z) * double(v.z) + double(v.w) * double(v.w);
              *tp = tv;
            }
          }
        }
        __syncthreads();
      }
      __threadfence();
      __syncthreads();
    }

    // measurements M 0 .. M m-1 from the FP64 sums
    const double* draws = P.draws + tr.draw0;
    uint32_t used = 0;  // meaningful in thread 0
    uint32_t o = 0;
    double z0 = 0.0, norm = 0.0;
    const uint32_t kl = min(tr.nmeas, TILE_BITS);
    for (uint32_t k = 0; k < max(kl, 1u); ++k) {
      double s0 = 0.0, s1 = 0.0;
      const uint32_t cnt = TILE >> k;
      for (uint32_t r = tid; r < cnt; r += THREADS) {
        const double v = T[spos(o | (r << k))];
        if (r & 1u) s1 += v;
        else s0 += v;
      }
      block_sum2(s0, s1, red, tid);
      if (tid == 0) {
        const double e = s0 - s1, nn = s0 + s1;
        if (k == 0) {
          z0 = e / nn;
          norm = nn;
        }
        s_bit = k < tr.nmeas ? decide(e, nn, draws, used) : 0u;
      }
      __syncthreads();
      o |= s_bit << k;
      __syncthreads();
    }
    uint64_t rec = o;
    if (tr.nmeas > TILE_BITS) {
      const uint32_t nh = ntiles;
      for (uint32_t h = tid; h < nh; h += THREADS) {
        const float2 v = st[o | (h << TILE_BITS)];
        G[h] = double(v.x) * double(v.x) + double(v.y) * double(v.y);
      }
      __syncthreads();
      uint32_t oh = 0;
      for (uint32_t k = TILE_BITS; k < tr.nmeas; ++k) {
        const uint32_t kk = k - TILE_BITS;
        double s0 = 0.0, s1 = 0.0;
        for (uint32_t r = tid; r < (nh >> kk); r += THREADS) {
          const double v = G[oh | (r << kk)];
          if (r & 1u) s1 += v;
          else s0 += v;
        }
        block_sum2(s0, s1, red, tid);
        if (tid == 0) s_bit = decide(s0 - s1, s0 + s1, draws, used);
        __syncthreads();
        oh |= s_bit << kk;
        __syncthreads();
      }
      rec |= uint64_t(oh) << TILE_BITS;
    }
    if (tid == 0) {
      P.out_rec[t] = rec;
      P.out_z0[t] = z0;
      P.out_norm[t] = norm;
    }
  }
}

constexpr size_t SMEM_NBUF2 = 3 * TILE * 8;  // two tiles and the FP64 sums
constexpr size_t SMEM_NBUF1 = TILE * 8;

}  // namespace

// ---------------------------------------------------------------------------
// device buffers of freed batches, kept for the next batch on the same device:
// a batch's trajectory states take up to tens of GB, and allocating and
// freeing them cost the driver tens to hundreds of milliseconds per batch.  At
// most four buffers per device are kept; they are released when an allocation
// runs out of memory (and the allocation is retried), else at process exit.
// ---------------------------------------------------------------------------
namespace {
struct CachedBuf {
  int dev;
  size_t bytes;
  void* p;
};
std::mutex g_buf_mu;
std::vector<CachedBuf> g_bufs;
constexpr size_t BUFS_PER_DEVICE = 4;

// a device buffer of at least `bytes` (its capacity in *cap)
void* buf_alloc(size_t bytes, size_t* cap) {
  int dev = 0;
  NCSIM_CUDA(cudaGetDevice(&dev));
  bytes = std::max<size_t>(bytes, 256);
  {
    std::lock_guard<std::mutex> lk(g_buf_mu);
    size_t best = g_bufs.size();
    for (size_t i = 0; i < g_bufs.size(); ++i) {
      const CachedBuf& c = g_bufs[i];
      if (c.dev != dev || c.bytes < bytes || c.bytes > 2 * bytes + (size_t(64) << 20)) continue;
      if (best == g_bufs.size() || c.bytes < g_bufs[best].bytes) best = i;
    }
    if (best < g_bufs.size()) {
      void* p = g_bufs[best].p;
      *cap = g_bufs[best].bytes;
      g_bufs.erase(g_bufs.begin() + long(best));
      return p;
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e == cudaErrorMemoryAllocation) {  // give the kept buffers of this device back and retry
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(g_buf_mu);
    for (size_t i = 0; i < g_bufs.size();) {
      if (g_bufs[i].dev == dev) {
        cudaFree(g_bufs[i].p);
        g_bufs.erase(g_bufs.begin() + long(i));
      } else {
        ++i;
      }
    }
    e = cudaMalloc(&p, bytes);
  }
  NCSIM_CUDA(e);
  *cap = bytes;
  return p;
}

// returns an idle buffer (its work finished) for reuse on the current device
void buf_free(void* p, size_t cap) {
  if (!p) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(p);
    return;
  }
  std::lock_guard<std::mutex> lk(g_buf_mu);
  g_bufs.push_back({dev, cap, p});
  size_t kept = 0;
  for (const CachedBuf& c : g_bufs) kept += c.dev == dev;
  if (kept > BUFS_PER_DEVICE) {  // drop the oldest of this device
    for (size_t i = 0; i < g_bufs.size(); ++i)
      if (g_bufs[i].dev == dev) {
        cudaFree(g_bufs[i].p);
        g_bufs.erase(g_bufs.begin() + long(i));
        break;
      }
  }
}
}  // namespace

// ---------------------------------------------------------------------------
// the batch object
// ---------------------------------------------------------------------------
struct ncsim_batch {
  Program prog;
  // the folded trajectories, kept until the planner's knobs are final (the
  // autotuner recompiles the program with other knobs), then dropped
  std::vector<Trajectory> ts;
  std::vector<PlanKnobs> knobs_by_n = std::vector<PlanKnobs>(MAX_QUBITS + 1);
  std::vector<int> knob_set_by_n = std::vector<int>(MAX_QUBITS + 1, 0);
  std::vector<std::array<double, NUM_KNOB_SETS>> knob_ms =
      std::vector<std::array<double, NUM_KNOB_SETS>>(MAX_QUBITS + 1);  // timed per size class and knob set
  bool knobs_final = false;
  std::vector<uint32_t> order_lpt, order_seq;
  std::mutex mu;
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  char* d_prog = nullptr;
  size_t off_traj = 0, off_pass = 0, off_stage = 0, off_op = 0, off_draws = 0, off_lpt = 0, off_seq = 0,
         off_sample = 0;
  uint32_t* d_queue = nullptr;  // [0] work counter, [1] error flags
  uint64_t* d_rec = nullptr;
  double* d_z0 = nullptr;
  double* d_norm = nullptr;
  float2* d_slots = nullptr;
  double* d_scratch = nullptr;
  size_t prog_cap = 0, slots_cap = 0, scratch_cap = 0;  // capacities of the kept-buffer allocations
  uint32_t slot_ctas = 0;
  uint64_t* h_rec = nullptr;
  double* h_z0 = nullptr;
  double* h_norm = nullptr;
  uint32_t* h_err = nullptr;
  ncsim_batch_config cfg{0, 0, 0};  // unset until tuned or set
  cudaGraphExec_t graph = nullptr;
  ncsim_batch_config graph_cfg{0, 0, 0};
  uint32_t sample_count = 0;
  bool have_results = false;
  double last_ms = 0.0;

  ~ncsim_batch() { release(); }
  // Frees every device and pinned resource on the batch's device and leaves
  // the object as if it had never run (all pointers null, all capacities 0),
  // so the next run sets everything up again on the then-current device.  The
  // calling thread's current device is restored.
  void release() {
    if (device < 0) return;
    int caller = -1;
    if (cudaGetDevice(&caller) != cudaSuccess) caller = -1;
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamSynchronize(stream);
    buf_free(d_prog, prog_cap);
    cudaFree(d_queue);
    cudaFree(d_rec);
    cudaFree(d_z0);
    cudaFree(d_norm);
    buf_free(d_slots, slots_cap);
    buf_free(d_scratch, scratch_cap);
    d_prog = nullptr;
    d_queue = nullptr;
    d_rec = nullptr;
    d_z0 = nullptr;
    d_norm = nullptr;
    d_slots = nullptr;
    d_scratch = nullptr;
    prog_cap = slots_cap = scratch_cap = 0;
    slot_ctas = 0;
    cudaFreeHost(h_rec);
    cudaFreeHost(h_z0);
    cudaFreeHost(h_norm);
    cudaFreeHost(h_err);
    h_rec = nullptr;
    h_z0 = nullptr;
    h_norm = nullptr;
    h_err = nullptr;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
    ev0 = ev1 = nullptr;
    stream = nullptr;
    graph = nullptr;
    have_results = false;
    device = -1;
    cudaGetLastError();
    if (caller >= 0) cudaSetDevice(caller);
  }
  uint32_t count() const { return uint32_t(prog.traj.size()); }
};

namespace {

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

template <class T>
T* dev_ptr(ncsim_batch* b, size_t off) {
  return reinterpret_cast<T*>(b->d_prog + off);
}

// (Re)uploads the program and the trajectory orders to the device (the
// batch's device must be current).  A captured graph holds the old pointers.
void upload_program(ncsim_batch* b) {
  if (b->graph) {
    NCSIM_CUDA(cudaStreamSynchronize(b->stream));
    NCSIM_CUDA(cudaGraphExecDestroy(b->graph));
    b->graph = nullptr;
  }
  if (b->d_prog) {
    NCSIM_CUDA(cudaStreamSynchronize(b->stream));
    buf_free(b->d_prog, b->prog_cap);
    b->d_prog = nullptr;
    b->prog_cap = 0;
  }
  const Program& P = b->prog;
  const uint32_t c = b->count();
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  b->off_traj = take(P.traj.size() * sizeof(DevTraj));
  b->off_pass = take(P.pass.size() * sizeof(DevPass));
  b->off_stage = take(P.stage.size() * sizeof(DevStage));
  b->off_op = take(std::max<size_t>(1, P.op.size()) * sizeof(DevOp));
  b->off_draws = take(std::max<size_t>(1, P.draws.size()) * sizeof(double));
  b->off_lpt = take(size_t(c) * 4);
  b->off_seq = take(size_t(c) * 4);
  b->off_sample = take(size_t(c) * 4);
  b->d_prog = static_cast<char*>(buf_alloc(off, &b->prog_cap));
  auto up = [&](size_t o, const void* src, size_t bytes) {
    if (bytes) NCSIM_CUDA(cudaMemcpyAsync(b->d_prog + o, src, bytes, cudaMemcpyHostToDevice, b->stream));
  };
  up(b->off_traj, P.traj.data(), P.traj.size() * sizeof(DevTraj));
  up(b->off_pass, P.pass.data(), P.pass.size() * sizeof(DevPass));
  up(b->off_stage, P.stage.data(), P.stage.size() * sizeof(DevStage));
  up(b->off_op, P.op.data(), P.op.size() * sizeof(DevOp));
  up(b->off_draws, P.draws.data(), P.draws.size() * sizeof(double));
  up(b->off_lpt, b->order_lpt.data(), size_t(c) * 4);
  up(b->off_seq, b->order_seq.data(), size_t(c) * 4);
  NCSIM_CUDA(cudaStreamSynchronize(b->stream));
}

void ensure_device(ncsim_batch* b) {
  int dev = 0;
  NCSIM_CUDA(cudaGetDevice(&dev));
  if (b->device == dev) return;
  if (b->device >= 0) b->release();  // on its old device; the caller's device stays current
  b->device = dev;
  NCSIM_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  NCSIM_CUDA(cudaEventCreate(&b->ev0));
  NCSIM_CUDA(cudaEventCreate(&b->ev1));
  const uint32_t c = b->count();
  upload_program(b);
  NCSIM_CUDA(cudaMalloc(&b->d_queue, 2 * sizeof(uint32_t)));
  NCSIM_CUDA(cudaMalloc(&b->d_rec, size_t(c) * 8));
  NCSIM_CUDA(cudaMalloc(&b->d_z0, size_t(c) * 8));
  NCSIM_CUDA(cudaMalloc(&b->d_norm, size_t(c) * 8));
  NCSIM_CUDA(cudaMallocHost(&b->h_rec, size_t(c) * 8));
  NCSIM_CUDA(cudaMallocHost(&b->h_z0, size_t(c) * 8));
  NCSIM_CUDA(cudaMallocHost(&b->h_norm, size_t(c) * 8));
  NCSIM_CUDA(cudaMallocHost(&b->h_err, sizeof(uint32_t)));
  static std::mutex attr_mu;  // batches on several host threads may race here
  static bool attr_done[64] = {};
  std::lock_guard<std::mutex> lk(attr_mu);
  if (dev < 0 || dev >= 64 || !attr_done[dev]) {
    NCSIM_CUDA(cudaFuncSetAttribute(k_batch<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_NBUF2)));
    NCSIM_CUDA(cudaFuncSetAttribute(k_batch<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_NBUF1)));
    if (dev >= 0 && dev < 64) attr_done[dev] = true;
  }
}

uint32_t grid_for(const ncsim_batch_config& cfg) {
  return uint32_t(sm_count()) * std::max<uint32_t>(1, cfg.ctas_per_sm);
}

void ensure_slots(ncsim_batch* b, uint32_t ctas) {
  if (b->slot_ctas >= ctas && b->d_slots && b->d_scratch) return;
  NCSIM_CUDA(cudaStreamSynchronize(b->stream));
  if (b->graph) {  // the captured launch holds the old slot pointers
    NCSIM_CUDA(cudaGraphExecDestroy(b->graph));
    b->graph = nullptr;
  }
  buf_free(b->d_slots, b->slots_cap);
  buf_free(b->d_scratch, b->scratch_cap);
  b->d_slots = nullptr;
  b->d_scratch = nullptr;
  b->slot_ctas = 0;
  const size_t elems = size_t(1) << b->prog.max_n;
  b->d_slots = static_cast<float2*>(buf_alloc(size_t(ctas) * elems * sizeof(float2), &b->slots_cap));
  b->d_scratch = static_cast<double*>(buf_alloc(size_t(ctas) * TILE * sizeof(double), &b->scratch_cap));
  b->slot_ctas = ctas;
}

// every device buffer a launch reads or writes must exist (a batch released
// from its device is set up again by ensure_device/ensure_slots before this)
void check_launch_buffers(const ncsim_batch* b) {
  if (!b->d_prog || !b->d_queue || !b->d_rec || !b->d_z0 || !b->d_norm || !b->d_slots || !b->d_scratch || !b->stream)
    throw Error(NCSIM_ERR_DEVICE, "batch launch without its device buffers (released and not set up again)");
}

// one launch of the kernel over `count` jobs of the order array at order_off
void enqueue_kernel(ncsim_batch* b, const ncsim_batch_config& cfg, size_t order_off, uint32_t count) {
  check_launch_buffers(b);
  KParams k{};
  k.traj = dev_ptr<DevTraj>(b, b->off_traj);
  k.pass = dev_ptr<DevPass>(b, b->off_pass);
  k.stage = dev_ptr<DevStage>(b, b->off_stage);
  k.op = dev_ptr<DevOp>(b, b->off_op);
  k.draws = dev_ptr<double>(b, b->off_draws);
  k.order = dev_ptr<uint32_t>(b, order_off);
  k.count = count;
  k.max_n = b->prog.max_n;
  k.slots = b->d_slots;
  k.slot_elems = uint64_t(1) << b->prog.max_n;
  k.gscratch = b->d_scratch;
  k.queue = b->d_queue;
  k.err = b->d_queue + 1;
  k.out_rec = b->d_rec;
  k.out_z0 = b->d_z0;
  k.out_norm = b->d_norm;
  const uint32_t grid = std::min<uint32_t>(grid_for(cfg), std::max<uint32_t>(1, count));
  if (cfg.buffers == 1) k_batch<1><<<grid, THREADS, SMEM_NBUF1, b->stream>>>(k);
  else k_batch<2><<<grid, THREADS, SMEM_NBUF2, b->stream>>>(k);
  NCSIM_LAUNCHED("k_batch");
}

size_t order_offset(const ncsim_batch* b, const ncsim_batch_config& cfg) {
  return cfg.order == NCSIM_BATCH_ORDER_GIVEN ? b->off_seq : b->off_lpt;
}

// enqueue: reset counters, the kernel (between the two events when timed
// directly; a graph launch is timed around the whole graph), results to the host
void enqueue_run(ncsim_batch* b, const ncsim_batch_config& cfg, size_t order_off, uint32_t count, bool copy_back,
                 bool events = true) {
  NCSIM_CUDA(cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(uint32_t), b->stream));
  if (events) NCSIM_CUDA(cudaEventRecord(b->ev0, b->stream));
  enqueue_kernel(b, cfg, order_off, count);
  if (events) NCSIM_CUDA(cudaEventRecord(b->ev1, b->stream));
  NCSIM_CUDA(cudaMemcpyAsync(b->h_err, b->d_queue + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream));
  if (copy_back) {
    const size_t c = b->count();
    NCSIM_CUDA(cudaMemcpyAsync(b->h_rec, b->d_rec, c * 8, cudaMemcpyDeviceToHost, b->stream));
    NCSIM_CUDA(cudaMemcpyAsync(b->h_z0, b->d_z0, c * 8, cudaMemcpyDeviceToHost, b->stream));
    NCSIM_CUDA(cudaMemcpyAsync(b->h_norm, b->d_norm, c * 8, cudaMemcpyDeviceToHost, b->stream));
  }
}

double finish_run(ncsim_batch* b) {
  NCSIM_CUDA(cudaStreamSynchronize(b->stream));
  if (*b->h_err) throw Error(NCSIM_ERR_DEVICE, "batched trajectory kernel rejected a trajectory descriptor");
  float ms = 0.f;
  NCSIM_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  return double(ms);
}

bool same_cfg(const ncsim_batch_config& a, const ncsim_batch_config& c) {
  return a.ctas_per_sm == c.ctas_per_sm && a.buffers == c.buffers && a.order == c.order;
}

void validate_cfg(const ncsim_batch_config& c) {
  if (c.buffers != 1 && c.buffers != 2) throw Error(NCSIM_ERR_INVALID, "batch config: buffers must be 1 or 2");
  if (c.ctas_per_sm < 1 || c.ctas_per_sm > (c.buffers == 2 ? 1u : 2u))
    throw Error(NCSIM_ERR_INVALID, "batch config: 1 CTA per SM double-buffered, 1..2 single-buffered");
  if (c.order != NCSIM_BATCH_ORDER_LARGEST_FIRST && c.order != NCSIM_BATCH_ORDER_GIVEN)
    throw Error(NCSIM_ERR_INVALID, "batch config: unknown order");
}

// tuned configurations, per (device, trajectory count, largest register)
std::mutex g_tune_mu;
std::map<std::tuple<int, uint32_t, uint32_t>, ncsim_batch_config> g_tuned;

ncsim_batch_config tune(ncsim_batch* b, uint32_t sample) {
  const uint32_t c = b->count();
  // a small sample is all tail (the last CTAs' registers decide its time), so
  // the default times the whole batch once per candidate after a warm-up
  if (sample == 0) sample = c;
  sample = std::max<uint32_t>(1, std::min(sample, c));
  // an evenly strided sample keeps the batch's register-size mix
  std::vector<uint32_t> pick(sample);
  for (uint32_t i = 0; i < sample; ++i) pick[i] = uint32_t(uint64_t(i) * c / sample);
  std::vector<uint32_t> lpt = pick;
  std::stable_sort(lpt.begin(), lpt.end(),
                   [&](uint32_t x, uint32_t y) { return b->prog.traj[x].n > b->prog.traj[y].n; });
  const ncsim_batch_config cands[] = {{1, 2, NCSIM_BATCH_ORDER_LARGEST_FIRST},
                                      {2, 1, NCSIM_BATCH_ORDER_LARGEST_FIRST},
                                      {1, 1, NCSIM_BATCH_ORDER_LARGEST_FIRST},
                                      {1, 2, NCSIM_BATCH_ORDER_GIVEN}};
  ncsim_batch_config best = cands[0];
  double best_ms = 1e300;
  for (const auto& cf : cands) {
    ensure_slots(b, grid_for(cf));
    const auto& ord = cf.order == NCSIM_BATCH_ORDER_GIVEN ? pick : lpt;
    NCSIM_CUDA(cudaMemcpyAsync(b->d_prog + b->off_sample, ord.data(), size_t(sample) * 4, cudaMemcpyHostToDevice,
                               b->stream));
    double ms = 1e300;
    for (int rep = 0; rep < 2; ++rep) {  // the first is a warm-up
      enqueue_run(b, cf, b->off_sample, sample, false);
      const double t = finish_run(b);
      if (rep > 0) ms = std::min(ms, t);
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = cf;
    }
  }
  b->sample_count = sample;
  return best;
}

// ---------------------------------------------------------------------------
// planner knobs per register size: timed per size class, kept in a cache file
// ---------------------------------------------------------------------------
// The file holds one "key knob_set" line per (device, register size, program
// size): NCSIM_TUNE_CACHE names it, else $XDG_CACHE_HOME (or ~/.cache)
// /ncsim_b200/batch_knobs.txt.
std::string knob_cache_path() {
  if (const char* p = std::getenv("NCSIM_TUNE_CACHE")) return p;
  std::string base;
  if (const char* x = std::getenv("XDG_CACHE_HOME")) base = x;
  else if (const char* h = std::getenv("HOME")) base = std::string(h) + "/.cache";
  else return "";
  return base + "/ncsim_b200/batch_knobs.txt";
}

std::map<std::string, int> read_knob_cache() {
  std::map<std::string, int> m;
  const std::string path = knob_cache_path();
  if (path.empty()) return m;
  std::ifstream f(path);
  std::string key;
  int v;
  while (f >> key >> v)
    if (v >= 0 && v < int(NUM_KNOB_SETS)) m[key] = v;
  return m;
}

void write_knob_cache(const std::map<std::string, int>& add) {
  const std::string path = knob_cache_path();
  if (path.empty()) return;
  std::map<std::string, int> m = read_knob_cache();
  for (const auto& kv : add) m[kv.first] = kv.second;
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    std::string dir = path.substr(0, slash), cmd;
    for (size_t i = 1; i <= dir.size(); ++i)  // mkdir -p, one component at a time
      if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
  }
  const std::string tmp = path + ".tmp" + std::to_string(getpid());
  {
    std::ofstream f(tmp);
    for (const auto& kv : m) f << kv.first << " " << kv.second << "\n";
    if (!f) return;
  }
  std::rename(tmp.c_str(), path.c_str());  // a whole file or none
}

std::mutex g_knob_mu;
std::map<std::string, int> g_knob_mem;  // this process's choices (and the file's, once read)
bool g_knob_file_read = false;

// the cache key of size class n: device, register size, and the class's mean
// folded ops per trajectory on a log2 scale
std::string knob_key(const std::string& device, uint32_t n, double mean_ops) {
  std::ostringstream k;
  k << device << "|n" << n << "|ops2^" << int(std::floor(std::log2(std::max(1.0, mean_ops))));
  return k.str();
}

std::string device_tag() {
  int dev = 0;
  cudaDeviceProp pr{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess) {
    cudaGetLastError();
    return "";
  }
  std::string name = pr.name;
  for (char& ch : name)
    if (ch == ' ' || ch == '|') ch = '_';
  return name + "_sm" + std::to_string(pr.multiProcessorCount);
}

// knob sets found in the cache for every size class of the batch (false: some missing)
bool knobs_from_cache(ncsim_batch* b, const std::string& dev) {
  if (dev.empty() || b->ts.empty()) return false;
  std::map<uint32_t, std::pair<double, uint32_t>> ops;  // n -> (sum ops, count)
  for (const Trajectory& t : b->ts) ops[t.n].first += double(t.ops.size()), ops[t.n].second += 1;
  std::lock_guard<std::mutex> lk(g_knob_mu);
  if (!g_knob_file_read) {
    for (const auto& kv : read_knob_cache()) g_knob_mem.insert(kv);
    g_knob_file_read = true;
  }
  for (const auto& kv : ops) {
    auto it = g_knob_mem.find(knob_key(dev, kv.first, kv.second.first / kv.second.second));
    if (it == g_knob_mem.end()) return false;
    b->knob_set_by_n[kv.first] = it->second;
    b->knobs_by_n[kv.first] = knob_set(uint32_t(it->second));
  }
  return true;
}

void set_orders(ncsim_batch* b) {
  const uint32_t c = b->count();
  b->order_seq.resize(c);
  std::iota(b->order_seq.begin(), b->order_seq.end(), 0u);
  b->order_lpt = b->order_seq;
  std::stable_sort(b->order_lpt.begin(), b->order_lpt.end(),
                   [&](uint32_t x, uint32_t y) { return b->prog.traj[x].n > b->prog.traj[y].n; });
}

void finalize_knobs(ncsim_batch* b) {
  b->knobs_final = true;
  std::vector<Trajectory>().swap(b->ts);
}

// Times every candidate knob set on every size class of the batch (each class's
// trajectories alone, an evenly strided sample of at most 512, double-buffered
// at one CTA per SM) and keeps, per class, the fastest; the program is then
// compiled with the chosen knobs.  Runs on the batch's device.
void tune_knobs(ncsim_batch* b) {
  if (b->ts.empty()) return;
  std::map<uint32_t, std::vector<uint32_t>> cls;
  std::map<uint32_t, double> ops;
  for (uint32_t i = 0; i < b->ts.size(); ++i) {
    cls[b->ts[i].n].push_back(i);
    ops[b->ts[i].n] += double(b->ts[i].ops.size());
  }
  const ncsim_batch_config cf{1, 2, NCSIM_BATCH_ORDER_GIVEN};
  ensure_slots(b, grid_for(cf));
  for (uint32_t k = 0; k < NUM_KNOB_SETS; ++k) {
    b->prog = compile(b->ts, knob_set(k));
    upload_program(b);
    for (auto& kv : cls) {
      const std::vector<uint32_t>& all = kv.second;
      const size_t m = std::min<size_t>(all.size(), 512);
      std::vector<uint32_t> pick(m);
      for (size_t i = 0; i < m; ++i) pick[i] = all[i * all.size() / m];
      NCSIM_CUDA(cudaMemcpyAsync(b->d_prog + b->off_sample, pick.data(), m * 4, cudaMemcpyHostToDevice, b->stream));
      double best = 1e300;
      for (int rep = 0; rep < 2; ++rep) {  // the first is a warm-up
        enqueue_run(b, cf, b->off_sample, uint32_t(m), false);
        const double t = finish_run(b);
        if (rep > 0) best = std::min(best, t);
      }
      b->knob_ms[kv.first][k] = best;
    }
  }
  const std::string dev = device_tag();
  std::map<std::string, int> chosen;
  for (auto& kv : cls) {
    const auto& t = b->knob_ms[kv.first];
    const int best = int(std::min_element(t.begin(), t.end()) - t.begin());
    b->knob_set_by_n[kv.first] = best;
    b->knobs_by_n[kv.first] = knob_set(uint32_t(best));
    if (!dev.empty()) chosen[knob_key(dev, kv.first, ops[kv.first] / double(kv.second.size()))] = best;
  }
  b->prog = compile(b->ts, b->knobs_by_n);
  upload_program(b);
  {
    std::lock_guard<std::mutex> lk(g_knob_mu);
    for (const auto& kv : chosen) g_knob_mem[kv.first] = kv.second;
  }
  write_knob_cache(chosen);
}

// the planner's knobs final: from the cache, else timed (once per batch)
void ensure_knobs(ncsim_batch* b) {
  if (b->knobs_final) return;
  tune_knobs(b);
  finalize_knobs(b);
}

void ensure_config(ncsim_batch* b) {
  if (b->cfg.buffers != 0) return;
  const auto key = std::make_tuple(b->device, b->count(), b->prog.max_n);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      b->cfg = it->second;
      return;
    }
  }
  b->cfg = tune(b, 0);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[key] = b->cfg;
}

// The program is compiled with the knobs the cache holds for the current
// device; when it lacks a size class of the batch, the default knobs are used
// and the trajectories are kept for the autotuner, which runs on first use.
ncsim_batch* make_batch(std::vector<Trajectory>&& ts) {
  auto* b = new ncsim_batch();
  try {
    b->ts = std::move(ts);
    const bool cached = knobs_from_cache(b, device_tag());
    b->prog = compile(b->ts, b->knobs_by_n);
    set_orders(b);
    if (cached) finalize_knobs(b);
  } catch (...) {
    delete b;
    throw;
  }
  return b;
}

template <class F>
void parallel_for(size_t count, F&& f) {
  std::atomic<size_t> next{0};
  std::vector<std::string> errs(count);
  auto work = [&] {
    for (size_t i; (i = next.fetch_add(1)) < count;) {
      try {
        f(i);
      } catch (const std::exception& e) {
        errs[i] = e.what();
      }
    }
  };
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const unsigned nth = unsigned(std::min<size_t>(hw, std::max<size_t>(1, count / 8)));
  std::vector<std::thread> th;
  for (unsigned k = 1; k < nth; ++k) th.emplace_back(work);
  work();
  for (auto& x : th) x.join();
  for (auto& e : errs)
    if (!e.empty()) throw Error(NCSIM_ERR_UNSUPPORTED, e);
}

}  // namespace

namespace ncsim {
namespace batch {
ncsim_batch* batch_random_layers(uint32_t count, uint64_t seed0, uint32_t n_lo, uint32_t n_span, uint32_t depth,
                                 double p) {
  if (count == 0) throw Error(NCSIM_ERR_INVALID, "a batch needs at least one trajectory");
  if (n_span < 1) throw Error(NCSIM_ERR_INVALID, "register span must be at least 1");
  if (n_lo < MIN_QUBITS || n_lo + n_span - 1 > MAX_QUBITS)
    throw Error(NCSIM_ERR_UNSUPPORTED, "batched trajectories need 13..26 qubits");
  if (!(p >= 0.0 && p <= 1.0)) throw Error(NCSIM_ERR_INVALID, "noise probability outside [0, 1]");
  std::vector<Trajectory> ts(count);
  parallel_for(count, [&](size_t i) { ts[i] = make_random_layers(seed0 + i, n_lo, n_span, depth, p); });
  return make_batch(std::move(ts));
}
}  // namespace batch
}  // namespace ncsim

extern "C" {

ncsim_status ncsim_batch_from_circuits(uint32_t count, const ncsim_circuit* const* circuits, const uint64_t* seeds,
                                       ncsim_batch** out) {
  return guarded([&] {
    if (!out || !circuits || !seeds) throw Error(NCSIM_ERR_INVALID, "null argument");
    *out = nullptr;
    if (count == 0) throw Error(NCSIM_ERR_INVALID, "a batch needs at least one trajectory");
    for (uint32_t i = 0; i < count; ++i)
      if (!circuits[i]) throw Error(NCSIM_ERR_INVALID, "null circuit");
    std::vector<Trajectory> ts(count);
    parallel_for(count, [&](size_t i) { ts[i] = make_from_circuit(*circuits[i], seeds[i]); });
    *out = make_batch(std::move(ts));
  });
}

ncsim_status ncsim_batch_free(ncsim_batch* b) {
  return guarded([&] { delete b; });
}

ncsim_status ncsim_batch_release(ncsim_batch* b) {
  return guarded([&] {
    if (!b) throw Error(NCSIM_ERR_INVALID, "null batch");
    std::lock_guard<std::mutex> lk(b->mu);
    b->release();
  });
}

ncsim_status ncsim_batch_info(const ncsim_batch* b, ncsim_batch_stats* st) {
  return guarded([&] {
    if (!b || !st) throw Error(NCSIM_ERR_INVALID, "null argument");
    const Program& P = b->prog;
    st->trajectories = P.traj.size();
    st->source_gates = P.source_gates;
    st->noise_events = P.noise_events;
    st->folded_ops = P.folded_ops;
    st->passes = P.pass.size();
    st->tile_passes = P.tile_passes;
    st->tile_stages = P.tile_stages;
    st->state_bytes = P.state_bytes;
    st->max_qubits = P.max_n;
    st->program_bytes = P.traj.size() * sizeof(DevTraj) + P.pass.size() * sizeof(DevPass) +
                        P.stage.size() * sizeof(DevStage) + P.op.size() * sizeof(DevOp) + P.draws.size() * 8;
  });
}

ncsim_status ncsim_batch_knobs(const ncsim_batch* b, uint32_t n, ncsim_batch_knobs_info* out) {
  return guarded([&] {
    if (!b || !out) throw Error(NCSIM_ERR_INVALID, "null argument");
    if (n > MAX_QUBITS) throw Error(NCSIM_ERR_INVALID, "register size above 26");
    const PlanKnobs& k = b->knobs_by_n[n];
    out->knob_set = uint32_t(b->knob_set_by_n[n]);
    out->window_step = k.window_step;
    out->greedy_windows = k.greedy_windows;
    out->greedy_stages = k.greedy_stages;
    out->final_ = b->knobs_final;
    for (uint32_t i = 0; i < 4; ++i) out->timed_ms[i] = i < NUM_KNOB_SETS ? b->knob_ms[n][i] : 0.0;
  });
}

ncsim_status ncsim_batch_set_knob_set(ncsim_batch* b, uint32_t n, uint32_t knob_set_index, int32_t final_) {
  return guarded([&] {
    if (!b) throw Error(NCSIM_ERR_INVALID, "null batch");
    if (n > MAX_QUBITS) throw Error(NCSIM_ERR_INVALID, "register size above 26");
    if (knob_set_index >= NUM_KNOB_SETS) throw Error(NCSIM_ERR_INVALID, "unknown knob set");
    std::lock_guard<std::mutex> lk(b->mu);
    if (b->knobs_final) throw Error(NCSIM_ERR_INVALID, "the batch's knobs are final (its trajectories were dropped)");
    b->knob_set_by_n[n] = int(knob_set_index);
    b->knobs_by_n[n] = knob_set(knob_set_index);
    b->prog = compile(b->ts, b->knobs_by_n);
    if (b->device >= 0) {
      int cur = 0;
      NCSIM_CUDA(cudaGetDevice(&cur));
      if (cur == b->device) upload_program(b);
      else b->release();
    }
    if (final_) finalize_knobs(b);
  });
}

ncsim_status ncsim_batch_set_config(ncsim_batch* b, const ncsim_batch_config* cfg) {
  return guarded([&] {
    if (!b || !cfg) throw Error(NCSIM_ERR_INVALID, "null argument");
    validate_cfg(*cfg);
    std::lock_guard<std::mutex> lk(b->mu);
    b->cfg = *cfg;
  });
}

ncsim_status ncsim_batch_get_config(ncsim_batch* b, ncsim_batch_config* cfg) {
  return guarded([&] {
    if (!b || !cfg) throw Error(NCSIM_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    ensure_device(b);
    ensure_knobs(b);
    ensure_config(b);
    *cfg = b->cfg;
  });
}

ncsim_status ncsim_batch_tune(ncsim_batch* b, uint32_t sample, ncsim_batch_config* best) {
  return guarded([&] {
    if (!b) throw Error(NCSIM_ERR_INVALID, "null batch");
    std::lock_guard<std::mutex> lk(b->mu);
    ensure_device(b);
    if (!b->ts.empty()) tune_knobs(b);  // the planner's knobs too, while the trajectories are kept
    finalize_knobs(b);
    b->cfg = tune(b, sample);
    {
      std::lock_guard<std::mutex> g(g_tune_mu);
      g_tuned[std::make_tuple(b->device, b->count(), b->prog.max_n)] = b->cfg;
    }
    if (best) *best = b->cfg;
  });
}

ncsim_status ncsim_batch_run(ncsim_batch* b, double* device_ms) {
  return guarded([&] {
    if (!b) throw Error(NCSIM_ERR_INVALID, "null batch");
    std::lock_guard<std::mutex> lk(b->mu);
    ensure_device(b);
    ensure_knobs(b);
    ensure_config(b);
    ensure_slots(b, grid_for(b->cfg));
    if (!b->graph || !same_cfg(b->graph_cfg, b->cfg)) {
      if (b->graph) {
        NCSIM_CUDA(cudaGraphExecDestroy(b->graph));
        b->graph = nullptr;
      }
      cudaGraph_t g = nullptr;
      NCSIM_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      try {
        enqueue_run(b, b->cfg, order_offset(b, b->cfg), b->count(), true, false);
      } catch (...) {
        cudaStreamEndCapture(b->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      NCSIM_CUDA(cudaStreamEndCapture(b->stream, &g));
      const cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      NCSIM_CUDA(e);
      b->graph_cfg = b->cfg;
    }
    NCSIM_CUDA(cudaEventRecord(b->ev0, b->stream));
    NCSIM_CUDA(cudaGraphLaunch(b->graph, b->stream));
    NCSIM_CUDA(cudaEventRecord(b->ev1, b->stream));
    b->last_ms = finish_run(b);
    b->have_results = true;
    if (device_ms) *device_ms = b->last_ms;
  });
}

ncsim_status ncsim_batch_results(ncsim_batch* b, uint32_t* n, uint64_t* records, double* z0, double* norm) {
  return guarded([&] {
    if (!b) throw Error(NCSIM_ERR_INVALID, "null batch");
    std::lock_guard<std::mutex> lk(b->mu);
    if (!b->have_results) throw Error(NCSIM_ERR_INVALID, "the batch has not run");
    const uint32_t c = b->count();
    for (uint32_t i = 0; i < c; ++i) {
      if (n) n[i] = b->prog.traj[i].n;
      if (records) records[i] = b->h_rec[i];
      if (z0) z0[i] = b->h_z0[i];
      if (norm) norm[i] = b->h_norm[i];
    }
  });
}

ncsim_status ncsim_batch_emulate(const ncsim_batch* b, uint32_t t, uint64_t* record, double* z0, double* norm) {
  return guarded([&] {
    if (!b) throw Error(NCSIM_ERR_INVALID, "null batch");
    if (t >= b->prog.traj.size()) throw Error(NCSIM_ERR_INVALID, "trajectory index out of range");
    if (b->prog.traj[t].n > 22) throw Error(NCSIM_ERR_UNSUPPORTED, "host emulation is limited to 22 qubits");
    const EmuResult r = emulate(b->prog, t);
    if (record) *record = r.record;
    if (z0) *z0 = r.z0;
    if (norm) *norm = r.norm;
  });
}

ncsim_status ncsim_batch_trajectory_qubits(const ncsim_batch* b, uint32_t* n) {
  return guarded([&] {
    if (!b || !n) throw Error(NCSIM_ERR_INVALID, "null argument");
    for (size_t i = 0; i < b->prog.traj.size(); ++i) n[i] = b->prog.traj[i].n;
  });
}

}  // extern "C"
