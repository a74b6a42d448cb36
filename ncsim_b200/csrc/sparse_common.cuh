// Shared pieces of the sparse form (sparse.cu: registers of up to 64 qubits,
// one 64-bit word per basis key; sparse_wide.cu: wider registers, several
// words per key): the state object, launch shapes, complex helpers, the
// local-index helpers of a gate's qubits, phase-polynomial evaluation, the
// key-independent kernels (scale, keep flags, norms, weights) and the host
// helpers (locks, stream-ordered buffers, fixed-order sums).
#pragma once

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

#include "engine.cuh"
#include "host/ir.hpp"
#include "host/rng.hpp"

struct ncsim_sparse {
  uint32_t n = 0;
  uint32_t words = 1;  // 64-bit words per basis key: 1 up to 64 qubits, 4 up to 256, 16 up to 1024
  uint64_t m = 0;      // entries
  uint64_t cap = 0;    // capacity of key/amp (entries)
  uint64_t* key = nullptr;  // m keys of `words` words each (qubit q: bit q % 64 of word q / 64)
  double2* amp = nullptr;
  bool sorted = true;
  double cutoff = 0.0;
  cudaStream_t stream = nullptr;
  int device = 0;
  double* partials = nullptr;       // device: SP_BLOCKS * 2 doubles
  double* host_partials = nullptr;  // pinned mirror
  cudaEvent_t timer0 = nullptr, timer1 = nullptr;
  mutable std::recursive_mutex mu;
};

namespace {
using namespace ncsim;

constexpr int SP_THREADS = 256;
constexpr int SP_BLOCKS = 1024;  // reduction blocks (partials)
constexpr uint32_t SP_MAX_K = 10;

unsigned sp_grid(uint64_t items) {
  uint64_t b = (items + SP_THREADS - 1) / SP_THREADS;
  const uint64_t cap = uint64_t(sm_count()) * 16;
  return unsigned(std::max<uint64_t>(1, std::min(b, cap)));
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 ipow(double2 v, uint32_t k) {  // i^k v
  switch (k & 3u) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
  }
}

// the qubits of a gate and the local index of a key on them (sparse.rs:243-258)
struct Qubits {
  uint32_t k;
  uint8_t q[SP_MAX_K];
};
__device__ __forceinline__ uint32_t local_of(uint64_t key, const Qubits& qs) {
  uint32_t x = 0;
  for (uint32_t j = 0; j < qs.k; ++j) x |= uint32_t((key >> qs.q[j]) & 1u) << j;
  return x;
}
__device__ __forceinline__ uint64_t with_local(uint64_t key, const Qubits& qs, uint32_t y) {
  for (uint32_t j = 0; j < qs.k; ++j)
    key = (key & ~(uint64_t(1) << qs.q[j])) | (uint64_t((y >> j) & 1u) << qs.q[j]);
  return key;
}


// exp(2 pi i f / 2^bits) with exact quarter and eighth turns
__device__ double2 turn_root(uint64_t f, uint32_t bits) {
  const uint64_t mk = bits >= 64 ? ~uint64_t(0) : (uint64_t(1) << bits) - 1;
  f &= mk;
  if (bits >= 2 && (f & (mk >> 2)) == 0) {
    switch ((f >> (bits - 2)) & 3u) {
      case 0: return make_double2(1.0, 0.0);
      case 1: return make_double2(0.0, 1.0);
      case 2: return make_double2(-1.0, 0.0);
      default: return make_double2(0.0, -1.0);
    }
  }
  if (bits >= 3 && (f & (mk >> 3)) == 0) {
    const double h = 0.70710678118654752440;
    switch ((f >> (bits - 3)) & 7u) {
      case 1: return make_double2(h, h);
      case 3: return make_double2(-h, h);
      case 5: return make_double2(-h, -h);
      default: return make_double2(h, -h);
    }
  }
  if (bits == 1) return f ? make_double2(-1.0, 0.0) : make_double2(1.0, 0.0);
  double s, c;
  sincospi(2.0 * double(f) / double(uint64_t(1) << std::min<uint32_t>(bits, 63)), &s, &c);
  return make_double2(c, s);
}


// amp *= scalar * zeta^f for the polynomial's value f (reduced mod 2^bits here)
__device__ __forceinline__ void poly_finish(uint64_t f, double2& amp, uint32_t bits, bool scalar_is_one,
                                            double2 scalar, bool use_table, const double2* table) {
  const uint64_t mk = bits >= 64 ? ~uint64_t(0) : (uint64_t(1) << bits) - 1;
  f &= mk;
  double2 c;
  if (use_table) {
    c = table[f];
  } else {
    if (f == 0 && scalar_is_one) return;
    c = turn_root(f, bits);
    if (!scalar_is_one) c = zmul(scalar, c);
  }
  if (c.x == 1.0 && c.y == 0.0) return;
  amp = zmul(c, amp);
}

// amp *= scalar * zeta^f(key), f = constant + sum_t coeff_t prod_l [par_l . key] mod 2^bits
// (and_mask, when given: a term whose parities are all single bits is the AND of
// those bits, one compare instead of a popcount per parity; 0 for other terms)
template <class Start>
__device__ __forceinline__ void poly_apply(uint64_t kk, double2& amp, uint32_t bits, uint32_t nterms, uint64_t constant,
                                           bool scalar_is_one, double2 scalar, bool use_table, const Start* start,
                                           const uint64_t* par, const uint64_t* coeff, const double2* table,
                                           const uint64_t* and_mask = nullptr) {
  uint64_t f = constant;
#pragma unroll 4
  for (uint32_t t = 0; t < nterms; ++t) {
    uint32_t all = 1;
    const uint64_t am = and_mask ? and_mask[t] : 0;
    if (am) {
      all = (kk & am) == am;
    } else {
      for (uint32_t l = start[t]; l < start[t + 1]; ++l) all &= uint32_t(__popcll(par[l] & kk)) & 1u;
    }
    if (all) f += coeff[t];
  }
  poly_finish(f, amp, bits, scalar_is_one, scalar, use_table, table);
}

// The sum of poly_apply with the warp sharing the term loads: lane j loads term
// t0 + j of each group of 32 and the terms reach every lane by shuffles, so a
// polynomial of many terms costs one round of dependent loads per 32 terms
// instead of one per term (integer sums: the same f in any order).  All 32 lanes
// of the warp call it with the same polynomial.
__device__ __forceinline__ uint64_t poly_sum_warp(uint64_t kk, uint32_t nterms, uint64_t constant,
                                                  const uint32_t* start, const uint64_t* par, const uint64_t* coeff,
                                                  const uint64_t* and_mask) {
  const uint32_t lane = threadIdx.x & 31u;
  uint64_t f = constant;
  for (uint32_t t0 = 0; t0 < nterms; t0 += 32) {
    const uint32_t t = t0 + lane;
    uint64_t am = 0, co = 0;
    uint32_t s0 = 0, s1 = 0;
    if (t < nterms) {
      am = and_mask[t];
      co = coeff[t];
      s0 = start[t];
      s1 = start[t + 1];
    }
    const uint32_t cnt = min(32u, nterms - t0);
    for (uint32_t j = 0; j < cnt; ++j) {
      const uint64_t amj = __shfl_sync(0xffffffffu, am, int(j));
      const uint64_t coj = __shfl_sync(0xffffffffu, co, int(j));
      uint32_t all = 1;
      if (amj) {  // warp-uniform
        all = (kk & amj) == amj;
      } else {
        const uint32_t a0 = __shfl_sync(0xffffffffu, s0, int(j));
        const uint32_t a1 = __shfl_sync(0xffffffffu, s1, int(j));
        for (uint32_t l = a0; l < a1; ++l) all &= uint32_t(__popcll(par[l] & kk)) & 1u;
      }
      if (all) f += coj;
    }
  }
  return f;
}

__global__ void k_sp_scale(double2* amp, uint64_t m, double2 c) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    amp[i] = zmul(c, amp[i]);
}


// ---- normalisation helpers ----
struct ZAdd {
  __device__ __forceinline__ double2 operator()(const double2& a, const double2& b) const {
    return make_double2(a.x + b.x, a.y + b.y);
  }
};
// Keep flags over a reduce-by-key output whose run count is still on the device:
// an entry stays when its amplitude is nonzero and |a|^2 >= cutoff^2 (or the
// cutoff is 0); positions at or past the count are dropped, so the selection can
// run over the input's size without the host waiting for the count.
__global__ void k_sp_keep(const double2* amp, const int* d_runs, uint64_t cap, double cut2, uint8_t* flag) {
  const uint64_t runs = uint64_t(*d_runs);
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < cap; i += uint64_t(gridDim.x) * blockDim.x) {
    if (i >= runs) {
      flag[i] = 0;
      continue;
    }
    const double2 a = amp[i];
    const bool zero = a.x == 0.0 && a.y == 0.0;
    flag[i] = !zero && (cut2 == 0.0 || a.x * a.x + a.y * a.y >= cut2);
  }
}


// ---- sums (block partials, FP64) ----
__device__ __forceinline__ void block_add2(double a, double b, double* out) {
  __shared__ double red[SP_THREADS / 32][2];
  for (int o = 16; o; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w][0] = a, red[w][1] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0;
    for (int i = 0; i < SP_THREADS / 32; ++i) s0 += red[i][0], s1 += red[i][1];
    out[2 * blockIdx.x] = s0;
    out[2 * blockIdx.x + 1] = s1;
  }
}
__global__ void k_sp_norm(const double2* amp, uint64_t m, double* part) {
  double s = 0;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const double2 a = amp[i];
    s += a.x * a.x + a.y * a.y;
  }
  block_add2(s, 0.0, part);
}

__global__ void k_sp_abs2(const double2* amp, uint64_t m, double* out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const double2 a = amp[i];
    out[i] = a.x * a.x + a.y * a.y;
  }
}

struct Lock {
  std::lock_guard<std::recursive_mutex> g;
  explicit Lock(const ncsim_sparse* s) : g(s->mu) { NCSIM_CUDA(cudaSetDevice(s->device)); }
};
// two states locked together without an order between them (no deadlock when
// other threads lock the same pair the other way round); a's device current
struct PairLock {
  std::unique_lock<std::recursive_mutex> la, lb;
  PairLock(const ncsim_sparse* a, const ncsim_sparse* b) : la(a->mu, std::defer_lock), lb(b->mu, std::defer_lock) {
    if (a == b) la.lock();
    else std::lock(la, lb);
    NCSIM_CUDA(cudaSetDevice(a->device));
  }
};

template <class T>
T* dalloc(size_t count, cudaStream_t st) {
  void* p = nullptr;
  NCSIM_CUDA(pool_alloc(&p, std::max<size_t>(1, count) * sizeof(T), st));
  return static_cast<T*>(p);
}
void dfree(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}
template <class T>
T* upload(const std::vector<T>& v, cudaStream_t st) {
  T* d = dalloc<T>(v.size(), st);
  if (!v.empty()) NCSIM_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return d;
}


// the host sum of the block partials (fixed order)
void sp_sum(const ncsim_sparse* s, unsigned blocks, double* out2) {
  NCSIM_CUDA(cudaMemcpyAsync(s->host_partials, s->partials, size_t(blocks) * 2 * sizeof(double),
                             cudaMemcpyDeviceToHost, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  double a = 0, b = 0;
  for (unsigned i = 0; i < blocks; ++i) a += s->host_partials[2 * i], b += s->host_partials[2 * i + 1];
  out2[0] = a;
  out2[1] = b;
}
unsigned red_grid(uint64_t m) { return unsigned(std::min<uint64_t>(SP_BLOCKS, std::max<uint64_t>(1, (m + SP_THREADS - 1) / SP_THREADS))); }

double sp_norm(const ncsim_sparse* s) {
  const unsigned g = red_grid(s->m);
  k_sp_norm<<<g, SP_THREADS, 0, s->stream>>>(s->amp, s->m, s->partials);
  NCSIM_LAUNCHED("sparse norm");
  double r[2];
  sp_sum(s, g, r);
  return r[0];
}


void need(const void* p, const char* what) {
  if (!p) throw Error(NCSIM_ERR_INVALID, std::string(what) + " is null");
}

// A dense view with one nonzero per column on distinct rows (a permutation with
// phases, as CCX): every entry moves to one entry (sparse.rs:176-199).
bool permutation_view(const std::vector<CplxD>& mat, size_t gd, std::vector<uint32_t>& image, std::vector<CplxD>& ph) {
  image.assign(gd, 0);
  ph.assign(gd, CplxD{0, 0});
  std::vector<uint8_t> hit(gd, 0);
  for (size_t b = 0; b < gd; ++b) {
    int found = 0;
    for (size_t a = 0; a < gd; ++a) {
      const CplxD e = mat[a * gd + b];
      if (e.re == 0.0 && e.im == 0.0) continue;
      if (++found > 1 || hit[a]) return false;
      hit[a] = 1;
      image[b] = uint32_t(a);
      ph[b] = e;
    }
    if (found != 1) return false;
  }
  return true;
}

}  // namespace

// The sparse form on registers wider than 64 qubits (sparse_wide.cu).  Keys
// and Pauli masks are `s->words` 64-bit words; keys order lexicographically
// from word 0 (the order of ncsim's Bits = Vec<u64>, bits.rs:11).  Gates are
// lowered on their own qubits (lower_gate with local qubits 0..k-1).
namespace ncsim {
namespace spw {
constexpr uint32_t MAX_QUBITS = 1024;
uint32_t words_for(uint32_t n);  // 1 (n <= 64), 4 (n <= 256), 16 (n <= 1024)
void set_entries(ncsim_sparse* s, const uint64_t* keys, const double* amps, uint64_t count);
void normalize(ncsim_sparse* s);
void sort(ncsim_sparse* s);
void apply_gate(ncsim_sparse* s, const GateIR& g, const std::vector<uint32_t>& qubits);
void pauli(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase);
void amplitude(const ncsim_sparse* s, const uint64_t* index, double* re_im);
void expectation(const ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, double* re_im);
void inner(const ncsim_sparse* a, const ncsim_sparse* b, double* re_im);
double project(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, bool outcome);
void tensor(const ncsim_sparse* a, const ncsim_sparse* b, ncsim_sparse* c);
void sample(const ncsim_sparse* s, ncsim_rng& rng, uint64_t shots, uint64_t* out);
bool measure(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, ncsim_rng& rng);
void run(ncsim_sparse* s, const ncsim_circuit& c, ncsim_rng& rng, uint8_t* rec, size_t& m);
}  // namespace spw
}  // namespace ncsim
