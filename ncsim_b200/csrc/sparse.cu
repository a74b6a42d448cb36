// The reference's SparseVector<C64> (src/state/sparse.rs) on the device: the
// nonzero amplitudes of a register of up to 64 qubits as (basis index,
// complex128) pairs in HBM, for circuits whose states stay sparse (permutation
// and diagonal gates: reversible arithmetic, the C3 family).
//
// Entry order follows the reference: operations that move each entry to one
// entry (monomial gates, permutations with phases, Paulis, diagonals) work in
// place and keep the order (unsorted afterwards when a key changed); the ones
// that create entries (a dense gate, a projection, a tensor product) expand
// into a new array that is then normalised: sorted by key, duplicates summed,
// exact zeros (and amplitudes under the cutoff) dropped (sparse.rs:114-128).
// Sums over entries (norm, expectation, inner product) are FP64 block partials
// added on the host in a fixed order; Born sampling takes the cumulative
// weights in entry order on the host, as sparse.rs:407-424 does.
#include "sparse_common.cuh"

using namespace ncsim;

namespace {

// ---- kernels that move each entry to one entry (order kept) ----
// monomial: entry with local pattern x goes to image[x] with phase[x]
__global__ void k_sp_monomial(uint64_t* key, double2* amp, uint64_t m, Qubits qs, const uint32_t* image,
                              const double2* phase, const uint8_t* unit) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t kk = key[i];
    const uint32_t x = local_of(kk, qs);
    if (!unit[x]) amp[i] = zmul(phase[x], amp[i]);
    const uint32_t y = image[x];
    if (y != x) key[i] = with_local(kk, qs, y);
  }
}

// the same with the tables in the kernel parameters (no per-gate upload)
template <int N>
struct MonoParams {
  Qubits qs;
  uint32_t unit[(N + 31) / 32];  // bit x: phase[x] == 1
  uint16_t image[N];
  double2 phase[N];
};
template <int N>
__global__ void k_sp_monomial_p(uint64_t* key, double2* amp, uint64_t m, const __grid_constant__ MonoParams<N> P) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t kk = key[i];
    const uint32_t x = local_of(kk, P.qs);
    if (!((P.unit[x >> 5] >> (x & 31)) & 1u)) amp[i] = zmul(P.phase[x], amp[i]);
    const uint32_t y = P.image[x];
    if (y != x) key[i] = with_local(kk, P.qs, y);
  }
}

// i^phase X^x Z^z (sparse.rs:216-231)
__global__ void k_sp_pauli(uint64_t* key, double2* amp, uint64_t m, uint64_t x, uint64_t z, uint32_t phase) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t kk = key[i];
    const uint32_t k = (phase + 2u * uint32_t(__popcll(z & kk))) & 3u;
    if (k) amp[i] = ipow(amp[i], k);
    key[i] = kk ^ x;
  }
}

// diagonal phase polynomial over global index parities (Diagonal(PhasePoly))
struct SpPoly {
  uint32_t bits, nterms, scalar_is_one, use_table;
  uint64_t constant;
  double2 scalar;
  const uint32_t* start;
  const uint64_t* par;
  const uint64_t* coeff;
  const double2* table;
};
__global__ void k_sp_phasepoly(const uint64_t* key, double2* amp, uint64_t m, SpPoly P) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    poly_apply(key[i], amp[i], P.bits, P.nterms, P.constant, P.scalar_is_one, P.scalar, P.use_table, P.start, P.par,
               P.coeff, P.table);
}

// the same with the terms in the kernel parameters
constexpr int SP_POLY_TERMS = 128, SP_POLY_PARS = 256;
struct PolyParamsSp {
  uint32_t bits, nterms, scalar_is_one, use_table;
  uint64_t constant;
  double2 scalar;
  uint16_t start[SP_POLY_TERMS + 1];
  uint64_t par[SP_POLY_PARS];
  uint64_t coeff[SP_POLY_TERMS];
  double2 table[256];
};
__global__ void k_sp_phasepoly_p(const uint64_t* key, double2* amp, uint64_t m, const __grid_constant__ PolyParamsSp P) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    poly_apply(key[i], amp[i], P.bits, P.nterms, P.constant, P.scalar_is_one, P.scalar, P.use_table, P.start, P.par,
               P.coeff, P.table);
}

// ---- expansions (new entries, normalised afterwards) ----
// dense matrix: entry (key, v) with local column b gives (key with row a, m_ab v)
// for every nonzero m_ab of column b (sparse.rs:162-214)
__global__ void k_sp_count(const uint64_t* key, uint64_t m, Qubits qs, const uint32_t* col_start, uint32_t* cnt) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t b = local_of(key[i], qs);
    cnt[i] = col_start[b + 1] - col_start[b];
  }
}
__global__ void k_sp_expand(const uint64_t* key, const double2* amp, uint64_t m, Qubits qs, const uint32_t* col_start,
                            const uint32_t* col_row, const double2* col_val, const uint32_t* off, uint32_t per,
                            uint64_t* okey, double2* oamp) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t kk = key[i];
    const double2 v = amp[i];
    const uint32_t b = local_of(kk, qs);
    uint64_t o = off ? uint64_t(off[i]) : i * per;  // per: every column's count, when they are all equal
    for (uint32_t j = col_start[b]; j < col_start[b + 1]; ++j, ++o) {
      okey[o] = with_local(kk, qs, col_row[j]);
      oamp[o] = zmul(col_val[j], v);
    }
  }
}
// (1 ± P)/2: entry c gives (c, psi(c)/2) and (c ^ x, ±i^k(c) psi(c)/2) (sparse.rs:351-380)
__global__ void k_sp_project(const uint64_t* key, const double2* amp, uint64_t m, uint64_t x, uint64_t z,
                             uint32_t phase, double sgn, uint64_t* okey, double2* oamp) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t c = key[i];
    const double2 a = amp[i];
    const uint32_t k = (phase + 2u * uint32_t(__popcll(z & c))) & 3u;
    const double2 h = make_double2(0.5 * a.x, 0.5 * a.y);
    okey[2 * i] = c;
    oamp[2 * i] = h;
    const double2 t = ipow(h, k);
    okey[2 * i + 1] = c ^ x;
    oamp[2 * i + 1] = make_double2(sgn * t.x, sgn * t.y);
  }
}
// a (x) b: for each entry of b (outer), each entry of a (inner) (sparse.rs:388-405)
__global__ void k_sp_tensor(const uint64_t* ka, const double2* va, uint64_t ma, uint32_t na, const uint64_t* kb,
                            const double2* vb, uint64_t mb, uint64_t* okey, double2* oamp) {
  const uint64_t tot = ma * mb;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t jb = i / ma, ia = i - jb * ma;
    okey[i] = ka[ia] | (na >= 64 ? 0 : (kb[jb] << na));
    oamp[i] = zmul(va[ia], vb[jb]);
  }
}

// ---- a run of one-to-one ops in one pass ----
// Monomial gates, diagonals and Paulis map each entry to one entry, so a run of
// them is applied entry by entry: one thread walks the run's op list with its
// entry in registers (one launch and one read and write of the entries per run).
enum : uint32_t { RUN_MONO = 0, RUN_POLY = 1, RUN_PAULI = 2 };
struct RunOp {
  uint32_t type;
  uint32_t k;        // MONO: qubits; POLY: terms
  uint8_t q[SP_MAX_K];
  uint16_t pad;
  uint32_t off;      // MONO: first pattern in image/phase/unit; POLY: first term in start
  uint32_t bits;     // POLY
  uint32_t flags;    // POLY: bit 0 scalar is one, bit 1 phasor table; PAULI: the phase
  uint32_t toff;     // POLY: first entry of its phasor table in RunData::table
  uint64_t x, z;     // PAULI; POLY: x = constant
  double2 scalar;    // POLY
  // MONO on at most 3 qubits: the 8 images (16 bits each: patterns 0..3, 4..7) and unit flags
  // (byte x: the phase of pattern x is exactly 1), packed on the host
  uint64_t img_lo, img_hi, unit8;
};
struct RunData {
  const RunOp* ops;
  uint32_t nops;
  const uint16_t* image;  // monomial tables (image, phase, unit share the op's offset)
  const double2* phase;
  const uint8_t* unit;
  const double2* table;   // polynomial phasor tables
  const uint32_t* start;  // polynomial term starts (absolute indices into par)
  const uint64_t* par;
  const uint64_t* coeff;
  const uint64_t* and_mask;  // per term (aligned with coeff): the AND of single-bit parities, or 0
};
// The block stages the run's op descriptors RUN_STAGE at a time in shared
// memory, so each thread's walk reads them as broadcasts instead of a chain of
// dependent global loads per op; monomials on at most 3 qubits carry their image
// and unit tables in the descriptor, a wider monomial's three table loads issue
// together, and a phase polynomial's terms are loaded 32 at a time by the warp.
// Every lane walks the ops (lanes past the last entry on a dummy entry) so that
// the warp's shuffles see all 32 lanes.
constexpr uint32_t RUN_STAGE = SP_THREADS;
__global__ void __launch_bounds__(SP_THREADS) k_sp_run(uint64_t* key, double2* amp, uint64_t m, RunData d) {
  __shared__ RunOp s_op[RUN_STAGE];
  for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x; base < m; base += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t i = base + threadIdx.x;
    const bool live = i < m;
    uint64_t kk = live ? key[i] : 0;
    double2 a = live ? amp[i] : make_double2(0.0, 0.0);
    for (uint32_t o0 = 0; o0 < d.nops; o0 += RUN_STAGE) {
      const uint32_t cnt = min(RUN_STAGE, d.nops - o0);
      __syncthreads();
      if (threadIdx.x < cnt) s_op[threadIdx.x] = d.ops[o0 + threadIdx.x];
      __syncthreads();
      for (uint32_t c = 0; c < cnt; ++c) {
        const RunOp& op = s_op[c];
        if (op.type == RUN_MONO) {
          const uint32_t k = op.k;
          uint32_t x = 0;
          for (uint32_t j = 0; j < k; ++j) x |= uint32_t((kk >> op.q[j]) & 1u) << j;
          uint32_t y;
          bool unit;
          double2 ph = make_double2(1.0, 0.0);
          if (k <= 3) {
            y = uint32_t((x < 4 ? op.img_lo : op.img_hi) >> (16 * (x & 3))) & 0xffffu;
            unit = (op.unit8 >> (8 * x)) & 1u;
            if (!unit) ph = d.phase[op.off + x];
          } else {
            y = d.image[op.off + x];
            unit = d.unit[op.off + x];
            ph = d.phase[op.off + x];
          }
          if (!unit) a = zmul(ph, a);
          if (y != x)
            for (uint32_t j = 0; j < k; ++j)
              kk = (kk & ~(uint64_t(1) << op.q[j])) | (uint64_t((y >> j) & 1u) << op.q[j]);
        } else if (op.type == RUN_POLY) {
          const uint64_t f =
              poly_sum_warp(kk, op.k, op.x, d.start + op.off, d.par, d.coeff + op.off, d.and_mask + op.off);
          poly_finish(f, a, op.bits, op.flags & 1u, op.scalar, (op.flags >> 1) & 1u, d.table + op.toff);
        } else {
          const uint32_t ph = (op.flags + 2u * uint32_t(__popcll(op.z & kk))) & 3u;
          if (ph) a = ipow(a, ph);
          kk ^= op.x;
        }
      }
    }
    if (live) {
      key[i] = kk;
      amp[i] = a;
    }
  }
}

__device__ __forceinline__ int64_t find_key(const uint64_t* sk, uint64_t m, uint64_t x) {
  uint64_t lo = 0, hi = m;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (sk[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < m && sk[lo] == x ? int64_t(lo) : -1;
}
// <psi|P|psi> = sum_c conj psi(c ^ x) i^k(c) psi(c) over the sorted view (sparse.rs:316-336)
__global__ void k_sp_expect(const uint64_t* sk, const double2* sa, uint64_t m, uint64_t x, uint64_t z, uint32_t phase,
                            double* part) {
  double re = 0, im = 0;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t c = sk[i];
    const int64_t j = x ? find_key(sk, m, c ^ x) : int64_t(i);
    if (j < 0) continue;
    const uint32_t k = (phase + 2u * uint32_t(__popcll(z & c))) & 3u;
    const double2 t = ipow(sa[i], k);
    const double2 b = sa[j];
    re += b.x * t.x + b.y * t.y;  // conj(b) t
    im += b.x * t.y - b.y * t.x;
  }
  block_add2(re, im, part);
}
// <a|b> = sum over a's entries of conj a(c) b(c) (sparse.rs:338-349)
__global__ void k_sp_inner(const uint64_t* ka, const double2* va, uint64_t ma, const uint64_t* skb, const double2* svb,
                           uint64_t mb, double* part) {
  double re = 0, im = 0;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < ma; i += uint64_t(gridDim.x) * blockDim.x) {
    const int64_t j = find_key(skb, mb, ka[i]);
    if (j < 0) continue;
    const double2 a = va[i], b = svb[j];
    re += a.x * b.x + a.y * b.y;
    im += a.x * b.y - a.y * b.x;
  }
  block_add2(re, im, part);
}
__global__ void k_sp_find(const uint64_t* key, const double2* amp, uint64_t m, uint64_t x, int sorted, double2* out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double2 r = make_double2(0.0, 0.0);
    if (sorted) {
      const int64_t j = find_key(key, m, x);
      if (j >= 0) r = amp[j];
    } else {
      for (uint64_t i = 0; i < m; ++i)
        if (key[i] == x) {
          r = amp[i];
          break;
        }
    }
    *out = r;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void sp_reserve(ncsim_sparse* s, uint64_t need) {
  if (need <= s->cap) return;
  const uint64_t cap = std::max<uint64_t>(need, std::max<uint64_t>(1024, 2 * s->cap));
  uint64_t* k = dalloc<uint64_t>(cap * s->words, s->stream);
  double2* a = dalloc<double2>(cap, s->stream);
  if (s->m) {
    NCSIM_CUDA(cudaMemcpyAsync(k, s->key, s->m * 8 * s->words, cudaMemcpyDeviceToDevice, s->stream));
    NCSIM_CUDA(cudaMemcpyAsync(a, s->amp, s->m * 16, cudaMemcpyDeviceToDevice, s->stream));
  }
  dfree(s->key, s->stream);
  dfree(s->amp, s->stream);
  s->key = k;
  s->amp = a;
  s->cap = cap;
}

// replaces the entries by the normalised form of (key, amp)[0, cnt): sorted by
// key, duplicates summed, exact zeros and entries under the cutoff dropped
// (sparse.rs:114-128).  Takes ownership of key/amp (stream-ordered buffers).
void sp_normalize_from(ncsim_sparse* s, uint64_t* key, double2* amp, uint64_t cnt) {
  cudaStream_t st = s->stream;
  if (cnt > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  const int num = int(cnt);
  uint64_t* k2 = dalloc<uint64_t>(cnt, st);
  double2* a2 = dalloc<double2>(cnt, st);
  uint64_t* k3 = dalloc<uint64_t>(cnt, st);
  double2* a3 = dalloc<double2>(cnt, st);
  uint8_t* flag = dalloc<uint8_t>(cnt, st);
  int* d_num = dalloc<int>(2, st);
  size_t t1 = 0, t2 = 0, t3 = 0, t4 = 0;
  const int end_bit = int(std::max<uint32_t>(1, s->n));
  NCSIM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, key, k2, amp, a2, num, 0, end_bit, st));
  NCSIM_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, t2, k2, k3, a2, a3, d_num, ZAdd(), num, st));
  NCSIM_CUDA(cub::DeviceSelect::Flagged(nullptr, t3, k3, flag, key, d_num + 1, num, st));
  NCSIM_CUDA(cub::DeviceSelect::Flagged(nullptr, t4, a3, flag, amp, d_num + 1, num, st));
  const size_t tb = std::max(std::max(t1, t2), std::max(t3, t4));
  void* tmp = dalloc<uint8_t>(tb, st);
  int kept = 0;
  if (num > 0) {
    NCSIM_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t1, key, k2, amp, a2, num, 0, end_bit, st));
    NCSIM_CUDA(cub::DeviceReduce::ReduceByKey(tmp, t2, k2, k3, a2, a3, d_num, ZAdd(), num, st));
    // the run count stays on the device: the keep flags drop the positions past it
    k_sp_keep<<<sp_grid(cnt), SP_THREADS, 0, st>>>(a3, d_num, cnt, s->cutoff * s->cutoff, flag);
    NCSIM_LAUNCHED("sparse keep");
    NCSIM_CUDA(cub::DeviceSelect::Flagged(tmp, t3, k3, flag, key, d_num + 1, num, st));
    NCSIM_CUDA(cub::DeviceSelect::Flagged(tmp, t4, a3, flag, amp, d_num + 1, num, st));
    NCSIM_CUDA(cudaMemcpyAsync(&kept, d_num + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    NCSIM_CUDA(cudaStreamSynchronize(st));
  }
  dfree(tmp, st);
  dfree(k2, st);
  dfree(a2, st);
  dfree(k3, st);
  dfree(a3, st);
  dfree(flag, st);
  dfree(d_num, st);
  dfree(s->key, st);
  dfree(s->amp, st);
  s->key = key;
  s->amp = amp;
  s->cap = std::max<uint64_t>(cnt, 1);
  s->m = uint64_t(kept);
  s->sorted = true;
}

void sp_normalize(ncsim_sparse* s) {
  if (s->words > 1) return spw::normalize(s);
  cudaStream_t st = s->stream;
  uint64_t* k = dalloc<uint64_t>(s->m, st);
  double2* a = dalloc<double2>(s->m, st);
  if (s->m) {
    NCSIM_CUDA(cudaMemcpyAsync(k, s->key, s->m * 8, cudaMemcpyDeviceToDevice, st));
    NCSIM_CUDA(cudaMemcpyAsync(a, s->amp, s->m * 16, cudaMemcpyDeviceToDevice, st));
  }
  sp_normalize_from(s, k, a, s->m);
}

// a sorted copy of m entries of an n-qubit register, made on stream st (owned by
// the caller, stream-ordered)
void sorted_copy(const uint64_t* key, const double2* amp, uint64_t m, uint32_t n, cudaStream_t st, uint64_t*& k,
                 double2*& a) {
  k = dalloc<uint64_t>(m, st);
  a = dalloc<double2>(m, st);
  if (!m) return;
  size_t tb = 0;
  const int num = int(m);
  const int end_bit = int(std::max<uint32_t>(1, n));
  NCSIM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, k, amp, a, num, 0, end_bit, st));
  void* tmp = dalloc<uint8_t>(tb, st);
  NCSIM_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, k, amp, a, num, 0, end_bit, st));
  dfree(tmp, st);
}
void sp_sorted_copy(const ncsim_sparse* s, uint64_t*& k, double2*& a) {
  sorted_copy(s->key, s->amp, s->m, s->n, s->stream, k, a);
}

void sp_sort(ncsim_sparse* s) {
  if (s->sorted) return;
  if (s->words > 1) return spw::sort(s);
  uint64_t* k;
  double2* a;
  sp_sorted_copy(s, k, a);
  dfree(s->key, s->stream);
  dfree(s->amp, s->stream);
  s->key = k;
  s->amp = a;
  s->cap = std::max<uint64_t>(s->m, 1);
  s->sorted = true;
}


void sp_expect(const ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, double* out) {
  const uint64_t* k = s->key;
  const double2* a = s->amp;
  uint64_t* kc = nullptr;
  double2* ac = nullptr;
  if (x && !s->sorted) {  // the sorted view (a copy, the entries keep their order)
    sp_sorted_copy(s, kc, ac);
    k = kc;
    a = ac;
  }
  const unsigned g = red_grid(s->m);
  k_sp_expect<<<g, SP_THREADS, 0, s->stream>>>(k, a, s->m, x, z, phase, s->partials);
  NCSIM_LAUNCHED("sparse expectation");
  sp_sum(s, g, out);
  dfree(kc, s->stream);
  dfree(ac, s->stream);
}

// a gate's monomial view: image and phases per local pattern
void sp_monomial(ncsim_sparse* s, const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& image,
                 const std::vector<CplxD>& phase) {
  const uint32_t k = uint32_t(qubits.size());
  if (k > SP_MAX_K) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse monomial gate on more than 10 qubits");
  Qubits qs{};
  qs.k = k;
  for (uint32_t j = 0; j < k; ++j) qs.q[j] = uint8_t(qubits[j]);
  const size_t gd = size_t(1) << k;
  std::vector<double2> ph(gd);
  std::vector<uint8_t> unit(gd);
  bool moves = false;
  for (size_t x = 0; x < gd; ++x) {
    ph[x] = make_double2(phase[x].re, phase[x].im);
    unit[x] = phase[x].re == 1.0 && phase[x].im == 0.0;
    moves |= image[x] != x;
  }
  if (s->m && gd <= 256) {
    auto launch = [&](auto& P) {
      P.qs = qs;
      for (size_t x = 0; x < gd; ++x) {
        P.image[x] = uint16_t(image[x]);
        P.phase[x] = ph[x];
        if (unit[x]) P.unit[x >> 5] |= 1u << (x & 31);
      }
      return &P;
    };
    if (gd <= 16) {
      MonoParams<16> P{};
      k_sp_monomial_p<16><<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(s->key, s->amp, s->m, *launch(P));
    } else {
      MonoParams<256> P{};
      k_sp_monomial_p<256><<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(s->key, s->amp, s->m, *launch(P));
    }
    NCSIM_LAUNCHED("sparse monomial");
  } else if (s->m) {
    cudaStream_t st = s->stream;
    uint32_t* di = upload(image, st);
    double2* dp = upload(ph, st);
    uint8_t* du = upload(unit, st);
    k_sp_monomial<<<sp_grid(s->m), SP_THREADS, 0, st>>>(s->key, s->amp, s->m, qs, di, dp, du);
    NCSIM_LAUNCHED("sparse monomial");
    dfree(di, st);
    dfree(dp, st);
    dfree(du, st);
  }
  if (moves) s->sorted = false;
}

// a dense matrix (row-major 2^k x 2^k): permutations with phases in place, others by expansion
void sp_matrix(ncsim_sparse* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& mat) {
  const uint32_t k = uint32_t(qubits.size());
  if (k > SP_MAX_K) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse dense gate on more than 10 qubits");
  const size_t gd = size_t(1) << k;
  std::vector<uint32_t> col_start(gd + 1, 0), col_row;
  std::vector<double2> col_val;
  for (size_t b = 0; b < gd; ++b) {
    col_start[b] = uint32_t(col_row.size());
    for (size_t a = 0; a < gd; ++a) {
      const CplxD e = mat[a * gd + b];
      if (e.re == 0.0 && e.im == 0.0) continue;
      col_row.push_back(uint32_t(a));
      col_val.push_back(make_double2(e.re, e.im));
    }
  }
  col_start[gd] = uint32_t(col_row.size());
  // one nonzero per column on distinct rows: every entry moves to one entry
  bool perm = col_row.size() == gd;
  for (size_t b = 0; b < gd && perm; ++b) perm = col_start[b + 1] - col_start[b] == 1;
  if (perm) {
    std::vector<uint32_t> rows(col_row);
    std::sort(rows.begin(), rows.end());
    perm = std::adjacent_find(rows.begin(), rows.end()) == rows.end();
  }
  if (perm) {
    std::vector<CplxD> ph(gd);
    for (size_t b = 0; b < gd; ++b) ph[b] = CplxD{col_val[b].x, col_val[b].y};
    sp_monomial(s, qubits, col_row, ph);
    return;
  }
  Qubits qs{};
  qs.k = k;
  for (uint32_t j = 0; j < k; ++j) qs.q[j] = uint8_t(qubits[j]);
  cudaStream_t st = s->stream;
  const uint64_t m = s->m;
  if (m > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  uint32_t* dcs = upload(col_start, st);
  uint32_t* dcr = upload(col_row, st);
  double2* dcv = upload(col_val, st);
  // every column with the same count (H, SQRT_X, rotations): entry i's images start at i * per,
  // so the counts, their scan and the host's wait for the total are not needed
  const uint32_t per = col_start[1] - col_start[0];
  bool uniform = true;
  for (size_t b = 0; b < gd && uniform; ++b) uniform = col_start[b + 1] - col_start[b] == per;
  uint32_t* cnt = uniform ? nullptr : dalloc<uint32_t>(m + 1, st);
  uint32_t* off = uniform ? nullptr : dalloc<uint32_t>(m + 1, st);
  uint64_t total = uniform ? m * per : 0;
  if (m && !uniform) {
    k_sp_count<<<sp_grid(m), SP_THREADS, 0, st>>>(s->key, m, qs, dcs, cnt);
    NCSIM_LAUNCHED("sparse count");
    NCSIM_CUDA(cudaMemsetAsync(cnt + m, 0, sizeof(uint32_t), st));
    size_t tb = 0;
    NCSIM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, int(m + 1), st));
    void* tmp = dalloc<uint8_t>(tb, st);
    NCSIM_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, int(m + 1), st));
    uint32_t t32 = 0;
    NCSIM_CUDA(cudaMemcpyAsync(&t32, off + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    NCSIM_CUDA(cudaStreamSynchronize(st));
    dfree(tmp, st);
    total = t32;
  }
  if (total > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  uint64_t* okey = dalloc<uint64_t>(total, st);
  double2* oamp = dalloc<double2>(total, st);
  if (total) {
    k_sp_expand<<<sp_grid(m), SP_THREADS, 0, st>>>(s->key, s->amp, m, qs, dcs, dcr, dcv, off, per, okey, oamp);
    NCSIM_LAUNCHED("sparse expand");
  }
  dfree(dcs, st);
  dfree(dcr, st);
  dfree(dcv, st);
  dfree(cnt, st);
  dfree(off, st);
  sp_normalize_from(s, okey, oamp, total);
}

// the host side of a run: ops and their tables, launched in one kernel
struct RunBuilder {
  std::vector<RunOp> ops;
  std::vector<uint16_t> image;
  std::vector<double2> phase;
  std::vector<uint8_t> unit;
  std::vector<double2> table;
  std::vector<uint32_t> start;
  std::vector<uint64_t> par, coeff, and_mask;
  bool moves = false;

  bool empty() const { return ops.empty(); }
  // empties the builder and keeps its buffers' capacity for the next run
  void reset() {
    ops.clear();
    image.clear();
    phase.clear();
    unit.clear();
    table.clear();
    start.clear();
    par.clear();
    coeff.clear();
    and_mask.clear();
    moves = false;
  }
  void add_mono(const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& img, const std::vector<CplxD>& ph) {
    RunOp op{};
    op.type = RUN_MONO;
    op.k = uint32_t(qubits.size());
    for (uint32_t j = 0; j < op.k; ++j) op.q[j] = uint8_t(qubits[j]);
    op.off = uint32_t(image.size());
    for (size_t x = 0; x < img.size(); ++x) {
      image.push_back(uint16_t(img[x]));
      phase.push_back(make_double2(ph[x].re, ph[x].im));
      const bool one = ph[x].re == 1.0 && ph[x].im == 0.0;
      unit.push_back(one);
      moves |= img[x] != x;
      if (op.k <= 3) {
        (x < 4 ? op.img_lo : op.img_hi) |= uint64_t(img[x]) << (16 * (x & 3));
        op.unit8 |= uint64_t(one) << (8 * x);
      }
    }
    ops.push_back(op);
  }
  void add_poly(const PolyTerms& t) {
    RunOp op{};
    op.type = RUN_POLY;
    op.k = uint32_t(t.coeffs.size());
    op.bits = t.bits;
    op.x = t.constant;
    op.scalar = make_double2(t.scalar.re, t.scalar.im);
    op.flags = (t.scalar_is_one ? 1u : 0u) | (t.root_table.empty() ? 0u : 2u);
    op.off = uint32_t(start.size());
    const uint32_t pbase = uint32_t(par.size());
    for (size_t i = 0; i < t.coeffs.size(); ++i) {
      start.push_back(pbase + (t.term_start.empty() ? 0 : t.term_start[i]));
      coeff.push_back(t.coeffs[i]);
      uint64_t am = 0;
      bool single = !t.term_start.empty() && t.term_start[i + 1] > t.term_start[i];
      for (uint32_t l = single ? t.term_start[i] : 0; single && l < t.term_start[i + 1]; ++l) {
        single = __builtin_popcountll(t.parities[l]) == 1;
        am |= t.parities[l];
      }
      and_mask.push_back(single ? am : 0);
    }
    start.push_back(pbase + (t.term_start.empty() ? 0 : t.term_start[t.coeffs.size()]));
    // start[] holds nterms + 1 entries per polynomial, coeff[] and and_mask[] nterms: keep them aligned
    coeff.push_back(0);
    and_mask.push_back(0);
    for (uint64_t pm : t.parities) par.push_back(pm);
    op.toff = uint32_t(table.size());
    for (const CplxD& c : t.root_table) table.push_back(make_double2(c.re, c.im));
    ops.push_back(op);
  }
  void add_pauli(uint64_t x, uint64_t z, uint32_t ph) {
    RunOp op{};
    op.type = RUN_PAULI;
    op.x = x;
    op.z = z;
    op.flags = ph & 3u;
    moves |= x != 0;
    ops.push_back(op);
  }
  void launch(ncsim_sparse* s) {
    if (ops.empty()) return;
    cudaStream_t st = s->stream;
    if (s->m) {
      RunOp* d_ops = upload(ops, st);
      uint16_t* d_img = upload(image, st);
      double2* d_ph = upload(phase, st);
      uint8_t* d_unit = upload(unit, st);
      double2* d_tab = upload(table, st);
      uint32_t* d_start = upload(start, st);
      uint64_t* d_par = upload(par, st);
      uint64_t* d_coeff = upload(coeff, st);
      uint64_t* d_and = upload(and_mask, st);
      RunData d{d_ops, uint32_t(ops.size()), d_img, d_ph, d_unit, d_tab, d_start, d_par, d_coeff, d_and};
      k_sp_run<<<sp_grid(s->m), SP_THREADS, 0, st>>>(s->key, s->amp, s->m, d);
      NCSIM_LAUNCHED("sparse run");
      dfree(d_ops, st);
      dfree(d_img, st);
      dfree(d_ph, st);
      dfree(d_unit, st);
      dfree(d_tab, st);
      dfree(d_start, st);
      dfree(d_par, st);
      dfree(d_coeff, st);
      dfree(d_and, st);
    }
    if (moves) s->sorted = false;
    reset();
  }
};

void sp_pauli(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase) {
  if (s->m) {
    k_sp_pauli<<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(s->key, s->amp, s->m, x, z, phase & 3u);
    NCSIM_LAUNCHED("sparse pauli");
  }
  if (x) s->sorted = false;
}

void sp_phasepoly(ncsim_sparse* s, const PolyTerms& t) {
  if (!s->m) return;
  cudaStream_t st = s->stream;
  if (t.coeffs.size() <= size_t(SP_POLY_TERMS) && t.parities.size() <= size_t(SP_POLY_PARS) &&
      t.root_table.size() <= 256) {
    auto P = std::make_unique<PolyParamsSp>();
    P->bits = t.bits;
    P->nterms = uint32_t(t.coeffs.size());
    P->constant = t.constant;
    P->scalar = make_double2(t.scalar.re, t.scalar.im);
    P->scalar_is_one = t.scalar_is_one;
    P->use_table = !t.root_table.empty();
    for (size_t i = 0; i < t.term_start.size(); ++i) P->start[i] = uint16_t(t.term_start[i]);
    if (t.term_start.empty()) P->start[0] = 0;
    for (size_t i = 0; i < t.parities.size(); ++i) P->par[i] = t.parities[i];
    for (size_t i = 0; i < t.coeffs.size(); ++i) P->coeff[i] = t.coeffs[i];
    for (size_t i = 0; i < t.root_table.size(); ++i) P->table[i] = make_double2(t.root_table[i].re, t.root_table[i].im);
    k_sp_phasepoly_p<<<sp_grid(s->m), SP_THREADS, 0, st>>>(s->key, s->amp, s->m, *P);
    NCSIM_LAUNCHED("sparse phasepoly");
    return;
  }
  SpPoly P{};
  P.bits = t.bits;
  P.nterms = uint32_t(t.coeffs.size());
  P.constant = t.constant;
  P.scalar = make_double2(t.scalar.re, t.scalar.im);
  P.scalar_is_one = t.scalar_is_one;
  P.use_table = !t.root_table.empty();
  std::vector<double2> tab(t.root_table.size());
  for (size_t i = 0; i < tab.size(); ++i) tab[i] = make_double2(t.root_table[i].re, t.root_table[i].im);
  uint32_t* ds = upload(t.term_start.empty() ? std::vector<uint32_t>{0} : t.term_start, st);
  uint64_t* dp = upload(t.parities, st);
  uint64_t* dc = upload(t.coeffs, st);
  double2* dt = upload(tab, st);
  P.start = ds;
  P.par = dp;
  P.coeff = dc;
  P.table = dt;
  k_sp_phasepoly<<<sp_grid(s->m), SP_THREADS, 0, st>>>(s->key, s->amp, s->m, P);
  NCSIM_LAUNCHED("sparse phasepoly");
  dfree(ds, st);
  dfree(dp, st);
  dfree(dc, st);
  dfree(dt, st);
}

void sp_apply_lowered(ncsim_sparse* s, const LoweredOp& op) {
  switch (op.kind) {
    case LoweredKind::Nothing: return;
    case LoweredKind::Dense: sp_matrix(s, op.qubits, op.matrix); return;
    case LoweredKind::Monomial: sp_monomial(s, op.qubits, op.image, op.matrix); return;
    case LoweredKind::PhasePoly: sp_phasepoly(s, op.poly); return;
    case LoweredKind::Pauli: sp_pauli(s, op.x, op.z, op.phase); return;
  }
}

double sp_project(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, bool outcome) {
  cudaStream_t st = s->stream;
  const uint64_t m = s->m;
  uint64_t* okey = dalloc<uint64_t>(2 * m, st);
  double2* oamp = dalloc<double2>(2 * m, st);
  if (m) {
    k_sp_project<<<sp_grid(m), SP_THREADS, 0, st>>>(s->key, s->amp, m, x, z, phase & 3u, outcome ? -1.0 : 1.0, okey,
                                                    oamp);
    NCSIM_LAUNCHED("sparse project");
  }
  sp_normalize_from(s, okey, oamp, 2 * m);
  return sp_norm(s);
}

// QuantumState::measure (mod.rs:113-131)
bool sp_measure(ncsim_sparse* s, const PauliOp& p, ncsim_rng& rng) {
  if (!p.hermitian()) throw Error(NCSIM_ERR_INVALID, "measured operator is not Hermitian");
  if (p.n != s->n) throw Error(NCSIM_ERR_INVALID, "expectation: operator on the wrong register");
  double e[2];
  sp_expect(s, p.x, p.z, p.phase, e);
  const double nn = sp_norm(s);
  double p_plus = (1.0 + e[0] / nn) / 2.0;
  if (!std::isnan(p_plus)) p_plus = std::min(1.0, std::max(0.0, p_plus));
  bool outcome;
  if (p_plus > 1.0 - 1e-12) outcome = false;
  else if (p_plus < 1e-12) outcome = true;
  else outcome = rng.f64() >= p_plus;
  sp_project(s, p.x, p.z, p.phase, outcome);
  return outcome;
}

// QuantumState::apply_op (mod.rs:134-165); -1, 0 or 1
int sp_apply_op(ncsim_sparse* s, const OpIR& op, ncsim_rng& rng) {
  switch (op.kind) {
    case OpKind::Gate: sp_apply_lowered(s, op.lowered); return -1;
    case OpKind::Measure: return sp_measure(s, op.pauli, rng) ? 1 : 0;
    case OpKind::Reset: {
      PauliOp z;
      z.n = s->n;
      z.z = uint64_t(1) << op.qubits[0];
      if (sp_measure(s, z, rng)) sp_pauli(s, uint64_t(1) << op.qubits[0], 0, 0);
      return -1;
    }
    case OpKind::Noise: {
      const int e = op.noise.sample(rng);
      if (e >= 0) {
        uint64_t x = 0, z = 0;
        for (size_t j = 0; j < op.qubits.size(); ++j) {
          x |= uint64_t((e >> j) & 1) << op.qubits[j];
          z |= uint64_t((e >> (8 + j)) & 1) << op.qubits[j];
        }
        sp_pauli(s, x, z, 0);
      }
      return -1;
    }
    default: return -1;
  }
}

ncsim_sparse* sp_new(uint32_t n) {
  const uint32_t words = spw::words_for(n);  // checks 1 <= n <= 1024
  auto s = std::make_unique<ncsim_sparse>();
  s->n = n;
  s->words = words;
  NCSIM_CUDA(cudaGetDevice(&s->device));
  NCSIM_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  NCSIM_CUDA(cudaMalloc(&s->partials, SP_BLOCKS * 2 * sizeof(double)));
  NCSIM_CUDA(cudaMallocHost(&s->host_partials, SP_BLOCKS * 2 * sizeof(double)));
  NCSIM_CUDA(cudaEventCreate(&s->timer0));
  NCSIM_CUDA(cudaEventCreate(&s->timer1));
  return s.release();
}

void sp_release(ncsim_sparse* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaFree(s->key);
  cudaFree(s->amp);
  cudaFree(s->partials);
  cudaFreeHost(s->host_partials);
  if (s->timer0) cudaEventDestroy(s->timer0);
  if (s->timer1) cudaEventDestroy(s->timer1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

void set_entries(ncsim_sparse* s, const uint64_t* keys, const double* amps, uint64_t count) {
  if (s->words > 1) return spw::set_entries(s, keys, amps, count);
  const uint64_t mask = s->n >= 64 ? ~uint64_t(0) : (uint64_t(1) << s->n) - 1;
  std::vector<uint64_t> k(count);
  for (uint64_t i = 0; i < count; ++i) k[i] = keys[i] & mask;
  uint64_t* dk = upload(k, s->stream);
  double2* da = dalloc<double2>(count, s->stream);
  if (count) NCSIM_CUDA(cudaMemcpyAsync(da, amps, count * 16, cudaMemcpyHostToDevice, s->stream));
  sp_normalize_from(s, dk, da, count);
}


// a one-word mask on a register of any width (qubits 0..63)
std::vector<uint64_t> word0(const ncsim_sparse* s, uint64_t v) {
  std::vector<uint64_t> w(s->words, 0);
  w[0] = v;
  return w;
}
// checks a caller's word arrays: their count is the register's and no bit lies outside it
void check_words(const ncsim_sparse* s, uint32_t words, std::initializer_list<const uint64_t*> masks) {
  if (words != s->words)
    throw Error(NCSIM_ERR_INVALID, "masks of " + std::to_string(words) + " words on a register keyed by " +
                                       std::to_string(s->words));
  for (const uint64_t* m : masks) {
    need(m, "mask");
    for (uint32_t w = 0; w < words; ++w) {
      const uint32_t lo = 64 * w;
      const uint64_t keep = s->n >= lo + 64 ? ~uint64_t(0) : s->n <= lo ? 0 : (uint64_t(1) << (s->n - lo)) - 1;
      if (m[w] & ~keep) throw Error(NCSIM_ERR_INVALID, "Pauli on qubits outside the register");
    }
  }
}

}  // namespace

extern "C" {

ncsim_status ncsim_sparse_create(uint32_t n, ncsim_sparse** out) {
  return guarded([&] {
    need(out, "out");
    ncsim_sparse* s = sp_new(n);
    try {
      const std::vector<uint64_t> zero(s->words, 0);
      const double one[2] = {1.0, 0.0};
      set_entries(s, zero.data(), one, 1);
    } catch (...) {
      sp_release(s);
      throw;
    }
    *out = s;
  });
}

ncsim_status ncsim_sparse_from_entries(uint32_t n, const uint64_t* keys, const double* amps, uint64_t count,
                                       ncsim_sparse** out) {
  return guarded([&] {
    need(out, "out");
    if (count) {
      need(keys, "keys");
      need(amps, "amps");
    }
    ncsim_sparse* s = sp_new(n);
    try {
      set_entries(s, keys, amps, count);
    } catch (...) {
      sp_release(s);
      throw;
    }
    *out = s;
  });
}

ncsim_status ncsim_sparse_destroy(ncsim_sparse* s) {
  return guarded([&] { sp_release(s); });
}

ncsim_status ncsim_sparse_clone(const ncsim_sparse* s, ncsim_sparse** out) {
  return guarded([&] {
    need(s, "state");
    need(out, "out");
    Lock lk(s);
    ncsim_sparse* c = sp_new(s->n);
    try {
      c->cutoff = s->cutoff;
      NCSIM_CUDA(cudaStreamSynchronize(s->stream));
      sp_reserve(c, s->m);
      if (s->m) {
        NCSIM_CUDA(cudaMemcpyAsync(c->key, s->key, s->m * 8 * s->words, cudaMemcpyDeviceToDevice, c->stream));
        NCSIM_CUDA(cudaMemcpyAsync(c->amp, s->amp, s->m * 16, cudaMemcpyDeviceToDevice, c->stream));
      }
      c->m = s->m;
      c->sorted = s->sorted;
      NCSIM_CUDA(cudaStreamSynchronize(c->stream));
    } catch (...) {
      sp_release(c);
      throw;
    }
    *out = c;
  });
}

ncsim_status ncsim_sparse_set_cutoff(ncsim_sparse* s, double cutoff) {
  return guarded([&] {
    need(s, "state");
    if (!(cutoff >= 0.0)) throw Error(NCSIM_ERR_INVALID, "cutoff must be >= 0");
    Lock lk(s);
    s->cutoff = cutoff;
    sp_normalize(s);
  });
}

ncsim_status ncsim_sparse_num_qubits(const ncsim_sparse* s, uint32_t* n) {
  return guarded([&] {
    need(s, "state");
    need(n, "n");
    *n = s->n;
  });
}

ncsim_status ncsim_sparse_num_entries(const ncsim_sparse* s, uint64_t* count) {
  return guarded([&] {
    need(s, "state");
    need(count, "count");
    *count = s->m;
  });
}

ncsim_status ncsim_sparse_get_entries(const ncsim_sparse* s, uint64_t* keys, double* amps, uint64_t cap) {
  return guarded([&] {
    need(s, "state");
    Lock lk(s);
    if (cap < s->m) throw Error(NCSIM_ERR_INVALID, "entry buffers too small");
    if (s->m) {
      need(keys, "keys");
      need(amps, "amps");
      NCSIM_CUDA(cudaMemcpyAsync(keys, s->key, s->m * 8 * s->words, cudaMemcpyDeviceToHost, s->stream));
      NCSIM_CUDA(cudaMemcpyAsync(amps, s->amp, s->m * 16, cudaMemcpyDeviceToHost, s->stream));
    }
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  });
}

ncsim_status ncsim_sparse_sort(ncsim_sparse* s) {
  return guarded([&] {
    need(s, "state");
    Lock lk(s);
    sp_sort(s);
  });
}

ncsim_status ncsim_sparse_apply_gate(ncsim_sparse* s, const ncsim_gate* g, const uint32_t* qubits, uint32_t k) {
  return guarded([&] {
    need(s, "state");
    need(g, "gate");
    if (k) need(qubits, "qubits");
    Lock lk(s);
    if (s->words > 1) return spw::apply_gate(s, g->g, std::vector<uint32_t>(qubits, qubits + k));
    const LoweredOp op = lower_gate(g->g, std::vector<uint32_t>(qubits, qubits + k), s->n);
    sp_apply_lowered(s, op);
  });
}

ncsim_status ncsim_sparse_apply_pauli(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase) {
  return guarded([&] {
    need(s, "state");
    const uint64_t mask = s->n >= 64 ? ~uint64_t(0) : (uint64_t(1) << s->n) - 1;
    if ((x | z) & ~mask) throw Error(NCSIM_ERR_INVALID, "Pauli on qubits outside the register");
    Lock lk(s);
    if (s->words > 1) return spw::pauli(s, word0(s, x).data(), word0(s, z).data(), phase);
    sp_pauli(s, x, z, phase);
  });
}

ncsim_status ncsim_sparse_norm_sq(const ncsim_sparse* s, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    Lock lk(s);
    re_im[0] = sp_norm(s);
    re_im[1] = 0.0;
  });
}

ncsim_status ncsim_sparse_amplitude(const ncsim_sparse* s, uint64_t index, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    Lock lk(s);
    if (s->words > 1) return spw::amplitude(s, word0(s, index).data(), re_im);
    const uint64_t mask = s->n >= 64 ? ~uint64_t(0) : (uint64_t(1) << s->n) - 1;
    double2* d = dalloc<double2>(1, s->stream);
    k_sp_find<<<1, 32, 0, s->stream>>>(s->key, s->amp, s->m, index & mask, s->sorted ? 1 : 0, d);
    NCSIM_LAUNCHED("sparse amplitude");
    double2 h;
    NCSIM_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    dfree(d, s->stream);
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    re_im[0] = h.x;
    re_im[1] = h.y;
  });
}

ncsim_status ncsim_sparse_expectation(const ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    const uint64_t mask = s->n >= 64 ? ~uint64_t(0) : (uint64_t(1) << s->n) - 1;
    if ((x | z) & ~mask) throw Error(NCSIM_ERR_INVALID, "expectation: operator on the wrong register");
    Lock lk(s);
    if (s->words > 1) return spw::expectation(s, word0(s, x).data(), word0(s, z).data(), phase & 3u, re_im);
    sp_expect(s, x, z, phase & 3u, re_im);
  });
}

ncsim_status ncsim_sparse_inner(const ncsim_sparse* a, const ncsim_sparse* b, double* re_im) {
  return guarded([&] {
    need(a, "a");
    need(b, "b");
    need(re_im, "out");
    if (a->n != b->n) throw Error(NCSIM_ERR_INVALID, "inner: register sizes differ");
    PairLock lk(a, b);
    NCSIM_CUDA(cudaStreamSynchronize(b->stream));
    if (a->words > 1) return spw::inner(a, b, re_im);
    uint64_t* kb = b->key;
    double2* vb = b->amp;
    uint64_t* kc = nullptr;
    double2* vc = nullptr;
    if (!b->sorted) {  // b's sorted view, made on a's stream
      sorted_copy(b->key, b->amp, b->m, b->n, a->stream, kc, vc);
      kb = kc;
      vb = vc;
    }
    const unsigned g = red_grid(a->m);
    k_sp_inner<<<g, SP_THREADS, 0, a->stream>>>(a->key, a->amp, a->m, kb, vb, b->m, a->partials);
    NCSIM_LAUNCHED("sparse inner");
    sp_sum(a, g, re_im);
    dfree(kc, a->stream);
    dfree(vc, a->stream);
  });
}

ncsim_status ncsim_sparse_project(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, int32_t outcome,
                                  double* weight_re_im) {
  return guarded([&] {
    need(s, "state");
    PauliOp p;
    p.n = s->n;
    p.x = x;
    p.z = z;
    p.phase = phase & 3u;
    if (!p.hermitian()) throw Error(NCSIM_ERR_INVALID, "projector of a non-Hermitian Pauli");
    Lock lk(s);
    const double w = s->words > 1 ? spw::project(s, word0(s, x).data(), word0(s, z).data(), phase, outcome != 0)
                                  : sp_project(s, x, z, phase, outcome != 0);
    if (weight_re_im) weight_re_im[0] = w, weight_re_im[1] = 0.0;
  });
}

ncsim_status ncsim_sparse_scale(ncsim_sparse* s, double re, double im) {
  return guarded([&] {
    need(s, "state");
    Lock lk(s);
    if (s->m) {
      k_sp_scale<<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(s->amp, s->m, make_double2(re, im));
      NCSIM_LAUNCHED("sparse scale");
    }
    sp_normalize(s);
  });
}

ncsim_status ncsim_sparse_tensor(const ncsim_sparse* a, const ncsim_sparse* b, ncsim_sparse** out) {
  return guarded([&] {
    need(a, "a");
    need(b, "b");
    need(out, "out");
    if (a->n + b->n > spw::MAX_QUBITS)
      throw Error(NCSIM_ERR_UNSUPPORTED, "sparse tensor product of more than " + std::to_string(spw::MAX_QUBITS) + " qubits");
    PairLock lk(a, b);
    NCSIM_CUDA(cudaStreamSynchronize(a->stream));
    NCSIM_CUDA(cudaStreamSynchronize(b->stream));
    if (a->n + b->n > 64) {  // keys of several words
      ncsim_sparse* c = sp_new(a->n + b->n);
      try {
        c->cutoff = a->cutoff;
        spw::tensor(a, b, c);
        NCSIM_CUDA(cudaStreamSynchronize(c->stream));
      } catch (...) {
        sp_release(c);
        throw;
      }
      *out = c;
      return;
    }
    const uint64_t tot = a->m * b->m;
    if (tot > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
    ncsim_sparse* c = sp_new(a->n + b->n);
    try {
      c->cutoff = a->cutoff;
      sp_reserve(c, tot);
      if (tot) {
        k_sp_tensor<<<sp_grid(tot), SP_THREADS, 0, c->stream>>>(a->key, a->amp, a->m, a->n, b->key, b->amp, b->m,
                                                                 c->key, c->amp);
        NCSIM_LAUNCHED("sparse tensor");
      }
      c->m = tot;
      c->sorted = false;
      NCSIM_CUDA(cudaStreamSynchronize(c->stream));
    } catch (...) {
      sp_release(c);
      throw;
    }
    *out = c;
  });
}

ncsim_status ncsim_sparse_sample(const ncsim_sparse* s, ncsim_rng* rng, uint64_t shots, uint64_t* out) {
  return guarded([&] {
    need(s, "state");
    need(rng, "rng");
    if (shots) need(out, "out");
    Lock lk(s);
    if (s->words > 1) return spw::sample(s, *rng, shots, out);
    std::vector<double> w(s->m);
    std::vector<uint64_t> keys(s->m);
    if (s->m) {
      double* dw = dalloc<double>(s->m, s->stream);
      k_sp_abs2<<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(s->amp, s->m, dw);
      NCSIM_LAUNCHED("sparse weights");
      NCSIM_CUDA(cudaMemcpyAsync(w.data(), dw, s->m * 8, cudaMemcpyDeviceToHost, s->stream));
      NCSIM_CUDA(cudaMemcpyAsync(keys.data(), s->key, s->m * 8, cudaMemcpyDeviceToHost, s->stream));
      dfree(dw, s->stream);
      NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    }
    // cumulative weights in entry order, a draw per shot (sparse.rs:407-424)
    double acc = 0.0;
    for (double& v : w) {
      acc += v;
      v = acc;
    }
    if (acc <= 0.0) throw Error(NCSIM_ERR_ZERO_STATE, "sample: the state vanished");
    for (uint64_t k = 0; k < shots; ++k) {
      const double u = rng->f64() * acc;
      size_t i = size_t(std::upper_bound(w.begin(), w.end(), u) - w.begin());
      if (i >= w.size()) i = w.size() - 1;
      out[k] = keys[i];
    }
  });
}

ncsim_status ncsim_sparse_to_vector(const ncsim_sparse* s, double* amps, uint64_t len) {
  return guarded([&] {
    need(s, "state");
    need(amps, "amps");
    if (s->n > 26) throw Error(NCSIM_ERR_UNSUPPORTED, "dense vector of more than 26 qubits");
    if (len != (uint64_t(1) << s->n)) throw Error(NCSIM_ERR_INVALID, "amplitude buffer length differs from 2^n");
    Lock lk(s);
    std::vector<uint64_t> k(s->m);
    std::vector<double2> a(s->m);
    if (s->m) {
      NCSIM_CUDA(cudaMemcpyAsync(k.data(), s->key, s->m * 8, cudaMemcpyDeviceToHost, s->stream));
      NCSIM_CUDA(cudaMemcpyAsync(a.data(), s->amp, s->m * 16, cudaMemcpyDeviceToHost, s->stream));
    }
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    std::memset(amps, 0, size_t(len) * 16);
    for (uint64_t i = 0; i < s->m; ++i) amps[2 * k[i]] = a[i].x, amps[2 * k[i] + 1] = a[i].y;
  });
}

ncsim_status ncsim_sparse_measure(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, ncsim_rng* rng,
                                  int32_t* outcome) {
  return guarded([&] {
    need(s, "state");
    need(rng, "rng");
    Lock lk(s);
    PauliOp p;
    p.n = s->n;
    p.x = x;
    p.z = z;
    p.phase = phase & 3u;
    const bool o = s->words > 1 ? spw::measure(s, word0(s, x).data(), word0(s, z).data(), phase & 3u, *rng)
                                : sp_measure(s, p, *rng);
    if (outcome) *outcome = o ? 1 : 0;
  });
}

ncsim_status ncsim_sparse_run(ncsim_sparse* s, const ncsim_circuit* c, ncsim_rng* rng, uint8_t* rec, size_t cap,
                              size_t* len) {
  return guarded([&] {
    need(s, "state");
    need(c, "circuit");
    need(rng, "rng");
    if (c->n != s->n) throw Error(NCSIM_ERR_INVALID, "circuit on a different register");
    if (c->num_measurements() > cap) throw Error(NCSIM_ERR_INVALID, "record buffer too small");
    if (c->num_measurements()) need(rec, "record");
    Lock lk(s);
    size_t m = 0;
    if (s->words > 1) {
      spw::run(s, *c, *rng, rec, m);
      NCSIM_CUDA(cudaStreamSynchronize(s->stream));
      if (len) *len = m;
      return;
    }
    // runs of one-to-one ops (gates with a monomial, diagonal or Pauli view, and the
    // Paulis of sampled noise) go to the device as one pass each; a measurement, a
    // reset or a gate that creates entries ends a run
    // one builder per host thread, reused so that its tables keep their capacity across runs
    static thread_local RunBuilder run;
    run.reset();
    std::vector<uint32_t> img;
    std::vector<CplxD> ph;
    for (const OpIR& op : c->ops) {
      if (op.kind == OpKind::Gate) {
        const LoweredOp& lo = op.lowered;
        switch (lo.kind) {
          case LoweredKind::Nothing: continue;
          case LoweredKind::Monomial:
            if (lo.qubits.size() <= SP_MAX_K) {
              run.add_mono(lo.qubits, lo.image, lo.matrix);
              continue;
            }
            break;
          case LoweredKind::PhasePoly: run.add_poly(lo.poly); continue;
          case LoweredKind::Pauli: run.add_pauli(lo.x, lo.z, lo.phase); continue;
          case LoweredKind::Dense:
            if (lo.qubits.size() <= SP_MAX_K && permutation_view(lo.matrix, size_t(1) << lo.qubits.size(), img, ph)) {
              run.add_mono(lo.qubits, img, ph);
              continue;
            }
            break;
        }
      } else if (op.kind == OpKind::Noise) {
        // the draws do not depend on the state: a sampled error joins the run
        const int e = op.noise.sample(*rng);
        if (e >= 0) {
          uint64_t x = 0, z = 0;
          for (size_t j = 0; j < op.qubits.size(); ++j) {
            x |= uint64_t((e >> j) & 1) << op.qubits[j];
            z |= uint64_t((e >> (8 + j)) & 1) << op.qubits[j];
          }
          run.add_pauli(x, z, 0);
        }
        continue;
      } else if (op.kind != OpKind::Measure && op.kind != OpKind::Reset) {
        continue;
      }
      run.launch(s);
      const int r = sp_apply_op(s, op, *rng);
      if (r >= 0) rec[m++] = uint8_t(r);
    }
    run.launch(s);
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    if (len) *len = m;
  });
}

ncsim_status ncsim_sparse_num_words(const ncsim_sparse* s, uint32_t* words) {
  return guarded([&] {
    need(s, "state");
    need(words, "words");
    *words = s->words;
  });
}

ncsim_status ncsim_sparse_apply_pauli_words(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t words,
                                            uint32_t phase) {
  return guarded([&] {
    need(s, "state");
    check_words(s, words, {x, z});
    Lock lk(s);
    if (s->words > 1) return spw::pauli(s, x, z, phase);
    sp_pauli(s, x[0], z[0], phase);
  });
}

ncsim_status ncsim_sparse_amplitude_words(const ncsim_sparse* s, const uint64_t* index, uint32_t words,
                                          double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    need(index, "index");
    if (words != s->words) throw Error(NCSIM_ERR_INVALID, "index of the wrong word count");
    if (s->words == 1) {
      const ncsim_status r = ncsim_sparse_amplitude(s, index[0], re_im);
      if (r) throw Error(r, ncsim_last_error());
      return;
    }
    std::vector<uint64_t> idx(index, index + words);
    const uint32_t top = s->n - 64 * (words - 1);  // bits of the register in the last word
    if (top < 64) idx[words - 1] &= (uint64_t(1) << top) - 1;
    Lock lk(s);
    spw::amplitude(s, idx.data(), re_im);
  });
}

ncsim_status ncsim_sparse_expectation_words(const ncsim_sparse* s, const uint64_t* x, const uint64_t* z,
                                            uint32_t words, uint32_t phase, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    check_words(s, words, {x, z});
    Lock lk(s);
    if (s->words > 1) return spw::expectation(s, x, z, phase & 3u, re_im);
    sp_expect(s, x[0], z[0], phase & 3u, re_im);
  });
}

ncsim_status ncsim_sparse_project_words(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t words,
                                        uint32_t phase, int32_t outcome, double* weight_re_im) {
  return guarded([&] {
    need(s, "state");
    check_words(s, words, {x, z});
    uint32_t c = 0;
    for (uint32_t w = 0; w < words; ++w) c += uint32_t(__builtin_popcountll(x[w] & z[w]));
    if (((phase & 1u) == 1u) != bool(c & 1u)) throw Error(NCSIM_ERR_INVALID, "projector of a non-Hermitian Pauli");
    Lock lk(s);
    const double w = s->words > 1 ? spw::project(s, x, z, phase, outcome != 0)
                                  : sp_project(s, x[0], z[0], phase, outcome != 0);
    if (weight_re_im) weight_re_im[0] = w, weight_re_im[1] = 0.0;
  });
}

ncsim_status ncsim_sparse_measure_words(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t words,
                                        uint32_t phase, ncsim_rng* rng, int32_t* outcome) {
  return guarded([&] {
    need(s, "state");
    need(rng, "rng");
    check_words(s, words, {x, z});
    Lock lk(s);
    bool o;
    if (s->words > 1) {
      o = spw::measure(s, x, z, phase & 3u, *rng);
    } else {
      PauliOp p;
      p.n = s->n;
      p.x = x[0];
      p.z = z[0];
      p.phase = phase & 3u;
      o = sp_measure(s, p, *rng);
    }
    if (outcome) *outcome = o ? 1 : 0;
  });
}

ncsim_status ncsim_sparse_synchronize(const ncsim_sparse* s) {
  return guarded([&] {
    need(s, "state");
    Lock lk(s);
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  });
}

ncsim_status ncsim_sparse_timer_start(ncsim_sparse* s) {
  return guarded([&] {
    need(s, "state");
    Lock lk(s);
    NCSIM_CUDA(cudaEventRecord(s->timer0, s->stream));
  });
}

ncsim_status ncsim_sparse_timer_stop(ncsim_sparse* s, double* milliseconds) {
  return guarded([&] {
    need(s, "state");
    need(milliseconds, "out");
    Lock lk(s);
    NCSIM_CUDA(cudaEventRecord(s->timer1, s->stream));
    NCSIM_CUDA(cudaEventSynchronize(s->timer1));
    float ms = 0;
    NCSIM_CUDA(cudaEventElapsedTime(&ms, s->timer0, s->timer1));
    *milliseconds = ms;
  });
}

}  // extern "C"
