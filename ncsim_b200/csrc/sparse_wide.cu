// The sparse form on registers of 65..1024 qubits: ncsim's SparseVector<C64>
// keys entries by Bits (a Vec<u64>, src/bits.rs:11), so its registers have any
// width (src/state/sparse.rs:28-34); this file keeps W = 4 or 16 words per key
// in HBM (interleaved: entry i's key is words [W i, W i + W)).
//
// Semantics are the 64-qubit form's (sparse.cu): one-to-one ops in place, entry
// order kept; expansions normalised by sort, duplicate sum and zero/cutoff drop
// (sparse.rs:114-128); keys order lexicographically from word 0, the order of
// Vec<u64>.  Gates arrive lowered on their own qubits (local qubit j is
// qubits[j]): monomial tables and dense columns index the local pattern, phase
// polynomials are evaluated on it, Paulis are embedded into key-wide masks.
//
// Sorting: the keys of a sparse state usually differ in few bit positions, so
// the sort first ORs every key's difference from the first one; the varying
// positions, most significant first, are cut into chunks of 64, and a stable
// 64-bit radix sort of the index permutation by each chunk, least significant
// chunk first, orders the keys (one pass when at most 64 positions vary); a
// gather then moves keys and amplitudes.
#include "sparse_common.cuh"

using namespace ncsim;

namespace {

template <int W>
struct alignas(16) WKey {
  uint64_t w[W];
};
template <int W>
__host__ __device__ inline bool operator==(const WKey<W>& a, const WKey<W>& b) {
  for (int i = 0; i < W; ++i)
    if (a.w[i] != b.w[i]) return false;
  return true;
}
template <int W>
__host__ __device__ inline bool operator!=(const WKey<W>& a, const WKey<W>& b) {
  return !(a == b);
}
// Vec<u64>'s order: the first differing word decides
template <int W>
__device__ inline bool key_less(const WKey<W>& a, const WKey<W>& b) {
  for (int i = 0; i < W; ++i)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i];
  return false;
}
template <int W>
__device__ inline uint32_t kbit(const WKey<W>& k, uint32_t q) {
  return uint32_t(k.w[q >> 6] >> (q & 63)) & 1u;
}
template <int W>
__device__ inline uint32_t and_popc(const WKey<W>& a, const WKey<W>& b) {
  uint32_t c = 0;
  for (int i = 0; i < W; ++i) c += uint32_t(__popcll(a.w[i] & b.w[i]));
  return c;
}
template <int W>
__device__ inline void kxor(WKey<W>& a, const WKey<W>& b) {
  for (int i = 0; i < W; ++i) a.w[i] ^= b.w[i];
}

// a gate's qubits on a wide register
struct QubitsW {
  uint32_t k;
  uint16_t q[SP_MAX_K];
};
template <int W>
__device__ inline uint32_t local_w(const WKey<W>& key, const QubitsW& qs) {
  uint32_t x = 0;
  for (uint32_t j = 0; j < qs.k; ++j) x |= kbit(key, qs.q[j]) << j;
  return x;
}
template <int W>
__device__ inline void set_local_w(WKey<W>& key, const QubitsW& qs, uint32_t y) {
  for (uint32_t j = 0; j < qs.k; ++j) {
    const uint32_t q = qs.q[j];
    const uint64_t b = uint64_t(1) << (q & 63);
    uint64_t& w = key.w[q >> 6];
    w = ((y >> j) & 1u) ? (w | b) : (w & ~b);
  }
}
// the local pattern of up to 64 qubits (phase polynomials)
template <int W>
__device__ inline uint64_t local_w64(const WKey<W>& key, const uint16_t* q, uint32_t nq) {
  uint64_t x = 0;
  for (uint32_t j = 0; j < nq; ++j) x |= uint64_t(kbit(key, q[j])) << j;
  return x;
}

#define NCSIM_GRID_LOOP(i, m) \
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (m); i += uint64_t(gridDim.x) * blockDim.x)

// ---- one-to-one ops (order kept) ----
template <int W>
__global__ void k_w_monomial(WKey<W>* key, double2* amp, uint64_t m, QubitsW qs, const uint16_t* image,
                             const double2* phase, const uint8_t* unit) {
  NCSIM_GRID_LOOP(i, m) {
    WKey<W> kk = key[i];
    const uint32_t x = local_w(kk, qs);
    if (!unit[x]) amp[i] = zmul(phase[x], amp[i]);
    const uint32_t y = image[x];
    if (y != x) {
      set_local_w(kk, qs, y);
      key[i] = kk;
    }
  }
}
// i^phase X^x Z^z (sparse.rs:216-231)
template <int W>
__global__ void k_w_pauli(WKey<W>* key, double2* amp, uint64_t m, WKey<W> x, WKey<W> z, uint32_t phase) {
  NCSIM_GRID_LOOP(i, m) {
    WKey<W> kk = key[i];
    const uint32_t k = (phase + 2u * and_popc(z, kk)) & 3u;
    if (k) amp[i] = ipow(amp[i], k);
    kxor(kk, x);
    key[i] = kk;
  }
}
// Diagonal(PhasePoly) on up to 64 qubits: the polynomial of the local pattern
struct PolyW {
  uint32_t nq;
  uint16_t q[64];
  uint32_t bits, nterms, scalar_is_one, use_table;
  uint64_t constant;
  double2 scalar;
  const uint32_t* start;
  const uint64_t* par;
  const uint64_t* coeff;
  const double2* table;
};
template <int W>
__global__ void k_w_poly(const WKey<W>* key, double2* amp, uint64_t m, const __grid_constant__ PolyW P) {
  NCSIM_GRID_LOOP(i, m) {
    const uint64_t x = local_w64(key[i], P.q, P.nq);
    poly_apply(x, amp[i], P.bits, P.nterms, P.constant, P.scalar_is_one, P.scalar, P.use_table, P.start, P.par,
               P.coeff, P.table);
  }
}

// ---- runs of one-to-one ops in one launch ----
enum : uint32_t { RW_MONO = 0, RW_POLY = 1, RW_PAULI = 2 };
struct RunOpW {
  uint32_t type;
  uint32_t k;         // MONO: qubits; POLY: terms
  uint16_t q[SP_MAX_K];
  uint32_t off;       // MONO: first pattern of its tables; POLY: first term start
  uint32_t bits;      // POLY
  uint32_t flags;     // POLY: bit 0 scalar is one, bit 1 phasor table; PAULI: the phase
  uint32_t toff;      // POLY: its phasor table
  uint32_t nq, qoff;  // POLY: its qubits in RunDataW::qlist; PAULI: its masks (index into px/pz)
  uint64_t constant;  // POLY
  double2 scalar;     // POLY
  // MONO on at most 3 qubits: the 8 images (16 bits each: patterns 0..3, 4..7) and unit flags
  // (byte x: the phase of pattern x is exactly 1), packed on the host
  uint64_t img_lo, img_hi, unit8;
};
struct RunDataW {
  const RunOpW* ops;
  uint32_t nops;
  const uint16_t* image;
  const double2* phase;
  const uint8_t* unit;
  const double2* table;
  const uint32_t* start;
  const uint64_t* par;
  const uint64_t* coeff;
  const uint16_t* qlist;
  const void* px;  // WKey<W>[]: the runs' Pauli masks
  const void* pz;
};
// One warp per block, one entry per lane.  The run's op descriptors (monomials on at most 3
// qubits carry their image and unit tables packed into words) are staged 32 at a time into
// shared memory, one op per lane, so the walk reads them as broadcasts instead of a chain of
// dependent global loads per op.
constexpr int RW_STAGE = 32;
// One lane's key held in shared memory, word w at col[w * RW_STAGE] (consecutive lanes in
// consecutive words: conflict-free), so the walk's bit reads and writes stay on chip.
struct SKeyCol {
  uint64_t* col;
  __device__ uint32_t bit(uint32_t q) const { return uint32_t(col[(q >> 6) * RW_STAGE] >> (q & 63)) & 1u; }
  __device__ void set(uint32_t q, uint32_t v) const {
    uint64_t& w = col[(q >> 6) * RW_STAGE];
    const uint64_t b = uint64_t(1) << (q & 63);
    w = v ? (w | b) : (w & ~b);
  }
};
template <int W>
__global__ void __launch_bounds__(RW_STAGE) k_w_run(WKey<W>* key, double2* amp, uint64_t m, RunDataW d) {
  __shared__ RunOpW s_op[RW_STAGE];
  __shared__ uint64_t s_key[W * RW_STAGE];
  const WKey<W>* px = static_cast<const WKey<W>*>(d.px);
  const WKey<W>* pz = static_cast<const WKey<W>*>(d.pz);
  const uint32_t lane = threadIdx.x;
  const SKeyCol kk{s_key + lane};
  for (uint64_t base = uint64_t(blockIdx.x) * RW_STAGE; base < m; base += uint64_t(gridDim.x) * RW_STAGE) {
    const uint64_t i = base + lane;
    const bool live = i < m;
    double2 a = make_double2(0.0, 0.0);
    {
      WKey<W> k0{};
      if (live) {
        k0 = key[i];
        a = amp[i];
      }
#pragma unroll
      for (int w = 0; w < W; ++w) kk.col[w * RW_STAGE] = k0.w[w];
    }
    for (uint32_t o0 = 0; o0 < d.nops; o0 += RW_STAGE) {
      const uint32_t cnt = min(uint32_t(RW_STAGE), d.nops - o0);
      __syncwarp();
      if (lane < cnt) s_op[lane] = d.ops[o0 + lane];
      __syncwarp();
      if (!live) continue;
      for (uint32_t c = 0; c < cnt; ++c) {
        const RunOpW& op = s_op[c];
        if (op.type == RW_MONO) {
          const uint32_t k = op.k;
          uint32_t x = 0;
          for (uint32_t j = 0; j < k; ++j) x |= kk.bit(op.q[j]) << j;
          uint32_t y;
          bool unit;
          if (k <= 3) {
            y = uint32_t((x < 4 ? op.img_lo : op.img_hi) >> (16 * (x & 3))) & 0xffffu;
            unit = (op.unit8 >> (8 * x)) & 1u;
          } else {
            y = d.image[op.off + x];
            unit = d.unit[op.off + x];
          }
          if (!unit) a = zmul(d.phase[op.off + x], a);
          if (y != x)
            for (uint32_t j = 0; j < k; ++j) kk.set(op.q[j], (y >> j) & 1u);
        } else if (op.type == RW_POLY) {
          uint64_t x = 0;
          for (uint32_t j = 0; j < op.nq; ++j) x |= uint64_t(kk.bit(d.qlist[op.qoff + j])) << j;
          poly_apply(x, a, op.bits, op.k, op.constant, op.flags & 1u, op.scalar, (op.flags >> 1) & 1u,
                     d.start + op.off, d.par, d.coeff + op.off, d.table + op.toff);
        } else {
          const WKey<W>& zx = pz[op.qoff];
          const WKey<W>& xx = px[op.qoff];
          uint32_t cz = 0;
#pragma unroll
          for (int w = 0; w < W; ++w) {
            cz += uint32_t(__popcll(zx.w[w] & kk.col[w * RW_STAGE]));
            kk.col[w * RW_STAGE] ^= xx.w[w];
          }
          const uint32_t ph = (op.flags + 2u * cz) & 3u;
          if (ph) a = ipow(a, ph);
        }
      }
    }
    if (live) {
      WKey<W> k1;
#pragma unroll
      for (int w = 0; w < W; ++w) k1.w[w] = kk.col[w * RW_STAGE];
      key[i] = k1;
      amp[i] = a;
    }
  }
}

// ---- expansions ----
template <int W>
__global__ void k_w_count(const WKey<W>* key, uint64_t m, QubitsW qs, const uint32_t* col_start, uint32_t* cnt) {
  NCSIM_GRID_LOOP(i, m) {
    const uint32_t b = local_w(key[i], qs);
    cnt[i] = col_start[b + 1] - col_start[b];
  }
}
template <int W>
__global__ void k_w_expand(const WKey<W>* key, const double2* amp, uint64_t m, QubitsW qs, const uint32_t* col_start,
                           const uint32_t* col_row, const double2* col_val, const uint32_t* off, uint32_t per,
                           WKey<W>* okey, double2* oamp) {
  NCSIM_GRID_LOOP(i, m) {
    const WKey<W> kk = key[i];
    const double2 v = amp[i];
    const uint32_t b = local_w(kk, qs);
    uint64_t o = off ? uint64_t(off[i]) : uint64_t(i) * per;  // per: every column's count, when they are all equal
    for (uint32_t j = col_start[b]; j < col_start[b + 1]; ++j, ++o) {
      WKey<W> nk = kk;
      set_local_w(nk, qs, col_row[j]);
      okey[o] = nk;
      oamp[o] = zmul(col_val[j], v);
    }
  }
}
// (1 ± P)/2 (sparse.rs:351-380)
template <int W>
__global__ void k_w_project(const WKey<W>* key, const double2* amp, uint64_t m, WKey<W> x, WKey<W> z, uint32_t phase,
                            double sgn, WKey<W>* okey, double2* oamp) {
  NCSIM_GRID_LOOP(i, m) {
    const WKey<W> c = key[i];
    const double2 a = amp[i];
    const uint32_t k = (phase + 2u * and_popc(z, c)) & 3u;
    const double2 h = make_double2(0.5 * a.x, 0.5 * a.y);
    okey[2 * i] = c;
    oamp[2 * i] = h;
    const double2 t = ipow(h, k);
    WKey<W> cx = c;
    kxor(cx, x);
    okey[2 * i + 1] = cx;
    oamp[2 * i + 1] = make_double2(sgn * t.x, sgn * t.y);
  }
}
// a (x) b on keys of any word counts (sparse.rs:388-405): b's key shifted up by na bits
__global__ void k_w_tensor(const uint64_t* ka, uint32_t wa, const double2* va, uint64_t ma, uint32_t na,
                           const uint64_t* kb, uint32_t wb, const double2* vb, uint64_t mb, uint64_t* okey,
                           uint32_t wo, double2* oamp) {
  const uint64_t tot = ma * mb;
  NCSIM_GRID_LOOP(i, tot) {
    const uint64_t jb = i / ma, ia = i - jb * ma;
    const uint64_t* a = ka + ia * wa;
    const uint64_t* b = kb + jb * wb;
    for (uint32_t w = 0; w < wo; ++w) {
      uint64_t v = w < wa ? a[w] : 0;
      // bits [64 w - na, 64 w - na + 64) of b
      const int64_t lo = int64_t(w) * 64 - int64_t(na);
      if (lo <= -64) {
      } else if (lo < 0) {
        v |= b[0] << uint32_t(-lo);
      } else {
        const uint64_t wi = uint64_t(lo) >> 6;
        const uint32_t sh = uint32_t(lo) & 63u;
        if (wi < wb) v |= b[wi] >> sh;
        if (sh && wi + 1 < wb) v |= b[wi + 1] << (64u - sh);
      }
      okey[i * wo + w] = v;
    }
    oamp[i] = zmul(va[ia], vb[jb]);
  }
}

// ---- sums over the sorted view ----
template <int W>
__device__ inline int64_t find_w(const WKey<W>* sk, uint64_t m, const WKey<W>& x) {
  uint64_t lo = 0, hi = m;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (key_less(sk[mid], x)) lo = mid + 1;
    else hi = mid;
  }
  return lo < m && sk[lo] == x ? int64_t(lo) : -1;
}
// <psi|P|psi> = sum_c conj psi(c ^ x) i^k(c) psi(c) (sparse.rs:316-336)
template <int W>
__global__ void k_w_expect(const WKey<W>* sk, const double2* sa, uint64_t m, WKey<W> x, WKey<W> z, uint32_t phase,
                           int has_x, double* part) {
  double re = 0, im = 0;
  NCSIM_GRID_LOOP(i, m) {
    const WKey<W> c = sk[i];
    int64_t j = int64_t(i);
    if (has_x) {
      WKey<W> cx = c;
      kxor(cx, x);
      j = find_w(sk, m, cx);
    }
    if (j < 0) continue;
    const uint32_t k = (phase + 2u * and_popc(z, c)) & 3u;
    const double2 t = ipow(sa[i], k);
    const double2 b = sa[j];
    re += b.x * t.x + b.y * t.y;
    im += b.x * t.y - b.y * t.x;
  }
  block_add2(re, im, part);
}
// <a|b> (sparse.rs:338-349)
template <int W>
__global__ void k_w_inner(const WKey<W>* ka, const double2* va, uint64_t ma, const WKey<W>* skb, const double2* svb,
                          uint64_t mb, double* part) {
  double re = 0, im = 0;
  NCSIM_GRID_LOOP(i, ma) {
    const int64_t j = find_w(skb, mb, ka[i]);
    if (j < 0) continue;
    const double2 a = va[i], b = svb[j];
    re += a.x * b.x + a.y * b.y;
    im += a.x * b.y - a.y * b.x;
  }
  block_add2(re, im, part);
}
template <int W>
__global__ void k_w_find(const WKey<W>* key, const double2* amp, uint64_t m, WKey<W> x, int sorted, double2* out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double2 r = make_double2(0.0, 0.0);
    if (sorted) {
      const int64_t j = find_w(key, m, x);
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

// ---- sorting ----
// OR over all keys of key ^ key[0]: the bit positions that vary
template <int W>
__global__ void k_w_varying(const WKey<W>* key, uint64_t m, unsigned long long* acc) {
  const WKey<W> k0 = key[0];
  uint64_t v[W];
  for (int w = 0; w < W; ++w) v[w] = 0;
  NCSIM_GRID_LOOP(i, m) {
    const WKey<W> k = key[i];
    for (int w = 0; w < W; ++w) v[w] |= k.w[w] ^ k0.w[w];
  }
  for (int w = 0; w < W; ++w) {
    uint64_t x = v[w];
    for (int o = 16; o; o >>= 1) x |= __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicOr(acc + w, (unsigned long long)x);
  }
}
struct Varying {
  uint32_t cnt;
  uint16_t pos[64];  // most significant first
};
// up to 64 varying bits, most significant first, of key idx[i] (idx null: key i) as a
// 64-bit key of the same order
template <int W>
__global__ void k_w_compact(const WKey<W>* key, const uint32_t* idx, uint64_t m, const __grid_constant__ Varying V,
                            uint64_t* ck, uint32_t* idx_out) {
  NCSIM_GRID_LOOP(i, m) {
    const uint32_t src = idx ? idx[i] : uint32_t(i);
    const WKey<W> k = key[src];
    uint64_t c = 0;
    for (uint32_t j = 0; j < V.cnt; ++j) c = (c << 1) | kbit(k, V.pos[j]);
    ck[i] = c;
    if (!idx) idx_out[i] = uint32_t(i);
  }
}
template <int W>
__global__ void k_w_gather(const WKey<W>* kin, const double2* ain, const uint32_t* idx, uint64_t m, WKey<W>* kout,
                           double2* aout) {
  NCSIM_GRID_LOOP(i, m) {
    const uint32_t j = idx[i];
    kout[i] = kin[j];
    aout[i] = ain[j];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int W>
WKey<W>* keys_of(const ncsim_sparse* s) {
  return reinterpret_cast<WKey<W>*>(s->key);
}

template <class F>
void with_words(uint32_t words, F&& f) {
  if (words == 4) f(std::integral_constant<int, 4>{});
  else if (words == 16) f(std::integral_constant<int, 16>{});
  else throw Error(NCSIM_ERR_INVALID, "sparse state of " + std::to_string(words) + " words per key");
}

template <int W>
WKey<W> host_key(const uint64_t* words) {
  WKey<W> k{};
  for (int w = 0; w < W; ++w) k.w[w] = words ? words[w] : 0;
  return k;
}

// (kin, ain)[0, m) sorted by key into (kout, aout), stream-ordered on st
template <int W>
void sort_pairs(const WKey<W>* kin, const double2* ain, WKey<W>* kout, double2* aout, uint64_t m, cudaStream_t st) {
  if (m == 0) return;
  if (m > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  if (m == 1) {
    NCSIM_CUDA(cudaMemcpyAsync(kout, kin, sizeof(WKey<W>), cudaMemcpyDeviceToDevice, st));
    NCSIM_CUDA(cudaMemcpyAsync(aout, ain, sizeof(double2), cudaMemcpyDeviceToDevice, st));
    return;
  }
  const int num = int(m);
  unsigned long long* acc = dalloc<unsigned long long>(W, st);
  NCSIM_CUDA(cudaMemsetAsync(acc, 0, W * sizeof(unsigned long long), st));
  k_w_varying<W><<<sp_grid(m), SP_THREADS, 0, st>>>(kin, m, acc);
  NCSIM_LAUNCHED("sparse varying bits");
  uint64_t vary[W];
  NCSIM_CUDA(cudaMemcpyAsync(vary, acc, sizeof(vary), cudaMemcpyDeviceToHost, st));
  NCSIM_CUDA(cudaStreamSynchronize(st));
  dfree(acc, st);
  // the varying positions, most significant first, in chunks of 64; a stable radix sort
  // of the index permutation by each chunk, least significant chunk first
  std::vector<uint16_t> pos;
  for (int w = 0; w < W; ++w)
    for (int b = 63; b >= 0; --b)
      if ((vary[w] >> b) & 1) pos.push_back(uint16_t(64 * w + b));
  if (pos.empty()) pos.push_back(0);  // all keys equal: any order
  uint64_t* ck = dalloc<uint64_t>(m, st);
  uint64_t* ck2 = dalloc<uint64_t>(m, st);
  uint32_t* idx = dalloc<uint32_t>(m, st);
  uint32_t* idx2 = dalloc<uint32_t>(m, st);
  size_t tb = 0;
  NCSIM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, ck, ck2, idx, idx2, num, 0, 64, st));
  void* tmp = dalloc<uint8_t>(tb, st);
  bool first = true;
  for (size_t hi = pos.size(); hi > 0;) {
    const size_t lo = hi > 64 ? hi - 64 : 0;
    Varying V{};
    V.cnt = uint32_t(hi - lo);
    for (size_t j = lo; j < hi; ++j) V.pos[j - lo] = pos[j];
    k_w_compact<W><<<sp_grid(m), SP_THREADS, 0, st>>>(kin, first ? nullptr : idx, m, V, ck, idx);
    NCSIM_LAUNCHED("sparse compact keys");
    NCSIM_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, ck, ck2, idx, idx2, num, 0, int(V.cnt), st));
    std::swap(idx, idx2);
    first = false;
    hi = lo;
  }
  k_w_gather<W><<<sp_grid(m), SP_THREADS, 0, st>>>(kin, ain, idx, m, kout, aout);
  NCSIM_LAUNCHED("sparse gather");
  dfree(tmp, st);
  dfree(ck, st);
  dfree(ck2, st);
  dfree(idx, st);
  dfree(idx2, st);
}

// replaces the entries by the normalised (key, amp)[0, cnt) (takes ownership)
template <int W>
void normalize_from(ncsim_sparse* s, WKey<W>* key, double2* amp, uint64_t cnt) {
  cudaStream_t st = s->stream;
  if (cnt > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  const int num = int(cnt);
  WKey<W>* k2 = dalloc<WKey<W>>(cnt, st);
  double2* a2 = dalloc<double2>(cnt, st);
  WKey<W>* k3 = dalloc<WKey<W>>(cnt, st);
  double2* a3 = dalloc<double2>(cnt, st);
  uint8_t* flag = dalloc<uint8_t>(cnt, st);
  int* d_num = dalloc<int>(2, st);
  int kept = 0;
  if (num > 0) {
    sort_pairs<W>(key, amp, k2, a2, cnt, st);
    size_t t2 = 0, t3 = 0, t4 = 0;
    NCSIM_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, t2, k2, k3, a2, a3, d_num, ZAdd(), num, st));
    NCSIM_CUDA(cub::DeviceSelect::Flagged(nullptr, t3, k3, flag, key, d_num + 1, num, st));
    NCSIM_CUDA(cub::DeviceSelect::Flagged(nullptr, t4, a3, flag, amp, d_num + 1, num, st));
    void* tmp = dalloc<uint8_t>(std::max(t2, std::max(t3, t4)), st);
    NCSIM_CUDA(cub::DeviceReduce::ReduceByKey(tmp, t2, k2, k3, a2, a3, d_num, ZAdd(), num, st));
    // the run count stays on the device: the keep flags drop the positions past it
    k_sp_keep<<<sp_grid(cnt), SP_THREADS, 0, st>>>(a3, d_num, cnt, s->cutoff * s->cutoff, flag);
    NCSIM_LAUNCHED("sparse keep");
    NCSIM_CUDA(cub::DeviceSelect::Flagged(tmp, t3, k3, flag, key, d_num + 1, num, st));
    NCSIM_CUDA(cub::DeviceSelect::Flagged(tmp, t4, a3, flag, amp, d_num + 1, num, st));
    NCSIM_CUDA(cudaMemcpyAsync(&kept, d_num + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    NCSIM_CUDA(cudaStreamSynchronize(st));
    dfree(tmp, st);
  }
  dfree(k2, st);
  dfree(a2, st);
  dfree(k3, st);
  dfree(a3, st);
  dfree(flag, st);
  dfree(d_num, st);
  dfree(s->key, st);
  dfree(s->amp, st);
  s->key = reinterpret_cast<uint64_t*>(key);
  s->amp = amp;
  s->cap = std::max<uint64_t>(cnt, 1);
  s->m = uint64_t(kept);
  s->sorted = true;
}

template <int W>
void normalize_w(ncsim_sparse* s) {
  cudaStream_t st = s->stream;
  WKey<W>* k = dalloc<WKey<W>>(s->m, st);
  double2* a = dalloc<double2>(s->m, st);
  if (s->m) {
    NCSIM_CUDA(cudaMemcpyAsync(k, s->key, s->m * sizeof(WKey<W>), cudaMemcpyDeviceToDevice, st));
    NCSIM_CUDA(cudaMemcpyAsync(a, s->amp, s->m * 16, cudaMemcpyDeviceToDevice, st));
  }
  normalize_from<W>(s, k, a, s->m);
}

// a sorted copy of the entries on stream st (owned by the caller)
template <int W>
void sorted_copy_w(const ncsim_sparse* s, cudaStream_t st, WKey<W>*& k, double2*& a) {
  k = dalloc<WKey<W>>(s->m, st);
  a = dalloc<double2>(s->m, st);
  sort_pairs<W>(keys_of<W>(s), s->amp, k, a, s->m, st);
}

template <int W>
void sort_w(ncsim_sparse* s) {
  if (s->sorted) return;
  WKey<W>* k;
  double2* a;
  sorted_copy_w<W>(s, s->stream, k, a);
  dfree(s->key, s->stream);
  dfree(s->amp, s->stream);
  s->key = reinterpret_cast<uint64_t*>(k);
  s->amp = a;
  s->cap = std::max<uint64_t>(s->m, 1);
  s->sorted = true;
}

QubitsW qubits_w(const std::vector<uint32_t>& local, const std::vector<uint32_t>& qubits) {
  if (local.size() > SP_MAX_K) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse gate on more than 10 qubits");
  QubitsW qs{};
  qs.k = uint32_t(local.size());
  for (size_t j = 0; j < local.size(); ++j) qs.q[j] = uint16_t(qubits[local[j]]);
  return qs;
}

template <int W>
void monomial_w(ncsim_sparse* s, const QubitsW& qs, const std::vector<uint32_t>& image, const std::vector<CplxD>& phase) {
  const size_t gd = size_t(1) << qs.k;
  std::vector<uint16_t> img(gd);
  std::vector<double2> ph(gd);
  std::vector<uint8_t> unit(gd);
  bool moves = false;
  for (size_t x = 0; x < gd; ++x) {
    img[x] = uint16_t(image[x]);
    ph[x] = make_double2(phase[x].re, phase[x].im);
    unit[x] = phase[x].re == 1.0 && phase[x].im == 0.0;
    moves |= image[x] != x;
  }
  if (s->m) {
    cudaStream_t st = s->stream;
    uint16_t* di = upload(img, st);
    double2* dp = upload(ph, st);
    uint8_t* du = upload(unit, st);
    k_w_monomial<W><<<sp_grid(s->m), SP_THREADS, 0, st>>>(keys_of<W>(s), s->amp, s->m, qs, di, dp, du);
    NCSIM_LAUNCHED("sparse monomial (wide)");
    dfree(di, st);
    dfree(dp, st);
    dfree(du, st);
  }
  if (moves) s->sorted = false;
}

template <int W>
void matrix_w(ncsim_sparse* s, const QubitsW& qs, const std::vector<CplxD>& mat) {
  const size_t gd = size_t(1) << qs.k;
  std::vector<uint32_t> img;
  std::vector<CplxD> ph;
  if (permutation_view(mat, gd, img, ph)) return monomial_w<W>(s, qs, img, ph);
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
  cudaStream_t st = s->stream;
  const uint64_t m = s->m;
  if (m > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  uint32_t* dcs = upload(col_start, st);
  uint32_t* dcr = upload(col_row, st);
  double2* dcv = upload(col_val, st);
  // every column with the same count: entry i's images start at i * per (no counts, scan or wait)
  const uint32_t per = col_start[1] - col_start[0];
  bool uniform = true;
  for (size_t b = 0; b < gd && uniform; ++b) uniform = col_start[b + 1] - col_start[b] == per;
  uint32_t* cnt = uniform ? nullptr : dalloc<uint32_t>(m + 1, st);
  uint32_t* off = uniform ? nullptr : dalloc<uint32_t>(m + 1, st);
  uint64_t total = uniform ? m * per : 0;
  if (m && !uniform) {
    k_w_count<W><<<sp_grid(m), SP_THREADS, 0, st>>>(keys_of<W>(s), m, qs, dcs, cnt);
    NCSIM_LAUNCHED("sparse count (wide)");
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
  WKey<W>* okey = dalloc<WKey<W>>(total, st);
  double2* oamp = dalloc<double2>(total, st);
  if (total) {
    k_w_expand<W><<<sp_grid(m), SP_THREADS, 0, st>>>(keys_of<W>(s), s->amp, m, qs, dcs, dcr, dcv, off, per,
                                                     okey, oamp);
    NCSIM_LAUNCHED("sparse expand (wide)");
  }
  dfree(dcs, st);
  dfree(dcr, st);
  dfree(dcv, st);
  dfree(cnt, st);
  dfree(off, st);
  normalize_from<W>(s, okey, oamp, total);
}

void check_poly_width(const std::vector<uint32_t>& qubits) {
  if (qubits.size() > 64) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse phase polynomial on more than 64 qubits");
}

template <int W>
void poly_w(ncsim_sparse* s, const std::vector<uint32_t>& qubits, const PolyTerms& t) {
  check_poly_width(qubits);
  if (!s->m) return;
  cudaStream_t st = s->stream;
  PolyW P{};
  P.nq = uint32_t(qubits.size());
  for (size_t j = 0; j < qubits.size(); ++j) P.q[j] = uint16_t(qubits[j]);
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
  k_w_poly<W><<<sp_grid(s->m), SP_THREADS, 0, st>>>(keys_of<W>(s), s->amp, s->m, P);
  NCSIM_LAUNCHED("sparse phasepoly (wide)");
  dfree(ds, st);
  dfree(dp, st);
  dfree(dc, st);
  dfree(dt, st);
}

// the words of a Pauli given on local qubits (bit j = qubits[j])
void embed(const std::vector<uint32_t>& qubits, uint64_t lx, uint64_t lz, uint32_t words, std::vector<uint64_t>& x,
           std::vector<uint64_t>& z) {
  x.assign(words, 0);
  z.assign(words, 0);
  for (size_t j = 0; j < qubits.size() && j < 64; ++j) {
    const uint32_t q = qubits[j];
    x[q >> 6] |= ((lx >> j) & 1ull) << (q & 63);
    z[q >> 6] |= ((lz >> j) & 1ull) << (q & 63);
  }
}

template <int W>
void pauli_w(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase) {
  const WKey<W> kx = host_key<W>(x), kz = host_key<W>(z);
  if (s->m) {
    k_w_pauli<W><<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(keys_of<W>(s), s->amp, s->m, kx, kz, phase & 3u);
    NCSIM_LAUNCHED("sparse pauli (wide)");
  }
  bool moves = false;
  for (int w = 0; w < W; ++w) moves |= x[w] != 0;
  if (moves) s->sorted = false;
}

template <int W>
void apply_lowered_w(ncsim_sparse* s, const LoweredOp& lo, const std::vector<uint32_t>& qubits) {
  switch (lo.kind) {
    case LoweredKind::Nothing: return;
    case LoweredKind::Dense: return matrix_w<W>(s, qubits_w(lo.qubits, qubits), lo.matrix);
    case LoweredKind::Monomial: return monomial_w<W>(s, qubits_w(lo.qubits, qubits), lo.image, lo.matrix);
    case LoweredKind::PhasePoly: return poly_w<W>(s, qubits, lo.poly);
    case LoweredKind::Pauli: {
      std::vector<uint64_t> x, z;
      embed(qubits, lo.x, lo.z, W, x, z);
      return pauli_w<W>(s, x.data(), z.data(), lo.phase);
    }
  }
}

template <int W>
void expect_w(const ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, double* out) {
  bool has_x = false;
  for (int w = 0; w < W; ++w) has_x |= x[w] != 0;
  const WKey<W>* k = keys_of<W>(s);
  const double2* a = s->amp;
  WKey<W>* kc = nullptr;
  double2* ac = nullptr;
  if (has_x && !s->sorted) {
    sorted_copy_w<W>(s, s->stream, kc, ac);
    k = kc;
    a = ac;
  }
  const unsigned g = red_grid(s->m);
  k_w_expect<W><<<g, SP_THREADS, 0, s->stream>>>(k, a, s->m, host_key<W>(x), host_key<W>(z), phase & 3u,
                                                   has_x ? 1 : 0, s->partials);
  NCSIM_LAUNCHED("sparse expectation (wide)");
  sp_sum(s, g, out);
  dfree(kc, s->stream);
  dfree(ac, s->stream);
}

template <int W>
double project_w(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, bool outcome) {
  cudaStream_t st = s->stream;
  const uint64_t m = s->m;
  WKey<W>* okey = dalloc<WKey<W>>(2 * m, st);
  double2* oamp = dalloc<double2>(2 * m, st);
  if (m) {
    k_w_project<W><<<sp_grid(m), SP_THREADS, 0, st>>>(keys_of<W>(s), s->amp, m, host_key<W>(x), host_key<W>(z),
                                                      phase & 3u, outcome ? -1.0 : 1.0, okey, oamp);
    NCSIM_LAUNCHED("sparse project (wide)");
  }
  normalize_from<W>(s, okey, oamp, 2 * m);
  return sp_norm(s);
}

bool hermitian_words(const uint64_t* x, const uint64_t* z, uint32_t words, uint32_t phase) {
  uint32_t c = 0;
  for (uint32_t w = 0; w < words; ++w) c += uint32_t(__builtin_popcountll(x[w] & z[w]));
  return ((phase & 1u) == 1u) == bool(c & 1u);
}

// QuantumState::measure (mod.rs:113-131)
template <int W>
bool measure_w(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, ncsim_rng& rng) {
  if (!hermitian_words(x, z, W, phase)) throw Error(NCSIM_ERR_INVALID, "measured operator is not Hermitian");
  double e[2];
  expect_w<W>(s, x, z, phase, e);
  const double nn = sp_norm(s);
  double p_plus = (1.0 + e[0] / nn) / 2.0;
  if (!std::isnan(p_plus)) p_plus = std::min(1.0, std::max(0.0, p_plus));
  bool outcome;
  if (p_plus > 1.0 - 1e-12) outcome = false;
  else if (p_plus < 1e-12) outcome = true;
  else outcome = rng.f64() >= p_plus;
  project_w<W>(s, x, z, phase, outcome);
  return outcome;
}

// the words of a measured Pauli given by its sites (Y = i X Z: a Y site adds one to the phase)
void sites_words(const PauliSites& ps, uint32_t words, std::vector<uint64_t>& x, std::vector<uint64_t>& z,
                 uint32_t& phase) {
  x.assign(words, 0);
  z.assign(words, 0);
  uint32_t ys = 0;
  for (const auto& st : ps.sites) {
    const uint32_t q = st.first;
    if (st.second & 1) x[q >> 6] |= uint64_t(1) << (q & 63);
    if (st.second & 2) z[q >> 6] |= uint64_t(1) << (q & 63);
    ys += st.second == 3;
  }
  phase = (ps.phase + ys) & 3u;
}

// the host side of a run of one-to-one ops
template <int W>
struct RunBuilderW {
  std::vector<RunOpW> ops;
  std::vector<uint16_t> image, qlist;
  std::vector<double2> phase, table;
  std::vector<uint8_t> unit;
  std::vector<uint32_t> start;
  std::vector<uint64_t> par, coeff;
  std::vector<WKey<W>> px, pz;
  bool moves = false;

  void add_mono(const QubitsW& qs, const std::vector<uint32_t>& img, const std::vector<CplxD>& ph) {
    RunOpW op{};
    op.type = RW_MONO;
    op.k = qs.k;
    for (uint32_t j = 0; j < qs.k; ++j) op.q[j] = qs.q[j];
    op.off = uint32_t(image.size());
    for (size_t x = 0; x < img.size(); ++x) {
      image.push_back(uint16_t(img[x]));
      phase.push_back(make_double2(ph[x].re, ph[x].im));
      const bool one = ph[x].re == 1.0 && ph[x].im == 0.0;
      unit.push_back(one);
      moves |= img[x] != x;
      if (qs.k <= 3) {
        (x < 4 ? op.img_lo : op.img_hi) |= uint64_t(img[x]) << (16 * (x & 3));
        op.unit8 |= uint64_t(one) << (8 * x);
      }
    }
    ops.push_back(op);
  }
  void add_poly(const std::vector<uint32_t>& qubits, const PolyTerms& t) {
    check_poly_width(qubits);
    RunOpW op{};
    op.type = RW_POLY;
    op.k = uint32_t(t.coeffs.size());
    op.bits = t.bits;
    op.constant = t.constant;
    op.scalar = make_double2(t.scalar.re, t.scalar.im);
    op.flags = (t.scalar_is_one ? 1u : 0u) | (t.root_table.empty() ? 0u : 2u);
    op.nq = uint32_t(qubits.size());
    op.qoff = uint32_t(qlist.size());
    for (uint32_t q : qubits) qlist.push_back(uint16_t(q));
    op.off = uint32_t(start.size());
    const uint32_t pbase = uint32_t(par.size());
    for (size_t i = 0; i <= t.coeffs.size(); ++i) start.push_back(pbase + (t.term_start.empty() ? 0 : t.term_start[i]));
    for (uint64_t c : t.coeffs) coeff.push_back(c);
    coeff.push_back(0);  // keeps coeff aligned with start (nterms + 1 per polynomial)
    for (uint64_t pm : t.parities) par.push_back(pm);
    op.toff = uint32_t(table.size());
    for (const CplxD& c : t.root_table) table.push_back(make_double2(c.re, c.im));
    ops.push_back(op);
  }
  void add_pauli(const uint64_t* x, const uint64_t* z, uint32_t ph) {
    RunOpW op{};
    op.type = RW_PAULI;
    op.flags = ph & 3u;
    op.qoff = uint32_t(px.size());
    px.push_back(host_key<W>(x));
    pz.push_back(host_key<W>(z));
    for (int w = 0; w < W; ++w) moves |= x[w] != 0;
    ops.push_back(op);
  }
  void launch(ncsim_sparse* s) {
    if (ops.empty()) return;
    cudaStream_t st = s->stream;
    if (s->m) {
      RunOpW* d_ops = upload(ops, st);
      uint16_t* d_img = upload(image, st);
      double2* d_ph = upload(phase, st);
      uint8_t* d_unit = upload(unit, st);
      double2* d_tab = upload(table, st);
      uint32_t* d_start = upload(start, st);
      uint64_t* d_par = upload(par, st);
      uint64_t* d_coeff = upload(coeff, st);
      uint16_t* d_q = upload(qlist, st);
      WKey<W>* d_px = upload(px, st);
      WKey<W>* d_pz = upload(pz, st);
      RunDataW d{d_ops, uint32_t(ops.size()), d_img, d_ph, d_unit, d_tab, d_start, d_par, d_coeff, d_q, d_px, d_pz};
      // one warp per block walks the run for 32 entries (up to 32 blocks per SM)
      const unsigned grid =
          unsigned(std::min<uint64_t>((s->m + RW_STAGE - 1) / RW_STAGE, uint64_t(sm_count()) * 32));
      k_w_run<W><<<grid, RW_STAGE, 0, st>>>(keys_of<W>(s), s->amp, s->m, d);
      NCSIM_LAUNCHED("sparse run (wide)");
      dfree(d_ops, st);
      dfree(d_img, st);
      dfree(d_ph, st);
      dfree(d_unit, st);
      dfree(d_tab, st);
      dfree(d_start, st);
      dfree(d_par, st);
      dfree(d_coeff, st);
      dfree(d_q, st);
      dfree(d_px, st);
      dfree(d_pz, st);
    }
    if (moves) s->sorted = false;
    *this = RunBuilderW();
  }
};

// QuantumState::run (mod.rs:168-183) with runs of one-to-one ops in one launch each
template <int W>
void run_w(ncsim_sparse* s, const ncsim_circuit& c, ncsim_rng& rng, uint8_t* rec, size_t& m) {
  RunBuilderW<W> run;
  std::vector<uint32_t> img;
  std::vector<CplxD> ph;
  std::vector<uint64_t> x, z;
  for (const OpIR& op : c.ops) {
    if (op.kind == OpKind::Gate) {
      const LoweredOp& lo = op.lowered;  // on local qubits: local j is op.qubits[j]
      switch (lo.kind) {
        case LoweredKind::Nothing: continue;
        case LoweredKind::Monomial:
          if (lo.qubits.size() <= SP_MAX_K) {
            run.add_mono(qubits_w(lo.qubits, op.qubits), lo.image, lo.matrix);
            continue;
          }
          break;
        case LoweredKind::PhasePoly:
          run.add_poly(op.qubits, lo.poly);
          continue;
        case LoweredKind::Pauli:
          embed(op.qubits, lo.x, lo.z, W, x, z);
          run.add_pauli(x.data(), z.data(), lo.phase);
          continue;
        case LoweredKind::Dense:
          if (lo.qubits.size() <= SP_MAX_K && permutation_view(lo.matrix, size_t(1) << lo.qubits.size(), img, ph)) {
            run.add_mono(qubits_w(lo.qubits, op.qubits), img, ph);
            continue;
          }
          break;
      }
      run.launch(s);
      apply_lowered_w<W>(s, lo, op.qubits);
      continue;
    }
    if (op.kind == OpKind::Noise) {
      // Noise::sample (circuit.rs:136-146): the draws do not depend on the state
      const int e = op.noise.sample(rng);
      if (e >= 0) {
        x.assign(W, 0);
        z.assign(W, 0);
        for (size_t j = 0; j < op.qubits.size(); ++j) {
          const uint32_t q = op.qubits[j];
          x[q >> 6] |= uint64_t((e >> j) & 1) << (q & 63);
          z[q >> 6] |= uint64_t((e >> (8 + j)) & 1) << (q & 63);
        }
        run.add_pauli(x.data(), z.data(), 0);
      }
      continue;
    }
    if (op.kind == OpKind::Measure) {
      run.launch(s);
      uint32_t phase = 0;
      sites_words(op.sites, W, x, z, phase);
      rec[m++] = uint8_t(measure_w<W>(s, x.data(), z.data(), phase, rng) ? 1 : 0);
      continue;
    }
    if (op.kind == OpKind::Reset) {  // measure Z, flip on 1 (mod.rs:150-157)
      run.launch(s);
      const uint32_t q = op.qubits[0];
      x.assign(W, 0);
      z.assign(W, 0);
      z[q >> 6] = uint64_t(1) << (q & 63);
      if (measure_w<W>(s, x.data(), z.data(), 0, rng)) {
        std::vector<uint64_t> fx(W, 0), fz(W, 0);
        fx[q >> 6] = uint64_t(1) << (q & 63);
        pauli_w<W>(s, fx.data(), fz.data(), 0);
      }
      continue;
    }
  }
  run.launch(s);
}

}  // namespace

namespace ncsim {
namespace spw {

uint32_t words_for(uint32_t n) {
  if (n == 0 || n > MAX_QUBITS)
    throw Error(NCSIM_ERR_INVALID, "sparse register of " + std::to_string(n) + " qubits (1.." +
                                       std::to_string(MAX_QUBITS) + ")");
  return n <= 64 ? 1u : n <= 256 ? 4u : 16u;
}

void set_entries(ncsim_sparse* s, const uint64_t* keys, const double* amps, uint64_t count) {
  const uint32_t W = s->words;
  // each key masked to the register (bits::mask_to, sparse.rs:58-62)
  std::vector<uint64_t> k(size_t(count) * W);
  for (uint64_t i = 0; i < count; ++i)
    for (uint32_t w = 0; w < W; ++w) {
      const uint32_t lo = 64 * w;
      const uint64_t mask = s->n >= lo + 64 ? ~uint64_t(0) : s->n <= lo ? 0 : (uint64_t(1) << (s->n - lo)) - 1;
      k[size_t(i) * W + w] = keys[size_t(i) * W + w] & mask;
    }
  with_words(W, [&](auto wc) {
    constexpr int WW = decltype(wc)::value;
    WKey<WW>* dk = dalloc<WKey<WW>>(count, s->stream);
    if (count) NCSIM_CUDA(cudaMemcpyAsync(dk, k.data(), k.size() * 8, cudaMemcpyHostToDevice, s->stream));
    double2* da = dalloc<double2>(count, s->stream);
    if (count) NCSIM_CUDA(cudaMemcpyAsync(da, amps, count * 16, cudaMemcpyHostToDevice, s->stream));
    normalize_from<WW>(s, dk, da, count);
  });
}

void normalize(ncsim_sparse* s) {
  with_words(s->words, [&](auto wc) { normalize_w<decltype(wc)::value>(s); });
}

void sort(ncsim_sparse* s) {
  with_words(s->words, [&](auto wc) { sort_w<decltype(wc)::value>(s); });
}

void apply_gate(ncsim_sparse* s, const GateIR& g, const std::vector<uint32_t>& qubits) {
  // check_qubits and the arity check (vector.rs:365-372 for every state form)
  for (size_t i = 0; i < qubits.size(); ++i) {
    if (qubits[i] >= s->n) throw qubit_out_of_range(qubits[i], s->n);
    for (size_t j = 0; j < i; ++j)
      if (qubits[j] == qubits[i]) throw duplicate_qubit(qubits[i]);
  }
  if (qubits.size() != g.arity()) throw arity_error(g.text(), g.arity(), qubits.size());
  if (qubits.size() > 64) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse gate on more than 64 qubits");
  std::vector<uint32_t> local(qubits.size());
  for (size_t j = 0; j < local.size(); ++j) local[j] = uint32_t(j);
  const LoweredOp lo = lower_gate(g, local, uint32_t(local.size()));
  with_words(s->words, [&](auto wc) { apply_lowered_w<decltype(wc)::value>(s, lo, qubits); });
}

void pauli(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase) {
  with_words(s->words, [&](auto wc) { pauli_w<decltype(wc)::value>(s, x, z, phase); });
}

void amplitude(const ncsim_sparse* s, const uint64_t* index, double* re_im) {
  with_words(s->words, [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    double2* d = dalloc<double2>(1, s->stream);
    k_w_find<W><<<1, 32, 0, s->stream>>>(keys_of<W>(s), s->amp, s->m, host_key<W>(index), s->sorted ? 1 : 0, d);
    NCSIM_LAUNCHED("sparse amplitude (wide)");
    double2 h;
    NCSIM_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    dfree(d, s->stream);
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    re_im[0] = h.x;
    re_im[1] = h.y;
  });
}

void expectation(const ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, double* re_im) {
  with_words(s->words, [&](auto wc) { expect_w<decltype(wc)::value>(s, x, z, phase, re_im); });
}

void inner(const ncsim_sparse* a, const ncsim_sparse* b, double* re_im) {
  with_words(a->words, [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    const WKey<W>* kb = keys_of<W>(b);
    const double2* vb = b->amp;
    WKey<W>* kc = nullptr;
    double2* vc = nullptr;
    if (!b->sorted) {  // b's sorted view, made on a's stream
      sorted_copy_w<W>(b, a->stream, kc, vc);
      kb = kc;
      vb = vc;
    }
    const unsigned g = red_grid(a->m);
    k_w_inner<W><<<g, SP_THREADS, 0, a->stream>>>(keys_of<W>(a), a->amp, a->m, kb, vb, b->m, a->partials);
    NCSIM_LAUNCHED("sparse inner (wide)");
    sp_sum(a, g, re_im);
    dfree(kc, a->stream);
    dfree(vc, a->stream);
  });
}

double project(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, bool outcome) {
  double w = 0;
  with_words(s->words, [&](auto wc) { w = project_w<decltype(wc)::value>(s, x, z, phase, outcome); });
  return w;
}

void tensor(const ncsim_sparse* a, const ncsim_sparse* b, ncsim_sparse* c) {
  const uint64_t tot = a->m * b->m;
  if (tot > uint64_t(INT32_MAX)) throw Error(NCSIM_ERR_UNSUPPORTED, "sparse state of more than 2^31 entries");
  cudaStream_t st = c->stream;
  uint64_t* okey = dalloc<uint64_t>(tot * c->words, st);
  double2* oamp = dalloc<double2>(tot, st);
  if (tot) {
    k_w_tensor<<<sp_grid(tot), SP_THREADS, 0, st>>>(a->key, a->words, a->amp, a->m, a->n, b->key, b->words, b->amp,
                                                     b->m, okey, c->words, oamp);
    NCSIM_LAUNCHED("sparse tensor (wide)");
  }
  dfree(c->key, st);
  dfree(c->amp, st);
  c->key = okey;
  c->amp = oamp;
  c->cap = std::max<uint64_t>(tot, 1);
  c->m = tot;
  c->sorted = false;
}

void sample(const ncsim_sparse* s, ncsim_rng& rng, uint64_t shots, uint64_t* out) {
  const uint32_t W = s->words;
  std::vector<double> w(s->m);
  std::vector<uint64_t> keys(size_t(s->m) * W);
  if (s->m) {
    double* dw = dalloc<double>(s->m, s->stream);
    k_sp_abs2<<<sp_grid(s->m), SP_THREADS, 0, s->stream>>>(s->amp, s->m, dw);
    NCSIM_LAUNCHED("sparse weights");
    NCSIM_CUDA(cudaMemcpyAsync(w.data(), dw, s->m * 8, cudaMemcpyDeviceToHost, s->stream));
    NCSIM_CUDA(cudaMemcpyAsync(keys.data(), s->key, keys.size() * 8, cudaMemcpyDeviceToHost, s->stream));
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
    const double u = rng.f64() * acc;
    size_t i = size_t(std::upper_bound(w.begin(), w.end(), u) - w.begin());
    if (i >= w.size()) i = w.size() - 1;
    std::copy(keys.begin() + i * W, keys.begin() + (i + 1) * W, out + k * W);
  }
}

bool measure(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t phase, ncsim_rng& rng) {
  bool o = false;
  with_words(s->words, [&](auto wc) { o = measure_w<decltype(wc)::value>(s, x, z, phase, rng); });
  return o;
}

void run(ncsim_sparse* s, const ncsim_circuit& c, ncsim_rng& rng, uint8_t* rec, size_t& m) {
  with_words(s->words, [&](auto wc) { run_w<decltype(wc)::value>(s, c, rng, rec, m); });
}

}  // namespace spw
}  // namespace ncsim
