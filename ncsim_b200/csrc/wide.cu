// Wide gates on the plain path: dense matrices on 6..13 qubits and monomial
// (permutation-with-phase) tables on more than 10 qubits, the gates whose
// matrices or tables do not fit a kernel's parameters or a shared-memory tile
// (the reference applies any k through one fiber kernel: apply_matrix,
// src/state/vector.rs:67-93, and apply_monomial's permutation branch,
// vector.rs:130-137; 12-qubit Clifford unitaries reach it through
// src/clifford/mod.rs:317-318 and src/gate.rs:732).
//
// A fiber is the 2^k amplitudes that agree off the gate qubits.  The register
// is processed in chunks of C fibers (C * 2^k <= 2^24 amplitudes):
//   gather   X[b][f] = amp[base(f0 + f) | off(b)]   (f fastest: coalesced when
//                                                    the low index bits are not
//                                                    gate bits)
//   dense    Y = M X, a tiled complex GEMM (FP64 for complex128 registers,
//            FP32 for complex64), 64 x 64 output tiles, 4 x 4 per thread
//   scatter  amp[base(f0 + f) | off(a)] = Y[a][f]
// and for a monomial table, one pass that writes amp[base | off(y)] =
// phase(y) * X[pre(y)][f] from the gathered chunk.  The matrix or table lives
// in device memory from the library's pool for the duration of the call.
#include "engine.cuh"

#include <algorithm>

namespace ncsim {

namespace {

constexpr int WIDE_THREADS = 256;
constexpr int MAX_WIDE_POS = 24;             // gate qubits of a wide gate
constexpr uint64_t CHUNK_AMPS = 1ull << 24;  // amplitudes per gathered chunk

template <class R>
using V = typename VecOf<R>::T;

struct FiberGeom {
  int k;                       // gate qubits
  uint8_t pos[MAX_WIDE_POS];   // their positions, ascending
};

__device__ __forceinline__ uint64_t fiber_base(uint64_t f, const FiberGeom& g) {
  for (int i = 0; i < g.k; ++i) {
    const int b = g.pos[i];
    f = ((f >> b) << (b + 1)) | (f & ((uint64_t(1) << b) - 1));
  }
  return f;
}

// X[b * ld + f] = amp[base(f0 + f) | off[b]] for b < 2^k, f < c
template <class R>
__global__ void __launch_bounds__(WIDE_THREADS) k_wide_gather(const V<R>* __restrict__ amp, V<R>* __restrict__ X,
                                                              const uint64_t* __restrict__ off, uint64_t f0, uint64_t c,
                                                              uint64_t ld, const FiberGeom g) {
  const uint64_t total = c << g.k;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    const uint64_t b = i / c, f = i - b * c;
    X[b * ld + f] = amp[fiber_base(f0 + f, g) | off[b]];
  }
}

template <class R>
__global__ void __launch_bounds__(WIDE_THREADS) k_wide_scatter(V<R>* __restrict__ amp, const V<R>* __restrict__ Y,
                                                               const uint64_t* __restrict__ off, uint64_t f0, uint64_t c,
                                                               uint64_t ld, const FiberGeom g) {
  const uint64_t total = c << g.k;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    const uint64_t a = i / c, f = i - a * c;
    amp[fiber_base(f0 + f, g) | off[a]] = Y[a * ld + f];
  }
}

// amp[base(f) | off[y]] = phase[y] * X[pre[y]][f] (unit[y]: the phase is exactly 1)
template <class R>
__global__ void __launch_bounds__(WIDE_THREADS) k_wide_permute(V<R>* __restrict__ amp, const V<R>* __restrict__ X,
                                                               const uint64_t* __restrict__ off,
                                                               const uint32_t* __restrict__ pre,
                                                               const V<R>* __restrict__ phase,
                                                               const uint8_t* __restrict__ unit, uint64_t f0,
                                                               uint64_t c, uint64_t ld, const FiberGeom g) {
  const uint64_t total = c << g.k;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    const uint64_t y = i / c, f = i - y * c;
    const V<R> v = X[uint64_t(pre[y]) * ld + f];
    amp[fiber_base(f0 + f, g) | off[y]] = unit[y] ? v : cmul(phase[y], v);
  }
}

// Y[a][f] = sum_b M[a][b] X[b][f]: M is K x K (row-major), X and Y are K x ld
// with c valid columns.  64 x 64 output tiles, K in steps of 16 staged in
// shared memory (M transposed so that a thread's four rows are one read).
constexpr int GT = 64, GK = 16;

template <class R>
__global__ void __launch_bounds__(WIDE_THREADS) k_wide_gemm(const V<R>* __restrict__ M, const V<R>* __restrict__ X,
                                                            V<R>* __restrict__ Y, uint32_t K, uint64_t c, uint64_t ld) {
  __shared__ V<R> As[GK][GT];  // As[kk][row]
  __shared__ V<R> Bs[GK][GT];  // Bs[kk][col]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const uint64_t col0 = uint64_t(blockIdx.x) * GT;
  const uint32_t row0 = blockIdx.y * GT;
  V<R> acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j].x = acc[i][j].y = R(0);
  for (uint32_t k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int e = threadIdx.x + r * WIDE_THREADS;  // 0..1023
      const int ar = e >> 4, ak = e & 15;            // M tile: 64 rows x 16 columns
      As[ak][ar] = M[uint64_t(row0 + ar) * K + k0 + ak];
      const int bk = e >> 6, bc = e & 63;  // X tile: 16 rows x 64 columns
      const uint64_t col = col0 + bc;
      V<R> v;
      v.x = v.y = R(0);
      if (col < c) v = X[uint64_t(k0 + bk) * ld + col];
      Bs[bk][bc] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      V<R> a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint64_t col = col0 + tx + 16 * j;
      if (col < c) Y[uint64_t(row0 + ty * 4 + i) * ld + col] = acc[i][j];
    }
}

template <class T>
T* pool_upload(const std::vector<T>& v, cudaStream_t st) {
  T* d = nullptr;
  NCSIM_CUDA(pool_alloc(&d, std::max<size_t>(1, v.size()) * sizeof(T), st));
  if (!v.empty()) NCSIM_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return d;
}

struct WidePlan {
  FiberGeom g{};
  std::vector<uint64_t> off;  // local index -> global offset bits
  uint64_t nfib = 0, chunk = 0;
};

WidePlan wide_plan(const ncsim_state* s, const std::vector<uint32_t>& qubits) {
  WidePlan p;
  const int k = int(qubits.size());
  if (k > MAX_WIDE_POS) throw Error(NCSIM_ERR_UNSUPPORTED, "gates on more than 24 qubits");
  p.g.k = k;
  std::vector<uint32_t> sq(qubits);
  std::sort(sq.begin(), sq.end());
  for (int i = 0; i < k; ++i) p.g.pos[i] = uint8_t(sq[i]);
  const uint64_t K = uint64_t(1) << k;
  p.off.resize(K);
  for (uint64_t b = 0; b < K; ++b) {
    uint64_t o = 0;
    for (int j = 0; j < k; ++j)
      if ((b >> j) & 1) o |= uint64_t(1) << qubits[j];
    p.off[b] = o;
  }
  p.nfib = s->len >> k;
  p.chunk = std::max<uint64_t>(1, std::min<uint64_t>(p.nfib, CHUNK_AMPS >> k));
  return p;
}

template <class R>
V<R> to_vr(const CplxD& c) {
  V<R> r;
  r.x = R(c.re);
  r.y = R(c.im);
  return r;
}

template <class R>
void dense_wide(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& m) {
  const WidePlan p = wide_plan(s, qubits);
  const int k = p.g.k;
  const uint32_t K = 1u << k;
  cudaStream_t st = s->stream;
  std::vector<V<R>> mh(size_t(K) * K);
  for (size_t i = 0; i < mh.size(); ++i) mh[i] = to_vr<R>(m[i]);
  V<R>* dM = pool_upload(mh, st);
  uint64_t* doff = pool_upload(p.off, st);
  V<R>*X = nullptr, *Y = nullptr;
  const uint64_t ld = p.chunk;
  NCSIM_CUDA(pool_alloc(&X, size_t(ld) * K * sizeof(V<R>), st));
  NCSIM_CUDA(pool_alloc(&Y, size_t(ld) * K * sizeof(V<R>), st));
  V<R>* a = reinterpret_cast<V<R>*>(s->amp);
  for (uint64_t f0 = 0; f0 < p.nfib; f0 += ld) {
    const uint64_t c = std::min(ld, p.nfib - f0);
    const unsigned gs = grid_for(c << k, WIDE_THREADS);
    k_wide_gather<R><<<gs, WIDE_THREADS, 0, st>>>(a, X, doff, f0, c, ld, p.g);
    const dim3 gg(unsigned((c + GT - 1) / GT), K / GT);
    k_wide_gemm<R><<<gg, WIDE_THREADS, 0, st>>>(dM, X, Y, K, c, ld);
    k_wide_scatter<R><<<gs, WIDE_THREADS, 0, st>>>(a, Y, doff, f0, c, ld, p.g);
  }
  NCSIM_LAUNCHED("dense_wide");
  for (void* q : {(void*)dM, (void*)doff, (void*)X, (void*)Y}) NCSIM_CUDA(cudaFreeAsync(q, st));
}

template <class R>
void perm_wide(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& image,
               const std::vector<CplxD>& phase) {
  const WidePlan p = wide_plan(s, qubits);
  const int k = p.g.k;
  const uint64_t K = uint64_t(1) << k;
  cudaStream_t st = s->stream;
  std::vector<uint32_t> pre(K);
  std::vector<V<R>> ph(K);
  std::vector<uint8_t> unit(K);
  for (uint64_t x = 0; x < K; ++x) {
    const uint32_t y = image[x];
    pre[y] = uint32_t(x);
    ph[y] = to_vr<R>(phase[x]);
    unit[y] = phase[x].re == 1.0 && phase[x].im == 0.0;
  }
  uint32_t* dpre = pool_upload(pre, st);
  V<R>* dph = pool_upload(ph, st);
  uint8_t* dunit = pool_upload(unit, st);
  uint64_t* doff = pool_upload(p.off, st);
  V<R>* X = nullptr;
  const uint64_t ld = p.chunk;
  NCSIM_CUDA(pool_alloc(&X, size_t(ld) * K * sizeof(V<R>), st));
  V<R>* a = reinterpret_cast<V<R>*>(s->amp);
  for (uint64_t f0 = 0; f0 < p.nfib; f0 += ld) {
    const uint64_t c = std::min(ld, p.nfib - f0);
    const unsigned gs = grid_for(c << k, WIDE_THREADS);
    k_wide_gather<R><<<gs, WIDE_THREADS, 0, st>>>(a, X, doff, f0, c, ld, p.g);
    k_wide_permute<R><<<gs, WIDE_THREADS, 0, st>>>(a, X, doff, dpre, dph, dunit, f0, c, ld, p.g);
  }
  NCSIM_LAUNCHED("perm_wide");
  for (void* q : {(void*)dpre, (void*)dph, (void*)dunit, (void*)doff, (void*)X}) NCSIM_CUDA(cudaFreeAsync(q, st));
}

}  // namespace

void launch_dense_wide(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& m) {
  if (qubits.size() < 6 || qubits.size() > MAX_WIDE_DENSE_K)
    throw Error(NCSIM_ERR_UNSUPPORTED, "wide dense gates take 6 to 13 qubits");
  ProfScope ps(s, K_DENSE_WIDE, 2.0 * double(s->bytes()));
  if (s->precision == NCSIM_C128) dense_wide<double>(s, qubits, m);
  else dense_wide<float>(s, qubits, m);
}

void launch_perm_wide(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& image,
                      const std::vector<CplxD>& phase) {
  if (qubits.size() > MAX_WIDE_MONOMIAL_K) throw Error(NCSIM_ERR_UNSUPPORTED, "monomial gates on more than 24 qubits");
  ProfScope ps(s, K_PERM_WIDE, 2.0 * double(s->bytes()));
  if (s->precision == NCSIM_C128) perm_wide<double>(s, qubits, image, phase);
  else perm_wide<float>(s, qubits, image, phase);
}

}  // namespace ncsim
