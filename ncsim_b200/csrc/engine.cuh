// Shared definitions of the B200 statevector engine: the state handle, error
// plumbing, device complex arithmetic and launch geometry.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ncsim_cuda.h"

namespace ncsim {

// ---------------------------------------------------------------------------
// errors: a status code (SimError variant, src/error.rs:7-42) and a message
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  ncsim_status code;
  // the fields of the variants that carry them (error.rs:17-33):
  // QubitOutOfRange {qubit, num_qubits}, DuplicateQubit(qubit), Arity {gate, expected, got}
  uint64_t qubit = 0, num_qubits = 0, expected = 0, got = 0;
  std::string gate;
  Error(ncsim_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// check_qubits's errors and apply_gate's arity error (error.rs:69-82, vector.rs:366-372)
inline Error qubit_out_of_range(uint64_t q, uint64_t n) {
  Error e(NCSIM_ERR_QUBIT_OUT_OF_RANGE, "qubit " + std::to_string(q) + " out of range for " + std::to_string(n) + " qubits");
  e.qubit = q;
  e.num_qubits = n;
  return e;
}
inline Error duplicate_qubit(uint64_t q) {
  Error e(NCSIM_ERR_DUPLICATE_QUBIT, "qubit " + std::to_string(q) + " listed twice");
  e.qubit = q;
  return e;
}
inline Error arity_error(const std::string& gate, uint64_t expected, uint64_t got) {
  Error e(NCSIM_ERR_ARITY, "gate " + gate + " acts on " + std::to_string(expected) + " qubits, " + std::to_string(got) + " given");
  e.gate = gate;
  e.expected = expected;
  e.got = got;
  return e;
}

void set_last_error(const std::string& m);
void set_last_error(const Error& e);

template <class F>
ncsim_status guarded(F&& f) {
  try {
    f();
    return NCSIM_OK;
  } catch (const Error& e) {
    set_last_error(e);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return NCSIM_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return NCSIM_ERR_INVALID;
  }
}

inline void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    throw Error(NCSIM_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
  }
  throw Error(NCSIM_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}
#define NCSIM_CUDA(call) ::ncsim::cuda_check((call), #call)
#define NCSIM_LAUNCHED(name) ::ncsim::cuda_check(cudaGetLastError(), name)

// ---------------------------------------------------------------------------
// device facts
// ---------------------------------------------------------------------------
int sm_count();
// the library's own stream-ordered pool on the current device (created on
// first use; keeps freed memory until trim_lib_pools)
cudaMemPool_t lib_pool();
void trim_lib_pools();
template <class T>
inline cudaError_t pool_alloc(T** p, size_t bytes, cudaStream_t st) {
  return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, lib_pool(), st);
}

// ---------------------------------------------------------------------------
// the state handle
// ---------------------------------------------------------------------------
constexpr int REDUCE_THREADS = 512;
constexpr int MAX_REDUCE_BLOCKS = 4096;
constexpr int PARTIAL_SLOTS = 4;  // doubles per block partial

}  // namespace ncsim

namespace ncsim {
// Kernel classes of the launch profiler.
enum KernelClass : int {
  K_DENSE1, K_DENSE2, K_DENSE_FIBER, K_DIAG, K_PAIRSWAP, K_PERM_TILE, K_PHASEPOLY, K_PAULI, K_NORM, K_EXPECT,
  K_INNER, K_PROJECT, K_SCALE, K_SAMPLE, K_FUSED_GEMM, K_FUSED_REMAP, K_OTHER, K_DENSE_WIDE, K_PERM_WIDE,
  K_PLAIN_PASS, K_NUM_CLASSES
};
const char* kernel_class_name(int c);
struct ProfRecord {
  int cls;
  double bytes;
  cudaEvent_t e0, e1;
};
}  // namespace ncsim

struct ncsim_state {
  uint32_t n = 0;
  int32_t precision = NCSIM_C128;
  uint64_t len = 0;         // 2^n amplitudes
  void* amp = nullptr;      // device: double2[len] or float2[len]
  cudaStream_t stream = nullptr;
  int device = 0;
  double* partials = nullptr;       // device scratch: MAX_REDUCE_BLOCKS * PARTIAL_SLOTS
  double* host_partials = nullptr;  // pinned mirror of `partials`
  int* dev_flag = nullptr;          // device word: a pass kernel's error code (kept for the state's life)
  mutable std::recursive_mutex mu;
  // launch profiler: an event pair per launch while enabled
  mutable bool prof = false;
  mutable std::vector<ncsim::ProfRecord> prof_recs;
  mutable std::vector<cudaEvent_t> prof_pool;
  cudaEvent_t timer0 = nullptr, timer1 = nullptr;
  uint64_t uid = 0;  // unique over the process: keys the circuits' captured gate graphs
  bool tile_passes = true;  // runs of gates go through tiled passes (plain_pass.cu)

  size_t elem_bytes() const { return precision == NCSIM_C128 ? 16 : 8; }
  size_t bytes() const { return size_t(len) * elem_bytes(); }
};

namespace ncsim {
// Records an event pair around the launches in its scope (when profiling).
struct ProfScope {
  const ncsim_state* s;
  int cls;
  double bytes;
  cudaEvent_t e0 = nullptr;
  ProfScope(const ncsim_state* st, int c, double b);
  ~ProfScope();
};
}  // namespace ncsim

namespace ncsim {

// ---------------------------------------------------------------------------
// device complex arithmetic (interleaved re/im), FP32 or FP64
// ---------------------------------------------------------------------------
template <class R> struct VecOf;
template <> struct VecOf<double> { using T = double2; };
template <> struct VecOf<float> { using T = float2; };

// Products and sums with a fixed rounding sequence (no contraction left to the
// compiler): every kernel that applies a gate computes the same bits for it,
// whichever kernel that is (the gate-by-gate kernels and the tiled passes).
#ifdef __CUDA_ARCH__
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
#else
inline double mul_rn(double a, double b) { return a * b; }
inline float mul_rn(float a, float b) { return a * b; }
inline double fma_rn(double a, double b, double c) { return __builtin_fma(a, b, c); }
inline float fma_rn(float a, float b, float c) { return __builtin_fmaf(a, b, c); }
inline double add_rn(double a, double b) { return a + b; }
inline float add_rn(float a, float b) { return a + b; }
#endif

template <class V>
__host__ __device__ __forceinline__ V cmul(V a, V b) {
  V r;
  r.x = fma_rn(a.x, b.x, -mul_rn(a.y, b.y));
  r.y = fma_rn(a.x, b.y, mul_rn(a.y, b.x));
  return r;
}
template <class V>
__host__ __device__ __forceinline__ V cadd(V a, V b) {
  V r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <class V>
__host__ __device__ __forceinline__ V cfma(V m, V x, V acc) {  // acc + m*x, two fused steps per part
  V r;
  r.x = fma_rn(m.x, x.x, fma_rn(-m.y, x.y, acc.x));
  r.y = fma_rn(m.x, x.y, fma_rn(m.y, x.x, acc.y));
  return r;
}
// Both parts +-0.  On the device an integer test of the bits (the floating-point
// compare would occupy the FP64 pipe next to the products).
template <class V>
__host__ __device__ __forceinline__ bool is_zero(V a) {
  return a.x == 0 && a.y == 0;
}
template <>
__host__ __device__ __forceinline__ bool is_zero<double2>(double2 a) {
#ifdef __CUDA_ARCH__
  return ((uint64_t(__double_as_longlong(a.x)) | uint64_t(__double_as_longlong(a.y))) << 1) == 0;
#else
  return a.x == 0 && a.y == 0;
#endif
}
template <>
__host__ __device__ __forceinline__ bool is_zero<float2>(float2 a) {
#ifdef __CUDA_ARCH__
  return ((__float_as_uint(a.x) | __float_as_uint(a.y)) << 1) == 0;
#else
  return a.x == 0 && a.y == 0;
#endif
}
// exactly 1 + 0i (either sign of the zero)
__host__ __device__ __forceinline__ bool is_one_v(double2 c) {
#ifdef __CUDA_ARCH__
  return uint64_t(__double_as_longlong(c.x)) == 0x3FF0000000000000ull && (uint64_t(__double_as_longlong(c.y)) << 1) == 0;
#else
  return c.x == 1.0 && c.y == 0.0;
#endif
}
__host__ __device__ __forceinline__ bool is_one_v(float2 c) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(c.x) == 0x3F800000u && (__float_as_uint(c.y) << 1) == 0;
#else
  return c.x == 1.0f && c.y == 0.0f;
#endif
}
// i^k * a for k mod 4
template <class V>
__host__ __device__ __forceinline__ V ipow_mul(int k, V a) {
  V r;
  switch (k & 3) {
    case 0: r = a; break;
    case 1: r.x = -a.y; r.y = a.x; break;
    case 2: r.x = -a.x; r.y = -a.y; break;
    default: r.x = a.y; r.y = -a.x; break;
  }
  return r;
}

// v with zero bits inserted at the ascending positions pos[0..cnt)
__host__ __device__ __forceinline__ uint64_t insert_zeros(uint64_t v, const uint8_t* pos, int cnt) {
  for (int i = 0; i < cnt; ++i) {
    int b = pos[i];
    v = ((v >> b) << (b + 1)) | (v & ((uint64_t(1) << b) - 1));
  }
  return v;
}

// grid of `blocks` for `items` work items at `per_thread` items per thread
inline unsigned grid_for(uint64_t items, int threads, int per_thread = 1, int max_waves = 32) {
  uint64_t b = (items + uint64_t(threads) * per_thread - 1) / (uint64_t(threads) * per_thread);
  uint64_t cap = uint64_t(sm_count()) * max_waves;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return unsigned(b);
}

// ---------------------------------------------------------------------------
// kernel launchers (kernels_plain.cu); all enqueue on s->stream
// ---------------------------------------------------------------------------
struct CplxD {
  double re, im;
};

void launch_dense(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& m);
// wide gates (wide.cu): dense matrices on 6..MAX_WIDE_DENSE_K qubits, monomial
// tables on up to MAX_WIDE_MONOMIAL_K qubits, through gathered chunks of fibers
constexpr int MAX_WIDE_DENSE_K = 13;
constexpr int MAX_WIDE_MONOMIAL_K = 24;
void launch_dense_wide(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& m);
void launch_perm_wide(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& image,
                      const std::vector<CplxD>& phase);
void launch_diag_table(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<CplxD>& diag);
void launch_perm_table(ncsim_state* s, const std::vector<uint32_t>& qubits, const std::vector<uint32_t>& image,
                       const std::vector<CplxD>& phase);
struct PolyTerms {
  uint32_t bits = 1;
  uint64_t constant = 0;
  std::vector<uint32_t> term_start;  // nterms + 1
  std::vector<uint64_t> parities;    // global index masks
  std::vector<uint64_t> coeffs;
  CplxD scalar{1.0, 0.0};
  bool scalar_is_one = true;
  std::vector<CplxD> root_table;     // exact phasor values scalar*zeta^f, when bits <= 8
};
void launch_phasepoly(ncsim_state* s, const PolyTerms& t);
void launch_pauli(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase);
void launch_scale(ncsim_state* s, CplxD c);
void launch_fill_plus(ncsim_state* s, double v);
void launch_set_basis(ncsim_state* s, uint64_t index);
void launch_convert_in(ncsim_state* s, const double2* src_dev, uint64_t offset, uint64_t count);
void launch_convert_out(const ncsim_state* s, double2* dst_dev, uint64_t offset, uint64_t count);
void launch_gather(const ncsim_state* s, const uint64_t* idx_dev, double2* out_dev, uint64_t count);
void launch_kron(const ncsim_state* a, const ncsim_state* b, ncsim_state* out);

// reductions: write per-block partials into s->partials, return the block count
int launch_norm_partials(const ncsim_state* s);
int launch_expect_partials(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, bool with_norm);
int launch_inner_partials(const ncsim_state* a, const ncsim_state* b);
int launch_project_partials(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, bool outcome);
// slots: <a|b> re, im, <a|a>, <b|b>; the per-block max |a-b| goes to maxdiff_dev[block]
int launch_compare_partials(const ncsim_state* a, const ncsim_state* b, double* maxdiff_dev);
// sampling
void launch_block_weights(const ncsim_state* s, double* weights_dev, uint64_t nblocks, uint64_t block);
void launch_sample_walk(const ncsim_state* s, const double* u_dev, const uint64_t* blk_dev, const double* acc_dev,
                        uint64_t shots, uint64_t block, uint64_t* out_dev);

// sum of `nb` partial slots (slot j of every block) in a fixed order on the host
void fetch_partials(const ncsim_state* s, int nb, int slots, double* out);

// state operations shared by both C ABI layers (capi_state.cu); the caller
// holds the state's lock
ncsim_state* state_new(uint32_t n, int32_t precision);
void state_free(ncsim_state* s);
CplxD state_norm_sq(const ncsim_state* s);
CplxD state_expectation(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase);
void state_measure_stats(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, double* e, double* nn);
CplxD state_project(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, bool outcome);
void state_set_amplitudes(ncsim_state* s, const double* amps, uint64_t len);
void state_get_amplitudes(const ncsim_state* s, double* amps, uint64_t len);
void state_gather(const ncsim_state* s, const uint64_t* idx, uint64_t count, double* out);
void state_sample(const ncsim_state* s, const double* uniforms, uint64_t shots, uint64_t* out);

}  // namespace ncsim
