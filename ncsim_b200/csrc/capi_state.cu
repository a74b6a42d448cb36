// C ABI, layer 1: state operations with plain-old-data arguments.  Each
// function validates its arguments on the host (the reference's checks in
// src/error.rs:69-82 and src/state/vector.rs), enqueues kernels on the state's
// stream, and waits only when it returns a value.
#include <atomic>
#include "engine.cuh"
#include "host_math.hpp"

#include <algorithm>
#include <numeric>

using namespace ncsim;

namespace ncsim {

thread_local std::string g_last_error;
thread_local ncsim_error_info g_last_info{};
void set_last_error(const std::string& m) {
  g_last_error = m;
  g_last_info = ncsim_error_info{};
  g_last_info.code = NCSIM_ERR_INVALID;
}
void set_last_error(const Error& e) {
  g_last_error = e.what();
  g_last_info = ncsim_error_info{};
  g_last_info.code = e.code;
  g_last_info.qubit = e.qubit;
  g_last_info.num_qubits = e.num_qubits;
  g_last_info.expected = e.expected;
  g_last_info.got = e.got;
  std::strncpy(g_last_info.gate, e.gate.c_str(), sizeof(g_last_info.gate) - 1);
}

int sm_count() {
  static int count = [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      cudaGetLastError();
      return 148;
    }
    return v > 0 ? v : 148;
  }();
  return count;
}

// The library's temporaries (readouts, staging buffers, the sparse form's
// sort buffers) come from a stream-ordered pool the library owns, one per
// device, created on first use.  A pool with the default release threshold of
// 0 hands freed memory back at every synchronisation, and the next allocation
// maps it again, which stalled runs by 100 ms and more at times; this pool
// keeps what it has (threshold UINT64_MAX) until ncsim_trim_memory or process
// exit.  The device's default pool, which other code in the process may use,
// is left as it is.
namespace {
constexpr int POOL_DEVICES = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[POOL_DEVICES] = {};
}  // namespace

cudaMemPool_t lib_pool() {
  int dev = 0;
  NCSIM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= POOL_DEVICES) throw Error(NCSIM_ERR_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    NCSIM_CUDA(cudaMemPoolCreate(&p, &props));
    uint64_t keep = UINT64_MAX;
    NCSIM_CUDA(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pool[dev] = p;
  }
  return g_pool[dev];
}

void trim_lib_pools() {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (int d = 0; d < POOL_DEVICES; ++d)
    if (g_pool[d]) NCSIM_CUDA(cudaMemPoolTrimTo(g_pool[d], 0));
}

namespace {

void need(const void* p, const char* what) {
  if (!p) throw Error(NCSIM_ERR_INVALID, std::string(what) + " is null");
}

// check_qubits (src/error.rs:69-82)
void check_qubits(const uint32_t* qubits, uint32_t k, uint32_t n) {
  if (k && !qubits) throw Error(NCSIM_ERR_INVALID, "qubit list is null");
  for (uint32_t i = 0; i < k; ++i) {
    if (qubits[i] >= n) throw qubit_out_of_range(qubits[i], n);
    for (uint32_t j = 0; j < i; ++j)
      if (qubits[j] == qubits[i]) throw duplicate_qubit(qubits[i]);
  }
}

uint64_t reg_mask(uint32_t n) { return n >= 64 ? ~uint64_t(0) : ((uint64_t(1) << n) - 1); }

void check_pauli(const ncsim_state* s, uint64_t x, uint64_t z) {
  if ((x | z) & ~reg_mask(s->n)) throw Error(NCSIM_ERR_INVALID, "Pauli acts outside the register");
}

bool hermitian(uint64_t x, uint64_t z, uint32_t phase) {  // src/pauli/ops.rs:25-27
  return ((phase & 1) == 1) == bool(__builtin_popcountll(x & z) & 1);
}

}  // namespace

const char* kernel_class_name(int c) {
  static const char* names[K_NUM_CLASSES] = {"dense1", "dense2", "dense_fiber", "diag", "pairswap", "perm_tile",
                                             "phasepoly", "pauli", "norm", "expect", "inner", "project", "scale",
                                             "sample", "fused_gemm", "fused_remap", "other", "dense_wide",
                                             "perm_wide", "plain_pass"};
  return (c >= 0 && c < K_NUM_CLASSES) ? names[c] : "other";
}

static cudaEvent_t prof_event(const ncsim_state* s) {
  if (!s->prof_pool.empty()) {
    cudaEvent_t e = s->prof_pool.back();
    s->prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  NCSIM_CUDA(cudaEventCreate(&e));
  return e;
}

ProfScope::ProfScope(const ncsim_state* st, int c, double b) : s(st), cls(c), bytes(b) {
  if (!s->prof) return;
  e0 = prof_event(s);
  NCSIM_CUDA(cudaEventRecord(e0, s->stream));
}

ProfScope::~ProfScope() {
  if (!e0) return;
  cudaEvent_t e1 = nullptr;
  try {
    e1 = prof_event(s);
  } catch (...) {
    return;
  }
  if (cudaEventRecord(e1, s->stream) != cudaSuccess) return;
  s->prof_recs.push_back({cls, bytes, e0, e1});
}

// state lifecycle (shared with the host layer)
ncsim_state* state_new(uint32_t n, int32_t precision) {
  if (precision != NCSIM_C128 && precision != NCSIM_C64) throw Error(NCSIM_ERR_INVALID, "precision must be C128 or C64");
  const uint32_t cap = precision == NCSIM_C128 ? 33 : 34;
  if (n > cap) throw Error(NCSIM_ERR_INVALID, "state vector of " + std::to_string(n) + " qubits exceeds " + std::to_string(cap));
  static std::atomic<uint64_t> next_uid{1};
  auto* s = new ncsim_state();
  s->uid = next_uid.fetch_add(1);
  s->n = n;
  s->precision = precision;
  s->len = uint64_t(1) << n;
  try {
    NCSIM_CUDA(cudaGetDevice(&s->device));
    NCSIM_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    NCSIM_CUDA(cudaMalloc(&s->amp, s->bytes()));
    NCSIM_CUDA(cudaMalloc(&s->partials, sizeof(double) * MAX_REDUCE_BLOCKS * PARTIAL_SLOTS));
    NCSIM_CUDA(cudaMallocHost(&s->host_partials, sizeof(double) * MAX_REDUCE_BLOCKS * PARTIAL_SLOTS));
    NCSIM_CUDA(cudaMalloc(&s->dev_flag, 256));
  } catch (...) {
    if (s->amp) cudaFree(s->amp);
    if (s->partials) cudaFree(s->partials);
    if (s->dev_flag) cudaFree(s->dev_flag);
    if (s->host_partials) cudaFreeHost(s->host_partials);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    throw;
  }
  return s;
}

void state_free(ncsim_state* s) {
  if (!s) return;
  cudaStreamSynchronize(s->stream);
  for (auto& r : s->prof_recs) cudaEventDestroy(r.e0), cudaEventDestroy(r.e1);
  for (auto e : s->prof_pool) cudaEventDestroy(e);
  if (s->timer0) cudaEventDestroy(s->timer0);
  if (s->timer1) cudaEventDestroy(s->timer1);
  cudaFree(s->amp);
  cudaFree(s->partials);
  cudaFree(s->dev_flag);
  cudaFreeHost(s->host_partials);
  cudaStreamDestroy(s->stream);
  delete s;
}

CplxD state_norm_sq(const ncsim_state* s) {
  double v;
  int nb = launch_norm_partials(s);
  fetch_partials(s, nb, 1, &v);
  return {v, 0.0};
}

CplxD state_expectation(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase) {
  check_pauli(s, x, z);
  double v[2];
  int nb = launch_expect_partials(s, x, z, phase, false);
  fetch_partials(s, nb, 2, v);
  return {v[0], v[1]};
}

void state_measure_stats(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, double* e, double* nn) {
  check_pauli(s, x, z);
  double v[3];
  int nb = launch_expect_partials(s, x, z, phase, true);
  fetch_partials(s, nb, 3, v);
  e[0] = v[0];
  e[1] = v[1];
  *nn = v[2];
}

CplxD state_project(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, bool outcome) {
  check_pauli(s, x, z);
  if (!hermitian(x, z, phase)) throw Error(NCSIM_ERR_INVALID, "projector of a non-Hermitian Pauli");
  double v;
  int nb = launch_project_partials(s, x, z, phase, outcome);
  fetch_partials(s, nb, 1, &v);
  return {v, 0.0};
}

static void state_apply_matrix(ncsim_state* s, const std::vector<uint32_t>& q, const std::vector<CplxD>& m) {
  launch_dense(s, q, m);
}

void state_set_amplitudes(ncsim_state* s, const double* amps, uint64_t len) {
  if (len != s->len) throw Error(NCSIM_ERR_INVALID, std::to_string(len) + " amplitudes for " + std::to_string(s->n) + " qubits");
  need(amps, "amplitudes");
  if (s->precision == NCSIM_C128) {
    NCSIM_CUDA(cudaMemcpyAsync(s->amp, amps, s->bytes(), cudaMemcpyHostToDevice, s->stream));
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    return;
  }
  const uint64_t chunk = std::min<uint64_t>(len, uint64_t(1) << 24);
  double2* stage = nullptr;
  NCSIM_CUDA(pool_alloc(&stage, chunk * sizeof(double2), s->stream));
  for (uint64_t off = 0; off < len; off += chunk) {
    uint64_t c = std::min(chunk, len - off);
    NCSIM_CUDA(cudaMemcpyAsync(stage, amps + 2 * off, c * sizeof(double2), cudaMemcpyHostToDevice, s->stream));
    launch_convert_in(s, stage, off, c);
  }
  NCSIM_CUDA(cudaFreeAsync(stage, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
}

// amplitudes [first, first + count) as complex128 into host memory
static void state_get_range(const ncsim_state* s, uint64_t first, uint64_t count, double* amps) {
  if (first > s->len || count > s->len - first) throw Error(NCSIM_ERR_INVALID, "amplitude range outside the register");
  if (count == 0) return;
  need(amps, "amplitudes");
  if (s->precision == NCSIM_C128) {
    NCSIM_CUDA(cudaMemcpyAsync(amps, static_cast<const double2*>(s->amp) + first, count * sizeof(double2),
                               cudaMemcpyDeviceToHost, s->stream));
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    return;
  }
  const uint64_t chunk = std::min<uint64_t>(count, uint64_t(1) << 24);
  double2* stage = nullptr;
  NCSIM_CUDA(pool_alloc(&stage, chunk * sizeof(double2), s->stream));
  for (uint64_t off = 0; off < count; off += chunk) {
    uint64_t c = std::min(chunk, count - off);
    launch_convert_out(s, stage, first + off, c);
    NCSIM_CUDA(cudaMemcpyAsync(amps + 2 * off, stage, c * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  }
  NCSIM_CUDA(cudaFreeAsync(stage, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
}

void state_get_amplitudes(const ncsim_state* s, double* amps, uint64_t len) {
  if (len != s->len) throw Error(NCSIM_ERR_INVALID, "amplitude buffer length differs from 2^n");
  state_get_range(s, 0, len, amps);
}

void state_gather(const ncsim_state* s, const uint64_t* idx, uint64_t count, double* out) {
  if (count == 0) return;
  need(idx, "indices");
  need(out, "output");
  uint64_t* d_idx = nullptr;
  double2* d_out = nullptr;
  NCSIM_CUDA(pool_alloc(&d_idx, count * sizeof(uint64_t), s->stream));
  NCSIM_CUDA(pool_alloc(&d_out, count * sizeof(double2), s->stream));
  NCSIM_CUDA(cudaMemcpyAsync(d_idx, idx, count * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream));
  launch_gather(s, d_idx, d_out, count);
  NCSIM_CUDA(cudaMemcpyAsync(out, d_out, count * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  NCSIM_CUDA(cudaFreeAsync(d_idx, s->stream));
  NCSIM_CUDA(cudaFreeAsync(d_out, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
}

// StateVector::sample (vector.rs:494-540): block weights on the device, the
// block of every shot on the host (the reference's sequential running sum),
// the walk inside the block on the device.
void state_sample(const ncsim_state* s, const double* uniforms, uint64_t shots, uint64_t* out) {
  const uint64_t block = std::min<uint64_t>(4096, s->len);
  const uint64_t nblocks = s->len / block;
  std::vector<double> w(nblocks);
  double* d_w = nullptr;
  NCSIM_CUDA(pool_alloc(&d_w, nblocks * sizeof(double), s->stream));
  launch_block_weights(s, d_w, nblocks, block);
  NCSIM_CUDA(cudaMemcpyAsync(w.data(), d_w, nblocks * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  NCSIM_CUDA(cudaFreeAsync(d_w, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  std::vector<double> hi(nblocks);
  double total = 0.0;
  for (uint64_t b = 0; b < nblocks; ++b) {
    total += w[b];
    hi[b] = total;
  }
  if (!(total > 0.0)) throw Error(NCSIM_ERR_ZERO_STATE, "state vanished: sample");
  if (shots == 0) return;
  need(uniforms, "uniforms");
  need(out, "output");
  std::vector<double> u(shots), acc(shots);
  std::vector<uint64_t> blk(shots);
  for (uint64_t k = 0; k < shots; ++k) {
    u[k] = uniforms[k] * total;
    // the first block whose running sum exceeds u, else the last block
    uint64_t b = uint64_t(std::upper_bound(hi.begin(), hi.end(), u[k]) - hi.begin());
    if (b >= nblocks) b = nblocks - 1;
    blk[k] = b;
    acc[k] = b ? hi[b - 1] : 0.0;
  }
  double *d_u = nullptr, *d_acc = nullptr;
  uint64_t *d_blk = nullptr, *d_out = nullptr;
  NCSIM_CUDA(pool_alloc(&d_u, shots * sizeof(double), s->stream));
  NCSIM_CUDA(pool_alloc(&d_acc, shots * sizeof(double), s->stream));
  NCSIM_CUDA(pool_alloc(&d_blk, shots * sizeof(uint64_t), s->stream));
  NCSIM_CUDA(pool_alloc(&d_out, shots * sizeof(uint64_t), s->stream));
  NCSIM_CUDA(cudaMemcpyAsync(d_u, u.data(), shots * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  NCSIM_CUDA(cudaMemcpyAsync(d_acc, acc.data(), shots * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  NCSIM_CUDA(cudaMemcpyAsync(d_blk, blk.data(), shots * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream));
  launch_sample_walk(s, d_u, d_blk, d_acc, shots, block, d_out);
  NCSIM_CUDA(cudaMemcpyAsync(out, d_out, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
  for (void* p : {(void*)d_u, (void*)d_acc, (void*)d_blk, (void*)d_out}) NCSIM_CUDA(cudaFreeAsync(p, s->stream));
  NCSIM_CUDA(cudaStreamSynchronize(s->stream));
}

// the host-side views of a monomial table (vector.rs:96-139)
static void state_apply_monomial(ncsim_state* s, const std::vector<uint32_t>& q, const std::vector<uint32_t>& image,
                          const std::vector<CplxD>& phase) {
  launch_perm_table(s, q, image, phase);
}

}  // namespace ncsim

// ===========================================================================
extern "C" {

const char* ncsim_last_error(void) { return ncsim::g_last_error.c_str(); }
ncsim_status ncsim_last_error_info(ncsim_error_info* out) {
  if (!out) return NCSIM_ERR_INVALID;
  *out = ncsim::g_last_info;
  return NCSIM_OK;
}
int32_t ncsim_abi_version(void) { return 10000; }

ncsim_status ncsim_device_info(int32_t* sm, uint64_t* free_b, uint64_t* total_b) {
  return guarded([&] {
    int dev = 0;
    NCSIM_CUDA(cudaGetDevice(&dev));
    int v = 0;
    NCSIM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    size_t f = 0, t = 0;
    NCSIM_CUDA(cudaMemGetInfo(&f, &t));
    if (sm) *sm = v;
    if (free_b) *free_b = f;
    if (total_b) *total_b = t;
  });
}

ncsim_status ncsim_trim_memory(void) {
  return guarded([&] { trim_lib_pools(); });
}

ncsim_status ncsim_pool_info(uint64_t* reserved_bytes, uint64_t* used_bytes) {
  return guarded([&] {
    cudaMemPool_t p = lib_pool();
    uint64_t r = 0, u = 0;
    NCSIM_CUDA(cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &r));
    NCSIM_CUDA(cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &u));
    if (reserved_bytes) *reserved_bytes = r;
    if (used_bytes) *used_bytes = u;
  });
}

ncsim_status ncsim_sv_create(uint32_t n, int32_t precision, ncsim_state** out) {
  return guarded([&] {
    need(out, "out");
    *out = nullptr;
    ncsim_state* s = state_new(n, precision);
    try {
      launch_set_basis(s, 0);
      NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    } catch (...) {
      state_free(s);
      throw;
    }
    *out = s;
  });
}

ncsim_status ncsim_sv_destroy(ncsim_state* s) {
  return guarded([&] { state_free(s); });
}

ncsim_status ncsim_sv_clone(const ncsim_state* s, ncsim_state** out) {
  return guarded([&] {
    need(s, "state");
    need(out, "out");
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    ncsim_state* c = state_new(s->n, s->precision);
    try {
      NCSIM_CUDA(cudaStreamSynchronize(s->stream));
      NCSIM_CUDA(cudaMemcpyAsync(c->amp, s->amp, s->bytes(), cudaMemcpyDeviceToDevice, c->stream));
      NCSIM_CUDA(cudaStreamSynchronize(c->stream));
    } catch (...) {
      state_free(c);
      throw;
    }
    *out = c;
  });
}

ncsim_status ncsim_sv_num_qubits(const ncsim_state* s, uint32_t* n) {
  return guarded([&] {
    need(s, "state");
    need(n, "out");
    *n = s->n;
  });
}

ncsim_status ncsim_sv_precision(const ncsim_state* s, int32_t* p) {
  return guarded([&] {
    need(s, "state");
    need(p, "out");
    *p = s->precision;
  });
}

ncsim_status ncsim_sv_set_basis(ncsim_state* s, uint64_t index) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    launch_set_basis(s, index & reg_mask(s->n));
  });
}

ncsim_status ncsim_sv_set_plus(ncsim_state* s) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    launch_fill_plus(s, sqrt2_power(-int64_t(s->n)));
  });
}

ncsim_status ncsim_sv_set_amplitudes(ncsim_state* s, const double* amps, uint64_t len) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_set_amplitudes(s, amps, len);
  });
}

ncsim_status ncsim_sv_get_amplitudes(const ncsim_state* s, double* amps, uint64_t len) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_get_amplitudes(s, amps, len);
  });
}

ncsim_status ncsim_sv_get_amplitudes_range(const ncsim_state* s, uint64_t first, uint64_t count, double* amps) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_get_range(s, first, count, amps);
  });
}

ncsim_status ncsim_sv_get_amplitude(const ncsim_state* s, uint64_t index, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    uint64_t i = index & reg_mask(s->n);
    state_gather(s, &i, 1, re_im);
  });
}

ncsim_status ncsim_sv_gather_amplitudes(const ncsim_state* s, const uint64_t* idx, uint64_t count, double* out) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_gather(s, idx, count, out);
  });
}

ncsim_status ncsim_sv_apply_matrix(ncsim_state* s, const uint32_t* qubits, uint32_t k, const double* m) {
  return guarded([&] {
    need(s, "state");
    check_qubits(qubits, k, s->n);
    if (k == 0) return;
    if (k > uint32_t(MAX_WIDE_DENSE_K))
      throw Error(NCSIM_ERR_UNSUPPORTED, "dense matrices on more than " + std::to_string(MAX_WIDE_DENSE_K) + " qubits");
    need(m, "matrix");
    std::vector<uint32_t> q(qubits, qubits + k);
    const size_t gd = size_t(1) << k;
    std::vector<CplxD> mm(gd * gd);
    for (size_t i = 0; i < gd * gd; ++i) mm[i] = {m[2 * i], m[2 * i + 1]};
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_apply_matrix(s, q, mm);
  });
}

ncsim_status ncsim_sv_apply_monomial(ncsim_state* s, const uint32_t* qubits, uint32_t k, const uint64_t* image,
                                     const double* phase) {
  return guarded([&] {
    need(s, "state");
    check_qubits(qubits, k, s->n);
    if (k == 0) return;
    if (k > uint32_t(MAX_WIDE_MONOMIAL_K))
      throw Error(NCSIM_ERR_UNSUPPORTED, "monomial tables on more than " + std::to_string(MAX_WIDE_MONOMIAL_K) + " qubits");
    need(image, "image");
    need(phase, "phase");
    const size_t gd = size_t(1) << k;
    std::vector<uint32_t> img(gd);
    std::vector<char> seen(gd, 0);
    std::vector<CplxD> ph(gd);
    for (size_t x = 0; x < gd; ++x) {
      if (image[x] >= gd || seen[image[x]]) throw Error(NCSIM_ERR_INVALID, "monomial image is not a permutation");
      seen[image[x]] = 1;
      img[x] = uint32_t(image[x]);
      ph[x] = {phase[2 * x], phase[2 * x + 1]};
    }
    std::vector<uint32_t> q(qubits, qubits + k);
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_apply_monomial(s, q, img, ph);
  });
}

ncsim_status ncsim_sv_apply_phasepoly(ncsim_state* s, const uint32_t* qubits, uint32_t k, uint32_t bits, uint64_t constant,
                                      uint32_t nterms, const uint32_t* term_start, const uint64_t* parities,
                                      const uint64_t* coeffs, int32_t s2, uint64_t sphase, uint32_t sbits) {
  return guarded([&] {
    need(s, "state");
    check_qubits(qubits, k, s->n);
    if (bits < 1 || bits > 32) throw Error(NCSIM_ERR_INVALID, "phase bits must be in 1..=32");
    if (sbits > 62) throw Error(NCSIM_ERR_INVALID, "scalar phase bits must be at most 62");
    PolyTerms t;
    t.bits = bits;
    const uint64_t modmask = (uint64_t(1) << bits) - 1;
    t.constant = constant & modmask;
    if (nterms) {
      need(term_start, "term_start");
      need(coeffs, "coeffs");
    }
    t.term_start.push_back(0);
    for (uint32_t i = 0; i < nterms; ++i) {
      if (term_start[i + 1] < term_start[i]) throw Error(NCSIM_ERR_INVALID, "term_start must be non-decreasing");
      if (i == 0 && term_start[0] != 0) throw Error(NCSIM_ERR_INVALID, "term_start[0] must be 0");
      bool vanishes = false;
      std::vector<uint64_t> glob;
      for (uint32_t l = term_start[i]; l < term_start[i + 1]; ++l) {
        uint64_t lm = parities[l] & reg_mask(k);
        if (lm == 0) vanishes = true;  // a zero parity makes the term vanish (phasepoly.rs:605)
        uint64_t g = 0;
        for (uint32_t j = 0; j < k; ++j)
          if ((lm >> j) & 1) g |= uint64_t(1) << qubits[j];
        glob.push_back(g);
      }
      uint64_t c = coeffs[i] & modmask;
      if (vanishes || c == 0) continue;
      if (glob.empty()) {  // an empty product is the constant 1
        t.constant = (t.constant + c) & modmask;
        continue;
      }
      t.parities.insert(t.parities.end(), glob.begin(), glob.end());
      t.coeffs.push_back(c);
      t.term_start.push_back(uint32_t(t.parities.size()));
    }
    Phase sc = Phase::make(s2, int64_t(sphase % (uint64_t(1) << sbits)), sbits);
    t.scalar_is_one = sc.is_one();
    Cd sv = sc.value();
    t.scalar = {sv.re, sv.im};
    if (bits <= 8) {
      t.root_table.resize(size_t(1) << bits);
      for (uint64_t f = 0; f < (uint64_t(1) << bits); ++f) {
        Cd v = sc.times(Phase::make(0, int64_t(f), bits)).value();
        t.root_table[f] = {v.re, v.im};
      }
    }
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    launch_phasepoly(s, t);
  });
}

ncsim_status ncsim_sv_apply_pauli(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase) {
  return guarded([&] {
    need(s, "state");
    check_pauli(s, x, z);
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    launch_pauli(s, x, z, phase & 3);
  });
}

ncsim_status ncsim_sv_norm_sq(const ncsim_state* s, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    CplxD v = state_norm_sq(s);
    re_im[0] = v.re;
    re_im[1] = v.im;
  });
}

ncsim_status ncsim_sv_expectation(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, double* re_im) {
  return guarded([&] {
    need(s, "state");
    need(re_im, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    CplxD v = state_expectation(s, x, z, phase & 3);
    re_im[0] = v.re;
    re_im[1] = v.im;
  });
}

ncsim_status ncsim_sv_measure_stats(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, double* e, double* nn) {
  return guarded([&] {
    need(s, "state");
    need(e, "out");
    need(nn, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_measure_stats(s, x, z, phase & 3, e, nn);
  });
}

ncsim_status ncsim_sv_inner(const ncsim_state* a, const ncsim_state* b, double* re_im) {
  return guarded([&] {
    need(a, "state");
    need(b, "state");
    need(re_im, "out");
    if (a->n != b->n) throw Error(NCSIM_ERR_INVALID, "inner: register sizes differ");
    if (a->precision != b->precision) throw Error(NCSIM_ERR_INVALID, "inner: precisions differ");
    std::unique_lock<std::recursive_mutex> la(a->mu, std::defer_lock), lb(b->mu, std::defer_lock);
    if (a == b) la.lock();
    else std::lock(la, lb);
    if (a != b) NCSIM_CUDA(cudaStreamSynchronize(b->stream));
    double v[2];
    int nb = launch_inner_partials(a, b);
    fetch_partials(a, nb, 2, v);
    re_im[0] = v[0];
    re_im[1] = v[1];
  });
}

ncsim_status ncsim_sv_project(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, int32_t outcome, double* w) {
  return guarded([&] {
    need(s, "state");
    need(w, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    CplxD v = state_project(s, x, z, phase & 3, outcome != 0);
    w[0] = v.re;
    w[1] = v.im;
  });
}

ncsim_status ncsim_sv_scale(ncsim_state* s, double re, double im) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    launch_scale(s, {re, im});
  });
}

ncsim_status ncsim_sv_sample(const ncsim_state* s, const double* uniforms, uint64_t shots, uint64_t* out) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    state_sample(s, uniforms, shots, out);
  });
}

ncsim_status ncsim_sv_kron(const ncsim_state* a, const ncsim_state* b, ncsim_state** out) {
  return guarded([&] {
    need(a, "state");
    need(b, "state");
    need(out, "out");
    *out = nullptr;
    if (a->precision != b->precision) throw Error(NCSIM_ERR_INVALID, "kron: precisions differ");
    std::unique_lock<std::recursive_mutex> la(a->mu, std::defer_lock), lb(b->mu, std::defer_lock);
    if (a == b) la.lock();
    else std::lock(la, lb);
    ncsim_state* o = state_new(a->n + b->n, a->precision);
    try {
      NCSIM_CUDA(cudaStreamSynchronize(a->stream));
      NCSIM_CUDA(cudaStreamSynchronize(b->stream));
      launch_kron(a, b, o);
      NCSIM_CUDA(cudaStreamSynchronize(o->stream));
    } catch (...) {
      state_free(o);
      throw;
    }
    *out = o;
  });
}

ncsim_status ncsim_sv_device_pointer(const ncsim_state* s, void** ptr, uint64_t* bytes) {
  return guarded([&] {
    need(s, "state");
    need(ptr, "out");
    *ptr = s->amp;
    if (bytes) *bytes = s->bytes();
  });
}

ncsim_status ncsim_sv_block_weights(const ncsim_state* s, uint64_t block, double* out, uint64_t nblocks) {
  return guarded([&] {
    need(s, "state");
    need(out, "out");
    if (block == 0 || (block & (block - 1)) || block > s->len) throw Error(NCSIM_ERR_INVALID, "block must be a power of two <= 2^n");
    if (nblocks != s->len / block) throw Error(NCSIM_ERR_INVALID, "output holds 2^n / block weights");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    double* d_w = nullptr;
    NCSIM_CUDA(pool_alloc(&d_w, nblocks * sizeof(double), s->stream));
    launch_block_weights(s, d_w, nblocks, block);
    NCSIM_CUDA(cudaMemcpyAsync(out, d_w, nblocks * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    NCSIM_CUDA(cudaFreeAsync(d_w, s->stream));
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  });
}

ncsim_status ncsim_sv_sample_walk(const ncsim_state* s, uint64_t block, const double* targets, const uint64_t* blocks,
                                  const double* accs, uint64_t shots, uint64_t* out) {
  return guarded([&] {
    need(s, "state");
    if (block == 0 || (block & (block - 1)) || block > s->len) throw Error(NCSIM_ERR_INVALID, "block must be a power of two <= 2^n");
    if (shots == 0) return;
    need(targets, "targets");
    need(blocks, "blocks");
    need(accs, "accs");
    need(out, "out");
    for (uint64_t k = 0; k < shots; ++k)
      if (blocks[k] >= s->len / block) throw Error(NCSIM_ERR_INVALID, "block index outside the register");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    double *d_u = nullptr, *d_acc = nullptr;
    uint64_t *d_blk = nullptr, *d_out = nullptr;
    NCSIM_CUDA(pool_alloc(&d_u, shots * sizeof(double), s->stream));
    NCSIM_CUDA(pool_alloc(&d_acc, shots * sizeof(double), s->stream));
    NCSIM_CUDA(pool_alloc(&d_blk, shots * sizeof(uint64_t), s->stream));
    NCSIM_CUDA(pool_alloc(&d_out, shots * sizeof(uint64_t), s->stream));
    NCSIM_CUDA(cudaMemcpyAsync(d_u, targets, shots * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    NCSIM_CUDA(cudaMemcpyAsync(d_acc, accs, shots * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    NCSIM_CUDA(cudaMemcpyAsync(d_blk, blocks, shots * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream));
    launch_sample_walk(s, d_u, d_blk, d_acc, shots, block, d_out);
    NCSIM_CUDA(cudaMemcpyAsync(out, d_out, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
    for (void* p : {(void*)d_u, (void*)d_acc, (void*)d_blk, (void*)d_out}) NCSIM_CUDA(cudaFreeAsync(p, s->stream));
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  });
}

ncsim_status ncsim_sv_synchronize(const ncsim_state* s) {
  return guarded([&] {
    need(s, "state");
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
  });
}

ncsim_status ncsim_sv_timer_start(ncsim_state* s) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    if (!s->timer0) NCSIM_CUDA(cudaEventCreate(&s->timer0));
    if (!s->timer1) NCSIM_CUDA(cudaEventCreate(&s->timer1));
    NCSIM_CUDA(cudaEventRecord(s->timer0, s->stream));
  });
}

ncsim_status ncsim_sv_timer_stop(ncsim_state* s, double* ms) {
  return guarded([&] {
    need(s, "state");
    need(ms, "out");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    if (!s->timer0) throw Error(NCSIM_ERR_INVALID, "timer was not started");
    NCSIM_CUDA(cudaEventRecord(s->timer1, s->stream));
    NCSIM_CUDA(cudaEventSynchronize(s->timer1));
    float f = 0.f;
    NCSIM_CUDA(cudaEventElapsedTime(&f, s->timer0, s->timer1));
    *ms = f;
  });
}

ncsim_status ncsim_sv_compare(const ncsim_state* a, const ncsim_state* b, double* inner, double* na, double* nb,
                              double* maxdiff) {
  return guarded([&] {
    need(a, "state");
    need(b, "state");
    if (a->n != b->n) throw Error(NCSIM_ERR_INVALID, "compare: register sizes differ");
    std::unique_lock<std::recursive_mutex> la(a->mu, std::defer_lock), lb(b->mu, std::defer_lock);
    if (a == b) la.lock();
    else std::lock(la, lb);
    if (a != b) NCSIM_CUDA(cudaStreamSynchronize(b->stream));
    double* d_max = nullptr;
    NCSIM_CUDA(pool_alloc(&d_max, sizeof(double) * MAX_REDUCE_BLOCKS, a->stream));
    int g = launch_compare_partials(a, b, d_max);
    std::vector<double> mx(g);
    NCSIM_CUDA(cudaMemcpyAsync(mx.data(), d_max, sizeof(double) * g, cudaMemcpyDeviceToHost, a->stream));
    NCSIM_CUDA(cudaFreeAsync(d_max, a->stream));
    double v[4];
    fetch_partials(a, g, 4, v);
    if (inner) inner[0] = v[0], inner[1] = v[1];
    if (na) *na = v[2];
    if (nb) *nb = v[3];
    if (maxdiff) *maxdiff = *std::max_element(mx.begin(), mx.end());
  });
}

ncsim_status ncsim_sv_set_tile_passes(ncsim_state* s, int32_t enable) {
  return guarded([&] {
    if (!s) throw Error(NCSIM_ERR_INVALID, "null state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    s->tile_passes = enable != 0;
  });
}

ncsim_status ncsim_sv_profile_enable(ncsim_state* s, int32_t enable) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    for (auto& r : s->prof_recs) s->prof_pool.push_back(r.e0), s->prof_pool.push_back(r.e1);
    s->prof_recs.clear();
    s->prof = enable != 0;
  });
}

ncsim_status ncsim_sv_profile_read(ncsim_state* s, ncsim_kernel_stat* out, uint32_t cap, uint32_t* count) {
  return guarded([&] {
    need(s, "state");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    NCSIM_CUDA(cudaStreamSynchronize(s->stream));
    std::vector<ncsim_kernel_stat> agg(K_NUM_CLASSES);
    for (int c = 0; c < K_NUM_CLASSES; ++c) {
      std::memset(&agg[c], 0, sizeof(ncsim_kernel_stat));
      std::strncpy(agg[c].name, kernel_class_name(c), sizeof(agg[c].name) - 1);
    }
    for (auto& r : s->prof_recs) {
      float ms = 0.f;
      NCSIM_CUDA(cudaEventElapsedTime(&ms, r.e0, r.e1));
      auto& a = agg[r.cls];
      a.launches += 1;
      a.milliseconds += ms;
      a.bytes += r.bytes;
    }
    uint32_t m = 0;
    for (int c = 0; c < K_NUM_CLASSES; ++c)
      if (agg[c].launches) {
        if (out && m < cap) out[m] = agg[c];
        ++m;
      }
    if (count) *count = m;
  });
}

}  // extern "C"
