/*
 * ncsim_cuda.h — C ABI of the B200 dense statevector engine (libncsim_cuda.so).
 *
 * The engine is a drop-in for ncsim's `StateVector<C64>` behind the
 * `QuantumState<C64>` trait (reference: src/state/mod.rs:41-234,
 * src/state/vector.rs:16-549).  A thin Rust crate (`ncsim-cuda`) binds these
 * functions and implements `GpuStateVector: QuantumState<C64>`; the core crate
 * keeps `#![forbid(unsafe_code)]` (src/lib.rs:36).
 *
 * Three layers are exported:
 *   1. state operations with plain-old-data arguments (pointers, sizes, bit
 *      masks, row-major complex128 arrays): what the Rust crate calls after it
 *      lowers a `Gate` through the reference's own views
 *      (`Gate::monomial/matrix`, src/gate.rs:519-747);
 *   2. a C++ host mirror of the trait's provided methods (run, measure,
 *      sample with a seeded StdRng, text circuits) for hosts that have no
 *      Rust toolchain, and the two GPU-only forms (fused precision form,
 *      batched trajectories);
 *   3. the sparse form: SparseVector<C64> (src/state/sparse.rs) with its
 *      entries in device memory;
 *   4. the Pauli-frame sampler (FrameSampler, src/frame.rs) for noisy
 *      Clifford circuits of up to 2^24 qubits.
 * The seeded synthetic workloads of the benchmark and the tests are not part
 * of this interface: they live in libncsim_workloads.so (ncsim_workloads.h).
 *
 * Conventions (src/state/vector.rs:14, src/pauli/ops.rs:5):
 *   - qubit q is bit q of a basis index; a k-qubit gate matrix is row-major,
 *     2^k x 2^k, over the local index whose bit j is qubits[j];
 *   - complex numbers are interleaved (re, im) doubles;
 *   - a Pauli is i^phase * X^x * Z^z with x, z bit masks over the register
 *     (so Y_q has x = z = 1<<q and phase 1).
 *
 * Every function returns an ncsim_status; NCSIM_OK is 0.  On error,
 * ncsim_last_error() returns a thread-local message.  No function aborts or
 * throws across the ABI.  Handles may be used from several threads: each
 * state serialises its own calls (the trait requires Send + Sync; read-only
 * calls such as expectation are issued from rayon threads by
 * src/state/mod.rs:93-101 and src/bridge.rs:456-464).
 */
#ifndef NCSIM_CUDA_H
#define NCSIM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes mirror SimError (src/error.rs:7-42) plus device errors. */
typedef int32_t ncsim_status;
#define NCSIM_OK 0
#define NCSIM_ERR_UNSUPPORTED 1         /* SimError::Unsupported */
#define NCSIM_ERR_QUBIT_OUT_OF_RANGE 2  /* SimError::QubitOutOfRange */
#define NCSIM_ERR_ARITY 3               /* SimError::Arity */
#define NCSIM_ERR_DUPLICATE_QUBIT 4     /* SimError::DuplicateQubit */
#define NCSIM_ERR_NOT_REPRESENTABLE 5   /* SimError::NotRepresentable */
#define NCSIM_ERR_ZERO_STATE 6          /* SimError::ZeroState */
#define NCSIM_ERR_PARSE 7               /* SimError::Parse */
#define NCSIM_ERR_INVALID 8             /* SimError::Invalid */
#define NCSIM_ERR_DEVICE 9              /* CUDA error (maps to SimError::Invalid on the Rust side) */
#define NCSIM_ERR_OUT_OF_MEMORY 10      /* device allocation failed */

/* Amplitude storage. */
#define NCSIM_C128 0 /* complex<double>: the drop-in for StateVector<C64> */
#define NCSIM_C64 1  /* complex<float>: storage of the fused precision form and the batched form */

typedef struct ncsim_state ncsim_state;
typedef struct ncsim_rng ncsim_rng;
typedef struct ncsim_circuit ncsim_circuit;
typedef struct ncsim_gate ncsim_gate;

/* Thread-local message of the last failed call on this thread. */
const char* ncsim_last_error(void);
/* The fields of the last error on this thread, for the SimError variants
 * that carry them (src/error.rs:17-33): QubitOutOfRange {qubit, num_qubits},
 * DuplicateQubit(qubit), Arity {gate, expected, got}.  Fields a variant does
 * not carry are zero (gate: empty). */
typedef struct ncsim_error_info {
  ncsim_status code;
  uint64_t qubit;
  uint64_t num_qubits;
  uint64_t expected;
  uint64_t got;
  char gate[64]; /* the gate's text name, zero-terminated */
} ncsim_error_info;
ncsim_status ncsim_last_error_info(ncsim_error_info* out);
/* ABI version (major * 10000 + minor * 100 + patch). */
int32_t ncsim_abi_version(void);
/* Streaming multiprocessors, free and total device memory of the current device. */
ncsim_status ncsim_device_info(int32_t* sm_count, uint64_t* free_bytes, uint64_t* total_bytes);
/* Temporaries (readouts, staging, the sparse form's sort buffers) come from a
 * stream-ordered pool that the library creates per device and that keeps
 * freed memory for the next call; the device's default pool is not touched.
 * This gives the kept memory of every such pool back to the device (call it
 * when no library work is queued). */
ncsim_status ncsim_trim_memory(void);
/* Bytes the current device's library pool holds from the device, and bytes of
 * it in use by queued or running library calls. */
ncsim_status ncsim_pool_info(uint64_t* reserved_bytes, uint64_t* used_bytes);

/* ======================================================================
 * 1. State operations (the QuantumState<C64> boundary)
 * ====================================================================== */

/* |0...0> on n qubits (StateVector::zero_state, vector.rs:25). n <= 33 for
 * C128 and n <= 34 for C64 (device memory bound; the reference caps at 30,
 * vector.rs:30).  Fails with NCSIM_ERR_OUT_OF_MEMORY when it does not fit. */
ncsim_status ncsim_sv_create(uint32_t n, int32_t precision, ncsim_state** out);
/* Frees the handle and its device memory (Drop). */
ncsim_status ncsim_sv_destroy(ncsim_state* s);
/* A device-to-device copy (Clone, vector.rs:15): needs a second state's memory. */
ncsim_status ncsim_sv_clone(const ncsim_state* s, ncsim_state** out);
/* Register size (QuantumState::num_qubits, mod.rs:46) and storage precision. */
ncsim_status ncsim_sv_num_qubits(const ncsim_state* s, uint32_t* n);
ncsim_status ncsim_sv_precision(const ncsim_state* s, int32_t* precision);
/* |x> (StateVector::basis_state, vector.rs:29-34). */
ncsim_status ncsim_sv_set_basis(ncsim_state* s, uint64_t index);
/* |+>^n with amplitude sqrt2_pow(-n) (StateVector::plus_state, vector.rs:36-42). */
ncsim_status ncsim_sv_set_plus(ncsim_state* s);
/* From 2^n interleaved complex128 host amplitudes (StateVector::from_amplitudes, vector.rs:44-52). */
ncsim_status ncsim_sv_set_amplitudes(ncsim_state* s, const double* amps, uint64_t len);
/* All 2^n amplitudes to host memory as complex128 (to_vector, vector.rs:542-544). */
ncsim_status ncsim_sv_get_amplitudes(const ncsim_state* s, double* amps, uint64_t len);
/* Amplitudes first .. first+count-1 as complex128 (a slice of to_vector, for
 * registers too large to copy to the host at once). */
ncsim_status ncsim_sv_get_amplitudes_range(const ncsim_state* s, uint64_t first, uint64_t count, double* amps);
/* One amplitude <x|psi> (QuantumState::amplitude, vector.rs:408-410). */
ncsim_status ncsim_sv_get_amplitude(const ncsim_state* s, uint64_t index, double* re_im);
/* count amplitudes at the given indices (amplitude called in a loop). */
ncsim_status ncsim_sv_gather_amplitudes(const ncsim_state* s, const uint64_t* indices, uint64_t count, double* out);

/* Dense 2^k x 2^k complex128 matrix on qubits (StateVector::apply_matrix,
 * vector.rs:67-93).  k <= 13 (gates on 6..13 qubits run as a complex GEMM
 * over gathered chunks of fibers, with the matrix in device memory for the
 * call).  Exact-zero entries contribute nothing (a zero product), as in the
 * reference's row-sparse product. */
ncsim_status ncsim_sv_apply_matrix(ncsim_state* s, const uint32_t* qubits, uint32_t k, const double* matrix);
/* Monomial gate given by its basis images (StateVector::apply_monomial,
 * vector.rs:96-139): U|x> = phase[x] |image[x]> over the local index x.
 * image must be a permutation of 0..2^k; phase is complex128.  Diagonal
 * tables (image[x] == x) touch only amplitudes whose phase is not exactly 1.
 * k <= 24 (tables on more than 10 qubits run through gathered chunks of
 * fibers, with the table in device memory for the call). */
ncsim_status ncsim_sv_apply_monomial(ncsim_state* s, const uint32_t* qubits, uint32_t k, const uint64_t* image,
                                     const double* phase);
/* Diagonal(PhasePoly) evaluated from each basis index (gate.rs:557 with
 * phasepoly.rs:670-678): amplitude x is multiplied by
 *   scalar * exp(2 pi i f(x) / 2^bits),  f(x) = constant + sum_t coeff[t] * prod_{l in t} parity(l . x)
 * over the local index x of `qubits`.  Term t owns parity masks
 * parities[term_start[t] .. term_start[t+1]) (masks over the k local
 * variables); term_start has nterms+1 entries.  1 <= bits <= 32, any k <= n.
 * The scalar is the exact phasor sqrt2^s2 * exp(2 pi i sphase / 2^sbits).
 * Amplitudes whose factor is exactly 1, and exact zeros, are not rewritten. */
ncsim_status ncsim_sv_apply_phasepoly(ncsim_state* s, const uint32_t* qubits, uint32_t k, uint32_t bits,
                                      uint64_t constant, uint32_t nterms, const uint32_t* term_start,
                                      const uint64_t* parities, const uint64_t* coeffs, int32_t scalar_s2,
                                      uint64_t scalar_phase, uint32_t scalar_bits);
/* psi <- P psi for P = i^phase X^x Z^z over the register (vector.rs:143-164). */
ncsim_status ncsim_sv_apply_pauli(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase);
/* <psi|psi> as complex (imaginary part 0) (vector.rs:397-406), FP64 reduction. */
ncsim_status ncsim_sv_norm_sq(const ncsim_state* s, double* re_im);
/* <psi|P|psi> (vector.rs:412-429), FP64 reduction. */
ncsim_status ncsim_sv_expectation(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, double* re_im);
/* <psi|P|psi> and <psi|psi> in one pass (what QuantumState::measure reads, mod.rs:119-120). */
ncsim_status ncsim_sv_measure_stats(const ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase,
                                    double* expectation_re_im, double* norm_sq);
/* <a|b> (vector.rs:431-443). Registers must have equal size. */
ncsim_status ncsim_sv_inner(const ncsim_state* a, const ncsim_state* b, double* re_im);
/* psi <- (1 + (-1)^outcome P)/2 psi for Hermitian P; writes the branch weight
 * <psi|psi> after projection (vector.rs:445-479), projection and norm fused
 * in one pass. */
ncsim_status ncsim_sv_project(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, int32_t outcome,
                              double* weight_re_im);
/* psi <- c psi (vector.rs:481-488). */
ncsim_status ncsim_sv_scale(ncsim_state* s, double re, double im);
/* Born sampling in one pass (StateVector::sample, vector.rs:494-540): the
 * caller draws the shots' uniforms u[k] in [0,1) (rng.gen::<f64>(), in shot
 * order); shot k is the basis index whose cumulative weight interval holds
 * u[k] * total.  Zero-weight indices are never returned.  Fails with
 * NCSIM_ERR_ZERO_STATE when the state vanished. */
ncsim_status ncsim_sv_sample(const ncsim_state* s, const double* uniforms, uint64_t shots, uint64_t* out);
/* psi (x) phi with psi on the low qubits (StateVector::kron, vector.rs:168-188). */
ncsim_status ncsim_sv_kron(const ncsim_state* a, const ncsim_state* b, ncsim_state** out);
/* Waits for the state's queued device work. */
ncsim_status ncsim_sv_synchronize(const ncsim_state* s);
/* The device address and size in bytes of the state's amplitude array (for
 * zero-copy views by a communication layer: the sharded register exchanges
 * halves of it between devices).  Work queued on the state must be finished
 * (ncsim_sv_synchronize) before another stream touches the array. */
ncsim_status ncsim_sv_device_pointer(const ncsim_state* s, void** ptr, uint64_t* bytes);
/* Sum |a|^2 over each block of `block` consecutive amplitudes (a power of
 * two), FP64, into nblocks = 2^n / block host doubles: the first step of
 * StateVector::sample (vector.rs:494-501), for a sampler that spans several
 * registers. */
ncsim_status ncsim_sv_block_weights(const ncsim_state* s, uint64_t block, double* out, uint64_t nblocks);
/* The last step of StateVector::sample (vector.rs:508-538) for given shots:
 * shot k walks block blocks[k] from the running sum accs[k] (the weight of
 * everything before that block) to the first index whose running sum exceeds
 * targets[k]; zero-weight indices are never returned. */
ncsim_status ncsim_sv_sample_walk(const ncsim_state* s, uint64_t block, const double* targets, const uint64_t* blocks,
                                  const double* accs, uint64_t shots, uint64_t* out);
/* Device time on the state's stream: start records an event; stop records a
 * second one, waits for it and writes the milliseconds between them. */
ncsim_status ncsim_sv_timer_start(ncsim_state* s);
ncsim_status ncsim_sv_timer_stop(ncsim_state* s, double* milliseconds);
/* One FP64 pass over two registers of equal size and any precisions:
 * <a|b>, <a|a>, <b|b> and max_i |a_i - b_i|, for infidelity
 * 1 - |<a|b>|^2 / (<a|a><b|b>) and the largest amplitude error. */
ncsim_status ncsim_sv_compare(const ncsim_state* a, const ncsim_state* b, double* inner_re_im, double* norm_a,
                              double* norm_b, double* max_abs_diff);

/* Launch profiler: while enabled, every kernel launched for the state is
 * bracketed by CUDA events on the state's stream.  Reading waits for the
 * stream and returns, per kernel class, the launch count, the summed device
 * time and the summed algorithmic bytes (read + written amplitudes in the
 * 32-byte sectors an operation changes).  Enabling clears earlier records. */
typedef struct ncsim_kernel_stat {
  char name[32];
  uint64_t launches;
  double milliseconds;
  double bytes;
} ncsim_kernel_stat;
/* Runs of 16 or more consecutive gates in ncsim_sv_run go through tiled passes
 * (on by default): a pass applies a run's gates to 4096-amplitude tiles in
 * shared memory, one HBM read and write for many gates, each gate with the
 * arithmetic of its own kernel (the amplitudes equal the gate-by-gate ones). */
ncsim_status ncsim_sv_set_tile_passes(ncsim_state* s, int32_t enable);
ncsim_status ncsim_sv_profile_enable(ncsim_state* s, int32_t enable);
ncsim_status ncsim_sv_profile_read(ncsim_state* s, ncsim_kernel_stat* out, uint32_t cap, uint32_t* count);

/* <psi|P|psi> and <psi|psi> of 2^n amplitudes that the caller already holds
 * in its own device memory (interleaved complex128 or complex64, per
 * `precision`), computed on the caller's stream (`stream` is a cudaStream_t;
 * NULL is the default stream), with no device or host allocation.
 * This entry point has no counterpart in the reference: it serves callers
 * that cannot let a library call cudaMalloc, because their amplitudes live in
 * memory they manage themselves (a framework's pool, a fixed device budget)
 * where an allocation or free could synchronize the device, fragment the pool
 * or exceed the budget.  The reduction scratch is a file-scope device array of
 * 1024 block partials (32 KB); registers of up to 34 qubits are accepted and
 * larger ones are rejected with NCSIM_ERR_INVALID.  `amps` must be device
 * (or managed) memory of the current device holding all 2^n amplitudes inside
 * one allocation, and a non-NULL `stream` must belong to the current device:
 * a host pointer, a shorter buffer or another device's stream is rejected
 * with NCSIM_ERR_INVALID before anything is launched.  The first call on a
 * device resolves the array's device address (set-up), so make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race and must be serialized by the caller. */
ncsim_status ncsim_measure_stats_noalloc(const void* amps, uint32_t n, int32_t precision, uint64_t x, uint64_t z,
                                         uint32_t phase, void* stream, double* expectation_re_im, double* norm_sq);

/* ======================================================================
 * 2. Host mirror of the reference interface (C++), and the GPU-only forms
 * ====================================================================== */

/* rand 0.8 StdRng (ChaCha12) seeded as StdRng::seed_from_u64. */
ncsim_status ncsim_rng_new(uint64_t seed, ncsim_rng** out);
ncsim_status ncsim_rng_free(ncsim_rng* r);
ncsim_status ncsim_rng_next_u64(ncsim_rng* r, uint64_t* out);
ncsim_status ncsim_rng_next_u32(ncsim_rng* r, uint32_t* out);
ncsim_status ncsim_rng_gen_f64(ncsim_rng* r, double* out);
ncsim_status ncsim_rng_gen_range(ncsim_rng* r, uint64_t lo, uint64_t hi, uint64_t* out);

/* Circuit::parse (src/circuit.rs:459-565), plus DIAG(...) / MONOMIAL(...)
 * lines for the reference's Diagonal and Monomial gates. */
ncsim_status ncsim_circuit_parse(const char* text, ncsim_circuit** out);
ncsim_status ncsim_circuit_free(ncsim_circuit* c);
ncsim_status ncsim_circuit_info(const ncsim_circuit* c, uint32_t* num_qubits, uint64_t* num_ops, uint64_t* num_gates,
                                uint64_t* num_measurements);
/* The circuit in text form (circuit.rs:693-728); *len receives the length
 * without the terminating zero, written only when cap > len. */
ncsim_status ncsim_circuit_to_text(const ncsim_circuit* c, char* buf, size_t cap, size_t* len);

/* A gate from one text token ("H", "RZ(0.5)", "PHASE(3,4)", "DIAG(...)",
 * "MONOMIAL(...)") and its arity. */
ncsim_status ncsim_gate_parse(const char* token, uint32_t arity_hint, ncsim_gate** out, uint32_t* arity);
/* Gate::Unitary (gate.rs:427-428): a dense complex128 matrix on k <= 13 qubits. */
ncsim_status ncsim_gate_unitary(uint32_t k, const double* matrix, ncsim_gate** out);
/* Gate::Pauli (gate.rs:417-418): i^phase X^x Z^z on k local qubits. */
ncsim_status ncsim_gate_pauli(uint32_t k, uint64_t x, uint64_t z, uint32_t phase, ncsim_gate** out);
ncsim_status ncsim_gate_free(ncsim_gate* g);
/* The dense 2^k x 2^k complex128 matrix that the engine's lowering of the
 * gate applies on qubits 0..k-1 (host only, k <= 8): the dense view, the
 * permutation table, the phase polynomial or the Pauli, as launched.  For
 * checking the lowering against Gate::matrix (gate.rs:670-747). */
ncsim_status ncsim_gate_lowered_matrix(const ncsim_gate* g, double* out, size_t cap_doubles, uint32_t* k);

/* Pauli::from_string(n, text) (pauli/mod.rs:349-414) as (x, z, phase). */
ncsim_status ncsim_pauli_parse(const char* text, uint32_t n, uint64_t* x, uint64_t* z, uint32_t* phase);
/* The same on registers of any width: x and z as `words` 64-bit words each
 * (qubit q: bit q % 64 of word q / 64), words * 64 >= n. */
ncsim_status ncsim_pauli_parse_words(const char* text, uint32_t n, uint64_t* x, uint64_t* z, uint32_t words,
                                     uint32_t* phase);

/* QuantumState::apply_gate through the gate's views (vector.rs:364-395). */
ncsim_status ncsim_sv_apply_gate(ncsim_state* s, const ncsim_gate* g, const uint32_t* qubits, uint32_t k);
/* QuantumState::measure (mod.rs:113-131): one pass for <P> and <psi|psi>, a
 * draw only when the outcome is uncertain, then the fused projection. */
ncsim_status ncsim_sv_measure(ncsim_state* s, uint64_t x, uint64_t z, uint32_t phase, ncsim_rng* rng,
                              int32_t* outcome);
/* QuantumState::run (mod.rs:168-183): the record (one byte per measurement,
 * 1 = eigenvalue -1) is written to rec (cap bytes); *len receives its length. */
ncsim_status ncsim_sv_run(ncsim_state* s, const ncsim_circuit* c, ncsim_rng* rng, uint8_t* rec, size_t cap,
                          size_t* len);
/* StateVector::sample with draws from rng (vector.rs:494-540). */
ncsim_status ncsim_sv_sample_rng(const ncsim_state* s, ncsim_rng* rng, uint64_t shots, uint64_t* out);
/* QuantumState::normalize (mod.rs:220-233) and probability (mod.rs:104-108). */
ncsim_status ncsim_sv_normalize(ncsim_state* s);
ncsim_status ncsim_sv_probability(const ncsim_state* s, uint64_t index, double* out);
/* QuantumState::expectation_sum (mod.rs:93-101): sum_k c_k <P_k>, summed pairwise. */
ncsim_status ncsim_sv_expectation_sum(const ncsim_state* s, uint64_t count, const uint64_t* x, const uint64_t* z,
                                      const uint32_t* phase, const double* coeffs, double* re_im);

/* ---- precision form: fused k<=5 unitaries on tensor cores (C64 states) ----
 * Runs of gates are fused on the host (FP64) into unitaries of at most
 * max_fuse qubits, grouped into passes over a qubit window held in shared
 * memory, and applied as BF16x3 split-precision complex GEMMs (tcgen05, FP32
 * accumulation) to FP32 amplitudes.  Measurements, resets and noise go
 * through the plain kernels with FP64 reductions.  Same record semantics as
 * ncsim_sv_run. */
typedef struct ncsim_fused_stats {
  uint64_t source_gates;     /* Op::Gate count of the circuit */
  uint64_t fused_unitaries;  /* unitaries after fusion */
  uint64_t passes;           /* HBM read+write passes over the state */
  uint64_t remap_passes;     /* of which qubit-permutation passes */
  uint64_t gemm_launches;    /* tensor-core pass kernel launches */
  uint64_t diagonal_terms;   /* elementwise phase terms left after folding diagonals into unitaries */
} ncsim_fused_stats;
ncsim_status ncsim_sv_run_fused(ncsim_state* s, const ncsim_circuit* c, ncsim_rng* rng, uint32_t max_fuse,
                                uint8_t* rec, size_t cap, size_t* len, ncsim_fused_stats* stats);
/* Host-only check of the fusion planner: applies the fused form's plan of a
 * gates-only circuit (n <= 22) to complex128 host amplitudes in FP64, in the
 * pass, tile and op order the device uses.  With amps NULL it only plans
 * (any n) and fills the statistics. */
ncsim_status ncsim_fused_emulate(const ncsim_circuit* c, uint32_t max_fuse, double* amps, uint64_t len,
                                 ncsim_fused_stats* stats);

/* ---- batching form: many independent noisy trajectories ----
 * Each trajectory is QuantumState::run (src/state/mod.rs:168-183) of a circuit
 * on a register of 13..26 qubits that starts at |0...0>, with its own StdRng:
 * one-qubit gates, two-qubit controlled phases (CZ, CS, CS_DAG, CPHASE), Pauli
 * noise channels (one draw per application, src/circuit.rs:136-146) and a
 * trailing block M 0, M 1, ..., M m-1 (a draw only when the outcome is
 * uncertain, src/state/mod.rs:113-131).  All trajectories run in one
 * persistent kernel (complex64 amplitudes, FP64 reductions) replayed through a
 * CUDA graph, with a launch configuration picked by timing (autotuner).
 * Results per trajectory: the record (bit k = outcome of M k), <Z0>/<psi|psi>
 * just before the measurements, and <psi|psi> there. */
typedef struct ncsim_batch ncsim_batch;
typedef struct ncsim_batch_stats {
  uint64_t trajectories;
  uint64_t source_gates;   /* Op::Gate count over all circuits */
  uint64_t noise_events;   /* sampled Pauli errors */
  uint64_t folded_ops;     /* device ops after folding one-qubit runs */
  uint64_t passes;         /* passes over trajectory states */
  uint64_t tile_passes;    /* 8192-amplitude tiles streamed, over all passes */
  uint64_t tile_stages;    /* register stages applied to tiles */
  double state_bytes;      /* algorithmic HBM bytes of one run */
  uint64_t program_bytes;  /* device program size */
  uint32_t max_qubits;
} ncsim_batch_stats;
enum { NCSIM_BATCH_ORDER_LARGEST_FIRST = 0, NCSIM_BATCH_ORDER_GIVEN = 1 };
typedef struct ncsim_batch_config {
  uint32_t ctas_per_sm; /* 1, or 2 when single-buffered */
  uint32_t buffers;     /* 2: tile prefetch, FP64 sums in shared memory; 1: no prefetch */
  uint32_t order;       /* NCSIM_BATCH_ORDER_* */
} ncsim_batch_config;
/* Trajectory t: circuits[t] run with StdRng::seed_from_u64(seeds[t]). */
ncsim_status ncsim_batch_from_circuits(uint32_t count, const ncsim_circuit* const* circuits, const uint64_t* seeds,
                                       ncsim_batch** out);
ncsim_status ncsim_batch_free(ncsim_batch* b);
/* Gives back the batch's device and pinned memory, its stream and its graph
 * (results of earlier runs are dropped); the batch keeps its program, and the
 * next run sets everything up again on the device current at that time (so a
 * batch can move between devices).  The caller's current device is kept. */
ncsim_status ncsim_batch_release(ncsim_batch* b);
ncsim_status ncsim_batch_info(const ncsim_batch* b, ncsim_batch_stats* st);
ncsim_status ncsim_batch_trajectory_qubits(const ncsim_batch* b, uint32_t* n);
/* The host planner's knobs for registers of n qubits, chosen per size class by
 * the autotuner: candidate windows (qubits 0..3 and 9 consecutive qubits every
 * window_step qubits), the window and stage choice rules, and the device
 * milliseconds each candidate knob set took on that class (0 when not timed).
 * The choice is made on first use, or read from a cache file keyed by device,
 * register size and program size (NCSIM_TUNE_CACHE, else
 * $XDG_CACHE_HOME or ~/.cache /ncsim_b200/batch_knobs.txt). */
typedef struct ncsim_batch_knobs_info {
  uint32_t knob_set;
  uint32_t window_step;
  uint32_t greedy_windows;
  uint32_t greedy_stages;
  uint32_t final_;  /* 1: the program is compiled with these knobs */
  double timed_ms[4];
} ncsim_batch_knobs_info;
ncsim_status ncsim_batch_knobs(const ncsim_batch* b, uint32_t n, ncsim_batch_knobs_info* out);
/* Compiles registers of n qubits with candidate knob set `knob_set` (0..3)
 * instead of the tuned one, while the batch still holds its trajectories;
 * final_ != 0 makes the knobs final (no tuning on first use, trajectories
 * dropped). */
ncsim_status ncsim_batch_set_knob_set(ncsim_batch* b, uint32_t n, uint32_t knob_set, int32_t final_);
ncsim_status ncsim_batch_set_config(ncsim_batch* b, const ncsim_batch_config* cfg);
/* The configuration the next run uses (tuned on the current device if unset). */
ncsim_status ncsim_batch_get_config(ncsim_batch* b, ncsim_batch_config* cfg);
/* Times each candidate launch configuration on an evenly strided sample of
 * the batch (0 = the whole batch) and keeps the fastest; runs on first use
 * when no configuration was set, once per (device, count, largest register).
 * While the batch still holds its trajectories (before its first run, when
 * the knob cache lacked a size class), the planner's knobs are timed again
 * per size class first. */
ncsim_status ncsim_batch_tune(ncsim_batch* b, uint32_t sample, ncsim_batch_config* best);
/* Runs every trajectory on the current device (one CUDA graph launch: counter
 * reset, the kernel, result copies to pinned host memory); device_ms
 * (optional) is the graph's time between CUDA events on its stream. */
ncsim_status ncsim_batch_run(ncsim_batch* b, double* device_ms);
/* Per trajectory (arrays of the batch's count; NULL skips): n, record, <Z0>/norm, norm. */
ncsim_status ncsim_batch_results(ncsim_batch* b, uint32_t* n, uint64_t* records, double* z0, double* norm);
/* Host-only check: trajectory t's device program run in FP64 on the host in
 * the device's pass, tile, stage and op order (n <= 22). */
ncsim_status ncsim_batch_emulate(const ncsim_batch* b, uint32_t t, uint64_t* record, double* z0, double* norm);

/* ---- sparse form: SparseVector<C64> (src/state/sparse.rs) on the device ----
 * The nonzero amplitudes of a register of 1..1024 qubits as (basis index,
 * complex128) entries in device memory (at most 2^31 entries).  A basis index
 * is W = ncsim_sparse_num_words() 64-bit words (1 up to 64 qubits, 4 up to
 * 256, 16 up to 1024), qubit q being bit q % 64 of word q / 64, the layout of
 * ncsim's Bits (bits.rs:1-17); every key array below holds W words per entry,
 * and keys order lexicographically from word 0, as Vec<u64> does.  The
 * functions taking one uint64_t mask or index address qubits 0..63 of any
 * register; the _words variants take W words.  Operations
 * that move each entry to one entry (monomial gates, permutations with
 * phases, Paulis, diagonals) keep the entry order and leave it unsorted when
 * a key changed; operations that create entries (dense gates, projections)
 * normalise: entries sorted by index, duplicates summed, exact zeros and
 * amplitudes under the cutoff dropped (sparse.rs:114-128). */
typedef struct ncsim_sparse ncsim_sparse;
/* SparseVector::zero_state (sparse.rs:50-52). */
ncsim_status ncsim_sparse_create(uint32_t n, ncsim_sparse** out);
/* SparseVector::from_entries (sparse.rs:54-72): amps are (re, im) pairs; duplicates add. */
ncsim_status ncsim_sparse_from_entries(uint32_t n, const uint64_t* keys, const double* amps, uint64_t count,
                                       ncsim_sparse** out);
ncsim_status ncsim_sparse_destroy(ncsim_sparse* s);
/* Clone (sparse.rs:27, #[derive(Clone)]). */
ncsim_status ncsim_sparse_clone(const ncsim_sparse* s, ncsim_sparse** out);
/* SparseVector::with_cutoff (sparse.rs:74-78): drop |a| < cutoff after each normalisation. */
ncsim_status ncsim_sparse_set_cutoff(ncsim_sparse* s, double cutoff);
ncsim_status ncsim_sparse_num_qubits(const ncsim_sparse* s, uint32_t* n);
/* SparseVector::num_entries (sparse.rs:84-86). */
ncsim_status ncsim_sparse_num_entries(const ncsim_sparse* s, uint64_t* count);
/* SparseVector::entries (sparse.rs:88-90), in the current entry order; cap >= num_entries. */
ncsim_status ncsim_sparse_get_entries(const ncsim_sparse* s, uint64_t* keys, double* amps, uint64_t cap);
/* SparseVector::sort (sparse.rs:92-97). */
ncsim_status ncsim_sparse_sort(ncsim_sparse* s);
/* QuantumState::apply_gate for SparseVector (sparse.rs:266-297): Pauli, monomial, matrix views. */
ncsim_status ncsim_sparse_apply_gate(ncsim_sparse* s, const ncsim_gate* g, const uint32_t* qubits, uint32_t k);
/* SparseVector::apply_pauli (sparse.rs:216-231): psi <- i^phase X^x Z^z psi. */
ncsim_status ncsim_sparse_apply_pauli(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase);
/* norm_sq (sparse.rs:299-302), FP64 reduction. */
ncsim_status ncsim_sparse_norm_sq(const ncsim_sparse* s, double* re_im);
/* amplitude (sparse.rs:304-314): 0 for an index without an entry. */
ncsim_status ncsim_sparse_amplitude(const ncsim_sparse* s, uint64_t index, double* re_im);
/* expectation (sparse.rs:316-336) over the sorted view. */
ncsim_status ncsim_sparse_expectation(const ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, double* re_im);
/* inner (sparse.rs:338-349): <a|b>. */
ncsim_status ncsim_sparse_inner(const ncsim_sparse* a, const ncsim_sparse* b, double* re_im);
/* project (sparse.rs:351-380): psi <- (1 + (-1)^outcome P)/2 psi for Hermitian P; the weight after it. */
ncsim_status ncsim_sparse_project(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, int32_t outcome,
                                  double* weight_re_im);
/* scale (sparse.rs:382-386). */
ncsim_status ncsim_sparse_scale(ncsim_sparse* s, double re, double im);
/* tensor (sparse.rs:388-405): a on the low qubits, b above them (n_a + n_b <= 1024). */
ncsim_status ncsim_sparse_tensor(const ncsim_sparse* a, const ncsim_sparse* b, ncsim_sparse** out);
/* sample (sparse.rs:407-424): cumulative weights in entry order, one rng.gen::<f64>() per shot;
 * out holds W words per shot. */
ncsim_status ncsim_sparse_sample(const ncsim_sparse* s, ncsim_rng* rng, uint64_t shots, uint64_t* out);
/* to_vector (sparse.rs:426-434), n <= 26. */
ncsim_status ncsim_sparse_to_vector(const ncsim_sparse* s, double* amps, uint64_t len);
/* QuantumState::measure (mod.rs:113-131) and run (mod.rs:168-183) on the sparse state. */
ncsim_status ncsim_sparse_measure(ncsim_sparse* s, uint64_t x, uint64_t z, uint32_t phase, ncsim_rng* rng,
                                  int32_t* outcome);
ncsim_status ncsim_sparse_run(ncsim_sparse* s, const ncsim_circuit* c, ncsim_rng* rng, uint8_t* rec, size_t cap,
                              size_t* len);
/* Words per basis key: Bits' nwords(n) rounded up to 1, 4 or 16 (bits.rs:14-17). */
ncsim_status ncsim_sparse_num_words(const ncsim_sparse* s, uint32_t* words);
/* apply_pauli, amplitude, expectation, project and measure with W-word masks
 * and indices (words must equal ncsim_sparse_num_words; sparse.rs:216-380,
 * mod.rs:113-131). */
ncsim_status ncsim_sparse_apply_pauli_words(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t words,
                                            uint32_t phase);
ncsim_status ncsim_sparse_amplitude_words(const ncsim_sparse* s, const uint64_t* index, uint32_t words,
                                          double* re_im);
ncsim_status ncsim_sparse_expectation_words(const ncsim_sparse* s, const uint64_t* x, const uint64_t* z,
                                            uint32_t words, uint32_t phase, double* re_im);
ncsim_status ncsim_sparse_project_words(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t words,
                                        uint32_t phase, int32_t outcome, double* weight_re_im);
ncsim_status ncsim_sparse_measure_words(ncsim_sparse* s, const uint64_t* x, const uint64_t* z, uint32_t words,
                                        uint32_t phase, ncsim_rng* rng, int32_t* outcome);
/* Waits for the state's queued device work; device-time events on its stream. */
ncsim_status ncsim_sparse_synchronize(const ncsim_sparse* s);
ncsim_status ncsim_sparse_timer_start(ncsim_sparse* s);
ncsim_status ncsim_sparse_timer_stop(ncsim_sparse* s, double* milliseconds);

/* ---- Pauli-frame sampler: FrameSampler (src/frame.rs:34-300) on the device ----
 * Circuits of any width up to 2^24 qubits; every gate Clifford.  Shots run in
 * batches of 16384 (frame.rs:31), each with its own StdRng seeded by one u64
 * drawn from the caller's generator per batch, in order (frame.rs:72-74).
 * Packed outputs: measurement (detector, observable) k's bits over the shots
 * are nwords = ceil(shots / 64) words at out[k * nwords] (bit s of word
 * s / 64 = shot s).  The sampler keeps its device buffers on the device that
 * is current at its first sample call. */
typedef struct ncsim_frames ncsim_frames;
/* FrameSampler::new (frame.rs:41-60): NCSIM_ERR_UNSUPPORTED for a non-Clifford
 * gate; the reference record of the noiseless circuit, random outcomes drawn
 * from StdRng::seed_from_u64(reference_seed) as the stabilizer tableau draws
 * them (stabilizer.rs:591). */
ncsim_status ncsim_frames_new(const ncsim_circuit* c, uint64_t reference_seed, ncsim_frames** out);
/* The same with a reference record given by the caller (m = the circuit's
 * measurements, one byte 0/1 each), e.g. ncsim's own FrameSampler::reference(). */
ncsim_status ncsim_frames_with_reference(const ncsim_circuit* c, const uint8_t* reference, uint64_t m,
                                         ncsim_frames** out);
ncsim_status ncsim_frames_free(ncsim_frames* f);
/* num_measurements, detectors() and observables() counts (circuit.rs:297-327),
 * and the dependency layers of the device program. */
ncsim_status ncsim_frames_info(const ncsim_frames* f, uint32_t* num_qubits, uint64_t* num_measurements,
                               uint64_t* num_detectors, uint64_t* num_observables, uint64_t* num_layers);
/* FrameSampler::reference (frame.rs:66-68): cap >= num_measurements bytes. */
ncsim_status ncsim_frames_reference(const ncsim_frames* f, uint8_t* out, uint64_t cap);
/* sample_packed (frame.rs:69-89) into host memory: cap >= num_measurements * nwords. */
ncsim_status ncsim_frames_sample_packed(ncsim_frames* f, uint64_t shots, ncsim_rng* rng, uint64_t* out, uint64_t cap);
/* The same with the batch seeds given (nseeds = ceil(shots / 16384)): what a
 * caller with its own generator passes after drawing one u64 per batch. */
ncsim_status ncsim_frames_sample_packed_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds,
                                              uint64_t* out, uint64_t cap);
/* The same into device memory on the sampler's device (d_out: cap words). */
ncsim_status ncsim_frames_sample_packed_device(ncsim_frames* f, uint64_t shots, const uint64_t* seeds, uint64_t nseeds,
                                               uint64_t* d_out, uint64_t cap);
/* sample (frame.rs:90-102): shot s's record is ceil(m / 64) words at
 * out[s * ceil(m / 64)], bit k = measurement k; cap >= shots * ceil(m / 64). */
ncsim_status ncsim_frames_sample(ncsim_frames* f, uint64_t shots, ncsim_rng* rng, uint64_t* out, uint64_t cap);
/* sample_detectors (frame.rs:155-205): detector and observable flips, packed. */
ncsim_status ncsim_frames_sample_detectors(ncsim_frames* f, uint64_t shots, ncsim_rng* rng, uint64_t* det,
                                           uint64_t det_cap, uint64_t* obs, uint64_t obs_cap);
/* The same with the batch seeds given. */
ncsim_status ncsim_frames_sample_detectors_seeds(ncsim_frames* f, uint64_t shots, const uint64_t* seeds,
                                                 uint64_t nseeds, uint64_t* det, uint64_t det_cap, uint64_t* obs,
                                                 uint64_t obs_cap);
/* Device time of the last call's mask and frame kernels (CUDA events on its stream). */
ncsim_status ncsim_frames_last_kernel_ms(const ncsim_frames* f, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* NCSIM_CUDA_H */
