//! Raw bindings of `include/ncsim_cuda.h` (libncsim_cuda.so), one to one:
//! every function, constant and struct of the header, with the same names.
//! Safe wrappers live in `lib.rs`.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_void};

/// Status of every call: 0 is success; the others mirror `SimError`
/// (src/error.rs:7-42) plus device errors.
pub type ncsim_status = i32;
pub const NCSIM_OK: ncsim_status = 0;
pub const NCSIM_ERR_UNSUPPORTED: ncsim_status = 1;
pub const NCSIM_ERR_QUBIT_OUT_OF_RANGE: ncsim_status = 2;
pub const NCSIM_ERR_ARITY: ncsim_status = 3;
pub const NCSIM_ERR_DUPLICATE_QUBIT: ncsim_status = 4;
pub const NCSIM_ERR_NOT_REPRESENTABLE: ncsim_status = 5;
pub const NCSIM_ERR_ZERO_STATE: ncsim_status = 6;
pub const NCSIM_ERR_PARSE: ncsim_status = 7;
pub const NCSIM_ERR_INVALID: ncsim_status = 8;
pub const NCSIM_ERR_DEVICE: ncsim_status = 9;
pub const NCSIM_ERR_OUT_OF_MEMORY: ncsim_status = 10;

/// Amplitude storage.
pub const NCSIM_C128: i32 = 0;
pub const NCSIM_C64: i32 = 1;

pub const NCSIM_BATCH_ORDER_LARGEST_FIRST: u32 = 0;
pub const NCSIM_BATCH_ORDER_GIVEN: u32 = 1;

macro_rules! opaque {
    ($($name:ident),*) => {$(
        #[repr(C)]
        pub struct $name {
            _private: [u8; 0],
        }
    )*};
}
opaque!(ncsim_state, ncsim_rng, ncsim_circuit, ncsim_gate, ncsim_batch, ncsim_sparse, ncsim_frames);

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ncsim_error_info {
    pub code: ncsim_status,
    pub qubit: u64,
    pub num_qubits: u64,
    pub expected: u64,
    pub got: u64,
    pub gate: [c_char; 64],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ncsim_kernel_stat {
    pub name: [c_char; 32],
    pub launches: u64,
    pub milliseconds: f64,
    pub bytes: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ncsim_fused_stats {
    pub source_gates: u64,
    pub fused_unitaries: u64,
    pub passes: u64,
    pub remap_passes: u64,
    pub gemm_launches: u64,
    pub diagonal_terms: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ncsim_batch_stats {
    pub trajectories: u64,
    pub source_gates: u64,
    pub noise_events: u64,
    pub folded_ops: u64,
    pub passes: u64,
    pub tile_passes: u64,
    pub tile_stages: u64,
    pub state_bytes: f64,
    pub program_bytes: u64,
    pub max_qubits: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ncsim_batch_config {
    pub ctas_per_sm: u32,
    pub buffers: u32,
    pub order: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ncsim_batch_knobs_info {
    pub knob_set: u32,
    pub window_step: u32,
    pub greedy_windows: u32,
    pub greedy_stages: u32,
    pub final_: u32,
    pub timed_ms: [f64; 4],
}

#[link(name = "ncsim_cuda")]
extern "C" {
    pub fn ncsim_last_error() -> *const c_char;
    pub fn ncsim_last_error_info(out: *mut ncsim_error_info) -> ncsim_status;
    pub fn ncsim_abi_version() -> i32;
    pub fn ncsim_device_info(sm_count: *mut i32, free_bytes: *mut u64, total_bytes: *mut u64) -> ncsim_status;
    pub fn ncsim_trim_memory() -> ncsim_status;
    pub fn ncsim_pool_info(reserved_bytes: *mut u64, used_bytes: *mut u64) -> ncsim_status;
    pub fn ncsim_sv_create(n: u32, precision: i32, out: *mut *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_destroy(s: *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_clone(s: *const ncsim_state, out: *mut *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_num_qubits(s: *const ncsim_state, n: *mut u32) -> ncsim_status;
    pub fn ncsim_sv_precision(s: *const ncsim_state, precision: *mut i32) -> ncsim_status;
    pub fn ncsim_sv_set_basis(s: *mut ncsim_state, index: u64) -> ncsim_status;
    pub fn ncsim_sv_set_plus(s: *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_set_amplitudes(s: *mut ncsim_state, amps: *const f64, len: u64) -> ncsim_status;
    pub fn ncsim_sv_get_amplitudes(s: *const ncsim_state, amps: *mut f64, len: u64) -> ncsim_status;
    pub fn ncsim_sv_get_amplitudes_range(s: *const ncsim_state, first: u64, count: u64, amps: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_get_amplitude(s: *const ncsim_state, index: u64, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_gather_amplitudes(s: *const ncsim_state, indices: *const u64, count: u64, out: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_apply_matrix(s: *mut ncsim_state, qubits: *const u32, k: u32, matrix: *const f64) -> ncsim_status;
    pub fn ncsim_sv_apply_monomial(s: *mut ncsim_state, qubits: *const u32, k: u32, image: *const u64, phase: *const f64) -> ncsim_status;
    pub fn ncsim_sv_apply_phasepoly(s: *mut ncsim_state, qubits: *const u32, k: u32, bits: u32, constant: u64, nterms: u32, term_start: *const u32, parities: *const u64, coeffs: *const u64, scalar_s2: i32, scalar_phase: u64, scalar_bits: u32) -> ncsim_status;
    pub fn ncsim_sv_apply_pauli(s: *mut ncsim_state, x: u64, z: u64, phase: u32) -> ncsim_status;
    pub fn ncsim_sv_norm_sq(s: *const ncsim_state, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_expectation(s: *const ncsim_state, x: u64, z: u64, phase: u32, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_measure_stats(s: *const ncsim_state, x: u64, z: u64, phase: u32, expectation_re_im: *mut f64, norm_sq: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_inner(a: *const ncsim_state, b: *const ncsim_state, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_project(s: *mut ncsim_state, x: u64, z: u64, phase: u32, outcome: i32, weight_re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_scale(s: *mut ncsim_state, re: f64, im: f64) -> ncsim_status;
    pub fn ncsim_sv_sample(s: *const ncsim_state, uniforms: *const f64, shots: u64, out: *mut u64) -> ncsim_status;
    pub fn ncsim_sv_kron(a: *const ncsim_state, b: *const ncsim_state, out: *mut *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_synchronize(s: *const ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_device_pointer(s: *const ncsim_state, ptr: *mut *mut c_void, bytes: *mut u64) -> ncsim_status;
    pub fn ncsim_sv_block_weights(s: *const ncsim_state, block: u64, out: *mut f64, nblocks: u64) -> ncsim_status;
    pub fn ncsim_sv_sample_walk(s: *const ncsim_state, block: u64, targets: *const f64, blocks: *const u64, accs: *const f64, shots: u64, out: *mut u64) -> ncsim_status;
    pub fn ncsim_sv_timer_start(s: *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_timer_stop(s: *mut ncsim_state, milliseconds: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_compare(a: *const ncsim_state, b: *const ncsim_state, inner_re_im: *mut f64, norm_a: *mut f64, norm_b: *mut f64, max_abs_diff: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_set_tile_passes(s: *mut ncsim_state, enable: i32) -> ncsim_status;
    pub fn ncsim_sv_profile_enable(s: *mut ncsim_state, enable: i32) -> ncsim_status;
    pub fn ncsim_sv_profile_read(s: *mut ncsim_state, out: *mut ncsim_kernel_stat, cap: u32, count: *mut u32) -> ncsim_status;
    pub fn ncsim_measure_stats_noalloc(amps: *const c_void, n: u32, precision: i32, x: u64, z: u64, phase: u32, stream: *mut c_void, expectation_re_im: *mut f64, norm_sq: *mut f64) -> ncsim_status;
    pub fn ncsim_rng_new(seed: u64, out: *mut *mut ncsim_rng) -> ncsim_status;
    pub fn ncsim_rng_free(r: *mut ncsim_rng) -> ncsim_status;
    pub fn ncsim_rng_next_u64(r: *mut ncsim_rng, out: *mut u64) -> ncsim_status;
    pub fn ncsim_rng_next_u32(r: *mut ncsim_rng, out: *mut u32) -> ncsim_status;
    pub fn ncsim_rng_gen_f64(r: *mut ncsim_rng, out: *mut f64) -> ncsim_status;
    pub fn ncsim_rng_gen_range(r: *mut ncsim_rng, lo: u64, hi: u64, out: *mut u64) -> ncsim_status;
    pub fn ncsim_circuit_parse(text: *const c_char, out: *mut *mut ncsim_circuit) -> ncsim_status;
    pub fn ncsim_circuit_free(c: *mut ncsim_circuit) -> ncsim_status;
    pub fn ncsim_circuit_info(c: *const ncsim_circuit, num_qubits: *mut u32, num_ops: *mut u64, num_gates: *mut u64, num_measurements: *mut u64) -> ncsim_status;
    pub fn ncsim_circuit_to_text(c: *const ncsim_circuit, buf: *mut c_char, cap: usize, len: *mut usize) -> ncsim_status;
    pub fn ncsim_gate_parse(token: *const c_char, arity_hint: u32, out: *mut *mut ncsim_gate, arity: *mut u32) -> ncsim_status;
    pub fn ncsim_gate_unitary(k: u32, matrix: *const f64, out: *mut *mut ncsim_gate) -> ncsim_status;
    pub fn ncsim_gate_pauli(k: u32, x: u64, z: u64, phase: u32, out: *mut *mut ncsim_gate) -> ncsim_status;
    pub fn ncsim_gate_free(g: *mut ncsim_gate) -> ncsim_status;
    pub fn ncsim_gate_lowered_matrix(g: *const ncsim_gate, out: *mut f64, cap_doubles: usize, k: *mut u32) -> ncsim_status;
    pub fn ncsim_pauli_parse(text: *const c_char, n: u32, x: *mut u64, z: *mut u64, phase: *mut u32) -> ncsim_status;
    pub fn ncsim_pauli_parse_words(text: *const c_char, n: u32, x: *mut u64, z: *mut u64, words: u32, phase: *mut u32) -> ncsim_status;
    pub fn ncsim_sv_apply_gate(s: *mut ncsim_state, g: *const ncsim_gate, qubits: *const u32, k: u32) -> ncsim_status;
    pub fn ncsim_sv_measure(s: *mut ncsim_state, x: u64, z: u64, phase: u32, rng: *mut ncsim_rng, outcome: *mut i32) -> ncsim_status;
    pub fn ncsim_sv_run(s: *mut ncsim_state, c: *const ncsim_circuit, rng: *mut ncsim_rng, rec: *mut u8, cap: usize, len: *mut usize) -> ncsim_status;
    pub fn ncsim_sv_sample_rng(s: *const ncsim_state, rng: *mut ncsim_rng, shots: u64, out: *mut u64) -> ncsim_status;
    pub fn ncsim_sv_normalize(s: *mut ncsim_state) -> ncsim_status;
    pub fn ncsim_sv_probability(s: *const ncsim_state, index: u64, out: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_expectation_sum(s: *const ncsim_state, count: u64, x: *const u64, z: *const u64, phase: *const u32, coeffs: *const f64, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sv_run_fused(s: *mut ncsim_state, c: *const ncsim_circuit, rng: *mut ncsim_rng, max_fuse: u32, rec: *mut u8, cap: usize, len: *mut usize, stats: *mut ncsim_fused_stats) -> ncsim_status;
    pub fn ncsim_fused_emulate(c: *const ncsim_circuit, max_fuse: u32, amps: *mut f64, len: u64, stats: *mut ncsim_fused_stats) -> ncsim_status;
    pub fn ncsim_batch_from_circuits(count: u32, circuits: *const *const ncsim_circuit, seeds: *const u64, out: *mut *mut ncsim_batch) -> ncsim_status;
    pub fn ncsim_batch_free(b: *mut ncsim_batch) -> ncsim_status;
    pub fn ncsim_batch_release(b: *mut ncsim_batch) -> ncsim_status;
    pub fn ncsim_batch_info(b: *const ncsim_batch, st: *mut ncsim_batch_stats) -> ncsim_status;
    pub fn ncsim_batch_trajectory_qubits(b: *const ncsim_batch, n: *mut u32) -> ncsim_status;
    pub fn ncsim_batch_knobs(b: *const ncsim_batch, n: u32, out: *mut ncsim_batch_knobs_info) -> ncsim_status;
    pub fn ncsim_batch_set_knob_set(b: *mut ncsim_batch, n: u32, knob_set: u32, final_: i32) -> ncsim_status;
    pub fn ncsim_batch_set_config(b: *mut ncsim_batch, cfg: *const ncsim_batch_config) -> ncsim_status;
    pub fn ncsim_batch_get_config(b: *mut ncsim_batch, cfg: *mut ncsim_batch_config) -> ncsim_status;
    pub fn ncsim_batch_tune(b: *mut ncsim_batch, sample: u32, best: *mut ncsim_batch_config) -> ncsim_status;
    pub fn ncsim_batch_run(b: *mut ncsim_batch, device_ms: *mut f64) -> ncsim_status;
    pub fn ncsim_batch_results(b: *mut ncsim_batch, n: *mut u32, records: *mut u64, z0: *mut f64, norm: *mut f64) -> ncsim_status;
    pub fn ncsim_batch_emulate(b: *const ncsim_batch, t: u32, record: *mut u64, z0: *mut f64, norm: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_create(n: u32, out: *mut *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_from_entries(n: u32, keys: *const u64, amps: *const f64, count: u64, out: *mut *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_destroy(s: *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_clone(s: *const ncsim_sparse, out: *mut *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_set_cutoff(s: *mut ncsim_sparse, cutoff: f64) -> ncsim_status;
    pub fn ncsim_sparse_num_qubits(s: *const ncsim_sparse, n: *mut u32) -> ncsim_status;
    pub fn ncsim_sparse_num_entries(s: *const ncsim_sparse, count: *mut u64) -> ncsim_status;
    pub fn ncsim_sparse_get_entries(s: *const ncsim_sparse, keys: *mut u64, amps: *mut f64, cap: u64) -> ncsim_status;
    pub fn ncsim_sparse_sort(s: *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_apply_gate(s: *mut ncsim_sparse, g: *const ncsim_gate, qubits: *const u32, k: u32) -> ncsim_status;
    pub fn ncsim_sparse_apply_pauli(s: *mut ncsim_sparse, x: u64, z: u64, phase: u32) -> ncsim_status;
    pub fn ncsim_sparse_norm_sq(s: *const ncsim_sparse, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_amplitude(s: *const ncsim_sparse, index: u64, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_expectation(s: *const ncsim_sparse, x: u64, z: u64, phase: u32, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_inner(a: *const ncsim_sparse, b: *const ncsim_sparse, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_project(s: *mut ncsim_sparse, x: u64, z: u64, phase: u32, outcome: i32, weight_re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_scale(s: *mut ncsim_sparse, re: f64, im: f64) -> ncsim_status;
    pub fn ncsim_sparse_tensor(a: *const ncsim_sparse, b: *const ncsim_sparse, out: *mut *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_sample(s: *const ncsim_sparse, rng: *mut ncsim_rng, shots: u64, out: *mut u64) -> ncsim_status;
    pub fn ncsim_sparse_to_vector(s: *const ncsim_sparse, amps: *mut f64, len: u64) -> ncsim_status;
    pub fn ncsim_sparse_measure(s: *mut ncsim_sparse, x: u64, z: u64, phase: u32, rng: *mut ncsim_rng, outcome: *mut i32) -> ncsim_status;
    pub fn ncsim_sparse_run(s: *mut ncsim_sparse, c: *const ncsim_circuit, rng: *mut ncsim_rng, rec: *mut u8, cap: usize, len: *mut usize) -> ncsim_status;
    pub fn ncsim_sparse_num_words(s: *const ncsim_sparse, words: *mut u32) -> ncsim_status;
    pub fn ncsim_sparse_apply_pauli_words(s: *mut ncsim_sparse, x: *const u64, z: *const u64, words: u32, phase: u32) -> ncsim_status;
    pub fn ncsim_sparse_amplitude_words(s: *const ncsim_sparse, index: *const u64, words: u32, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_expectation_words(s: *const ncsim_sparse, x: *const u64, z: *const u64, words: u32, phase: u32, re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_project_words(s: *mut ncsim_sparse, x: *const u64, z: *const u64, words: u32, phase: u32, outcome: i32, weight_re_im: *mut f64) -> ncsim_status;
    pub fn ncsim_sparse_measure_words(s: *mut ncsim_sparse, x: *const u64, z: *const u64, words: u32, phase: u32, rng: *mut ncsim_rng, outcome: *mut i32) -> ncsim_status;
    pub fn ncsim_sparse_synchronize(s: *const ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_timer_start(s: *mut ncsim_sparse) -> ncsim_status;
    pub fn ncsim_sparse_timer_stop(s: *mut ncsim_sparse, milliseconds: *mut f64) -> ncsim_status;
    pub fn ncsim_frames_new(c: *const ncsim_circuit, reference_seed: u64, out: *mut *mut ncsim_frames) -> ncsim_status;
    pub fn ncsim_frames_with_reference(c: *const ncsim_circuit, reference: *const u8, m: u64, out: *mut *mut ncsim_frames) -> ncsim_status;
    pub fn ncsim_frames_free(f: *mut ncsim_frames) -> ncsim_status;
    pub fn ncsim_frames_info(f: *const ncsim_frames, num_qubits: *mut u32, num_measurements: *mut u64, num_detectors: *mut u64, num_observables: *mut u64, num_layers: *mut u64) -> ncsim_status;
    pub fn ncsim_frames_reference(f: *const ncsim_frames, out: *mut u8, cap: u64) -> ncsim_status;
    pub fn ncsim_frames_sample_packed(f: *mut ncsim_frames, shots: u64, rng: *mut ncsim_rng, out: *mut u64, cap: u64) -> ncsim_status;
    pub fn ncsim_frames_sample_packed_seeds(f: *mut ncsim_frames, shots: u64, seeds: *const u64, nseeds: u64, out: *mut u64, cap: u64) -> ncsim_status;
    pub fn ncsim_frames_sample_packed_device(f: *mut ncsim_frames, shots: u64, seeds: *const u64, nseeds: u64, d_out: *mut u64, cap: u64) -> ncsim_status;
    pub fn ncsim_frames_sample(f: *mut ncsim_frames, shots: u64, rng: *mut ncsim_rng, out: *mut u64, cap: u64) -> ncsim_status;
    pub fn ncsim_frames_sample_detectors(f: *mut ncsim_frames, shots: u64, rng: *mut ncsim_rng, det: *mut u64, det_cap: u64, obs: *mut u64, obs_cap: u64) -> ncsim_status;
    pub fn ncsim_frames_sample_detectors_seeds(f: *mut ncsim_frames, shots: u64, seeds: *const u64, nseeds: u64, det: *mut u64, det_cap: u64, obs: *mut u64, obs_cap: u64) -> ncsim_status;
    pub fn ncsim_frames_last_kernel_ms(f: *const ncsim_frames, ms: *mut f64) -> ncsim_status;
}
