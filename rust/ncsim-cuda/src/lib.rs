//! `GpuStateVector`: ncsim's dense `StateVector<C64>` (src/state/vector.rs)
//! held in B200 memory and driven by hand-written sm_100a kernels through the
//! C ABI of `include/ncsim_cuda.h` (libncsim_cuda.so).
//!
//! It implements the same `QuantumState<C64>` trait (src/state/mod.rs:41-234)
//! and lowers each `Gate` through the reference's own views, in the order
//! `StateVector::apply_gate` uses (src/state/vector.rs:364-395): Pauli, then
//! monomial, then dense matrix, then decomposition.  The random generator
//! stays on this side: `measure` and `sample` draw from the caller's
//! `RngCore` exactly as the reference does (src/state/mod.rs:113-131,
//! src/state/vector.rs:505) and pass the uniforms down.  There is no CPU
//! fallback.
//!
//! All `unsafe` lives in this crate, so the core crate keeps
//! `#![forbid(unsafe_code)]` (src/lib.rs:36).
//!
//! This crate is written against the reference's public API; the build
//! environment it was developed in had no Rust toolchain, so it has not been
//! compiled there.

pub mod ffi;

use std::ffi::{CStr, CString};
use std::fmt;
use std::os::raw::c_char;

use ncsim::bits::{self, Bits};
use ncsim::{Amplitude, Circuit, Gate, MonomialGate, Op, Pauli, Phasor, QuantumState, Result, SimError, C64};
use rand::{Rng, RngCore};

const BACKEND: &str = "GpuStateVector";

/// Storage of the device register: complex128 (the drop-in for
/// `StateVector<C64>`) or complex64 (the fused precision form's storage).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Precision {
    C128,
    C64,
}

impl Precision {
    fn code(self) -> i32 {
        match self {
            Precision::C128 => ffi::NCSIM_C128,
            Precision::C64 => ffi::NCSIM_C64,
        }
    }
}

fn c_text(s: &[c_char]) -> String {
    let bytes: Vec<u8> = s.iter().take_while(|&&c| c != 0).map(|&c| c as u8).collect();
    String::from_utf8_lossy(&bytes).into_owned()
}

/// The `SimError` of a failed call, with the fields of the variants that
/// carry them (src/error.rs:7-42).  Device and allocation failures become
/// `SimError::Invalid`, which is the closest variant the enum has.
fn last_error(status: ffi::ncsim_status) -> SimError {
    // SAFETY: the library returns a pointer to its thread-local, zero-terminated message.
    let msg = unsafe { CStr::from_ptr(ffi::ncsim_last_error()) }.to_string_lossy().into_owned();
    let mut info = std::mem::MaybeUninit::<ffi::ncsim_error_info>::zeroed();
    // SAFETY: `info` is a valid, writable ncsim_error_info.
    let info = unsafe {
        ffi::ncsim_last_error_info(info.as_mut_ptr());
        info.assume_init()
    };
    let strip = |m: &str, prefix: &str| m.strip_prefix(prefix).unwrap_or(m).to_string();
    match status {
        ffi::NCSIM_ERR_UNSUPPORTED => SimError::Unsupported { backend: BACKEND, what: msg },
        ffi::NCSIM_ERR_QUBIT_OUT_OF_RANGE => SimError::QubitOutOfRange {
            qubit: info.qubit as usize,
            num_qubits: info.num_qubits as usize,
        },
        ffi::NCSIM_ERR_ARITY => SimError::Arity {
            gate: c_text(&info.gate),
            expected: info.expected as usize,
            got: info.got as usize,
        },
        ffi::NCSIM_ERR_DUPLICATE_QUBIT => SimError::DuplicateQubit(info.qubit as usize),
        ffi::NCSIM_ERR_NOT_REPRESENTABLE => SimError::NotRepresentable(msg),
        ffi::NCSIM_ERR_ZERO_STATE => SimError::ZeroState(strip(&msg, "state vanished: ")),
        ffi::NCSIM_ERR_PARSE => SimError::Parse(msg),
        ffi::NCSIM_ERR_DEVICE => SimError::Invalid(format!("device: {msg}")),
        ffi::NCSIM_ERR_OUT_OF_MEMORY => SimError::Invalid(format!("out of device memory: {msg}")),
        _ => SimError::Invalid(msg),
    }
}

fn check(status: ffi::ncsim_status) -> Result<()> {
    if status == ffi::NCSIM_OK {
        Ok(())
    } else {
        Err(last_error(status))
    }
}

/// `check_qubits` (src/error.rs:69-82): in range, no repeats.  The library
/// repeats the check; it is done here first so that the error is the
/// reference's for any gate, whatever view it takes below.
fn check_qubits(qubits: &[usize], n: usize) -> Result<()> {
    for (i, &q) in qubits.iter().enumerate() {
        if q >= n {
            return Err(SimError::QubitOutOfRange { qubit: q, num_qubits: n });
        }
        if qubits[..i].contains(&q) {
            return Err(SimError::DuplicateQubit(q));
        }
    }
    Ok(())
}

/// `(x, z, phase)` of a Pauli on at most 64 qubits (as `pauli_masks`,
/// src/state/vector.rs:353-355).
fn pauli_masks(p: &Pauli) -> (u64, u64, u32) {
    (p.x_bits()[0], p.z_bits()[0], u32::from(p.phase()))
}

fn phasor_c64(p: Phasor) -> C64 {
    C64::from_phasor(p).expect("every phasor is a complex double")
}

/// A dense state vector of `n` qubits in B200 memory.
pub struct GpuStateVector {
    h: *mut ffi::ncsim_state,
    n: usize,
    precision: Precision,
}

// SAFETY: a handle owns its device memory and stream; the library serialises
// the calls made on one handle (a mutex per state), so it may move between
// threads and be shared by the `&self` readers that `expectation_sum`
// (src/state/mod.rs:93-101) and the bridge (src/bridge.rs:456-464) run on
// rayon threads.
unsafe impl Send for GpuStateVector {}
unsafe impl Sync for GpuStateVector {}

impl GpuStateVector {
    /// `|0…0⟩` (StateVector::zero_state, vector.rs:25).  Up to 33 qubits in
    /// complex128 and 34 in complex64 (device memory bound); the reference
    /// stops at 30 (vector.rs:30).
    pub fn zero_state(n: usize) -> Result<Self> {
        Self::with_precision(n, Precision::C128)
    }

    pub fn with_precision(n: usize, precision: Precision) -> Result<Self> {
        let mut h = std::ptr::null_mut();
        // SAFETY: `h` is a valid out pointer.
        check(unsafe { ffi::ncsim_sv_create(n as u32, precision.code(), &mut h) })?;
        Ok(GpuStateVector { h, n, precision })
    }

    /// `|x⟩` (vector.rs:29-34).
    pub fn basis_state(n: usize, x: &[u64]) -> Result<Self> {
        let s = Self::zero_state(n)?;
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_sv_set_basis(s.h, bits::to_u64(x, n)) })?;
        Ok(s)
    }

    /// `|+⟩^n` with amplitude `sqrt2_pow(-n)` (vector.rs:36-42).
    pub fn plus_state(n: usize) -> Result<Self> {
        let s = Self::zero_state(n)?;
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_sv_set_plus(s.h) })?;
        Ok(s)
    }

    /// From `2^n` amplitudes (vector.rs:44-52).
    pub fn from_amplitudes(n: usize, amps: &[C64]) -> Result<Self> {
        if amps.len() != 1usize << n {
            return Err(SimError::Invalid(format!("{} amplitudes for {n} qubits", amps.len())));
        }
        let s = Self::zero_state(n)?;
        let flat: Vec<f64> = amps.iter().flat_map(|a| [a.re, a.im]).collect();
        // SAFETY: `flat` holds 2^n interleaved complex numbers.
        check(unsafe { ffi::ncsim_sv_set_amplitudes(s.h, flat.as_ptr(), amps.len() as u64) })?;
        Ok(s)
    }

    pub fn precision(&self) -> Precision {
        self.precision
    }

    /// `StateVector::apply_matrix` (vector.rs:67-93): a dense `2^k x 2^k`
    /// row-major matrix over the local index whose bit `j` is `qubits[j]`.
    pub fn apply_matrix(&mut self, m: &[C64], qubits: &[usize]) -> Result<()> {
        let k = qubits.len();
        if m.len() != 1usize << (2 * k) {
            return Err(SimError::Invalid("matrix size".into()));
        }
        let q: Vec<u32> = qubits.iter().map(|&q| q as u32).collect();
        let flat: Vec<f64> = m.iter().flat_map(|a| [a.re, a.im]).collect();
        // SAFETY: `q` holds k qubits and `flat` 4^k complex numbers.
        check(unsafe { ffi::ncsim_sv_apply_matrix(self.h, q.as_ptr(), k as u32, flat.as_ptr()) })
    }

    /// `StateVector::apply_monomial` (vector.rs:96-139).  A diagonal gate on
    /// more than 10 qubits goes down as its phase polynomial, evaluated on the
    /// device from each basis index (the reference's `2^k` table would not
    /// fit); everything else as the table of `MonomialGate::apply_to_basis`
    /// (gate.rs:157-169).
    pub fn apply_monomial(&mut self, m: &MonomialGate, qubits: &[usize]) -> Result<()> {
        let k = m.num_qubits();
        let q: Vec<u32> = qubits.iter().map(|&q| q as u32).collect();
        if m.is_diagonal() && k > 10 {
            let poly = m.phase();
            let mut term_start = vec![0u32];
            let mut parities = Vec::new();
            let mut coeffs = Vec::new();
            for (lams, c) in poly.terms() {
                for l in lams {
                    parities.push(l[0]);
                }
                term_start.push(parities.len() as u32);
                coeffs.push(c);
            }
            let (s2, sphase, sbits) = match m.scalar() {
                Phasor::Value { sqrt2_power, phase, bits } => (sqrt2_power, phase, bits),
                Phasor::Zero => return self.scale(&C64::new(0.0, 0.0)),
            };
            // SAFETY: the arrays hold the term_start (nterms + 1), parity and coefficient lists.
            return check(unsafe {
                ffi::ncsim_sv_apply_phasepoly(
                    self.h,
                    q.as_ptr(),
                    k as u32,
                    poly.bits(),
                    poly.constant(),
                    coeffs.len() as u32,
                    term_start.as_ptr(),
                    parities.as_ptr(),
                    coeffs.as_ptr(),
                    s2,
                    sphase,
                    sbits,
                )
            });
        }
        let d = 1usize << k;
        let mut image = Vec::with_capacity(d);
        let mut phase = Vec::with_capacity(2 * d);
        for x in 0..d as u64 {
            let (s, y) = m.apply_to_basis(&bits::from_u64(x, k));
            image.push(bits::to_u64(&y, k));
            let c = phasor_c64(s);
            phase.push(c.re);
            phase.push(c.im);
        }
        // SAFETY: `image` holds 2^k images and `phase` 2^k complex numbers.
        check(unsafe { ffi::ncsim_sv_apply_monomial(self.h, q.as_ptr(), k as u32, image.as_ptr(), phase.as_ptr()) })
    }

    /// `StateVector::apply_pauli` (vector.rs:143-164) of a Pauli on the register.
    pub fn apply_pauli(&mut self, p: &Pauli) -> Result<()> {
        let (x, z, ph) = pauli_masks(p);
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_sv_apply_pauli(self.h, x, z, ph) })
    }

    /// `⟨ψ|P|ψ⟩` and `⟨ψ|ψ⟩` in one pass over the register.
    pub fn measure_stats(&self, p: &Pauli) -> Result<(C64, f64)> {
        let (x, z, ph) = pauli_masks(p);
        let mut e = [0.0f64; 2];
        let mut nn = 0.0f64;
        // SAFETY: the outputs are valid.
        check(unsafe { ffi::ncsim_sv_measure_stats(self.h, x, z, ph, e.as_mut_ptr(), &mut nn) })?;
        Ok((C64::new(e[0], e[1]), nn))
    }

    /// The fused precision form on a complex64 register: runs of gates fused
    /// into unitaries of at most 5 qubits and applied as BF16x3 tensor-core
    /// products.  Its measurements draw from the library's restatement of
    /// `StdRng::seed_from_u64(seed)`.
    pub fn run_fused(&mut self, circuit: &Circuit, seed: u64) -> Result<(Vec<bool>, ffi::ncsim_fused_stats)> {
        let c = CCircuit::from_circuit(circuit)?;
        let rng = CRng::new(seed)?;
        let m = circuit.num_measurements();
        let mut rec = vec![0u8; m.max(1)];
        let mut len = 0usize;
        let mut st = ffi::ncsim_fused_stats::default();
        // SAFETY: every pointer is live; `rec` holds `m` bytes.
        check(unsafe { ffi::ncsim_sv_run_fused(self.h, c.0, rng.0, 5, rec.as_mut_ptr(), m, &mut len, &mut st) })?;
        Ok((rec[..len].iter().map(|&b| b != 0).collect(), st))
    }

    /// Waits for the register's queued device work.
    pub fn synchronize(&self) -> Result<()> {
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_sv_synchronize(self.h) })
    }

    fn scalar_call(
        &self,
        f: impl FnOnce(*mut f64) -> ffi::ncsim_status,
    ) -> Result<C64> {
        let mut v = [0.0f64; 2];
        check(f(v.as_mut_ptr()))?;
        Ok(C64::new(v[0], v[1]))
    }
}

impl Drop for GpuStateVector {
    fn drop(&mut self) {
        // SAFETY: the handle is owned and dropped once.
        unsafe {
            ffi::ncsim_sv_destroy(self.h);
        }
    }
}

impl Clone for GpuStateVector {
    /// A device-to-device copy (vector.rs:15).  It needs a second register's
    /// device memory; `Clone` cannot return an error, so running out of it
    /// panics (at n = 34 in complex64 it always does).
    fn clone(&self) -> Self {
        let mut h = std::ptr::null_mut();
        // SAFETY: the handle is live and `h` is a valid out pointer.
        let st = unsafe { ffi::ncsim_sv_clone(self.h, &mut h) };
        if st != ffi::NCSIM_OK {
            panic!("GpuStateVector::clone: {}", last_error(st));
        }
        GpuStateVector { h, n: self.n, precision: self.precision }
    }
}

impl fmt::Debug for GpuStateVector {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "GpuStateVector({} qubits, {:?})", self.n, self.precision)
    }
}

impl QuantumState<C64> for GpuStateVector {
    const BACKEND: &'static str = BACKEND;

    fn num_qubits(&self) -> usize {
        self.n
    }

    /// vector.rs:364-395: check_qubits, the arity check, then the views in
    /// the reference's order.
    fn apply_gate(&mut self, gate: &Gate, qubits: &[usize]) -> Result<()> {
        check_qubits(qubits, self.n)?;
        if qubits.len() != gate.arity() {
            return Err(SimError::Arity { gate: gate.name(), expected: gate.arity(), got: qubits.len() });
        }
        if let Gate::Pauli(p) = gate {
            return self.apply_pauli(&p.embed(self.n, qubits));
        }
        if let Some(m) = gate.monomial() {
            return self.apply_monomial(&m, qubits);
        }
        if let Some(m) = gate.matrix::<C64>() {
            return self.apply_matrix(&m, qubits);
        }
        if let Some(c) = gate.decomposition() {
            for op in c.ops() {
                if let Op::Gate { gate: g, qubits: qs } = op {
                    let mapped: Vec<usize> = qs.iter().map(|&q| qubits[q]).collect();
                    self.apply_gate(g, &mapped)?;
                }
            }
            return Ok(());
        }
        Err(SimError::NotRepresentable(format!("gate {gate} in the scalar type")))
    }

    fn norm_sq(&self) -> Result<C64> {
        // SAFETY: the output holds two doubles.
        self.scalar_call(|out| unsafe { ffi::ncsim_sv_norm_sq(self.h, out) })
    }

    fn amplitude(&self, x: &[u64]) -> Result<C64> {
        let i = bits::to_u64(x, self.n);
        // SAFETY: the output holds two doubles.
        self.scalar_call(|out| unsafe { ffi::ncsim_sv_get_amplitude(self.h, i, out) })
    }

    fn expectation(&self, p: &Pauli) -> Result<C64> {
        if p.num_qubits() != self.n {
            return Err(SimError::Invalid("expectation: operator on the wrong register".into()));
        }
        let (x, z, ph) = pauli_masks(p);
        // SAFETY: the output holds two doubles.
        self.scalar_call(|out| unsafe { ffi::ncsim_sv_expectation(self.h, x, z, ph, out) })
    }

    fn inner(&self, other: &Self) -> Result<C64> {
        if other.n != self.n {
            return Err(SimError::Invalid("inner: register sizes differ".into()));
        }
        // SAFETY: both handles are live; the output holds two doubles.
        self.scalar_call(|out| unsafe { ffi::ncsim_sv_inner(self.h, other.h, out) })
    }

    fn project(&mut self, p: &Pauli, outcome: bool) -> Result<C64> {
        if !p.is_hermitian() {
            return Err(SimError::Invalid(format!("projector of non-Hermitian {p}")));
        }
        let (x, z, ph) = pauli_masks(p);
        let h = self.h;
        // SAFETY: the output holds two doubles.
        self.scalar_call(|out| unsafe { ffi::ncsim_sv_project(h, x, z, ph, i32::from(outcome), out) })
    }

    fn scale(&mut self, c: &C64) -> Result<()> {
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_sv_scale(self.h, c.re, c.im) })
    }

    fn tensor(&self, other: &Self) -> Result<Self> {
        let mut h = std::ptr::null_mut();
        // SAFETY: both handles are live; `h` is a valid out pointer.
        check(unsafe { ffi::ncsim_sv_kron(self.h, other.h, &mut h) })?;
        Ok(GpuStateVector { h, n: self.n + other.n, precision: self.precision })
    }

    /// `measure` (src/state/mod.rs:113-131) with ⟨P⟩ and ⟨ψ|ψ⟩ from one pass:
    /// the same clamp, the same certainty thresholds, a draw only when the
    /// outcome is uncertain, then the projection.
    fn measure(&mut self, p: &Pauli, rng: &mut dyn RngCore) -> Result<bool> {
        if !p.is_hermitian() {
            return Err(SimError::Invalid(format!("measured operator {p} is not Hermitian")));
        }
        if p.num_qubits() != self.n {
            return Err(SimError::Invalid("expectation: operator on the wrong register".into()));
        }
        let (e, nn) = self.measure_stats(p)?;
        let p_plus = ((1.0 + e.re / nn) / 2.0).clamp(0.0, 1.0);
        let outcome = if p_plus > 1.0 - 1e-12 {
            false
        } else if p_plus < 1e-12 {
            true
        } else {
            rng.gen::<f64>() >= p_plus
        };
        self.project(p, outcome)?;
        Ok(outcome)
    }

    /// One-pass Born sampling (vector.rs:494-540): the shots' uniforms are
    /// drawn here in shot order, the block weights and walks run on the device.
    fn sample(&self, rng: &mut dyn RngCore, shots: usize) -> Result<Vec<Bits>> {
        let u: Vec<f64> = (0..shots).map(|_| rng.gen::<f64>()).collect();
        let mut out = vec![0u64; shots];
        // SAFETY: `u` and `out` hold `shots` values.
        check(unsafe { ffi::ncsim_sv_sample(self.h, u.as_ptr(), shots as u64, out.as_mut_ptr()) })?;
        Ok(out.into_iter().map(|i| bits::from_u64(i, self.n)).collect())
    }

    fn to_vector(&self) -> Result<Vec<C64>> {
        let len = 1usize << self.n;
        let mut flat = vec![0.0f64; 2 * len];
        // SAFETY: `flat` holds 2^n complex numbers.
        check(unsafe { ffi::ncsim_sv_get_amplitudes(self.h, flat.as_mut_ptr(), len as u64) })?;
        Ok(flat.chunks_exact(2).map(|c| C64::new(c[0], c[1])).collect())
    }
}

/// A circuit in the library's own form, parsed from the reference's text
/// format (src/circuit.rs:459-565, printed by its `Display`, :693-728).
struct CCircuit(*mut ffi::ncsim_circuit);

impl CCircuit {
    fn from_circuit(c: &Circuit) -> Result<Self> {
        let text = CString::new(c.to_string()).map_err(|e| SimError::Invalid(e.to_string()))?;
        let mut h = std::ptr::null_mut();
        // SAFETY: `text` is zero-terminated and `h` a valid out pointer.
        check(unsafe { ffi::ncsim_circuit_parse(text.as_ptr(), &mut h) })?;
        Ok(CCircuit(h))
    }
}

impl Drop for CCircuit {
    fn drop(&mut self) {
        // SAFETY: owned, dropped once.
        unsafe {
            ffi::ncsim_circuit_free(self.0);
        }
    }
}

/// The library's restatement of `StdRng::seed_from_u64` (rand 0.8, ChaCha12).
struct CRng(*mut ffi::ncsim_rng);

impl CRng {
    fn new(seed: u64) -> Result<Self> {
        let mut h = std::ptr::null_mut();
        // SAFETY: `h` is a valid out pointer.
        check(unsafe { ffi::ncsim_rng_new(seed, &mut h) })?;
        Ok(CRng(h))
    }
}

impl Drop for CRng {
    fn drop(&mut self) {
        // SAFETY: owned, dropped once.
        unsafe {
            ffi::ncsim_rng_free(self.0);
        }
    }
}

/// Many independent noisy trajectories in one persistent kernel (the
/// batching form): trajectory `t` is `QuantumState::run` of `circuits[t]`
/// with `StdRng::seed_from_u64(seeds[t])` (the library's restatement).
pub struct TrajectoryBatch(*mut ffi::ncsim_batch);

// SAFETY: the library serialises the calls made on one batch.
unsafe impl Send for TrajectoryBatch {}

/// Per trajectory: the register size, the record (bit k = outcome of `M k`),
/// ⟨Z0⟩/⟨ψ|ψ⟩ just before the measurements and ⟨ψ|ψ⟩ there.
#[derive(Clone, Debug, Default)]
pub struct TrajectoryResults {
    pub qubits: Vec<u32>,
    pub records: Vec<u64>,
    pub z0: Vec<f64>,
    pub norm: Vec<f64>,
}

impl TrajectoryBatch {
    pub fn from_circuits(circuits: &[Circuit], seeds: &[u64]) -> Result<Self> {
        if circuits.len() != seeds.len() {
            return Err(SimError::Invalid("one seed per circuit".into()));
        }
        let cs: Vec<CCircuit> = circuits.iter().map(CCircuit::from_circuit).collect::<Result<_>>()?;
        let ptrs: Vec<*const ffi::ncsim_circuit> = cs.iter().map(|c| c.0 as *const _).collect();
        let mut h = std::ptr::null_mut();
        // SAFETY: `ptrs` and `seeds` hold `len` entries; `h` is a valid out pointer.
        check(unsafe { ffi::ncsim_batch_from_circuits(ptrs.len() as u32, ptrs.as_ptr(), seeds.as_ptr(), &mut h) })?;
        Ok(TrajectoryBatch(h))
    }

    /// Runs every trajectory; returns the device milliseconds.
    pub fn run(&mut self) -> Result<f64> {
        let mut ms = 0.0;
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_batch_run(self.0, &mut ms) })?;
        Ok(ms)
    }

    pub fn results(&mut self) -> Result<TrajectoryResults> {
        let mut st = ffi::ncsim_batch_stats::default();
        // SAFETY: the handle is live.
        check(unsafe { ffi::ncsim_batch_info(self.0, &mut st) })?;
        let c = st.trajectories as usize;
        let mut r = TrajectoryResults {
            qubits: vec![0; c],
            records: vec![0; c],
            z0: vec![0.0; c],
            norm: vec![0.0; c],
        };
        // SAFETY: every array holds `c` entries.
        check(unsafe {
            ffi::ncsim_batch_results(
                self.0,
                r.qubits.as_mut_ptr(),
                r.records.as_mut_ptr(),
                r.z0.as_mut_ptr(),
                r.norm.as_mut_ptr(),
            )
        })?;
        Ok(r)
    }
}

impl Drop for TrajectoryBatch {
    fn drop(&mut self) {
        // SAFETY: owned, dropped once.
        unsafe {
            ffi::ncsim_batch_free(self.0);
        }
    }
}

/// The Pauli-frame sampler on the device: the drop-in for ncsim's
/// `FrameSampler` (src/frame.rs:34-300).  The reference record comes from
/// ncsim's own `FrameSampler::new` (its stabilizer tableau), so the records
/// are those of the reference for the same `reference_seed`; the batches'
/// seeds are drawn from the caller's generator, one `next_u64` per batch of
/// 16384 shots in order (frame.rs:72-74), and the frames run on the device.
pub struct GpuFrameSampler {
    h: *mut ffi::ncsim_frames,
    reference: Vec<bool>,
    detectors: usize,
    observables: usize,
}

// SAFETY: the library serialises the calls made on one sampler.
unsafe impl Send for GpuFrameSampler {}

const FRAME_BATCH: usize = 1 << 14;

impl GpuFrameSampler {
    /// `FrameSampler::new` (frame.rs:41-60): Unsupported for a non-Clifford gate.
    pub fn new(circuit: &Circuit, reference_seed: u64) -> Result<Self> {
        let reference = ncsim::FrameSampler::new(circuit, reference_seed)?.reference().to_vec();
        let c = CCircuit::from_circuit(circuit)?;
        let bytes: Vec<u8> = reference.iter().map(|&b| b as u8).collect();
        let mut h = std::ptr::null_mut();
        // SAFETY: `bytes` holds `len` entries; `h` is a valid out pointer.
        check(unsafe { ffi::ncsim_frames_with_reference(c.0, bytes.as_ptr(), bytes.len() as u64, &mut h) })?;
        Ok(GpuFrameSampler {
            h,
            reference,
            detectors: circuit.detectors().len(),
            observables: circuit.observables().len(),
        })
    }

    /// The noiseless reference record.
    pub fn reference(&self) -> &[bool] {
        &self.reference
    }

    fn seeds(shots: usize, rng: &mut dyn RngCore) -> Vec<u64> {
        (0..shots.div_ceil(FRAME_BATCH)).map(|_| rng.next_u64()).collect()
    }

    fn unpack(flat: &[u64], rows: usize, shots: usize) -> Vec<Bits> {
        let w = bits::nwords(shots);
        (0..rows).map(|k| flat[k * w..(k + 1) * w].to_vec()).collect()
    }

    /// `sample_packed` (frame.rs:69-89): entry `k` holds measurement `k` over the shots.
    pub fn sample_packed(&self, shots: usize, rng: &mut dyn RngCore) -> Result<Vec<Bits>> {
        let seeds = Self::seeds(shots, rng);
        let m = self.reference.len();
        let mut flat = vec![0u64; m * bits::nwords(shots)];
        // SAFETY: `seeds` and `flat` hold the lengths passed.
        check(unsafe {
            ffi::ncsim_frames_sample_packed_seeds(
                self.h,
                shots as u64,
                seeds.as_ptr(),
                seeds.len() as u64,
                flat.as_mut_ptr(),
                flat.len() as u64,
            )
        })?;
        Ok(Self::unpack(&flat, m, shots))
    }

    /// `sample` (frame.rs:90-102): one record per shot (bit `k` = measurement `k`).
    pub fn sample(&self, shots: usize, rng: &mut dyn RngCore) -> Result<Vec<Bits>> {
        let packed = self.sample_packed(shots, rng)?;
        let m = self.reference.len();
        let mut out = vec![bits::zero(m); shots];
        for (k, col) in packed.iter().enumerate() {
            for s in bits::ones(col) {
                if s < shots {
                    bits::set(&mut out[s], k, true);
                }
            }
        }
        Ok(out)
    }

    /// `sample_detectors` (frame.rs:155-205): detector and observable flips, packed.
    pub fn sample_detectors(&self, shots: usize, rng: &mut dyn RngCore) -> Result<(Vec<Bits>, Vec<Bits>)> {
        let seeds = Self::seeds(shots, rng);
        let w = bits::nwords(shots);
        let mut det = vec![0u64; self.detectors * w];
        let mut obs = vec![0u64; self.observables * w];
        // SAFETY: `seeds`, `det` and `obs` hold the lengths passed.
        check(unsafe {
            ffi::ncsim_frames_sample_detectors_seeds(
                self.h,
                shots as u64,
                seeds.as_ptr(),
                seeds.len() as u64,
                det.as_mut_ptr(),
                det.len() as u64,
                obs.as_mut_ptr(),
                obs.len() as u64,
            )
        })?;
        Ok((Self::unpack(&det, self.detectors, shots), Self::unpack(&obs, self.observables, shots)))
    }
}

impl Drop for GpuFrameSampler {
    fn drop(&mut self) {
        // SAFETY: owned, dropped once.
        unsafe {
            ffi::ncsim_frames_free(self.h);
        }
    }
}
