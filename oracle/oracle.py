"""CPU ORACLE — test infrastructure only.

ctypes access to ``liboracle.so``, the C++ restatement of ncsim's dense
``StateVector<C64>`` path (``src/state/vector.rs``, ``src/state/mod.rs``,
``src/gate.rs``, ``src/phasepoly.rs``, ``src/scalar.rs``, ``src/circuit.rs``,
``src/pauli/``).  Only the tests, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` import this module; the product package never
does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build() -> str:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, dbl, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_double, C.c_int
        P = C.POINTER
        sig = {
            "oracle_last_error": (C.c_char_p, []),
            "oracle_num_threads": (i32, []),
            "oracle_set_threads": (None, [i32]),
            "oracle_rng_new": (vp, [u64]),
            "oracle_rng_free": (None, [vp]),
            "oracle_rng_next_u64": (u64, [vp]),
            "oracle_rng_next_u32": (u32, [vp]),
            "oracle_rng_gen_f64": (dbl, [vp]),
            "oracle_rng_gen_range": (u64, [vp, u64, u64]),
            "oracle_chacha_block": (None, [P(u32), u64, i32, P(u32)]),
            "oracle_random_circuit_text": (i32, [u32, u32, u64, dbl, u32, u32, C.c_char_p, C.c_size_t]),
            "oracle_reversible_circuit_text": (i32, [u32, u32, u64, C.c_char_p, C.c_size_t]),
            "oracle_frames_circuit_text": (i32, [u32, u32, u32, dbl, u64, C.c_char_p, C.c_size_t]),
            "oracle_circuit_parse": (vp, [C.c_char_p]),
            "oracle_circuit_free": (None, [vp]),
            "oracle_circuit_num_qubits": (u32, [vp]),
            "oracle_circuit_num_gates": (u32, [vp]),
            "oracle_circuit_num_measurements": (u32, [vp]),
            "oracle_gate_matrix": (i32, [C.c_char_p, P(dbl), C.c_size_t]),
            "oracle_gate_dagger_matrix": (i32, [C.c_char_p, P(dbl), C.c_size_t]),
            "oracle_sv_new": (vp, [u32]),
            "oracle_sv_plus": (vp, [u32]),
            "oracle_sv_clone": (vp, [vp]),
            "oracle_sv_free": (None, [vp]),
            "oracle_sv_set_amplitudes": (i32, [vp, P(dbl), u64]),
            "oracle_sv_get_amplitudes": (i32, [vp, P(dbl), u64]),
            "oracle_sv_set_range": (i32, [vp, P(dbl), u64, u64]),
            "oracle_sv_max_abs_diff": (i32, [vp, P(dbl), u64, u64, P(dbl)]),
            "oracle_sv_apply_gate_text": (i32, [vp, C.c_char_p]),
            "oracle_sv_apply_matrix": (i32, [vp, P(u32), u32, P(dbl)]),
            "oracle_sv_apply_pauli": (i32, [vp, C.c_char_p]),
            "oracle_sv_apply_pauli_raw": (i32, [vp, u64, u64, u32]),
            "oracle_sv_norm_sq": (i32, [vp, P(dbl)]),
            "oracle_sv_expectation": (i32, [vp, C.c_char_p, P(dbl)]),
            "oracle_sv_expectation_raw": (i32, [vp, u64, u64, u32, P(dbl)]),
            "oracle_sv_inner": (i32, [vp, vp, P(dbl)]),
            "oracle_sv_project_raw": (i32, [vp, u64, u64, u32, i32, P(dbl)]),
            "oracle_sv_scale": (i32, [vp, dbl, dbl]),
            "oracle_sv_normalize": (i32, [vp]),
            "oracle_sv_measure": (i32, [vp, C.c_char_p, vp, P(i32)]),
            "oracle_sv_sample": (i32, [vp, vp, u64, P(u64)]),
            "oracle_sv_sample_uniforms": (i32, [vp, P(dbl), u64, P(u64)]),
            "oracle_sv_kron": (vp, [vp, vp]),
            "oracle_sv_run": (i32, [vp, vp, vp, P(C.c_uint8), C.c_size_t]),
            "oracle_sv_run_gates_timed": (dbl, [vp, vp, u64]),
            "oracle_trajectory": (i32, [u64, u32, u32, u32, dbl, P(u32), P(dbl), P(C.c_uint8), C.c_size_t]),
            "oracle_sparse_run": (vp, [C.c_char_p]),
            "oracle_sparse_len": (u64, [vp]),
            "oracle_sparse_get": (None, [vp, P(u64), P(dbl)]),
            "oracle_sparse_free": (None, [vp]),
            "oracle_wsparse_run": (vp, [C.c_char_p, u64, P(C.c_uint8), C.c_size_t, P(C.c_size_t)]),
            "oracle_wsparse_len": (u64, [vp]),
            "oracle_wsparse_words": (u32, [vp]),
            "oracle_wsparse_get": (None, [vp, P(u64), P(dbl)]),
            "oracle_wsparse_expect": (i32, [vp, C.c_char_p, P(dbl)]),
            "oracle_wsparse_sample": (i32, [vp, u64, u64, P(u64)]),
            "oracle_wsparse_free": (None, [vp]),
            "oracle_frames_reference": (i32, [C.c_char_p, u64, P(C.c_uint8), C.c_size_t]),
            "oracle_frames_sample_packed": (i32, [C.c_char_p, P(C.c_uint8), C.c_size_t, u64, P(u64), C.c_size_t, i32,
                                                  P(u64)]),
            "oracle_frames_sample_detectors": (i32, [C.c_char_p, P(C.c_uint8), C.c_size_t, u64, P(u64), C.c_size_t,
                                                     P(u64), C.c_size_t, P(u64), C.c_size_t]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"oracle status {status}: {msg}")
        self.status = status


def _check(st: int) -> int:
    if st < 0:
        raise OracleError(st, lib().oracle_last_error().decode())
    return st


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class StdRng:
    """rand 0.8 StdRng restatement (ChaCha12, PCG32 seed expansion)."""

    def __init__(self, seed: int):
        self.h = lib().oracle_rng_new(seed)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_rng_free(self.h)

    def next_u64(self) -> int:
        return lib().oracle_rng_next_u64(self.h)

    def next_u32(self) -> int:
        return lib().oracle_rng_next_u32(self.h)

    def gen_f64(self) -> float:
        return lib().oracle_rng_gen_f64(self.h)

    def gen_range(self, lo: int, hi: int) -> int:
        return lib().oracle_rng_gen_range(self.h, lo, hi)


def chacha_block(key_words, counter: int, rounds: int) -> list[int]:
    k = (C.c_uint32 * 8)(*key_words)
    out = (C.c_uint32 * 16)()
    lib().oracle_chacha_block(k, counter, rounds, out)
    return list(out)


def _text(fn, *args) -> str:
    n = fn(*args, None, 0)
    buf = C.create_string_buffer(n + 1)
    fn(*args, buf, n + 1)
    return buf.value.decode()


def random_circuit_text(n: int, depth: int, seed: int, noise_p: float = 0.0, m_lo: int = 0, m_hi: int = 0) -> str:
    return _text(lib().oracle_random_circuit_text, n, depth, seed, noise_p, m_lo, m_hi)


def frames_circuit_text(n: int = 1000, rounds: int = 20, meas: int = 100, p: float = 1e-3, seed: int = 9) -> str:
    """The reference's frame-sampler benchmark circuit (examples/bench.rs:264-294)."""
    return _text(lib().oracle_frames_circuit_text, n, rounds, meas, p, seed)


def reversible_circuit_text(n: int, gates: int, seed: int) -> str:
    return _text(lib().oracle_reversible_circuit_text, n, gates, seed)


class Circuit:
    def __init__(self, text: str):
        self.h = lib().oracle_circuit_parse(text.encode())
        if not self.h:
            raise OracleError(-7, lib().oracle_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_circuit_free(self.h)

    @property
    def num_qubits(self) -> int:
        return lib().oracle_circuit_num_qubits(self.h)

    @property
    def num_gates(self) -> int:
        return lib().oracle_circuit_num_gates(self.h)

    @property
    def num_measurements(self) -> int:
        return lib().oracle_circuit_num_measurements(self.h)


def gate_matrix(text: str, dagger: bool = False) -> np.ndarray:
    buf = np.zeros(2 * 4 ** 10, dtype=np.float64)
    fn = lib().oracle_gate_dagger_matrix if dagger else lib().oracle_gate_matrix
    k = _check(fn(text.encode(), _dp(buf), buf.size))
    d = 1 << k
    return (buf[0 : 2 * d * d : 2] + 1j * buf[1 : 2 * d * d : 2]).reshape(d, d)


class StateVector:
    """The dense restatement (``StateVector<C64>``)."""

    def __init__(self, n: int, _h=None):
        self.n = n
        self.h = _h if _h is not None else lib().oracle_sv_new(n)
        if not self.h:
            raise OracleError(-8, lib().oracle_last_error().decode())

    @classmethod
    def plus_state(cls, n: int) -> "StateVector":
        return cls(n, lib().oracle_sv_plus(n))

    @classmethod
    def from_amplitudes(cls, a: np.ndarray) -> "StateVector":
        n = int(a.size).bit_length() - 1
        s = cls(n)
        s.set_amplitudes(a)
        return s

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_sv_free(self.h)

    def clone(self) -> "StateVector":
        return StateVector(self.n, lib().oracle_sv_clone(self.h))

    def set_amplitudes(self, a: np.ndarray) -> None:
        b = np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64)
        _check(lib().oracle_sv_set_amplitudes(self.h, _dp(b), 1 << self.n))

    def to_vector(self) -> np.ndarray:
        b = np.zeros(2 << self.n, dtype=np.float64)
        _check(lib().oracle_sv_get_amplitudes(self.h, _dp(b), 1 << self.n))
        return b.view(np.complex128)

    def set_range(self, first: int, a: np.ndarray) -> None:
        """Amplitudes first .. first+len(a)-1 from complex128 values."""
        b = np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64)
        _check(lib().oracle_sv_set_range(self.h, _dp(b), first, b.size // 2))

    def max_abs_diff(self, first: int, a: np.ndarray) -> float:
        """max |amp[first + i] - a[i]| over the slice."""
        b = np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64)
        out = C.c_double()
        _check(lib().oracle_sv_max_abs_diff(self.h, _dp(b), first, b.size // 2, C.byref(out)))
        return out.value

    def apply_gate_text(self, text: str) -> None:
        _check(lib().oracle_sv_apply_gate_text(self.h, text.encode()))

    def apply_matrix(self, m: np.ndarray, qubits) -> None:
        q = (C.c_uint32 * len(qubits))(*qubits)
        b = np.ascontiguousarray(np.asarray(m, dtype=np.complex128)).view(np.float64)
        _check(lib().oracle_sv_apply_matrix(self.h, q, len(qubits), _dp(b)))

    def apply_pauli(self, p: str) -> None:
        _check(lib().oracle_sv_apply_pauli(self.h, p.encode()))

    def apply_pauli_raw(self, x: int, z: int, phase: int) -> None:
        _check(lib().oracle_sv_apply_pauli_raw(self.h, x, z, phase))

    def norm_sq(self) -> complex:
        o = np.zeros(2)
        _check(lib().oracle_sv_norm_sq(self.h, _dp(o)))
        return complex(o[0], o[1])

    def expectation(self, p: str) -> complex:
        o = np.zeros(2)
        _check(lib().oracle_sv_expectation(self.h, p.encode(), _dp(o)))
        return complex(o[0], o[1])

    def expectation_raw(self, x: int, z: int, phase: int) -> complex:
        o = np.zeros(2)
        _check(lib().oracle_sv_expectation_raw(self.h, x, z, phase, _dp(o)))
        return complex(o[0], o[1])

    def inner(self, other: "StateVector") -> complex:
        o = np.zeros(2)
        _check(lib().oracle_sv_inner(self.h, other.h, _dp(o)))
        return complex(o[0], o[1])

    def project_raw(self, x: int, z: int, phase: int, outcome: bool) -> complex:
        o = np.zeros(2)
        _check(lib().oracle_sv_project_raw(self.h, x, z, phase, int(outcome), _dp(o)))
        return complex(o[0], o[1])

    def scale(self, c: complex) -> None:
        _check(lib().oracle_sv_scale(self.h, c.real, c.imag))

    def normalize(self) -> None:
        _check(lib().oracle_sv_normalize(self.h))

    def measure(self, p: str, rng: StdRng) -> bool:
        o = C.c_int(0)
        _check(lib().oracle_sv_measure(self.h, p.encode(), rng.h, C.byref(o)))
        return bool(o.value)

    def sample(self, rng: StdRng, shots: int) -> np.ndarray:
        out = np.zeros(shots, dtype=np.uint64)
        _check(lib().oracle_sv_sample(self.h, rng.h, shots, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def sample_uniforms(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(u.size, dtype=np.uint64)
        _check(lib().oracle_sv_sample_uniforms(self.h, _dp(u), u.size, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def kron(self, other: "StateVector") -> "StateVector":
        h = lib().oracle_sv_kron(self.h, other.h)
        if not h:
            raise OracleError(-8, lib().oracle_last_error().decode())
        return StateVector(self.n + other.n, h)

    def run(self, circuit: Circuit, rng: StdRng) -> list[bool]:
        cap = max(1, circuit.num_measurements)
        rec = (C.c_uint8 * cap)()
        m = _check(lib().oracle_sv_run(self.h, circuit.h, rng.h, rec, cap))
        return [bool(rec[i]) for i in range(m)]

    def run_gates_timed(self, circuit: Circuit, max_gates: int) -> float:
        return lib().oracle_sv_run_gates_timed(self.h, circuit.h, max_gates)


def trajectory(seed: int, n_lo: int = 16, n_span: int = 7, depth: int = 30, p: float = 1e-3):
    """(n, <Z0>/norm before the final measurements, record) of one noisy trajectory."""
    n = C.c_uint32(0)
    z0 = C.c_double(0.0)
    cap = n_lo + n_span + 1
    rec = (C.c_uint8 * cap)()
    m = _check(lib().oracle_trajectory(seed, n_lo, n_span, depth, p, C.byref(n), C.byref(z0), rec, cap))
    return n.value, z0.value, [bool(rec[i]) for i in range(m)]


def sparse_run(text: str):
    """(indices, amplitudes) of the sparse restatement after a gates-only circuit."""
    h = lib().oracle_sparse_run(text.encode())
    if not h:
        raise OracleError(-8, lib().oracle_last_error().decode())
    try:
        m = lib().oracle_sparse_len(h)
        idx = np.zeros(m, dtype=np.uint64)
        amp = np.zeros(2 * m, dtype=np.float64)
        lib().oracle_sparse_get(h, idx.ctypes.data_as(C.POINTER(C.c_uint64)), _dp(amp))
        return idx, amp.view(np.complex128)
    finally:
        lib().oracle_sparse_free(h)


class WideSparse:
    """The sparse restatement on a register of any width after running a circuit
    text from |0...0> with StdRng::seed_from_u64(seed): the record, the entries in
    entry order (keys as Python integers), expectations and samples."""

    def __init__(self, text: str, seed: int, max_record: int = 4096):
        rec = (C.c_uint8 * max(1, max_record))()
        ln = C.c_size_t()
        h = lib().oracle_wsparse_run(text.encode(), seed, rec, max_record, C.byref(ln))
        if not h:
            raise OracleError(-8, lib().oracle_last_error().decode())
        self._h = h
        self.record = [bool(rec[i]) for i in range(ln.value)]
        self.words = lib().oracle_wsparse_words(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_wsparse_free(h)
            self._h = None

    def _ints(self, arr):
        return [sum(int(w) << (64 * j) for j, w in enumerate(row)) for row in arr.reshape(-1, self.words)]

    def entries(self):
        m = lib().oracle_wsparse_len(self._h)
        k = np.zeros(m * self.words, dtype=np.uint64)
        a = np.zeros(2 * m, dtype=np.float64)
        lib().oracle_wsparse_get(self._h, k.ctypes.data_as(C.POINTER(C.c_uint64)), _dp(a))
        return self._ints(k), a.view(np.complex128)

    def expectation(self, pauli: str) -> complex:
        o = (C.c_double * 2)()
        _check(lib().oracle_wsparse_expect(self._h, pauli.encode(), o))
        return complex(o[0], o[1])

    def sample(self, seed: int, shots: int):
        out = np.zeros(shots * self.words, dtype=np.uint64)
        _check(lib().oracle_wsparse_sample(self._h, seed, shots, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return self._ints(out)


FRAME_BATCH = 1 << 14


def frame_reference(text: str, seed: int) -> list[bool]:
    """FrameSampler::new's reference record (frame.rs:41-60) on the oracle's tableau."""
    cap = text.count("\n") * 64 + 64
    out = np.zeros(cap, dtype=np.uint8)
    m = _check(lib().oracle_frames_reference(text.encode(), seed, out.ctypes.data_as(C.POINTER(C.c_uint8)), cap))
    return [bool(v) for v in out[:m]]


def _frame_args(reference, seeds):
    r = np.ascontiguousarray(np.asarray(list(reference), dtype=np.uint8))
    sd = np.ascontiguousarray(np.asarray(list(seeds), dtype=np.uint64))
    return r, sd


def frame_sample_packed(text: str, reference, shots: int, seeds, threads: int = 1) -> np.ndarray:
    """sample_packed (frame.rs:69-89) with the batch seeds given: (measurements, words) uint64."""
    r, sd = _frame_args(reference, seeds)
    out = np.zeros((r.size, (shots + 63) // 64), dtype=np.uint64)
    P = C.POINTER
    _check(lib().oracle_frames_sample_packed(text.encode(), r.ctypes.data_as(P(C.c_uint8)), r.size, shots,
                                             sd.ctypes.data_as(P(C.c_uint64)), sd.size, threads,
                                             out.ctypes.data_as(P(C.c_uint64))))
    return out


def frame_sample_detectors(text: str, reference, shots: int, seeds, num_detectors: int, num_observables: int):
    """sample_detectors (frame.rs:155-205) with the batch seeds given."""
    r, sd = _frame_args(reference, seeds)
    w = (shots + 63) // 64
    det = np.zeros((num_detectors, w), dtype=np.uint64)
    obs = np.zeros((num_observables, w), dtype=np.uint64)
    P = C.POINTER
    _check(lib().oracle_frames_sample_detectors(text.encode(), r.ctypes.data_as(P(C.c_uint8)), r.size, shots,
                                                sd.ctypes.data_as(P(C.c_uint64)), sd.size,
                                                det.ctypes.data_as(P(C.c_uint64)), num_detectors,
                                                obs.ctypes.data_as(P(C.c_uint64)), num_observables))
    return det, obs
