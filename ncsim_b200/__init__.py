"""ncsim_b200 — a B200 dense statevector engine behind ncsim's ``QuantumState<C64>`` interface.

Python binding (ctypes) of ``libncsim_cuda.so``.  The names follow the
reference's trait and types (``src/state/mod.rs:41-234``,
``src/state/vector.rs``, ``src/gate.rs``, ``src/circuit.rs``): a
``GpuStateVector`` offers ``apply_gate``, ``run``, ``amplitude``,
``expectation``, ``expectation_sum``, ``norm_sq``, ``inner``, ``project``,
``scale``, ``measure``, ``sample``, ``to_vector``, ``normalize``,
``probability`` and ``tensor``.

There is no CPU fallback: every operation runs the CUDA kernels of the
library, and importing this module fails loudly when the library is absent.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Iterable, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libncsim_cuda.so")

C128 = 0
C64 = 1

# status codes (include/ncsim_cuda.h), mirroring SimError (src/error.rs:7-42)
STATUS_NAMES = {
    1: "Unsupported",
    2: "QubitOutOfRange",
    3: "Arity",
    4: "DuplicateQubit",
    5: "NotRepresentable",
    6: "ZeroState",
    7: "Parse",
    8: "Invalid",
    9: "Device",
    10: "OutOfMemory",
}


class SimError(RuntimeError):
    """An error status of the engine; ``kind`` names the SimError variant and
    ``fields`` holds the variant's fields where it has some (src/error.rs:17-33):
    ``{"qubit", "num_qubits"}`` for QubitOutOfRange, ``{"qubit"}`` for
    DuplicateQubit, ``{"gate", "expected", "got"}`` for Arity."""

    def __init__(self, status: int, message: str, fields: dict | None = None):
        self.status = status
        self.kind = STATUS_NAMES.get(status, f"status{status}")
        self.fields = fields or {}
        super().__init__(f"{self.kind}: {message}")


class ErrorInfo(C.Structure):
    _fields_ = [("code", C.c_int32), ("qubit", C.c_uint64), ("num_qubits", C.c_uint64), ("expected", C.c_uint64),
                ("got", C.c_uint64), ("gate", C.c_char * 64)]


_lib = None
_wlib = None
WORKLOADS_PATH = os.path.join(_HERE, "libncsim_workloads.so")

_P = C.POINTER
_u32, _u64, _i32, _dbl, _vp = C.c_uint32, C.c_uint64, C.c_int32, C.c_double, C.c_void_p

_SIGNATURES = {
    "ncsim_last_error": (C.c_char_p, []),
    "ncsim_last_error_info": (_i32, [_vp]),
    "ncsim_abi_version": (_i32, []),
    "ncsim_device_info": (_i32, [_P(_i32), _P(_u64), _P(_u64)]),
    "ncsim_trim_memory": (_i32, []),
    "ncsim_pool_info": (_i32, [_P(_u64), _P(_u64)]),
    "ncsim_sv_create": (_i32, [_u32, _i32, _P(_vp)]),
    "ncsim_sv_destroy": (_i32, [_vp]),
    "ncsim_sv_clone": (_i32, [_vp, _P(_vp)]),
    "ncsim_sv_num_qubits": (_i32, [_vp, _P(_u32)]),
    "ncsim_sv_precision": (_i32, [_vp, _P(_i32)]),
    "ncsim_sv_set_basis": (_i32, [_vp, _u64]),
    "ncsim_sv_set_plus": (_i32, [_vp]),
    "ncsim_sv_set_amplitudes": (_i32, [_vp, _P(_dbl), _u64]),
    "ncsim_sv_get_amplitudes": (_i32, [_vp, _P(_dbl), _u64]),
    "ncsim_sv_get_amplitudes_range": (_i32, [_vp, _u64, _u64, _P(_dbl)]),
    "ncsim_sv_device_pointer": (_i32, [_vp, _P(_vp), _P(_u64)]),
    "ncsim_sv_block_weights": (_i32, [_vp, _u64, _P(_dbl), _u64]),
    "ncsim_sv_sample_walk": (_i32, [_vp, _u64, _P(_dbl), _P(_u64), _P(_dbl), _u64, _P(_u64)]),
    "ncsim_sv_get_amplitude": (_i32, [_vp, _u64, _P(_dbl)]),
    "ncsim_sv_gather_amplitudes": (_i32, [_vp, _P(_u64), _u64, _P(_dbl)]),
    "ncsim_sv_apply_matrix": (_i32, [_vp, _P(_u32), _u32, _P(_dbl)]),
    "ncsim_sv_apply_monomial": (_i32, [_vp, _P(_u32), _u32, _P(_u64), _P(_dbl)]),
    "ncsim_sv_apply_phasepoly": (
        _i32,
        [_vp, _P(_u32), _u32, _u32, _u64, _u32, _P(_u32), _P(_u64), _P(_u64), _i32, _u64, _u32],
    ),
    "ncsim_sv_apply_pauli": (_i32, [_vp, _u64, _u64, _u32]),
    "ncsim_sv_norm_sq": (_i32, [_vp, _P(_dbl)]),
    "ncsim_sv_expectation": (_i32, [_vp, _u64, _u64, _u32, _P(_dbl)]),
    "ncsim_sv_measure_stats": (_i32, [_vp, _u64, _u64, _u32, _P(_dbl), _P(_dbl)]),
    "ncsim_sv_inner": (_i32, [_vp, _vp, _P(_dbl)]),
    "ncsim_sv_project": (_i32, [_vp, _u64, _u64, _u32, _i32, _P(_dbl)]),
    "ncsim_sv_scale": (_i32, [_vp, _dbl, _dbl]),
    "ncsim_sv_sample": (_i32, [_vp, _P(_dbl), _u64, _P(_u64)]),
    "ncsim_sv_kron": (_i32, [_vp, _vp, _P(_vp)]),
    "ncsim_sv_synchronize": (_i32, [_vp]),
    "ncsim_rng_new": (_i32, [_u64, _P(_vp)]),
    "ncsim_rng_free": (_i32, [_vp]),
    "ncsim_rng_next_u64": (_i32, [_vp, _P(_u64)]),
    "ncsim_rng_next_u32": (_i32, [_vp, _P(_u32)]),
    "ncsim_rng_gen_f64": (_i32, [_vp, _P(_dbl)]),
    "ncsim_rng_gen_range": (_i32, [_vp, _u64, _u64, _P(_u64)]),
    "ncsim_circuit_parse": (_i32, [C.c_char_p, _P(_vp)]),
    "ncsim_circuit_free": (_i32, [_vp]),
    "ncsim_circuit_info": (_i32, [_vp, _P(_u32), _P(_u64), _P(_u64), _P(_u64)]),
    "ncsim_circuit_to_text": (_i32, [_vp, C.c_char_p, C.c_size_t, _P(C.c_size_t)]),
    "ncsim_gate_parse": (_i32, [C.c_char_p, _u32, _P(_vp), _P(_u32)]),
    "ncsim_gate_unitary": (_i32, [_u32, _P(_dbl), _P(_vp)]),
    "ncsim_gate_pauli": (_i32, [_u32, _u64, _u64, _u32, _P(_vp)]),
    "ncsim_gate_free": (_i32, [_vp]),
    "ncsim_gate_lowered_matrix": (_i32, [_vp, _P(_dbl), C.c_size_t, _P(_u32)]),
    "ncsim_pauli_parse": (_i32, [C.c_char_p, _u32, _P(_u64), _P(_u64), _P(_u32)]),
    "ncsim_pauli_parse_words": (_i32, [C.c_char_p, _u32, _P(_u64), _P(_u64), _u32, _P(_u32)]),
    "ncsim_sv_apply_gate": (_i32, [_vp, _vp, _P(_u32), _u32]),
    "ncsim_sv_measure": (_i32, [_vp, _u64, _u64, _u32, _vp, _P(_i32)]),
    "ncsim_sv_run": (_i32, [_vp, _vp, _vp, _P(C.c_uint8), C.c_size_t, _P(C.c_size_t)]),
    "ncsim_sv_sample_rng": (_i32, [_vp, _vp, _u64, _P(_u64)]),
    "ncsim_sv_normalize": (_i32, [_vp]),
    "ncsim_sv_probability": (_i32, [_vp, _u64, _P(_dbl)]),
    "ncsim_sv_expectation_sum": (_i32, [_vp, _u64, _P(_u64), _P(_u64), _P(_u32), _P(_dbl), _P(_dbl)]),
    "ncsim_sv_run_fused": (_i32, [_vp, _vp, _vp, _u32, _P(C.c_uint8), C.c_size_t, _P(C.c_size_t), _vp]),
    "ncsim_fused_emulate": (_i32, [_vp, _u32, _P(_dbl), _u64, _vp]),
    "ncsim_sv_timer_start": (_i32, [_vp]),
    "ncsim_sv_timer_stop": (_i32, [_vp, _P(_dbl)]),
    "ncsim_sv_compare": (_i32, [_vp, _vp, _P(_dbl), _P(_dbl), _P(_dbl), _P(_dbl)]),
    "ncsim_sv_profile_enable": (_i32, [_vp, _i32]),
    "ncsim_sv_profile_read": (_i32, [_vp, _vp, _u32, _P(_u32)]),
    "ncsim_measure_stats_noalloc": (_i32, [_vp, _u32, _i32, _u64, _u64, _u32, _vp, _P(_dbl), _P(_dbl)]),
    "ncsim_batch_from_circuits": (_i32, [_u32, _P(_vp), _P(_u64), _P(_vp)]),
    "ncsim_batch_free": (_i32, [_vp]),
    "ncsim_batch_release": (_i32, [_vp]),
    "ncsim_batch_knobs": (_i32, [_vp, _u32, _vp]),
    "ncsim_batch_set_knob_set": (_i32, [_vp, _u32, _u32, _i32]),
    "ncsim_batch_info": (_i32, [_vp, _vp]),
    "ncsim_batch_trajectory_qubits": (_i32, [_vp, _P(_u32)]),
    "ncsim_batch_set_config": (_i32, [_vp, _vp]),
    "ncsim_batch_get_config": (_i32, [_vp, _vp]),
    "ncsim_batch_tune": (_i32, [_vp, _u32, _vp]),
    "ncsim_batch_run": (_i32, [_vp, _P(_dbl)]),
    "ncsim_batch_results": (_i32, [_vp, _P(_u32), _P(_u64), _P(_dbl), _P(_dbl)]),
    "ncsim_batch_emulate": (_i32, [_vp, _u32, _P(_u64), _P(_dbl), _P(_dbl)]),
    "ncsim_sparse_create": (_i32, [_u32, _P(_vp)]),
    "ncsim_sparse_from_entries": (_i32, [_u32, _P(_u64), _P(_dbl), _u64, _P(_vp)]),
    "ncsim_sparse_destroy": (_i32, [_vp]),
    "ncsim_sparse_clone": (_i32, [_vp, _P(_vp)]),
    "ncsim_sparse_set_cutoff": (_i32, [_vp, _dbl]),
    "ncsim_sparse_num_qubits": (_i32, [_vp, _P(_u32)]),
    "ncsim_sparse_num_entries": (_i32, [_vp, _P(_u64)]),
    "ncsim_sparse_get_entries": (_i32, [_vp, _P(_u64), _P(_dbl), _u64]),
    "ncsim_sparse_sort": (_i32, [_vp]),
    "ncsim_sparse_apply_gate": (_i32, [_vp, _vp, _P(_u32), _u32]),
    "ncsim_sparse_apply_pauli": (_i32, [_vp, _u64, _u64, _u32]),
    "ncsim_sparse_norm_sq": (_i32, [_vp, _P(_dbl)]),
    "ncsim_sparse_amplitude": (_i32, [_vp, _u64, _P(_dbl)]),
    "ncsim_sparse_expectation": (_i32, [_vp, _u64, _u64, _u32, _P(_dbl)]),
    "ncsim_sparse_inner": (_i32, [_vp, _vp, _P(_dbl)]),
    "ncsim_sparse_project": (_i32, [_vp, _u64, _u64, _u32, _i32, _P(_dbl)]),
    "ncsim_sparse_scale": (_i32, [_vp, _dbl, _dbl]),
    "ncsim_sparse_tensor": (_i32, [_vp, _vp, _P(_vp)]),
    "ncsim_sparse_sample": (_i32, [_vp, _vp, _u64, _P(_u64)]),
    "ncsim_sparse_to_vector": (_i32, [_vp, _P(_dbl), _u64]),
    "ncsim_sparse_measure": (_i32, [_vp, _u64, _u64, _u32, _vp, _P(_i32)]),
    "ncsim_sparse_run": (_i32, [_vp, _vp, _vp, _P(C.c_uint8), C.c_size_t, _P(C.c_size_t)]),
    "ncsim_sparse_synchronize": (_i32, [_vp]),
    "ncsim_sparse_timer_start": (_i32, [_vp]),
    "ncsim_sparse_timer_stop": (_i32, [_vp, _P(_dbl)]),
    "ncsim_sparse_num_words": (_i32, [_vp, _P(_u32)]),
    "ncsim_sparse_apply_pauli_words": (_i32, [_vp, _P(_u64), _P(_u64), _u32, _u32]),
    "ncsim_sparse_amplitude_words": (_i32, [_vp, _P(_u64), _u32, _P(_dbl)]),
    "ncsim_sparse_expectation_words": (_i32, [_vp, _P(_u64), _P(_u64), _u32, _u32, _P(_dbl)]),
    "ncsim_sparse_project_words": (_i32, [_vp, _P(_u64), _P(_u64), _u32, _u32, _i32, _P(_dbl)]),
    "ncsim_sparse_measure_words": (_i32, [_vp, _P(_u64), _P(_u64), _u32, _u32, _vp, _P(_i32)]),
    "ncsim_sv_set_tile_passes": (_i32, [_vp, _i32]),
    "ncsim_frames_new": (_i32, [_vp, _u64, _P(_vp)]),
    "ncsim_frames_with_reference": (_i32, [_vp, _P(C.c_uint8), _u64, _P(_vp)]),
    "ncsim_frames_free": (_i32, [_vp]),
    "ncsim_frames_info": (_i32, [_vp, _P(_u32), _P(_u64), _P(_u64), _P(_u64), _P(_u64)]),
    "ncsim_frames_reference": (_i32, [_vp, _P(C.c_uint8), _u64]),
    "ncsim_frames_sample_packed": (_i32, [_vp, _u64, _vp, _P(_u64), _u64]),
    "ncsim_frames_sample_packed_seeds": (_i32, [_vp, _u64, _P(_u64), _u64, _P(_u64), _u64]),
    "ncsim_frames_sample_packed_device": (_i32, [_vp, _u64, _P(_u64), _u64, _vp, _u64]),
    "ncsim_frames_sample": (_i32, [_vp, _u64, _vp, _P(_u64), _u64]),
    "ncsim_frames_sample_detectors": (_i32, [_vp, _u64, _vp, _P(_u64), _u64, _P(_u64), _u64]),
    "ncsim_frames_sample_detectors_seeds": (_i32, [_vp, _u64, _P(_u64), _u64, _P(_u64), _u64, _P(_u64), _u64]),
    "ncsim_frames_last_kernel_ms": (_i32, [_vp, _P(_dbl)]),
}


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", _u64), ("milliseconds", _dbl), ("bytes", _dbl)]


def lib():
    """The loaded C library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m ncsim_b200.build` "
                "(there is no CPU fallback)"
            )
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


# the seeded synthetic workloads (libncsim_workloads.so, include/ncsim_workloads.h)
_WORKLOAD_SIGNATURES = {
    "ncsim_workload_random_circuit": (_i32, [_u32, _u32, _u64, _dbl, _u32, _u32, _P(_vp)]),
    "ncsim_workload_random_circuit_rng": (_i32, [_vp, _u32, _u32, _dbl, _u32, _u32, _P(_vp)]),
    "ncsim_workload_reversible_circuit": (_i32, [_u32, _u32, _u64, _P(_vp)]),
    "ncsim_workload_frames_circuit": (_i32, [_u32, _u32, _u32, _dbl, _u64, _P(_vp)]),
    "ncsim_batch_random_layers": (_i32, [_u32, _u64, _u32, _u32, _u32, _dbl, _P(_vp)]),
}


def workloads_lib():
    """The workloads library (seeded synthetic circuits of the benchmark and the tests)."""
    global _wlib
    if _wlib is None:
        lib()  # the engine first: the workloads library resolves its symbols from it
        if not os.path.exists(WORKLOADS_PATH):
            raise ImportError(f"{WORKLOADS_PATH} is missing: build it with `python -m ncsim_b200.build`")
        L = C.CDLL(WORKLOADS_PATH)
        for name, (res, args) in _WORKLOAD_SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _wlib = L
    return _wlib


def _check(status: int) -> None:
    if status != 0:
        msg = lib().ncsim_last_error().decode(errors="replace")
        info = ErrorInfo()
        lib().ncsim_last_error_info(C.byref(info))
        fields = {}
        if status == 2:
            fields = {"qubit": info.qubit, "num_qubits": info.num_qubits}
        elif status == 4:
            fields = {"qubit": info.qubit}
        elif status == 3:
            fields = {"gate": info.gate.decode(errors="replace"), "expected": info.expected, "got": info.got}
        raise SimError(status, msg, fields)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_P(_dbl))


def _u32s(v: Sequence[int]):
    return (_u32 * max(1, len(v)))(*v)


# ---------------------------------------------------------------------------
# Paulis: (x, z, phase) with P = i^phase X^x Z^z (src/pauli/ops.rs:5)
# ---------------------------------------------------------------------------
class Pauli:
    """A Pauli operator on ``n`` qubits in ncsim's stored form."""

    __slots__ = ("n", "x", "z", "phase")

    def __init__(self, n: int, x: int = 0, z: int = 0, phase: int = 0):
        self.n, self.x, self.z, self.phase = n, x, z, phase & 3

    @classmethod
    def from_string(cls, n: int, text: str) -> "Pauli":
        """``Pauli::from_string`` (src/pauli/mod.rs:349-351); x and z are Python
        integers of n bits, so registers wider than 64 qubits work too."""
        if n > 64:
            words = (n + 63) // 64
            xw, zw, ph = (_u64 * words)(), (_u64 * words)(), _u32()
            _check(lib().ncsim_pauli_parse_words(text.encode(), n, xw, zw, words, C.byref(ph)))
            return cls(n, words_to_int(xw), words_to_int(zw), ph.value)
        x, z, ph = _u64(), _u64(), _u32()
        _check(lib().ncsim_pauli_parse(text.encode(), n, C.byref(x), C.byref(z), C.byref(ph)))
        return cls(n, x.value, z.value, ph.value)

    @classmethod
    def z_on(cls, n: int, q: int) -> "Pauli":
        return cls(n, 0, 1 << q, 0)

    def is_hermitian(self) -> bool:
        return ((self.phase & 1) == 1) == (bin(self.x & self.z).count("1") & 1 == 1)

    def __repr__(self) -> str:
        return f"Pauli(n={self.n}, x={self.x:#x}, z={self.z:#x}, phase={self.phase})"


def int_to_words(v: int, words: int):
    """A basis index or Pauli mask as `words` little-endian 64-bit words (ncsim's Bits)."""
    return (_u64 * words)(*[(v >> (64 * w)) & 0xFFFFFFFFFFFFFFFF for w in range(words)])


def words_to_int(ws) -> int:
    return sum(int(w) << (64 * i) for i, w in enumerate(ws))


# ---------------------------------------------------------------------------
class StdRng:
    """rand 0.8 ``StdRng`` seeded with ``seed_from_u64`` (C++ in the library)."""

    def __init__(self, seed: int):
        h = _vp()
        _check(lib().ncsim_rng_new(seed, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_rng_free(h)

    def next_u64(self) -> int:
        v = _u64()
        _check(lib().ncsim_rng_next_u64(self._h, C.byref(v)))
        return v.value

    def next_u32(self) -> int:
        v = _u32()
        _check(lib().ncsim_rng_next_u32(self._h, C.byref(v)))
        return v.value

    def gen_f64(self) -> float:
        v = _dbl()
        _check(lib().ncsim_rng_gen_f64(self._h, C.byref(v)))
        return v.value

    def gen_range(self, lo: int, hi: int) -> int:
        v = _u64()
        _check(lib().ncsim_rng_gen_range(self._h, lo, hi, C.byref(v)))
        return v.value


class Gate:
    """A gate (``src/gate.rs:356-431``): a text token, a dense unitary or a Pauli."""

    def __init__(self, handle, arity: int, label: str):
        self._h, self.arity, self.label = handle, arity, label

    @classmethod
    def parse(cls, token: str, arity: int = 0) -> "Gate":
        """A gate from its circuit-text token: ``H``, ``RZ(0.5)``, ``CCZ``, ``DIAG(...)``.

        ``arity`` is the qubit count of DIAG/MONOMIAL tokens (other gates know theirs).
        """
        h, k = _vp(), _u32()
        _check(lib().ncsim_gate_parse(token.encode(), arity, C.byref(h), C.byref(k)))
        return cls(h, k.value, token)

    @classmethod
    def unitary(cls, m: np.ndarray) -> "Gate":
        """``Gate::Unitary``: a dense 2^k x 2^k matrix, row-major, little-endian."""
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128))
        k = int(round(np.log2(m.shape[0])))
        h = _vp()
        _check(lib().ncsim_gate_unitary(k, _dp(m.view(np.float64)), C.byref(h)))
        return cls(h, k, f"UNITARY[{k}]")

    @classmethod
    def pauli(cls, p: Pauli) -> "Gate":
        """``Gate::Pauli`` on ``p.n`` local qubits."""
        h = _vp()
        _check(lib().ncsim_gate_pauli(p.n, p.x, p.z, p.phase, C.byref(h)))
        return cls(h, p.n, "PAULI")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_gate_free(h)

    def lowered_matrix(self) -> np.ndarray:
        """The dense matrix the engine's lowering applies (host only)."""
        d = 1 << self.arity
        buf = np.zeros(2 * d * d, dtype=np.float64)
        k = _u32()
        _check(lib().ncsim_gate_lowered_matrix(self._h, _dp(buf), buf.size, C.byref(k)))
        return buf.view(np.complex128).reshape(d, d)

    def __repr__(self) -> str:
        return f"Gate({self.label})"


class Circuit:
    """``Circuit`` (src/circuit.rs:151): parsed from ncsim's text format."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def parse(cls, text: str) -> "Circuit":
        h = _vp()
        _check(lib().ncsim_circuit_parse(text.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def random_layers(cls, n: int, depth: int, seed: int, noise_p: float = 0.0, m_lo: int = 0, m_hi: int = 0):
        """The seeded random layer family (H/S/T/SQRT_X/RZ on every qubit, CZ matching)."""
        h = _vp()
        _check(workloads_lib().ncsim_workload_random_circuit(n, depth, seed, noise_p, m_lo, m_hi, C.byref(h)))
        return cls(h)

    @classmethod
    def random_layers_from(cls, rng: "StdRng", n: int, depth: int, noise_p: float = 0.0, m_lo: int = 0, m_hi: int = 0):
        """The random layer family drawn from ``rng``, which keeps its state."""
        h = _vp()
        _check(workloads_lib().ncsim_workload_random_circuit_rng(rng._h, n, depth, noise_p, m_lo, m_hi, C.byref(h)))
        return cls(h)

    @classmethod
    def frames_workload(cls, n: int = 1000, rounds: int = 20, meas: int = 100, p: float = 1e-3,
                        seed: int = 9) -> "Circuit":
        """The reference's frame-sampler benchmark circuit (examples/bench.rs:264-294)."""
        h = _vp()
        _check(workloads_lib().ncsim_workload_frames_circuit(n, rounds, meas, p, seed, C.byref(h)))
        return cls(h)

    @classmethod
    def reversible(cls, n: int, gates: int, seed: int) -> "Circuit":
        """The seeded permutation/diagonal family (CX, CCX, CCZ, DIAG, MONOMIAL)."""
        h = _vp()
        _check(workloads_lib().ncsim_workload_reversible_circuit(n, gates, seed, C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_circuit_free(h)

    def _info(self):
        nq, no, ng, nm = _u32(), _u64(), _u64(), _u64()
        _check(lib().ncsim_circuit_info(self._h, C.byref(nq), C.byref(no), C.byref(ng), C.byref(nm)))
        return nq.value, no.value, ng.value, nm.value

    @property
    def num_qubits(self) -> int:
        return self._info()[0]

    @property
    def num_gates(self) -> int:
        return self._info()[2]

    @property
    def num_measurements(self) -> int:
        return self._info()[3]

    def fused_emulate(self, amps: np.ndarray, max_fuse: int = 5):
        """The fused form's plan applied on the host in FP64 (planner check)."""
        b = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128)).copy().view(np.float64)
        st = FusedStats()
        _check(lib().ncsim_fused_emulate(self._h, max_fuse, _dp(b), b.size // 2, C.byref(st)))
        return b.view(np.complex128), st

    def to_text(self) -> str:
        n = C.c_size_t()
        _check(lib().ncsim_circuit_to_text(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value + 1)
        _check(lib().ncsim_circuit_to_text(self._h, buf, n.value + 1, C.byref(n)))
        return buf.value.decode()


class FusedStats(C.Structure):
    _fields_ = [
        ("source_gates", _u64),
        ("fused_unitaries", _u64),
        ("passes", _u64),
        ("remap_passes", _u64),
        ("gemm_launches", _u64),
        ("diagonal_terms", _u64),
    ]


def _complex(buf) -> complex:
    return complex(buf[0], buf[1])


class GpuStateVector:
    """A dense state vector in B200 memory: the drop-in for ``StateVector<C64>``.

    ``precision`` is ``C128`` (complex128, the drop-in) or ``C64`` (complex64,
    the storage of the fused precision form).
    """

    BACKEND = "GpuStateVector"

    def __init__(self, n: int, precision: int = C128, _handle=None):
        if _handle is None:
            h = _vp()
            _check(lib().ncsim_sv_create(n, precision, C.byref(h)))
            _handle = h
        self._h = _handle
        self.n = n
        self.precision = precision

    # ---- constructors (vector.rs:25-52) ----
    @classmethod
    def zero_state(cls, n: int, precision: int = C128) -> "GpuStateVector":
        return cls(n, precision)

    @classmethod
    def basis_state(cls, n: int, index: int, precision: int = C128) -> "GpuStateVector":
        s = cls(n, precision)
        _check(lib().ncsim_sv_set_basis(s._h, index))
        return s

    @classmethod
    def plus_state(cls, n: int, precision: int = C128) -> "GpuStateVector":
        s = cls(n, precision)
        _check(lib().ncsim_sv_set_plus(s._h))
        return s

    @classmethod
    def from_amplitudes(cls, amps: np.ndarray, precision: int = C128) -> "GpuStateVector":
        amps = np.asarray(amps, dtype=np.complex128)
        n = int(amps.size).bit_length() - 1
        if (1 << n) != amps.size:
            raise SimError(8, f"{amps.size} amplitudes for {n} qubits")
        s = cls(n, precision)
        s.set_amplitudes(amps)
        return s

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_sv_destroy(h)
            self._h = None

    def clone(self) -> "GpuStateVector":
        h = _vp()
        _check(lib().ncsim_sv_clone(self._h, C.byref(h)))
        return GpuStateVector(self.n, self.precision, h)

    def num_qubits(self) -> int:
        return self.n

    def set_amplitudes(self, amps: np.ndarray) -> None:
        b = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128)).view(np.float64)
        _check(lib().ncsim_sv_set_amplitudes(self._h, _dp(b), 1 << self.n))

    def device_pointer(self) -> tuple[int, int]:
        """(device address, bytes) of the amplitude array."""
        p, b = _vp(), _u64()
        _check(lib().ncsim_sv_device_pointer(self._h, C.byref(p), C.byref(b)))
        return int(p.value or 0), b.value

    def torch_view(self):
        """A torch tensor over the amplitude array, without a copy (complex128 or
        complex64, on this state's device).  The state's queued work must be
        finished (``synchronize``) before torch touches it, and torch's work
        before the state's next call."""
        import torch

        ptr, nbytes = self.device_pointer()
        dt = "<c16" if self.precision == C128 else "<c8"

        class _View:
            __cuda_array_interface__ = {"shape": (1 << self.n,), "typestr": dt, "data": (ptr, False),
                                        "version": 3, "strides": None}

        return torch.as_tensor(_View(), device="cuda")

    def block_weights(self, block: int = 4096) -> np.ndarray:
        """|a|^2 summed over each block of ``block`` consecutive amplitudes (FP64)."""
        nbl = (1 << self.n) // block
        out = np.empty(nbl)
        _check(lib().ncsim_sv_block_weights(self._h, block, _dp(out), nbl))
        return out

    def sample_walk(self, block: int, targets, blocks, accs) -> np.ndarray:
        """The in-block walk of one-pass sampling for the given shots (vector.rs:508-538)."""
        t = np.ascontiguousarray(targets, dtype=np.float64)
        b = np.ascontiguousarray(blocks, dtype=np.uint64)
        a = np.ascontiguousarray(accs, dtype=np.float64)
        out = np.empty(t.size, dtype=np.uint64)
        _check(lib().ncsim_sv_sample_walk(self._h, block, _dp(t), b.ctypes.data_as(_P(_u64)), _dp(a), t.size,
                                          out.ctypes.data_as(_P(_u64))))
        return out

    def set_basis(self, index: int) -> None:
        """The register becomes the basis state |index> (in place)."""
        _check(lib().ncsim_sv_set_basis(self._h, index))

    def to_vector(self) -> np.ndarray:
        """All amplitudes as complex128 (``to_vector``, vector.rs:542)."""
        b = np.empty(2 << self.n, dtype=np.float64)
        _check(lib().ncsim_sv_get_amplitudes(self._h, _dp(b), 1 << self.n))
        return b.view(np.complex128)

    def to_vector_range(self, first: int, count: int, out: np.ndarray | None = None) -> np.ndarray:
        """Amplitudes ``first .. first+count-1`` as complex128 (a slice of ``to_vector``)."""
        if out is None:
            out = np.empty(count, dtype=np.complex128)
        if out.dtype != np.complex128 or out.size < count or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous complex128 array of at least count elements")
        _check(lib().ncsim_sv_get_amplitudes_range(self._h, first, count, _dp(out.view(np.float64))))
        return out[:count]

    def amplitude(self, index: int) -> complex:
        o = (_dbl * 2)()
        _check(lib().ncsim_sv_get_amplitude(self._h, index, o))
        return _complex(o)

    def amplitudes_at(self, indices: Iterable[int]) -> np.ndarray:
        idx = np.ascontiguousarray(np.asarray(list(indices), dtype=np.uint64))
        out = np.empty(2 * idx.size, dtype=np.float64)
        _check(lib().ncsim_sv_gather_amplitudes(self._h, idx.ctypes.data_as(_P(_u64)), idx.size, _dp(out)))
        return out.view(np.complex128)

    # ---- gates ----
    def apply_gate(self, gate: Gate, qubits: Sequence[int]) -> None:
        """``apply_gate`` through the gate's views (vector.rs:364-395)."""
        _check(lib().ncsim_sv_apply_gate(self._h, gate._h, _u32s(qubits), len(qubits)))

    def apply_matrix(self, m: np.ndarray, qubits: Sequence[int]) -> None:
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128))
        _check(lib().ncsim_sv_apply_matrix(self._h, _u32s(qubits), len(qubits), _dp(m.view(np.float64))))

    def apply_monomial(self, qubits: Sequence[int], image: Sequence[int], phase: np.ndarray) -> None:
        img = np.ascontiguousarray(np.asarray(image, dtype=np.uint64))
        ph = np.ascontiguousarray(np.asarray(phase, dtype=np.complex128))
        _check(
            lib().ncsim_sv_apply_monomial(
                self._h, _u32s(qubits), len(qubits), img.ctypes.data_as(_P(_u64)), _dp(ph.view(np.float64))
            )
        )

    def apply_phasepoly(self, qubits, bits, constant, terms, scalar=(0, 0, 0)) -> None:
        """Diagonal(PhasePoly) from the bit index; ``terms`` = [(coeff, [parity masks])]."""
        starts, pars, coeffs = [0], [], []
        for c, ps in terms:
            pars.extend(ps)
            starts.append(len(pars))
            coeffs.append(c)
        st = (_u32 * len(starts))(*starts)
        pa = (_u64 * max(1, len(pars)))(*pars)
        co = (_u64 * max(1, len(coeffs)))(*coeffs)
        _check(
            lib().ncsim_sv_apply_phasepoly(
                self._h, _u32s(qubits), len(qubits), bits, constant, len(coeffs), st, pa, co, *scalar
            )
        )

    def apply_pauli(self, p: Pauli) -> None:
        _check(lib().ncsim_sv_apply_pauli(self._h, p.x, p.z, p.phase))

    # ---- readouts ----
    def norm_sq(self) -> complex:
        o = (_dbl * 2)()
        _check(lib().ncsim_sv_norm_sq(self._h, o))
        return _complex(o)

    def expectation(self, p: Pauli) -> complex:
        if p.n != self.n:
            raise SimError(8, "expectation: operator on the wrong register")
        o = (_dbl * 2)()
        _check(lib().ncsim_sv_expectation(self._h, p.x, p.z, p.phase, o))
        return _complex(o)

    def measure_stats(self, p: Pauli):
        e = (_dbl * 2)()
        nn = _dbl()
        _check(lib().ncsim_sv_measure_stats(self._h, p.x, p.z, p.phase, e, C.byref(nn)))
        return _complex(e), nn.value

    def expectation_sum(self, terms: Sequence[tuple[complex, Pauli]]) -> complex:
        k = len(terms)
        xs = (_u64 * max(1, k))(*[p.x for _, p in terms])
        zs = (_u64 * max(1, k))(*[p.z for _, p in terms])
        ph = (_u32 * max(1, k))(*[p.phase for _, p in terms])
        cs = np.array([[complex(c).real, complex(c).imag] for c, _ in terms] or [[0.0, 0.0]], dtype=np.float64)
        o = (_dbl * 2)()
        _check(lib().ncsim_sv_expectation_sum(self._h, k, xs, zs, ph, _dp(cs), o))
        return _complex(o)

    def inner(self, other: "GpuStateVector") -> complex:
        o = (_dbl * 2)()
        _check(lib().ncsim_sv_inner(self._h, other._h, o))
        return _complex(o)

    def project(self, p: Pauli, outcome: bool) -> complex:
        o = (_dbl * 2)()
        _check(lib().ncsim_sv_project(self._h, p.x, p.z, p.phase, int(bool(outcome)), o))
        return _complex(o)

    def scale(self, c: complex) -> None:
        c = complex(c)
        _check(lib().ncsim_sv_scale(self._h, c.real, c.imag))

    def normalize(self) -> None:
        _check(lib().ncsim_sv_normalize(self._h))

    def probability(self, index: int) -> float:
        o = _dbl()
        _check(lib().ncsim_sv_probability(self._h, index, C.byref(o)))
        return o.value

    def measure(self, p: Pauli, rng: StdRng) -> bool:
        o = _i32()
        _check(lib().ncsim_sv_measure(self._h, p.x, p.z, p.phase, rng._h, C.byref(o)))
        return bool(o.value)

    def run(self, circuit: Circuit, rng: StdRng) -> list[bool]:
        m = circuit.num_measurements
        rec = (C.c_uint8 * max(1, m))()
        ln = C.c_size_t()
        _check(lib().ncsim_sv_run(self._h, circuit._h, rng._h, rec, m, C.byref(ln)))
        return [bool(rec[i]) for i in range(ln.value)]

    def run_fused(self, circuit: Circuit, rng: StdRng, max_fuse: int = 5):
        m = circuit.num_measurements
        rec = (C.c_uint8 * max(1, m))()
        ln = C.c_size_t()
        st = FusedStats()
        _check(lib().ncsim_sv_run_fused(self._h, circuit._h, rng._h, max_fuse, rec, m, C.byref(ln), C.byref(st)))
        return [bool(rec[i]) for i in range(ln.value)], st

    def sample(self, rng: StdRng, shots: int) -> np.ndarray:
        out = np.empty(shots, dtype=np.uint64)
        _check(lib().ncsim_sv_sample_rng(self._h, rng._h, shots, out.ctypes.data_as(_P(_u64))))
        return out

    def sample_uniforms(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty(u.size, dtype=np.uint64)
        _check(lib().ncsim_sv_sample(self._h, _dp(u), u.size, out.ctypes.data_as(_P(_u64))))
        return out

    def tensor(self, other: "GpuStateVector") -> "GpuStateVector":
        h = _vp()
        _check(lib().ncsim_sv_kron(self._h, other._h, C.byref(h)))
        return GpuStateVector(self.n + other.n, self.precision, h)

    kron = tensor

    def synchronize(self) -> None:
        _check(lib().ncsim_sv_synchronize(self._h))

    def timer_start(self) -> None:
        """Records a start event on the state's stream."""
        _check(lib().ncsim_sv_timer_start(self._h))

    def timer_stop(self) -> float:
        """Device milliseconds since timer_start (waits for the stream)."""
        ms = _dbl()
        _check(lib().ncsim_sv_timer_stop(self._h, C.byref(ms)))
        return ms.value

    def compare(self, other: "GpuStateVector") -> dict:
        """<a|b>, norms, infidelity and max amplitude difference, in one FP64 pass."""
        inner = (_dbl * 2)()
        na, nb_, mx = _dbl(), _dbl(), _dbl()
        _check(lib().ncsim_sv_compare(self._h, other._h, inner, C.byref(na), C.byref(nb_), C.byref(mx)))
        ip = _complex(inner)
        return {
            "inner": ip,
            "norm_a": na.value,
            "norm_b": nb_.value,
            "infidelity": 1.0 - abs(ip) ** 2 / (na.value * nb_.value),
            "max_abs_diff": mx.value,
        }

    # ---- launch profiler (CUDA events on the state's stream) ----
    def set_tile_passes(self, enable: bool = True) -> None:
        """Runs of gates through tiled passes (default) or gate by gate."""
        _check(lib().ncsim_sv_set_tile_passes(self._h, int(enable)))

    def profile(self, enable: bool = True) -> None:
        """Start (clearing earlier records) or stop per-launch event timing."""
        _check(lib().ncsim_sv_profile_enable(self._h, int(enable)))

    def profile_read(self) -> dict:
        """{kernel class: {"launches", "ms", "bytes"}} since profiling was enabled."""
        arr = (KernelStat * 32)()
        cnt = _u32()
        _check(lib().ncsim_sv_profile_read(self._h, C.cast(arr, _vp), 32, C.byref(cnt)))
        return {
            arr[i].name.decode(): {"launches": arr[i].launches, "ms": arr[i].milliseconds, "bytes": arr[i].bytes}
            for i in range(min(cnt.value, 32))
        }


# ---------------------------------------------------------------------------
# batching form: many noisy trajectories in one persistent kernel
# ---------------------------------------------------------------------------
class BatchStats(C.Structure):
    _fields_ = [
        ("trajectories", _u64),
        ("source_gates", _u64),
        ("noise_events", _u64),
        ("folded_ops", _u64),
        ("passes", _u64),
        ("tile_passes", _u64),
        ("tile_stages", _u64),
        ("state_bytes", _dbl),
        ("program_bytes", _u64),
        ("max_qubits", _u32),
    ]


class BatchConfig(C.Structure):
    _fields_ = [("ctas_per_sm", _u32), ("buffers", _u32), ("order", _u32)]

    def as_dict(self) -> dict:
        return {"ctas_per_sm": self.ctas_per_sm, "buffers": self.buffers,
                "order": "largest_first" if self.order == 0 else "given"}


class BatchKnobs(C.Structure):
    _fields_ = [("knob_set", C.c_uint32), ("window_step", C.c_uint32), ("greedy_windows", C.c_uint32),
                ("greedy_stages", C.c_uint32), ("final_", C.c_uint32), ("timed_ms", C.c_double * 4)]


class TrajectoryBatch:
    """Independent noisy trajectories, each ``QuantumState::run`` of its circuit
    with its own ``StdRng`` (src/state/mod.rs:168-183), run together on the GPU.

    ``results()`` gives per trajectory the register size, the record (bit k =
    outcome of ``M k``), <Z0>/<psi|psi> just before the measurements and
    <psi|psi> there."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def random_layers(cls, count: int, seed0: int = 1, n_lo: int = 16, n_span: int = 7, depth: int = 30,
                      p: float = 1e-3) -> "TrajectoryBatch":
        """Trajectory t: StdRng(seed0 + t), n = n_lo + gen_range(0..n_span), the random
        layer circuit with DEPOLARIZE2(p) after every CZ and M on every qubit."""
        h = _vp()
        _check(workloads_lib().ncsim_batch_random_layers(count, seed0, n_lo, n_span, depth, p, C.byref(h)))
        return cls(h)

    @classmethod
    def from_circuits(cls, circuits: Sequence[Circuit], seeds: Sequence[int]) -> "TrajectoryBatch":
        if len(circuits) != len(seeds):
            raise ValueError("one seed per circuit")
        hs = (_vp * len(circuits))(*[c._h for c in circuits])
        sd = (_u64 * len(seeds))(*seeds)
        h = _vp()
        _check(lib().ncsim_batch_from_circuits(len(circuits), hs, sd, C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_batch_free(h)

    def release(self) -> None:
        """Gives back the batch's device memory, stream and graph; the next run
        sets them up again on the then-current device."""
        _check(lib().ncsim_batch_release(self._h))

    def knobs(self, n: int) -> dict:
        """The planner's knobs for registers of n qubits (and what each candidate took)."""
        k = BatchKnobs()
        _check(lib().ncsim_batch_knobs(self._h, n, C.byref(k)))
        return {"knob_set": k.knob_set, "window_step": k.window_step, "greedy_windows": bool(k.greedy_windows),
                "greedy_stages": bool(k.greedy_stages), "final": bool(k.final_), "timed_ms": list(k.timed_ms)}

    def set_knob_set(self, n: int, knob_set: int, final: bool = False) -> None:
        _check(lib().ncsim_batch_set_knob_set(self._h, n, knob_set, int(final)))

    def info(self) -> dict:
        st = BatchStats()
        _check(lib().ncsim_batch_info(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in BatchStats._fields_}

    def __len__(self) -> int:
        return int(self.info()["trajectories"])

    def qubits(self) -> np.ndarray:
        n = np.empty(len(self), dtype=np.uint32)
        _check(lib().ncsim_batch_trajectory_qubits(self._h, n.ctypes.data_as(_P(_u32))))
        return n

    def set_config(self, ctas_per_sm: int = 1, buffers: int = 2, order: str = "largest_first") -> None:
        cfg = BatchConfig(ctas_per_sm, buffers, 0 if order == "largest_first" else 1)
        _check(lib().ncsim_batch_set_config(self._h, C.byref(cfg)))

    def config(self) -> dict:
        cfg = BatchConfig()
        _check(lib().ncsim_batch_get_config(self._h, C.byref(cfg)))
        return cfg.as_dict()

    def tune(self, sample: int = 0) -> dict:
        cfg = BatchConfig()
        _check(lib().ncsim_batch_tune(self._h, sample, C.byref(cfg)))
        return cfg.as_dict()

    def run(self) -> float:
        """Runs every trajectory; returns the kernel's device milliseconds."""
        ms = _dbl()
        _check(lib().ncsim_batch_run(self._h, C.byref(ms)))
        return ms.value

    def results(self):
        c = len(self)
        n = np.empty(c, dtype=np.uint32)
        rec = np.empty(c, dtype=np.uint64)
        z0 = np.empty(c)
        nn = np.empty(c)
        _check(lib().ncsim_batch_results(self._h, n.ctypes.data_as(_P(_u32)), rec.ctypes.data_as(_P(_u64)),
                                         _dp(z0), _dp(nn)))
        return n, rec, z0, nn

    def emulate(self, t: int):
        """Host FP64 run of trajectory t's device program (tests): (record, z0, norm)."""
        r, z, nn = _u64(), _dbl(), _dbl()
        _check(lib().ncsim_batch_emulate(self._h, t, C.byref(r), C.byref(z), C.byref(nn)))
        return r.value, z.value, nn.value


class GpuSparseVector:
    """The nonzero amplitudes of a register of up to 1024 qubits in B200 memory:
    the drop-in for ``SparseVector<C64>`` (``src/state/sparse.rs``).

    Basis indices are Python integers; on the device they are ``words`` 64-bit
    words (1 up to 64 qubits, 4 up to 256, 16 up to 1024), ordered as ncsim's
    ``Bits`` (``Vec<u64>``) order them.

    Entries are (basis index, complex128) pairs.  Gates that move each entry to
    one entry (monomials, permutations with phases, Paulis, diagonals) keep the
    entry order; dense gates and projections sort, sum duplicates and drop
    zeros, as the reference does.
    """

    BACKEND = "GpuSparseVector"

    def __init__(self, n: int, _handle=None):
        if _handle is None:
            h = _vp()
            _check(lib().ncsim_sparse_create(n, C.byref(h)))
            _handle = h
        self._h = _handle
        self.n = n
        w = _u32()
        _check(lib().ncsim_sparse_num_words(self._h, C.byref(w)))
        self.words = w.value

    def _w(self, v: int):
        return int_to_words(v, self.words)

    @classmethod
    def zero_state(cls, n: int) -> "GpuSparseVector":
        return cls(n)

    @classmethod
    def from_entries(cls, n: int, keys: Sequence[int], amps: Sequence[complex]) -> "GpuSparseVector":
        """``SparseVector::from_entries`` (sparse.rs:54-72): duplicates are added."""
        words = 1 if n <= 64 else 4 if n <= 256 else 16
        if words == 1:
            k = np.ascontiguousarray(np.asarray(list(keys), dtype=np.uint64))
        else:
            ks = [int(v) for v in keys]
            k = np.zeros((len(ks), words), dtype=np.uint64)
            for i, v in enumerate(ks):
                for w in range(words):
                    k[i, w] = (v >> (64 * w)) & 0xFFFFFFFFFFFFFFFF
        a = np.ascontiguousarray(np.asarray(list(amps), dtype=np.complex128))
        h = _vp()
        _check(lib().ncsim_sparse_from_entries(n, k.ctypes.data_as(_P(_u64)), _dp(a.view(np.float64)), a.size,
                                               C.byref(h)))
        return cls(n, h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_sparse_destroy(h)
            self._h = None

    def clone(self) -> "GpuSparseVector":
        h = _vp()
        _check(lib().ncsim_sparse_clone(self._h, C.byref(h)))
        return GpuSparseVector(self.n, h)

    def with_cutoff(self, cutoff: float) -> "GpuSparseVector":
        _check(lib().ncsim_sparse_set_cutoff(self._h, cutoff))
        return self

    def num_qubits(self) -> int:
        return self.n

    def num_entries(self) -> int:
        m = _u64()
        _check(lib().ncsim_sparse_num_entries(self._h, C.byref(m)))
        return m.value

    def entries(self):
        """(indices, amplitudes) in the current entry order: indices as a uint64
        array (one word per entry) up to 64 qubits, as Python integers beyond."""
        m = self.num_entries()
        k = np.empty((m, self.words), dtype=np.uint64)
        a = np.empty(2 * m, dtype=np.float64)
        _check(lib().ncsim_sparse_get_entries(self._h, k.ctypes.data_as(_P(_u64)), _dp(a), m))
        if self.words == 1:
            return k[:, 0].copy(), a.view(np.complex128)
        return [words_to_int(row) for row in k], a.view(np.complex128)

    def sort(self) -> None:
        _check(lib().ncsim_sparse_sort(self._h))

    def apply_gate(self, gate: Gate, qubits: Sequence[int]) -> None:
        _check(lib().ncsim_sparse_apply_gate(self._h, gate._h, _u32s(qubits), len(qubits)))

    def apply_pauli(self, p: Pauli) -> None:
        if self.words > 1:
            _check(lib().ncsim_sparse_apply_pauli_words(self._h, self._w(p.x), self._w(p.z), self.words, p.phase))
            return
        _check(lib().ncsim_sparse_apply_pauli(self._h, p.x, p.z, p.phase))

    def norm_sq(self) -> complex:
        o = (_dbl * 2)()
        _check(lib().ncsim_sparse_norm_sq(self._h, o))
        return _complex(o)

    def amplitude(self, index: int) -> complex:
        o = (_dbl * 2)()
        if self.words > 1:
            _check(lib().ncsim_sparse_amplitude_words(self._h, self._w(index), self.words, o))
        else:
            _check(lib().ncsim_sparse_amplitude(self._h, index, o))
        return _complex(o)

    def expectation(self, p: Pauli) -> complex:
        if p.n != self.n:
            raise SimError(8, "expectation: operator on the wrong register")
        o = (_dbl * 2)()
        if self.words > 1:
            _check(lib().ncsim_sparse_expectation_words(self._h, self._w(p.x), self._w(p.z), self.words, p.phase, o))
        else:
            _check(lib().ncsim_sparse_expectation(self._h, p.x, p.z, p.phase, o))
        return _complex(o)

    def inner(self, other: "GpuSparseVector") -> complex:
        o = (_dbl * 2)()
        _check(lib().ncsim_sparse_inner(self._h, other._h, o))
        return _complex(o)

    def project(self, p: Pauli, outcome: bool) -> complex:
        o = (_dbl * 2)()
        if self.words > 1:
            _check(lib().ncsim_sparse_project_words(self._h, self._w(p.x), self._w(p.z), self.words, p.phase,
                                                    int(bool(outcome)), o))
        else:
            _check(lib().ncsim_sparse_project(self._h, p.x, p.z, p.phase, int(bool(outcome)), o))
        return _complex(o)

    def scale(self, c: complex) -> None:
        c = complex(c)
        _check(lib().ncsim_sparse_scale(self._h, c.real, c.imag))

    def tensor(self, other: "GpuSparseVector") -> "GpuSparseVector":
        h = _vp()
        _check(lib().ncsim_sparse_tensor(self._h, other._h, C.byref(h)))
        return GpuSparseVector(self.n + other.n, h)

    def sample(self, rng: StdRng, shots: int):
        """Shots as a uint64 array up to 64 qubits, as Python integers beyond."""
        out = np.empty((shots, self.words), dtype=np.uint64)
        _check(lib().ncsim_sparse_sample(self._h, rng._h, shots, out.ctypes.data_as(_P(_u64))))
        if self.words == 1:
            return out[:, 0].copy()
        return [words_to_int(row) for row in out]

    def to_vector(self) -> np.ndarray:
        b = np.empty(2 << self.n, dtype=np.float64)
        _check(lib().ncsim_sparse_to_vector(self._h, _dp(b), 1 << self.n))
        return b.view(np.complex128)

    def measure(self, p: Pauli, rng: StdRng) -> bool:
        o = _i32()
        if self.words > 1:
            _check(lib().ncsim_sparse_measure_words(self._h, self._w(p.x), self._w(p.z), self.words, p.phase, rng._h,
                                                    C.byref(o)))
        else:
            _check(lib().ncsim_sparse_measure(self._h, p.x, p.z, p.phase, rng._h, C.byref(o)))
        return bool(o.value)

    def run(self, circuit: Circuit, rng: StdRng) -> list[bool]:
        m = circuit.num_measurements
        rec = (C.c_uint8 * max(1, m))()
        ln = C.c_size_t()
        _check(lib().ncsim_sparse_run(self._h, circuit._h, rng._h, rec, m, C.byref(ln)))
        return [bool(rec[i]) for i in range(ln.value)]

    def synchronize(self) -> None:
        _check(lib().ncsim_sparse_synchronize(self._h))

    def timer_start(self) -> None:
        _check(lib().ncsim_sparse_timer_start(self._h))

    def timer_stop(self) -> float:
        ms = _dbl()
        _check(lib().ncsim_sparse_timer_stop(self._h, C.byref(ms)))
        return ms.value


class FrameSampler:
    """Bulk sampler of a noisy Clifford circuit by Pauli frames on the GPU: the
    drop-in for ncsim's ``FrameSampler`` (``src/frame.rs:34-300``).

    Records come packed as the reference returns them: row k of the
    ``(measurements, ceil(shots / 64))`` uint64 array holds measurement k over
    the shots (bit s of word s // 64 = shot s).  Shots run in batches of 16384,
    each seeded by one ``next_u64`` of the caller's generator.
    """

    BATCH = 1 << 14

    def __init__(self, circuit: Circuit, reference_seed: int = 0, reference: Sequence[int] | None = None):
        h = _vp()
        if reference is None:
            _check(lib().ncsim_frames_new(circuit._h, reference_seed, C.byref(h)))
        else:
            r = np.ascontiguousarray(np.asarray(list(reference), dtype=np.uint8))
            _check(lib().ncsim_frames_with_reference(circuit._h, r.ctypes.data_as(_P(C.c_uint8)), r.size, C.byref(h)))
        self._h = h
        n, m, d, o, layers = _u32(), _u64(), _u64(), _u64(), _u64()
        _check(lib().ncsim_frames_info(h, C.byref(n), C.byref(m), C.byref(d), C.byref(o), C.byref(layers)))
        self.n, self.m = n.value, m.value
        self.num_detectors, self.num_observables, self.num_layers = d.value, o.value, layers.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ncsim_frames_free(h)
            self._h = None

    def reference(self) -> list[bool]:
        """``FrameSampler::reference`` (frame.rs:66-68): the noiseless record."""
        r = np.zeros(max(self.m, 1), dtype=np.uint8)
        _check(lib().ncsim_frames_reference(self._h, r.ctypes.data_as(_P(C.c_uint8)), r.size))
        return [bool(v) for v in r[: self.m]]

    @staticmethod
    def words(shots: int) -> int:
        return (shots + 63) // 64

    def sample_packed(self, shots: int, rng: StdRng) -> np.ndarray:
        """``sample_packed`` (frame.rs:69-89): (measurements, words) uint64."""
        out = np.zeros((self.m, self.words(shots)), dtype=np.uint64)
        _check(lib().ncsim_frames_sample_packed(self._h, shots, rng._h, out.ctypes.data_as(_P(_u64)), out.size))
        return out

    def sample_packed_seeds(self, shots: int, seeds: Sequence[int], out: np.ndarray | None = None) -> np.ndarray:
        """The same with the per-batch seeds given (one per 16384 shots)."""
        sd = np.ascontiguousarray(np.asarray(list(seeds), dtype=np.uint64))
        if out is None:
            out = np.zeros((self.m, self.words(shots)), dtype=np.uint64)
        _check(lib().ncsim_frames_sample_packed_seeds(self._h, shots, sd.ctypes.data_as(_P(_u64)), sd.size,
                                                      out.ctypes.data_as(_P(_u64)), out.size))
        return out

    def sample_packed_device(self, shots: int, seeds: Sequence[int], d_out: int, cap_words: int) -> None:
        """The same into device memory (``d_out``: a device pointer of ``cap_words`` words)."""
        sd = np.ascontiguousarray(np.asarray(list(seeds), dtype=np.uint64))
        _check(lib().ncsim_frames_sample_packed_device(self._h, shots, sd.ctypes.data_as(_P(_u64)), sd.size,
                                                       _vp(d_out), cap_words))

    def sample(self, shots: int, rng: StdRng) -> np.ndarray:
        """``sample`` (frame.rs:90-102): (shots, ceil(m / 64)) uint64, bit k = measurement k."""
        mw = (self.m + 63) // 64
        out = np.zeros((shots, mw), dtype=np.uint64)
        _check(lib().ncsim_frames_sample(self._h, shots, rng._h, out.ctypes.data_as(_P(_u64)), out.size))
        return out

    def sample_detectors(self, shots: int, rng: StdRng):
        """``sample_detectors`` (frame.rs:155-205): packed detector and observable flips."""
        w = self.words(shots)
        det = np.zeros((self.num_detectors, w), dtype=np.uint64)
        obs = np.zeros((self.num_observables, w), dtype=np.uint64)
        _check(lib().ncsim_frames_sample_detectors(self._h, shots, rng._h, det.ctypes.data_as(_P(_u64)), det.size,
                                                   obs.ctypes.data_as(_P(_u64)), obs.size))
        return det, obs

    def last_kernel_ms(self) -> float:
        """Device time of the last call's mask and frame kernels."""
        ms = _dbl()
        _check(lib().ncsim_frames_last_kernel_ms(self._h, C.byref(ms)))
        return ms.value


def packed_bit(packed: np.ndarray, k: int, s: int) -> bool:
    """Bit s of packed row k (``bits::get``)."""
    return bool((int(packed[k, s // 64]) >> (s % 64)) & 1)


def device_info() -> dict:
    sm, fr, tot = _i32(), _u64(), _u64()
    _check(lib().ncsim_device_info(C.byref(sm), C.byref(fr), C.byref(tot)))
    return {"sm_count": sm.value, "free_bytes": fr.value, "total_bytes": tot.value}


def trim_memory() -> None:
    """Gives the memory kept by the library's per-device pools back to the device."""
    _check(lib().ncsim_trim_memory())


def pool_info() -> dict:
    """Bytes the current device's library pool holds, and bytes of it in use."""
    r, u = _u64(), _u64()
    _check(lib().ncsim_pool_info(C.byref(r), C.byref(u)))
    return {"reserved_bytes": r.value, "used_bytes": u.value}
