"""The fused precision form on the device (complex64 amplitudes, BF16x3
tensor-core products with FP32 accumulation) against the FP64 oracle.

Bar: infidelity 1 - |<psi64|psi32>|^2 / (<psi64|psi64><psi32|psi32>) at most
1e-6 and every amplitude of a unit-norm register within 2e-5 of the FP64
result; measurement records identical to the complex128 plain path for the
same seed (no outcome probability is within 1e-5 of its draw here).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

INFIDELITY = 1e-6
AMP_TOL = 2e-5


def _fidelity(a, b):
    ip = np.vdot(a, b)
    return 1 - abs(ip) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


@pytest.mark.parametrize("n,depth,seed", [(12, 4, 1), (14, 10, 2), (18, 20, 3)])
def test_fused_random_layers_match_fp64(nb, oracle, n, depth, seed):
    text = oracle.random_circuit_text(n, depth, seed)
    g = nb.GpuStateVector(n, nb.C64)
    rec, st = g.run_fused(nb.Circuit.parse(text), nb.StdRng(0))
    o = oracle.StateVector(n)
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    a, b = g.to_vector(), o.to_vector()
    assert _fidelity(b, a) < INFIDELITY
    assert np.abs(a - b).max() < AMP_TOL
    assert st.source_gates == depth * (n + n // 2) and st.passes >= 1


def test_fused_reuses_tile_buffers(nb):
    """n = 21: 512 tiles, so CTAs take more than one set of tiles and every
    rotating tile buffer and operand slot is reused; against the complex128
    plain path on the same circuit."""
    n = 21
    c = nb.Circuit.random_layers(n, 12, 4)
    f = nb.GpuStateVector(n, nb.C64)
    rec, st = f.run_fused(c, nb.StdRng(0))
    ref = nb.GpuStateVector(n, nb.C128)
    ref.run(c, nb.StdRng(0))
    cmp = ref.compare(f)
    assert cmp["infidelity"] < INFIDELITY
    assert cmp["max_abs_diff"] < AMP_TOL * 2 ** (-(n - 12) / 2)
    assert st.passes >= 2


def test_fused_random_state_every_gate_kind(nb, oracle):
    n = 13
    r = np.random.default_rng(4)
    v = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    v /= np.linalg.norm(v)
    text = (
        "QUBITS 13\nH 0 1 2 3 4 5 6 7 8 9 10 11 12\nCY 0 11\nSWAP 1 12\nPHASE(3,4) 2\nCPHASE(5,3) 0 9\nRX(0.3) 1\n"
        "RY(1.1) 12\nSQRT_Y 3\nCS 2 10\nCCX 3 11 0\nCCZ 4 12 7\nCX 12 0\nT_DAG 11\nS_DAG 12\nCZ 11 12\nRZ(0.7) 12\nH 12\n"
    )
    g = nb.GpuStateVector.from_amplitudes(v, nb.C64)
    g.run_fused(nb.Circuit.parse(text), nb.StdRng(0))
    o = oracle.StateVector.from_amplitudes(v)
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    a, b = g.to_vector(), o.to_vector()
    assert _fidelity(b, a) < INFIDELITY
    assert np.abs(a - b).max() < AMP_TOL


def test_fused_reversible_family(nb, oracle):
    text = oracle.reversible_circuit_text(15, 120, 6)
    g = nb.GpuStateVector(15, nb.C64)
    g.run_fused(nb.Circuit.parse(text), nb.StdRng(0))
    idx, amp = oracle.sparse_run(text)
    a = g.to_vector()
    assert np.abs(a[idx.astype(np.int64)] - amp).max() < AMP_TOL
    assert abs(np.sum(np.abs(a) ** 2) - 1) < 1e-5


def test_fused_measurement_records_match_plain(nb, oracle):
    n = 16
    text = oracle.random_circuit_text(n, 12, 9, 0.0, n - 4, n)
    text += "".join(f"H {q}\n" for q in range(6)) + "M 0 1 2\n"
    c = nb.Circuit.parse(text)
    g = nb.GpuStateVector(n, nb.C64)
    rec_f, _ = g.run_fused(c, nb.StdRng(21))
    o = oracle.StateVector(n)
    rec_o = o.run(oracle.Circuit(text), oracle.StdRng(21))
    assert rec_f == rec_o
    a, b = g.to_vector(), o.to_vector()
    assert _fidelity(b, a) < INFIDELITY


def test_fused_noisy_trajectory_matches_oracle(nb, oracle):
    seed = 4
    n_o, z0_o, rec_o = oracle.trajectory(seed, 12, 3, 10, 0.05)
    rng = nb.StdRng(seed)
    n = 12 + rng.gen_range(0, 3)
    c = nb.Circuit.random_layers_from(rng, n, 10, 0.05, 0, 0)
    s = nb.GpuStateVector(n, nb.C64)
    s.run_fused(c, rng)
    e = s.expectation(nb.Pauli(n, 0, 1, 0)).real / s.norm_sq().real
    assert abs(e - z0_o) < 1e-5
    m = nb.Circuit.parse(f"QUBITS {n}\n" + "".join(f"M {q}\n" for q in range(n)))
    assert s.run(m, rng) == rec_o


def test_fused_compare_reduction_and_refusals(nb):
    n = 14
    c = nb.Circuit.random_layers(n, 6, 5)
    a = nb.GpuStateVector(n, nb.C64)
    b = nb.GpuStateVector(n, nb.C128)
    a.run_fused(c, nb.StdRng(0))
    b.run(c, nb.StdRng(0))
    d = b.compare(a)
    assert d["infidelity"] < INFIDELITY and d["max_abs_diff"] < AMP_TOL
    with pytest.raises(nb.SimError):
        b.run_fused(c, nb.StdRng(0))  # complex128 registers take the plain path
