"""The batching form's host side on CPU: trajectory generation, folding and
the pass/stage plan, run by the FP64 host emulator of the device program and
compared with the oracle's trajectories (src/state/mod.rs:113-183,
src/circuit.rs:136-146).

Bar: the same register size and record for every trajectory, <Z0>/<psi|psi>
within 1e-6 (the program's gate coefficients are FP32).
"""
from __future__ import annotations

import pytest

Z0_TOL = 1e-6


def _bits(rec):
    return sum(int(v) << k for k, v in enumerate(rec))


def test_random_layer_trajectories_match_oracle(nb, oracle):
    b = nb.TrajectoryBatch.random_layers(10, seed0=1, n_lo=13, n_span=3, depth=8, p=0.05)
    nq = b.qubits()
    for t in range(10):
        rec, z0, norm = b.emulate(t)
        n_o, z0_o, rec_o = oracle.trajectory(1 + t, 13, 3, 8, 0.05)
        assert nq[t] == n_o
        assert rec == _bits(rec_o)
        assert abs(z0 - z0_o) < Z0_TOL
        assert abs(norm - 1) < 1e-5


def test_noise_free_and_noisy_draw_streams(nb, oracle):
    """p = 0 draws nothing for noise; a large p samples many errors."""
    for p in (0.0, 0.3):
        b = nb.TrajectoryBatch.random_layers(3, seed0=7, n_lo=13, n_span=2, depth=6, p=p)
        st = b.info()
        assert (st["noise_events"] == 0) == (p == 0.0)
        for t in range(3):
            rec, z0, _ = b.emulate(t)
            n_o, z0_o, rec_o = oracle.trajectory(7 + t, 13, 2, 6, p)
            assert rec == _bits(rec_o) and abs(z0 - z0_o) < Z0_TOL


def test_circuit_trajectories_match_oracle(nb, oracle):
    """Given circuits (other one-qubit gates, controlled phases, one- and
    two-qubit channels, a partial measurement block) with their own seeds."""
    n = 14
    body = []
    for q in range(n):
        body.append(["H", "RX(0.3)", "SQRT_Y", "RY(1.1)", "S_DAG", "X", "PHASE(1,3)"][q % 7] + f" {q}")
    body += [f"CZ {q} {(q + 5) % n}" for q in range(0, n, 2)]
    body += [f"CS {q} {(q + 3) % n}" for q in range(1, n, 3)]
    body += ["DEPOLARIZE1(0.2) 3", "X_ERROR(0.4) 12", "DEPOLARIZE2(0.3) 4 11", "PAULI_CHANNEL_1(0.1,0.2,0.3) 7"]
    body += [f"CPHASE(3,4) {q} {(q + 1) % n}" for q in range(0, n, 4)]
    body += [["SQRT_X", "H", "T", "RZ(2.5)"][q % 4] + f" {q}" for q in range(n)]
    meas = [f"M {q}" for q in range(9)]
    text = f"QUBITS {n}\n" + "\n".join(body + meas) + "\n"
    gates_only = f"QUBITS {n}\n" + "\n".join(body) + "\n"
    seeds = [3, 4, 5, 6]
    b = nb.TrajectoryBatch.from_circuits([nb.Circuit.parse(text)] * len(seeds), seeds)
    for t, seed in enumerate(seeds):
        rec, z0, _ = b.emulate(t)
        o = oracle.StateVector(n)
        rng = oracle.StdRng(seed)
        o.run(oracle.Circuit(gates_only), rng)
        z0_o = o.expectation("Z" + "_" * (n - 1)).real / o.norm_sq().real
        rec_o = o.run(oracle.Circuit(f"QUBITS {n}\n" + "\n".join(meas) + "\n"), rng)
        assert rec == _bits(rec_o)
        assert abs(z0 - z0_o) < Z0_TOL


def test_plan_statistics(nb):
    depth = 5
    b = nb.TrajectoryBatch.random_layers(6, seed0=11, n_lo=16, n_span=4, depth=depth, p=1e-3)
    st = b.info()
    nq = b.qubits()
    assert st["trajectories"] == 6
    assert st["source_gates"] == sum(depth * (int(n) + int(n) // 2) for n in nq)
    assert st["max_qubits"] == max(nq) and 16 <= min(nq)
    # every pass streams 2^(n-13) tiles; at least one pass per trajectory
    assert st["tile_passes"] >= sum(2 ** (int(n) - 13) for n in nq)
    assert st["folded_ops"] < st["source_gates"]


@pytest.mark.parametrize("text,kind", [
    ("QUBITS 14\nCX 0 1\nM 0\n", "Unsupported"),
    ("QUBITS 14\nH 0\nM 1\n", "Unsupported"),
    ("QUBITS 14\nM 0\nH 0\n", "Unsupported"),
    ("QUBITS 12\nH 0\nM 0\n", "Unsupported"),
    ("QUBITS 14\nH 0\nR 0\n", "Unsupported"),
])
def test_unsupported_circuits_refused(nb, text, kind):
    with pytest.raises(nb.SimError) as e:
        nb.TrajectoryBatch.from_circuits([nb.Circuit.parse(text)], [1])
    assert e.value.kind == kind


def test_register_range_refused(nb):
    with pytest.raises(nb.SimError) as e:
        nb.TrajectoryBatch.random_layers(2, 1, 10, 2, 3, 0.0)
    assert e.value.kind == "Unsupported"
    with pytest.raises(nb.SimError):
        nb.TrajectoryBatch.random_layers(0, 1, 16, 2, 3, 0.0)


@pytest.mark.parametrize("knob_set", [1, 2, 3])
def test_every_knob_set_plans_correct_programs(nb, oracle, knob_set):
    """The autotuner's candidate planner knob sets (overlapping windows every 3 or
    5 qubits, cycled stage register sets) give programs with the same results."""
    b = nb.TrajectoryBatch.random_layers(8, seed0=21, n_lo=15, n_span=4, depth=10, p=0.02)
    nq = b.qubits()
    for n in set(int(v) for v in nq):
        b.set_knob_set(n, knob_set)
        assert b.knobs(n)["knob_set"] == knob_set
    for t in range(8):
        rec, z0, norm = b.emulate(t)
        n_o, z0_o, rec_o = oracle.trajectory(21 + t, 15, 4, 10, 0.02)
        assert rec == _bits(rec_o) and abs(z0 - z0_o) < Z0_TOL
    b.set_knob_set(int(nq[0]), 0, final=True)
    assert b.knobs(int(nq[0]))["final"]
    with pytest.raises(nb.SimError):
        b.set_knob_set(int(nq[0]), 1)  # final: the trajectories were dropped
