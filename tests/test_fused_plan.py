"""The fused form's planner on the CPU: its passes, 5-qubit unitaries and
diagonal terms, replayed in FP64 with the device's tile and op order
(ncsim_fused_emulate), must equal the oracle's StateVector<C64> run."""
from __future__ import annotations

import numpy as np
import pytest

MISC = (
    "QUBITS 13\nH 0 1 2 3 4 5 6 7 8 9 10 11 12\nCY 0 11\nSWAP 1 12\nPHASE(3,4) 2\nCPHASE(5,3) 0 9\nRX(0.3) 1\n"
    "RY(1.1) 12\nSQRT_Y 3\nCS 2 10\nCCX 3 11 0\nCCZ 4 12 7\nCX 12 0\nT_DAG 11\nS_DAG 12\nCZ 11 12\nRZ(0.7) 12\nH 12\n"
)


def _state(n, seed):
    r = np.random.default_rng(seed)
    v = r.normal(size=1 << n) + 1j * r.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("max_fuse", [5, 3, 1])
@pytest.mark.parametrize("which", ["layers12", "layers16", "layers20", "reversible", "misc"])
def test_plan_replays_to_the_oracle(nb, oracle, which, max_fuse):
    text = {
        "layers12": lambda: oracle.random_circuit_text(12, 6, 1),
        "layers16": lambda: oracle.random_circuit_text(16, 12, 3),
        "layers20": lambda: oracle.random_circuit_text(20, 20, 1),
        "reversible": lambda: oracle.reversible_circuit_text(13, 60, 2),
        "misc": lambda: MISC,
    }[which]()
    c = nb.Circuit.parse(text)
    v = _state(c.num_qubits, 5)
    got, st = c.fused_emulate(v, max_fuse)
    o = oracle.StateVector.from_amplitudes(v)
    o.run(oracle.Circuit(text), oracle.StdRng(0))
    assert np.abs(got - o.to_vector()).max() < 1e-12
    assert st.source_gates == c.num_gates
    assert 1 <= st.passes and st.fused_unitaries >= 1


def test_plan_is_compact_on_the_random_layer_family(nb):
    """Diagonal gates apply from any pass: the 20-layer circuit at n = 20 needs few passes."""
    c = nb.Circuit.random_layers(20, 20, 1)
    _, st = c.fused_emulate(_state(20, 1))
    assert st.source_gates == 600
    assert st.passes <= 12 and st.fused_unitaries <= 80


def test_small_registers_are_refused(nb):
    c = nb.Circuit.parse("QUBITS 8\nH 0\n")
    with pytest.raises(nb.SimError) as e:
        c.fused_emulate(_state(8, 1))
    assert e.value.kind == "Unsupported"
