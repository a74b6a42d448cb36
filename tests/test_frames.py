"""The frame sampler's host side and its oracle, on CPU.

- The oracle's restatement of frame.rs is pinned by the reference's own tests
  of it (frame.rs:309-462): the repetition-code rates, the noiseless
  detectors, and the record histograms against trajectories (total variation
  below 0.03), here against the oracle's dense StateVector trajectories.
- The reference record (FrameSampler::new): the engine's bit-sliced column
  tableau and the oracle's row tableau agree bit for bit on random Clifford
  circuits (up to 300 qubits), and on small registers every recorded outcome
  is one the dense oracle state allows, drawn from the generator exactly when
  it is random (Stabilizer::collapse, stabilizer.rs:571-591).
- Circuits of more than 64 qubits parse, print and re-parse; non-Clifford
  gates are refused as the reference refuses them.
"""
from __future__ import annotations

import random

import numpy as np
import pytest

from frames_cases import batch_seeds, random_clifford_text


def _tv(a: dict, b: dict, shots: int) -> float:
    keys = set(a) | set(b)
    return sum(abs(a.get(k, 0) - b.get(k, 0)) for k in keys) / (2 * shots)


def _histogram_frames(oracle, text, shots, seed, rng_seed):
    ref = oracle.frame_reference(text, seed)
    r = oracle.StdRng(rng_seed)
    packed = oracle.frame_sample_packed(text, ref, shots, batch_seeds(r, shots), threads=4)
    m = packed.shape[0]
    h = {}
    for s in range(shots):
        key = tuple((int(packed[k, s // 64]) >> (s % 64)) & 1 for k in range(m))
        h[key] = h.get(key, 0) + 1
    return h


def _histogram_trajectories(oracle, text, shots, seed):
    c = oracle.Circuit(text)
    n = c.num_qubits
    rng = oracle.StdRng(seed)
    h = {}
    for _ in range(shots):
        s = oracle.StateVector(n)
        key = tuple(int(b) for b in s.run(c, rng))
        h[key] = h.get(key, 0) + 1
    return h


@pytest.mark.parametrize("text,shots", [
    ("QUBITS 3\nH 0\nCX 0 1\nCX 1 2\nM 0 1 2\nMX 0\nM 2\n", 20000),
    ("QUBITS 2\nH 0\nS 0\nCX 0 1\nMY 0\nMPP X0*X1 Z0*Z1\nR 0\nM 0\nH 1\nM 1\n", 20000),
    ("QUBITS 3\nH 0\nDEPOLARIZE1(0.1) 0\nCX 0 1\nDEPOLARIZE2(0.2) 0 1\nCX 1 2\nX_ERROR(0.15) 2\nM 0 1 2\nMPP Z0*Z1\n",
     40000),
    ("QUBITS 2\nH 0\nCX 0 1\nPAULI_CHANNEL_1(0.05,0.1,0.15) 1\nSQRT_X 0\nCY 0 1\nMX 0 1\nZ_ERROR(0.3) 0\nR 1\nMX 0\n"
     "M 1\n", 40000),
])
def test_oracle_records_match_trajectories(oracle, text, shots):
    """frame.rs:317-370: frame histograms against trajectory histograms, TV < 0.03."""
    hf = _histogram_frames(oracle, text, shots, 7, 11)
    ht = _histogram_trajectories(oracle, text, shots // 4, 12)
    # the trajectory side runs a quarter of the shots: compare frequencies
    keys = set(hf) | set(ht)
    tv = sum(abs(hf.get(k, 0) / shots - ht.get(k, 0) / (shots // 4)) for k in keys) / 2
    assert tv < 0.03, (tv, hf, ht)


def test_oracle_repetition_code_rates(oracle):
    """frame.rs:403-460: distance-3 majority vote and a two-measurement detector."""
    p = 0.1
    text = f"QUBITS 3\nX_ERROR({p}) 0 1 2\nM 0 1 2\n"
    shots = 200_000
    ref = oracle.frame_reference(text, 0)
    packed = oracle.frame_sample_packed(text, ref, shots, batch_seeds(oracle.StdRng(3), shots), threads=8)
    bits = np.unpackbits(packed.view(np.uint8), axis=1, bitorder="little")[:, :shots]
    fails = int((bits.sum(axis=0) >= 2).sum())
    want = 3 * p * p * (1 - p) + p ** 3
    assert abs(fails / shots - want) < 4 * (want / shots) ** 0.5
    d = (bits[0] ^ bits[1]).mean()
    assert abs(d - 2 * p * (1 - p)) < 0.01


def _repetition_text(d=5, rounds=3, p=0.02):
    text = f"QUBITS {2 * d - 1}\n"
    for r in range(rounds):
        text += f"X_ERROR({p})" + "".join(f" {q}" for q in range(d)) + "\n"
        for a in range(d - 1):
            anc = d + a
            text += f"CX {a} {anc}\nCX {a + 1} {anc}\nM {anc}\nR {anc}\n"
        for a in range(d - 1):
            if r == 0:
                text += f"DETECTOR rec[-{d - 1 - a}]\n"
            else:
                text += f"DETECTOR rec[-{d - 1 - a}] rec[-{2 * (d - 1) - a}]\n"
    text += "M" + "".join(f" {q}" for q in range(d)) + "\nOBSERVABLE_INCLUDE(0) rec[-1]\n"
    return text


def test_oracle_repetition_code_memory_with_detectors(oracle):
    """frame.rs:372-401: quiet without noise; first-round detector and observable rates."""
    d, rounds, p = 5, 3, 0.02
    text = _repetition_text(d, rounds, p)
    quiet = "\n".join(ln for ln in text.split("\n") if not ln.startswith("X_ERROR")) + "\n"
    ref = oracle.frame_reference(quiet, 5)
    dq, oq = oracle.frame_sample_detectors(quiet, ref, 1000, batch_seeds(oracle.StdRng(1), 1000), rounds * (d - 1), 1)
    assert not dq.any() and not oq.any()
    shots = 100_000
    ref = oracle.frame_reference(text, 5)
    det, obs = oracle.frame_sample_detectors(text, ref, shots, batch_seeds(oracle.StdRng(2), shots),
                                             rounds * (d - 1), 1)
    pop = lambda row: int(np.unpackbits(row.view(np.uint8)).sum())  # noqa: E731
    assert abs(pop(det[0]) / shots - 2 * p * (1 - p)) < 0.005
    q = 1 - (1 - 2 * p) ** rounds
    assert abs(pop(obs[0]) / shots - q / 2) < 0.005


def test_reference_records_engine_and_oracle_agree(nb, oracle):
    r = random.Random(1)
    for trial in range(150):
        n = r.choice([1, 2, 3, 5, 8, 70, 300])
        text = random_clifford_text(r, n, r.randint(5, 80))
        seed = r.randrange(1 << 40)
        got = nb.FrameSampler(nb.Circuit.parse(text), seed).reference()
        assert got == oracle.frame_reference(text, seed), text


def _pauli_of(line: str, n: int, nb):
    name, rest = line.split(" ", 1)
    if name == "MPP":
        return nb.Pauli.from_string(n, rest.strip())
    q = int(rest)
    letter = {"M": "Z", "MZ": "Z", "MX": "X", "MY": "Y"}[name]
    return nb.Pauli.from_string(n, f"{letter}{q}")


def test_reference_record_is_physical_and_draws_like_the_tableau(nb, oracle):
    """Each recorded outcome has nonzero probability in the dense oracle state;
    the outcomes of probability 1/2 are the generator's successive gen::<bool>()."""
    r = random.Random(5)
    for trial in range(40):
        n = r.choice([1, 2, 3, 4, 6])
        text = random_clifford_text(r, n, r.randint(5, 40), noise=False)
        seed = r.randrange(1 << 30)
        rec = nb.FrameSampler(nb.Circuit.parse(text), seed).reference()
        draws = oracle.StdRng(seed)
        s = oracle.StateVector(n)
        k = 0

        def settle(p, outcome=None):
            e = s.expectation_raw(p.x, p.z, p.phase).real / s.norm_sq().real
            p_plus = (1 + e) / 2
            random_outcome = abs(p_plus - 0.5) < 1e-9
            if random_outcome:
                drawn = int(draws.next_u32()) >= 1 << 31  # (next_u32 as i32) < 0
                if outcome is None:
                    outcome = drawn
                assert outcome == drawn, (text, k)
            else:
                assert abs(p_plus - round(p_plus)) < 1e-9
                det = p_plus < 0.5
                if outcome is None:
                    outcome = det
                assert outcome == det, (text, k)
            s.project_raw(p.x, p.z, p.phase, outcome)
            s.normalize()
            return outcome

        for line in text.strip().split("\n")[1:]:
            head = line.split(" ")[0].split("(")[0]
            if head in ("M", "MZ", "MX", "MY", "MPP"):
                settle(_pauli_of(line, n, nb), rec[k])
                k += 1
            elif head == "R":
                q = int(line.split()[1])
                if settle(nb.Pauli.from_string(n, f"Z{q}")):
                    s.apply_gate_text(f"X {q}")
            elif head not in ("DETECTOR", "OBSERVABLE_INCLUDE", "TICK"):
                s.apply_gate_text(line)
        assert k == len(rec)


def test_wide_circuits_parse_and_print(nb):
    text = "QUBITS 1000\nH 0\nCX 0 999\nDEPOLARIZE2(0.001) 0 999\nM 999\nMPP -X0*Y500*Z999\nR 998\nDETECTOR rec[-1]\n"
    c = nb.Circuit.parse(text)
    assert c.num_qubits == 1000 and c.num_measurements == 2
    out = c.to_text()
    assert "MZ 999" in out and "MPP -X0*Y500*Z999" in out
    assert nb.Circuit.parse(out).to_text() == out
    with pytest.raises(nb.SimError):
        nb.Circuit.parse("QUBITS 1000\nCX 5 5\n")
    with pytest.raises(nb.SimError):
        nb.Circuit.parse("QUBITS 1000\nMPP iX0*Z999\n")


@pytest.mark.parametrize("gate", ["T 0", "T_DAG 0", "CS 0 1", "CCZ 0 1 2", "CCX 0 1 2", "RX(0.5) 0", "RZ(1.5707963267948966) 0",
                                  "PHASE(1,3) 0", "CPHASE(1,2) 0 1"])
def test_non_clifford_gates_are_refused(nb, oracle, gate):
    text = f"QUBITS 3\n{gate}\nM 0\n"
    with pytest.raises(nb.SimError) as e:
        nb.FrameSampler(nb.Circuit.parse(text), 0)
    assert e.value.kind == "Unsupported" and "non-Clifford" in str(e.value)
    with pytest.raises(oracle.OracleError):
        oracle.frame_reference(text, 0)


def test_frame_workload_matches_the_oracle_generator(nb, oracle):
    """The reference's frame benchmark circuit (examples/bench.rs:264-294) from both generators."""
    c = nb.Circuit.frames_workload(1000, 20, 100, 1e-3, 9)
    assert c.num_qubits == 1000 and c.num_gates == 10_500 and c.num_measurements == 2000
    assert nb.Circuit.parse(oracle.frames_circuit_text(1000, 20, 100, 1e-3, 9)).to_text() == c.to_text()


def test_reference_record_given_by_the_caller(nb):
    c = nb.Circuit.parse("QUBITS 2\nH 0\nM 0\nM 1\n")
    f = nb.FrameSampler(c, reference=[1, 0])
    assert f.reference() == [True, False]
    with pytest.raises(nb.SimError):
        nb.FrameSampler(c, reference=[1])
