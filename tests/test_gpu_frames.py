"""The GPU frame sampler against the oracle's restatement of frame.rs: packed
records, per-shot records and detector/observable flips bit-exact for the same
batch seeds, on random Clifford circuits with every noise channel, at shot
counts around the word and batch edges, with the frame tables in shared memory
and in global memory, and on the reference's frame benchmark (1000 qubits,
10 500 noisy gates, 2000 measurements) at its full 100 000 shots."""
from __future__ import annotations

import random

import numpy as np
import pytest

from frames_cases import batch_seeds, random_clifford_text

pytestmark = pytest.mark.gpu


def _both(nb, oracle, text, shots, seed, rng_seed, threads=8):
    f = nb.FrameSampler(nb.Circuit.parse(text), seed)
    seeds = batch_seeds(nb.StdRng(rng_seed), shots)
    got = f.sample_packed(shots, nb.StdRng(rng_seed))
    want = oracle.frame_sample_packed(text, f.reference(), shots, seeds, threads=threads)
    return f, got, want


@pytest.mark.parametrize("shots", [1, 63, 64, 65, 1000, 16384, 16385, 40000])
def test_packed_records_match_oracle(nb, oracle, shots):
    r = random.Random(shots)
    for trial in range(6):
        n = r.choice([1, 2, 5, 9, 40, 130])
        text = random_clifford_text(r, n, r.randint(10, 120))
        _, got, want = _both(nb, oracle, text, shots, r.randrange(1 << 30), r.randrange(1 << 30))
        assert np.array_equal(got, want), text


def test_per_shot_records_and_detectors_match_oracle(nb, oracle):
    r = random.Random(77)
    for trial in range(8):
        n = r.choice([3, 7, 33])
        text = random_clifford_text(r, n, 80)
        shots = r.choice([500, 20000])
        f = nb.FrameSampler(nb.Circuit.parse(text), 3)
        packed = f.sample_packed(shots, nb.StdRng(9))
        per_shot = f.sample(shots, nb.StdRng(9))
        m = f.m
        bits = np.unpackbits(packed.view(np.uint8), axis=1, bitorder="little")[:, :shots]  # (m, shots)
        want = np.zeros((shots, (m + 63) // 64), dtype=np.uint64)
        if m:
            padded = np.zeros((shots, want.shape[1] * 64), dtype=np.uint8)
            padded[:, :m] = bits.T
            want = np.packbits(padded, axis=1, bitorder="little").view(np.uint64)
        assert np.array_equal(per_shot, want)
        det, obs = f.sample_detectors(shots, nb.StdRng(10))
        seeds = batch_seeds(nb.StdRng(10), shots)
        wd, wo = oracle.frame_sample_detectors(text, f.reference(), shots, seeds, f.num_detectors, f.num_observables)
        assert np.array_equal(det, wd) and np.array_equal(obs, wo), text


def test_channels_used_often_match_oracle(nb, oracle):
    """Channels used on 64 or more ops draw their skips and picks from exact step
    tables (zero probabilities, p >= 0.25 and the two-qubit channel included)."""
    r = random.Random(8)
    n = 24
    chans1 = ["X_ERROR(0.1)", "DEPOLARIZE1(0.05)", "PAULI_CHANNEL_1(0.02,0,0.07)", "Z_ERROR(0.4)", "Y_ERROR(0.001)"]
    lines = [f"QUBITS {n}"] + [f"H {q}" for q in range(0, n, 3)]
    for _ in range(900):
        a, b = r.sample(range(n), 2)
        lines.append(f"CX {a} {b}")
        lines.append(f"{r.choice(chans1)} {a}")
        lines.append(f"DEPOLARIZE2({r.choice([0.003, 0.3])}) {a} {b}")
        if r.random() < 0.2:
            lines.append(f"M {r.randrange(n)}")
    text = "\n".join(lines) + "\n"
    for shots in (5000, 40000):
        _, got, want = _both(nb, oracle, text, shots, 2, 3 + shots)
        assert np.array_equal(got, want)


def test_tables_in_global_memory_match_oracle(nb, oracle):
    """13 000 qubits: 16 n bytes per shot-word exceed the shared-memory budget."""
    n = 13000
    r = random.Random(4)
    lines = [f"QUBITS {n}"] + [f"H {q}" for q in range(0, n, 7)]
    for _ in range(400):
        a, b = r.sample(range(n), 2)
        lines.append(f"CX {a} {b}")
        lines.append(f"DEPOLARIZE2(0.01) {a} {b}")
        if r.random() < 0.3:
            lines.append(f"M {r.randrange(n)}")
    text = "\n".join(lines) + "\n"
    _, got, want = _both(nb, oracle, text, 3000, 1, 2)
    assert np.array_equal(got, want)


def test_repetition_code_rates_on_device(nb):
    """frame.rs:403-460 on the device sampler."""
    p = 0.1
    f = nb.FrameSampler(nb.Circuit.parse(f"QUBITS 3\nX_ERROR({p}) 0 1 2\nM 0 1 2\n"), 0)
    shots = 200_000
    packed = f.sample_packed(shots, nb.StdRng(3))
    bits = np.unpackbits(packed.view(np.uint8), axis=1, bitorder="little")[:, :shots]
    want = 3 * p * p * (1 - p) + p ** 3
    assert abs((bits.sum(axis=0) >= 2).mean() - want) < 4 * (want / shots) ** 0.5
    assert abs((bits[0] ^ bits[1]).mean() - 2 * p * (1 - p)) < 0.01


def test_reference_benchmark_at_full_size_matches_oracle(nb, oracle):
    """The reference's frame benchmark (examples/bench.rs:264-294): 100 000 shots, bit-exact."""
    c = nb.Circuit.frames_workload(1000, 20, 100, 1e-3, 9)
    f = nb.FrameSampler(c, 0)
    shots = 100_000
    seeds = batch_seeds(nb.StdRng(9), shots)
    got = f.sample_packed_seeds(shots, seeds)
    want = oracle.frame_sample_packed(c.to_text(), f.reference(), shots, seeds, threads=16)
    assert got.shape == (2000, (shots + 63) // 64)
    assert np.array_equal(got, want)
    print(f"frames n=1000: {f.num_layers} layers, kernels {f.last_kernel_ms():.3f} ms")


def test_argument_errors(nb):
    f = nb.FrameSampler(nb.Circuit.parse("QUBITS 2\nH 0\nM 0 1\n"), 0)
    with pytest.raises(nb.SimError):
        f.sample_packed_seeds(20000, [1])  # two batches need two seeds
    with pytest.raises(nb.SimError):
        f.sample_packed_seeds(100, [1], out=np.zeros((1, 2), dtype=np.uint64))  # room for one measurement
    assert f.sample_packed(0, nb.StdRng(0)).shape == (2, 0)
    with pytest.raises(nb.SimError):
        nb.GpuStateVector(4).run(nb.Circuit.parse("QUBITS 1000\nH 999\n"), nb.StdRng(0))
