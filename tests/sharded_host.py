"""Test support for the sharded register on CPU ranks (gloo): a shard that
keeps its 2^(n-g) amplitudes in a host array and applies each gate through the
engine's own host-side lowering (``Gate.lowered_matrix``, the dense matrix the
kernels apply), so that the partition, exchange and reduction logic of
``ncsim_b200.sharded`` runs without a GPU.  Also the per-rank worker that the
multi-rank tests launch.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

BLOCK = 4096


class HostShard:
    device = "cpu"

    def __init__(self, nl: int):
        self.nl = nl
        self.a = np.zeros(1 << nl, dtype=np.complex128)
        self.a[0] = 1.0

    def _local(self, qubits):
        idx = np.arange(1 << self.nl, dtype=np.int64)
        loc = np.zeros_like(idx)
        for j, q in enumerate(qubits):
            loc |= ((idx >> q) & 1) << j
        rest = idx.copy()
        for q in qubits:
            rest &= ~(1 << q)
        return loc, rest

    def apply_gate(self, gate, qubits):
        m = gate.lowered_matrix()
        k = len(qubits)
        loc, rest = self._local(qubits)
        order = np.lexsort((loc, rest))
        fib = self.a[order].reshape(-1, 1 << k)  # fibers, local index last
        fib = fib @ m.T
        self.a[order] = fib.reshape(-1)

    def _pauli_phase(self, z, phase):
        idx = np.arange(1 << self.nl, dtype=np.int64)
        pc = np.array([bin(int(v)).count("1") for v in (idx & z)], dtype=np.int64) if z else np.zeros_like(idx)
        return (1j) ** ((phase + 2 * pc) & 3)

    def _apply_p(self, x, z, phase, a):
        # (P psi)(c) = i^{k(c ^ x)} psi(c ^ x), k(c) = phase + 2 popcount(z & c)
        idx = np.arange(1 << self.nl, dtype=np.int64)
        src = idx ^ x
        return self._pauli_phase(z, phase)[src] * a[src]

    def apply_pauli(self, x, z, phase):
        self.a = self._apply_p(x, z, phase, self.a)

    def expectation(self, x, z, phase):
        return complex(np.vdot(self.a, self._apply_p(x, z, phase, self.a)))

    def measure_stats(self, x, z, phase):
        return self.expectation(x, z, phase), float(np.vdot(self.a, self.a).real)

    def project(self, x, z, phase, outcome):
        pa = self._apply_p(x, z, phase, self.a)
        self.a = (self.a + (-pa if outcome else pa)) / 2
        return float(np.vdot(self.a, self.a).real)

    def norm_sq(self):
        return float(np.vdot(self.a, self.a).real)

    def scale(self, c):
        self.a *= c

    def amplitude(self, i):
        return complex(self.a[i])

    def to_vector(self):
        return self.a.copy()

    def block_weights(self):
        w = (np.abs(self.a) ** 2).reshape(-1, BLOCK)
        return np.array([sum(float(v) for v in row) for row in w])

    def sample_walk(self, targets, blocks, accs):
        out = []
        for t, b, acc in zip(targets, blocks, accs):
            run = acc
            start = int(b) * BLOCK
            pick = start + BLOCK - 1
            for i in range(start, start + BLOCK - 1):
                run += abs(self.a[i]) ** 2
                if run > t:
                    pick = i
                    break
            while pick > start and self.a[pick] == 0:
                pick -= 1
            out.append(pick)
        return np.array(out, dtype=np.uint64)

    def half(self, l, c):
        import torch

        v = self.a.reshape(1 << (self.nl - l - 1), 2, 1 << l)[:, c, :]
        return torch.from_numpy(np.ascontiguousarray(v).reshape(-1))

    def set_half(self, l, c, data):
        v = self.a.reshape(1 << (self.nl - l - 1), 2, 1 << l)
        v[:, c, :] = data.numpy().reshape(1 << (self.nl - l - 1), 1 << l)

    def empty_like_half(self, l):
        import torch

        return torch.empty(1 << (self.nl - 1), dtype=torch.complex128)


def worker(spec_path: str, out_path: str) -> None:
    """One rank: runs the spec's circuit and readouts on a sharded register."""
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import ncsim_b200 as nb
    from ncsim_b200.sharded import ShardedStateVector

    spec = json.load(open(spec_path))
    dist.init_process_group("gloo")
    s = ShardedStateVector(spec["n"], shard_factory=HostShard)
    rng = nb.StdRng(spec["seed"])
    rec = s.run(nb.Circuit.parse(spec["text"]), rng)
    out = {"rank": dist.get_rank(), "record": rec, "exchanges": s.exchanges}
    out["expectations"] = [[e.real, e.imag] for e in
                           (s.expectation(nb.Pauli.from_string(spec["n"], p)) for p in spec["paulis"])]
    out["amplitudes"] = [[a.real, a.imag] for a in (s.amplitude(i) for i in spec["indices"])]
    out["norm"] = s.norm_sq()
    out["samples"] = [int(v) for v in s.sample(nb.StdRng(spec["seed"] + 1), spec["shots"])]
    v = s.to_vector()
    if dist.get_rank() == 0:
        np.save(out_path + ".npy", v)
        json.dump(out, open(out_path, "w"))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    worker(sys.argv[1], sys.argv[2])
