"""The sharded register (ncsim_b200.sharded) on 2 and 4 CPU ranks over gloo,
against the oracle's single StateVector of the same circuit.

Each rank holds 2^(n-g) amplitudes in a host array (tests/sharded_host.py);
the exchanges of halves between partner ranks, the qubit map, the rank-bit
phases of Pauli operators, the all-reduced sums and the distributed sampling
are the product's own code.  Bar: every amplitude within 1e-12, records and
sampled indices identical, expectations within 1e-12.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-12


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _circuit(oracle, n: int) -> str:
    base = oracle.random_circuit_text(n, 5, 3)
    t = n - 1
    extra = (f"CCX {t} {t - 1} 0\nCCZ {t - 2} {t} 1\nSWAP {t} 2\nCX {t - 1} {t}\nH {t}\nRX(0.7) {t - 1}\n"
             f"MPP X{t}*Z{t - 1}\nM {t}\nR {t - 1}\nH {t - 1}\nT {t - 1}\nCX {t - 1} 3\nM 0\nMX {t - 1}\n"
             f"CY 5 {t}\nS {t}\nH 4\n")
    return base + extra


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_register_matches_the_oracle(tmp_path, oracle, world):
    n, seed, shots = 15, 11, 200
    text = _circuit(oracle, n)
    spec = {"n": n, "seed": seed, "text": text, "shots": shots,
            "paulis": ["X14*Y13*Z0", "Z13*Z14", "X0*X5*Y9", "Y14*X2"],
            "indices": [0, 1, (1 << n) - 1, 0b101100110011001, 12345, 1 << (n - 1)]}
    sp = tmp_path / "spec.json"
    sp.write_text(json.dumps(spec))
    out = tmp_path / "out.json"
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "sharded_host.py"), str(sp),
                                       str(out)], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                      text=True))
    logs = [p.communicate(timeout=600)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), logs
    got = json.loads(out.read_text())
    vec = np.load(str(out) + ".npy")

    o = oracle.StateVector(n)
    rec = o.run(oracle.Circuit(text), oracle.StdRng(seed))
    assert got["record"] == rec
    assert got["exchanges"] > 0
    assert np.abs(vec - o.to_vector()).max() < TOL
    for p, e in zip(spec["paulis"], got["expectations"]):
        assert abs(complex(*e) - o.expectation(p)) < TOL
    ov = o.to_vector()
    for i, a in zip(spec["indices"], got["amplitudes"]):
        assert abs(complex(*a) - ov[i]) < TOL
    assert abs(got["norm"] - o.norm_sq().real) < TOL
    assert got["samples"] == [int(v) for v in o.sample(oracle.StdRng(seed + 1), shots)]
