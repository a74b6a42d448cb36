"""One launch of every plain-path kernel class on a dense n-qubit register,
each timed by the launch profiler (CUDA events on the state's stream) with its
algorithmic bytes, for per-class roofline figures and for ncu captures:

    python -m ncsim_b200.kernel_cases --n 27
    ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum \\
        --clock-control none -k regex:^k_ python -m ncsim_b200.kernel_cases --n 27 --reps 1

Each case runs `--reps` times after one untimed warm-up and prints one JSON
line per case: the kernel class, launches, milliseconds per launch, GB/s of
algorithmic bytes, and the fraction of the measured copy bandwidth.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import C128, Circuit, Gate, GpuStateVector, Pauli, StdRng


def _unitary(k: int, seed: int) -> np.ndarray:
    r = np.random.default_rng(seed)
    z = r.normal(size=(1 << k, 1 << k)) + 1j * r.normal(size=(1 << k, 1 << k))
    q, rr = np.linalg.qr(z)
    return q * (np.diag(rr) / np.abs(np.diag(rr)))


def cases(n: int):
    """(name, action) pairs; each action launches one kernel of its class on the state."""
    h, cx, cz, rz = Gate.parse("H"), Gate.parse("CX"), Gate.parse("CZ"), Gate.parse("RZ(0.3)")
    ccx = Gate.parse("CCX")
    layers = Circuit.random_layers(n, 4, 1)
    u2, u3, u6 = _unitary(2, 1), _unitary(3, 2), _unitary(6, 3)
    u4, u5 = _unitary(4, 4), _unitary(5, 6)
    r = np.random.default_rng(5)
    perm6 = r.permutation(64)
    ph6 = np.exp(2j * np.pi * r.integers(0, 8, 64) / 8)
    perm11 = r.permutation(1 << 11)
    ph11 = np.exp(2j * np.pi * r.integers(0, 8, 1 << 11) / 8)
    diag_terms = [(1 + (t % 7), [1 << (t % n), 1 << ((3 * t + 1) % n)]) for t in range(40)]
    return [
        ("dense1", lambda s: s.apply_gate(h, [n - 3])),
        ("dense1_low", lambda s: s.apply_gate(h, [0])),
        ("dense2", lambda s: s.apply_matrix(u2, [3, n - 5])),
        ("dense_fiber3", lambda s: s.apply_matrix(u3, [2, 9, n - 4])),
        ("dense_fiber4", lambda s: s.apply_matrix(u4, [0, 6, 13, n - 3])),
        ("dense_fiber5", lambda s: s.apply_matrix(u5, [1, 4, 10, 16, n - 1])),
        ("dense_wide", lambda s: s.apply_matrix(u6, [1, 5, 8, 12, 17, n - 2])),
        ("diag_const", lambda s: s.apply_gate(cz, [4, n - 6])),
        ("diag_1q", lambda s: s.apply_gate(rz, [n - 7])),
        ("pairswap", lambda s: s.apply_gate(cx, [6, n - 8])),
        ("pairswap_ccx", lambda s: s.apply_gate(ccx, [7, 11, n - 9])),
        ("perm_tile", lambda s: s.apply_monomial([2, 4, 10, 13, 19, n - 1], perm6, ph6)),
        ("perm_wide", lambda s: s.apply_monomial(list(range(3, 3 + 11)), perm11, ph11)),
        ("phasepoly", lambda s: s.apply_phasepoly(list(range(n)), 3, 0, diag_terms)),
        ("pauli_pair", lambda s: s.apply_pauli(Pauli(n, (1 << 3) | (1 << (n - 2)), 1 << 5, 1))),
        ("pauli_diag", lambda s: s.apply_pauli(Pauli(n, 0, (1 << 2) | (1 << (n - 3)), 0))),
        ("norm", lambda s: s.norm_sq()),
        ("expect_diag", lambda s: s.expectation(Pauli(n, 0, (1 << 1) | (1 << (n - 1)), 0))),
        ("expect_pair", lambda s: s.expectation(Pauli(n, (1 << 4) | (1 << (n - 2)), 1 << 7, 0))),
        # the projection zeroes half the register; H on that qubit makes it dense again (a dense1 line)
        ("project_diag", lambda s: (s.project(Pauli(n, 0, 1 << (n - 4), 0), False), s.apply_gate(h, [n - 4]))),
        ("project_pair", lambda s: s.project(Pauli(n, 1 << (n - 5), 0, 0), False)),
        ("sample", lambda s: s.sample(StdRng(3), 1024)),
        # a run of gates through tiled passes (one layer of the random layer family per pass or so)
        ("run_layers", lambda s: s.run(layers, StdRng(0))),
    ]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=27)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--only", default="", help="comma-separated case names")
    args = ap.parse_args(argv)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    peak = None
    p = os.path.join(root, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peak = float(json.load(open(p))["hbm_gbs"])
    n = args.n
    s = GpuStateVector.plus_state(n, C128)
    s.apply_gate(Gate.parse("RZ(0.7)"), [0])  # a dense register without exact zeros or exact ones
    only = set(filter(None, args.only.split(",")))
    for name, act in cases(n):
        if only and name not in only:
            continue
        act(s)  # warm-up (and any one-time set-up)
        s.synchronize()
        s.profile(True)
        for _ in range(args.reps):
            act(s)
        prof = s.profile_read()
        s.profile(False)
        for cls, v in prof.items():
            ms = v["ms"] / max(1, v["launches"])
            gbs = v["bytes"] / max(v["ms"], 1e-9) / 1e6
            print(json.dumps({"case": name, "class": cls, "n": n, "launches": v["launches"],
                              "ms_per_launch": round(ms, 4), "GBps": round(gbs, 1),
                              "frac_of_measured_copy": round(gbs / peak, 4) if peak else None}), flush=True)
        if name.startswith("project"):
            s.normalize()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
