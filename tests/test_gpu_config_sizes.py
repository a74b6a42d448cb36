"""Parity at the workloads' full sizes.

- C1: the random layer family at n = 30, depth 20, complex128 (16 GiB), with M
  on qubits 26..29.  The oracle takes about a second per gate at this size on
  the host, so it checks three of the twenty layers at full size, each started
  from the engine's own register before that layer (the first, a middle and
  the last), and the final measurement block started from the engine's
  register before it: every amplitude within 1e-12 after each checked step,
  and the four records identical for the same seed.  The other layers are
  covered by the n <= 24 whole-circuit parity tests of the same family.
- C2: the fused precision form at n = 32 (complex64, 32 GiB) against the plain
  complex128 path on the same circuit (64 GiB): 1 - F <= 1e-6, with the
  largest amplitude error reported and bounded.
- C2 capacity: n = 34 complex64 (128 GiB): the circuit and then its inverse on
  the fused form return the register to |0...0> (1 - |<0|psi>|^2 / <psi|psi>
  <= 1e-6), and the norm drifts by less than 1e-4 per circuit.
- C4: all 4096 noisy trajectories of the batching form against per-trajectory
  complex128 runs of the same draws on the plain path: the averaged <Z0>
  within 1e-6, every trajectory's <Z0> within 1e-4.

Each test needs its register's memory on the device (and the C1 test 16 GiB
of host memory for the oracle); a test whose memory is not there is skipped
with the reason printed.
"""
from __future__ import annotations

import concurrent.futures as cf
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL = 1e-12
CHUNK = 1 << 24  # amplitudes per host transfer (256 MiB of complex128)


def _host_available() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def _need_device(nb, nbytes: int):
    free = nb.device_info()["free_bytes"]
    if free < nbytes + (2 << 30):
        pytest.skip(f"needs {nbytes / 2**30:.0f} GiB of device memory, {free / 2**30:.0f} GiB free")


def _split_layers(text: str, n: int):
    """The random layer text as (header, [layer texts], measurement text)."""
    lines = text.strip().split("\n")
    header, body = lines[0] + "\n", lines[1:]
    per = n + n // 2
    gates = [ln for ln in body if not ln.startswith("M ")]
    meas = [ln for ln in body if ln.startswith("M ")]
    assert len(gates) % per == 0
    layers = ["\n".join(gates[i:i + per]) + "\n" for i in range(0, len(gates), per)]
    return header, layers, "\n".join(meas) + "\n"


def _copy_into_oracle(g, o, n):
    buf = np.empty(CHUNK, dtype=np.complex128)
    for first in range(0, 1 << n, CHUNK):
        o.set_range(first, g.to_vector_range(first, CHUNK, buf))


def _max_diff(g, o, n) -> float:
    buf = np.empty(CHUNK, dtype=np.complex128)
    return max(o.max_abs_diff(first, g.to_vector_range(first, CHUNK, buf)) for first in range(0, 1 << n, CHUNK))


def test_c1_n30_layers_and_records_match_oracle(nb, oracle):
    n = 30
    if _host_available() < (20 << 30):
        pytest.skip(f"the oracle's 16 GiB register does not fit: {_host_available() / 2**30:.0f} GiB available")
    _need_device(nb, 16 << n)
    text = oracle.random_circuit_text(n, 20, 1, 0.0, n - 4, n)
    header, layers, meas = _split_layers(text, n)
    assert len(layers) == 20
    g = nb.GpuStateVector(n)
    o = oracle.StateVector(n)
    checked = {0, 10, 19}
    diffs = {}
    for L, body in enumerate(layers):
        if L in checked:
            _copy_into_oracle(g, o, n)
            o.run(oracle.Circuit(header + body), oracle.StdRng(0))
        g.run(nb.Circuit.parse(header + body), nb.StdRng(0))
        if L in checked:
            diffs[L] = _max_diff(g, o, n)
            assert diffs[L] < TOL, (L, diffs[L])
    _copy_into_oracle(g, o, n)
    rec_g = g.run(nb.Circuit.parse(header + meas), nb.StdRng(5))
    rec_o = o.run(oracle.Circuit(header + meas), oracle.StdRng(5))
    assert len(rec_g) == 4 and rec_g == rec_o
    d = _max_diff(g, o, n)
    assert d < TOL
    print(f"C1 n=30: layer errors {diffs}, after M 26..29 {d:.2e}, records {rec_g}")


def test_c2_n32_fused_fidelity_against_complex128(nb):
    n = 32
    _need_device(nb, (16 + 8) << n)
    c = nb.Circuit.random_layers(n, 20, 1)
    ref = nb.GpuStateVector(n, nb.C128)
    ref.run(c, nb.StdRng(7))
    f = nb.GpuStateVector(n, nb.C64)
    f.run_fused(c, nb.StdRng(7))
    cmp = ref.compare(f)
    print(f"C2 n=32: 1-F {cmp['infidelity']:.3e}, max |da| {cmp['max_abs_diff']:.3e}, norm {cmp['norm_b']:.9f}")
    assert cmp["infidelity"] <= 1e-6
    # amplitudes are about 2^-16 here: 2e-5 of a unit amplitude scaled the same way
    assert cmp["max_abs_diff"] < 2e-5 * 2.0 ** (-(n - 12) / 2)


def _inverse_text(text: str) -> str:
    inv = {"H": "H", "S": "S_DAG", "T": "T_DAG", "SQRT_X": "SQRT_X_DAG", "CZ": "CZ"}
    lines = text.strip().split("\n")
    out = [lines[0]]
    for ln in reversed(lines[1:]):
        name, rest = ln.split(" ", 1)
        if name.startswith("RZ("):
            out.append(f"RZ({-float(name[3:-1])!r}) {rest}")
        else:
            out.append(f"{inv[name]} {rest}")
    return "\n".join(out) + "\n"


def test_c2_n34_capacity_round_trip(nb):
    n = 34
    _need_device(nb, 8 << n)
    c = nb.Circuit.random_layers(n, 20, 1)
    ci = nb.Circuit.parse(_inverse_text(c.to_text()))
    f = nb.GpuStateVector(n, nb.C64)
    _, st = f.run_fused(c, nb.StdRng(0))
    nn = f.norm_sq().real
    f.run_fused(ci, nb.StdRng(0))
    a0 = f.amplitude(0)
    nn2 = f.norm_sq().real
    back = 1.0 - abs(a0) ** 2 / nn2  # the infidelity with |0...0>, normalised as 1 - F is
    print(f"C2 n=34: {st.source_gates} gates, {st.passes} passes, norm after the circuit {nn:.9f}, after its "
          f"inverse {nn2:.9f}, 1 - |<0|psi>|^2/<psi|psi> {back:.3e}")
    # the BF16x3 products are not exactly norm-preserving: about 2e-5 of norm per
    # circuit of this depth (reported; 1 - F is normalised and is the accuracy bar)
    assert abs(nn - 1.0) < 1e-4 and abs(nn2 - 1.0) < 2e-4
    assert back <= 1e-6


def _plain_reference(nb, count, seed0, depth, p, workers=8):
    """<Z0>/<psi|psi> before the final measurements and the record of trajectory
    t (StdRng(seed0 + t)), on the plain complex128 path, registers reused per size."""
    z = np.empty(count)
    rec = np.empty(count, dtype=np.uint64)

    def work(start):
        states, meas = {}, {}
        for t in range(start, count, workers):
            rng = nb.StdRng(seed0 + t)
            n = 16 + rng.gen_range(0, 7)
            c = nb.Circuit.random_layers_from(rng, n, depth, p, 0, 0)
            s = states.get(n)
            if s is None:
                s = states[n] = nb.GpuStateVector(n, nb.C128)
                meas[n] = nb.Circuit.parse(f"QUBITS {n}\n" + "".join(f"M {q}\n" for q in range(n)))
            else:
                s.set_basis(0)
            s.run(c, rng)
            z[t] = s.expectation(nb.Pauli(n, 0, 1, 0)).real / s.norm_sq().real
            r = s.run(meas[n], rng)
            rec[t] = sum(int(v) << k for k, v in enumerate(r))

    with cf.ThreadPoolExecutor(workers) as ex:
        list(ex.map(work, range(workers)))
    return z, rec


def test_c4_all_trajectories_against_complex128(nb):
    count, seed0, depth, p = 4096, 1, 30, 1e-3
    tb = nb.TrajectoryBatch.random_layers(count, seed0, 16, 7, depth, p)
    tb.run()
    _, rec, z0, norm = tb.results()
    z_ref, rec_ref = _plain_reference(nb, count, seed0, depth, p)
    mean_err = abs(float(z0.mean()) - float(z_ref.mean()))
    max_err = float(np.abs(z0 - z_ref).max())
    same = int((rec == rec_ref).sum())
    print(f"C4: mean <Z0> error {mean_err:.2e}, max {max_err:.2e}, records identical {same}/{count}, "
          f"norm drift {float(np.abs(norm - 1).max()):.2e}")
    assert mean_err < 1e-6
    assert max_err < 1e-4
    # complex64 against complex128: a record may differ only where a draw lies
    # within the single-precision error of its outcome probability
    assert same >= count - 2
