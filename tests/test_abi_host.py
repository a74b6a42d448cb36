"""CPU tests of the engine library: it loads, exports every symbol the header
declares, and its host layer (StdRng, circuit parsing, gate parsing,
workloads, argument validation) agrees with the oracle.  No kernel runs."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols(header="ncsim_cuda.h"):
    hdr = open(os.path.join(ROOT, "include", header)).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(ncsim_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(nb):
    syms = _declared_symbols()
    assert len(syms) >= 50
    lib = C.CDLL(nb.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) <= set(nb._SIGNATURES), set(syms) - set(nb._SIGNATURES)


def test_workloads_live_in_their_own_library(nb):
    """The seeded workloads are declared in ncsim_workloads.h and exported by
    libncsim_workloads.so, not by the engine's drop-in library."""
    syms = _declared_symbols("ncsim_workloads.h")
    assert set(syms) == set(nb._WORKLOAD_SIGNATURES)
    assert not set(syms) & set(_declared_symbols())
    w = nb.workloads_lib()
    assert all(hasattr(w, s) for s in syms)
    engine = C.CDLL(nb.LIB_PATH)
    assert not any(hasattr(engine, s) for s in syms)


def test_rng_matches_oracle(nb, oracle):
    for seed in (0, 1, 7, 2**63 + 5):
        a, b = nb.StdRng(seed), oracle.StdRng(seed)
        seq_a = [a.next_u64() for _ in range(70)] + [a.next_u32() for _ in range(3)] + [a.gen_f64() for _ in range(70)]
        seq_b = [b.next_u64() for _ in range(70)] + [b.next_u32() for _ in range(3)] + [b.gen_f64() for _ in range(70)]
        assert seq_a == seq_b
        assert [a.gen_range(0, 7) for _ in range(50)] == [b.gen_range(0, 7) for _ in range(50)]


@pytest.mark.parametrize(
    "n,depth,seed,p,lo,hi",
    [(20, 40, 1, 0.0, 0, 0), (30, 20, 1, 0.0, 26, 30), (32, 20, 1, 0.0, 0, 0), (22, 30, 5, 1e-3, 0, 22), (7, 3, 2, 0.0, 2, 5)],
)
def test_random_layer_workload_matches_oracle(nb, oracle, n, depth, seed, p, lo, hi):
    c = nb.Circuit.random_layers(n, depth, seed, p, lo, hi)
    ref = nb.Circuit.parse(oracle.random_circuit_text(n, depth, seed, p, lo, hi))
    assert c.to_text() == ref.to_text()
    assert c.num_gates == depth * (n + n // 2)


def test_reversible_workload_matches_oracle(nb, oracle):
    for n, g, s in [(31, 80, 1), (12, 40, 9)]:
        assert nb.Circuit.reversible(n, g, s).to_text() == oracle.reversible_circuit_text(n, g, s)


def test_circuit_text_round_trip(nb):
    """src/circuit.rs:772-785."""
    text = "H 0\nCX 0 1 1 2\nT 2\nPHASE(3,4) 1\nM 0\nMX 1\nMPP X0*Z2\nR 2\nTICK\n"
    c = nb.Circuit.parse(text)
    assert (c.num_qubits, c.num_gates, c.num_measurements) == (3, 5, 3)
    assert nb.Circuit.parse(c.to_text()).to_text() == c.to_text()
    full = text + "DEPOLARIZE2(0.01) 0 1\nX_ERROR(0.5) 2\nPAULI_CHANNEL_1(0.1,0,0.2) 1\nDETECTOR rec[-1] rec[-2]\nOBSERVABLE_INCLUDE(0) rec[-1]\n"
    c2 = nb.Circuit.parse(full)
    assert nb.Circuit.parse(c2.to_text()).to_text() == c2.to_text()


@pytest.mark.parametrize(
    "bad,kind",
    [
        ("CX 0", "Parse"),
        ("QUBITS 1\nH 3", "Parse"),
        ("FOO 1", "Parse"),
        ("MPP X0*Z1*X0", "Parse"),
        ("RZ 0", "Parse"),
        ("DEPOLARIZE1(2) 0", "Parse"),
        ("CX 1 1", "Parse"),
        ("M 0\nDETECTOR rec[-2]", "Parse"),
        ("PHASE(1,40) 0", "Parse"),
    ],
)
def test_parse_errors(nb, bad, kind):
    with pytest.raises(nb.SimError) as e:
        nb.Circuit.parse(bad)
    assert e.value.kind == kind


def test_pauli_parse_and_hermiticity(nb):
    """src/pauli/mod.rs:462-483."""
    p = nb.Pauli.from_string(3, "-i*X0*Z2")
    assert (p.x, p.z, p.phase) == (1, 4, 3)
    y = nb.Pauli.from_string(1, "Y0")
    assert (y.x, y.z, y.phase) == (1, 1, 1) and y.is_hermitian()
    assert not nb.Pauli(1, 1, 1, 0).is_hermitian()
    q = nb.Pauli.from_string(4, "+XZ_Y")
    assert (q.x, q.z, q.phase) == (0b1001, 0b1010, 1)
    with pytest.raises(nb.SimError):
        nb.Pauli.from_string(3, "X0*X0")


def test_gate_tokens(nb):
    assert nb.Gate.parse("CCZ").arity == 3
    assert nb.Gate.parse("rz(0.25)").arity == 1
    assert nb.Gate.parse("DIAG(3;1;5:1,2;7:4)", 3).arity == 3
    with pytest.raises(nb.SimError) as e:
        nb.Gate.parse("MONOMIAL(1,1;0;1;0;0,0,0)", 2)  # singular affine map
    assert e.value.kind == "Invalid"
    with pytest.raises(nb.SimError):
        nb.Gate.parse("NOPE")


def test_state_argument_errors_need_no_device(nb):
    import ctypes

    h = ctypes.c_void_p()
    assert nb.lib().ncsim_sv_create(40, nb.C128, ctypes.byref(h)) == 8
    assert nb.lib().ncsim_sv_create(10, 7, ctypes.byref(h)) == 8
    assert nb.lib().ncsim_sv_norm_sq(None, (ctypes.c_double * 2)()) == 8
    assert "null" in nb.lib().ncsim_last_error().decode()
    # the sparse form: register sizes 1..1024 and null handles, checked before any device call
    assert nb.lib().ncsim_sparse_create(1025, ctypes.byref(h)) == 8
    assert nb.lib().ncsim_sparse_create(0, ctypes.byref(h)) == 8
    assert nb.lib().ncsim_sparse_norm_sq(None, (ctypes.c_double * 2)()) == 8
    assert nb.lib().ncsim_sparse_run(None, None, None, None, 0, None) == 8


LOWERED = ["I", "X", "Y", "Z", "H", "S", "S_DAG", "SQRT_X", "SQRT_X_DAG", "SQRT_Y", "SQRT_Y_DAG", "T", "T_DAG",
           "CX", "CY", "CZ", "SWAP", "CS", "CS_DAG", "CCZ", "CCX", "PHASE(3,4)", "PHASE(-5,9)", "CPHASE(1,3)",
           "CPHASE(7,2)", "RX(0.3)", "RY(-1.1)", "RZ(2.2)"]


@pytest.mark.parametrize("name", LOWERED)
def test_lowering_of_named_gates_matches_gate_matrix(nb, oracle, name):
    """The kernel descriptors built on the host equal the oracle's Gate::matrix (gate.rs:670-747)."""
    import numpy as np

    g = nb.Gate.parse(name)
    k = g.arity
    want = oracle.gate_matrix(f"QUBITS {k}\n{name} " + " ".join(map(str, range(k))) + "\n")
    assert np.abs(g.lowered_matrix() - want).max() < 1e-15


def test_lowering_of_random_diagonals_and_monomials(nb, oracle):
    import numpy as np

    text = oracle.reversible_circuit_text(8, 40, 21)
    for line in text.splitlines()[1:]:
        toks = line.split()
        if not toks[0].startswith(("DIAG", "MONOMIAL")):
            continue
        k = len(toks) - 1
        local = f"QUBITS {k}\n{toks[0]} " + " ".join(map(str, range(k))) + "\n"
        g = nb.Gate.parse(toks[0], k)
        want = np.eye(1 << k, dtype=complex)
        s = oracle.StateVector(k)
        for col in range(1 << k):
            e = np.zeros(1 << k, dtype=complex)
            e[col] = 1
            s.set_amplitudes(e)
            s.apply_gate_text(local.split("\n", 1)[1])
            want[:, col] = s.to_vector()
        assert np.abs(g.lowered_matrix() - want).max() < 1e-15, toks[0][:40]
