"""The Rust crate `ncsim-cuda` (rust/ncsim-cuda) against the C header it binds.

No Rust toolchain exists here, so the crate cannot be compiled; these checks
keep it in step with include/ncsim_cuda.h: the extern block declares exactly
the header's functions with the same parameter counts, the structs have the
header's fields in order, and GpuStateVector implements every required method
of QuantumState<C64> (src/state/mod.rs:41-70) plus the overrides StateVector
has (sample, to_vector, tensor), with check_qubits and the arity check ahead
of the gate views as in src/state/vector.rs:364-395.
"""
from __future__ import annotations

import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CRATE = os.path.join(ROOT, "rust", "ncsim-cuda")


def _header():
    h = open(os.path.join(ROOT, "include", "ncsim_cuda.h")).read()
    return re.sub(r"/\*.*?\*/", "", h, flags=re.S)


def _header_functions():
    fns = re.findall(r"^\s*(?:const char\*|int32_t|ncsim_status)\s+(ncsim_\w+)\s*\(([^;]*?)\);", _header(),
                     flags=re.M | re.S)
    return {n: (0 if " ".join(a.split()) == "void" else len(a.split(","))) for n, a in fns}


def _rust_functions():
    src = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    block = src[src.index('extern "C" {'):]
    fns = re.findall(r"pub fn (ncsim_\w+)\(([^)]*)\)", block)
    return {n: (len([p for p in a.split(",") if p.strip()])) for n, a in fns}


def test_extern_block_mirrors_the_header():
    h, r = _header_functions(), _rust_functions()
    assert len(h) >= 90
    assert set(h) == set(r), (set(h) - set(r), set(r) - set(h))
    assert {n: h[n] for n in h} == {n: r[n] for n in h}


def test_structs_mirror_the_header():
    hdr = _header()
    src = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    for name in ("ncsim_error_info", "ncsim_kernel_stat", "ncsim_fused_stats", "ncsim_batch_stats",
                 "ncsim_batch_config", "ncsim_batch_knobs_info"):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), hdr, flags=re.S).group(1)
        c_fields = re.findall(r"(\w+)(?:\[\d+\])?;", body)
        rbody = re.search(r"pub struct %s \{(.*?)\}" % name, src, flags=re.S).group(1)
        r_fields = re.findall(r"pub (\w+):", rbody)
        assert c_fields == r_fields, name
    for const in re.findall(r"#define (NCSIM_\w+) (-?\d+)", hdr):
        assert re.search(r"pub const %s: \w+ = %s;" % const, src), const


def test_gpu_state_vector_implements_the_trait():
    src = open(os.path.join(CRATE, "src", "lib.rs")).read()
    impl = src[src.index("impl QuantumState<C64> for GpuStateVector"):]
    impl = impl[:impl.index("\n}\n")]
    for m in ("num_qubits", "apply_gate", "norm_sq", "amplitude", "expectation", "inner", "project", "scale",
              "tensor", "sample", "to_vector", "measure"):
        assert re.search(r"fn %s\b" % m, impl), m
    body = impl[impl.index("fn apply_gate"):impl.index("fn norm_sq")]
    order = [body.index(s) for s in ("check_qubits(", "gate.arity()", "Gate::Pauli", "gate.monomial()",
                                     "gate.matrix::<C64>()", "gate.decomposition()", "NotRepresentable")]
    assert order == sorted(order)
    # every SimError variant with fields is rebuilt from the library's error info
    for v in ("QubitOutOfRange {", "Arity {", "DuplicateQubit(", "ZeroState(", "Parse(", "Unsupported {"):
        assert v in src, v
    assert "#![forbid(unsafe_code)]\n" not in src  # the unsafe calls live here, not in the core crate
