"""The no-allocation entry point, ncsim_measure_stats_noalloc, against the
regular state API.

It is for callers that keep the amplitudes in device memory they manage
themselves and cannot let a library allocate there; here that memory is a
torch tensor, so the engine never sees a handle.  Two calls in a row (the
static scratch keeps the previous call's contents) must each agree with
ncsim_sv_measure_stats on the same amplitudes to the tolerance of the other
parity tests.  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(nb, ptr, n, precision, p):
    e = (C.c_double * 2)()
    nn = C.c_double()
    st = nb.lib().ncsim_measure_stats_noalloc(C.c_void_p(ptr), n, precision, p.x, p.z, p.phase, None, e, C.byref(nn))
    return st, complex(e[0], e[1]), nn.value


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_measure_stats_twice_in_a_row(nb, precision):
    torch = pytest.importorskip("torch")
    n = 15
    rng = np.random.default_rng(17 + precision)
    amps = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    amps /= np.linalg.norm(amps)
    dtype = torch.complex128 if precision == nb.C128 else torch.complex64
    dev = torch.from_numpy(amps).to(dtype).to("cuda")
    torch.cuda.synchronize()
    host = dev.cpu().numpy().astype(np.complex128)  # what the device holds, for the regular API
    ref = nb.GpuStateVector.from_amplitudes(host, precision)
    paulis = [nb.Pauli(n, 0, 0b1011, 0), nb.Pauli(n, 0b100101, 0b110, 3), nb.Pauli(n, 0b100101, 0b110, 3)]
    for p in paulis:
        st, e, nn = _noalloc(nb, dev.data_ptr(), n, precision, p)
        assert st == 0, nb.lib().ncsim_last_error().decode()
        e_ref, nn_ref = ref.measure_stats(p)
        assert abs(e - e_ref) < TOL and abs(nn - nn_ref) < TOL


def test_noalloc_rejects_registers_above_its_maximum(nb):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(4, dtype=torch.complex128, device="cuda")
    st, _, _ = _noalloc(nb, buf.data_ptr(), 35, nb.C128, nb.Pauli(35, 0, 1, 0))
    assert st == 8 and "maximum" in nb.lib().ncsim_last_error().decode()
