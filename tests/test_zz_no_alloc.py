"""The no-allocation entry point, ncsim_measure_stats_noalloc, against the
regular state API.

It is for callers that keep the amplitudes in device memory they manage
themselves and cannot let a library allocate there; here that memory is a
torch tensor, so the engine never sees a handle.  Two calls in a row (the
static scratch keeps the previous call's contents) must each agree with
ncsim_sv_measure_stats on the same amplitudes to the tolerance of the other
parity tests, and must leave the device's free memory, torch's allocator and
the library's own pool exactly as they were.  Wrong buffers (host memory, a
buffer shorter than the register) are rejected on the host before any
launch.  This file is collected last on purpose.
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
    expected = [ref.measure_stats(p) for p in paulis]
    # the first call on the device does the set-up (the scratch array's address)
    st, _, _ = _noalloc(nb, dev.data_ptr(), n, precision, paulis[0])
    assert st == 0, nb.lib().ncsim_last_error().decode()
    nb.pool_info()  # creates the library's pool on this device, if no call has yet
    torch.cuda.synchronize()
    before = (torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved(), nb.pool_info())
    for p, (e_ref, nn_ref) in zip(paulis, expected):
        st, e, nn = _noalloc(nb, dev.data_ptr(), n, precision, p)
        assert st == 0, nb.lib().ncsim_last_error().decode()
        assert abs(e - e_ref) < TOL and abs(nn - nn_ref) < TOL
    torch.cuda.synchronize()
    after = (torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved(), nb.pool_info())
    assert after == before, (before, after)


def test_noalloc_rejects_wrong_buffers_before_launching(nb):
    n = 12
    p = nb.Pauli(n, 0, 1, 0)
    host = np.zeros(1 << n, dtype=np.complex128)  # pageable host memory
    st, _, _ = _noalloc(nb, host.ctypes.data, n, nb.C128, p)
    assert st == 8 and "host" in nb.lib().ncsim_last_error().decode()
    # a buffer of its own allocation (not carved by torch's caching allocator),
    # holding half the register
    from cuda.bindings import runtime as cudart

    err, ptr = cudart.cudaMalloc(16 << (n - 1))
    assert err == cudart.cudaError_t.cudaSuccess
    try:
        st, _, _ = _noalloc(nb, int(ptr), n, nb.C128, p)
        msg = nb.lib().ncsim_last_error().decode()
        assert st == 8 and "short" in msg, msg
        st, _, _ = _noalloc(nb, int(ptr), n - 1, nb.C128, nb.Pauli(n - 1, 0, 1, 0))  # the right size passes
        assert st == 0, nb.lib().ncsim_last_error().decode()
    finally:
        cudart.cudaFree(ptr)
