"""The GPU side of the sharded register on one device: the shard's halves
(zero-copy torch views of the library's amplitude array) leave and re-enter
the register in index order, its block weights and in-block walks follow the
single-register sampler, and a one-rank ShardedStateVector runs a circuit as
the plain GpuStateVector does.  The exchanges between ranks are covered on
CPU ranks (tests/test_sharded.py)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_gpu_shard_halves_round_trip(nb):
    torch = pytest.importorskip("torch")
    from ncsim_b200.sharded import GpuShard

    nl = 14
    rng = np.random.default_rng(3)
    v = rng.normal(size=1 << nl) + 1j * rng.normal(size=1 << nl)
    sh = GpuShard(nl)
    sh.s.set_amplitudes(v)
    for l, c in ((0, 1), (5, 0), (13, 1)):
        h = sh.half(l, c).cpu().numpy()
        want = v.reshape(1 << (nl - l - 1), 2, 1 << l)[:, c, :].reshape(-1)
        assert np.array_equal(h, want)
    # write the c = 1 half of bit 7 into the c = 0 half
    sh.set_half(7, 0, sh.half(7, 1))
    w = v.reshape(1 << (nl - 8), 2, 1 << 7).copy()
    w[:, 0, :] = w[:, 1, :]
    assert np.array_equal(sh.to_vector(), w.reshape(-1))
    assert torch.cuda.is_available()


def test_block_weights_and_walk_follow_the_sampler(nb):
    n = 15
    c = nb.Circuit.random_layers(n, 6, 2)
    s = nb.GpuStateVector(n)
    s.run(c, nb.StdRng(0))
    w = s.block_weights(4096)
    a = s.to_vector()
    assert np.abs(w - (np.abs(a) ** 2).reshape(-1, 4096).sum(1)).max() < 1e-14
    hi = np.cumsum(w)  # sequential, as the sampler's running sum (vector.rs:501)
    total = hi[-1]
    rng = nb.StdRng(9)
    us = np.array([rng.gen_f64() for _ in range(100)]) * total
    blk = np.minimum(np.searchsorted(hi, us, side="right"), w.size - 1)
    acc = np.where(blk > 0, hi[np.maximum(blk - 1, 0)], 0.0)
    got = s.sample_walk(4096, us, blk, acc)
    assert np.array_equal(got, s.sample(nb.StdRng(9), 100))


def test_one_rank_sharded_register_is_the_plain_register(nb):
    from ncsim_b200.sharded import ShardedStateVector

    n = 16
    text = nb.Circuit.random_layers(n, 8, 5).to_text() + "CCX 15 14 0\nMPP X15*Z3\nM 2\n"
    s = ShardedStateVector(n)
    g = nb.GpuStateVector(n)
    c = nb.Circuit.parse(text)
    assert s.run(c, nb.StdRng(4)) == g.run(c, nb.StdRng(4))
    assert np.abs(s.to_vector() - g.to_vector()).max() < TOL
    p = nb.Pauli.from_string(n, "X15*Y2*Z9")
    assert abs(s.expectation(p) - g.expectation(p)) < TOL
    assert np.array_equal(s.sample(nb.StdRng(8), 300), g.sample(nb.StdRng(8), 300))
