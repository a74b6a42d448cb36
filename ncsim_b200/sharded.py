"""A dense register sharded over 2^g processes, one GPU each.

The reference's ``StateVector`` (src/state/vector.rs) holds one array of 2^n
amplitudes; here rank r of a process group of W = 2^g ranks holds the 2^(n-g)
amplitudes whose top g physical index bits equal r, in a ``GpuStateVector``
on its own GPU.  Logical qubit q sits at physical position ``pos[q]``:
positions below n - g are local bits, the others are rank bits.

- A gate whose qubits are all local runs on every rank's shard with no
  communication (the same kernels as the single-GPU register).
- A gate on a global qubit first swaps that qubit with a local one that the
  gate does not use: each rank sends the half of its shard whose local bit
  differs from its rank bit to the partner rank across that bit and receives
  the partner's matching half (a point-to-point exchange of 2^(n-g-1)
  amplitudes per rank), and the qubit map is updated.  No amplitude moves
  otherwise.
- Pauli operators (expectation, projection, measurement) map their X part
  into local bits the same way; their Z part on rank bits becomes a phase
  i^(2 popcount(z_rank & r)) per rank.
- Sums (norm, expectations, projection weights) are per-shard FP64 sums and
  one all-reduce.
- Sampling restores the identity layout, gathers every shard's block weights
  (blocks of 4096 amplitudes, none spanning two ranks), runs the reference's
  sequential running sum over all blocks on every rank (vector.rs:494-540),
  and lets the owner of each shot's block walk it.

Measurements draw from the generator each rank passes (all ranks pass
generators in the same state, so every rank draws the same uniform and takes
the same branch).  The shard object is injectable so that the partition and
exchange logic can run on CPU ranks (gloo) with a host array per rank; the
product path is the GPU shard over NCCL.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import C128, GpuStateVector, Pauli, SimError, Circuit, Gate, StdRng

BLOCK = 4096


class GpuShard:
    """One rank's part of the register: a ``GpuStateVector`` on this process's GPU,
    with zero-copy torch views of its halves for the exchanges."""

    device = "cuda"

    def __init__(self, nl: int, precision: int = C128):
        self.nl = nl
        self.s = GpuStateVector(nl, precision)

    # ---- state operations (local qubit positions) ----
    def apply_gate(self, gate: Gate, qubits: Sequence[int]) -> None:
        self.s.apply_gate(gate, qubits)

    def apply_pauli(self, x: int, z: int, phase: int) -> None:
        self.s.apply_pauli(Pauli(self.nl, x, z, phase))

    def measure_stats(self, x: int, z: int, phase: int):
        return self.s.measure_stats(Pauli(self.nl, x, z, phase))

    def expectation(self, x: int, z: int, phase: int) -> complex:
        return self.s.expectation(Pauli(self.nl, x, z, phase))

    def project(self, x: int, z: int, phase: int, outcome: bool) -> float:
        return self.s.project(Pauli(self.nl, x, z, phase), outcome).real

    def norm_sq(self) -> float:
        return self.s.norm_sq().real

    def scale(self, c: complex) -> None:
        self.s.scale(c)

    def amplitude(self, i: int) -> complex:
        return self.s.amplitude(i)

    def to_vector(self) -> np.ndarray:
        return self.s.to_vector()

    def block_weights(self) -> np.ndarray:
        return self.s.block_weights(BLOCK)

    def sample_walk(self, targets, blocks, accs) -> np.ndarray:
        return self.s.sample_walk(BLOCK, targets, blocks, accs)

    # ---- halves for the exchanges ----
    def _half_view(self, l: int, c: int):
        v = self.s.torch_view()
        return v.view(1 << (self.nl - l - 1), 2, 1 << l)[:, c, :]

    def half(self, l: int, c: int):
        """A contiguous copy of the amplitudes whose local bit l is c, in index order."""
        import torch

        self.s.synchronize()
        out = self._half_view(l, c).contiguous().view(-1)
        torch.cuda.synchronize()
        return out

    def set_half(self, l: int, c: int, data) -> None:
        import torch

        self._half_view(l, c).copy_(data.view(1 << (self.nl - l - 1), 1 << l))
        torch.cuda.synchronize()

    def empty_like_half(self, l: int):
        import torch

        return torch.empty(1 << (self.nl - 1), dtype=torch.complex128, device="cuda")


def _check_qubits(qubits: Sequence[int], n: int) -> None:
    """check_qubits (src/error.rs:69-82)."""
    for i, q in enumerate(qubits):
        if q >= n:
            raise SimError(2, f"qubit {q} out of range for {n} qubits", {"qubit": q, "num_qubits": n})
        if q in qubits[:i]:
            raise SimError(4, f"qubit {q} listed twice", {"qubit": q})


class ShardedStateVector:
    """|0...0> on ``n`` qubits over the ranks of ``group`` (a power-of-two count)."""

    BACKEND = "ShardedStateVector"

    def __init__(self, n: int, group=None, shard_factory=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.world = dist.get_world_size(group)
            self.rank = dist.get_rank(group)
        else:
            self.world, self.rank = 1, 0
        g = self.world.bit_length() - 1
        if (1 << g) != self.world:
            raise SimError(8, f"a sharded register needs a power-of-two number of ranks, not {self.world}")
        if n - g < 13:
            raise SimError(8, f"{n} qubits over {self.world} ranks leave fewer than 13 local qubits")
        self.n, self.g, self.nl = n, g, n - g
        self.shard = (shard_factory or GpuShard)(self.nl)
        if self.rank != 0:
            self.shard.scale(0.0)  # |0...0> lives in rank 0's first amplitude
        self.pos = list(range(n))  # logical qubit -> physical position
        self.at = list(range(n))   # physical position -> logical qubit
        self.exchanges = 0         # half-shard exchanges so far

    # ---- communication ----
    def _comm_device(self):
        return getattr(self.shard, "device", "cpu")

    def _allreduce(self, values: Sequence[float]) -> np.ndarray:
        import torch

        t = torch.tensor(list(values), dtype=torch.float64, device=self._comm_device())
        if self.world > 1:
            self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def _swap(self, p: int, l: int) -> None:
        """Swaps physical positions p (a rank bit) and l (a local bit)."""
        import torch.distributed as dist

        j = p - self.nl
        b = (self.rank >> j) & 1
        partner = self.rank ^ (1 << j)
        if self.group is not None:
            partner = dist.get_global_rank(self.group, partner)
        send = self.shard.half(l, 1 - b)
        recv = self.shard.empty_like_half(l)
        ops = [dist.P2POp(dist.isend, send, partner, self.group), dist.P2POp(dist.irecv, recv, partner, self.group)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        self.shard.set_half(l, 1 - b, recv)
        qa, qb = self.at[p], self.at[l]
        self.pos[qa], self.pos[qb] = l, p
        self.at[l], self.at[p] = qa, qb
        self.exchanges += 1

    def _localize(self, logical: Sequence[int], keep: Sequence[int] = ()) -> None:
        """Brings the given logical qubits into local positions, swapping each global one
        with the highest local position that holds none of them (preferring one that
        holds none of `keep` either, whose qubits are only moved when nothing else is free)."""
        need = {self.pos[q] for q in logical}
        pref = {self.pos[q] for q in keep}
        for q in logical:
            p = self.pos[q]
            if p < self.nl:
                continue
            free = [l for l in range(self.nl - 1, -1, -1) if l not in need]
            if not free:
                raise SimError(1, "the operator touches every local qubit and a global one")
            l = next((f for f in free if f not in pref), free[0])
            self._swap(p, l)
            need.add(l)

    def _restore_layout(self) -> None:
        """The identity layout (logical qubit q at physical position q)."""
        for p in range(self.n - 1, -1, -1):
            q = self.at[p]
            if q == p:
                continue
            src = self.pos[p]  # where logical qubit p sits now
            a, b = min(src, p), max(src, p)
            if b < self.nl:  # both local: a SWAP gate on every shard
                self.shard.apply_gate(Gate.parse("SWAP"), [a, b])
                qa, qb = self.at[a], self.at[b]
                self.pos[qa], self.pos[qb] = b, a
                self.at[a], self.at[b] = qb, qa
            elif a < self.nl:
                self._swap(b, a)
            else:  # both global: through a local position
                t = self.nl - 1
                self._swap(a, t)
                self._swap(b, t)
                self._swap(a, t)

    # ---- masks ----
    def _phys_mask(self, m: int) -> int:
        out = 0
        for q in range(self.n):
            if (m >> q) & 1:
                out |= 1 << self.pos[q]
        return out

    def _local_pauli(self, p: Pauli):
        """(x, z, phase) on the local bits of a Pauli whose X part is local."""
        xs = [q for q in range(self.n) if (p.x >> q) & 1]
        zs = [q for q in range(self.n) if (p.z >> q) & 1]
        self._localize(xs, keep=zs)
        x, z = self._phys_mask(p.x), self._phys_mask(p.z)
        lmask = (1 << self.nl) - 1
        zr = z >> self.nl
        ph = (p.phase + 2 * bin(zr & self.rank).count("1")) & 3
        return x & lmask, z & lmask, ph

    # ---- the QuantumState<C64> methods ----
    def num_qubits(self) -> int:
        return self.n

    def apply_gate(self, gate: Gate, qubits: Sequence[int]) -> None:
        """vector.rs:364-372 checks, then the gate on local positions."""
        qubits = list(qubits)
        _check_qubits(qubits, self.n)
        if len(qubits) != gate.arity:
            raise SimError(3, f"gate {gate.label} acts on {gate.arity} qubits, {len(qubits)} given",
                           {"gate": gate.label, "expected": gate.arity, "got": len(qubits)})
        self._localize(qubits)
        self.shard.apply_gate(gate, [self.pos[q] for q in qubits])

    def apply_pauli(self, p: Pauli) -> None:
        self.shard.apply_pauli(*self._local_pauli(p))

    def norm_sq(self) -> float:
        return float(self._allreduce([self.shard.norm_sq()])[0])

    def expectation(self, p: Pauli) -> complex:
        e = self.shard.expectation(*self._local_pauli(p))
        r = self._allreduce([e.real, e.imag])
        return complex(r[0], r[1])

    def project(self, p: Pauli, outcome: bool) -> float:
        if not p.is_hermitian():
            raise SimError(8, "projector of a non-Hermitian Pauli")
        w = self.shard.project(*self._local_pauli(p), outcome)
        return float(self._allreduce([w])[0])

    def measure(self, p: Pauli, rng: StdRng) -> bool:
        """QuantumState::measure (src/state/mod.rs:113-131): <P> and <psi|psi> from
        one pass and one all-reduce, a draw only when the outcome is uncertain."""
        if not p.is_hermitian():
            raise SimError(8, "measured operator is not Hermitian")
        x, z, ph = self._local_pauli(p)
        e, nn = self.shard.measure_stats(x, z, ph)
        r = self._allreduce([e.real, nn])
        p_plus = min(1.0, max(0.0, (1.0 + float(r[0]) / float(r[1])) / 2.0))
        if p_plus > 1.0 - 1e-12:
            outcome = False
        elif p_plus < 1e-12:
            outcome = True
        else:
            outcome = bool(rng.gen_f64() >= p_plus)
        self.shard.project(x, z, ph, outcome)
        return outcome

    def scale(self, c: complex) -> None:
        self.shard.scale(c)

    def amplitude(self, index: int) -> complex:
        phys = self._phys_mask(index)
        owner, local = phys >> self.nl, phys & ((1 << self.nl) - 1)
        a = self.shard.amplitude(local) if owner == self.rank else 0j
        r = self._allreduce([a.real, a.imag])
        return complex(r[0], r[1])

    def run(self, circuit: Circuit, rng: StdRng) -> list[bool]:
        """QuantumState::run (src/state/mod.rs:168-183) for circuits of gates, Pauli
        measurements, resets and annotations."""
        if circuit.num_qubits != self.n:
            raise SimError(8, f"circuit on {circuit.num_qubits} qubits, state on {self.n}")
        rec = []
        for line in circuit.to_text().splitlines()[1:]:
            toks = line.split()
            if not toks:
                continue
            name, args = toks[0], toks[1:]
            if name in ("TICK", "DETECTOR") or name.startswith("OBSERVABLE_INCLUDE"):
                continue
            if name in ("MX", "MY", "MZ"):
                rec.append(self.measure(Pauli.from_string(self.n, f"{name[1]}{args[0]}"), rng))
            elif name == "MPP":
                rec.append(self.measure(Pauli.from_string(self.n, args[0]), rng))
            elif name == "R":
                q = int(args[0])
                if self.measure(Pauli.z_on(self.n, q), rng):
                    self.apply_gate(Gate.parse("X"), [q])
            elif name.split("(")[0] in ("X_ERROR", "Y_ERROR", "Z_ERROR", "DEPOLARIZE1", "DEPOLARIZE2",
                                        "PAULI_CHANNEL_1"):
                raise SimError(1, "noise channels on the sharded register")
            else:
                qs = [int(a) for a in args]
                self.apply_gate(Gate.parse(name, len(qs)), qs)
        return rec

    def sample(self, rng: StdRng, shots: int) -> np.ndarray:
        """StateVector::sample (vector.rs:494-540) over all shards: the same blocks,
        the same sequential running sum, the same walk inside each shot's block."""
        import torch

        self._restore_layout()
        w = np.ascontiguousarray(self.shard.block_weights(), dtype=np.float64)
        per = w.size
        if self.world > 1:
            t = torch.from_numpy(w).to(self._comm_device())
            parts = [torch.empty_like(t) for _ in range(self.world)]
            self.dist.all_gather(parts, t, group=self.group)
            w = torch.cat(parts).cpu().numpy()
        hi = np.empty_like(w)
        total = 0.0
        for b in range(w.size):  # the reference's sequential sum (vector.rs:501)
            total += w[b]
            hi[b] = total
        if not total > 0.0:
            raise SimError(6, "state vanished: sample")
        u = np.array([rng.gen_f64() for _ in range(shots)]) * total
        blk = np.minimum(np.searchsorted(hi, u, side="right"), w.size - 1)
        acc = np.where(blk > 0, hi[np.maximum(blk - 1, 0)], 0.0)
        mine = (blk // per) == self.rank
        out = np.zeros(shots, dtype=np.int64)
        if mine.any():
            idx = self.shard.sample_walk(u[mine], (blk[mine] % per).astype(np.uint64), acc[mine])
            out[mine] = (np.int64(self.rank) << self.nl) | idx.astype(np.int64)
        if self.world > 1:
            t = torch.from_numpy(out).to(self._comm_device())
            self.dist.all_reduce(t, group=self.group)
            out = t.cpu().numpy()
        return out.astype(np.uint64)

    def to_vector(self) -> np.ndarray:
        """All 2^n amplitudes in logical order (every rank gets them; small registers)."""
        import torch

        self._restore_layout()
        v = self.shard.to_vector()
        if self.world == 1:
            return v
        t = torch.from_numpy(np.ascontiguousarray(v).view(np.float64)).to(self._comm_device())
        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(parts, t, group=self.group)
        return torch.cat(parts).cpu().numpy().view(np.complex128)
