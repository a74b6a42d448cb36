"""The multi-GPU path on CPU: `bench.py --gpus N` runs N independent replicas
(the path has no data exchange between replicas), one rank per GPU, timed as
the max over ranks.  These tests run its rank plumbing with the gloo backend
and two ranks on 127.0.0.1; no GPU is needed.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_and_barrier_gloo():
    port = _free_port()
    script = textwrap.dedent(f"""
        import os, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        dist = bench.dist_init()
        v = bench.max_over_ranks(dist, 1.5 + bench.RANK)
        bench.barrier(dist)
        print("RESULT", bench.RANK, bench.WORLD, v, flush=True)
        dist.destroy_process_group()
    """)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=300)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    got = sorted(tuple(l.split()[1:]) for o in outs for l in o.splitlines() if l.startswith("RESULT"))
    assert got == [("0", "2", "2.5"), ("1", "2", "2.5")]


def test_reference_arm_prints_once_on_two_ranks():
    """`--impl reference` under torchrun: rank 0 times the CPU path and prints the
    one JSON line; the other rank exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--qubits", "14",
           "--cpu-budget", "0.2", "--no-trajectories"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port"
