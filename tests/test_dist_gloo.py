"""The multi-rank path of bench.py on CPU: two gloo ranks (127.0.0.1) -- process-group
set-up, the max-over-ranks timing reduction, the barrier, and the reference arm under
torchrun (rank 0 prints the one JSON line, the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, _ = bench.dist_setup(None)
    value = bench.max_over_ranks(1.5 + r, w)
    bench.barrier(w)
    q.put((r, w, value, dist.get_backend()))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_the_max():
    port = free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2, 2.5, "gloo"), (1, 2, 2.5, "gloo")]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "honei_ref"))
                    and not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")),
                    reason="neither the reference build nor the oracle library is built")
def test_reference_arm_under_torchrun_prints_one_line():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--level", "4"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] in ("reference", "port")
