"""The bench's multi-rank path on CPU (gloo, world size 2): replicas only, so
the only collectives are the timing reductions (max of device times, sum of
attempts) and barriers; each rank builds its own seeded batch. The reference
arm under two ranks prints one line from rank 0 and exits 0 on the others."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local = bench.dist_setup()
    d = bench.Dist(ws, r, "gloo")
    d.barrier()
    mx = d.max(10.0 + r)
    sm = d.sum(1.0 + r)
    models, seeds, _ = bench.make_workload(3, 5 + 7919 * r, 4)
    out.put((r, mx, sm, [m.num_vars for m in models], int(seeds[0])))
    d.close()


def test_timing_reductions_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[1] for x in res] == [11.0, 11.0]  # device time: max over ranks
    assert [x[2] for x in res] == [3.0, 3.0]    # attempts: sum over ranks
    assert res[0][3] != res[1][3] or res[0][4] != res[1][4]  # each rank its own batch


@pytest.mark.timeout(600)
def test_reference_arm_two_ranks():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--count", "16", "--sweeps", "20", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0
