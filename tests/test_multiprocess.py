"""The multi-process (N > 1) host logic of bench.py on CPU with the gloo backend, two ranks: the
process-group set-up from the torchrun environment, the barrier, the max over ranks that every timed
figure goes through, and the reference arm under torchrun (rank 0 alone measures and prints one JSON
line, the other rank exits 0 without work).  The B200 arm runs independent replicas (no collective on
the data path), so these are the only cross-rank steps."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    e = dict(os.environ)
    e.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
             MASTER_PORT=str(port), DH_BENCH_BACKEND="gloo", CUDA_VISIBLE_DEVICES="")
    return e


def test_barrier_and_max_over_ranks_gloo():
    port = _free_port()
    code = ("import sys; sys.path.insert(0, %r); import bench, torch.distributed as d; "
            "w, r, l = bench.dist_setup(); bench.barrier(w); "
            "print('max', bench.reduce_max(1.5 + 2.0 * r, w)); d.destroy_process_group()") % ROOT
    procs = [subprocess.Popen([sys.executable, "-c", code], env=_env(r, 2, port), stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err
        assert "max 3.5" in out


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_tool")),
                    reason="the reference is not built here (make -C oracle ref)")
def test_reference_arm_under_torchrun_two_ranks():
    env = dict(os.environ, DH_BENCH_BACKEND="gloo", DH_BENCH_REFERENCE_SECONDS="2", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, env=env, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
