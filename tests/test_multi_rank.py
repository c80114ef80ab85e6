"""The multi-rank path of bench.py on CPU: two gloo ranks (one process per GPU on a
GPU box, NCCL there).  Every rank takes the same collective steps; timing is the
max over ranks; under torchrun only rank 0 runs the reference arm and prints."""

import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_and_barrier_gloo():
    port = _free_port()
    code = (
        "import os, sys; sys.path.insert(0, %r); import bench\n"
        "w, r, l = bench.dist_init()\n"
        "m = bench.max_over_ranks(1.5 + r, w)\n"
        "bench.barrier(w)\n"
        "print('RESULT', r, m, bench._BACKEND, flush=True)\n"
        "import torch.distributed as dist; dist.destroy_process_group()\n" % ROOT)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CVDV_DIST_BACKEND="gloo")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=120)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    for rank, out in enumerate(outs):
        line = [x for x in out.splitlines() if x.startswith("RESULT")][0].split()
        assert int(line[1]) == rank and float(line[2]) == 2.5 and line[3] == "gloo"


def test_reference_arm_two_ranks_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--workload", "small"]
    env = dict(os.environ, CVDV_DIST_BACKEND="gloo", OMP_NUM_THREADS="2")
    res = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
