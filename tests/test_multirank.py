"""The multi-process path of bench.py on the CPU: two ranks over gloo
(127.0.0.1).  Photons shard across ranks with no data-path collective; the
only collectives are the barrier and the maximum of the step times over
ranks, and the reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO


def free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


WORKER = r"""
import os, sys, json
sys.path.insert(0, {repo!r})
import torch.distributed as dist
import bench
world, rank, local = bench.init_dist()
assert dist.get_backend() == "gloo"
bench.barrier(world)
m = bench.max_over_ranks(float(10 + rank), world)
print(json.dumps({{"rank": rank, "world": world, "max": m}}), flush=True)
dist.destroy_process_group()
"""


def run_ranks(code: str, n: int = 2, timeout: int = 120):
    port = free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=REPO,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_max_over_ranks_and_barrier_over_gloo():
    outs = run_ranks(WORKER.format(repo=REPO))
    lines = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    assert all(l["world"] == 2 and l["max"] == 11.0 for l in lines)


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_build", "libmerlict_oracle.so")),
                    reason="oracle not built")
def test_reference_arm_prints_one_line_from_rank_zero():
    """--impl reference under two ranks: rank 0 times the CPU path and prints
    the one JSON line; rank 1 exits 0 without work."""
    code = (f"import sys; sys.path.insert(0, {REPO!r}); sys.argv = ['bench.py', '--impl', "
            "'reference', '--gpus', '2', '--steps', '1', '--warmup', '0', '--ref-photons', '2000']; "
            "import bench; bench.main()")
    outs = run_ranks(code, timeout=600)
    printed = [o for o in outs if o.strip()]
    assert len(printed) == 1
    line = json.loads(printed[0].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["cpu_baseline"]["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
