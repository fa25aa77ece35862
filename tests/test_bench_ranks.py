"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): every rank
takes the same collective steps, the device time is the max over ranks and
the units are summed; the reference arm runs on rank 0 only."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


_WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
rank, world, local = bench.dist_setup()
assert world == 2 and rank in (0, 1)
bench.barrier(world)
elapsed, units = bench.aggregate(0.5 + rank, 100.0 * (rank + 1), world)
# the reference arm: rank 0 prints, rank 1 returns without work
bench.cpu_reference_run = lambda steps, warmup: {{"value": 1.0, "unit": bench.UNIT, "cores": 1, "kind": "reference",
                                                   "sample": "stub"}}
class A: steps = 2; warmup = 1; grid = "64x128x64"
rc = bench.reference_arm(A, rank, world)
print(json.dumps({{"rank": rank, "elapsed": elapsed, "units": units, "rc": rc}}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def test_two_gloo_ranks_take_max_time_and_summed_units(tmp_path):
    port = _free_port()
    script = tmp_path / "worker.py"
    script.write_text(_WORKER.format(root=ROOT))
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("gloo ranks did not finish")
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    lines = [[json.loads(l) for l in o.splitlines() if l.startswith("{")] for o in outs]
    res = {d["rank"]: d for ls in lines for d in ls if "rank" in d}
    assert res[0]["elapsed"] == res[1]["elapsed"] == 1.5
    assert res[0]["units"] == res[1]["units"] == 300.0
    ref0 = [d for d in lines[0] if d.get("impl") == "reference"]
    ref1 = [d for d in lines[1] if d.get("impl") == "reference"]
    assert len(ref0) == 1 and ref1 == []
    assert ref0[0]["n_gpus"] == 2 and ref0[0]["e2e"]["h2d_bytes_per_step"] == 0
