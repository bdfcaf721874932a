"""bench.py's rotation-sharded step (GPU): two ranks that share the one GPU here
(gloo collectives on host copies, MD_BENCH_BACKEND=gloo; nothing waits across
the ranks on the device) each dock half of the 54,000 rotations; the
all-gathered records of the timed step equal the reference's goldens at every
checked rotation and the line reports the two-rank job."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def test_bench_two_rotation_shards(built, gpu):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2", "--master-addr",
           "127.0.0.1", f"--master-port={port}", "bench.py", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--batch", "64", "--no-cpu-baseline", "--no-cufft"]
    res = subprocess.run(cmd, cwd=ROOT, env=dict(os.environ, MD_BENCH_BACKEND="gloo"), capture_output=True,
                         text=True, timeout=1200)
    assert res.returncode == 0, res.stderr[-3000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, res.stdout[-2000:]
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["scaling"] == "strong"
    assert line["config"]["parallelism"].startswith("rotation shards x2")
    par = line["parity"]
    assert par["rotation_indices_ok"] and par["within_1e-4"] and par["cells_equal"] == par["poses_checked"] == 10800
    assert line["value"] > 0 and line["e2e"]["value"] > 0
