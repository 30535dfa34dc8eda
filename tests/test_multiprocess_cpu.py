"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the max-over-ranks timing
reduction, and the reference arm under torchrun -- rank 0 alone runs the CPU reference and
prints one JSON line, the other ranks exit 0 without work."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=rank, world_size=world)
m = bench.max_over_ranks(1.5 + rank, world, "cpu")
print("MAX", rank, m, flush=True)
class A:
    config, steps, warmup = "c1", 1, 1
rc = bench.run_reference(A(), rank, world)
print("RC", rank, rc, flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo(oa, tmp_path):
    pytest.importorskip("torch.distributed")
    port = _free_port()
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=str(ROOT), port=port))
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=300)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    for rank, out in enumerate(outs):
        assert f"MAX {rank} 2.5" in out
        assert f"RC {rank} 0" in out
    lines0 = [ln for ln in outs[0].splitlines() if ln.startswith("{")]
    lines1 = [ln for ln in outs[1].splitlines() if ln.startswith("{")]
    assert len(lines0) == 1 and not lines1
    rec = json.loads(lines0[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] == "port"
