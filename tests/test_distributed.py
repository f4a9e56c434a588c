"""The multi-process path of bench.py on the CPU (gloo, world size 2): the
workload does not shard across GPUs, so N ranks run N replicas and the only
collective is the max-over-ranks of the timed region; the reference arm runs
on rank 0 while the other ranks exit without work."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as tmp

from _oracle import have_reference

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    r, ws, _ = bench.init_dist()
    t = bench.max_over_ranks(float(10 * (rank + 1)))
    bench.barrier()
    Path(out_dir, f"rank{r}.json").write_text(json.dumps({"rank": r, "world": ws, "max": t}))
    bench._dist.destroy_process_group()


def test_max_over_ranks_with_gloo(tmp_path):
    world = 2
    tmp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    assert [g["world"] for g in got] == [world, world]
    assert [g["max"] for g in got] == [20.0, 20.0]


@pytest.mark.skipif(not have_reference("wilson"), reason="reference build absent")
def test_reference_arm_runs_on_rank_zero_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--workload", "n8"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 prints, rank 1 exits without work
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
