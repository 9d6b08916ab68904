"""bench.py starts its own ranks: ``--gpus N`` without WORLD_SIZE re-launches
the script under torch.distributed.run with N processes (127.0.0.1
rendezvous); ``--launch-check`` makes each rank report RANK / WORLD_SIZE and
exit before touching a GPU, so this runs on CPU."""

import json
import os
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _ranks(extra_env=None, gpus=2):
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env.update(extra_env or {})
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", str(gpus),
                        "--launch-check"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    # the ranks write concurrently: take every JSON object, however the lines interleave
    return [json.loads(m) for m in re.findall(r"\{[^{}]*\}", r.stdout)]


def test_gpus_2_starts_two_ranks():
    got = _ranks()
    assert sorted(g["rank"] for g in got) == [0, 1]
    assert all(g["world"] == 2 for g in got)


def test_gpus_1_runs_in_process():
    got = _ranks(gpus=1)
    assert got == [{"rank": 0, "local_rank": 0, "world": 1}]


def test_world_size_mismatch_is_an_error():
    env = {k: v for k, v in os.environ.items()}
    env.update({"WORLD_SIZE": "3", "RANK": "0", "LOCAL_RANK": "0"})
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--launch-check"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode != 0
    assert "WORLD_SIZE=3" in r.stderr
