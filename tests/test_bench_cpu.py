"""bench.py's launcher and rank logic on the CPU (gloo, no GPU work): `--gpus N` re-runs the
command as N ranks under torch.distributed.run, every rank takes the barrier and the
max-reduction of the timed arms, and the one printed line reports n_gpus = N."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO


def _run(*args, env=None):
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        e.pop(k, None)
    e.update(env or {})
    res = subprocess.run([sys.executable, str(REPO / "bench.py"), *args], capture_output=True,
                         text=True, timeout=300, env=e, cwd=str(REPO))
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    return res, lines


@pytest.mark.parametrize("n", [1, 2])
def test_gpus_flag_launches_that_many_ranks(n):
    res, lines = _run("--gpus", str(n), "--dry")
    assert res.returncode == 0, res.stderr[-2000:]
    assert len(lines) == 1, res.stdout  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["n_gpus"] == n and line["gpus_requested"] == n
    assert line["ranks_seen"] == n and line["max_rank"] == n - 1


def test_world_size_must_match_gpus():
    res, lines = _run("--gpus", "2", "--dry",
                      env={"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert res.returncode != 0
    assert "--gpus 2 but 1 rank(s)" in (res.stderr + res.stdout)
    assert not lines
