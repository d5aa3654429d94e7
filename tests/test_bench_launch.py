"""bench.py honours --gpus N: it starts N ranks itself when no launcher did, and refuses a launcher
whose world size differs, so a run never reports a GPU count other than the one requested."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_launch_plan():
    assert bench.launch_plan(1, {}) == "run"
    assert bench.launch_plan(2, {}) == "spawn"
    assert bench.launch_plan(8, {"WORLD_SIZE": "8"}) == "run"
    assert bench.launch_plan(1, {"WORLD_SIZE": "1"}) == "run"
    with pytest.raises(SystemExit):
        bench.launch_plan(2, {"WORLD_SIZE": "1"})
    with pytest.raises(SystemExit):
        bench.launch_plan(0, {})


def _run(env_extra, *args):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env.update(env_extra)
    env["CUDA_VISIBLE_DEVICES"] = ""  # no device: every rank stops before any model is built
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=env, cwd=ROOT,
                          capture_output=True, text=True, timeout=600)


def test_gpus_2_under_a_one_rank_launcher_is_refused():
    r = _run({"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"}, "--gpus", "2", "--steps", "1")
    assert r.returncode != 0
    assert "WORLD_SIZE=1" in r.stderr
    assert '"n_gpus"' not in r.stdout


def test_gpus_2_without_a_launcher_starts_two_ranks():
    r = _run({}, "--gpus", "2", "--steps", "1")
    # torch.distributed.run started two ranks (it reports the per-process thread setting only for
    # more than one process, and names local rank 1 when it ends them); a rank stops for want of a
    # CUDA device, the launcher ends the other, and nothing is reported
    out = r.stdout + r.stderr
    assert r.returncode != 0
    assert "for each process" in out, out[-2000:]
    assert "no CUDA device" in out, out[-2000:]
    assert "local_rank: 1" in out, out[-2000:]
    assert '"n_gpus"' not in r.stdout
