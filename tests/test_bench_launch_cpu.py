"""bench.py --gpus N: the rank launcher (CPU, gloo).  Without a process group
the script starts N ranks itself; inside one, --gpus must match WORLD_SIZE."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(REPO, "bench.py")


def _env():
    return {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}


def test_gpus_two_starts_two_ranks():
    r = subprocess.run([sys.executable, BENCH, "--gpus", "2", "--launch-check"], env=_env(), capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert line == {"n_gpus": 2, "max_over_ranks": 2.0}


def test_gpus_one_runs_in_process():
    r = subprocess.run([sys.executable, BENCH, "--gpus", "1", "--launch-check"], env=_env(), capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1]) == {"n_gpus": 1, "max_over_ranks": 1.0}


def test_gpus_must_match_the_process_group():
    env = dict(_env(), WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, BENCH, "--gpus", "4", "--launch-check"], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 2
    assert "WORLD_SIZE" in r.stderr


def test_launch_command_uses_loopback():
    sys.path.insert(0, REPO)
    import bench
    cmd = bench.launch_command(["--gpus", "8", "--steps", "5"], 8, 12345)
    assert cmd[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert cmd[cmd.index("--nproc-per-node") + 1] == "8"
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-4:] == ["--gpus", "8", "--steps", "5"]
