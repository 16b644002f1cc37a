"""The multi-GPU launcher of bench.py (dice_b200.launch) on the CPU: a
script started as one process and asked for two ranks re-runs itself under
torch.distributed.run, and both ranks meet in a world_size-2 gloo group."""
import os
import subprocess
import sys
import textwrap

import pytest

from dice_b200 import launch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import os, sys
    sys.path.insert(0, {root!r})
    from datetime import timedelta
    from dice_b200 import launch
    n = int(sys.argv[1])
    out = sys.argv[2]
    rank, world, local = launch.ensure_ranks(n)
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("gloo", timeout=timedelta(seconds=60))
        t = torch.tensor([rank + 1.0])
        dist.all_reduce(t)
        total = float(t.item())
        dist.destroy_process_group()
    else:
        total = 1.0
    with open(os.path.join(out, "rank%d.txt" % rank), "w") as f:
        f.write("%d %d %d %g" % (rank, world, local, total))
""")


def _run(tmp_path, n):
    script = tmp_path / "ranks.py"
    script.write_text(SCRIPT.format(root=ROOT))
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, str(script), str(n), str(tmp_path)], env=env, capture_output=True,
                       text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    return sorted(p.read_text() for p in tmp_path.glob("rank*.txt"))


def test_two_ranks_from_one_process(tmp_path):
    got = _run(tmp_path, 2)
    assert got == ["0 2 0 3", "1 2 1 3"]


def test_one_rank_runs_in_place(tmp_path):
    assert _run(tmp_path, 1) == ["0 1 0 1"]


def test_world_size_mismatch_fails(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "2")
    with pytest.raises(RuntimeError):
        launch.ensure_ranks(4)


def test_launch_command_bounds_the_ranks():
    cmd = launch.launch_command(8, "bench.py", ["--gpus", "8"], limit_s=900)
    assert "torch.distributed.run" in cmd and "--nproc-per-node" in cmd
    assert cmd[cmd.index("--nproc-per-node") + 1] == "8"
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    if cmd[0] == "timeout":
        assert cmd[1:4] == ["-k", "60", "900"]
