"""One process per GPU for a script started as a single process.

`ensure_ranks(n)` is the first call of a multi-GPU entry point such as
bench.py.  Started without a launcher (no WORLD_SIZE in the environment) and
asked for n > 1 ranks, it replaces the process with torch.distributed.run
over n local ranks, running the same script with the same arguments, under
`timeout -k 60` as the last bound on a rank that waits for good.  Inside the
ranks (or for n = 1) it returns (rank, world_size, local_rank) from the
environment and fails loudly when the launcher started a different number of
ranks than asked for.
"""
import os
import shutil
import socket
import sys


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_command(n, script, argv, limit_s=None):
    """The command that runs `script argv` as n local ranks."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), script] + list(argv)
    if limit_s and shutil.which("timeout"):
        cmd = ["timeout", "-k", "60", str(int(limit_s))] + cmd
    return cmd


def ensure_ranks(n, script=None, argv=None, limit_s=3600):
    n = int(n)
    if n < 1:
        raise ValueError("need at least one rank")
    env_world = os.environ.get("WORLD_SIZE")
    if env_world is None and n > 1:
        script = os.path.abspath(script or sys.argv[0])
        argv = sys.argv[1:] if argv is None else argv
        cmd = launch_command(n, script, argv, limit_s)
        sys.stdout.flush()
        sys.stderr.flush()
        os.execvp(cmd[0], cmd)   # does not return
    world = int(env_world or 1)
    if world != n:
        raise RuntimeError("started as %d ranks, asked for %d" % (world, n))
    return int(os.environ.get("RANK", "0")), world, int(os.environ.get("LOCAL_RANK", "0"))
