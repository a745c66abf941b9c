"""The multi-rank protocol of bench.py (one replica per GPU, max-over-ranks
timing, whole-job rate), run as two gloo ranks on the CPU; the rank != 0
exit of the CPU reference arm; and bench.py starting its own ranks when no
launcher set WORLD_SIZE."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from freeflow_b200 import replicas as R

    assert R.env_ranks() == (rank, world, rank)
    R.init("gloo", timeout_s=30.0)
    R.barrier()
    ms = 10.0 + 5.0 * rank                        # this rank's timed region
    ms_max = R.max_over_ranks(ms)
    rate = R.whole_job_rate(1000.0, ms_max * 1e-3, world)
    out.put((rank, ms_max, rate))
    R.shutdown()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    assert [r[1] for r in res] == [15.0, 15.0]      # both ranks see the maximum
    assert all(abs(r[2] - 2 * 1000.0 / 0.015) < 1e-6 for r in res)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from freeflow_b200 import replicas as R

    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        assert R.env_ranks() == (0, 1, 0)
        R.init("gloo")                               # no-op for one process
        assert R.max_over_ranks(3.5) == 3.5
        assert R.whole_job_rate(10.0, 2.0, 1) == 5.0
    finally:
        os.environ.update(env)


def test_reference_arm_exits_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_bench_starts_its_own_ranks():
    """`bench.py --gpus 2` without a launcher runs two processes, ranks 0 and 1
    of a world of 2, which meet over gloo (--check-ranks does no GPU work)."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--check-ranks"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1                        # rank 0 prints, rank 1 does not
    seen = json.loads(lines[0])["check_ranks"]
    assert [(x["rank"], x["world"], x["local_rank"]) for x in seen] == [(0, 2, 0), (1, 2, 1)]
    assert seen[0]["pid"] != seen[1]["pid"]       # two processes


def test_bench_launch_reports_a_failed_rank():
    """A rank that fails makes the launch fail (its exit code comes back)."""
    sys.path.insert(0, ROOT)
    from freeflow_b200 import replicas as R

    code = "import os, sys; sys.exit(3 if os.environ['RANK'] == '1' else 0)"
    assert R.launch_local_ranks(["-c", code], 2) == 3
