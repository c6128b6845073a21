"""Multi-GPU runs are independent replicas (diablo3_b200/replicas.py): the
host logic of a 2-rank job, run as two gloo processes on the CPU - the
MAX of the ranks' times, the whole-job rate, barriers and teardown - and the
reference arm's rule that only rank 0 works and prints."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
torch = pytest.importorskip("torch")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from diablo3_b200 import replicas
    r = replicas.from_env()
    replicas.init(r, "gloo", timeout_s=60.0)
    replicas.barrier(r)
    ms = 10.0 + 5.0 * rank                   # the slower rank sets the job time
    ms_max = replicas.max_over_ranks(r, ms, device="cpu")
    rate = replicas.job_rate(1000, 3, r, ms_max)
    out.put((rank, r.leader, ms_max, rate))
    replicas.finish(r)


def test_two_gloo_ranks_reduce_max_and_rate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [True, False]
    for _, _, ms_max, rate in got:
        assert ms_max == 15.0
        assert rate == pytest.approx(1000 * 3 * 2 / 0.015)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from diablo3_b200 import replicas
    r = replicas.Ranks(1, 0, 0)
    replicas.init(r)
    assert replicas.max_over_ranks(r, 7.5) == 7.5
    assert replicas.job_rate(10, 3, r, 1000.0) == 30.0
    replicas.finish(r)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
