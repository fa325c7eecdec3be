"""The multi-GPU form is independent replicas (one process per GPU, no data-path
collective).  Its host logic -- rank environment, barrier, maximum of the ranks'
timings, whole-job rate, only rank 0 reporting, a short process-group timeout -- is
tested here with two gloo ranks on the CPU (127.0.0.1), including a rank that fails
before the collective: the other rank must end with an error, not hang."""
import os
import socket
import time

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _setenv(rank, world, port):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))


def _timed_rank(rank, world, port, out):
    from lddmm_b200 import replicas

    _setenv(rank, world, port)
    env = replicas.rank_env()
    dist = replicas.init(env, "gloo", timeout_s=30)
    replicas.barrier(dist)
    seconds = 0.25 + 0.5 * rank  # rank 1 is the slow one
    slowest = replicas.max_over_ranks(dist, seconds)
    rate = replicas.job_rate(3, env.world, slowest)
    replicas.barrier(dist)
    replicas.finish(dist)
    out.put((env.rank, env.reports, slowest, rate))


def test_two_ranks_max_and_rate():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_timed_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    assert [g[1] for g in got] == [True, False]  # only rank 0 prints the line
    for _, _, slowest, rate in got:
        assert slowest == pytest.approx(0.75)          # the max over ranks, on every rank
        assert rate == pytest.approx(3 * 2 / 0.75)     # all ranks' units / slowest time


def _failing_rank(rank, world, port, out):
    from lddmm_b200 import replicas

    _setenv(rank, world, port)
    env = replicas.rank_env()
    dist = replicas.init(env, "gloo", timeout_s=5)
    if rank == 1:
        os._exit(3)  # dies before the collective, as a crashed rank would
    t0 = time.time()
    try:
        replicas.max_over_ranks(dist, 1.0)
        out.put(("no error", time.time() - t0))
    except Exception as e:  # the short process-group timeout turns the wait into an error
        out.put((type(e).__name__, time.time() - t0))


def test_failed_rank_ends_the_other_with_an_error():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_failing_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    kind, waited = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
    assert kind != "no error"
    assert waited < 60


def test_single_rank_needs_no_process_group(monkeypatch):
    from lddmm_b200 import replicas

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    env = replicas.rank_env()
    assert (env.world, env.rank, env.local, env.reports) == (1, 0, 0, True)
    assert replicas.init(env, "gloo") is None
    assert replicas.max_over_ranks(None, 2.5) == 2.5
    assert replicas.job_rate(5, 1, 2.0) == 2.5
