"""The N > 1 plumbing of the bench on CPU: two gloo ranks on 127.0.0.1, each a
replica with its own time; both must end with the slowest one, and a rank
that never arrives must end the other's barrier with an error, not a wait."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from felizjueves_b200 import replicas


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))


def _rank_max(rank, world, port, q):
    _env(rank, world, port)
    dist = replicas.init(world, "gloo", timeout_s=30)
    replicas.barrier(dist)
    ms = replicas.max_over_ranks(dist, 10.0 + 5.0 * rank)
    ms2 = replicas.max_over_ranks(dist, 3.0 if rank == 0 else 1.0)
    replicas.barrier(dist)
    replicas.finish(dist)
    q.put((rank, ms, ms2))


def _rank_absent(rank, world, port, q):
    _env(rank, world, port)
    dist = replicas.init(world, "gloo", timeout_s=5)
    if rank == 1:
        q.put((rank, "left"))  # leaves between steps: no collective in flight
        return
    try:
        replicas.barrier(dist)
        q.put((rank, "returned"))
    except Exception as e:  # the short process-group timeout ends the wait
        q.put((rank, type(e).__name__))


def _run(fn, world=2, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in ps:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_single_rank_is_identity():
    assert replicas.init(1) is None
    assert replicas.max_over_ranks(None, 2.5) == 2.5
    replicas.barrier(None)
    replicas.finish(None)


def test_two_ranks_max_over_ranks():
    out = _run(_rank_max)
    assert [o[0] for o in out] == [0, 1]
    for _, ms, ms2 in out:
        assert ms == 15.0  # the slower replica's time, on both ranks
        assert ms2 == 3.0


@pytest.mark.timeout(120)
def test_absent_rank_ends_barrier_with_error():
    out = dict(_run(_rank_absent))
    assert out[1] == "left"
    assert out[0] != "returned"


def test_reference_arm_other_ranks_do_no_work(capsys):
    """Under torchrun only rank 0 runs and prints the reference arm."""
    import sys

    import bench
    argv, sys.argv = sys.argv, ["bench.py", "--impl", "reference"]
    try:
        a = bench.parse()
    finally:
        sys.argv = argv
    assert bench.reference_arm(a, rank=1, world=2) is None
    assert capsys.readouterr().out == ""
