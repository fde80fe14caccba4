"""The replica path on CPU: two gloo ranks (spawned processes, rendezvous on 127.0.0.1) run the barrier, the
max-over-ranks of their timings and the whole-job rate exactly as bench.py does on GPUs over NCCL; a rank that never
joins ends the other's collective with an error within the group's timeout instead of hanging."""
import multiprocessing as mp
import os
import socket

import pytest

from opensol_b200.replicas import ReplicaGroup, replica_env


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR='127.0.0.1',
                      MASTER_PORT=str(port))
    group = ReplicaGroup('gloo', timeout_s=60)
    try:
        group.barrier()
        seconds = 1.0 + rank   # rank 1 is the slower replica
        slowest = group.reduce_max(seconds)
        rate = group.whole_job_rate(1000, slowest)
        group.barrier()
        out.put((rank, group.world, group.is_root, slowest, rate))
    finally:
        group.close()


def _lonely_rank(port, out):
    os.environ.update(RANK='0', WORLD_SIZE='2', LOCAL_RANK='0', MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    try:
        group = ReplicaGroup('gloo', timeout_s=3)
        group.barrier()
        out.put('no error')
    except Exception as exc:   # the store's wait for the missing rank, or the barrier, times out
        out.put(type(exc).__name__)


def test_single_process_needs_no_group(monkeypatch):
    for name in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK'):
        monkeypatch.delenv(name, raising=False)
    assert replica_env() == (0, 1, 0)
    group = ReplicaGroup('gloo')
    group.barrier()
    assert group.reduce_max(2.5) == 2.5
    assert group.whole_job_rate(10, 2.0) == 5.0
    group.close()


def test_two_gloo_ranks_take_the_max_and_count_every_rank():
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in results] == [0, 1]
    for rank, world, is_root, slowest, rate in results:
        assert world == 2 and is_root == (rank == 0)
        assert slowest == 2.0                 # the slower rank's time on every rank
        assert rate == 2 * 1000 / 2.0         # all ranks' units over the slowest rank's time


def test_missing_rank_ends_in_an_error_not_a_hang():
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    p = ctx.Process(target=_lonely_rank, args=(_free_port(), out))
    p.start()
    outcome = out.get(timeout=120)
    p.join(timeout=60)
    if p.is_alive():
        p.kill()
        pytest.fail('the lonely rank did not return')
    assert outcome != 'no error'
