"""The multi-GPU host path on the CPU: two ranks over gloo (127.0.0.1), each solving its shard
of the batch — the oracle standing in for a rank's GPU solve — and every rank getting the whole
batch's curves in the caller's order, equal to one process solving all of it; the slowest rank's
time by the max over ranks; a rank that fails raises on the host, never hangs its peer."""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from jaxdd_b200 import distributed  # noqa: E402

V = np.round(np.linspace(-0.2, 1.2, 5), 10)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_solve(batch, voltages, **kw):
    from oracle import dd
    return dd.solve_batch(dd.prepare(batch["devices"]), voltages, **kw)


def _failing_solve(batch, voltages, **kw):
    raise RuntimeError("this rank's solve failed")


def _rank(rank, world, port, out, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        from jaxdd_b200.workloads import drawn_devices
        devs = drawn_devices(5, NP=50)
        solve = _failing_solve if rank == fail_rank else _oracle_solve
        try:
            J, ok, its = distributed.solve_batch(devs, V, solve=solve)
        except Exception as e:  # noqa: BLE001 - reported to the test, which checks the kind
            out.put((rank, "error", type(e).__name__))
            return
        slowest = distributed.max_over_ranks(1.0 + rank)
        out.put((rank, J, ok, its, slowest))
    finally:
        dist.destroy_process_group()


def test_shards_cover_the_batch_in_order():
    for n, world in ((5, 2), (64, 3), (2, 4), (16384, 8)):
        parts = [distributed.shard(n, r, world) for r in range(world)]
        assert parts[0].start == 0 and parts[-1].stop == n
        assert all(a.stop == b.start for a, b in zip(parts, parts[1:]))
        sizes = [p.stop - p.start for p in parts]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        distributed.shard(5, 2, 2)


def test_two_ranks_give_the_single_process_curves():
    from oracle import dd
    from jaxdd_b200.workloads import drawn_devices
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out, -1)) for r in range(2)]
    for p in procs:
        p.start()
    got = [out.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    devs = drawn_devices(5, NP=50)
    J, ok, its = dd.solve_batch(dd.prepare(devs), V)
    for rank, Jr, okr, itsr, slowest in got:
        assert np.array_equal(Jr, J) and np.array_equal(okr, ok) and np.array_equal(itsr, its)
        assert slowest == 2.0


def test_a_failing_rank_ends_its_peer_with_an_error():
    """Rank 1's solve raises before the gather: it leaves the group, and rank 0's gather ends
    with an error from the process group (closed connection or its 20 s timeout) instead of
    waiting for good."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out, 1)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert got[0][:2] == (0, "error")
    assert got[1] == (1, "error", "RuntimeError")
