"""The N > 1 path of bench.py on the host: world-size-2 gloo ranks (replicas only, no data-path
collective; the only collectives are the barrier and the max over ranks of the timings)."""
import multiprocessing as mp
import socket

from helpers import replica_rank


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=replica_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert res[r]["env"] == (r, world, r)
        # every rank sees the slowest replica's time
        assert res[r]["max"] == 12.5
        assert res[r]["max_neg"] == -1.0
    # the reference arm runs on rank 0 alone: rank 1 returns 0 and prints nothing
    assert res[1]["ref_rc"] == 0
    assert res[1]["ref_out"] == ""


def test_rank_max_single_process():
    import bench
    assert bench.rank_max(3.25) == 3.25
