"""The multi-GPU plumbing of bench.py on CPU: two ranks over gloo (one
process each, spawned), as torchrun launches them on a node.  The path runs
independent replicas (no data-path collective); what the ranks share is the
barrier, the max-over-ranks reduction of the device time and the whole-job
value, and only rank 0 runs the reference arm."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks("gloo")
    r.barrier()
    ms = 10.0 + 3.0 * rank  # this rank's device time for 100 steps
    m = r.max(ms)
    q.put((rank, r.world, m, r.job_value(100, m)))
    r.close()


def test_two_ranks_max_and_job_value():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = 10.0 + 3.0 * (world - 1)
    for rank, w, m, v in got:
        assert w == world and m == slowest
        assert abs(v - world * 100 / (slowest / 1e3)) < 1e-9


def test_single_rank_has_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks("gloo")
    assert r.world == 1 and r.dist is None and r.max(4.5) == 4.5
    assert r.job_value(200, 200.0) == 1000.0
    r.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Ranks other than 0 leave the reference arm at once (no oracle work)."""
    monkeypatch.setenv("RANK", "1")
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup = 1, 0
    assert bench.run_reference(A()) == 0
