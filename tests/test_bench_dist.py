"""Multi-process (gloo, world_size 2) checks of the bench's replicas-only
aggregation: value = all ranks' mol-steps / slowest rank's device time, each
rank its own seeded workload, and the reference arm runs on rank 0 alone."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        local_ms = [120.0, 150.0][rank]
        local_units = [1.0e6, 3.0e6][rank]
        value, max_ms, total = bench.aggregate(local_ms, local_units, world)
        args = bench.parse_args(["--gpus", str(world), "--steps", "1", "--warmup", "0"])
        ens = bench.rank_workload(args, rank)
        sig = [(e.spec.nmol, e.spec.moltype.name, e.spec.confined, e.nreplica) for e in ens]
        buf = io.StringIO()
        if rank == 1:
            with redirect_stdout(buf):
                bench.reference_arm(args, rank, world)
        bench.barrier(world)
        q.put((rank, value, max_ms, total, sig, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_replicas_only_aggregation_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=240)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        _, value, max_ms, total, _, _ = out[r]
        assert max_ms == pytest.approx(150.0)
        assert total == pytest.approx(4.0e6)
        assert value == pytest.approx(4.0e6 / 0.150)
    # each rank its own seeded batch (same shape of grid, different draws)
    assert out[0][4] != out[1][4]
    # the reference arm prints only on rank 0
    assert out[1][5] == ""


def test_round_stats_split_and_normalisation():
    """Serving round statistics: raw p50/p99 milliseconds and milliseconds per
    million molecule-steps of the round's interval, per class of round."""
    import bench
    rounds = [(10.0, 2e6, False), (20.0, 2e6, False), (40.0, 1e6, True)]
    steady = bench.round_stats([r for r in rounds if not r[2]])
    changed = bench.round_stats([r for r in rounds if r[2]])
    assert steady["n"] == 2 and changed["n"] == 1
    assert steady["p50_ms"] == pytest.approx(15.0)
    assert steady["p50_ms_per_Mmolstep"] == pytest.approx(7.5)
    assert changed["p99_ms_per_Mmolstep"] == pytest.approx(40.0)
    assert bench.round_stats([]) == {"n": 0}


def test_cpu_model_names_the_host():
    import bench
    s = bench.cpu_model()
    assert s.endswith("logical CPUs") and str(os.cpu_count()) in s
