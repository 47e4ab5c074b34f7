"""Continuous batching (remd_server_*): jobs arriving while others run are
admitted as HBM frees up, share one batched launch per interval, and each
job's result is bit-identical to the same job run alone."""
import numpy as np
import pytest

from remd_b200 import engine as E
from remd_b200 import systems as S

pytestmark = pytest.mark.gpu


def _jobs():
    return [S.small_ensemble("tip4p", 1, nmol=90, ntemp=2, npress=2, seed=71, interval=10),
            S.small_ensemble("tip5p", 0, nmol=64, ntemp=4, npress=1, seed=72, interval=10),
            S.small_ensemble("tip3p", 2, nmol=150, ntemp=2, npress=1, seed=73, interval=10)]


def _alone(e, nint, seed):
    srv = E.Server(budget_bytes=8 << 30)
    jid = srv.submit(e, nint, seed=seed)
    while srv.step():
        pass
    out = srv.result(jid, e.nreplica)
    srv.close()
    return out


def test_mixed_arrivals_equal_alone_bitwise():
    ens = _jobs()
    nints = [5, 3, 4]
    srv = E.Server(budget_bytes=8 << 30)
    ids = [srv.submit(ens[0], nints[0], seed=1), srv.submit(ens[1], nints[1], seed=2)]
    srv.step()
    srv.step()
    ids.append(srv.submit(ens[2], nints[2], seed=3))   # arrives while the others run
    while srv.step():
        pass
    for e, jid, n, seed in zip(ens, ids, nints, [1, 2, 3]):
        info = srv.poll(jid)
        assert info.state == 2 and info.intervals_done == n
        avg, idx = srv.result(jid, e.nreplica)
        avg1, idx1 = _alone(e, n, seed)
        assert np.array_equal(avg, avg1)
        assert np.array_equal(idx, idx1)
        assert sorted(idx) == list(range(e.nreplica))
    st = srv.stats()
    assert st["jobs_done"] == 3 and st["p99_interval_ms"] >= st["p50_interval_ms"] > 0
    srv.close()


def test_budget_admission_and_cancel():
    ens = _jobs()
    ba, bb, bc = (E.Server.job_bytes(e) for e in ens)
    srv = E.Server(budget_bytes=max(ba, bb, bc) - 1)
    with pytest.raises(E.RemdError) as e:
        srv.submit(ens[int(np.argmax([ba, bb, bc]))], 2)   # larger than the whole budget
    assert e.value.status == 2
    srv.close()
    # a budget that holds a or b but not both: b waits for a
    srv = E.Server(budget_bytes=max(ba, bb) + min(ba, bb) // 2)
    a = srv.submit(ens[0], 2)
    b = srv.submit(ens[1], 2)
    srv.step()
    assert srv.poll(a).state == 1 and srv.poll(b).state == 0
    srv.step()     # a finishes at the end of this round
    assert srv.poll(a).state == 2
    c = srv.submit(ens[1], 50)
    srv.cancel(c)
    assert srv.poll(c).state == 4
    while srv.step():
        pass
    assert srv.poll(b).state == 2
    assert srv.poll(b).start_s >= srv.poll(a).end_s - 1e-9
    st = srv.stats()
    assert st["bytes_in_use"] == 0 and st["jobs_done"] == 2
    srv.close()


def test_jobs_of_different_interval_lengths_run_side_by_side():
    """Jobs whose MD interval lengths differ run as separate batches in the same
    rounds (their graphs side by side on their own streams); each result still
    equals the job run alone, bit for bit."""
    a = S.small_ensemble("tip4p", 0, nmol=80, ntemp=2, npress=1, seed=91, interval=10)
    b = S.small_ensemble("tip3p", 1, nmol=96, ntemp=2, npress=2, seed=92, interval=5)
    c = S.small_ensemble("tip5p", 2, nmol=90, ntemp=2, npress=1, seed=93, interval=10)
    srv = E.Server(budget_bytes=8 << 30)
    ids = [srv.submit(a, 3, seed=11), srv.submit(b, 4, seed=12)]
    srv.step()
    assert srv.poll(ids[0]).state == 1 and srv.poll(ids[1]).state == 1   # both running
    ids.append(srv.submit(c, 2, seed=13))
    while srv.step():
        pass
    for e, jid, n, seed in zip([a, b, c], ids, [3, 4, 2], [11, 12, 13]):
        assert srv.poll(jid).state == 2 and srv.poll(jid).intervals_done == n
        avg, idx = srv.result(jid, e.nreplica)
        avg1, idx1 = _alone(e, n, seed)
        assert np.array_equal(avg, avg1) and np.array_equal(idx, idx1)
    srv.close()
