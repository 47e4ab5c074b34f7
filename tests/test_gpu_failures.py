"""Failures stay local and are reported once.  Every failure here is made on
the host -- a NaN written into a replica's staged state before upload, a box
compressed far beyond liquid density, a histogram range no sample can fall
in -- and turned into a status by the engine's own checks: no kernel is made
to fault, trap or wait."""
import copy

import numpy as np
import pytest

from remd_b200 import engine as E
from remd_b200 import systems as S

pytestmark = pytest.mark.gpu


def _run_alone(e, nint, seed):
    srv = E.Server(budget_bytes=8 << 30)
    jid = srv.submit(e, nint, seed=seed)
    while srv.step():
        pass
    out = srv.result(jid, e.nreplica)
    srv.close()
    return out


def _with_nan_velocity(e, rep=1, mol=3):
    bad = copy.deepcopy(e)
    bad.states[rep].v[mol, 0] = np.nan
    return bad


def _dense(e, factor=0.6):
    """The same molecules in a box `factor` times as long (density / factor^3)."""
    d = copy.deepcopy(e)
    for st in d.states:
        st.L = st.L * factor
    return d


def test_nonfinite_replica_fails_its_job_alone():
    good = S.small_ensemble("tip4p", 1, nmol=90, ntemp=2, npress=2, seed=81, interval=10)
    other = S.small_ensemble("tip5p", 0, nmol=64, ntemp=2, npress=1, seed=82, interval=10)
    bad = _with_nan_velocity(other)
    srv = E.Server(budget_bytes=8 << 30)
    a = srv.submit(good, 4, seed=1)
    b = srv.submit(bad, 4, seed=2)
    while srv.step():
        pass
    ia, ib = srv.poll(a), srv.poll(b)
    assert ib.state == 3 and ib.status == 4          # failed, REMD_ERR_NONFINITE
    assert ia.state == 2 and ia.intervals_done == 4  # the batch mate finished
    avg, idx = srv.result(a, good.nreplica)
    avg1, idx1 = _run_alone(good, 4, 1)
    assert np.array_equal(avg, avg1) and np.array_equal(idx, idx1)
    assert srv.stats()["jobs_done"] == 1
    srv.close()


def test_nonfinite_replica_is_flagged_in_a_handle():
    e = _with_nan_velocity(S.small_ensemble("tip3p", 0, nmol=64, ntemp=2, npress=1, seed=83, interval=5))
    eng = E.REMDGPU([e], precision="fp32")
    with pytest.raises(E.RemdError) as err:
        eng.ExecuteSteps(e.T, e.P)
    assert err.value.status == 4
    assert eng.replica_status(1) == 4 and eng.replica_status(0) == 0
    eng.close()


def test_dense_input_overflows_the_neighbour_list():
    e = S.small_ensemble("tip3p", 0, nmol=1000, ntemp=1, npress=1, seed=84, interval=5)
    with pytest.raises(E.RemdError) as err:
        E.REMDGPU([_dense(e)], precision="fp32")
    assert err.value.status == 8                     # REMD_ERR_NEIGHBOR_OVERFLOW


def test_dense_job_fails_alone_in_the_server():
    good = S.small_ensemble("tip4p", 2, nmol=120, ntemp=2, npress=1, seed=85, interval=10)
    dense = _dense(S.small_ensemble("tip3p", 0, nmol=1000, ntemp=1, npress=1, seed=84, interval=10))
    srv = E.Server(budget_bytes=8 << 30)
    a = srv.submit(good, 3, seed=5)
    b = srv.submit(dense, 3, seed=6)
    while srv.step():
        pass
    assert srv.poll(b).state == 3 and srv.poll(b).status == 8
    assert srv.poll(a).state == 2
    avg, idx = srv.result(a, good.nreplica)
    avg1, idx1 = _run_alone(good, 3, 5)
    assert np.array_equal(avg, avg1) and np.array_equal(idx, idx1)
    srv.close()


def test_dense_job_arriving_mid_run_fails_alone():
    """The dense job joins a running batch: building the next batch handle fails
    in its initial force call, the previous handle stays usable, the dense job
    fails alone and the running job continues bit for bit."""
    good = S.small_ensemble("tip5p", 1, nmol=100, ntemp=2, npress=2, seed=86, interval=10)
    dense = _dense(S.small_ensemble("tip3p", 0, nmol=1000, ntemp=1, npress=1, seed=84, interval=10))
    srv = E.Server(budget_bytes=8 << 30)
    a = srv.submit(good, 4, seed=7)
    srv.step()
    srv.step()
    b = srv.submit(dense, 2, seed=8)
    while srv.step():
        pass
    assert srv.poll(b).state == 3 and srv.poll(b).status == 8
    assert srv.poll(a).state == 2 and srv.poll(a).intervals_done == 4
    avg, idx = srv.result(a, good.nreplica)
    avg1, idx1 = _run_alone(good, 4, 7)
    assert np.array_equal(avg, avg1) and np.array_equal(idx, idx1)
    srv.close()


def test_error_is_reported_once_then_cleared():
    """A histogram sample out of range is reported by the call that took it;
    the next interval, and an increment with a valid range, return REMD_OK."""
    e = S.small_ensemble("tip4p", 0, nmol=64, ntemp=2, npress=1, seed=74, interval=5)
    eng = E.REMDGPU([e], precision="fp32")
    eng.histogram_enable(0, 100.0, 200.0, 0.0, 1.0)   # no water sits there
    eng.ExecuteSteps(e.T, e.P)
    with pytest.raises(E.RemdError, match="RANGE"):
        eng.histogram_increment(np.arange(e.nreplica))
    eng.ExecuteSteps(e.T, e.P)                         # REMD_OK: the word was cleared
    a = eng.all_averages()
    pot = (a[:, 0] + a[:, 1] + a[:, 2]) / e.spec.nmol
    vol = a[:, 3] / e.spec.nmol
    eng.histogram_enable(0, pot.min() - 5, pot.max() + 5, vol.min() - 5, vol.max() + 5)
    eng.histogram_increment(np.arange(e.nreplica))
    b, hist, _ = eng.histogram(0, 0)
    assert b[4] == 1 and hist.sum() == 1
    eng.close()
