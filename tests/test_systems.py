"""The seeded synthetic workloads (remd_b200/systems.py)."""
import numpy as np
import pytest

from remd_b200 import systems as S
from remd_b200.inputs import UNIT_TEMP


def test_generator_is_deterministic():
    a = S.small_ensemble("tip4p", 1, nmol=40, seed=3)
    b = S.small_ensemble("tip4p", 1, nmol=40, seed=3)
    for sa, sb in zip(a.states, b.states):
        for k in ["r", "v", "q", "p"]:
            assert np.array_equal(getattr(sa, k), getattr(sb, k))


@pytest.mark.parametrize("model,confined", [("tip3p", 0), ("tip4p", 1), ("tip5p", 2)])
def test_start_state_is_valid(model, confined):
    e = S.small_ensemble(model, confined, nmol=50, ntemp=2, npress=2, seed=9)
    assert e.nreplica == 4 and len(e.states) == 4
    for st, T in zip(e.states, e.T):
        assert np.all((st.r >= 0) & (st.r < 1))
        assert np.allclose(np.linalg.norm(st.q, axis=1), 1.0, atol=1e-12)
        v = st.v / (st.L * st.s)
        tra = 0.5 * np.sum(st.m[:, None] * v * v)
        # the tube's angular-momentum removal after the scaling moves it slightly
        assert tra == pytest.approx(1.5 * st.nmol * T, rel=1e-10 if confined != 1 else 2e-2)
        mom = (st.v * st.m[:, None]).sum(0)
        free = {0: [0, 1, 2], 1: [2], 2: [0, 1]}[confined]
        assert np.allclose(mom[free], 0.0, atol=1e-9)
        # O-O spacing of the lattice start
        L = st.L
        x = st.r * L
        d = x[:, None] - x[None]
        d -= L * np.round(d / L)
        dd = np.sqrt((d ** 2).sum(-1)) + np.eye(st.nmol) * 1e9
        assert dd.min() >= 2.85


def test_condition_ladder_matches_reference_formula():
    T, P = S.conditions_geometrical(4, 4, 240, 360, 0.1e6, 200e6)
    assert T[0] * UNIT_TEMP == pytest.approx(240.0)
    assert T[3] * UNIT_TEMP == pytest.approx(360.0, rel=1e-6)
    assert np.all(np.diff(T[:4]) > 0) and np.all(P[4:8] > P[:4])


def test_config4_shape():
    ens = S.config4(seed=4)
    assert len(ens) == 8
    assert sum(e.nreplica for e in ens) == 256
    for e in ens:
        assert 64 <= e.spec.nmol <= 2048
        assert e.spec.moltype.nsite in (3, 4, 5)
        assert 8.5 <= e.spec.rcut <= 12.0
        assert e.spec.rcut - e.spec.rswitch in (1.0, 2.0)


def test_simg_tie_fixture_offsets():
    """The committed site-image tie configuration holds the ties it claims:
    |x| - L/2 for each listed site pair, recomputed in FP64."""
    import os
    from tests.common import GOLDEN
    z = np.load(os.path.join(GOLDEN, "simg_tie.npz"))
    b = S.load_model("tip3p").r
    r, q, L = z["r"], z["q"], z["L"]
    for (i, j, k, l, ax), off in zip(z["ties"], z["offsets"]):
        gr = (r[i] - r[j]) * L
        gr = np.where(gr >= 0.5 * L, gr - L, gr)
        gr = np.where(gr < -0.5 * L, gr + L, gr)
        rv = gr + S.body_to_space(q[i:i + 1], b)[0, k] - S.body_to_space(q[j:j + 1], b)[0, l]
        assert abs(rv[ax]) - 0.5 * L[ax] == pytest.approx(off, abs=1e-9)
        assert 1e-8 < abs(off) < 4e-6
