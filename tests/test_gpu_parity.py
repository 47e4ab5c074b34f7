"""CUDA engine vs the FP64 oracle, through the C-ABI (libremd_b200.so).

Tolerances (relative L2 norms over all molecules unless stated):
  FP64 engine: forces/torques 1e-10, energies 1e-11 -- same arithmetic as the
               oracle, different summation order;
  FP32 engine: forces and torques 1e-5, potential energy 1e-6 (the engine's
               FP32 accuracy gate), virial 1e-5;
  20-step trajectories (chaotic, errors grow ~e^(t/tau)): FP64 1e-8, FP32 see
  the per-quantity bounds in test_twenty_steps.
"""
import copy
import os

import numpy as np
import pytest

from oracle import oracle as O
from remd_b200 import engine as E
from remd_b200 import systems as S
from remd_b200.inputs import read_chk
from tests.common import CASES, GOLDEN, NSTEPS, golden_conditions, golden_line, golden_spec, load_case, rel

pytestmark = pytest.mark.gpu

SLIT_CASES = {"tip4p_slit_npxy": ("tip4p", 3, 1, 96, 201), "tip3p_slit_nvt": ("tip3p", 0, 1, 80, 202),
              "tip5p_slit_npxy": ("tip5p", 3, 1, 72, 203)}


def slit_case(name, interval=NSTEPS):
    model, pcon, tcon, nmol, seed = SLIT_CASES[name]
    e = S.small_ensemble(model=model, confined=2, nmol=nmol, ntemp=1, npress=1, seed=seed,
                         pconstant=pcon, tconstant=tcon, interval=interval)
    return e.spec, e.states[0]


def any_case(name):
    if name in CASES:
        spec, st, _ = load_case(name)
        return spec, st
    return slit_case(name)


ALL = list(CASES) + list(SLIT_CASES)


def single(spec, st):
    return S.Ensemble("t", spec, 1, 1, np.array([st.T]), np.array([st.P]), [st])


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("name", ALL)
def test_force_snapshot(name, prec):
    spec, st = any_case(name)
    eng = E.REMDGPU([single(spec, st)], precision=prec)
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(spec, st)
    orc.initialize_property()
    po = orc.prop()
    # The bulk fixtures are dilute (64 molecules in a 19 A box: gas density),
    # where the molecular forces are ~100x smaller than the site-site Coulomb
    # terms they cancel from; the FP32 representation of the site vectors alone
    # then gives ~1.5e-5.  The 1e-5 / 1e-6 gates are enforced on liquid-density
    # systems in test_fp32_accuracy_liquid.
    dilute = spec.confined == 0
    tf = (3e-5 if dilute else 1e-5) if prec == "fp32" else 1e-10
    te = (3e-6 if dilute else 1e-6) if prec == "fp32" else 1e-11
    assert rel(g["f"], orc.f) < tf
    assert rel(g["n"], orc.n) < tf
    assert g["pot"] == pytest.approx(po["pot"], rel=te)
    # components cancel against each other: bound them on the scale of their magnitudes
    scale = abs(po["lj"]) + abs(po["clmb"]) + abs(po["wall"])
    assert g["lj"] == pytest.approx(po["lj"], abs=te * scale)
    assert g["clmb"] == pytest.approx(po["clmb"], abs=te * scale)
    assert g["wall"] == pytest.approx(po["wall"], abs=te * scale)
    assert rel(g["vir"], po["vir"]) < tf
    assert g["H0"] == pytest.approx(po["H0"], rel=te * 10, abs=te * 10 * abs(po["pot"]))
    if prec == "fp64":
        assert eng.pair_count() == po["npairs"]
    else:
        assert abs(eng.pair_count() - po["npairs"]) <= 1
    eng.close()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("name", ALL)
def test_twenty_steps(name, prec):
    spec, st = any_case(name)
    eng = E.REMDGPU([single(spec, st)], precision=prec, interval=NSTEPS)
    eng.ExecuteSteps(np.array([st.T]), np.array([st.P]))
    a = eng.GetAverages(0)
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(spec, st)
    orc.initialize_property()
    orc.steps(NSTEPS)
    b = orc.average()
    if prec == "fp64":
        tr, tv, te = 1e-9, 1e-7, 1e-8
    else:
        tr, tv, te = 2e-5, 2e-3, 2e-4
    assert rel(g["r"], orc.r) < tr
    assert rel(g["q"], orc.q) < tr * 10
    assert rel(g["v"], orc.v) < tv
    assert rel(g["p"], orc.p) < tv
    pot_a, pot_b = a[0] + a[1] + a[2], b[0] + b[1] + b[2]
    assert pot_a == pytest.approx(pot_b, rel=te)
    for k in [3, 4, 5, 6, 13]:   # VOL TRA ROT T TSTs
        assert a[k] == pytest.approx(b[k], rel=te * 10), E.AVG_NAMES[k]
    # DRF: the Hamiltonian drift, compared in absolute terms against |H0|
    assert abs(a[12] - b[12]) < te * 10 * abs(orc.prop()["H0"]) + 1e-6
    assert eng.replica_status(0) == 0


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_engine_matches_reference_fixtures(name):
    """The FP64 engine against the reference's own outputs (tests/golden/ref_*.npz,
    compiled reference CPU code; slit systems from the build whose CPU slit wall is
    the reference GPU kernel's lookup): the force snapshot at the oracle's bounds and
    20 MD steps at the trajectory bounds."""
    spec, st, z = load_case(name)
    eng = E.REMDGPU([single(spec, st)], precision="fp64", interval=NSTEPS)
    g = eng.ConvertVariablesToHost(0)
    assert rel(g["f"], z["snap_f"]) < 1e-10
    assert rel(g["n"], z["snap_n"]) < 1e-10
    e = z["snap_ener"]
    scale = abs(e[0]) + abs(e[1]) + abs(e[2])
    assert g["lj"] == pytest.approx(e[0], abs=1e-11 * scale)
    assert g["clmb"] == pytest.approx(e[1], abs=1e-11 * scale)
    assert g["wall"] == pytest.approx(e[2], abs=1e-11 * scale)
    assert rel(g["vir"], e[3:6]) < 1e-10
    eng.ExecuteSteps(np.array([st.T]), np.array([st.P]))
    g = eng.ConvertVariablesToHost(0)
    assert rel(g["r"], z["after_r"]) < 1e-9
    assert rel(g["q"], z["after_q"]) < 1e-8
    assert rel(g["v"], z["after_v"]) < 1e-7
    assert rel(g["p"], z["after_p"]) < 1e-7
    sc = z["after_scal"]
    assert g["s"] == pytest.approx(sc[0], rel=1e-9)
    assert np.allclose(g["L"], sc[5:8], rtol=1e-12)
    eng.close()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_condition_change_applies_exchange_tail(prec):
    """ExecuteSteps with a new (T,P) runs ChangeTemperature, KillMomentum,
    SetPressure, CalcProperties, UpdateHamiltonian first (src/remd.cxx:526-536)."""
    for name in ["tip4p_tube_npz", "tip3p_bulk_npt", "tip5p_slit_npxy"]:
        spec, st = any_case(name)
        eng = E.REMDGPU([single(spec, st)], precision=prec, interval=5)
        T1, P1 = st.T * 1.07, st.P * 0.5 + 1e-4
        eng.ExecuteSteps(np.array([T1]), np.array([P1]))
        a = eng.GetAverages(0)
        orc = O.Oracle(spec, st)
        orc.initialize_property()
        orc.apply_condition(T1, P1)
        orc.steps(5)
        b = orc.average()
        tol = 1e-8 if prec == "fp64" else 1e-4
        for k in [4, 5, 6, 11, 13, 14]:
            assert a[k] == pytest.approx(b[k], rel=tol, abs=tol), (name, E.AVG_NAMES[k])
        g = eng.ConvertVariablesToHost(0)
        assert g["T"] == T1 and g["P"] == P1


def test_batch_equals_alone_bitwise():
    """Mixed ensembles in one launch: each replica's trajectory is bit-identical
    to the same replica run alone (deterministic fixed-order reductions)."""
    ens = [S.small_ensemble("tip3p", 0, nmol=70, ntemp=2, npress=1, seed=31, interval=10),
           S.small_ensemble("tip4p", 1, nmol=130, ntemp=1, npress=2, seed=32, interval=10),
           S.small_ensemble("tip5p", 2, nmol=200, ntemp=2, npress=1, seed=33, interval=10)]
    big = E.REMDGPU(ens, precision="fp32")
    T = np.concatenate([e.T for e in ens])
    P = np.concatenate([e.P for e in ens])
    big.ExecuteSteps(T, P)
    avg = big.all_averages()
    k = 0
    for e in ens:
        for j, st in enumerate(e.states):
            one = E.REMDGPU([S.Ensemble("a", e.spec, 1, 1, e.T[j:j + 1], e.P[j:j + 1], [st])],
                            precision="fp32")
            one.ExecuteSteps(e.T[j:j + 1], e.P[j:j + 1])
            assert np.array_equal(one.GetAverages(0), avg[k])
            assert np.array_equal(one.ConvertVariablesToHost(0)["r"], big.ConvertVariablesToHost(k)["r"])
            one.close()
            k += 1


def test_dependent_launch_and_plain_launch_agree_bitwise():
    """A step whose tile grid is no larger than the SM count is launched with
    programmatic stream serialisation, a larger one plainly.  A small ensemble
    alone (dependent launches) and the same ensemble inside a batch of more than
    148 tiles per interval-graph chain (plain launches) give the same bits."""
    small = S.small_ensemble("tip4p", 0, nmol=70, ntemp=2, npress=1, seed=34, interval=10)
    filler = S.make_ensemble("filler", "tip3p", 0, 512, 0.0, 9.0, 8.0, 16, 4, 250, 350, 0.1e6, 0.1e6, 35,
                             interval=10)
    alone = E.REMDGPU([small], precision="fp32")
    alone.set_tuning(32, 1.0)
    alone.ExecuteSteps(small.T, small.P)
    both = E.REMDGPU([small, filler], precision="fp32")
    both.set_tuning(32, 1.0)
    assert filler.nreplica * 16 // 4 > 148   # 512 molecules = 16 tiles of 32, over four chains
    both.ExecuteSteps(np.concatenate([small.T, filler.T]), np.concatenate([small.P, filler.P]))
    for r in range(small.nreplica):
        assert np.array_equal(alone.GetAverages(r), both.GetAverages(r))
        a, b = alone.ConvertVariablesToHost(r), both.ConvertVariablesToHost(r)
        assert np.array_equal(a["r"], b["r"]) and np.array_equal(a["p"], b["p"])
    alone.close()
    both.close()


def test_velocity_scaling_in_a_mixed_batch():
    """tconstant 2: Molecules::ExecuteSteps rescales the velocities before every
    step (src/integrator.cxx:713-723).  In a batch with Nose-Poincare replicas the
    scaled replicas follow the oracle, and the others stay bit-identical to a
    batch without them (their steps are split into closing kick, rescale
    launch and opening, with the same arithmetic as the fused step)."""
    vs = S.small_ensemble("tip3p", 1, nmol=72, ntemp=2, npress=1, seed=51, interval=NSTEPS,
                          pconstant=2, tconstant=2)
    npt = S.small_ensemble("tip4p", 0, nmol=70, ntemp=2, npress=1, seed=52, interval=NSTEPS)
    for prec in ["fp32", "fp64"]:
        mixed = E.REMDGPU([npt, vs], precision=prec)
        plain = E.REMDGPU([npt], precision=prec)
        # per step: integrate, replica head, force (two launches in FP32), and for
        # velocity scaling the rescale plus, after the first step, the closing kick;
        # then start + end
        per = 4 if prec == "fp32" else 3
        assert mixed.launches_per_interval() == (per + 1) * NSTEPS + NSTEPS - 1 + 2
        T = np.concatenate([npt.T, vs.T])
        P = np.concatenate([npt.P, vs.P])
        mixed.ExecuteSteps(T, P)
        plain.ExecuteSteps(npt.T, npt.P)
        for j in range(2):
            assert np.array_equal(mixed.GetAverages(j), plain.GetAverages(j))
            assert np.array_equal(mixed.ConvertVariablesToHost(j)["v"], plain.ConvertVariablesToHost(j)["v"])
        for j, st in enumerate(vs.states):
            orc = O.Oracle(vs.spec, st)
            orc.initialize_property()
            orc.steps(NSTEPS)
            a, b = mixed.GetAverages(2 + j), orc.average()
            g = mixed.ConvertVariablesToHost(2 + j)
            tr, te = (1e-9, 1e-8) if prec == "fp64" else (2e-5, 2e-4)
            assert rel(g["r"], orc.r) < tr
            assert a[0] + a[1] + a[2] == pytest.approx(b[0] + b[1] + b[2], rel=te)
            for k in [3, 4, 5, 6]:   # VOL TRA ROT T
                assert a[k] == pytest.approx(b[k], rel=te * 10), E.AVG_NAMES[k]
            # s and Ps are reset before every step and not integrated; Pv_z restarts from 0
            assert a[13] == 1.0 and a[14] == 0.0
            assert a[17] == pytest.approx(b[17], rel=te * 10, abs=1e-12)
        mixed.close()
        plain.close()


def test_velocity_scaling_modes_the_reference_does_not_integrate_are_rejected():
    """Slit and bulk-barostat *TSCALE* modes fall through the switch of
    Molecules::ExecuteSteps (src/integrator.cxx:730-787), which then integrates
    nothing; the engine refuses them."""
    for confined, pcon in [(2, 0), (2, 3), (0, 1)]:
        e = S.small_ensemble("tip4p", confined, nmol=64, ntemp=1, npress=1, seed=53, interval=5,
                             pconstant=pcon, tconstant=2)
        with pytest.raises(RuntimeError, match="tconstant 2"):
            E.REMDGPU([e], precision="fp32")


def test_wall_tables_are_shared_cached_and_bounded():
    """Ensembles with equal wall parameters share one table, a second handle
    takes its table from the engine's cache (a tube table of 65536 entries is
    about a second of host time), and neither changes a result; an nfwall
    beyond the engine's bound is refused before any table is computed."""
    a = S.small_ensemble("tip4p", 1, nmol=64, ntemp=1, npress=2, seed=57, interval=5, nfwall=65536)
    b = S.small_ensemble("tip3p", 1, nmol=64, ntemp=1, npress=2, seed=58, interval=5, nfwall=65536)
    alone = E.REMDGPU([a], precision="fp32")
    alone.ExecuteSteps(a.T, a.P)
    ref = [alone.ConvertVariablesToHost(r) for r in range(a.nreplica)]
    alone.close()
    both = E.REMDGPU([a, b], precision="fp32")
    both.ExecuteSteps(np.concatenate([a.T, b.T]), np.concatenate([a.P, b.P]))
    for r in range(a.nreplica):
        g = both.ConvertVariablesToHost(r)
        assert np.array_equal(g["r"], ref[r]["r"]) and np.array_equal(g["p"], ref[r]["p"])
    both.close()
    big = copy.deepcopy(a)
    big.spec.nfwall = (1 << 24) + 1
    with pytest.raises(RuntimeError, match="nfwall"):
        E.REMDGPU([big], precision="fp32")


def test_device_exchange_equals_host_exchange():
    ens = [S.small_ensemble("tip4p", 0, nmol=64, ntemp=4, npress=2, seed=41, interval=5),
           S.small_ensemble("tip3p", 1, nmol=80, ntemp=2, npress=3, seed=42, interval=5)]
    eng = E.REMDGPU(ens, precision="fp32")
    T = np.concatenate([e.T for e in ens])
    P = np.concatenate([e.P for e in ens])
    grids = [(e.ntemp, e.npress) for e in ens]
    eng.ExecuteSteps(T, P)
    rng = np.random.default_rng(7)
    idx_h = [np.arange(e.nreplica, dtype=np.int32) for e in ens]
    T_h = [e.T.copy() for e in ens]
    P_h = [e.P.copy() for e in ens]
    for step in range(8):
        avg = eng.all_averages()
        us, off = [], 0
        for i, e in enumerate(ens):
            pot = avg[off:off + e.nreplica, 0] + avg[off:off + e.nreplica, 1] + avg[off:off + e.nreplica, 2]
            vol = avg[off:off + e.nreplica, 3]
            u = rng.random(max(e.nreplica // 2, 1))
            n = E.exchange_host(e.ntemp, e.npress, e.spec.pconstant, step, idx_h[i], T_h[i], P_h[i],
                                pot, vol, u)
            us.append(u[:len(n)])
            off += e.nreplica
        eng.exchange_device(grids, step, u=np.concatenate(us))
        idx_d, T_d, P_d = eng.conditions()
        assert np.array_equal(idx_d, np.concatenate(idx_h))
        assert np.array_equal(T_d, np.concatenate(T_h)) and np.array_equal(P_d, np.concatenate(P_h))
        eng.execute_device()


def test_write_chk_on_the_reference_input(tmp_path):
    """remd_write_chk on the reference's test input (test/input/gpu0000.chk):
    every line but the last is the reference file's bytes; the last, the
    Property line, holds the engine's own numbers for that state, checked
    against the FP64 oracle."""
    from remd_b200.inputs import UNIT_PRESS, UNIT_TEMP
    spec = golden_spec()
    st = read_chk(f"{GOLDEN}/gpu0000.chk")
    st.T, st.P = golden_conditions()
    eng = E.REMDGPU([single(spec, st)], precision="fp64")
    eng.write_chk(0, str(tmp_path / "e.chk"))
    mine = open(tmp_path / "e.chk").read().splitlines()
    ref = open(f"{GOLDEN}/gpu0000.chk").read().splitlines()
    assert len(mine) == len(ref) and mine[:-1] == ref[:-1]
    prop = np.array([float(x) for x in mine[-1].split()])
    assert len(prop) == 26
    orc = O.Oracle(spec, st)
    orc.initialize_property()
    po, avg = orc.prop(), orc.average()
    assert prop[0] == 0.0                                       # time: no MD step yet
    for k, key in [(1, "pot"), (2, "tra"), (3, "rot"), (4, "kin"), (9, "tot")]:
        assert prop[k] == pytest.approx(po[key], rel=1e-6), key
    assert abs(prop[10]) <= 1e-6 * abs(po["tot"])               # ham = tot - H0 = 0
    assert prop[14] == pytest.approx(po["kin"] / (3 * spec.nmol) * UNIT_TEMP, rel=1e-6)
    prs = np.array([avg[8], avg[9], avg[10], avg[7]]) * UNIT_PRESS
    assert np.allclose(prop[15:19], prs, rtol=1e-5) and np.allclose(prop[22:26], prs, rtol=1e-5)
    assert np.allclose(prop[19:22], po["vir"], rtol=1e-6)
    tmo = (st.v * st.m[:, None] / (st.L * st.s)).sum(axis=0)  # Molecules::Momentum
    assert np.allclose(prop[11:14], tmo, rtol=1e-5, atol=1e-9 * np.abs(st.v * st.m[:, None] / st.L).sum())
    eng.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_reference_regression_input(prec):
    """test/input/gpu0000.chk through the engine: interval 0 against the
    reference's golden line (loose band) and the oracle (tight)."""
    spec = golden_spec()
    st = read_chk(f"{GOLDEN}/gpu0000.chk")
    st.T, st.P = golden_conditions()
    orc = O.Oracle(spec, st)
    orc.velocity_scaling()
    orc.ang_velocity_scaling()
    orc.set_tstat_mass(0.5)
    st0 = orc.state()
    orc.initialize_property()
    orc.steps(100)
    b = orc.average()
    eng = E.REMDGPU([single(spec, st0)], precision=prec)
    eng.ExecuteSteps(np.array([st0.T]), np.array([st0.P]))
    a = eng.GetAverages(0)
    g = dict(zip(golden_line()["columns"], golden_line()["values"]))
    assert a[0] + a[1] + a[2] == pytest.approx(g["pot"], rel=2e-4)
    assert a[3] == pytest.approx(g["vol"], rel=2e-4)
    tol = 1e-8 if prec == "fp64" else 1e-4
    assert a[0] + a[1] + a[2] == pytest.approx(b[0] + b[1] + b[2], rel=tol)
    assert a[3] == pytest.approx(b[3], rel=tol)


def test_rescale_matches_reference_init_scaling():
    spec, st, _ = load_case("tip4p_tube_npz")
    st = st.copy()
    st.T *= 1.3     # rescale to a different temperature than the start
    eng = E.REMDGPU([single(spec, st)], precision="fp64", interval=5)
    eng.rescale_velocities()
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(spec, st)
    orc.velocity_scaling()
    orc.ang_velocity_scaling()
    orc.initialize_property()
    assert rel(g["v"], orc.v) < 1e-12 and rel(g["p"], orc.p) < 1e-12
    assert (g["s"], g["Ps"]) == (1.0, 0.0)
    assert g["H0"] == pytest.approx(orc.prop()["H0"], rel=1e-11)


def test_rescale_after_thermostat_drift_restores_temperature():
    """With s != 1 the stored v, p are brought to s = 1 first, so the physical
    kinetic energy after the rescale is exactly 1.5 N T (translational and
    rotational each)."""
    spec, st, _ = load_case("tip4p_tube_npz")
    eng = E.REMDGPU([single(spec, st)], precision="fp64", interval=20)
    eng.ExecuteSteps(np.array([st.T]), np.array([st.P]))
    assert eng.ConvertVariablesToHost(0)["s"] != 1.0
    eng.rescale_velocities()
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(spec, st)
    orc.change_temperature(st.T)      # v, p -> s = 1 scale (coef = 1)
    # same state as the engine before its rescale is not available here; check
    # the invariant instead: translational energy 1.5 N T at s = 1
    v = g["v"] / g["L"]
    tra = 0.5 * np.sum(st.m[:, None] * v * v)
    assert g["s"] == 1.0
    assert tra == pytest.approx(1.5 * spec.nmol * st.T, rel=2e-2)


@pytest.mark.parametrize("idx", [0, 2, 6])
def test_long_fp64_trajectory_config4_ensembles(idx):
    """100 steps of a strongly relaxing config-4 lattice start: FP64 engine vs oracle."""
    e = S.config4(seed=4)[idx]
    st = e.states[0]
    eng = E.REMDGPU([single(e.spec, st)], precision="fp64", interval=50)
    orc = O.Oracle(e.spec, st)
    orc.initialize_property()
    for k in range(2):
        eng.ExecuteSteps(np.array([st.T]), np.array([st.P]))
        orc.steps(50)
        a, b = eng.GetAverages(0), orc.average()
        assert np.all(np.isfinite(a))
        assert a[0] + a[1] + a[2] == pytest.approx(b[0] + b[1] + b[2], rel=1e-6 * (10 ** k))


@pytest.mark.parametrize("idx", range(8))
def test_fp32_accuracy_liquid(idx):
    """The FP32 accuracy gate on the benchmark's own (liquid-density)
    ensembles: force and torque RMS error <= 1e-5 relative, potential energy
    within 1e-6 relative of the FP64 oracle, one replica per ensemble."""
    e = S.config4(seed=4)[idx]
    st = e.states[0]
    eng = E.REMDGPU([single(e.spec, st)], precision="fp32")
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(e.spec, st)
    orc.initialize_property()
    assert rel(g["f"], orc.f) < 1e-5
    assert rel(g["n"], orc.n) < 1e-5
    assert g["pot"] == pytest.approx(orc.prop()["pot"], rel=1e-6)
    assert rel(g["vir"], orc.prop()["vir"]) < 1e-5


def test_fp32_accuracy_tip5p_bulk_1728():
    """The precision-study system (TIP5P, N=1728, 12^3 simple cubic, rc 12 / rs 10)."""
    e = S.make_ensemble("c3", "tip5p", 0, 1728, 0.0, 12.0, 10.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 3)
    st = e.states[0]
    eng = E.REMDGPU([single(e.spec, st)], precision="fp32")
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(e.spec, st)
    orc.initialize_property()
    assert rel(g["f"], orc.f) < 1e-5
    assert rel(g["n"], orc.n) < 1e-5
    assert g["pot"] == pytest.approx(orc.prop()["pot"], rel=1e-6)


@pytest.mark.parametrize("model,confined,wall,rc", [("tip5p", 0, 0.0, 12.0), ("tip4p", 1, 7.0, 10.0),
                                                   ("tip3p", 2, 12.0, 11.0)])
def test_fp32_accuracy_large_systems(model, confined, wall, rc):
    """The largest systems of the serving stream (N = 4096: a 50 A bulk box, a
    1.4 um nanotube, a 115 A slit): FP32 forces, torques and energy against the
    FP64 oracle at the same gates as the liquid-density batch."""
    e = S.make_ensemble("big", model, confined, 4096, wall, rc, rc - 1.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 41)
    st = e.states[0]
    eng = E.REMDGPU([single(e.spec, st)], precision="fp32")
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(e.spec, st)
    orc.initialize_property()
    assert rel(g["f"], orc.f) < 1e-5
    assert rel(g["n"], orc.n) < 1e-5
    assert g["pot"] == pytest.approx(orc.prop()["pot"], rel=1e-6)
    assert abs(eng.pair_count() - orc.prop()["npairs"]) <= 2
    eng.close()


@pytest.mark.parametrize("wall", [4.5, 5.0])
def test_fp32_accuracy_narrow_tube(wall):
    """Single-file water in the narrowest tubes of the batch's radius range
    (4.5 and 5 A, 256 TIP4P molecules on a 768 A axis): the FP32 gates hold where
    the wall term is as large as the pair terms."""
    e = S.make_ensemble("nt", "tip4p", 1, 256, wall, 8.5, 7.5, 1, 1, 300, 300, 0.1e6, 0.1e6, 45)
    st = e.states[0]
    eng = E.REMDGPU([single(e.spec, st)], precision="fp32")
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(e.spec, st)
    orc.initialize_property()
    assert rel(g["f"], orc.f) < 1e-5
    assert rel(g["n"], orc.n) < 1e-5
    assert g["pot"] == pytest.approx(orc.prop()["pot"], rel=1e-6)
    assert g["wall"] == pytest.approx(orc.prop()["wall"], rel=1e-6)
    assert eng.pair_count() == orc.prop()["npairs"]
    eng.close()


def _simg_tie_case():
    z = np.load(os.path.join(GOLDEN, "simg_tie.npz"))
    e = S.make_ensemble("tie", "tip3p", 0, len(z["r"]), 0.0, float(z["rcut"]), float(z["rswitch"]),
                        1, 1, 300, 300, 0.1e6, 0.1e6, 4)
    st = e.states[0]
    st.r, st.q, st.L = z["r"].copy(), z["q"].copy(), z["L"].copy()
    st.v[:] = 0.0
    st.p[:] = 0.0
    return e.spec, st, z["ties"]


def test_fp32_site_image_ties_follow_oracle():
    """Site pairs with a component within 1e-7..3e-6 A of L/2 under the per-site
    minimum image (src/force_calculator.cxx:737-741): the FP32 form takes the
    oracle's image for each, so no site force flips direction."""
    spec, st, ties = _simg_tie_case()
    eng = E.REMDGPU([single(spec, st)], precision="fp32")
    g = eng.ConvertVariablesToHost(0)
    orc = O.Oracle(spec, st)
    orc.initialize_property()
    assert rel(g["f"], orc.f) < 1e-5
    assert rel(g["n"], orc.n) < 1e-5
    scale = np.median(np.linalg.norm(orc.f, axis=1))
    for i, j, _, _, _ in ties:
        for m in (i, j):
            assert np.linalg.norm(g["f"][m] - orc.f[m]) < 1e-5 * scale * 10


def _tuning_batch():
    return [S.small_ensemble("tip4p", 1, nmol=150, ntemp=2, npress=1, seed=81, interval=10),
            S.small_ensemble("tip5p", 0, nmol=100, ntemp=1, npress=2, seed=82, interval=10)]


def _run_intervals(eng, n):
    T = np.concatenate([e.T for e in eng.ensembles])
    P = np.concatenate([e.P for e in eng.ensembles])
    out = []
    for _ in range(n):
        eng.ExecuteSteps(T, P)
        out.append(eng.all_averages())
    return np.array(out)


def test_tile_and_skin_do_not_change_the_trajectory():
    """Forces are a function of the positions only and every partial sum is per
    32 molecules, so the same batch under different (tile, skin) choices gives
    bit-identical averages."""
    ens = _tuning_batch()
    runs = []
    for tuning in [None, (32, 0.6), (32, 1.4)]:
        eng = E.REMDGPU(ens, precision="fp32")
        if tuning:
            eng.set_tuning(*tuning)
        runs.append(_run_intervals(eng, 4))
        eng.close()
    assert np.array_equal(runs[0], runs[1])
    assert np.array_equal(runs[0], runs[2])


def test_autotune_keeps_the_trajectory():
    """remd_autotune times its candidates on the live batch and restores the
    state after each, so the run continues exactly as without it."""
    ens = _tuning_batch()
    a = E.REMDGPU(ens, precision="fp32")
    b = E.REMDGPU(ens, precision="fp32")
    ra, rb = [_run_intervals(a, 1)], [_run_intervals(b, 1)]
    tile, skin, ms = a.autotune(nsteps=5)
    assert tile in (32, 64, 96, 128) and skin in (0.2, 0.4, 0.6, 0.8, 1.0, 1.4) and ms > 0
    ra.append(_run_intervals(a, 3))
    rb.append(_run_intervals(b, 3))
    assert np.array_equal(np.concatenate(ra), np.concatenate(rb))
    a.close()
    b.close()


def test_graph_exchange_equals_explicit_exchange():
    """The exchange appended to the interval graph (device step counter, Philox
    uniforms) makes the same decisions as explicit per-interval calls."""
    ens = [S.small_ensemble("tip4p", 0, nmol=64, ntemp=4, npress=2, seed=51, interval=5),
           S.small_ensemble("tip5p", 1, nmol=72, ntemp=2, npress=2, seed=52, interval=5)]
    grids = [(e.ntemp, e.npress) for e in ens]
    a = E.REMDGPU(ens, precision="fp32")
    b = E.REMDGPU(ens, precision="fp32")
    a.enable_device_exchange(grids, seed=99)
    for step in range(8):
        a.execute_device()
        b.execute_device()
        b.exchange_device(grids, step, u=None, seed=99)
    ia, Ta, Pa = a.conditions()
    ib, Tb, Pb = b.conditions()
    assert np.array_equal(ia, ib) and np.array_equal(Ta, Tb) and np.array_equal(Pa, Pb)
    assert np.array_equal(a.all_averages(), b.all_averages())
    off = 0
    for e in ens:      # conditions stay a permutation within each ensemble
        assert sorted(ia[off:off + e.nreplica]) == list(range(e.nreplica))
        assert np.array_equal(np.sort(Ta[off:off + e.nreplica]), np.sort(e.T))
        off += e.nreplica


def test_write_gro_matches_reference_writer(tmp_path):
    """remd_write_gro of an advanced replica gives the bytes the reference's
    IOManager::UpdateOutputs path writes for the same state (restated
    ConvertMoleculesToAtoms, the reference's own write_gro_file when built)."""
    e = S.small_ensemble("tip4p", 2, nmol=90, ntemp=1, npress=1, seed=23, interval=10)
    eng = E.REMDGPU([e], precision="fp32")
    eng.ExecuteSteps(e.T, e.P)
    path = str(tmp_path / "engine.gro")
    mt = e.spec.moltype
    eng.write_gro(0, path, mt)
    g = eng.ConvertVariablesToHost(0)
    atoms = O.gro_atoms(mt.name, mt.names, g["r"], g["q"], g["L"], mt.r)
    text = O.gro_text(*atoms, L=g["L"] * 0.1)
    assert open(path).read() == text
    if O.reference_available():
        ref = str(tmp_path / "ref.gro")
        O.reference_write_gro(ref, *atoms, L=g["L"] * 0.1)
        assert open(ref).read() == text
    eng.close()


def test_output_cdv_matches_restatement(tmp_path):
    """remd_output_cdv (REMDGPU::OutputCDV, src/remdgpu.cu:700-804) over a batch of
    bulk, tube and slit replicas after an interval: one file per replica slot,
    byte-identical to the restatement on the engine's own state."""
    ens = [S.small_ensemble("tip3p", 0, nmol=70, ntemp=2, npress=1, seed=61, interval=10),
           S.small_ensemble("tip4p", 1, nmol=96, ntemp=1, npress=2, seed=62, interval=10),
           S.small_ensemble("tip5p", 2, nmol=80, ntemp=1, npress=1, seed=63, interval=10)]
    eng = E.REMDGPU(ens, precision="fp32")
    eng.ExecuteSteps(np.concatenate([e.T for e in ens]), np.concatenate([e.P for e in ens]))
    prefix = str(tmp_path / "snap")
    eng.OutputCDV(prefix, 12)
    k = 0
    for e in ens:
        for _ in e.states:
            g = eng.ConvertVariablesToHost(k)
            want = O.cdv_text(g["r"], g["q"], g["L"], e.spec.moltype.r, g["T"], g["P"],
                              e.spec.confined, e.spec.wall_length)
            got = open(f"{prefix}R{k:04d}s0000012.cdv").read()
            assert got == want, k
            assert len(got.splitlines()) == 1 + e.spec.nmol * e.spec.moltype.nsite
            k += 1
    assert not os.path.exists(f"{prefix}R{k:04d}s0000012.cdv")
    eng.close()


def _hist_ranges(avg, nmol):
    """energy / volume ranges per molecule that hold every sample of a short run."""
    pot = (avg[:, 0] + avg[:, 1] + avg[:, 2]) / nmol
    vol = avg[:, 3] / nmol
    return (float(np.floor(pot.min()) - 40.0), float(np.ceil(pot.max()) + 40.0), 0.0,
            float(np.ceil(vol.max()) * 1.5))


def test_histograms_host_index_match_oracle_and_reference(tmp_path):
    """remd_histogram_increment after each interval, with the conditions moved by
    the host exchange: counts, bounds and per-bin sums equal the restatement
    bit for bit, and remd_histogram_write gives the bytes the reference's
    REMDInfo::OutputHistogram writes for the same samples."""
    ens = [S.small_ensemble("tip4p", 1, nmol=96, ntemp=2, npress=2, seed=71, interval=10),
           S.small_ensemble("tip3p", 0, nmol=64, ntemp=3, npress=1, seed=72, interval=10)]
    eng = E.REMDGPU(ens, precision="fp32")
    offs = np.cumsum([0] + [e.nreplica for e in ens])
    a0 = eng.all_averages()
    ranges = [_hist_ranges(a0[offs[i]:offs[i + 1]], e.spec.nmol) for i, e in enumerate(ens)]
    eng.histogram_enable(0, *ranges[0])          # ensemble 1 keeps none
    orc = O.Histograms(ens[0].nreplica, *ranges[0])
    idx = [np.arange(e.nreplica, dtype=np.int32) for e in ens]
    T = [e.T.copy() for e in ens]
    P = [e.P.copy() for e in ens]
    rng = np.random.default_rng(3)
    samples = []
    for step in range(6):
        eng.ExecuteSteps(np.concatenate(T), np.concatenate(P))
        avg = eng.all_averages()
        eng.histogram_increment(np.concatenate(idx))
        a = avg[offs[0]:offs[1]]
        orc.increment(idx[0], a, ens[0].spec.nmol)
        samples.append((idx[0].copy(), T[0].copy(), P[0].copy(), a.copy()))
        for i, e in enumerate(ens):
            ai = avg[offs[i]:offs[i + 1]]
            O.replica_exchange(e.ntemp, e.npress, e.spec.pconstant, step, idx[i], T[i], P[i],
                               ai[:, 0] + ai[:, 1] + ai[:, 2], ai[:, 3], rng.random(e.nreplica))
    for c in range(ens[0].nreplica):
        b, hist, ave = eng.histogram(0, c)
        assert np.array_equal(b, orc.bounds[c]) and np.array_equal(hist, orc.hist[c])
        assert np.array_equal(ave, orc.ave[c])
    out = tmp_path / "eng"
    out.mkdir()
    eng.histogram_write(0, str(out))
    # the slot's condition is that of the replica the slot's index names
    Tc, Pc = T[0][idx[0]], P[0][idx[0]]
    for c in range(ens[0].nreplica):
        assert open(O.Histograms.file_name(str(out), Pc[c], Tc[c])).read() == orc.text(c)
    if O.reference_available():
        lib = O._ref_lib()
        ref = tmp_path / "ref"
        ref.mkdir()
        e = ens[0]
        inp = ("nmol %d\nntemp %d\nnpress %d\nnreplica %d\ntemp_min 250\ntemp_max 350\n"
               "press_min 1e5\npress_max 2e8\npconstant %d\nconfined 1\ntconstant 1\n"
               "energy_min %r\nenergy_max %r\nvolume_min %r\nvolume_max %r\n"
               "output_prefix %s\ninput_prefix %s\n"
               % ((e.spec.nmol, e.ntemp, e.npress, e.nreplica, e.spec.pconstant) + tuple(ranges[0]) + (ref, ref)))
        h = lib.ref_remdinfo_create(inp.encode())
        for ix, Ts, Ps, a in samples:
            lib.ref_remdinfo_set_arrays(h, O._ptr(ix, O._ip), O._ptr(Ts), O._ptr(Ps))
            pot = np.ascontiguousarray(a[:, 0] + a[:, 1] + a[:, 2])
            vol = np.ascontiguousarray(a[:, 3])
            lib.ref_remdinfo_increment_histogram(h, O._ptr(pot), O._ptr(vol), O._ptr(np.ascontiguousarray(a)))
        lib.ref_remdinfo_set_arrays(h, O._ptr(idx[0], O._ip), O._ptr(T[0]), O._ptr(P[0]))
        lib.ref_remdinfo_output_histogram(h)
        for c in range(e.nreplica):
            name = os.path.basename(O.Histograms.file_name("", Pc[c], Tc[c]))
            assert open(ref / name).read() == open(out / name).read()
    # ReadHistogramFromBackUp: counts and bounds back exactly, sums to the file's 7 digits
    eng.histogram_enable(0, *ranges[0])
    eng.histogram_read(0, str(out))
    for c in range(ens[0].nreplica):
        b, hist, ave = eng.histogram(0, c)
        assert np.array_equal(b, orc.bounds[c]) and np.array_equal(hist, orc.hist[c])
        assert np.allclose(ave, orc.ave[c], rtol=1e-6, atol=1e-300)
    with pytest.raises(E.RemdError, match="INVALID"):
        eng.histogram(1, 0)
    eng.close()


def test_histograms_in_the_interval_graph():
    """With the device exchange on, the interval graph samples every slot before
    exchanging (one more launch per interval); the result equals the restatement
    fed with the slot -> replica index each interval started from."""
    e = S.small_ensemble("tip5p", 2, nmol=80, ntemp=2, npress=2, seed=73, interval=10)
    eng = E.REMDGPU([e], precision="fp32")
    ranges = _hist_ranges(eng.all_averages(), e.spec.nmol)
    n0 = eng.launches_per_interval()
    eng.enable_device_exchange([(e.ntemp, e.npress)], seed=11)
    eng.histogram_enable(0, *ranges)
    assert eng.launches_per_interval() == n0 + 2
    orc = O.Histograms(e.nreplica, *ranges)
    for _ in range(8):
        idx_pre = eng.conditions()[0]
        eng.execute_device()
        orc.increment(idx_pre, eng.all_averages(), e.spec.nmol)
    for c in range(e.nreplica):
        b, hist, ave = eng.histogram(0, c)
        assert np.array_equal(b, orc.bounds[c]) and np.array_equal(hist, orc.hist[c])
        assert np.array_equal(ave, orc.ave[c])
    assert orc.bounds[:, 4].sum() == 8 * e.nreplica
    eng.close()


def test_histogram_sample_out_of_range_is_an_error():
    e = S.small_ensemble("tip4p", 0, nmol=64, ntemp=2, npress=1, seed=74, interval=5)
    eng = E.REMDGPU([e], precision="fp32")
    eng.histogram_enable(0, 100.0, 200.0, 0.0, 1.0)   # no water sits there
    eng.ExecuteSteps(e.T, e.P)
    with pytest.raises(E.RemdError, match="RANGE"):
        eng.histogram_increment(np.arange(e.nreplica))
    eng.close()
