"""The C oracle restates the reference's generic FP64 CPU path.  These tests pin
it against (a) fixtures the reference itself produced (tests/golden/ref_*.npz,
made by tests/golden/make_golden.py) and (b) the compiled reference, when
oracle/_ref is present."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.common import CASES, GOLDEN, HIST_RANGES, NSTEPS, histogram_samples, load_case, rel


@pytest.mark.parametrize("name", list(CASES))
def test_force_snapshot_matches_reference(name):
    spec, st, z = load_case(name)
    orc = O.Oracle(spec, st)
    orc.initialize_property()
    assert rel(orc.f, z["snap_f"]) < 1e-13
    assert rel(orc.n, z["snap_n"]) < 1e-12
    p = orc.prop()
    e = z["snap_ener"]
    assert p["lj"] == pytest.approx(e[0], rel=1e-13)
    assert p["clmb"] == pytest.approx(e[1], rel=1e-13)
    assert p["wall"] == pytest.approx(e[2], rel=1e-13, abs=1e-12)
    assert np.allclose(p["vir"], e[3:6], rtol=1e-12, atol=1e-9)
    assert p["tra"] == pytest.approx(e[6], rel=1e-13)
    assert p["rot"] == pytest.approx(e[7], rel=1e-13)


@pytest.mark.parametrize("name", list(CASES))
def test_twenty_steps_match_reference(name):
    spec, st, z = load_case(name)
    orc = O.Oracle(spec, st)
    orc.initialize_property()
    orc.steps(NSTEPS)
    # identical arithmetic up to the reference's uninitialised bulk wall term
    assert rel(orc.r, z["after_r"]) < 1e-12
    assert rel(orc.v, z["after_v"]) < 1e-10
    assert rel(orc.q, z["after_q"]) < 1e-12
    assert rel(orc.p, z["after_p"]) < 1e-10
    assert rel(orc.f, z["after_f"]) < 1e-9
    p = orc.prop()
    sc = z["after_scal"]
    assert p["s"] == pytest.approx(sc[0], rel=1e-11)
    assert p["Ps"] == pytest.approx(sc[1], rel=1e-8, abs=1e-10)
    assert np.allclose(p["Pv"], sc[2:5], rtol=1e-8, atol=1e-10)
    assert np.allclose(p["L"], sc[5:8], rtol=1e-13)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (no reference sources)")
@pytest.mark.parametrize("name", ["tip4p_tube_npz", "tip3p_bulk_npt", "tip4p_slit_nvt", "tip5p_slit_nvt",
                                  "tip3p_slit_nve"])
def test_live_reference_bitwise(name):
    """With the same compiler flags the restatement is bit-identical for tube
    and slit systems.  Slit systems run on the reference build whose broken CPU
    slit wall is replaced by the reference GPU kernel's lookup
    (oracle/ref_slit_wall.cxx): the pair forces, the wall table, the
    integrator and the properties there are the reference's own code."""
    spec, st, _ = load_case(name)
    variant = "slitwall" if spec.confined == 2 else "generic"
    if not O.reference_available(variant):
        pytest.skip(f"oracle/_ref {variant} build missing")
    ref = O.Reference(spec, st, spec.moltype_file, variant=variant)
    orc = O.Oracle(spec, st)
    ref.initialize_property()
    orc.initialize_property()
    ref.execute_steps(5)
    orc.steps(5)
    g = ref.get()
    pr, po = ref.prop(), orc.prop()
    if spec.confined:
        assert np.array_equal(g["r"], orc.r) and np.array_equal(g["p"], orc.p)
        assert np.array_equal(g["f"], orc.f) and np.array_equal(g["n"], orc.n)
        assert (pr["lj"], pr["clmb"], pr["wall"]) == (po["lj"], po["clmb"], po["wall"])
    else:
        assert rel(g["r"], orc.r) < 1e-13
        assert pr["lj"] == pytest.approx(po["lj"], rel=1e-12)


def test_exchange_matches_reference_remdinfo():
    """REMD::ReplicaExchange restatement vs the reference's REMDInfo pair lists."""
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(5)
    nt, npr = 4, 2
    inp = ("nmol 64\nntemp %d\nnpress %d\nnreplica %d\ntemp_min 250\ntemp_max 350\n"
           "press_min 1e5\npress_max 2e8\npconstant 1\nconfined 0\ntconstant 1\n" % (nt, npr, nt * npr))
    lib = O._ref_lib()
    h = lib.ref_remdinfo_create(inp.encode())
    n = nt * npr
    idx_r = np.zeros(n, dtype=np.int32)
    T_r, P_r = np.zeros(n), np.zeros(n)
    lib.ref_remdinfo_arrays(h, O._ptr(idx_r, O._ip), O._ptr(T_r), O._ptr(P_r))
    T_o, P_o = O.conditions_geometrical(nt, npr, 250, 350, 1e5, 2e8)
    assert np.array_equal(T_o, T_r) and np.array_equal(P_o, P_r)
    idx_o = np.arange(n, dtype=np.int32)
    for step in range(24):
        pot = rng.normal(-4000, 30, n)
        vol = rng.normal(3000, 20, n)
        u = rng.random(n)
        acc_r = np.zeros(n, dtype=np.int32)
        lib.ref_remdinfo_exchange(h, step, O._ptr(pot), O._ptr(vol), O._ptr(u), O._ptr(acc_r, O._ip))
        acc_o = O.replica_exchange(nt, npr, 1, step, idx_o, T_o, P_o, pot, vol, u)
        lib.ref_remdinfo_arrays(h, O._ptr(idx_r, O._ip), O._ptr(T_r), O._ptr(P_r))
        assert np.array_equal(acc_o, acc_r[:len(acc_o)])
        assert np.array_equal(idx_o, idx_r)
        assert np.array_equal(T_o, T_r) and np.array_equal(P_o, P_r)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (no reference sources)")
def test_gro_restatement_matches_reference_writer(tmp_path):
    """The .gro restatement (ConvertMoleculesToAtoms + write_gro_file) gives the
    same bytes as the reference's own writer on the same atoms, including
    coordinates that round at the last printed digit and negative ones."""
    from remd_b200 import systems as S
    e = S.small_ensemble("tip5p", 1, nmol=40, ntemp=1, npress=1, seed=17)
    st, mt = e.states[0], e.spec.moltype
    atoms = O.gro_atoms(mt.name, mt.names, st.r, st.q, st.L, mt.r)
    text = O.gro_text(*atoms, L=st.L * 0.1)
    path = str(tmp_path / "ref.gro")
    O.reference_write_gro(path, *atoms, L=st.L * 0.1)
    assert open(path).read() == text
    lines = text.splitlines()
    assert lines[0] == "test" and int(lines[1]) == 40 * 5 and len(lines) == 40 * 5 + 3
    assert lines[2][5:15] == "TIP5P   OW"


def test_cdv_restatement_known_answer():
    """REMDGPU::OutputCDV (src/remdgpu.cu:700-804), worked by hand for a tube box:
    the box spans +-wall_length in x and y, the centres come from the 32-bit
    fixed-point fraction (r = 0.1 of 30 A prints as -12 after the float
    rounding), and the sites are offset by R(q) b."""
    from remd_b200.inputs import UNIT_PRESS, UNIT_TEMP
    r = np.array([[0.5, 0.5, 0.5], [0.25, 0.75, 0.1]])
    q = np.array([[1.0, 0.0, 0.0, 0.0], [0.5, 0.5, 0.5, 0.5]])
    text = O.cdv_text(r, q, [20.0, 20.0, 30.0], [[0.0, 0.0, 0.0], [0.75, 0.5, 0.0]], 2.5, 0.0625,
                      confined=1, wall_length=6.0)
    lines = text.splitlines()
    assert lines[0] == ("' box_sx=-6 box_sy=-6 box_sz=-15 box_ex=6 box_ey=6 box_ez=15"
                        " r0=1.0 r1=0.8 r2=0.8 c0=(1.0,0.0,0.0) c1=(1.0,1.0,1.0) c2=(1.0,1.0,1.0)"
                        ' bond0_c=(1.0,1.0,1.0) st0="T=%g K, P=%g MPa" st0_pos=(-2.0,-2.0)'
                        % (2.5 * UNIT_TEMP, 0.0625 * UNIT_PRESS / 1e6))
    assert lines[1:] == ["0 0 0 0 0", "0 1 0.75 0.5 0", "1 0 -5 5 -12", "1 1 -5 5.75 -11.5"]
    # bulk and slit boxes
    bulk = O.cdv_text(r[:1], q[:1], [20.0, 20.0, 30.0], [[0.0, 0.0, 0.0]], 2.5, 0.0625, 0, 0.0)
    assert bulk.startswith("' box_sx=-10 box_sy=-10 box_sz=-15 box_ex=10 box_ey=10 box_ez=15 ")
    slit = O.cdv_text(r[:1], q[:1], [20.0, 20.0, 30.0], [[0.0, 0.0, 0.0]], 2.5, 0.0625, 2, 9.0)
    assert slit.startswith("' box_sx=-10 box_sy=-10 box_sz=-4.5 box_ex=10 box_ey=10 box_ez=4.5 ")


def test_histogram_restatement_matches_golden():
    """The restatement against the reference REMDInfo's own histogram files for
    the seeded samples (tests/golden/ref_histograms.json, make_golden.py)."""
    import json
    g = json.load(open(os.path.join(GOLDEN, "ref_histograms.json")))
    orc = O.Histograms(g["nrep"], *g["ranges"])
    for idx, avg in histogram_samples(np.random.default_rng(g["seed"]), g["nrep"], g["nmol"], g["nint"]):
        orc.increment(idx, avg, g["nmol"])
    for c in range(g["nrep"]):
        assert orc.text(c) == g["files"][c], c


def test_histogram_restatement_matches_reference_remdinfo(tmp_path):
    """REMD::IncrementHistogram + REMDInfo::OutputHistogram: the restatement and
    the reference's compiled REMDInfo, fed the same samples, write the same bytes."""
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    nt, npr, nmol = 3, 2, 50
    nrep = nt * npr
    inp = ("nmol %d\nntemp %d\nnpress %d\nnreplica %d\ntemp_min 250\ntemp_max 350\n"
           "press_min 1e5\npress_max 2e8\npconstant 1\nconfined 0\ntconstant 1\n"
           "energy_min -60\nenergy_max -20\nvolume_min 25\nvolume_max 35\n"
           "output_prefix %s\ninput_prefix %s\n" % (nmol, nt, npr, nrep, tmp_path, tmp_path))
    lib = O._ref_lib()
    h = lib.ref_remdinfo_create(inp.encode())
    Tc = np.linspace(2.0, 3.0, nrep)
    Pc = np.linspace(0.01, 0.1, nrep)
    orc = O.Histograms(nrep, *HIST_RANGES)
    rng = np.random.default_rng(9)
    for idx, avg in histogram_samples(rng, nrep, nmol, 40):
        T = np.zeros(nrep)
        P = np.zeros(nrep)
        T[idx], P[idx] = Tc, Pc           # replica idx[c] holds condition c
        lib.ref_remdinfo_set_arrays(h, O._ptr(idx, O._ip), O._ptr(T), O._ptr(P))
        pot = np.ascontiguousarray(avg[:, 0] + avg[:, 1] + avg[:, 2])
        vol = np.ascontiguousarray(avg[:, 3])
        lib.ref_remdinfo_increment_histogram(h, O._ptr(pot), O._ptr(vol), O._ptr(np.ascontiguousarray(avg)))
        orc.increment(idx, avg, nmol)
    lib.ref_remdinfo_output_histogram(h)
    for c in range(nrep):
        ref = open(O.Histograms.file_name(str(tmp_path), Pc[c], Tc[c])).read()
        assert ref == orc.text(c), c
    assert orc.bounds[:, 4].sum() == 40 * nrep
