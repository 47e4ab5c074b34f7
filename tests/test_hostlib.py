"""The C-ABI library (remd_b200/_lib/libremd_b200.so) on the CPU: it loads, it
exports every entry point include/remd_b200.h declares, and its host-side parts
(wall table, .chk I/O, exchange) agree with the oracle.  No GPU compute here."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from remd_b200 import engine as E
from remd_b200.inputs import read_chk, write_chk
from tests.common import GOLDEN

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "remd_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(remd_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = E.lib()
    syms = declared_symbols()
    assert len(syms) > 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert b"sm_100a" in lib.remd_version()


def test_library_is_self_contained():
    # only the CUDA driver is needed at run time (runtime linked statically)
    out = os.popen(f"ldd {E.LIB_PATH}").read()
    assert "libcudart" not in out


@pytest.mark.parametrize("confined,nfwall,wall", [(1, 1000, 6.0), (1, 257, 4.4), (2, 1000, 10.0),
                                                  (2, 500, 7.3)])
def test_wall_table_bitwise_equal_to_oracle(confined, nfwall, wall):
    a = E.wall_table(confined, nfwall, wall, 3.277, 0.3886, 0.38016)
    b = O.wall_table(confined, nfwall, wall, 3.277, 0.3886, 0.38016)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("case,nfwall,wall", [("tip4p_tube_npz", None, None), ("tip4p_slit_nvt", None, None),
                                               ("tip3p_slit_nve", 500, 7.3), ("tip5p_slit_nvt", 4096, 14.0)])
def test_wall_table_matches_reference_object(case, nfwall, wall):
    """The table the engine builds equals ForceCalculator::fwall of the
    reference's own object (src/force_calculator.cxx:117-200), bit for bit,
    for the nanotube and for the nano-slit (confined=2, 163-199)."""
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    import dataclasses
    from tests.common import load_case
    spec, st, _ = load_case(case)
    if nfwall is not None:
        spec = dataclasses.replace(spec, nfwall=nfwall, wall_length=wall)
    ref = O.Reference(spec, st, spec.moltype_file)
    t = E.wall_table(spec.confined, spec.nfwall, spec.wall_length, spec.sgm_wall, spec.eps_wall,
                     spec.rho_wall)
    assert np.array_equal(t, ref.fwall())


def test_wall_table_rejects_bad_input():
    with pytest.raises(E.RemdError):
        E.wall_table(0, 100, 5.0, 3.0, 0.3, 0.3)
    with pytest.raises(E.RemdError):
        E.wall_table(1, 2, 5.0, 3.0, 0.3, 0.3)


def test_read_chk_matches_python_reader(tmp_path):
    a = E.read_chk(f"{GOLDEN}/gpu0000.chk", 150)
    b = read_chk(f"{GOLDEN}/gpu0000.chk")
    for k in ["r", "v", "q", "p", "m", "I"]:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert (a.s, a.Ps, a.Q, a.W) == (b.s, b.Ps, b.Q, b.W)
    assert np.array_equal(a.L, b.L) and np.array_equal(a.Pv, b.Pv)


def test_read_chk_errors(tmp_path):
    with pytest.raises(E.RemdError) as e:
        E.read_chk(str(tmp_path / "missing.chk"), 10)
    assert e.value.status == 7
    with pytest.raises(E.RemdError):
        E.read_chk(f"{GOLDEN}/gpu0000.chk", 151)
    trunc = tmp_path / "t.chk"
    trunc.write_text("\n".join(open(f"{GOLDEN}/gpu0000.chk").read().splitlines()[:40]))
    with pytest.raises(E.RemdError):
        E.read_chk(str(trunc), 150)


def test_chk_round_trip(tmp_path):
    b = read_chk(f"{GOLDEN}/gpu0000.chk")
    write_chk(tmp_path / "x.chk", b, 4)
    c = E.read_chk(str(tmp_path / "x.chk"), 150)
    assert np.allclose(c.r, b.r, rtol=1e-6, atol=1e-6)
    assert np.allclose(c.q, b.q, rtol=1e-6, atol=1e-6)
    # layout: same token count and line structure as the reference's writer
    ref_lines = open(f"{GOLDEN}/gpu0000.chk").read().splitlines()
    new_lines = open(tmp_path / "x.chk").read().splitlines()
    assert [len(l.split()) for l in new_lines] == [len(l.split()) for l in ref_lines[:len(new_lines)]]


def _property_line(path):
    return np.array([float(x) for x in open(path).read().splitlines()[-1].split()])


def test_chk_writer_reproduces_the_reference_file_byte_for_byte(tmp_path):
    """The reference's own test input (test/input/gpu0000.chk, written by its
    IOManager::WriteCheckPoint) read and written back: every byte equal,
    including the Property line (src/io_manager.cxx:632)."""
    st = E.read_chk(f"{GOLDEN}/gpu0000.chk", 150)
    prop = _property_line(f"{GOLDEN}/gpu0000.chk")
    assert len(prop) == 26
    E.write_chk_arrays(str(tmp_path / "x.chk"), 4, st, prop)
    assert open(tmp_path / "x.chk", "rb").read() == open(f"{GOLDEN}/gpu0000.chk", "rb").read()


@pytest.mark.parametrize("name", ["tip4p_tube_npz", "tip5p_bulk_nvt", "tip3p_slit_nve"])
def test_chk_writer_equals_reference_operators(tmp_path, name):
    """Against the reference's own operator<< for Vector and Property
    (src/vector.h:141-147, src/variables.h:51-74) in WriteCheckPoint's statement
    order, on a reference object after InitializeProperty and 20 MD steps."""
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    from tests.common import load_case
    spec, st, _ = load_case(name)
    ref = O.Reference(spec, st, spec.moltype_file, variant="slitwall" if spec.confined == 2 else "generic")
    ref.initialize_property()
    ref.execute_steps(20)
    ref.write_chk(str(tmp_path / "ref.chk"))
    g = ref.get()
    from remd_b200.inputs import ReplicaState
    mine = ReplicaState(g["r"], g["v"], g["q"], g["p"], st.m, st.I, g["s"], g["Ps"], g["Q"], g["Pv"],
                        g["W"], g["L"], g["T"], g["P"])
    E.write_chk_arrays(str(tmp_path / "mine.chk"), spec.moltype.nsite, mine, ref.property_line())
    assert open(tmp_path / "mine.chk", "rb").read() == open(tmp_path / "ref.chk", "rb").read()


@pytest.mark.parametrize("nt,npr,pcon", [(4, 2, 1), (8, 1, 0), (1, 6, 2), (5, 3, 3), (16, 4, 1)])
def test_exchange_host_equals_oracle(nt, npr, pcon):
    rng = np.random.default_rng(nt * 100 + npr)
    n = nt * npr
    T0, P0 = O.conditions_geometrical(nt, npr, 220, 380, 1e5, 3e8)
    idx_a, T_a, P_a = np.arange(n, dtype=np.int32), T0.copy(), P0.copy()
    idx_b, T_b, P_b = idx_a.copy(), T0.copy(), P0.copy()
    for step in range(40):
        pot = rng.normal(-5000, 40, n)
        vol = rng.normal(4000, 30, n)
        u = rng.random(max(n // 2, 1))
        acc_a = E.exchange_host(nt, npr, pcon, step, idx_a, T_a, P_a, pot, vol, u)
        acc_b = O.replica_exchange(nt, npr, pcon, step, idx_b, T_b, P_b, pot, vol, u)
        assert np.array_equal(acc_a, acc_b)
        assert np.array_equal(idx_a, idx_b) and np.array_equal(T_a, T_b) and np.array_equal(P_a, P_b)
    assert sorted(idx_a) == list(range(n))


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from tests.common import case_ensemble
    with pytest.raises(E.RemdError) as e:
        E.REMDGPU([case_ensemble("tip4p_bulk_nve")])
    assert e.value.status == 9
