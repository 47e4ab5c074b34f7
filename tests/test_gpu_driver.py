"""The reference's own REMD driver (src/main.cxx, src/remd.cxx, unmodified) on
the engine: oracle/_ref/remd_driver links them with the REMDGPU shim and a
stand-in for the members of src/io_manager.cxx (which needs the unvendored VMD
molfile plugin).  It runs the reference's regression input (test/input/gpu.inp:
150 TIP4P waters in a 7.4 A nanotube, one GPU) and must reproduce the golden
line of test/correct, write the per-condition binary logs and the .chk / .gro
outputs of REMD::ExecuteREMD (src/remd.cxx:272-462)."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from remd_b200.inputs import DATA_DIR, UNIT_PRESS, UNIT_TEMP, read_chk
from tests.common import GOLDEN, golden_line

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "remd_driver")

# test/input/gpu.inp with two intervals; paths filled in below
INP = """input_prefix {inp}
output_prefix {out}
mtl_in moltype_tip4p.txt
gro_out gpu
chk_in  gpu
chk_out gpu
cdv_out gpu
nmol 150
natom 600
nsite 4
dt    2.0
rcut 8.655
rswitch 6.655
tconstant  1
temp_max 400
temp_min 200
tstat_mass 0.5
pconstant  2
press_max 5000000000
press_min 4000000000
bstat_mass 0.05
ninterval 2
interval  100
energy_interval 100
snap_interval 1000
chk_interval 10000
nreplica 1
ntemp  1
npress 1
energy_max 0.0
energy_min -80.0
volume_max 40.0
volume_min 0.0
gen_vel 0
cond_mode 0
restart 0
init_scaling 1
nthreads 1
nprocs 1
ngpus 1
gpu_offset 0
confined 1
nfwall 65536
wall_length 7.4
sgm_wall 3.277
eps_wall 0.3886
rho_wall 0.38016
"""


@pytest.mark.skipif(not os.path.exists(BIN), reason="remd_driver is built from the reference sources")
def test_reference_remd_driver_runs_on_the_engine(tmp_path):
    inp, out = tmp_path / "in", tmp_path / "out"
    inp.mkdir()
    out.mkdir()
    shutil.copy(os.path.join(DATA_DIR, "moltype_tip4p.txt"), inp)
    shutil.copy(os.path.join(GOLDEN, "gpu0000.chk"), inp)
    f = tmp_path / "gpu.inp"
    f.write_text(INP.format(inp=f"{inp}/", out=f"{out}/"))
    run = subprocess.run([BIN, str(f)], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    # " rep <rep> <interval> pot vol LJ CLMB WALL T Pz TRA ROT TSTs TSTv BSTz" (src/remd.cxx:302-327)
    rows = [ln.split() for ln in run.stdout.splitlines() if ln.startswith(" rep ")]
    assert [r[2] for r in rows] == ["0", "1"]
    v = np.array(rows[0][3:], dtype=float)
    g = dict(zip(golden_line()["columns"], golden_line()["values"]))
    assert v[0] == pytest.approx(g["pot"], rel=2e-4)
    assert v[1] == pytest.approx(g["vol"], rel=2e-4)
    assert v[0] == pytest.approx(v[2] + v[3] + v[4], rel=1e-5)   # printed to 6 digits
    # trajectory quantities of a different (FP32) build: loose band, as for the oracle
    assert v[5] == pytest.approx(g["T_red"], rel=1e-2)
    # per-condition binary log (REMD::OutputBinary): T, P, 1.0, NUM_ELEM, then 19 doubles
    # (the Average of the replica at that condition) per interval
    T, P = 200.0 / UNIT_TEMP, 4e9 / UNIT_PRESS
    logs = [n for n in os.listdir(out) if n.endswith(".log")]
    assert len(logs) == 1
    raw = open(out / logs[0], "rb").read()
    head = struct.unpack("3di", raw[:28])
    assert head[0] == pytest.approx(T) and head[1] == pytest.approx(P) and head[3] == 19
    recs = np.frombuffer(raw[28:], dtype=np.float64).reshape(-1, 19)
    assert recs.shape[0] == 2
    assert recs[0][0] + recs[0][1] + recs[0][2] == pytest.approx(v[0], rel=1e-5)
    # .chk and .gro of step 0 (UpdateOutputs at chk_interval), readable again
    st = read_chk(str(out / "gpu0000.chk"))
    assert st.r.shape == (150, 3) and np.all((st.r >= 0) & (st.r <= 1))
    gro = open(out / "gpu0000.gro").read().splitlines()
    assert gro[0] == "test" and int(gro[1]) == 600 and len(gro) == 603
    # .cdv snapshot of step 0 (snap_interval) through REMDGPU::OutputCDV
    cdv = open(out / "gpuR0000s0000000.cdv").read().splitlines()
    assert cdv[0].startswith("' box_sx=-7.4 box_sy=-7.4 ") and 'st0="T=200 K, P=4000 MPa"' in cdv[0]
    assert len(cdv) == 601 and cdv[1].split()[:2] == ["0", "0"] and cdv[600].split()[:2] == ["149", "3"]
    # the end-of-run files of REMD::ExecuteREMD (src/remd.cxx:448-460):
    # energy.dat (REMD::OutputEnergy, src/remd.cxx:838-849): the step, then per replica
    # the last interval's potential plus volume x pressure (barostat on), 16 digits
    last = np.array(rows[-1][3:5], dtype=float)   # pot, vol of interval 1 (6 digits)
    ene = open(out / "energy.dat").read().split()
    assert int(ene[0]) == 2 and len(ene) == 2
    assert float(ene[1]) == pytest.approx(last[0] + last[1] * P, rel=1e-5)
    # index_temp.dat / index_press.dat (REMD::OutputIndex, src/remd.cxx:851-879)
    it = open(out / "index_temp.dat").read().split()
    ip = open(out / "index_press.dat").read().split()
    assert int(it[0]) == 2 and int(ip[0]) == 2
    assert float(it[1]) == pytest.approx(T, abs=1e-6) and float(ip[1]) == pytest.approx(P, abs=1e-6)
    # accept_rate.dat and tunnel_count.dat (REMDInfo, src/remdinfo.cxx:762-832): one
    # condition, so no exchange pair and one tunnel counter
    assert open(out / "accept_rate.dat").read().startswith("#Ti,Pi,Tj,Pj,AR\n")
    assert len(open(out / "tunnel_count.dat").read().split()) == 1
