"""The reference's own host code driving the engine: oracle/_ref/shim_check
builds the reference's Molecules objects from test/input/gpu0000.chk, hands
them to the REMDGPU shim (remd_b200/shim, the drop-in for src/remdgpu.h) and
compares every interval with the reference's CPU Molecules::ExecuteSteps on
copies of the same replicas."""
import os
import subprocess

import numpy as np
import pytest

from remd_b200.inputs import DATA_DIR, UNIT_PRESS, UNIT_TEMP
from tests.common import GOLDEN

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "shim_check")


@pytest.mark.skipif(not os.path.exists(BIN), reason="shim_check is built from the reference sources")
def test_reference_host_code_drives_engine(tmp_path):
    inp = tmp_path / "g.inp"
    inp.write_text(f"input_prefix {DATA_DIR}/\nmtl_in moltype_tip4p.txt\n" +
                   open(os.path.join(GOLDEN, "shim_golden.inp")).read())
    out = subprocess.run([BIN, str(inp), os.path.join(GOLDEN, "gpu0000.chk"), "2"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    rows = [l.split() for l in out.stdout.splitlines() if l.startswith("rep ")]
    assert len(rows) == 2
    for r in rows:
        gpu = np.array(r[4:22], dtype=float)
        cpu = np.array(r[23:41], dtype=float)
        # REMDGPU reports T, P reduced; Molecules::GetAverage in K and Pa
        cpu[6] /= UNIT_TEMP
        cpu[7:11] /= UNIT_PRESS
        pot_g, pot_c = gpu[0] + gpu[1] + gpu[2], cpu[0] + cpu[1] + cpu[2]
        assert pot_g == pytest.approx(pot_c, rel=1e-4)
        assert gpu[3] == pytest.approx(cpu[3], rel=1e-5)        # volume
        assert gpu[4] == pytest.approx(cpu[4], rel=1e-3)        # translational KE
        assert gpu[13] == pytest.approx(cpu[13], rel=1e-4)      # thermostat s
