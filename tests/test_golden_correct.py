"""The reference's only regression test (test/test.sh, test/correct): 150 TIP4P
waters in a 7.4 A nanotube, NP thermostat + z barostat, one interval of 100
steps.  The golden line came from an old FP32 GPU build, so it is a loose
(2e-4) band on the potential energy and volume."""
import numpy as np
import pytest

from oracle import oracle as O
from remd_b200.inputs import read_chk
from tests.common import GOLDEN, golden_conditions, golden_line, golden_spec


@pytest.mark.slow
def test_oracle_reproduces_test_correct_line4():
    spec = golden_spec()
    st = read_chk(f"{GOLDEN}/gpu0000.chk")
    st.T, st.P = golden_conditions()
    orc = O.Oracle(spec, st)
    orc.velocity_scaling()          # init_scaling 1 in test/input/gpu.inp
    orc.ang_velocity_scaling()
    orc.set_tstat_mass(0.5)
    orc.initialize_property()
    orc.steps(100)
    a = orc.average()
    g = dict(zip(golden_line()["columns"], golden_line()["values"]))
    pot = a[0] + a[1] + a[2]
    assert pot == pytest.approx(g["pot"], rel=2e-4)
    assert a[3] == pytest.approx(g["vol"], rel=2e-4)
    # the remaining columns are trajectory quantities of a different (FP32) build
    assert a[6] == pytest.approx(g["T_red"], rel=1e-2)
    assert a[4] == pytest.approx(g["tra"], rel=1e-2)
    assert a[5] == pytest.approx(g["rot"], rel=1e-2)
