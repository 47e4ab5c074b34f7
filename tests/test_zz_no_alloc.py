"""remd_force_snapshot_noalloc: the force snapshot for callers that cannot
allocate device memory (a host program whose own allocator already owns the
GPU, or a loop that must not stall on cudaMalloc/cudaFree).  The test owns
every buffer; the entry point works only in its fixed device scratch.  Its
results must equal the regular snapshot of a one-replica FP32 handle
(remd_create + remd_compute_forces), call after call, although every call
reuses the scratch left by the previous one."""
import numpy as np
import pytest

from remd_b200 import engine as E
from remd_b200 import systems as S
from tests.common import rel

pytestmark = pytest.mark.gpu


def _systems():
    tube = S.make_ensemble("nt", "tip4p", 1, 362, 7.0, 10.3, 9.3, 1, 1, 300, 300, 0.1e6, 0.1e6, 61)
    bulk = S.make_ensemble("nb", "tip5p", 0, 512, 0.0, 11.0, 9.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 62)
    slit = S.make_ensemble("ns", "tip3p", 2, 300, 10.0, 9.0, 8.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 63)
    return [tube, bulk, slit]


def _regular(e):
    eng = E.REMDGPU([e], precision="fp32")
    g = eng.ConvertVariablesToHost(0)
    pairs = eng.pair_count()
    eng.close()
    return g, pairs


def _noalloc(e, torch):
    spec, st = e.spec, e.states[0]
    dev = torch.device("cuda")
    d_r = torch.tensor(st.r.reshape(-1), dtype=torch.float64, device=dev)
    d_q = torch.tensor(st.q.reshape(-1), dtype=torch.float64, device=dev)
    d_wall = None
    if spec.confined:
        w = E.wall_table(spec.confined, spec.nfwall, spec.wall_length, spec.sgm_wall, spec.eps_wall,
                         spec.rho_wall)
        d_wall = torch.tensor(w.reshape(-1), dtype=torch.float64, device=dev)
    n = spec.nmol
    d_f = torch.empty(3 * n, dtype=torch.float64, device=dev)
    d_n = torch.empty(4 * n, dtype=torch.float64, device=dev)
    d_out = torch.empty(8, dtype=torch.float64, device=dev)
    E.force_snapshot_noalloc(spec, d_r.data_ptr(), d_q.data_ptr(), st.L,
                             d_wall.data_ptr() if d_wall is not None else 0, d_f.data_ptr(),
                             d_n.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return (d_f.cpu().numpy().reshape(n, 3), d_n.cpu().numpy().reshape(n, 4), d_out.cpu().numpy())


def test_noalloc_snapshot_equals_regular_snapshot_on_consecutive_calls():
    import torch
    systems = _systems()
    expected = [_regular(e) for e in systems]
    # consecutive calls on different systems (and the first one again): each
    # call finds the previous call's contents in the shared scratch
    for k in [0, 1, 2, 0]:
        f, n, out = _noalloc(systems[k], torch)
        g, pairs = expected[k]
        assert out[7] == 0.0
        assert rel(f, g["f"]) < 1e-5 and rel(n, g["n"]) < 1e-5
        pot = out[0] + out[1] + out[2]
        assert pot == pytest.approx(g["pot"], rel=1e-6)
        assert rel(out[3:6], g["vir"]) < 1e-5
        assert int(out[6]) == pairs


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    big = S.make_ensemble("big", "tip4p", 0, 2100, 0.0, 10.0, 9.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 64)
    dev = torch.device("cuda")
    buf = torch.zeros(4 * 2100, dtype=torch.float64, device=dev)
    with pytest.raises(E.RemdError) as e:
        E.force_snapshot_noalloc(big.spec, buf.data_ptr(), buf.data_ptr(), big.states[0].L, 0,
                                 buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    assert e.value.status == 1 and "2048" in str(e.value)
