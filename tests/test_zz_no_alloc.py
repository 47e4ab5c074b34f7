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


class _Buffers:
    """Caller-owned device buffers for one system (allocated once, up front)."""

    def __init__(self, e, torch):
        spec, st = e.spec, e.states[0]
        dev = torch.device("cuda")
        self.spec, self.L, n = spec, st.L, spec.nmol
        self.r = torch.tensor(st.r.reshape(-1), dtype=torch.float64, device=dev)
        self.q = torch.tensor(st.q.reshape(-1), dtype=torch.float64, device=dev)
        self.wall = None
        if spec.confined:
            w = E.wall_table(spec.confined, spec.nfwall, spec.wall_length, spec.sgm_wall, spec.eps_wall,
                             spec.rho_wall)
            self.wall = torch.tensor(w.reshape(-1), dtype=torch.float64, device=dev)
        self.f = torch.empty(3 * n, dtype=torch.float64, device=dev)
        self.n = torch.empty(4 * n, dtype=torch.float64, device=dev)
        self.out = torch.empty(8, dtype=torch.float64, device=dev)

    def call(self, torch, wall_ptr=None):
        wp = wall_ptr if wall_ptr is not None else (self.wall.data_ptr() if self.wall is not None else 0)
        E.force_snapshot_noalloc(self.spec, self.r.data_ptr(), self.q.data_ptr(), self.L, wp,
                                 self.f.data_ptr(), self.n.data_ptr(), self.out.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        n = self.spec.nmol
        return (self.f.cpu().numpy().reshape(n, 3), self.n.cpu().numpy().reshape(n, 4),
                self.out.cpu().numpy())


def test_noalloc_snapshot_equals_regular_snapshot_on_consecutive_calls():
    """Bit for bit: the same FP32 arithmetic, and the results depend neither on
    the tile size nor on the neighbour skin (the per-step lists are exact)."""
    import torch
    systems = _systems()
    expected = [_regular(e) for e in systems]
    bufs = [_Buffers(e, torch) for e in systems]
    # consecutive calls on different systems (and the first one again): each
    # call finds the previous call's contents in the shared scratch
    free0 = None
    for k in [0, 1, 2, 0, 2]:
        f, n, out = bufs[k].call(torch)
        if free0 is None:
            free0 = torch.cuda.mem_get_info()[0]
        g, pairs = expected[k]
        assert out[7] == 0.0
        assert np.array_equal(f, g["f"]) and np.array_equal(n, g["n"])
        # energies and virial: the same per-32-molecule partial sums, added up in
        # another order (a warp butterfly here, a host loop in remd_get_state)
        for a, b in [(out[0], g["lj"]), (out[1], g["clmb"]), (out[2], g["wall"])]:
            assert a == pytest.approx(b, rel=1e-13, abs=1e-13)
        assert np.allclose(out[3:6], g["vir"], rtol=1e-13, atol=1e-13)
        assert int(out[6]) == pairs
    # the calls after the first allocated no device memory
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_reports_neighbour_overflow():
    """A box compressed to about 4.6x liquid density has more neighbours per
    molecule than the fixed capacity: the error word says so (out[7] = 1)."""
    import copy
    import torch
    e = S.make_ensemble("dense", "tip3p", 0, 1000, 0.0, 9.0, 8.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 65)
    d = copy.deepcopy(e)
    d.states[0].L = d.states[0].L * 0.6
    _, _, out = _Buffers(d, torch).call(torch)
    assert out[7] == 1.0
    # the next call on a normal system starts clean
    tube = _systems()[0]
    _, _, out = _Buffers(tube, torch).call(torch)
    assert out[7] == 0.0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    big = S.make_ensemble("big", "tip4p", 0, 2100, 0.0, 10.0, 9.0, 1, 1, 300, 300, 0.1e6, 0.1e6, 64)
    dev = torch.device("cuda")
    buf = torch.zeros(4 * 2100, dtype=torch.float64, device=dev)
    with pytest.raises(E.RemdError) as e:
        E.force_snapshot_noalloc(big.spec, buf.data_ptr(), buf.data_ptr(), big.states[0].L, 0,
                                 buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    assert e.value.status == 1 and "2048" in str(e.value)


def test_noalloc_rejects_a_misaligned_wall_table():
    """The wall table is read as 16-byte {f, U} pairs: a table starting 8 bytes
    into a buffer is refused before anything is launched."""
    import torch
    tube = _Buffers(_systems()[0], torch)
    with pytest.raises(E.RemdError) as e:
        tube.call(torch, wall_ptr=tube.wall.data_ptr() + 8)
    assert e.value.status == 1 and "aligned" in str(e.value)
