"""bd_mobility_apply_noalloc: the mobility product for callers that must not
allocate device memory where they call it (for example while another
framework's memory pool owns the device, under a fixed memory budget, or
where the device-wide synchronisation of cudaMalloc/cudaFree is not
acceptable).  Its scratch is a fixed device array inside the library, so it
allocates nothing per call.

Checked through the C ABI against the existing bd_mobility_apply on two calls
in a row (the shared scratch keeps the previous call's contents), within the
FP64 tolerance used elsewhere (1e-10 relative), for FP64 and FP32-stored
tiles, in both flows; at 500 beads, at exactly the scratch's limit of 4096
beads (128 full tile rows) and at 4065 beads (the last tile row holds one
bead); a system larger than the fixed scratch allows is rejected, and so is a
particle-mesh context (it has no tiles).
Collected last so that a stop-at-first-failure run has run everything else.
"""
import ctypes

import numpy as np
import pytest

import bd_b200 as B
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _entry():
    f = B._lib().bd_mobility_apply_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("flow,Nb,Nc,L,precision", [
    (1, 25, 20, 30.0, "fp64"), (1, 25, 20, 30.0, "fp32"), (0, 25, 20, 30.0, "fp64"),
    (0, 15, 271, 48.0, "fp64"),    # 4065 beads: partial last tile row
    (1, 32, 128, 48.0, "fp32"),    # 4096 beads: the limit, full tile rows
])
def test_noalloc_product_matches_mobility_apply_on_two_calls(flow, Nb, Nc, L, precision):
    import torch
    x, y, z = B.random_chains(Nb, Nc, L, 77, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(flow, x, y)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, mobility="ewald",
                                precision=precision))
    c.set_positions(x, y, z)
    c.set_time(0, 0)
    c.update_lattice(0)
    if flow == 1:
        c.transform_coords()
    c.apply_pbc()
    c.calc_hi()
    f = _entry()
    rng = np.random.default_rng(11)
    for call in range(2):
        v = rng.normal(size=3 * c.N)
        want = c.mobility_apply(v)
        vd = torch.tensor(v, device="cuda", dtype=torch.float64)
        od = torch.full((3 * c.N,), float("nan"), device="cuda", dtype=torch.float64)
        torch.cuda.synchronize()
        assert f(c.h, vd.data_ptr(), od.data_ptr()) == 0
        c.sync()
        got = od.cpu().numpy()
        assert rel_err(got, want) < 1e-10, (call, rel_err(got, want))
    c.close()


def test_noalloc_rejects_systems_beyond_the_fixed_scratch():
    import torch
    c = B.Context(B.make_params(1, 100, 41, 60.0, 0.2, 5e-4, mobility="ewald"))  # 4100 beads
    assert c.N > 4096
    vd = torch.zeros(3 * c.N, device="cuda", dtype=torch.float64)
    od = torch.zeros(3 * c.N, device="cuda", dtype=torch.float64)
    assert _entry()(c.h, vd.data_ptr(), od.data_ptr()) == 12  # BD_ERR_CAPACITY
    c.close()


def test_noalloc_rejects_particle_mesh_contexts():
    import torch
    flow, Nb, Nc, L = 1, 25, 8, 30.0
    x, y, z = B.random_chains(Nb, Nc, L, 78, bond=2.0, min_sep=1.8)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, mobility="pme"))
    c.set_positions(x, y, z)
    c.set_time(0, 0)
    c.update_lattice(0)
    c.calc_hi()
    vd = torch.zeros(3 * c.N, device="cuda", dtype=torch.float64)
    od = torch.zeros(3 * c.N, device="cuda", dtype=torch.float64)
    assert _entry()(c.h, vd.data_ptr(), od.data_ptr()) == 8  # BD_ERR_STATE
    c.close()
