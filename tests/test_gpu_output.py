"""Output files against the reference's own writers (oracle/_ref):
printTrajectory, printRestart, calcExt + printExt (with the unwrapping loop
of the reference's main) and printVisc produce the same text, and the
unwrapped coordinates are bit-identical; centres of mass and gyration
tensors are checked against numpy on the unwrapped coordinates (the
reference's calcCOM / calcRg accumulate from uninitialised values)."""
import glob
import os
import tempfile

import numpy as np
import pytest

import bd_b200 as B
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flow,t", [(0, 2900), (1, 2900)])
def test_output_files_match_reference(flow, t):
    if not O.ref_available(flow):
        pytest.skip("reference library not built")
    Nb, Nc, L = 25, 8, 20.0
    x, y, z = B.random_chains(Nb, Nc, L, 9, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    track = B.random_charges(Nb, Nc, 0.5, 10)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.05, 5e-4, Ncharges=len(track)))
    r = O.RefSim(flow, Nb, Nc, L, 0.05, 5e-4, Ncharges=len(track))
    for s in (c, r):
        s.set_t(t) if s is r else s.set_time(t, t)
        s.update_lattice(t)
    r.set_pos(x, y, z)
    c.set_positions(x, y, z)
    r.apply_pbc()
    c.apply_pbc()
    r.set_charges(np.ascontiguousarray(track, np.int32), len(track))
    c.set_charges(track)
    r.reset_force()
    r.bondforce()
    c.reset_force()
    c.bond_force()
    r.set_strain(0.25)
    with tempfile.TemporaryDirectory() as d:
        def both(name, fr, fc):
            pr, pc = os.path.join(d, "r_" + name), os.path.join(d, "c_" + name)
            fr(pr.encode())
            fc(pc)
            return open(pr).read(), open(pc).read()

        a, b = both("traj.xyz", r.lib.h_print_traj, lambda p: c.write_trajectory(p, t))
        assert a == b and a.count("\n") == Nb * Nc + 2
        a, b = both("ext.txt", r.lib.h_print_ext, lambda p: c.write_ext(p, t, 0.25))
        assert a == b
        ux, uy, uz = (np.zeros(Nb * Nc) for _ in range(3))
        r.lib.h_get_unwrapped(ux, uy, uz)
        p, e, com, rg = c.chain_props()
        assert np.array_equal(p, np.stack([ux, uy, uz]))
        P = p.reshape(3, Nc, Nb)
        assert np.allclose(com, P.mean(2).T, rtol=1e-13, atol=1e-12)
        D = P - P.mean(2, keepdims=True)
        g = np.stack([(D[0] * D[0]).mean(1), (D[0] * D[1]).mean(1), (D[0] * D[2]).mean(1),
                      (D[1] * D[1]).mean(1), (D[1] * D[2]).mean(1), (D[2] * D[2]).mean(1)], 1)
        assert np.allclose(rg, g, rtol=1e-12, atol=1e-12)
        a, b = both("visc.txt", lambda p: r.lib.h_print_visc(p, 10), lambda p: c.write_visc(p, t, 10))
        assert a == b and len(a.split()) == (2 if flow == 0 else 3)
        os.makedirs(os.path.join(d, "res"))
        assert r.lib.h_print_restart(d.encode()) == 0
        ref_restart = glob.glob(os.path.join(d, "res", "R*.xyz"))
        assert len(ref_restart) == 1
        c.write_restart(os.path.join(d, "c_restart.xyz"), t)
        assert open(ref_restart[0]).read() == open(os.path.join(d, "c_restart.xyz")).read()
