"""calcMSD on the GPU against the reference's own calcMSD (oracle/_ref):
a synthetic charge-displacement log written in the CH-file format, both
analyses run on it; the reference writes six decimals, so rows agree to
1e-6 (relative, or absolute below 1)."""
import os
import tempfile

import numpy as np
import pytest

import bd_b200 as B
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nch,Tmax,start", [(8, 60, 0), (30, 80, 10)])
def test_msd_matches_reference(nch, Tmax, start):
    if not O.ref_available(0):
        pytest.skip("reference library not built")
    r = np.random.default_rng(nch + Tmax)
    w = r.normal(0, 0.3, (nch * (Tmax + 1), 3)).round(6)
    got = B.msd(w, nch, Tmax, start)
    ref = O.RefSim(0, 10, 2, 20.0, 0.1, 5e-4)
    with tempfile.TemporaryDirectory() as d:
        ch, out = os.path.join(d, "CH.txt"), os.path.join(d, "MSD.txt")
        with open(ch, "w") as f:
            for i in range(Tmax + 1):
                for j in range(nch):
                    x, y, z = w[i * nch + j]
                    f.write("%d %d %d %d %.6f %.6f %.6f\n" % (i, j, 0, 0, x, y, z))
        ref.lib.h_msd(ch.encode(), out.encode(), nch, Tmax, 1, start, 5e-4)
        rows = np.array([list(map(float, l.split(","))) for l in open(out) if l.strip()])
    assert rows.shape == (Tmax - start, 5)
    assert np.allclose(rows[:, 0], 5e-4 * np.arange(1, Tmax - start + 1))
    assert np.allclose(got, rows[:, 1:], rtol=1e-6, atol=1e-6)
