"""The statistics of tests/stat_parity.py on synthetic samples (CPU): the
comparison of two runs reads no difference between draws of one
distribution, flags a shifted mean, and pooling independent runs keeps every
chain and stress block."""
import numpy as np

import stat_parity as S


def _run(rng, shift=0.0, chains=80, blocks=60):
    return {"ree_per_chain": (rng.normal(10.0, 1.0, chains) + shift).tolist(),
            "tau_blocks": (rng.normal(0.0, 1.0, (blocks, 3)) + shift).tolist(),
            "msd_z_per_chain": (rng.normal(2.0, 0.5, chains) + shift).tolist(),
            "samples": 40, "steps": 2000, "wall_s": 1.0}


def test_same_distribution_passes_and_shift_is_flagged():
    rng = np.random.default_rng(3)
    same = S.compare(_run(rng), _run(rng))
    assert same["ree_ks_p"] > 1e-3
    assert max(abs(z) for z in same["tau_z"]) < 4 and abs(same["msd_z_z"]) < 4
    moved = S.compare(_run(rng), _run(rng, shift=1.0))
    assert moved["ree_ks_p"] < 1e-3
    assert min(abs(z) for z in moved["tau_z"]) > 4 and abs(moved["msd_z_z"]) > 4


def test_merge_pools_chains_and_blocks():
    rng = np.random.default_rng(4)
    runs = [_run(rng, chains=20, blocks=10) for _ in range(3)]
    m = S.merge(runs)
    assert m["runs"] == 3
    assert len(m["ree_per_chain"]) == 60 and len(m["msd_z_per_chain"]) == 60
    assert len(m["tau_blocks"]) == 30
    assert m["wall_s"] == 3.0
