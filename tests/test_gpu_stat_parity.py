"""Statistical parity of long runs, short versions (tests/stat_parity.py
holds the statistics and the long runs' command lines).

* north: the headline path (FP32 particle-mesh products, learned
  preconditioner, noise blocks of 10) against the plain FP64 method (pme64) on
  the 4000-bead extensional workload, 600 steps each from the same
  configuration with independent Philox noise;
* reference: the GPU's reference-mode step (dense hybrid mobility, CA-TEA
  noise, Debye-Hueckel, sequential hop) against the reference's own routines
  on the host, 1000 steps each from the same 500-bead shear configuration with
  independent ran1 seeds.

Pass: per-chain end-to-end distances indistinguishable by the two-sample
Kolmogorov-Smirnov test (p > 0.001), mean stress components and the mean
z-MSD within 4 combined standard errors.
"""
import pytest

import stat_parity as S

pytestmark = pytest.mark.gpu


def _check(cmp_):
    assert cmp_["ree_ks_p"] > 1e-3, cmp_
    assert max(abs(z) for z in cmp_["tau_z"]) < 4.0, cmp_
    assert abs(cmp_["msd_z_z"]) < 4.0, cmp_


def test_north_star_path_matches_plain_fp64_statistics():
    a = S.run_gpu("c1s", "pme32-learned", 600, 20, noise_seed=11)
    b = S.run_gpu("c1s", "pme64", 600, 20, noise_seed=22)
    assert a["lanczos"]["maxed"] == 0 and b["lanczos"]["maxed"] == 0
    _check(S.compare(a, b))


def test_reference_mode_matches_reference_statistics():
    a = S.run_gpu("c0", "tea", 1000, 50, noise_seed=830062920, reference_step=True)
    b = S.run_reference_host("c0", 1000, 50, seed=123456789)
    _check(S.compare(a, b))
