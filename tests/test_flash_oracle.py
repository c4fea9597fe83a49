"""CPU: pins the flash oracle (oracle/flash_oracle.c) against the reference's
own device flash compiled for the host (oracle/_ref/libref_flash.so) on seeded
pure-N2O batches: phase labels bit-exact, success flags equal, p and T within
1e-9 relative."""
import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import cases
import flash_cases as F


@pytest.mark.parametrize("policy,n", [("exact", 1500), ("fixed", 300)])
def test_oracle_flash_matches_reference(policy, n):
    image = F.model_image()
    q, e, guess = cases.flash_batch(n, seed=77 + n, seed_policy=policy)
    ref, ref_ok, ref_cnt = oracle.ref_flash_recover(image, q, e, guess)
    out, ok, cnt = F.oracle_flash(oracle, image, q, e, guess)
    s = F.compare(out, ok, ref, ref_ok)
    assert s["success_equal"], s
    assert s["label_mismatch"] == 0, s
    assert s["p_rel"] <= F.P_T_TOL and s["T_rel"] <= F.P_T_TOL, s
    assert s["c_rel"] <= F.STATE_TOL, s
    if policy == "exact":
        assert ref_ok.all()
        assert min(s["labels"]) > 0  # gas, liquid and two-phase all present
    # the per-cell work counters follow the same candidate sequence
    assert np.mean(np.all(cnt[:, 2:5] == ref_cnt[:, 2:5], axis=1)) > 0.99


def test_oracle_flash_edge_inputs():
    image = F.model_image()
    q, e, guess = cases.flash_batch(8, seed=5)
    q[0] = 0.0            # empty cell
    e[1] = np.nan         # non-finite energy
    q[2] = -1.0           # negative mass
    e[3] = -1e12          # far outside the EOS domain
    ref, ref_ok, _ = oracle.ref_flash_recover(image, q, e, guess)
    out, ok, _ = F.oracle_flash(oracle, image, q, e, guess)
    assert np.array_equal(ok != 0, ref_ok != 0)
    assert not ok[:4].any()
