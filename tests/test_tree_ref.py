"""CPU checks of the restated reference tree (oracle/tree_ref.py), the
yardstick that tests/test_gpu_tree.py sets this library's tree mode beside:
its Peano-Hilbert order, its theta -> 0 limit (the direct sum), and its
errors on config 1 against the committed fixture."""
import json
import os

import numpy as np

import oracle
from conftest import ROOT, err_report
from oracle import tree_ref
from starsmasher_b200 import inputs


def test_hilbert_order_is_a_unit_step_walk():
    g = np.stack(np.meshgrid(np.arange(4), np.arange(4), np.arange(4), indexing="ij"), -1)
    g = g.reshape(-1, 3).astype(float)
    k = tree_ref.hilbert_keys(g, bits=2)
    assert len(np.unique(k)) == 64
    steps = np.abs(np.diff(g[np.argsort(k)], axis=0)).sum(axis=1)
    assert np.all(steps == 1)


def test_theta_zero_is_the_direct_sum():
    s = inputs.single_polytrope(3000, 1.5, seed=3)
    got = tree_ref.forces(s.x, s.y, s.z, s.m, s.range2, 0.0)
    want = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0)
    for a, b in zip(got, want):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)


def test_config1_errors_match_fixture():
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "tree_ref_errors.json")))["config1"]
    s = inputs.cached("config1")
    want = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0)
    r = err_report(*tree_ref.forces(s.x, s.y, s.z, s.m, s.range2, 0.3), *want)
    for k in ("acc_rms", "acc_max", "pot_rms", "pot_max"):
        assert abs(r[k] - ref["theta_0.3"][k]) <= 1e-3 * ref["theta_0.3"][k], (k, r[k], ref["theta_0.3"][k])


def test_sampled_groups_equal_the_full_walk():
    """Walking only the groups that hold chosen particles (how config 3 is
    sampled) gives exactly the full walk's rows and NaN elsewhere."""
    s = inputs.single_polytrope(3000, 1.5, seed=3)
    full = tree_ref.forces(s.x, s.y, s.z, s.m, s.range2, 0.3)
    part = tree_ref.forces(s.x, s.y, s.z, s.m, s.range2, 0.3, only=np.array([0, 5, 1000, 2999]))
    rows = np.flatnonzero(~np.isnan(part[0]))
    assert 4 <= rows.size <= 4 * tree_ref.NCRIT
    assert {0, 5, 1000, 2999} <= set(rows.tolist())
    for a, b in zip(part, full):
        np.testing.assert_array_equal(a[rows], b[rows])
