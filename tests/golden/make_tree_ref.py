"""Errors of the reference's Barnes-Hut algorithm (restated on the CPU in
oracle/tree_ref.py) against the direct FP64 sum (oracle row form), on the
benchmark's config 1 and config 2 inputs at theta 0.3, 0.5 and 0.7, and on
sampled groups of config 3 (the 1M-particle red giant: 63 random particles
and the point-mass core, every row of their groups).  Writes
tree_ref_errors.json beside this script; tests/test_tree_ref.py checks the
restatement against it and tests/test_gpu_tree.py sets this library's tree
mode beside it.

    python tests/golden/make_tree_ref.py [config1,config2,config3]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from conftest import err_report  # noqa: E402
from oracle import tree_ref  # noqa: E402
from starsmasher_b200 import inputs  # noqa: E402

THETAS = (0.3, 0.5, 0.7)


def sampled(name, nsample=63, seed=7):
    """Rows of the groups holding nsample random particles and particle 0."""
    s = inputs.cached(name)
    pick = np.concatenate([[0], np.random.default_rng(seed).choice(np.arange(1, s.n), nsample,
                                                                   replace=False)])
    res = {"n": int(s.n), "sampled_particles": int(pick.size)}
    rows = None
    for th in THETAS:
        t0 = time.time()
        got = tree_ref.forces(s.x, s.y, s.z, s.m, s.range2, th, only=pick)
        if rows is None:
            rows = np.flatnonzero(~np.isnan(got[0]))
            ex = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0, row_idx=rows)
            res["rows"] = int(rows.size)
        g = [a[rows] for a in got]
        r = err_report(*g, *ex)
        core = int(np.flatnonzero(rows == 0)[0])
        da = np.sqrt(sum((g[q][core] - ex[q][core]) ** 2 for q in range(3)))
        amag = np.sqrt(sum(ex[q][core] ** 2 for q in range(3)))
        r["core_acc_rel"] = float(da / amag)
        r["core_pot_rel"] = float(abs(g[3][core] - ex[3][core]) / abs(ex[3][core]))
        res[f"theta_{th:g}"] = {k: float("%.4g" % v) if isinstance(v, float) else v
                                for k, v in r.items()}
        print(name, "sampled", th, round(time.time() - t0, 1), res[f"theta_{th:g}"], flush=True)
    return res


def main(names):
    path = os.path.join(HERE, "tree_ref_errors.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for name in names:
        if name == "config3":
            out["config3_sampled"] = sampled(name)
            continue
        s = inputs.cached(name)
        t0 = time.time()
        ex = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0)
        res = {"n": int(s.n), "direct_seconds": round(time.time() - t0, 1)}
        for th in THETAS:
            t0 = time.time()
            got = tree_ref.forces(s.x, s.y, s.z, s.m, s.range2, th)
            r = err_report(*got, *ex)
            res[f"theta_{th:g}"] = {k: float("%.4g" % v) if isinstance(v, float) else v
                                    for k, v in r.items()}
            print(name, th, round(time.time() - t0, 1), res[f"theta_{th:g}"], flush=True)
        out[name] = res
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1].split(",") if len(sys.argv) > 1 else ["config1", "config2"])
