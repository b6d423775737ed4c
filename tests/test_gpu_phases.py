"""The split-FP32 kernel's phase accounting (diagnostic build).

The default library has no phase counters and says so; the diagnostic copy
(`python -m starsmasher_b200.build --phases`, the pair kernel compiled with
-DSG_PHASES) counts SM cycles per phase and must compute bit-identical
forces, so the phases it reports belong to the kernel that ships.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from starsmasher_b200 import _lib, api, inputs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import json, sys
import numpy as np
from starsmasher_b200 import api, inputs
s = inputs.single_polytrope(6000, 1.5, seed=31)
ctx = api.Context(0)
ctx.profile_enable(True)
ctx.phase_read()
res = ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
ph = ctx.phase_read()
np.save(sys.argv[1], np.stack(res))
print(json.dumps(ph))
"""


def test_default_build_has_no_phase_counters(gpu_ctx):
    with pytest.raises(_lib.SphgravError) as e:
        gpu_ctx.phase_read()
    assert e.value.status == _lib.ERR_UNSUPPORTED


def test_phase_build_counts_and_matches_default(gpu_ctx, tmp_path):
    from starsmasher_b200 import build
    build.build_phases()
    out = tmp_path / "phases_res.npy"
    env = dict(os.environ, SPHGRAV_B200_BUILD="phases")
    p = subprocess.run([sys.executable, "-c", _CHILD, str(out)], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    ph = json.loads(p.stdout.strip().splitlines()[-1])
    # every consumer warp started items and waited or worked on tiles
    assert ph["n_items"] > 0 and ph["n_far"] + ph["n_checked"] > 0, ph
    assert ph["far"] + ph["checked"] > 0 and ph["producer_work"] > 0, ph
    s = inputs.single_polytrope(6000, 1.5, seed=31)
    ref = np.stack(gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split"))
    got = np.load(out)
    assert np.array_equal(got, ref), np.max(np.abs(got - ref))
