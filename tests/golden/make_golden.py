"""Regenerate the golden fixtures from the reference's own snapshot files.

The reference ships binary particle dumps whose per-particle grpot was
written by its own gravity code (example_input/*/sph.start{1,2}u; format of
parallel_bleeding_edge/src/output.f:53-92).  This script copies x, y, z, am,
hp, u and grpot of each into tests/golden/snap_<case>.npz.  collision/ and
collision_elliptical/ hold byte-identical files, so only the first is kept.

Run where the reference tree is mounted:
    python tests/golden/make_golden.py [/path/to/reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from starsmasher_b200.snapshot import read_snapshot  # noqa: E402

CASES = {
    "collision_start1": "example_input/collision/sph.start1u",
    "collision_start2": "example_input/collision/sph.start2u",
    "3stars_start1": "example_input/3_stars/sph.start1u",
    "3stars_start2": "example_input/3_stars/sph.start2u",
}


def main(ref_root: str) -> None:
    for name, rel in CASES.items():
        snap = read_snapshot(os.path.join(ref_root, rel))
        d = snap.data
        out = os.path.join(HERE, f"snap_{name}.npz")
        np.savez_compressed(out, x=d["x"], y=d["y"], z=d["z"], am=d["am"], hp=d["hp"], u=d["u"],
                            grpot=d["grpot"], source=np.array(rel))
        print(f"{out}: ntot={snap.ntot}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
