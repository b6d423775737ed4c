"""Reader for StarSmasher binary particle dumps (sph.start*u, out*.sph).

Format written by ``dump`` (parallel_bleeding_edge/src/output.f:53-92):
Fortran unformatted sequential records, each framed by a 4-byte length
before and after.  Record 1 is the header (ntot first); then one record per
particle with 16 float64 (x, y, z, am, hp, rho, vx, vy, vz, vxdot, vydot,
vzdot, u, udot, grpot, meanmolecular), an int32 cc and a float64 divv
(140 bytes; with ncooling != 0 two more float64 ueq, tthermal); a last
record repeats ntot.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

FIELDS = ("x", "y", "z", "am", "hp", "rho", "vx", "vy", "vz", "vxdot", "vydot", "vzdot", "u",
          "udot", "grpot", "meanmolecular")


@dataclass
class Snapshot:
    ntot: int
    data: dict  # field name -> float64 array

    def range2(self) -> np.ndarray:
        """The softening argument the gravity call receives (grav.f:15-18)."""
        r2 = 4.0 * self.data["hp"] ** 2
        return np.where(self.data["u"] == 0.0, -r2, r2)


def read_snapshot(path: str) -> Snapshot:
    with open(path, "rb") as f:
        buf = f.read()
    recs = []
    off = 0
    while off < len(buf):
        (n,) = struct.unpack_from("<i", buf, off)
        off += 4
        recs.append((off, n))
        off += n
        (n2,) = struct.unpack_from("<i", buf, off)
        off += 4
        if n2 != n:
            raise ValueError(f"{path}: corrupt record framing at byte {off}")
    ntot = struct.unpack_from("<i", buf, recs[0][0])[0]
    body = recs[1:-1]
    if len(body) != ntot:
        raise ValueError(f"{path}: header says {ntot} particles, found {len(body)} records")
    tail = struct.unpack_from("<i", buf, recs[-1][0])[0]
    if tail != ntot:
        raise ValueError(f"{path}: trailing ntot {tail} != {ntot}")
    reclen = body[0][1]
    if reclen not in (140, 156):
        raise ValueError(f"{path}: unexpected particle record length {reclen}")
    start = body[0][0]
    stride = reclen + 8
    raw = np.frombuffer(buf, dtype=np.uint8, count=stride * ntot, offset=start)
    raw = raw.reshape(ntot, stride)[:, :reclen]
    vals = np.ascontiguousarray(raw[:, :128]).view("<f8").reshape(ntot, 16)
    data = {name: vals[:, k].copy() for k, name in enumerate(FIELDS)}
    data["cc"] = np.ascontiguousarray(raw[:, 128:132]).view("<i4").reshape(ntot).copy()
    data["divv"] = np.ascontiguousarray(raw[:, 132:140]).view("<f8").reshape(ntot).copy()
    return Snapshot(ntot, data)
