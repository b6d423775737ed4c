"""Reader and writer for StarSmasher binary particle dumps (sph.start*u,
out*.sph).

Format written by ``dump`` (parallel_bleeding_edge/src/output.f:53-92):
Fortran unformatted sequential records, each framed by a 4-byte length
before and after.  Record 1 is the header: ntot, nnopt, hco, hfloor, sep0,
tf, dtout, nout, nit, t, nav, alpha, beta, tjumpahead, ngr, nrelax, trelax,
dt, omega2, ncooling, erad, ndisplace, displacex, displacey, displacez
(output.f:69-71; integers int32, reals float64: 164 bytes; older dumps stop
after omega2, 124 bytes, and readin reads only up to dt, init.f:787-790).
Then one record per particle with 16 float64 (x, y, z, am, hp, rho, vx, vy,
vz, vxdot, vydot, vzdot, u, udot, grpot, meanmolecular), an int32 cc and a
float64 divv (140 bytes; with ncooling != 0 two more float64 ueq, tthermal);
a last record repeats ntot.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

FIELDS = ("x", "y", "z", "am", "hp", "rho", "vx", "vy", "vz", "vxdot", "vydot", "vzdot", "u",
          "udot", "grpot", "meanmolecular")
# header record, in order (output.f:69-71): (name, struct code)
HEADER = (("ntot", "i"), ("nnopt", "i"), ("hco", "d"), ("hfloor", "d"), ("sep0", "d"), ("tf", "d"),
          ("dtout", "d"), ("nout", "i"), ("nit", "i"), ("t", "d"), ("nav", "i"), ("alpha", "d"),
          ("beta", "d"), ("tjumpahead", "d"), ("ngr", "i"), ("nrelax", "i"), ("trelax", "d"),
          ("dt", "d"), ("omega2", "d"), ("ncooling", "i"), ("erad", "d"), ("ndisplace", "i"),
          ("displacex", "d"), ("displacey", "d"), ("displacez", "d"))
HEADER_FULL = 25    # fields of the current dump (164 bytes)
HEADER_OLD = 19     # older dumps end after omega2 (124 bytes)


def _header_format(nfields: int) -> str:
    return "<" + "".join(code for _, code in HEADER[:nfields])


@dataclass
class Snapshot:
    ntot: int
    data: dict  # field name -> array (float64; cc int32)
    header: dict = field(default_factory=dict)  # header record values (ntot included)
    header_fields: int = HEADER_FULL            # how many header fields the file carries

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
    if len(recs) < 2:
        raise ValueError(f"{path}: {len(recs)} records; a dump has a header and a trailer")
    header, nhf = {}, 0
    for nf in (HEADER_FULL, HEADER_OLD):
        if struct.calcsize(_header_format(nf)) == recs[0][1]:
            vals = struct.unpack_from(_header_format(nf), buf, recs[0][0])
            header = {name: v for (name, _), v in zip(HEADER[:nf], vals)}
            nhf = nf
            break
    if not nhf:
        raise ValueError(f"{path}: unexpected header length {recs[0][1]}")
    ntot = int(header["ntot"])
    body = recs[1:-1]
    if len(body) != ntot:
        raise ValueError(f"{path}: header says {ntot} particles, found {len(body)} records")
    if recs[-1][1] != 4:
        raise ValueError(f"{path}: trailing record of {recs[-1][1]} bytes, expected 4")
    tail = struct.unpack_from("<i", buf, recs[-1][0])[0]
    if tail != ntot:
        raise ValueError(f"{path}: trailing ntot {tail} != {ntot}")
    if ntot == 0:
        data = {name: np.zeros(0) for name in FIELDS}
        data["cc"] = np.zeros(0, dtype=np.int32)
        data["divv"] = np.zeros(0)
        return Snapshot(0, data, header, nhf)
    reclen = body[0][1]
    if reclen not in (140, 156) or any(r[1] != reclen for r in body):
        raise ValueError(f"{path}: unexpected particle record length {reclen}")
    start = body[0][0]
    stride = reclen + 8
    raw = np.frombuffer(buf, dtype=np.uint8, count=stride * ntot, offset=start)
    raw = raw.reshape(ntot, stride)[:, :reclen]
    vals = np.ascontiguousarray(raw[:, :128]).view("<f8").reshape(ntot, 16)
    data = {name: vals[:, k].copy() for k, name in enumerate(FIELDS)}
    data["cc"] = np.ascontiguousarray(raw[:, 128:132]).view("<i4").reshape(ntot).copy()
    data["divv"] = np.ascontiguousarray(raw[:, 132:140]).view("<f8").reshape(ntot).copy()
    if reclen == 156:
        extra = np.ascontiguousarray(raw[:, 140:156]).view("<f8").reshape(ntot, 2)
        data["ueq"] = extra[:, 0].copy()
        data["tthermal"] = extra[:, 1].copy()
    return Snapshot(ntot, data, header, nhf)


def write_snapshot(path: str, snap: Snapshot) -> None:
    """Write ``snap`` in dump's format (output.f:53-92).  Header values missing
    from ``snap.header`` are written as zero (ntot from the data); particle
    fields missing from ``snap.data`` as zero; the ncooling-dependent fields
    ueq and tthermal are written when the header's ncooling is non-zero."""
    n = int(snap.ntot)
    hdr = dict(snap.header)
    hdr["ntot"] = n
    nhf = snap.header_fields
    hvals = [hdr.get(name, 0) for name, _ in HEADER[:nhf]]
    cooling = int(hdr.get("ncooling", 0)) != 0
    reclen = 156 if cooling else 140
    rec = np.zeros((n, reclen + 8), dtype=np.uint8)
    rec[:, 0:4] = np.frombuffer(struct.pack("<i", reclen), np.uint8)
    rec[:, reclen + 4:] = np.frombuffer(struct.pack("<i", reclen), np.uint8)
    f8 = np.zeros((n, 16), dtype="<f8")
    for k, name in enumerate(FIELDS):
        if name in snap.data:
            f8[:, k] = snap.data[name]
    rec[:, 4:132] = f8.view(np.uint8)
    cc = np.asarray(snap.data.get("cc", np.zeros(n)), dtype="<i4").reshape(n, 1)
    rec[:, 132:136] = cc.view(np.uint8)
    dv = np.asarray(snap.data.get("divv", np.zeros(n)), dtype="<f8").reshape(n, 1)
    rec[:, 136:144] = dv.view(np.uint8)
    if cooling:
        ex = np.zeros((n, 2), dtype="<f8")
        ex[:, 0] = snap.data.get("ueq", 0.0)
        ex[:, 1] = snap.data.get("tthermal", 0.0)
        rec[:, 144:160] = ex.view(np.uint8)
    head = struct.pack(_header_format(nhf), *hvals)
    with open(path, "wb") as f:
        f.write(struct.pack("<i", len(head)) + head + struct.pack("<i", len(head)))
        f.write(rec.tobytes())
        f.write(struct.pack("<iii", 4, n, 4))
