"""CPU tests of the workload generators and the snapshot reader and writer."""
import os
import struct

import numpy as np
import pytest

from conftest import ROOT
from starsmasher_b200 import inputs
from starsmasher_b200.snapshot import HEADER_FULL, HEADER_OLD, Snapshot, read_snapshot, write_snapshot


@pytest.mark.parametrize("n_index,xi1", [(1.0, np.pi), (1.5, 3.65375), (3.0, 6.89685)])
def test_lane_emden_first_zero(n_index, xi1):
    _, _, _, got = inputs.lane_emden(n_index)
    assert got == pytest.approx(xi1, rel=1e-4)


def test_polytrope_mass_profile():
    rng = np.random.default_rng(0)
    pos, m = inputs.polytrope_equal_mass(rng, 20000, 3.0, 1.0, 1.0)
    r = np.linalg.norm(pos, axis=1)
    assert r.max() <= 1.0 + 1e-12
    assert m.sum() == pytest.approx(1.0)
    # n=3: half the mass inside ~0.0.28 R (centrally condensed)
    assert 0.2 < np.median(r) < 0.35


def test_knn_smoothing_counts():
    rng = np.random.default_rng(1)
    pos = rng.random((3000, 3))
    r2 = inputs.knn_range2(pos, 64)
    i = 17
    d2 = np.sum((pos - pos[i]) ** 2, axis=1)
    assert np.sum(d2 < r2[i] * (1 - 1e-12)) == 64  # 64 others + itself strictly inside
    assert np.sum(d2 <= r2[i]) == 65


def test_red_giant_spans():
    s = inputs.red_giant(20000, seed=3)
    assert s.m[0] == 0.3 and s.range2[0] == pytest.approx(-0.01)
    gas_m = s.m[1:]
    assert gas_m.max() / gas_m.min() == pytest.approx(1e4, rel=1e-6)
    assert s.m.sum() == pytest.approx(1.0)
    h = np.sqrt(s.range2[1:])
    assert h.max() / h.min() > 100  # ~1e3 at N=1M; fewer particles -> smaller span


def test_batch_and_snapshots_shapes():
    b = inputs.batch_models(5, 256, 1024, seed=4)
    assert b.nsets == 5 and b.offsets[0] == 0 and np.all(np.diff(b.offsets) >= 256)
    for s in range(b.nsets):
        a, e = b.offsets[s], b.offsets[s + 1]
        assert b.m[a:e].sum() == pytest.approx(1.0)
    c = inputs.collision_snapshots(3, 1000, 2000, seed=5)
    assert c.nsets == 3
    com = [np.sum(c.m[a:e] * c.x[a:e]) / np.sum(c.m[a:e])
           for a, e in zip(c.offsets[:-1], c.offsets[1:])]
    assert np.max(np.abs(com)) < 0.05


REF_SNAP = "/root/reference/example_input/3_stars/sph.start1u"


def test_snapshot_reader_roundtrip_against_fixture():
    g = np.load(os.path.join(ROOT, "tests", "golden", "snap_3stars_start1.npz"))
    if os.path.exists(REF_SNAP):
        s = read_snapshot(REF_SNAP)
        assert s.ntot == 4944
        for k in ("x", "y", "z", "am", "hp", "u", "grpot"):
            np.testing.assert_array_equal(s.data[k], g[k])
    assert g["x"].shape == (4944,)


@pytest.mark.parametrize("nfields,ncooling", [(HEADER_FULL, 0), (HEADER_FULL, 1), (HEADER_OLD, 0)])
def test_snapshot_writer_roundtrip(tmp_path, nfields, ncooling):
    """write_snapshot restates dump (output.f:53-92): both header layouts,
    140-byte records and, with ncooling != 0, 156-byte ones."""
    from starsmasher_b200.snapshot import FIELDS
    rng = np.random.default_rng(11)
    n = 257
    data = {k: rng.normal(size=n) for k in FIELDS}
    data["cc"] = rng.integers(0, 5, n).astype(np.int32)
    data["divv"] = rng.normal(size=n)
    if ncooling:
        data["ueq"] = rng.normal(size=n)
        data["tthermal"] = rng.normal(size=n)
    header = {"nnopt": 23, "hco": 1.0, "t": 12.5, "nav": 3, "ncooling": ncooling, "displacez": 0.25}
    path = str(tmp_path / "out0001.sph")
    write_snapshot(path, Snapshot(n, data, header, nfields))
    back = read_snapshot(path)
    assert back.ntot == n and back.header_fields == nfields
    for k, v in data.items():
        np.testing.assert_array_equal(back.data[k], v)
    for k, v in header.items():
        if k in dict(back.header):
            assert back.header[k] == v
    assert back.header["ntot"] == n
    reclen = 156 if ncooling else 140
    hbytes = 164 if nfields == HEADER_FULL else 124
    assert os.path.getsize(path) == (hbytes + 8) + n * (reclen + 8) + 12


@pytest.mark.parametrize("case", ["3_stars/sph.start1u", "3_stars/sph.start2u",
                                  "collision/sph.start1u", "collision/sph.start2u"])
def test_snapshot_writer_reproduces_reference_dumps(tmp_path, case):
    """Reading a dump the reference wrote and writing it back gives the same bytes."""
    src = os.path.join("/root/reference/example_input", case)
    if not os.path.exists(src):
        pytest.skip("reference example inputs not mounted")
    out = str(tmp_path / "copy.sph")
    write_snapshot(out, read_snapshot(src))
    with open(src, "rb") as a, open(out, "rb") as b:
        assert a.read() == b.read()


def test_snapshots_as_a_batch(tmp_path):
    """Dump files become one particle set each, range2 = +-4 hp^2 (grav.f:15-18)."""
    from starsmasher_b200.snapshot import FIELDS
    rng = np.random.default_rng(3)
    paths = []
    for k, n in enumerate((40, 75)):
        data = {f: rng.uniform(0.1, 1.0, n) for f in FIELDS}
        data["u"][::7] = 0.0  # point masses
        p = str(tmp_path / f"m{k}.sph")
        write_snapshot(p, Snapshot(n, data))
        paths.append((p, data))
    b = inputs.from_snapshots([p for p, _ in paths])
    assert b.nsets == 2 and list(b.offsets) == [0, 40, 115]
    for s, (_, d) in enumerate(paths):
        a, e = b.offsets[s], b.offsets[s + 1]
        np.testing.assert_array_equal(b.x[a:e], d["x"])
        np.testing.assert_array_equal(b.m[a:e], d["am"])
        want = np.where(d["u"] == 0.0, -4.0 * d["hp"] ** 2, 4.0 * d["hp"] ** 2)
        np.testing.assert_array_equal(b.range2[a:e], want)


def test_snapshot_empty_roundtrip(tmp_path):
    """A dump with ntot = 0 (which the writer produces) reads back as an empty
    snapshot; a file with a bad header length is rejected before its body is
    parsed."""
    from starsmasher_b200.snapshot import FIELDS
    path = str(tmp_path / "empty.sph")
    write_snapshot(path, Snapshot(0, {}, {"t": 1.5}))
    back = read_snapshot(path)
    assert back.ntot == 0 and back.header["t"] == 1.5
    for k in FIELDS:
        assert back.data[k].shape == (0,)
    bad = str(tmp_path / "bad.sph")
    with open(bad, "wb") as f:
        f.write(struct.pack("<i", 12) + b"\0" * 12 + struct.pack("<i", 12))
        f.write(struct.pack("<iii", 4, 0, 4))
    with pytest.raises(ValueError, match="header length"):
        read_snapshot(bad)
