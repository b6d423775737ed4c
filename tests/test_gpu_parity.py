"""GPU parity tests: the CUDA kernels (through the C-ABI) against the oracle.

Tolerances (per-particle relative errors, particles with |a| < 1e-3 median|a|
reported separately because cancellation makes their relative error
ill-conditioned):
  FP64 kernel      vs CPU-path triangle:  acc <= 1e-12, pot <= 1e-12
  split-FP32       vs FP64 oracle:        acc <= 1e-6,  pot <= 1e-6
"""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import GOLDEN_CASES, err_report, load_golden
from starsmasher_b200 import _lib, api, inputs

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
F32_TOL = 1e-6


def _torch():
    import torch
    return torch


def dev(a):
    t = _torch()
    return t.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.fixture(scope="module")
def star16k():
    return inputs.cached("config1")


@pytest.fixture(scope="module")
def tri16k(star16k):
    s = star16k
    return {nk: oracle.triangle(s.x, s.y, s.z, s.m, s.range2, nk) for nk in (0, 1, 2)}


@pytest.mark.parametrize("nkernel", [0, 1, 2])
def test_fp64_matches_cpu_path_config1(gpu_ctx, star16k, tri16k, nkernel):
    s = star16k
    ax, ay, az, pot = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, nkernel, "fp64")
    r = err_report(ax, ay, az, pot, *tri16k[nkernel])
    print("fp64 vs triangle", nkernel, r)
    assert r["acc_max"] <= FP64_TOL and r["pot_max"] <= FP64_TOL, r
    assert r["acc_max_ill"] <= 1e-9, r


@pytest.mark.parametrize("nkernel", [0, 1, 2])
def test_f32split_within_1e6_config1(gpu_ctx, star16k, tri16k, nkernel):
    s = star16k
    ax, ay, az, pot = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, nkernel, "f32split")
    r = err_report(ax, ay, az, pot, *tri16k[nkernel])
    print("f32split vs triangle", nkernel, r)
    assert r["acc_max"] <= F32_TOL and r["pot_max"] <= F32_TOL, r


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("precision", ["fp64", "f32split"])
def test_golden_snapshot_potential(gpu_ctx, name, precision):
    """Reference dumps: stored grpot (FP32-level) reproduced like the oracle does."""
    d = load_golden(name)
    ax, ay, az, pot = gpu_ctx.forces(d["x"], d["y"], d["z"], d["am"], d["range2"], 0, precision)
    rel = np.abs(pot - d["grpot"]) / np.abs(d["grpot"])
    assert rel.max() < 4e-7
    o = oracle.rows(d["x"], d["y"], d["z"], d["am"], d["range2"], 0)
    r = err_report(ax, ay, az, pot, *o)
    tol = FP64_TOL if precision == "fp64" else F32_TOL
    assert r["acc_max"] <= tol and r["pot_max"] <= tol, r


def test_gravforce_host_mirror_matches(gpu_ctx):
    """sphgrav_gravforce restates grav.f:15-26 + balAV3.f:418 (hp, u inputs)."""
    d = load_golden("3stars_start1")
    u = d["u"].copy()
    u[::50] = 0.0  # some point masses: negative range2
    out = gpu_ctx.gravforce(d["x"], d["y"], d["z"], d["am"], d["hp"], u, nkernel=0,
                            precision="fp64")
    r2 = 4 * d["hp"] ** 2
    r2 = np.where(u == 0, -r2, r2)
    o = oracle.triangle(d["x"], d["y"], d["z"], d["am"], r2, 0)
    r = err_report(*out, *o)
    assert r["acc_max"] <= FP64_TOL and r["pot_max"] <= FP64_TOL


@pytest.mark.parametrize("precision", ["fp64", "f32split", "tree"])
def test_gravforce_device_matches_host_mirror(gpu_ctx, precision):
    """sphgrav_gravforce_device (positions, hp, u on the device; range2 built
    there) gives the host mirror's rows bit for bit and leaves the others."""
    t = _torch()
    d = load_golden("3stars_start1")
    n = d["x"].shape[0]
    hp = d["hp"]
    u = d["u"].copy()
    u[::50] = 0.0  # some point masses: negative range2
    lo, hi = 11, n - 7
    want = gpu_ctx.gravforce(d["x"], d["y"], d["z"], d["am"], hp, u, lo, hi, 0, precision)
    outs = [t.full((n,), -7.0, dtype=t.float64, device="cuda") for _ in range(4)]
    gpu_ctx.gravforce_device(n, *(dev(a) for a in (d["x"], d["y"], d["z"], d["am"], hp, u)), *outs,
                             ngrav_lower=lo, ngrav_upper=hi, precision=precision)
    gpu_ctx.sync()
    for a, b in zip(outs, want):
        a = a.cpu().numpy()
        assert np.array_equal(a[lo - 1:hi], b[lo - 1:hi])
        assert np.all(a[:lo - 1] == -7.0) and np.all(a[hi:] == -7.0)


@pytest.mark.parametrize("precision", ["fp64", "f32split"])
def test_legacy_abi_row_slice(precision, star16k):
    """Fortran conventions: 1-based n_lower, only the listed rows written."""
    s = star16k
    n = s.n
    api.gpu_init_dev(0, 0.3)
    api.set_legacy_precision(precision)
    lo, length = 3001, 5003  # 1-based first row
    api.firsthalf_grav_forces(n, lo, length, s.x, s.y, s.z, s.m, s.range2, q=4, nkernel=0)
    outs = [np.full(n, 7.0) for _ in range(4)]
    api.lasthalf_grav_forces(n, *outs)
    rows = np.arange(lo - 1, lo - 1 + length)
    o = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0, row_idx=rows)
    r = err_report(*(a[rows] for a in outs), *o)
    tol = FP64_TOL if precision == "fp64" else F32_TOL
    assert r["acc_max"] <= tol and r["pot_max"] <= tol, r
    mask = np.ones(n, bool)
    mask[rows] = False
    for a in outs:
        assert np.all(a[mask] == 7.0)


@pytest.mark.parametrize("precision", ["fp64", "f32split"])
@pytest.mark.parametrize("nkernel", [0, 1, 2])
def test_edge_cases(gpu_ctx, precision, nkernel):
    """Coincident particles, point masses, tiny sets, ragged sizes, huge H."""
    rng = np.random.default_rng(7 + nkernel)
    cases = []
    # a few particles, including coincident pairs with different H and mass
    x = np.array([0.0, 0.0, 0.3, 0.3, 1.0])
    y = np.array([0.0, 0.0, 0.1, 0.1, -0.2])
    z = np.zeros(5)
    m = np.array([1.0, 2.0, 0.5, 0.5, 0.1])
    r2 = np.array([0.25, 0.0625, 0.04, -0.04, 0.5])
    cases.append((x, y, z, m, r2))
    cases.append((np.zeros(1), np.zeros(1), np.zeros(1), np.ones(1), np.ones(1)))
    cases.append((np.array([0.0, 1.0]), np.zeros(2), np.zeros(2), np.array([1.0, 3.0]),
                  np.array([4.0, -0.01])))
    for n in (255, 257, 1029):
        p = rng.normal(size=(n, 3))
        mm = rng.uniform(0.1, 1.0, n) / n
        rr = rng.uniform(0.01, 2.0, n) ** 2
        rr[::13] *= -1
        p[5] = p[9]  # a coincident pair
        cases.append((p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), mm, rr))
    tol = FP64_TOL if precision == "fp64" else F32_TOL
    for (x, y, z, m, r2) in cases:
        got = gpu_ctx.forces(x, y, z, m, r2, nkernel, precision)
        o = oracle.triangle(x, y, z, m, r2, nkernel)
        amag = np.sqrt(o[0] ** 2 + o[1] ** 2 + o[2] ** 2)
        scale = np.maximum(amag, 1e-300)
        da = np.sqrt((got[0] - o[0]) ** 2 + (got[1] - o[1]) ** 2 + (got[2] - o[2]) ** 2)
        ok = (da <= tol * scale + 1e-13 * np.max(amag))
        assert ok.all(), (x.shape[0], np.max(da / scale))
        np.testing.assert_allclose(got[3], o[3], rtol=tol, atol=0)


@pytest.mark.parametrize("precision", ["fp64", "f32split"])
def test_invalid_input_reported(gpu_ctx, precision):
    x = np.zeros(4)
    m = np.ones(4)
    bad = np.ones(4)
    bad[2] = 0.0
    with pytest.raises(_lib.SphgravError) as e:
        gpu_ctx.forces(np.arange(4.0), x, x, m, bad, 0, precision)
    assert e.value.status == _lib.ERR_INVALID_INPUT
    m2 = m.copy()
    m2[1] = -1.0
    with pytest.raises(_lib.SphgravError) as e:
        gpu_ctx.forces(np.arange(4.0), x, x, m2, np.ones(4), 0, precision)
    assert e.value.status == _lib.ERR_INVALID_INPUT
    # device path: the check runs on the device and is reported at sync
    t = _torch()
    dx = dev(np.arange(4.0))
    dz = dev(x)
    dm = dev(m2)
    dr = dev(np.ones(4))
    outs = [t.zeros(4, dtype=t.float64, device="cuda") for _ in range(4)]
    gpu_ctx.forces_device(4, dx, dz, dz, dm, dr, *outs, precision=precision)
    with pytest.raises(_lib.SphgravError) as e:
        gpu_ctx.sync()
    assert e.value.status == _lib.ERR_INVALID_INPUT
    gpu_ctx.sync()  # the flag was cleared


def test_protocol_errors(gpu_ctx):
    with pytest.raises(_lib.SphgravError) as e:
        _lib.check(gpu_ctx._lib.sphgrav_lasthalf(gpu_ctx._h, None, None, None, None), "lasthalf")
    assert e.value.status == _lib.ERR_PROTOCOL
    with pytest.raises(ValueError):
        gpu_ctx.forces(np.zeros(2), np.zeros(2), np.zeros(2), np.ones(2), np.ones(2), 0, "fp16")
    with pytest.raises(_lib.SphgravError) as e:
        gpu_ctx.forces(np.zeros(2), np.zeros(2), np.zeros(2), np.ones(2), np.ones(2), 5)
    assert e.value.status == _lib.ERR_INVALID_ARGUMENT


def test_device_wait_timeout_is_reported_and_recoverable(gpu_ctx):
    """The pair kernels' bounded mbarrier wait, run on a barrier that nothing
    arrives on (sphgrav_selftest_wait_timeout): it gives up after its polls,
    the host reads SPHGRAV_ERR_DEVICE_TIMEOUT, the flag is cleared and the
    context keeps working.  No fault and no hang is involved."""
    import time
    t0 = time.perf_counter()
    st = gpu_ctx.selftest_wait_timeout(1024)
    assert st == _lib.ERR_DEVICE_TIMEOUT
    assert time.perf_counter() - t0 < 20.0
    s = inputs.single_polytrope(700, 1.5, seed=5)
    got = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "fp64")
    o = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0)
    r = err_report(*got, *o)
    assert r["acc_max"] <= FP64_TOL and r["pot_max"] <= FP64_TOL
    with pytest.raises(_lib.SphgravError) as e:
        _lib.check(gpu_ctx._lib.sphgrav_selftest_wait_timeout(gpu_ctx._h, 0), "selftest")
    assert e.value.status == _lib.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("precision", ["fp64", "f32split"])
def test_deterministic(gpu_ctx, star16k, precision):
    s = star16k
    a = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, precision)
    b = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, precision)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_every_f32_variant_meets_tolerance(gpu_ctx, star16k, tri16k):
    s = star16k
    names = api.variant_names("f32split")
    try:
        for v, name in enumerate(names):
            gpu_ctx.force_variant("f32split", v)
            got = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
            r = err_report(*got, *tri16k[0])
            print(name, r)
            assert r["acc_max"] <= F32_TOL and r["pot_max"] <= F32_TOL, (name, r)
    finally:
        gpu_ctx.force_variant("f32split", -1)


def test_every_fp64_variant_meets_tolerance(gpu_ctx, star16k, tri16k):
    s = star16k
    try:
        for v, name in enumerate(api.variant_names("fp64")):
            gpu_ctx.force_variant("fp64", v)
            got = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "fp64")
            r = err_report(*got, *tri16k[0])
            assert r["acc_max"] <= FP64_TOL and r["pot_max"] <= FP64_TOL, (name, r)
    finally:
        gpu_ctx.force_variant("fp64", -1)


@pytest.mark.parametrize("hp_cluster", [1.0, 0.03])
def test_dense_near_cluster(gpu_ctx, hp_cluster):
    """A compact cluster inside a sparse halo: with hp = 1 every cluster pair is
    a near (FP64) pair, so every near mask of the cluster's warps is full and the
    warp-cooperative evaluation runs its largest compactions (32 lanes x 16
    sources per mask); with hp = 0.03 the masks are partly set."""
    rng = np.random.default_rng(11)
    nc, nh = 2048, 1000
    rc = 0.1 * rng.random(nc) ** (1 / 3)
    rh = 1.0 + 9.0 * rng.random(nh)
    dirs = rng.normal(size=(nc + nh, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pos = dirs * np.concatenate([rc, rh])[:, None]
    m = np.concatenate([rng.uniform(0.5, 1.5, nc), rng.uniform(0.1, 0.2, nh)]) / (nc + nh)
    hp = np.concatenate([np.full(nc, hp_cluster), np.full(nh, 0.2)])
    range2 = 4.0 * hp * hp
    x, y, z = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    o = oracle.rows(x, y, z, m, range2, 0)
    for precision, tol in (("fp64", FP64_TOL), ("f32split", F32_TOL)):
        got = gpu_ctx.forces(x, y, z, m, range2, 0, precision)
        r = err_report(*got, *o)
        print(precision, hp_cluster, r)
        assert r["acc_max"] <= tol and r["pot_max"] <= tol, (precision, r)


def test_red_giant_core_subset(gpu_ctx):
    """Config-3 physics (core point mass, h and m spanning decades) at
    N=65,536 on a row subset: split-FP32 within 1e-6 of the FP64 oracle."""
    s = inputs.red_giant(65536, seed=31)
    ax, ay, az, pot = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
    rows = np.concatenate([[0], np.random.default_rng(0).choice(s.n, 3000, replace=False)])
    o = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0, row_idx=rows)
    r = err_report(ax[rows], ay[rows], az[rows], pot[rows], *o)
    print("red giant 64k", r)
    assert r["acc_max"] <= F32_TOL and r["pot_max"] <= F32_TOL, r
    g = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "fp64")
    r64 = err_report(*(a[rows] for a in g), *o)
    assert r64["acc_max"] <= FP64_TOL and r64["pot_max"] <= FP64_TOL, r64


@pytest.mark.parametrize("band", [1.0, 1.5, 2.0, 3.0])
def test_fp64_band_setting(gpu_ctx, star16k, tri16k, band):
    """sphgrav_set_fp64_band moves pairs between two correct evaluations: every
    setting stays within 1e-6 (band 1, the default, keeps only the softened
    near field in FP64; the refine recomputes the rows whose FP32 sums are
    ill-conditioned)."""
    s = star16k
    try:
        gpu_ctx.set_fp64_band(band)
        got = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
    finally:
        gpu_ctx.set_fp64_band(1.0)
    r = err_report(*got, *tri16k[0])
    print("band", band, r)
    assert r["acc_rms"] <= 1e-7 and r["pot_max"] <= F32_TOL
    assert r["acc_max"] <= F32_TOL, r


@pytest.mark.parametrize("case", ["tiles", "row_chunks"])
def test_refine_recomputes_listed_rows_in_fp64(gpu_ctx, case):
    """The FP64 refine: with the refine off the split-FP32 sums stand for
    every row; with it on, exactly the rows whose error scale G exceeds
    |a| (or that lie far from their tile centre, G = inf) change, and
    those rows then agree with the CPU path to the FP64 tolerance; the
    others are bit-identical.  Both routes: a set with many listed rows
    (tiles of 128 rows) and sets with at most 32 (one warp per row and
    source chunk)."""
    if case == "tiles":
        s = inputs.collision_snapshots(1, 24000, 24000, seed=8)
    else:
        s = inputs.cached("config1")
    try:
        gpu_ctx.keep_error_scale(True)
        gpu_ctx.set_refine(0.0)
        off = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
        assert gpu_ctx.last_refine_rows() == 0
        G = gpu_ctx.error_scale(s.n)
        gpu_ctx.set_refine(1.0)
        on = gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
        nref = gpu_ctx.last_refine_rows()
    finally:
        gpu_ctx.keep_error_scale(False)
        gpu_ctx.set_refine(1.0)
    amag = np.sqrt(off[0] ** 2 + off[1] ** 2 + off[2] ** 2)
    listed = G > amag
    assert nref == int(listed.sum()) and nref > 0
    assert (nref > 32) == (case == "tiles"), nref
    same = np.all([np.equal(a, b) for a, b in zip(on, off)], axis=0)
    assert np.all(same[~listed])
    rows = np.nonzero(listed)[0].astype(np.int32)
    o = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0, row_idx=rows)
    r = err_report(*(a[rows] for a in on), *o)
    print("refined rows", nref, r)
    assert r["acc_max"] <= FP64_TOL and r["pot_max"] <= FP64_TOL, r


def test_error_scale_needs_keep(gpu_ctx, star16k):
    s = star16k
    gpu_ctx.keep_error_scale(False)
    gpu_ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "f32split")
    with pytest.raises(_lib.SphgravError) as e:
        gpu_ctx.error_scale(s.n)
    assert e.value.status == _lib.ERR_PROTOCOL
    for bad in (-0.5, float("nan"), 1e7):
        with pytest.raises(_lib.SphgravError):
            gpu_ctx.set_refine(bad)


def test_fp64_band_rejects_bad_values(gpu_ctx):
    for bad in (0.5, 0.0, -1.0, 100.0, float("nan")):
        with pytest.raises(_lib.SphgravError) as e:
            gpu_ctx.set_fp64_band(bad)
        assert e.value.status == _lib.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("shift", [(1.0e4, -2.0e4, 5.0e3), (3.0e6, 0.0, -1.0e6)])
def test_model_far_from_the_origin(gpu_ctx, shift):
    """A star model displaced far from the coordinate origin (a collision's
    stars sit at large separations): both kernels still agree with the CPU
    path on the same (displaced) inputs.  The split kernel forms separations
    from hi + lo position pairs relative to each tile's centre, so the
    displacement costs it nothing; the FP64 kernel rounds x_j - x_i as the
    CPU path does."""
    s = inputs.single_polytrope(6000, 1.5, seed=91)
    x, y, z = s.x + shift[0], s.y + shift[1], s.z + shift[2]
    tri = oracle.triangle(x, y, z, s.m, s.range2, 0)
    for precision, tol in (("fp64", FP64_TOL), ("f32split", F32_TOL)):
        got = gpu_ctx.forces(x, y, z, s.m, s.range2, 0, precision)
        r = err_report(*got, *tri)
        print("displaced by", shift, precision, r)
        assert r["acc_max"] <= tol and r["pot_max"] <= tol, (precision, r)
