"""GPU tests of the batched persistent launch, the potential-energy
diagnostic, device-resident graph-captured sweeps and the autotuner."""
import os

import numpy as np
import pytest

import oracle
from conftest import err_report
from starsmasher_b200 import inputs

pytestmark = pytest.mark.gpu


def _t():
    import torch
    return torch


def dev(a):
    t = _t()
    return t.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.fixture(scope="module")
def small_batch():
    """Uneven sets: 9 models, N log-uniform in [64, 6000] (ragged, tiny and
    multi-tile sizes), n in [1, 3]."""
    return inputs.batch_models(9, 64, 6000, seed=41)


@pytest.fixture(scope="module")
def small_batch_oracle(small_batch):
    b = small_batch
    res = []
    for s in range(b.nsets):
        p = b.subset(s)
        res.append(oracle.triangle(p.x, p.y, p.z, p.m, p.range2, 0))
    return res


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("f32split", 1e-6)])
def test_batch_host_api(gpu_ctx, small_batch, small_batch_oracle, precision, tol):
    b = small_batch
    ax, ay, az, pot, W = gpu_ctx.batch_forces(b.offsets, b.x, b.y, b.z, b.m, b.range2, 0,
                                              precision)
    for s in range(b.nsets):
        a, e = b.offsets[s], b.offsets[s + 1]
        o = small_batch_oracle[s]
        r = err_report(ax[a:e], ay[a:e], az[a:e], pot[a:e], *o)
        assert r["acc_max"] <= tol and r["pot_max"] <= tol, (s, r)
        w_ref = 0.5 * np.sum(b.m[a:e] * o[3])
        assert W[s] == pytest.approx(w_ref, rel=max(tol, 1e-13))


@pytest.mark.parametrize("precision", ["fp64", "f32split"])
def test_batch_equals_separate_calls(gpu_ctx, small_batch, precision):
    """One persistent launch over all sets == one call per set (same math,
    same chunking of each set only if the plan agrees, so compare at 1e-12/1e-6)."""
    b = small_batch
    ax, ay, az, pot, _ = gpu_ctx.batch_forces(b.offsets, b.x, b.y, b.z, b.m, b.range2, 0,
                                              precision)
    tol = 1e-13 if precision == "fp64" else 2e-7
    for s in range(b.nsets):
        p = b.subset(s)
        a, e = b.offsets[s], b.offsets[s + 1]
        g = gpu_ctx.forces(p.x, p.y, p.z, p.m, p.range2, 0, precision)
        np.testing.assert_allclose(pot[a:e], g[3], rtol=tol)


@pytest.mark.parametrize("precision", ["fp64", "f32split"])
def test_empty_inputs_and_empty_sets(gpu_ctx, precision):
    """N = 0 returns empty results; empty sets inside a batch get no rows and
    W = 0, and leave the other sets' results as separate calls give them."""
    e = np.zeros(0)
    got = gpu_ctx.forces(e, e, e, e, e, 0, precision)
    assert all(a.shape == (0,) for a in got)
    b = inputs.batch_models(2, 300, 700, seed=53)
    n0 = int(b.offsets[1])
    offs = [0, 0, n0, n0, b.n, b.n]  # sets 0, 2 and 4 are empty
    res = gpu_ctx.batch_forces(offs, b.x, b.y, b.z, b.m, b.range2, 0, precision)
    W = res[4]
    assert W[0] == 0.0 and W[2] == 0.0 and W[4] == 0.0
    for s, (a, c) in enumerate([(0, n0), (n0, b.n)]):
        one = gpu_ctx.forces(b.x[a:c], b.y[a:c], b.z[a:c], b.m[a:c], b.range2[a:c], 0, precision)
        for u, v in zip(res[:4], one):
            assert np.array_equal(u[a:c], v)
        assert W[2 * s + 1] == pytest.approx(0.5 * np.sum(b.m[a:c] * one[3]), rel=1e-12)


def test_batch_device_api_and_W(gpu_ctx, small_batch, small_batch_oracle):
    t = _t()
    b = small_batch
    X = [dev(a) for a in (b.x, b.y, b.z, b.m, b.range2)]
    outs = [t.zeros(b.n, dtype=t.float64, device="cuda") for _ in range(4)]
    W = t.zeros(b.nsets, dtype=t.float64, device="cuda")
    gpu_ctx.batch_forces_device(b.offsets, *X, *outs, W=W, precision="f32split")
    gpu_ctx.sync()
    pot = outs[3].cpu().numpy()
    Wh = W.cpu().numpy()
    for s in range(b.nsets):
        a, e = b.offsets[s], b.offsets[s + 1]
        o = small_batch_oracle[s]
        np.testing.assert_allclose(pot[a:e], o[3], rtol=1e-6)
        assert Wh[s] == pytest.approx(0.5 * np.sum(b.m[a:e] * o[3]), rel=1e-6)


def test_graph_captured_sweep_matches_eager(gpu_ctx):
    """kick + batched gravity captured once and replayed == the same calls
    issued eagerly; state stays on the device between calls."""
    t = _t()
    b = inputs.collision_snapshots(3, 2000, 6000, seed=51)
    n = b.n
    sigma, seed = 1e-3, 1234

    def fresh():
        return [dev(a) for a in (b.x, b.y, b.z, b.m, b.range2)]

    # eager reference
    X = fresh()
    outs_e = [t.zeros(n, dtype=t.float64, device="cuda") for _ in range(4)]
    W_e = t.zeros(b.nsets, dtype=t.float64, device="cuda")
    gpu_ctx.kick_reset(0)
    for _ in range(3):
        gpu_ctx.kick_device(n, X[0], X[1], X[2], sigma, seed)
        gpu_ctx.batch_forces_device(b.offsets, *X, *outs_e, W=W_e, precision="f32split")
    gpu_ctx.sync()
    pos_e = [a.cpu().numpy() for a in X[:3]]
    res_e = [a.cpu().numpy() for a in outs_e] + [W_e.cpu().numpy()]

    # captured
    X = fresh()
    outs = [t.zeros(n, dtype=t.float64, device="cuda") for _ in range(4)]
    W = t.zeros(b.nsets, dtype=t.float64, device="cuda")
    gpu_ctx.kick_reset(0)
    gpu_ctx.batch_forces_device(b.offsets, *X, *outs, W=W, precision="f32split")  # sizes buffers
    gpu_ctx.sync()
    with gpu_ctx.capture() as cap:
        gpu_ctx.kick_device(n, X[0], X[1], X[2], sigma, seed)
        gpu_ctx.batch_forces_device(b.offsets, *X, *outs, W=W, precision="f32split")
    cap.graph.launch(3)
    gpu_ctx.sync()
    for a, r in zip([a.cpu().numpy() for a in X[:3]], pos_e):
        assert np.array_equal(a, r)
    for a, r in zip([a.cpu().numpy() for a in outs] + [W.cpu().numpy()], res_e):
        assert np.array_equal(a, r)
    # kicks moved the particles by ~sigma (3 kicks)
    d = np.sqrt((pos_e[0] - b.x) ** 2 + (pos_e[1] - b.y) ** 2 + (pos_e[2] - b.z) ** 2)
    assert 0.5 * sigma < np.median(d) < 5 * sigma
    # physics of the kicked positions vs the oracle
    for s in range(b.nsets):
        a, e = b.offsets[s], b.offsets[s + 1]
        o = oracle.rows(pos_e[0][a:e], pos_e[1][a:e], pos_e[2][a:e], b.m[a:e], b.range2[a:e], 0)
        r = err_report(res_e[0][a:e], res_e[1][a:e], res_e[2][a:e], res_e[3][a:e], *o)
        assert r["acc_max"] <= 1e-6 and r["pot_max"] <= 1e-6, r
    cap.graph.close()


def test_capture_refuses_new_sizes(gpu_ctx):
    t = _t()
    from starsmasher_b200 import _lib
    X = [dev(np.arange(10.0) * 0.1) for _ in range(3)] + [dev(np.ones(10)), dev(np.ones(10))]
    outs = [t.zeros(10, dtype=t.float64, device="cuda") for _ in range(4)]
    gpu_ctx.sync()
    with pytest.raises(_lib.SphgravError) as e:
        with gpu_ctx.capture():
            gpu_ctx.batch_forces_device([0, 3, 10], *X, *outs, precision="fp64")
    assert e.value.status == _lib.ERR_PROTOCOL
    gpu_ctx.sync()


def test_graph_refuses_replay_after_plan_change():
    """A graph bakes in its context's work plan and buffer addresses.  Calls
    with the captured sizes may interleave with replays; once a call with
    another precision rebuilds the plan, or the context is destroyed, the
    graph reports itself invalid and sphgrav_graph_launch refuses.  Validity
    is asserted before every launch, so no stale graph is ever replayed."""
    from starsmasher_b200 import Context, _lib
    t = _t()
    b = inputs.batch_models(3, 500, 1500, seed=71)
    X = [dev(a) for a in (b.x, b.y, b.z, b.m, b.range2)]
    outs = [t.zeros(b.n, dtype=t.float64, device="cuda") for _ in range(4)]
    ctx = Context(0)  # its own context: the shared fixture's plan stays as it is
    try:
        ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
        with ctx.capture() as cap:
            ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
        g = cap.graph
        assert g.valid
        g.launch(1)
        ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")  # same plan
        assert g.valid
        g.launch(1)
        ctx.sync()
        ctx.batch_forces_device(b.offsets, *X, *outs, precision="fp64")  # plan rebuilt
        ctx.sync()
        assert not g.valid
        with pytest.raises(_lib.SphgravError) as e:
            g.launch(1)
        assert e.value.status == _lib.ERR_PROTOCOL
        g.close()
        with ctx.capture() as cap:
            ctx.batch_forces_device(b.offsets, *X, *outs, precision="fp64")
        g2 = cap.graph
        assert g2.valid
    finally:
        ctx.close()
    assert not g2.valid  # context destroyed
    with pytest.raises(_lib.SphgravError) as e:
        g2.launch(1)
    assert e.value.status == _lib.ERR_PROTOCOL
    g2.close()


def test_autotune_and_cache_file(gpu_ctx, tmp_path):
    b = inputs.batch_models(4, 2000, 4000, seed=61)
    X = [dev(a) for a in (b.x, b.y, b.z, b.m, b.range2)]
    gpu_ctx.autotune(b.offsets, *X, 0, "f32split")
    path = str(tmp_path / "tune.json")
    gpu_ctx.tuning_save(path)
    txt = open(path).read()
    assert "sphgrav_b200-tuning-1" in txt and "f32split" in txt
    gpu_ctx.tuning_load(path)
    got = gpu_ctx.batch_forces(b.offsets, b.x, b.y, b.z, b.m, b.range2, 0, "f32split")
    p = b.subset(0)
    o = oracle.rows(p.x, p.y, p.z, p.m, p.range2, 0)
    np.testing.assert_allclose(got[3][: p.n], o[3], rtol=1e-6)


def test_fp32_peak_probe_runs(gpu_ctx):
    tf = gpu_ctx.fp32_peak_probe(2000)
    assert 5.0 < tf < 200.0


def test_reference_gpu_library_is_less_accurate(gpu_ctx):
    """The reference's own SPHgrav_lib2 compiled for sm_100a (oracle/_ref, a
    comparator built from its sources) on a reference snapshot: the split-FP32
    path is at least as accurate against the FP64 oracle."""
    import ctypes
    from conftest import load_golden
    if not os.path.exists(oracle.REF_GPU_LIB):
        pytest.skip("reference GPU library not built")
    d = load_golden("3stars_start1")
    n = d["x"].shape[0]
    ref = ctypes.CDLL(oracle.REF_GPU_LIB, mode=ctypes.RTLD_LOCAL)
    P = ctypes.POINTER(ctypes.c_double)
    ia = [ctypes.c_int(v) for v in (n, 1, n, 1, 0)]
    arr = [np.ascontiguousarray(d[k]) for k in ("x", "y", "z", "am")] + [np.ascontiguousarray(d["range2"])]
    ref.firsthalf_grav_forces_(*(ctypes.byref(v) for v in ia[:3]), *(a.ctypes.data_as(P) for a in arr),
                               ctypes.byref(ia[3]), ctypes.byref(ia[4]))
    outs = [np.zeros(n) for _ in range(4)]
    rk = ctypes.c_int(0)
    ref.lasthalf_grav_forces_(ctypes.byref(ia[0]), *(a.ctypes.data_as(P) for a in outs), ctypes.byref(rk))
    o = oracle.rows(d["x"], d["y"], d["z"], d["am"], d["range2"], 0)
    r_ref = err_report(*outs, *o)
    ours = gpu_ctx.forces(d["x"], d["y"], d["z"], d["am"], d["range2"], 0, "f32split")
    r_our = err_report(*ours, *o)
    print("reference GPU lib", r_ref, "ours", r_our)
    assert r_our["acc_max"] <= r_ref["acc_max"]
    # potentials: both at the FP32 level (max ~5e-8 set by a rounding bias);
    # compare the typical error
    assert r_our["pot_rms"] <= r_ref["pot_rms"]
    assert r_our["pot_max"] <= 2 * r_ref["pot_max"]


def test_graph_destroyed_during_another_capture(gpu_ctx):
    """Releasing a graph while the same thread captures another one (what a
    garbage-collected handle does) waits until the capture ends instead of
    invalidating it."""
    from starsmasher_b200 import _lib
    t = _t()
    b = inputs.collision_snapshots(2, 2000, 3000, seed=53)
    X = [dev(a) for a in (b.x, b.y, b.z, b.m, b.range2)]
    outs = [t.zeros(b.n, dtype=t.float64, device="cuda") for _ in range(4)]
    gpu_ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
    gpu_ctx.sync()
    want = [o.cpu().numpy() for o in outs]
    with gpu_ctx.capture() as first:
        gpu_ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
    with gpu_ctx.capture() as second:
        _lib.load().sphgrav_graph_destroy(first.graph._h)
        first.graph._h = None
        gpu_ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
    for o in outs:
        o.zero_()
    second.graph.launch(1)
    gpu_ctx.sync()
    for o, w in zip(outs, want):
        assert np.array_equal(o.cpu().numpy(), w)


def test_graph_refuses_replay_after_a_setting_changes():
    """Settings a captured graph bakes in (the FP64 band, the refine
    threshold) cannot change under it: changing one invalidates the graph,
    and setting the same value again does not."""
    from starsmasher_b200 import Context, _lib
    t = _t()
    b = inputs.batch_models(2, 500, 1500, seed=77)
    X = [dev(a) for a in (b.x, b.y, b.z, b.m, b.range2)]
    outs = [t.zeros(b.n, dtype=t.float64, device="cuda") for _ in range(4)]
    ctx = Context(0)
    try:
        for change in (lambda c: c.set_fp64_band(1.5), lambda c: c.set_refine(2.0)):
            ctx.set_fp64_band(1.0)
            ctx.set_refine(1.0)
            ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
            ctx.sync()
            with ctx.capture() as cap:
                ctx.batch_forces_device(b.offsets, *X, *outs, precision="f32split")
            ctx.set_fp64_band(1.0)  # unchanged: the graph stays valid
            assert cap.graph.valid
            cap.graph.launch(1)
            change(ctx)
            assert not cap.graph.valid
            with pytest.raises(_lib.SphgravError) as e:
                cap.graph.launch(1)
            assert e.value.status == _lib.ERR_PROTOCOL
            cap.graph.close()
        ctx.sync()
    finally:
        ctx.set_fp64_band(1.0)
        ctx.set_refine(1.0)
        ctx.close()

