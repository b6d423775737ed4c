"""The persistent kernels' work plan (host-side arithmetic, no GPU needed):
every (set, row tile) has its source range split into chunks that cover it
exactly once, in order; every chunk owns one partial-sum slot, contiguous per
tile; the queue is longest first; and the split-FP32 kernel cuts only the
last half-wave of tiles into chunks when there are many tiles (so its
partial sums stay about the size of the outputs), while the FP64 kernel
keeps uniform chunks."""
import numpy as np
import pytest

from starsmasher_b200 import api

PAD_J = 256  # sets are padded to multiples of the 256-source j-tile


def _check_plan(offsets, precision, variant, resident):
    info = api.variant_names(precision)  # the library loads (no GPU touched)
    assert variant < len(info)
    p = api.plan_preview(offsets, precision, variant, resident)
    it = p["items"]
    assert p["nitems"] == len(it)
    sizes = np.diff(offsets)
    # slots: one per item, all distinct, 0 .. nslots-1
    assert sorted(it[:, 3].tolist()) == list(range(p["nslots"]))
    cost = []
    by_tile = {}
    for s_, t, c, slot, jb, je in it:
        by_tile.setdefault((s_, t), []).append((c, slot, jb, je))
        n = sizes[s_]
        assert 0 <= jb < je <= (n + 255) // 256 * 256 or (n == 0)
        cost.append(je - jb)
    for (s_, t), chunks in by_tile.items():
        chunks.sort()
        n = sizes[s_]
        npad = (n + PAD_J - 1) // PAD_J * PAD_J
        assert [c for c, *_ in chunks] == list(range(len(chunks)))
        # covers every source [0, n), whole j-tiles, within the padded set
        assert chunks[0][2] == 0 and n <= chunks[-1][3] <= npad and chunks[-1][3] % 64 == 0
        for a, b in zip(chunks, chunks[1:]):
            assert a[3] == b[2]                                      # no gap, no overlap
            assert b[1] == a[1] + 1                                  # slots contiguous
    # every non-empty set's row tiles are 0, 1, ..., all planned
    for s_ in range(len(sizes)):
        tiles = sorted(t for (ss, t) in by_tile if ss == s_)
        assert (len(tiles) > 0) == (sizes[s_] > 0)
        assert tiles == list(range(len(tiles)))
    return p, by_tile


@pytest.mark.parametrize("precision,variant", [("f32split", 0), ("f32split", 2), ("f32split", 5),
                                               ("fp64", 0), ("fp64", 9)])
def test_single_set_plans_cover_every_pair(precision, variant):
    for n in (1, 255, 257, 16384, 262144, 1048576):
        _check_plan([0, n], precision, variant, resident=148 * (1 if precision == "f32split" else 4))


def test_batch_plans_cover_every_pair():
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(100), np.log(131072), 64)).astype(int)
    sizes[[3, 17]] = 0  # empty sets
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for precision, variant in (("f32split", 2), ("fp64", 9)):
        p, by_tile = _check_plan(offs, precision, variant, resident=148)
        assert p["nitems"] >= len(by_tile) > 0


def test_split_kernel_chunks_only_the_tail():
    """Config 3's shape: 1M particles in 768-row tiles, 148 persistent CTAs:
    whole-j-range items except the last 74 tiles (half a wave), cut in 4."""
    p, by_tile = _check_plan([0, 1048576], "f32split", 0, resident=148)
    nch = sorted(len(v) for v in by_tile.values())
    ntiles = (1048576 + 767) // 768
    assert len(by_tile) == ntiles
    assert nch.count(4) == 74 and nch.count(1) == ntiles - 74
    assert p["nslots"] == ntiles + 3 * 74


def test_fp64_kernel_keeps_uniform_chunks():
    p, by_tile = _check_plan([0, 1048576], "fp64", 9, resident=148 * 12)
    assert len({len(v) for v in by_tile.values()}) == 1


def test_preview_rejects_bad_arguments():
    from starsmasher_b200 import _lib
    for offs, prec, var in (([1, 5], "f32split", 0), ([0, 5, 3], "f32split", 0),
                            ([0, 5], "f32split", 99)):
        with pytest.raises(_lib.SphgravError):
            api.plan_preview(offs, prec, var)


def test_fp64_small_set_fills_the_gpu():
    """The FP64 kernel's small sets take chunks down to 512 sources, so a
    16K set gives each of 592 persistent CTAs several items (with the
    split-FP32 minimum of 2,048 sources it had 1,024 items, under two per
    CTA, and a third of the SMs idle at the end)."""
    resident = 148 * 4
    p, by_tile = _check_plan([0, 16384], "fp64", 0, resident)
    assert p["nitems"] >= 4 * resident
    for chunks in by_tile.values():
        assert all(je - jb >= 512 for _, _, jb, je in chunks)
    # split-FP32 keeps its 2,048-source minimum
    p32, by32 = _check_plan([0, 16384], "f32split", 5, 148)
    assert all(je - jb >= 2048 for ch in by32.values() for _, _, jb, je in ch)
