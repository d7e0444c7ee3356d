"""Batched rendering on the GPU: many cameras of mixed resolution and
tolerance in one persistent launch, the compaction interval, the autotuner,
graph capture and replay, and the per-frame clock.

Every ray's arithmetic is independent of the lane, warp and launch that runs
it, so these launch-shape switches must leave the outputs bit-identical.
"""
import numpy as np
import pytest

from rtwca_b200 import abi, configs

pytestmark = pytest.mark.gpu

WANT = ("xyz", "class", "steps", "spectrum")


def _same(a, b):
    for k in WANT:
        assert np.array_equal(a[k], b[k]), k


def _small_batch(n=6):
    scene, cams, colors, meta = configs.batched_frames(n, seed=0, sizes=(16, 24, 32), tols=(1e-6, 1e-8))
    return scene, cams, configs.log_spaced_colors(16), meta


@pytest.mark.parametrize("precision", [abi.PREC_MIXED, abi.PREC_FP64])
def test_refill_interval_invariance(renderer, precision):
    scene, cam, _ = configs.workload("kerr_thin_disk", x_pix=48)
    colors = configs.log_spaced_colors(16)
    base = renderer.render(scene, [cam], colors, want=WANT, precision=precision)
    for refill in (4, 8, 32):
        g = renderer.render(scene, [cam], colors, want=WANT, precision=precision, refill_min=refill)
        assert renderer.stats()["refill_min"] == refill
        _same(base, g)


def test_batched_mixed_sizes_equal_single(renderer):
    scene, cams, colors, meta = _small_batch()
    batch = renderer.render(scene, cams, colors, want=WANT, precision=abi.PREC_MIXED, refill_min=4)
    off = 0
    for c in cams:
        one = renderer.render(scene, [c], colors, want=WANT, precision=abi.PREC_MIXED)
        n = c.x_pix * c.y_pix
        for k in WANT:
            assert np.array_equal(batch[k][off:off + n], one[k]), k
        off += n
    assert off == batch["class"].size


def test_frame_times(renderer):
    scene, cams, colors, meta = _small_batch()
    renderer.render(scene, cams, colors, want=("class",), precision=abi.PREC_MIXED)
    st = renderer.stats()
    ft = renderer.frame_times(len(cams))
    done, span = ft["done"], ft["span"]
    assert np.all(np.isfinite(done)) and np.all(np.isfinite(span))
    assert np.all(span >= 0) and np.all(done >= span - 1e-9)
    # every frame ends inside the kernel (global timer vs CUDA events: allow slack)
    assert done.max() <= st["kernel_ms"] * 1.05 + 0.5
    with pytest.raises(abi.RTWError):
        renderer.frame_times(len(cams) + 1)


def test_graph_replay_matches_direct_launch(renderer):
    scene, cams, colors, meta = _small_batch(3)
    a, b = cams[0], cams[1]
    b.x_pix = a.x_pix  # same shape: the captured launch is replayed for camera b
    ref_a = renderer.render(scene, [a], colors, want=WANT, precision=abi.PREC_MIXED)
    ref_b = renderer.render(scene, [b], colors, want=WANT, precision=abi.PREC_MIXED)
    g_a = renderer.render(scene, [a], colors, want=WANT, precision=abi.PREC_MIXED, graph=True)
    assert renderer.stats()["graph_replayed"] == 0
    g_b = renderer.render(scene, [b], colors, want=WANT, precision=abi.PREC_MIXED, graph=True)
    assert renderer.stats()["graph_replayed"] == 1
    g_a2 = renderer.render(scene, [a], colors, want=WANT, precision=abi.PREC_MIXED, graph=True)
    assert renderer.stats()["graph_replayed"] == 1
    _same(ref_a, g_a)
    _same(ref_b, g_b)
    _same(ref_a, g_a2)
    # another precision changes the kernel: captured again
    g_64 = renderer.render(scene, [a], colors, want=WANT, precision=abi.PREC_FP64, graph=True)
    assert renderer.stats()["graph_replayed"] == 0
    ref_64 = renderer.render(scene, [a], colors, want=WANT, precision=abi.PREC_FP64)
    _same(ref_64, g_64)


def test_autotune(renderer):
    scene, cam, _ = configs.workload("schwarzschild_disk", x_pix=40)
    colors = configs.log_spaced_colors(16)
    base = renderer.render(scene, [cam], colors, want=WANT, precision=abi.PREC_MIXED)
    g = renderer.render(scene, [cam], colors, want=WANT, precision=abi.PREC_MIXED, autotune=True)
    st = renderer.stats()
    assert st["block_warps"] in (2, 4) and st["refill_min"] in (1, 4, 8)
    _same(base, g)
    # cached: a second call does not tune again and picks the same shape
    renderer.render(scene, [cam], colors, want=("class",), precision=abi.PREC_MIXED, autotune=True)
    st2 = renderer.stats()
    assert (st2["block_warps"], st2["refill_min"]) == (st["block_warps"], st["refill_min"])
