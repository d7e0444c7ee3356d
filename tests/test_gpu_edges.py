"""Edge cases of the render call on the GPU: the largest bin count, the most
cameras in one launch, one-pixel frames, and the inputs rtw_render rejects
before any launch."""
import ctypes as C

import numpy as np
import pytest

from rtwca_b200 import abi, configs
from tests.parity import summarize

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_max_bins(renderer, oracle, precision):
    """RTW_MAX_BINS (128) bins: four bins per lane."""
    scene, cam, _ = configs.workload("kerr_thin_disk", x_pix=12)
    colors = configs.log_spaced_colors(abi.MAX_BINS)
    g = renderer.render(scene, [cam], colors, want=("xyz", "class", "steps", "spectrum"), precision=precision)
    r = oracle.render(scene, cam, colors)
    s = summarize(g, r)
    assert s["class_match"] >= 0.99 and s["frac_within_1e-3"] >= 0.99, s
    assert g["spectrum"].shape == (cam.x_pix * cam.y_pix, abi.MAX_BINS)


def test_max_cameras_in_one_launch(renderer):
    """RTW_MAX_FRAMES cameras of 2x2 pixels at varied positions in one launch;
    sampled frames equal their single-camera renders; one more is rejected."""
    rng = np.random.default_rng(4)
    cams = [configs.look_at_camera(float(rng.uniform(8, 40)), float(rng.uniform(0.3, 2.8)), 30.0, 2, 1e-6)
            for _ in range(abi.MAX_FRAMES)]
    scene = configs.kerr_disk_scene()
    colors = configs.log_spaced_colors(8)
    batch = renderer.render(scene, cams, colors, want=("xyz", "class", "steps"), precision=abi.PREC_MIXED)
    assert batch["class"].size == 4 * abi.MAX_FRAMES
    assert np.all(batch["class"] > 0)
    for f in (0, 1, 777, abi.MAX_FRAMES - 1):
        one = renderer.render(scene, [cams[f]], colors, want=("xyz", "class", "steps"), precision=abi.PREC_MIXED)
        for k in ("xyz", "class", "steps"):
            assert np.array_equal(batch[k][4 * f:4 * f + 4], one[k]), (f, k)
    with pytest.raises(abi.RTWError):
        renderer.render(scene, cams + cams[:1], colors, want=("class",), precision=abi.PREC_MIXED)


def test_one_pixel_frame(renderer, oracle):
    scene, cam, colors = configs.workload("schwarzschild_disk", x_pix=1)
    g = renderer.render(scene, [cam], colors, want=("xyz", "class", "steps"), precision=abi.PREC_FP64)
    r = oracle.render(scene, cam, colors)
    assert cam.y_pix == 1 and g["class"].size == 1
    assert g["class"][0] == r["class"][0]
    assert abs(g["xyz"][0, 1] - r["xyz"][0, 1]) <= 1e-3 * max(abs(r["xyz"][0, 1]), 1e-30)


def _call(renderer, scene, cams, params):
    arr = (abi.Camera * max(len(cams), 1))(*cams) if cams else (abi.Camera * 1)()
    out = abi.Outputs()
    out.on_device = 0
    return renderer._lib.rtw_render(renderer.handle, C.byref(scene), arr, len(cams), C.byref(params), C.byref(out))


def test_rejected_inputs(renderer):
    scene, cam, colors = configs.workload("kerr_thin_disk", x_pix=4)
    ok = renderer.params(colors, precision=abi.PREC_MIXED)
    assert _call(renderer, scene, [cam], ok) == abi.OK
    assert _call(renderer, scene, [], ok) == abi.ERR_INVALID_PARAM                # no camera
    bad = renderer.params(colors, precision=7)
    assert _call(renderer, scene, [cam], bad) == abi.ERR_INVALID_PARAM              # precision
    bad = renderer.params(colors, integrator=5)
    assert _call(renderer, scene, [cam], bad) == abi.ERR_INVALID_PARAM              # integrator
    bad = renderer.params(configs.log_spaced_colors(abi.MAX_BINS + 1))
    assert _call(renderer, scene, [cam], bad) == abi.ERR_INVALID_PARAM              # too many bins
    bad = renderer.params(colors, max_dt_scale=0.0)
    assert _call(renderer, scene, [cam], bad) == abi.ERR_INVALID_PARAM              # step cap
    spin = abi.Scene.from_buffer_copy(scene)
    spin.spin = 1.5
    assert _call(renderer, spin, [cam], ok) == abi.ERR_INVALID_PARAM                # |a| >= M
    tol = abi.Camera.from_buffer_copy(cam)
    tol.tolerance = 2.0
    assert _call(renderer, scene, [tol], ok) == abi.ERR_INVALID_PARAM               # tolerance
    pole = abi.Camera.from_buffer_copy(cam)
    pole.position[2] = 0.0
    assert _call(renderer, scene, [pole], ok) == abi.ERR_INVALID_CAMERA             # on the axis
    bundles = renderer.params(colors, ray_bundles=True)
    assert _call(renderer, scene, [cam], bundles) == abi.ERR_UNSUPPORTED            # wormhole only
    assert renderer.last_error() != ""


def test_frame_in_tiles_equals_whole_frame(renderer):
    """One frame rendered as interleaved 16 x 16 tiles (windowed cameras, the
    multi-GPU split of a frame; here both halves on this GPU) reassembles to
    the whole-frame render exactly: each ray's arithmetic does not depend on
    its batch."""
    from rtwca_b200 import shard
    scene, cam, colors = configs.workload("kerr_thin_disk", x_pix=72)
    whole = renderer.render(scene, [cam], colors, want=("xyz", "class", "steps"), precision=abi.PREC_MIXED)
    wins = shard.tile_windows(cam.x_pix, cam.y_pix, 16)
    tiles = {}
    for rank in range(2):  # the two ranks' shares, rendered one after the other
        mine = shard.tiles_of_rank(len(wins), 2, rank)
        res = renderer.render(scene, [abi.window(cam, *wins[t]) for t in mine], colors,
                              want=("xyz", "class", "steps"), precision=abi.PREC_MIXED)
        off = 0
        for t in mine:
            n = wins[t][2] * wins[t][3]
            tiles[t] = {k: res[k][off:off + n] for k in ("xyz", "class", "steps")}
            off += n
    got = shard.assemble_tiles(wins, tiles, cam.x_pix, cam.y_pix)
    for k in ("xyz", "class", "steps"):
        assert np.array_equal(got[k], whole[k]), k
    one = shard.render_frame_tiles(renderer, scene, cam, colors, precision=abi.PREC_MIXED)
    assert np.array_equal(one["xyz"], whole["xyz"])
    bad = abi.window(cam, cam.x_pix - 4, 0, 8, 8)  # past the image's edge
    with pytest.raises(abi.RTWError):
        renderer.render(scene, [bad], colors, want=("class",), precision=abi.PREC_MIXED)
