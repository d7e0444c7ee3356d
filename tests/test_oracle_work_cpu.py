"""The oracle's work count: its own integration run over a counting scalar
takes the plain FP64 run's path (same step attempts on the same pixels) and
counts the same operations on every run; per-bin scenes are refused."""
import numpy as np
import pytest

from oracle import oracle as O
from rtwca_b200 import abi, configs


@pytest.mark.parametrize("name", ["minkowski_sphere", "schwarzschild_disk", "kerr_thin_disk"])
def test_work_follows_the_oracle_path(name):
    scene, cam, colors = configs.workload(name, x_pix=48)
    P = cam.x_pix * abi.y_pixels(cam.x_pix, cam.fov_hor, cam.fov_vert)
    ids = np.linspace(0, P - 1, 96).astype(np.int64)
    r = O.render(scene, cam, colors, pixel_ids=ids, want=("steps",))
    w = O.work(scene, cam, colors, pixel_ids=ids)
    assert w["rays"] == ids.size
    assert w["attempts"] == int(r["counters"][0]) == int(r["steps"].sum())
    # a step attempt is at least its seven right-hand sides' geodesic
    # contraction (4 x 16 products and sums each) plus the stage sums over the
    # 8 + 2N state components
    L = 8 + 2 * len(colors)
    assert w["flops"] > w["attempts"] * (7 * 4 * 16 * 2 + 6 * L)
    assert w["transcendentals"] > 0
    assert O.work(scene, cam, colors, pixel_ids=ids, threads=1) == w


def test_work_refuses_per_bin_scenes():
    sc, cam, col = configs.torus_problem(x_pix=8, tol=1e-6)
    with pytest.raises(RuntimeError):
        O.work(sc, cam, col)
