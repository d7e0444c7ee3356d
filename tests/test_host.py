"""Host-side logic of the package (no GPU): workload definitions, the
reference-facing API mirror, the image orientation and helpers of bench.py."""
import math

import numpy as np
import pytest

import bench
from rtwca_b200 import abi, configs, render


def test_log_spaced_colors():
    c = configs.log_spaced_colors(64)
    assert c.size == 64 and np.all(np.diff(c) > 0)
    f = 299792458.0 / (c * 1e-9)
    assert f.max() == pytest.approx(8.6e14, rel=1e-12) and f.min() == pytest.approx(3.7e14, rel=1e-12)
    r = f[:-1] / f[1:]
    assert np.allclose(r, r[0])


def test_kerr_isco_and_orbit_speed():
    assert configs.kerr_isco(0.0) == pytest.approx(6.0)
    assert configs.kerr_isco(0.9) == pytest.approx(2.320883, rel=1e-6)
    assert configs.kerr_isco(0.998) == pytest.approx(1.2370, rel=1e-3)
    # Schwarzschild circular orbit speed seen by a static observer: 1/sqrt(r/M - 2)
    assert configs.circular_orbit_beta(10.0, 0.0) == pytest.approx(1 / math.sqrt(8.0))


def test_workloads_shapes():
    for name, (_, _, xp, tol) in configs.WORKLOADS.items():
        sc, cam, col = configs.workload(name)
        assert cam.x_pix == xp and cam.tolerance == tol and cam.y_pix == xp  # square FOVs
        assert col.size == 64
    _, cams, _, meta = configs.batched_frames()
    assert len(cams) == 96
    assert sorted({m["x_pix"] for m in meta}) == [256, 512, 1024]
    assert all(5 <= m["r"] <= 40 and 10 <= m["inclination_deg"] <= 85 for m in meta)
    assert sum(c.x_pix * c.y_pix for c in cams) == 32 * (256 ** 2 + 512 ** 2 + 1024 ** 2) == 44040192


def test_worlds_table():
    worlds = render.available_worlds()
    for w in ("kerr_boyer_lindquist", "m87", "synch", "wormhole", "minkowski_t,x,y,z_sphere"):
        assert w in worlds
    with pytest.raises(ValueError):
        render.initialize_world("no such world")


class FakeRenderer:
    """Stands in for the library in the orientation test: XYZ = pixel index."""

    def render(self, scene, cams, colors, want, **kw):
        c = cams[0]
        P = c.x_pix * c.y_pix
        n = len(colors)
        out = {"xyz": np.repeat(np.arange(P, dtype=np.float32)[:, None], 3, 1),
               "class": np.ones(P, np.uint8), "steps": np.ones(P, np.uint32)}
        if "state" in want:
            out["state"] = np.tile(np.arange(P, dtype=float)[:, None], (1, 8))
            out["spectrum"] = np.tile(np.arange(P, dtype=np.float32)[:, None], (1, n))
            out["tau"] = np.arange(P, dtype=np.float32)
        return out


def test_gen_image_orientation_and_returnrays(monkeypatch, rtwlib):
    render.set_scene(configs.kerr_disk_scene())
    img, rays = render.gen_image(camera_pos=[0, 30, 1.2, 0], x_pix=6, fov_hor=60, fov_vert=40, colors=[500, 600],
                                 returnrays=True, renderer=FakeRenderer())
    yp = abi.y_pixels(6, 60, 40)
    assert img.shape == (yp, 6, 3)
    # image row 0 is the top (j = y_pix - 1): transpose(reverse(img, dims=2))
    assert img[0, 0, 0] == (yp - 1) * 6 and img[-1, 0, 0] == 0 and img[-1, 5, 0] == 5
    assert rays.shape == (6, yp, 8 + 4)
    assert rays[2, 1, 0] == 2 + 6 * 1 and rays[2, 1, 8] == 2 + 6 and rays[2, 1, 9] == 2 + 6


def test_xyz_to_srgb():
    xyz = np.array([[[0.9505, 1.0, 1.089]], [[0.0, 0.0, 0.0]]])
    rgb = render.xyz_to_srgb(xyz)
    assert np.allclose(rgb[0, 0], 1.0, atol=2e-3) and np.all(rgb[1, 0] == 0)


def test_bench_cpu_sample_ids():
    ids = bench.cpu_sample_ids(1024 * 1024, 2048)
    assert ids.size == 2048 and ids[0] == 0 and ids[-1] == 1024 * 1024 - 1
    assert np.all(np.diff(ids) > 0)


def test_gen_image_passes_textures_to_skybox_worlds():
    """load_textures' maps reach the render call for the two skybox worlds,
    with ray_bundles, and no other world gets them."""
    seen = {}

    class Spy(FakeRenderer):
        def render(self, scene, cams, colors, want, **kw):
            seen["skybox"], seen["bundles"] = kw.get("skybox"), kw.get("ray_bundles")
            return super().render(scene, cams, colors, want, **kw)

    maps = (np.zeros((6, 8, 3), np.float32), np.ones((6, 8, 3), np.float32))
    render.load_textures(*maps)
    try:
        for world in ("wormhole", "minkowski_t,x,y,z_sphere", "synch"):
            pos, d, pt, beta = render.initialize_world(world)
            render.gen_image(camera_pos=pos, camera_dir=d, speed=beta, camera_point=pt, x_pix=4, ray_bundles=True,
                             renderer=Spy())
            if world == "synch":
                assert seen["skybox"] == (None, None)
            else:
                assert seen["skybox"][0] is maps[0] and seen["skybox"][1] is maps[1]
            assert seen["bundles"] is True
    finally:
        render.load_textures(None, None)
