"""Raw spectral output: cube layout, NPY with its sidecar, FITS round trip."""
import json

import numpy as np

from rtwca_b200 import io


def test_spectral_cube_layout():
    x, y, n = 5, 3, 4
    sp = np.arange(2 * x * y * n, dtype=np.float32).reshape(2 * x * y, n)  # two frames
    c = io.spectral_cube(sp, x, y, frame=1)
    assert c.shape == (y, x, n)
    # pixel i + x j of frame 1 is row y-1-j of the cube (rows reversed as in gen_image)
    assert np.array_equal(c[y - 1 - 2, 4], sp[x * y + 4 + x * 2])


def test_npy_and_fits_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    cube = rng.random((6, 7, 3)).astype(np.float32) * 1e15
    colors = [1086204.5, 1300000.0, 1629306.8]
    io.save_npy(str(tmp_path / "c.npy"), cube, colors, {"scene": "torus"})
    assert np.array_equal(np.load(tmp_path / "c.npy"), cube)
    side = json.load(open(str(tmp_path / "c.npy") + ".json"))
    assert side["colors_nm"] == colors and side["meta"]["scene"] == "torus"
    io.save_fits(str(tmp_path / "c.fits"), cube, colors, {"spin": 0.94, "scene": "torus"})
    raw = (tmp_path / "c.fits").read_bytes()
    assert len(raw) % 2880 == 0 and raw.startswith(b"SIMPLE  =                    T")
    back, hdr = io.load_fits(str(tmp_path / "c.fits"))
    assert np.array_equal(back, cube)
    assert (hdr["NAXIS1"], hdr["NAXIS2"], hdr["NAXIS3"], hdr["BITPIX"]) == (7, 6, 3, -32)
    assert abs(hdr["WAVE0001"] - 1300000.0) < 1e-6 and hdr["SPIN"] == 0.94 and hdr["SCENE"] == "torus"
