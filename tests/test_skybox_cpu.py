"""The wormhole's skybox lookup on the CPU: the library's cube-map neighbour
rule (the function the device's ray-bundle footprint runs, evaluated on the
host) against the oracle's separately written restatement of cube_wrap
(gen_geometry.jl:128-344) over every texel, face and footprint offset, and
properties of the oracle's ray-bundle lookup (calc_skybox_I_nu_beam!,
Wormhole.source/source_model.jl:266-358), and the oracle's Cartesian
blackbody sphere (Minkowski_Sphere_Cartesian.source) against the closed form
of a straight ray through it.
"""
import ctypes as C

import numpy as np
import pytest

from rtwca_b200 import abi, configs


def _lib_wrap(lib):
    f = lib.rtw_skybox_wrap
    f.argtypes = [C.c_int32] * 6 + [C.POINTER(C.c_int32)]
    f.restype = C.c_int
    out = (C.c_int32 * 3)()

    def wrap(i, j, face, x, y, n):
        assert f(i, j, face, x, y, n, out) == abi.OK
        return tuple(out)

    return wrap


def test_cube_wrap_library_matches_oracle(rtwlib, oracle):
    """Every texel of an 11-texel face, every face, every offset of the
    largest footprint (|x|, |y| <= 10): both restatements agree exactly."""
    wrap = _lib_wrap(rtwlib)
    n = 11
    bad = []
    for face in range(1, 7):
        for i in range(1, n + 1):
            for j in range(1, n + 1):
                for x in range(-10, 11):
                    for y in range(-10, 11):
                        a = wrap(i, j, face, x, y, n)
                        b = oracle.cube_wrap(i, j, face, x, y, n)
                        if a != b:
                            bad.append(((i, j, face, x, y), a, b))
    assert not bad, bad[:5]


def test_cube_wrap_properties(rtwlib):
    """Moves inside a face stay there; the ring of faces 1-4 along i is a
    cycle (a move and its reverse return to the start); crossing the top edge
    of face 2 enters face 6 and its bottom edge face 5."""
    wrap = _lib_wrap(rtwlib)
    n = 16
    assert wrap(5, 7, 3, 4, -3, n) == (9, 4, 3)
    for face in range(1, 5):
        for i in (1, 8, 16):
            for x in (-10, -1, 1, 10):
                i2, j2, f2 = wrap(i, 5, face, x, 0, n)
                assert f2 in (1, 2, 3, 4) and j2 == 5
                assert wrap(i2, j2, f2, -x, 0, n) == (i, 5, face)
    assert wrap(4, 16, 2, 0, 1, n)[2] == 6
    assert wrap(4, 1, 2, 0, -1, n)[2] == 5


def test_cube_wrap_rejects_bad_arguments(rtwlib, oracle):
    """A face outside 1..6, a face edge under 1 texel or no output buffer is
    RTW_ERR_INVALID_PARAM from the library's hook and the oracle's."""
    f = rtwlib.rtw_skybox_wrap
    out = (C.c_int32 * 3)()
    assert f(1, 1, 0, 0, 0, 4, out) == abi.ERR_INVALID_PARAM
    assert f(1, 1, 7, 0, 0, 4, out) == abi.ERR_INVALID_PARAM
    assert f(1, 1, 1, 0, 0, 0, out) == abi.ERR_INVALID_PARAM
    assert f(1, 1, 1, 0, 0, 4, None) == abi.ERR_INVALID_PARAM
    with pytest.raises(RuntimeError):
        oracle.cube_wrap(1, 1, 9, 0, 0, 4)


def _wormhole_case(H, seed):
    rng = np.random.default_rng(seed)
    sky = tuple(rng.uniform(0, 1, (3 * H, 4 * H, 3)).astype(np.float32) for _ in range(2))
    sc = configs.wormhole_scene()
    cam = configs.wormhole_camera(12, 1e-6)
    col = np.array([467.0, 532.0, 630.0])
    return sc, cam, col, sky


def test_oracle_bundle_lookup_properties(oracle):
    """With a uniform map the footprint only rescales the texel's spectrum:
    bundle / plain is the same in every bin of a pixel (the summed weights);
    with a random map the footprint changes the image; either way the
    geodesics and the step counts do not depend on the bundle (its components
    have zero slope and stay out of the error norm)."""
    sc, cam, col, sky = _wormhole_case(16, 7)
    ids = np.arange(0, 12 * 8, 5)
    flat = tuple(np.full_like(s, 0.5) for s in sky)
    kw = dict(integrator=abi.DP45_FSAL, pixel_ids=ids, want=("spectrum", "steps", "state"))
    p = oracle.render(sc, cam, col, skybox=flat, **kw)
    b = oracle.render(sc, cam, col, skybox=flat, ray_bundles=True, **kw)
    assert np.array_equal(p["steps"], b["steps"]) and np.array_equal(p["state"], b["state"])
    ratio = b["spectrum"] / p["spectrum"]
    assert np.all(ratio > 0.05) and np.all(ratio < 2)
    np.testing.assert_allclose(ratio, ratio[:, :1] * np.ones_like(ratio), rtol=1e-12)
    p = oracle.render(sc, cam, col, skybox=sky, **kw)
    b = oracle.render(sc, cam, col, skybox=sky, ray_bundles=True, **kw)
    assert np.median(np.abs(b["spectrum"] / p["spectrum"] - 1)) > 1e-2
    # the bundle flag is reset after each call
    again = oracle.render(sc, cam, col, skybox=sky, **kw)
    assert np.array_equal(again["spectrum"], p["spectrum"])


@pytest.mark.parametrize("H", [3, 16])
def test_oracle_bundle_lookup_small_maps(oracle, H):
    """Faces smaller than the footprint (3 texels: offsets wrap past a whole
    face, where the reference stops with an index error) give finite, positive
    spectra: texels whose coordinates leave the map are skipped."""
    sc, cam, col, sky = _wormhole_case(H, 11)
    r = oracle.render(sc, cam, col, integrator=abi.DP45_FSAL, skybox=sky, ray_bundles=True,
                      pixel_ids=np.arange(0, 96, 7), want=("spectrum",))
    assert np.all(np.isfinite(r["spectrum"])) and np.all(r["spectrum"] > 0)


def test_oracle_cart_sphere_closed_form(oracle):
    """The Cartesian blackbody sphere in the oracle against the closed form of
    a straight ray through a uniform, optically thin sphere at rest: tau is the
    chord 2 sqrt(r^2 - b^2) (a_nu = 1, k^t = 1) and I_c = B_c (1 - exp(-tau)),
    B_c = emission_scale / (exp(f_factor nu_c / T) - 1); rays that miss it stay
    dark without a skybox; with one, every ray adds the skybox texel it points
    at, attenuated by exp(-tau)."""
    sc = configs.cart_sphere_scene()
    cam = configs.cart_sphere_camera(24, 1e-8)
    col = np.array([450.0, 550.0, 650.0])
    x0 = oracle.camera_rays(sc, cam)
    p0, d = x0[:, 1:4], x0[:, 5:8] / x0[:, 4:5]
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    b2 = np.sum(p0 * p0, axis=1) - np.sum(p0 * d, axis=1) ** 2  # squared impact parameter
    chord = 2 * np.sqrt(np.maximum(0.0, 1.0 - b2))
    r = oracle.render(sc, cam, col, integrator=abi.DP45_FSAL, want=("spectrum", "tau", "class"))
    assert np.all(r["class"] == abi.CLASS_ESCAPE)
    es, ff = oracle.constants()
    B = es / np.expm1(ff / col / 5778.0)
    hit = chord > 0.05
    assert hit.sum() > 20 and (~hit).sum() > 20
    np.testing.assert_allclose(r["tau"][hit], np.repeat(chord[hit, None], 3, 1), rtol=2e-3, atol=2e-4)
    np.testing.assert_allclose(r["spectrum"][hit], B * -np.expm1(-r["tau"][hit]), rtol=1e-5)
    assert np.all(r["spectrum"][chord == 0] == 0) and np.all(r["tau"][chord == 0] == 0)
    H = 8
    flat = np.full((3 * H, 4 * H, 3), 0.5, np.float32)
    s = oracle.render(sc, cam, col, integrator=abi.DP45_FSAL, skybox=(flat, None), want=("spectrum", "tau"))
    sky = (s["spectrum"] - r["spectrum"]) / np.exp(-r["tau"])
    np.testing.assert_allclose(sky, np.repeat(sky[:1], len(sky), 0), rtol=1e-9)  # one colour, k^t = 1
    assert np.all(sky > 0)


def _hand_skybox(sky, h, state, freq_nm, tau):
    """The skybox term of a ray of the Cartesian sphere, written from the
    reference's functions by hand (Minkowski_Sphere_Cartesian.source/
    source_model.jl:175-188, 191-280, 406-424; gen_geometry.jl:347-370;
    my_special_functions.jl:20-22): face of the largest |direction|
    component, (u, v) on it, the texel (i, j), its place in the cross layout,
    the map's row 3h + 1 - j, and three Gaussian lines per texel colour."""
    v = np.asarray(state[4:8], dtype=np.float64)
    n = np.sqrt(v[1] ** 2 + v[2] ** 2 + v[3] ** 2)
    x, y, z = v[1] / n, v[2] / n, v[3] / n
    if abs(x) >= abs(y) and abs(x) >= abs(z):
        face = 1 if x > 0 else 3
    elif abs(y) >= abs(x) and abs(y) >= abs(z):
        face = 4 if y > 0 else 2
    else:
        face = 6 if z > 0 else 5
    if face == 1:
        u, w = -y / abs(x), z / abs(x)
    elif face == 2:
        u, w = -x / abs(y), z / abs(y)
    elif face == 3:
        u, w = y / abs(x), z / abs(x)
    elif face == 4:
        u, w = x / abs(y), z / abs(y)
    elif face == 5:
        u, w = -x / abs(z), -y / abs(z)
    else:
        u, w = -x / abs(z), y / abs(z)
    i = min(int(np.floor(h * (u + 1) / 2)) + 1, h)
    j = min(int(np.floor(h * (w + 1) / 2)) + 1, h)
    di, dj = {1: (0, h), 2: (h, h), 3: (2 * h, h), 4: (3 * h, h), 5: (h, 0), 6: (h, 2 * h)}[face]
    ia, ja = i + di, j + dj
    rgb = sky[3 * h + 1 - ja - 1, ia - 1].astype(np.float64)

    def ng(f, s, m):
        return np.exp(-(f - m) ** 2 / (2 * s * s)) / (s * np.sqrt(2 * np.pi))

    f = np.asarray(freq_nm) * v[0]  # freq_shift = -[1,0,0,0] g v = v^t in flat space
    I = 1e-12 * (1.0 * rgb[0] * ng(f, 5e-5, 0.001587) + 0.843 * rgb[1] * ng(f, 7e-5, 0.001879)
                 + 0.914 * rgb[2] * ng(f, 9e-5, 0.002141))
    return I * np.exp(-np.asarray(tau)) / f ** 3


def test_cart_sphere_skybox_against_hand_computation(oracle):
    """Pins the skybox lookup independently of the oracle's code (the skybox
    golden fixtures pin it only against itself): for every ray of the
    Cartesian sphere that misses the sphere (a straight line, tau = 0), the
    oracle's spectrum equals the hand computation of the texel its final
    direction points at, on a map whose every texel has its own colour."""
    h = 8
    rng = np.random.default_rng(21)
    sky = rng.uniform(0.05, 1.0, (3 * h, 4 * h, 3)).astype(np.float32)
    col = np.array([467.0, 532.0, 630.0])
    cam = configs.cart_sphere_camera(24, 1e-6)
    r = oracle.render(configs.cart_sphere_scene(), cam, col, integrator=abi.DP45_FSAL, skybox=(sky, None),
                      want=("spectrum", "state", "tau", "class"))
    miss = np.all(r["tau"] == 0, axis=1) & (r["class"] == abi.CLASS_ESCAPE)
    assert miss.sum() > 100
    for q in np.flatnonzero(miss):
        want = _hand_skybox(sky, h, r["state"][q], 1.0 / col, r["tau"][q])
        assert np.allclose(r["spectrum"][q], want, rtol=1e-12, atol=0), (q, r["spectrum"][q], want)
