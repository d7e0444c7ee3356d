"""ctypes wrapper of the CPU oracle (liboracle.so) - TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker of librtw_b200.so; the product never imports it.
Parity status: unpinned against the reference itself (see rtw_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    src = [HERE / "rtw_oracle.cpp", HERE.parent / "include" / "rtw.h"]
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in src):
        env = dict(os.environ)
        r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        lib.oracle_abi_version.restype = C.c_int
        lib.oracle_cie.argtypes = [D, C.c_int, D, D, D, D]
        lib.oracle_cie.restype = C.c_int
        lib.oracle_cie_eval.argtypes = [C.c_int, C.c_double]
        lib.oracle_cie_eval.restype = C.c_double
        lib.oracle_constants.argtypes = [D, D]
        lib.oracle_camera_rays.argtypes = [P, P, D, C.c_longlong]
        lib.oracle_camera_rays.restype = C.c_int
        lib.oracle_rhs.argtypes = [P, D, C.c_int, D, D]
        lib.oracle_rhs.restype = C.c_int
        lib.oracle_metric.argtypes = [P, D, D]
        lib.oracle_pad_max_dt.argtypes = [P, D, C.c_double]
        lib.oracle_pad_max_dt.restype = C.c_double
        lib.oracle_render.argtypes = [P, P, D, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_longlong), C.c_longlong,
                                      D, C.POINTER(C.c_ubyte), C.POINTER(C.c_uint), D, D, D,
                                      C.POINTER(C.c_longlong), C.c_int]
        lib.oracle_render.restype = C.c_int
        lib.oracle_work.argtypes = [P, P, D, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_longlong), C.c_longlong,
                                    C.POINTER(C.c_longlong), C.c_int]
        lib.oracle_work.restype = C.c_int
        lib.oracle_set_skybox.argtypes = [C.c_int, C.POINTER(C.c_float), C.c_int]
        lib.oracle_set_skybox.restype = C.c_int
        lib.oracle_torus_forward.argtypes = [P, P, D, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_longlong),
                                             C.c_longlong, D, D, C.POINTER(C.c_ubyte), C.POINTER(C.c_uint),
                                             C.POINTER(C.c_int), C.c_int]
        lib.oracle_torus_forward.restype = C.c_int
        lib.oracle_set_gaunt.argtypes = [C.POINTER(C.c_float)]
        lib.oracle_set_gaunt.restype = C.c_int
        lib.oracle_gaunt.argtypes = [C.c_double, C.c_double]
        lib.oracle_gaunt.restype = C.c_float
        lib.oracle_set_diagnostics.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.oracle_set_diagnostics.restype = C.c_int
        lib.oracle_set_ray_bundles.argtypes = [C.c_int]
        lib.oracle_set_ray_bundles.restype = C.c_int
        lib.oracle_cube_wrap.argtypes = [C.c_int] * 6 + [C.POINTER(C.c_int)]
        lib.oracle_cube_wrap.restype = C.c_int
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def constants():
    e, f = C.c_double(), C.c_double()
    load().oracle_constants(C.byref(e), C.byref(f))
    return e.value, f.value


def cie(colors_nm):
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    n = c.size
    out = [np.zeros(n) for _ in range(4)]
    st = load().oracle_cie(_dp(c), n, *[_dp(o) for o in out])
    assert st == 0
    return out


def cie_eval(which: int, wl: float) -> float:
    return load().oracle_cie_eval(which, wl)


def camera_rays(scene, cam):
    from rtwca_b200 import abi
    cam = abi.Camera.from_buffer_copy(cam)
    cam.y_pix = abi.y_pixels(cam.x_pix, cam.fov_hor, cam.fov_vert)
    n = cam.x_pix * cam.y_pix
    rays = np.zeros((n, 8))
    st = load().oracle_camera_rays(C.byref(scene), C.byref(cam), _dp(rays), n)
    assert st == 0, st
    return rays


def rhs(scene, colors_nm, state, gaunt_lut=None):
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    s = np.ascontiguousarray(state, dtype=np.float64)
    out = np.zeros_like(s)
    lut = None if gaunt_lut is None else np.ascontiguousarray(gaunt_lut, dtype=np.float32)
    load().oracle_set_gaunt(lut.ctypes.data_as(C.POINTER(C.c_float)) if lut is not None else None)
    try:
        load().oracle_rhs(C.byref(scene), _dp(c), c.size, _dp(s), _dp(out))
    finally:
        load().oracle_set_gaunt(None)
    return out


def metric(scene, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    g = np.zeros(16)
    load().oracle_metric(C.byref(scene), _dp(x), _dp(g))
    return g.reshape(4, 4)


def pad_max_dt(scene, x, scale):
    x = np.ascontiguousarray(x, dtype=np.float64)
    return load().oracle_pad_max_dt(C.byref(scene), _dp(x), scale)


def render(scene, cam, colors_nm, *, max_dt_scale=0.1, integrator=0, pixel_ids=None, threads=0,
           want=("xyz", "class", "steps", "spectrum", "tau", "state"), skybox=(None, None), ray_bundles=False,
           gaunt_lut=None):
    """Traces one camera (or the pixel subset `pixel_ids`) with the FP64 oracle.
    Returns a dict of arrays indexed like the pixel list, plus 'counters'
    (step attempts, rejected attempts, polar Euler sub-steps). ray_bundles:
    the Gaussian ray-bundle lookup of the wormhole's skyboxes. want may add
    "crossings" (steps that cross the equatorial plane, per pixel) and
    "escapes" (polar Euler sub-steps, per pixel)."""
    from rtwca_b200 import abi
    cam = abi.Camera.from_buffer_copy(cam)
    cam.y_pix = abi.y_pixels(cam.x_pix, cam.fov_hor, cam.fov_vert)
    P = cam.x_pix * cam.y_pix
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    N = c.size
    ids = None
    n = P
    if pixel_ids is not None:
        ids = np.ascontiguousarray(pixel_ids, dtype=np.int64)
        n = ids.size
    res = {}
    res["xyz"] = np.zeros((n, 3)) if "xyz" in want else None
    res["class"] = np.zeros(n, np.uint8) if "class" in want else None
    res["steps"] = np.zeros(n, np.uint32) if "steps" in want else None
    res["spectrum"] = np.zeros((n, N)) if "spectrum" in want else None
    res["tau"] = np.zeros((n, N)) if "tau" in want else None
    res["state"] = np.zeros((n, 8)) if "state" in want else None
    res["crossings"] = np.zeros(n, np.int32) if "crossings" in want else None
    res["escapes"] = np.zeros(n, np.int32) if "escapes" in want else None
    counters = np.zeros(3, np.int64)

    def ptr(a, t):
        return a.ctypes.data_as(C.POINTER(t)) if a is not None else None

    # the wormhole's skyboxes (float32 [3 h, 4 h, 3] cross layout), set for this call
    texs = [None if t is None else np.ascontiguousarray(t, dtype=np.float32) for t in skybox]
    for k, t in enumerate(texs):
        load().oracle_set_skybox(k, t.ctypes.data_as(C.POINTER(C.c_float)) if t is not None else None,
                                 t.shape[0] // 3 if t is not None else 0)
    load().oracle_set_ray_bundles(int(bool(ray_bundles)))
    load().oracle_set_diagnostics(ptr(res["crossings"], C.c_int), ptr(res["escapes"], C.c_int))
    lut = None if gaunt_lut is None else np.ascontiguousarray(gaunt_lut, dtype=np.float32)
    load().oracle_set_gaunt(lut.ctypes.data_as(C.POINTER(C.c_float)) if lut is not None else None)
    try:
        st = load().oracle_render(
            C.byref(scene), C.byref(cam), _dp(c), N, float(max_dt_scale), int(integrator),
            ids.ctypes.data_as(C.POINTER(C.c_longlong)) if ids is not None else None, n,
            ptr(res["xyz"], C.c_double), ptr(res["class"], C.c_ubyte), ptr(res["steps"], C.c_uint),
            ptr(res["spectrum"], C.c_double), ptr(res["tau"], C.c_double), ptr(res["state"], C.c_double),
            counters.ctypes.data_as(C.POINTER(C.c_longlong)), int(threads))
    finally:
        for k in range(2):
            load().oracle_set_skybox(k, None, 0)
        load().oracle_set_ray_bundles(0)
        load().oracle_set_diagnostics(None, None)
        load().oracle_set_gaunt(None)
    if st != 0:
        raise RuntimeError(f"oracle_render failed with status {st}")
    res = {k: v for k, v in res.items() if v is not None}
    res["counters"] = counters
    res["y_pix"] = cam.y_pix
    return res


def work(scene, cam, colors_nm, *, max_dt_scale=0.1, integrator=0, pixel_ids=None, threads=0):
    """Algorithmic work of the reference's form over one camera's pixels (or
    `pixel_ids`): the oracle's own integration of those rays run over a
    counting scalar (same path and step counts as render()). Thin-disk scenes
    only. Returns {"flops", "transcendentals", "attempts", "rays"}:
    add/sub/mul 1 flop; div/sqrt/exp/log/sin/cos 1 flop + 1 transcendental;
    pow 2 + 2."""
    from rtwca_b200 import abi
    cam = abi.Camera.from_buffer_copy(cam)
    cam.y_pix = abi.y_pixels(cam.x_pix, cam.fov_hor, cam.fov_vert)
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    ids = None
    n = cam.x_pix * cam.y_pix
    if pixel_ids is not None:
        ids = np.ascontiguousarray(pixel_ids, dtype=np.int64)
        n = ids.size
    out = np.zeros(4, np.int64)
    st = load().oracle_work(C.byref(scene), C.byref(cam), _dp(c), c.size, float(max_dt_scale), int(integrator),
                            ids.ctypes.data_as(C.POINTER(C.c_longlong)) if ids is not None else None, n,
                            out.ctypes.data_as(C.POINTER(C.c_longlong)), int(threads))
    if st != 0:
        raise RuntimeError(f"oracle_work failed with status {st}")
    return {"flops": int(out[0]), "transcendentals": int(out[1]), "attempts": int(out[2]), "rays": int(out[3])}


def torus_forward(scene, cam, colors_nm, *, mode=0, max_dt_scale=0.1, pixel_ids=None, threads=0):
    """Forward-mode derivatives of the synchrotron torus's FSAL render: dict of
    'spectrum' [n, N], 'tangents' [n, N, 5] = dI/d(spin, inclination (rad),
    n_e0, b_0, theta_e0), 'class', 'steps', 'escapes' (polar Euler sub-steps).
    mode 0 holds the controller's step sizes fixed and differentiates those
    set by pad_max_dt (the discrete adjoint's convention); mode 1 carries the
    tangents through every step size."""
    from rtwca_b200 import abi
    cam = abi.Camera.from_buffer_copy(cam)
    cam.y_pix = abi.y_pixels(cam.x_pix, cam.fov_hor, cam.fov_vert)
    P = cam.x_pix * cam.y_pix
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    N = c.size
    ids = None if pixel_ids is None else np.ascontiguousarray(pixel_ids, dtype=np.int64)
    n = P if ids is None else ids.size
    res = {"spectrum": np.zeros((n, N)), "tangents": np.zeros((n, N, 5)), "class": np.zeros(n, np.uint8),
           "steps": np.zeros(n, np.uint32), "escapes": np.zeros(n, np.int32)}
    st = load().oracle_torus_forward(
        C.byref(scene), C.byref(cam), _dp(c), N, float(max_dt_scale), int(mode),
        ids.ctypes.data_as(C.POINTER(C.c_longlong)) if ids is not None else None, n,
        _dp(res["spectrum"]), _dp(res["tangents"]), res["class"].ctypes.data_as(C.POINTER(C.c_ubyte)),
        res["steps"].ctypes.data_as(C.POINTER(C.c_uint)), res["escapes"].ctypes.data_as(C.POINTER(C.c_int)),
        int(threads))
    if st != 0:
        raise RuntimeError(f"oracle_torus_forward failed with status {st}")
    return res


def gaunt(lut, gam2, u):
    """The oracle's own gaunt_ei_therm_van_Hoof from a [146, 81] float32 table."""
    t = np.ascontiguousarray(lut, dtype=np.float32)
    load().oracle_set_gaunt(t.ctypes.data_as(C.POINTER(C.c_float)))
    try:
        return float(load().oracle_gaunt(float(gam2), float(u)))
    finally:
        load().oracle_set_gaunt(None)


def cube_wrap(i, j, face, x, y, n):
    """The oracle's cube_wrap (gen_geometry.jl:128-344): (i, j, face) after
    moving texel (i, j) of `face` by x along i and y along j, n texels a face."""
    out = (C.c_int * 3)()
    st = load().oracle_cube_wrap(int(i), int(j), int(face), int(x), int(y), int(n), out)
    if st != 0:
        raise RuntimeError(f"oracle_cube_wrap failed with status {st}")
    return tuple(out)
