"""ctypes mirror of include/rtw.h and the loader of librtw_b200.so.

The structures here are byte-for-byte the C structs of the public header; the
library is loaded lazily and a missing or unbuildable library raises (there is
no CPU fallback in the product path).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
# RTW_LIB_PATH selects another build of the same library (e.g. a tuning variant)
LIB_PATH = Path(os.environ.get("RTW_LIB_PATH", PKG / "librtw_b200.so"))

ABI_VERSION = 7
MAX_BINS = 128
MAX_FRAMES = 4096
TRACE_FIELDS = 15
NOALLOC_MAX_FRAMES = 64
NOALLOC_SCRATCH_BYTES = 24 << 20

# rtw_status
OK = 0
ERR_INVALID_CAMERA = 1
ERR_INVALID_PARAM = 2
ERR_CUDA = 3
ERR_ITER_LIMIT = 4
ERR_NAN = 5
ERR_NO_DEVICE = 6
ERR_UNSUPPORTED = 7
ERR_OOM = 8
STATUS_NAMES = {
    0: "RTW_OK", 1: "RTW_ERR_INVALID_CAMERA", 2: "RTW_ERR_INVALID_PARAM", 3: "RTW_ERR_CUDA",
    4: "RTW_ERR_ITER_LIMIT", 5: "RTW_ERR_NAN", 6: "RTW_ERR_NO_DEVICE", 7: "RTW_ERR_UNSUPPORTED",
    8: "RTW_ERR_OOM",
}

# rtw_scene_kind
SCENE_MINKOWSKI_SPHERE = 0
SCENE_SCHWARZSCHILD_DISK = 1
SCENE_KERR_DISK = 2
SCENE_KERR_THICK_DISK = 3
SCENE_KERR_SYNCHRO_TORUS = 4
SCENE_KERR_POWEHI = 5
SCENE_SYNCHRO_TEST = 6
SCENE_WORMHOLE = 7
SCENE_MINKOWSKI_CART_SPHERE = 8
SCENE_KERR_BREMS_TORUS = 9
GAUNT_ROWS = 146
GAUNT_COLS = 81
ADJOINT_PARAMS = ("spin", "inclination", "n_e0", "b_0", "theta_e0")

# rtw_term_class
CLASS_NONE = 0
CLASS_ESCAPE = 1
CLASS_HORIZON = 2
CLASS_THICK = 3
CLASS_WINDING = 4
CLASS_MAXSTEPS = 5
CLASS_NAN = 6
CLASS_NAMES = {0: "none", 1: "escape", 2: "horizon", 3: "thick", 4: "winding", 5: "maxsteps", 6: "nan"}

# rtw_precision / rtw_integrator
PREC_FP64 = 0
PREC_MIXED = 1
PREC_FP64_PLAIN = 2
DP45_REF_COMPAT = 0
DP45_FSAL = 1


class Scene(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("ref_precision", C.c_int32),
        ("mass", C.c_double), ("spin", C.c_double),
        ("r_in", C.c_double), ("r_out", C.c_double),
        ("theta_lo", C.c_double), ("theta_hi", C.c_double),
        ("temperature", C.c_double), ("a_nu", C.c_double),
        ("escape_radius", C.c_double), ("winding_limit", C.c_double),
        ("rho_r0", C.c_double), ("rho_h", C.c_double),
        ("rho_index", C.c_double), ("t_index", C.c_double),
        ("n_e0", C.c_double), ("b_0", C.c_double), ("theta_e0", C.c_double), ("b_index", C.c_double),
        ("edge_in", C.c_double), ("edge_out", C.c_double), ("length_cm", C.c_double),
    ]


class Camera(C.Structure):
    _fields_ = [
        ("position", C.c_double * 4), ("direction", C.c_double * 2), ("speed", C.c_double),
        ("pointing", C.c_double * 3), ("x_pix", C.c_int32), ("y_pix", C.c_int32),
        ("fov_hor", C.c_double), ("fov_vert", C.c_double),
        ("tolerance", C.c_double), ("max_steps", C.c_int64),
        ("win_x0", C.c_int32), ("win_y0", C.c_int32), ("win_w", C.c_int32), ("win_h", C.c_int32),
    ]


class RenderParams(C.Structure):
    _fields_ = [
        ("n_colors", C.c_int32), ("precision", C.c_int32), ("colors_nm", C.POINTER(C.c_double)),
        ("max_dt_scale", C.c_double), ("integrator", C.c_int32), ("ray_bundles", C.c_int32),
        ("promote_dr", C.c_double), ("promote_sin", C.c_double),
        ("block_warps", C.c_int32), ("ctas_per_sm", C.c_int32),
        ("stream", C.c_void_p), ("pixel_order", C.c_int32), ("refill_min", C.c_int32),
        ("trace_ray", C.c_int64), ("autotune", C.c_int32), ("graph", C.c_int32),
        ("skybox", C.POINTER(C.c_float) * 2), ("skybox_h", C.c_int32 * 2),
        ("gaunt_lut", C.POINTER(C.c_float)), ("tail_pass", C.c_int32),
    ]


class Outputs(C.Structure):
    _fields_ = [
        ("xyz", C.c_void_p), ("term_class", C.c_void_p), ("steps", C.c_void_p),
        ("spectrum", C.c_void_p), ("final_state", C.c_void_p), ("tau", C.c_void_p),
        ("on_device", C.c_int32), ("trace_capacity", C.c_int32), ("trace", C.c_void_p),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("rays", C.c_uint64), ("step_attempts", C.c_uint64), ("rejected_steps", C.c_uint64),
        ("promoted_steps", C.c_uint64), ("spectral_steps", C.c_uint64), ("emitting_steps", C.c_uint64),
        ("escape_substeps", C.c_uint64), ("nan_rays", C.c_uint64),
        ("kernel_ms", C.c_double), ("total_ms", C.c_double), ("phase_cycles", C.c_uint64 * 4),
        ("grid", C.c_int32), ("block_warps", C.c_int32), ("refill_min", C.c_int32), ("graph_replayed", C.c_int32),
        ("tail_rays", C.c_uint64), ("launches", C.c_int32), ("reserved0", C.c_int32),
    ]


class AdjointParams(C.Structure):
    _fields_ = [
        ("target", C.c_void_p), ("target_on_device", C.c_int32), ("checkpoint_every", C.c_int32),
        ("camera_delta", C.c_double), ("per_ray_grad", C.c_void_p), ("escape_rays", C.c_int32),
        ("reserved", C.c_int32), ("ray_begin", C.c_int64), ("ray_count", C.c_int64), ("ray_stride", C.c_int64),
    ]


class AdjointResult(C.Structure):
    _fields_ = [
        ("loss", C.c_double), ("grad", C.c_double * 5), ("forward_ms", C.c_double), ("record_ms", C.c_double),
        ("reverse_ms", C.c_double), ("total_ms", C.c_double), ("events", C.c_uint64), ("checkpoints", C.c_uint64),
        ("scratch_bytes", C.c_uint64), ("escape_rays", C.c_uint64), ("escape_cuts", C.c_uint64),
    ]


class OpCounts(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "rhs_vacuum", "rhs_vacuum_mufu", "rhs_emit", "rhs_emit_mufu", "step_overhead", "step_overhead_mufu",
        "bin_step", "bin_step_mufu")]


# Every function the header declares, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    "rtw_create": (C.c_int, [C.POINTER(_P), C.c_int32]),
    "rtw_destroy": (None, [_P]),
    "rtw_last_error": (C.c_char_p, [_P]),
    "rtw_abi_version": (C.c_int32, []),
    "rtw_scene_default": (C.c_int, [C.c_int32, C.POINTER(Scene)]),
    "rtw_camera_pixels": (C.c_int, [C.POINTER(Camera), C.POINTER(C.c_int64)]),
    "rtw_camera_rays": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(C.c_double), C.c_int64]),
    "rtw_cie_weights": (C.c_int, [C.POINTER(C.c_double), C.c_int32] + [C.POINTER(C.c_double)] * 4),
    "rtw_render": (C.c_int, [_P, C.POINTER(Scene), C.POINTER(Camera), C.c_int32,
                             C.POINTER(RenderParams), C.POINTER(Outputs)]),
    "rtw_get_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "rtw_get_frame_times": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "rtw_adjoint": (C.c_int, [_P, C.POINTER(Scene), C.POINTER(Camera), C.POINTER(RenderParams),
                              C.POINTER(AdjointParams), C.POINTER(Outputs), C.POINTER(AdjointResult)]),
    "rtw_torus_rhs": (C.c_int, [C.POINTER(Scene), C.POINTER(C.c_double), C.c_int32, C.c_int32,
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "rtw_torus_vjp": (C.c_int, [C.POINTER(Scene), C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "rtw_skybox_wrap": (C.c_int, [C.c_int32] * 6 + [C.POINTER(C.c_int32)]),
    "rtw_torus_step_vjp": (C.c_int, [C.POINTER(Scene), C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double),
                                     C.c_double, C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "rtw_torus_escape_vjp": (C.c_int, [C.POINTER(Scene), C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double),
                                       C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "rtw_measure_peaks": (C.c_int, [_P] + [C.POINTER(C.c_double)] * 3),
    "rtw_get_op_counts": (C.c_int, [C.c_int32, C.POINTER(OpCounts)]),
    "rtw_render_noalloc": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_int32, C.POINTER(RenderParams),
                                     C.POINTER(Outputs)]),
    "rtw_noalloc_last_error": (C.c_char_p, []),
    "rtw_scene_rhs": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                C.POINTER(C.c_double)]),
    "rtw_gaunt_lookup": (C.c_float, [C.POINTER(C.c_float), C.c_double, C.c_double]),
    "rtw_brems_rhs": (C.c_int, [C.POINTER(Scene), C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_float),
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}

_lib = None


def load(path: Path | str | None = None) -> C.CDLL:
    """Loads librtw_b200.so (built by rtwca_b200.build) and binds every symbol."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build the CUDA library first (python -m rtwca_b200.build or "
            "__graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.rtw_abi_version() != ABI_VERSION:
        raise RuntimeError("librtw_b200.so ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


class RTWError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


def check(status: int, msg: str = "") -> None:
    if status != OK:
        raise RTWError(status, msg)


def op_counts(kind: int) -> dict:
    oc = OpCounts()
    check(load().rtw_get_op_counts(kind, C.byref(oc)), "op_counts")
    return {f: getattr(oc, f) for f, _ in OpCounts._fields_}


def scene_rhs(scene: Scene, state, fp32: bool = False):
    """Host evaluation of the kernel's right-hand side: (slope[9], (A, X, ktau))."""
    import numpy as np
    st = np.ascontiguousarray(state, dtype=np.float64)
    out = np.zeros(9)
    em = np.zeros(3)
    D = C.POINTER(C.c_double)
    check(load().rtw_scene_rhs(C.byref(scene), int(fp32), st.ctypes.data_as(D), out.ctypes.data_as(D),
                               em.ctypes.data_as(D)), "scene_rhs")
    return out, em


def scene_default(kind: int) -> Scene:
    s = Scene()
    check(load().rtw_scene_default(kind, C.byref(s)), "scene_default")
    return s


def camera_pixels(c: "Camera") -> int:
    """Pixels a camera renders: its window (win_w x win_h) or the whole image
    (sets c.y_pix)."""
    c.y_pix = y_pixels(c.x_pix, c.fov_hor, c.fov_vert)
    if c.win_w or c.win_h:
        return int(c.win_w) * int(c.win_h)
    return c.x_pix * c.y_pix


def window(c: "Camera", x0: int, y0: int, w: int, h: int) -> "Camera":
    """A copy of camera c that renders pixels [x0, x0 + w) x [y0, y0 + h) of its image."""
    d = Camera.from_buffer_copy(c)
    d.win_x0, d.win_y0, d.win_w, d.win_h = int(x0), int(y0), int(w), int(h)
    return d


def make_camera(position, direction=(0.0, 0.0), speed=0.0, pointing=(0.0, 0.0, 0.0), x_pix=100,
                fov_hor=85.0, fov_vert=60.0, tolerance=1e-4, max_steps=1000) -> Camera:
    c = Camera()
    for i in range(4):
        c.position[i] = float(position[i])
    for i in range(2):
        c.direction[i] = float(direction[i])
    for i in range(3):
        c.pointing[i] = float(pointing[i])
    c.speed = float(speed)
    c.x_pix = int(x_pix)
    c.fov_hor = float(fov_hor)
    c.fov_vert = float(fov_vert)
    c.tolerance = float(tolerance)
    c.max_steps = int(max_steps)
    c.y_pix = y_pixels(c.x_pix, c.fov_hor, c.fov_vert)
    return c


def y_pixels(x_pix: int, fov_hor: float, fov_vert: float) -> int:
    """round(x_pix * tan(fov_vert/2) / tan(fov_hor/2)), ties to even (initialization.jl:197-200)."""
    W = math.tan(math.pi * fov_hor / 180 / 2)
    H = math.tan(math.pi * fov_vert / 180 / 2)
    return int(round(x_pix * H / W))


def torus_rhs(scene: Scene, colors_nm, state, form: int = 0):
    """Host FP64 torus right-hand side (reference layout: x, k, then (I, tau) per bin)."""
    import numpy as np
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    st = np.ascontiguousarray(state, dtype=np.float64)
    out = np.zeros_like(st)
    dp = C.POINTER(C.c_double)
    check(load().rtw_torus_rhs(C.byref(scene), c.ctypes.data_as(dp), int(c.size), int(form), st.ctypes.data_as(dp),
                               out.ctypes.data_as(dp)), "torus_rhs")
    return out


def gaunt_lookup(lut, gam2: float, u: float) -> float:
    """The library's Gaunt factor (gaunt_ei_therm_van_Hoof) from a
    [GAUNT_ROWS, GAUNT_COLS] float32 table."""
    import numpy as np
    t = np.ascontiguousarray(lut, dtype=np.float32)
    assert t.shape == (GAUNT_ROWS, GAUNT_COLS)
    return float(load().rtw_gaunt_lookup(t.ctypes.data_as(C.POINTER(C.c_float)), float(gam2), float(u)))


def brems_rhs(scene: Scene, colors_nm, lut, state):
    """Host FP64 right-hand side of the bremsstrahlung torus (layout of torus_rhs)."""
    import numpy as np
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    t = np.ascontiguousarray(lut, dtype=np.float32)
    st = np.ascontiguousarray(state, dtype=np.float64)
    out = np.zeros_like(st)
    dp = C.POINTER(C.c_double)
    check(load().rtw_brems_rhs(C.byref(scene), c.ctypes.data_as(dp), int(c.size),
                               t.ctypes.data_as(C.POINTER(C.c_float)), st.ctypes.data_as(dp),
                               out.ctypes.data_as(dp)), "brems_rhs")
    return out


def torus_vjp(scene: Scene, colors_nm, state, cot):
    """Host FP64 vector-Jacobian product of the torus right-hand side: (J^T cot, d/d params)."""
    import numpy as np
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    st = np.ascontiguousarray(state, dtype=np.float64)
    ct = np.ascontiguousarray(cot, dtype=np.float64)
    mu = np.zeros_like(st)
    pb = np.zeros(5)
    dp = C.POINTER(C.c_double)
    check(load().rtw_torus_vjp(C.byref(scene), c.ctypes.data_as(dp), int(c.size), st.ctypes.data_as(dp),
                               ct.ctypes.data_as(dp), mu.ctypes.data_as(dp), pb.ctypes.data_as(dp)), "torus_vjp")
    return mu, pb


def torus_escape_vjp(scene: Scene, colors_nm, state, n_sub: int, cot):
    """Host polar escape of the torus and its VJP: (end_state, J^T cot, d/d params, guard_ok)."""
    import numpy as np
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    st = np.ascontiguousarray(state, dtype=np.float64)
    ct = np.ascontiguousarray(cot, dtype=np.float64)
    end = np.zeros_like(st)
    mu = np.zeros_like(st)
    pb = np.zeros(5)
    dp = C.POINTER(C.c_double)
    r = load().rtw_torus_escape_vjp(C.byref(scene), c.ctypes.data_as(dp), int(c.size), st.ctypes.data_as(dp),
                                    int(n_sub), ct.ctypes.data_as(dp), end.ctypes.data_as(dp),
                                    mu.ctypes.data_as(dp), pb.ctypes.data_as(dp))
    if r not in (OK, ERR_NAN):
        check(r, "torus_escape_vjp")
    return end, mu, pb, r == OK


def torus_step_vjp(scene: Scene, colors_nm, state, h: float, cot, form: int = 0):
    """Host reverse of one torus DP45 step: (J^T cot, d/d params, d/d h)."""
    import numpy as np
    c = np.ascontiguousarray(colors_nm, dtype=np.float64)
    st = np.ascontiguousarray(state, dtype=np.float64)
    ct = np.ascontiguousarray(cot, dtype=np.float64)
    mu = np.zeros_like(st)
    pb = np.zeros(5)
    hb = C.c_double(0)
    dp = C.POINTER(C.c_double)
    check(load().rtw_torus_step_vjp(C.byref(scene), c.ctypes.data_as(dp), int(c.size), st.ctypes.data_as(dp),
                                    float(h), ct.ctypes.data_as(dp), int(form), mu.ctypes.data_as(dp),
                                    pb.ctypes.data_as(dp), C.byref(hb)), "torus_step_vjp")
    return mu, pb, hb.value
