"""Host side of the render call, mirroring the reference's Julia API.

``initialize_world(name)`` selects a scene the way the reference's
initialize_world (main/initialization.jl:78-172) ``include``s a ``.source``
folder, and returns its default camera (position, direction, pointing, beta).
``gen_image(...)`` takes the keyword arguments of the reference's gen_image
(main/Iterators/LttM/LttM.jl:104-107, main/Iterators/5P/5P.jl:135-138) with the
same meaning and defaults, and calls librtw_b200.so through its C ABI.

Differences, by design of the library: gen_image returns linear CIE XYZ
[y_pix, x_pix, 3] in the reference's image orientation (the reference converts
to xyY, normalises brightness and converts to RGB{N0f16}; ``xyz_to_srgb`` gives
that last step as an informational helper); the wormhole's skybox textures,
which the reference loads from PNG files that its repository does not hold,
are arrays the caller hands to ``load_textures``; and ``ray_bundles=True`` (the
Gaussian footprint lookup of those skyboxes) is built for the two skybox
scenes (the wormhole and the Cartesian sphere), whose images depend on it, and
raises RTW_ERR_UNSUPPORTED elsewhere.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import abi

PI = math.pi


class Renderer:
    """One library context (one CUDA device, one stream, cached device buffers)."""

    def __init__(self, device: int = 0):
        self._lib = abi.load()
        self._ctx = C.c_void_p()
        st = self._lib.rtw_create(C.byref(self._ctx), int(device))
        abi.check(st, f"rtw_create(device={device})")

    def close(self) -> None:
        if self._ctx:
            self._lib.rtw_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._ctx

    def last_error(self) -> str:
        return (self._lib.rtw_last_error(self._ctx) or b"").decode()

    @staticmethod
    def params(colors_nm, precision=abi.PREC_FP64, integrator=abi.DP45_REF_COMPAT, max_dt_scale=0.1,
               block_warps=0, ctas_per_sm=0, promote_dr=0.0, promote_sin=0.0, stream=None,
               pixel_order=0, ray_bundles=False, trace_ray=-1, refill_min=0, autotune=False, graph=False,
               skybox=(None, None), gaunt_lut=None, tail_pass=True):
        """skybox: the wormhole's two cube maps, each None or a float32 array
        [3 h, 4 h, 3] in the reference's cross layout (RGB in [0, 1])."""
        colors = np.ascontiguousarray(np.asarray(colors_nm, dtype=np.float64))
        p = abi.RenderParams()
        p.n_colors = int(colors.size)
        p.precision = int(precision)
        p.colors_nm = colors.ctypes.data_as(C.POINTER(C.c_double))
        p.max_dt_scale = float(max_dt_scale)
        p.integrator = int(integrator)
        p.ray_bundles = int(bool(ray_bundles))
        p.promote_dr = float(promote_dr)
        p.promote_sin = float(promote_sin)
        p.block_warps = int(block_warps)
        p.ctas_per_sm = int(ctas_per_sm)
        p.stream = stream
        p.pixel_order = int(pixel_order)
        p.trace_ray = int(trace_ray)
        p.refill_min = int(refill_min)
        p.autotune = int(bool(autotune))
        p.graph = int(bool(graph))
        p.tail_pass = 0 if tail_pass else -1
        keep = [colors]
        for k, tex in enumerate(skybox):
            if tex is None:
                continue
            t = np.ascontiguousarray(np.asarray(tex, dtype=np.float32))
            h = t.shape[0] // 3
            if t.ndim != 3 or t.shape != (3 * h, 4 * h, 3) or h < 1:
                raise ValueError("a skybox is a float32 array [3 h, 4 h, 3]")
            p.skybox[k] = t.ctypes.data_as(C.POINTER(C.c_float))
            p.skybox_h[k] = h
            keep.append(t)
        if gaunt_lut is not None:  # the bremsstrahlung torus's Gaunt-factor table
            t = np.ascontiguousarray(np.asarray(gaunt_lut, dtype=np.float32))
            if t.shape != (abi.GAUNT_ROWS, abi.GAUNT_COLS):
                raise ValueError(f"gaunt_lut is a float32 array [{abi.GAUNT_ROWS}, {abi.GAUNT_COLS}]")
            p.gaunt_lut = t.ctypes.data_as(C.POINTER(C.c_float))
            keep.append(t)
        p._keep = keep  # keep the arrays alive with the struct
        return p

    def render_raw(self, scene: abi.Scene, cams, params: abi.RenderParams, outputs: abi.Outputs) -> None:
        """rtw_render with caller-provided output pointers (host or device)."""
        cams = list(cams)
        arr = (abi.Camera * len(cams))(*cams)
        st = self._lib.rtw_render(self._ctx, C.byref(scene), arr, len(cams), C.byref(params), C.byref(outputs))
        abi.check(st, self.last_error())

    def render(self, scene: abi.Scene, cams, colors_nm, *, want=("xyz", "class", "steps"), **kw) -> dict:
        """Renders frames into new host numpy arrays; returns a dict of arrays
        indexed by global pixel (frames concatenated, pixel i + x_pix * j; a
        windowed camera contributes its window's pixels, i + win_w * j)."""
        cams = list(cams)
        total = 0
        for c in cams:
            total += abi.camera_pixels(c)
        n = len(np.atleast_1d(colors_nm))
        res = {}
        out = abi.Outputs()
        if "xyz" in want:
            res["xyz"] = np.zeros((total, 3), np.float32)
            out.xyz = res["xyz"].ctypes.data
        if "class" in want:
            res["class"] = np.zeros(total, np.uint8)
            out.term_class = res["class"].ctypes.data
        if "steps" in want:
            res["steps"] = np.zeros(total, np.uint32)
            out.steps = res["steps"].ctypes.data
        if "spectrum" in want:
            res["spectrum"] = np.zeros((total, n), np.float32)
            out.spectrum = res["spectrum"].ctypes.data
        if "state" in want:
            res["state"] = np.zeros((total, 8), np.float64)
            out.final_state = res["state"].ctypes.data
        if "tau" in want:
            res["tau"] = np.zeros(total, np.float32)
            out.tau = res["tau"].ctypes.data
        if kw.get("trace_ray", -1) >= 0:
            cap = int(kw.pop("trace_capacity", 20000))
            res["trace"] = np.zeros((cap, abi.TRACE_FIELDS))
            out.trace = res["trace"].ctypes.data
            out.trace_capacity = cap
        kw.pop("trace_capacity", None)
        out.on_device = 0
        self.render_raw(scene, cams, self.params(colors_nm, **kw), out)
        return res

    def stats(self) -> dict:
        s = abi.Stats()
        abi.check(self._lib.rtw_get_stats(self._ctx, C.byref(s)), self.last_error())
        d = {f: getattr(s, f) for f, _ in abi.Stats._fields_}
        d["phase_cycles"] = list(s.phase_cycles)
        return d

    def adjoint(self, scene: abi.Scene, cam: abi.Camera, colors_nm, target, *, precision=abi.PREC_MIXED,
                checkpoint_every: int = 16, camera_delta: float = 0.0, want=("spectrum",), per_ray: bool = False,
                exclude_escape_rays: bool = False, rays=(0, 0, 1), **kw) -> dict:
        """Loss sum (I - target)^2 of a synchrotron-torus render and its gradient
        in (spin, inclination, n_e0, b_0, theta_e0) through rtw_adjoint.
        target: [P, n_colors] float32 (host array or a CUDA tensor).
        rays = (begin, count, stride): the pixel subset (count 0: to the end)."""
        P = abi.camera_pixels(cam)
        n = len(np.atleast_1d(colors_nm))
        ap = abi.AdjointParams()
        on_dev = hasattr(target, "data_ptr")
        if on_dev:
            ap.target = target.data_ptr()
            ap.target_on_device = 1
        else:
            tgt = np.ascontiguousarray(target, dtype=np.float32).reshape(P, n)
            ap.target = tgt.ctypes.data
            ap.target_on_device = 0
        ap.checkpoint_every = int(checkpoint_every)
        ap.camera_delta = float(camera_delta)
        ap.escape_rays = int(bool(exclude_escape_rays))
        ap.ray_begin, ap.ray_count, ap.ray_stride = (int(v) for v in rays)
        res = {}
        if per_ray:
            res["per_ray_grad"] = np.zeros((P, 5))
            ap.per_ray_grad = res["per_ray_grad"].ctypes.data
        out = abi.Outputs()
        if "spectrum" in want:
            res["spectrum"] = np.zeros((P, n), np.float32)
            out.spectrum = res["spectrum"].ctypes.data
        if "class" in want:
            res["class"] = np.zeros(P, np.uint8)
            out.term_class = res["class"].ctypes.data
        if "steps" in want:
            res["steps"] = np.zeros(P, np.uint32)
            out.steps = res["steps"].ctypes.data
        out.on_device = 0
        kw.setdefault("integrator", abi.DP45_FSAL)
        prm = self.params(colors_nm, precision=precision, **kw)
        r = abi.AdjointResult()
        st = self._lib.rtw_adjoint(self._ctx, C.byref(scene), C.byref(cam), C.byref(prm), C.byref(ap), C.byref(out),
                                   C.byref(r))
        abi.check(st, self.last_error())
        res.update({f: getattr(r, f) for f, _ in abi.AdjointResult._fields_ if f != "grad"})
        res["grad"] = np.array(list(r.grad))
        return res

    def frame_times(self, n_frames: int) -> dict:
        """Per-frame times of the last render (ms, device global timer):
        'done' = batch start to the frame's last ray, 'span' = the frame's
        first ray start to its last ray end."""
        done = np.zeros(n_frames)
        span = np.zeros(n_frames)
        dp = done.ctypes.data_as(C.POINTER(C.c_double))
        sp = span.ctypes.data_as(C.POINTER(C.c_double))
        abi.check(self._lib.rtw_get_frame_times(self._ctx, int(n_frames), dp, sp), self.last_error())
        return {"done": done, "span": span}

    def op_counts(self, kind: int) -> dict:
        return abi.op_counts(kind)

    def measure_peaks(self) -> dict:
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        abi.check(self._lib.rtw_measure_peaks(self._ctx, C.byref(a), C.byref(b), C.byref(c)), self.last_error())
        return {"fp32_flops": a.value, "fp64_flops": b.value, "mufu_ops": c.value}


# ---------------------------------------------------------------------------
# The reference's world/scene selection and render call
# ---------------------------------------------------------------------------

@dataclass
class World:
    scene: abi.Scene
    position: list
    direction: list
    pointing: list
    beta: float


_WORLDS = {
    # initialization.jl:80-89
    "schwarzschild_t,r,θ,ϕ_simpledisk": (abi.SCENE_SCHWARZSCHILD_DISK, [0, 25, PI / 3, 0], [PI / 2, 0],
                                          [0.0, 0.0, -PI / 2], 0.0),
    # initialization.jl:90-99
    "kerr_boyer_lindquist": (abi.SCENE_KERR_DISK, [0, 25, 0.52 * PI, 0], [PI / 2, 0], [0.0, 0.0, -PI / 2], 0.0),
    # initialization.jl:110-119
    "minkowski_t,r,θ,ϕ_sphere": (abi.SCENE_MINKOWSKI_SPHERE, [0, 4, PI / 2, 0], [PI / 2, 0],
                                 [0.0, 0.0, -PI / 2], 0.0),
    # initialization.jl:100-109 (Powehi.source, the M87* model)
    "m87": (abi.SCENE_KERR_POWEHI, [0, 35, 0.3, 0], [PI / 2, PI / 6], [0.0, 0.0, PI], 0.0),
    # initialization.jl:120-128 (Synchro_Test.source, Cartesian t, x, y, z)
    "synch": (abi.SCENE_SYNCHRO_TEST, [0.0, 0.0, 0.0, 0.0], [0.0, 0.0], [PI / 8, 0.0, PI], 0.0),
    # initialization.jl:140-148 (Wormhole.source, coordinates t, l, theta, phi)
    "wormhole": (abi.SCENE_WORMHOLE, [0, 5, PI / 2, 0], [PI / 2, 0], [0.0, 0.0, -PI / 2], 0.0),
    # initialization.jl:130-138 (Minkowski_Sphere_Cartesian.source, Cartesian t, x, y, z)
    "minkowski_t,x,y,z_sphere": (abi.SCENE_MINKOWSKI_CART_SPHERE, [0.0, 0.0, 0.0, -4.0], [0.0, 0.0],
                                 [0.0, 0.0, 0.0], 0.0),
}

_current: World | None = None
_renderer: Renderer | None = None
_textures = (None, None)


def load_textures(skybox1=None, skybox2=None):
    """The skybox worlds' textures (load_textures, Wormhole.source/ and
    Minkowski_Sphere_Cartesian.source/source_model.jl): cube maps in the
    reference's cross layout, float32 [3 h, 4 h, 3] RGB in [0, 1], row 0 at the
    top. The wormhole's skybox1 lies beyond the throat's positive-l side; the
    Cartesian sphere uses skybox1 only. gen_image uses them until they are
    replaced."""
    global _textures
    _textures = (skybox1, skybox2)
    return _textures


def available_worlds() -> list:
    return sorted(_WORLDS)


def initialize_world(input_string: str):
    """Selects a scene and returns its default (position, direction, pointing, beta)
    (initialization.jl:78-172). The skybox worlds ("wormhole",
    "minkowski_t,x,y,z_sphere") take their textures from load_textures."""
    global _current
    key = input_string.lower()
    if key not in _WORLDS:
        raise ValueError(f"unknown or unsupported world {input_string!r}; available: {available_worlds()}")
    kind, pos, d, pt, beta = _WORLDS[key]
    _current = World(abi.scene_default(kind), list(pos), list(d), list(pt), beta)
    return list(pos), list(d), list(pt), beta


def set_scene(scene: abi.Scene) -> None:
    """Selects an explicit scene (runtime parameters instead of a .source folder)."""
    global _current
    _current = World(scene, [0, 0, 0, 0], [0, 0], [0, 0, 0], 0.0)


def _get_renderer() -> Renderer:
    global _renderer
    if _renderer is None:
        _renderer = Renderer(0)
    return _renderer


def gen_image(*, camera_pos=(0, 0, 0, 0), camera_dir=(0.0, 0.0), speed=0.0, camera_point=(0.0, 0.0, 0.0),
              x_pix=100, max_steps=1e3, colors=(400, 550, 700), returnrays=False, tolerance=1e-4,
              max_dt_scale=1e-1, fov_hor=85, fov_vert=60, print_num_pix=False, ray_bundles=False,
              precision="fp64", integrator="ref_compat", renderer: Renderer | None = None):
    """The reference's gen_image (LttM.jl:104-209 / 5P.jl:135-282) on the B200.

    Returns the linear XYZ image [y_pix, x_pix, 3] in the reference's orientation
    (transpose(reverse(img, dims=2))), and with ``returnrays`` also the final
    ray states [x_pix, y_pix, 8 + 2 len(colors)] in the reference's layout
    (t, r, theta, phi, k^t, k^r, k^theta, k^phi, I_1, tau_1, I_2, tau_2, ...).
    A camera on a coordinate singularity raises abi.RTWError(RTW_ERR_INVALID_CAMERA)
    (the reference prints and returns a blank image, 5P.jl:140-143)."""
    if _current is None:
        raise RuntimeError("call initialize_world(name) or set_scene(scene) first")
    r = renderer or _get_renderer()
    cam = abi.make_camera(camera_pos, camera_dir, speed, camera_point, int(x_pix), fov_hor, fov_vert,
                          tolerance, int(max_steps))
    if print_num_pix:
        print("Number of Pixels ", cam.x_pix * cam.y_pix)
    prec = {"fp64": abi.PREC_FP64, "mixed": abi.PREC_MIXED, "fp64_plain": abi.PREC_FP64_PLAIN}[precision]
    integ = {"ref_compat": abi.DP45_REF_COMPAT, "fsal": abi.DP45_FSAL}[integrator]
    want = ("xyz", "class", "steps") + (("spectrum", "state", "tau") if returnrays else ())
    sky = _textures if _current.scene.kind in (abi.SCENE_WORMHOLE, abi.SCENE_MINKOWSKI_CART_SPHERE) else (None, None)
    res = r.render(_current.scene, [cam], colors, want=want, precision=prec, integrator=integ,
                   max_dt_scale=max_dt_scale, ray_bundles=ray_bundles, skybox=sky)
    xp, yp = cam.x_pix, cam.y_pix
    img = res["xyz"].reshape(yp, xp, 3)[::-1].copy()
    if not returnrays:
        return img
    n = len(np.atleast_1d(colors))
    rays = np.zeros((xp, yp, 8 + 2 * n))
    st = res["state"].reshape(yp, xp, 8).transpose(1, 0, 2)
    rays[:, :, :8] = st
    rays[:, :, 8::2] = res["spectrum"].reshape(yp, xp, n).transpose(1, 0, 2)
    rays[:, :, 9::2] = res["tau"].reshape(yp, xp, 1).transpose(1, 0, 2)
    return img, rays


def xyz_to_srgb(xyz: np.ndarray) -> np.ndarray:
    """Informational: brightness-normalised sRGB of a linear XYZ image in the way
    gen_image finishes (Y scaled to [0, max Y], then XYZ -> sRGB, D65)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    ymax = np.nanmax(xyz[..., 1]) if xyz.size else 0.0
    if not ymax > 0:
        return np.zeros_like(xyz)
    x = xyz / ymax
    m = np.array([[3.2404542, -1.5371385, -0.4985314], [-0.9692660, 1.8760108, 0.0415560],
                  [0.0556434, -0.2040259, 1.0572252]])
    lin = np.clip(x @ m.T, 0, 1)
    return np.where(lin <= 0.0031308, 12.92 * lin, 1.055 * np.power(lin, 1 / 2.4) - 0.055)
