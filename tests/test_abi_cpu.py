"""The C ABI of librtw_b200.so without a GPU: every symbol of include/rtw.h is
exported, the ctypes structs match the C layout, and the host-side entry
points (scene defaults, camera set-up, CIE tables, the scene right-hand side)
agree with the oracle."""
import ctypes as C
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from rtwca_b200 import abi, configs
from tests.conftest import HAS_GPU, ROOT

HEADER = ROOT / "include" / "rtw.h"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:rtw_status|void|const char\*|int32_t)\s+(rtw_\w+)\(", text, re.M)))


def test_every_declared_symbol_is_exported(rtwlib):
    names = header_functions()
    assert len(names) >= 13
    lib = C.CDLL(str(abi.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), n
        assert n in abi.SIGNATURES, f"{n} has no ctypes binding"


def test_abi_version(rtwlib):
    assert rtwlib.rtw_abi_version() == abi.ABI_VERSION == 7


STRUCTS = {
    "rtw_scene": abi.Scene, "rtw_camera": abi.Camera, "rtw_render_params": abi.RenderParams,
    "rtw_outputs": abi.Outputs, "rtw_stats": abi.Stats, "rtw_op_counts": abi.OpCounts,
    "rtw_adjoint_params": abi.AdjointParams, "rtw_adjoint_result": abi.AdjointResult,
}


def test_struct_layouts_match_c(tmp_path):
    """Compile a C program against rtw.h and compare sizeof/offsetof with ctypes."""
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for cname, py in STRUCTS.items():
        assert int(got[f"{cname} size"]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


def test_scene_defaults_are_the_reference_constants(rtwlib):
    s = abi.scene_default(abi.SCENE_SCHWARZSCHILD_DISK)   # Schwarzschild ... source_model.jl:44-80
    assert (s.r_in, s.r_out, s.temperature, s.a_nu) == (6, 12, 5778, 1)
    assert s.theta_lo == pytest.approx(15 * math.pi / 32) and s.theta_hi == pytest.approx(17 * math.pi / 32)
    k = abi.scene_default(abi.SCENE_KERR_DISK)             # Kerr.source: spin 0.998f0, a_nu 1f-1
    assert k.spin == float(np.float32(0.998)) and k.a_nu == float(np.float32(0.1)) and k.r_out == 12
    m = abi.scene_default(abi.SCENE_MINKOWSKI_SPHERE)
    assert (m.r_out, m.temperature, m.a_nu, m.escape_radius) == (1, 5778, 1, 100)
    assert m.winding_limit == pytest.approx(8 * math.pi)
    with pytest.raises(abi.RTWError):
        abi.scene_default(17)


@pytest.mark.parametrize("x_pix,fh,fv,expect", [(500, 85, 60, 315), (256, 60, 60, 256), (1024, 45, 45, 1024),
                                                (7, 90, 53.13010235415598, 4)])
def test_camera_pixels_round_half_even(rtwlib, x_pix, fh, fv, expect):
    cam = abi.make_camera([0, 10, 1.0, 0], x_pix=x_pix, fov_hor=fh, fov_vert=fv)
    n = C.c_int64()
    abi.check(rtwlib.rtw_camera_pixels(C.byref(cam), C.byref(n)))
    assert cam.y_pix == expect == abi.y_pixels(x_pix, fh, fv)
    assert n.value == x_pix * expect


CAMERAS = [
    ("kerr_thin_disk", dict()),
    ("schwarzschild_disk", dict()),
    ("minkowski_sphere", dict()),
]


@pytest.mark.parametrize("name", ["kerr_thin_disk", "schwarzschild_disk", "minkowski_sphere", "kerr_thick_disk"])
def test_camera_rays_match_oracle(rtwlib, oracle, name):
    scene, cam, _ = configs.workload(name, x_pix=12)
    rays = np.zeros((cam.x_pix * cam.y_pix, 8))
    abi.check(rtwlib.rtw_camera_rays(C.byref(scene), C.byref(cam), rays.ctypes.data_as(C.POINTER(C.c_double)),
                                     rays.shape[0]))
    ref = oracle.camera_rays(scene, cam)
    assert np.allclose(rays, ref, rtol=1e-13, atol=1e-13)


def test_camera_rays_boosted_rotated(rtwlib, oracle):
    scene = configs.kerr_disk_scene()
    cam = abi.make_camera([0, 7.5, 1.2, 0.4], [1.1, 0.7], 0.6, [0.3, -0.2, 0.9], 9, 70, 50, 1e-6, 100)
    n = 9 * cam.y_pix
    rays = np.zeros((n, 8))
    abi.check(rtwlib.rtw_camera_rays(C.byref(scene), C.byref(cam), rays.ctypes.data_as(C.POINTER(C.c_double)), n))
    ref = oracle.camera_rays(scene, cam)
    assert np.allclose(rays, ref, rtol=1e-12, atol=1e-12)
    # every initial momentum is null
    for x in ref:
        g = oracle.metric(scene, x)
        k = x[4:]
        assert abs(k @ g @ k) < 1e-12 * (k[0] ** 2)


def test_cie_weights_match_oracle(rtwlib, oracle):
    for colors in (np.arange(350, 751, 30, dtype=float), configs.log_spaced_colors(64), np.array([550.0])):
        n = colors.size
        got = [np.zeros(n) for _ in range(4)]
        D = C.POINTER(C.c_double)
        abi.check(rtwlib.rtw_cie_weights(colors.ctypes.data_as(D), n, *[g.ctypes.data_as(D) for g in got]))
        ref = oracle.cie(colors)
        for g, r in zip(got, ref):
            assert np.allclose(g, r, rtol=1e-14, atol=0)


def test_scene_rhs_matches_oracle(rtwlib, oracle):
    """The kernel's own functors (factored Christoffel symbols, grey emitter
    numbers) against the oracle's literal calc_ray_derivative!."""
    rng = np.random.default_rng(0)
    colors = np.array([400.0, 500.0, 600.0, 700.0])
    for sc in (configs.minkowski_sphere_scene(), configs.schwarzschild_disk_scene(), configs.kerr_disk_scene(),
               configs.kerr_thick_disk_scene()):
        for t in range(150):
            r = rng.uniform(6, 20) if t % 3 == 0 else rng.uniform(2.5, 40)
            if sc.kind == abi.SCENE_MINKOWSKI_SPHERE and t % 3 == 0:
                r = rng.uniform(0.2, 1.0)
            th = rng.uniform(15 * np.pi / 32, 17 * np.pi / 32) if t % 2 else rng.uniform(0.05, np.pi - 0.05)
            st = np.array([0, r, th, 0.3, 1.2, rng.normal(), rng.normal() * 0.05, rng.normal() * 0.05,
                           rng.uniform(0, 3)])
            full = np.zeros(8 + 2 * colors.size)
            full[:8] = st[:8]
            full[9::2] = st[8]
            ref = oracle.rhs(sc, colors, full)
            g64, em = abi.scene_rhs(sc, st)
            g32, _ = abi.scene_rhs(sc, st, fp32=True)
            scale = np.abs(ref[:8]).max()
            assert np.abs(g64[:8] - ref[:8]).max() <= 1e-14 * scale
            assert np.abs(g32[:8] - ref[:8]).max() <= 1e-6 * scale
            assert g64[8] == pytest.approx(ref[9], rel=1e-13, abs=1e-300)
            for c, lam in enumerate(colors):
                kI = 0.0 if em[0] == 0 else -em[0] / (np.exp(em[1] / lam) - 1)
                assert kI == pytest.approx(ref[8 + 2 * c], rel=1e-11, abs=1e-300)


def test_op_counts(rtwlib):
    for k in range(4):
        oc = abi.op_counts(k)
        assert oc["rhs_vacuum"] > 10 and oc["rhs_emit"] >= oc["rhs_vacuum"] and oc["step_overhead"] > 100
    assert abi.op_counts(abi.SCENE_KERR_DISK)["rhs_vacuum"] > abi.op_counts(abi.SCENE_MINKOWSKI_SPHERE)["rhs_vacuum"]


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_create_without_device_fails_cleanly(rtwlib):
    ctx = C.c_void_p()
    st = rtwlib.rtw_create(C.byref(ctx), 0)
    assert st in (abi.ERR_NO_DEVICE, abi.ERR_CUDA)
    assert not ctx.value
    rtwlib.rtw_destroy(None)  # accepts NULL
    assert rtwlib.rtw_last_error(None) == b"null context"
