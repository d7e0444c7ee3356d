"""rtw_render_noalloc: the entry point for callers that cannot allocate device
memory (a host that owns all device memory up front, a real-time loop that
must not enter the allocator, code without an rtw_ctx). It keeps its scratch
in the library's own __device__ arrays; here its outputs must match those of
rtw_render on the same inputs, on two calls in a row (the second call reuses
the arrays the first one left behind), and requests beyond its fixed limits
must be refused. Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from rtwca_b200 import abi, configs

pytestmark = pytest.mark.gpu


def _device_outputs(torch, P, n_bins=0):
    dev = torch.device("cuda", 0)
    t = {"xyz": torch.zeros((P, 3), dtype=torch.float32, device=dev),
         "class": torch.zeros(P, dtype=torch.uint8, device=dev),
         "steps": torch.zeros(P, dtype=torch.int32, device=dev)}
    out = abi.Outputs()
    out.xyz, out.term_class, out.steps, out.on_device = (t["xyz"].data_ptr(), t["class"].data_ptr(),
                                                         t["steps"].data_ptr(), 1)
    if n_bins:
        t["spectrum"] = torch.zeros((P, n_bins), dtype=torch.float32, device=dev)
        out.spectrum = t["spectrum"].data_ptr()
    return t, out


def _host(t):
    return {k: v.cpu().numpy() for k, v in t.items()}


@pytest.mark.parametrize("name,x_pix,prec", [("kerr_thin_disk", 48, abi.PREC_MIXED),
                                             ("schwarzschild_disk", 32, abi.PREC_FP64)])
def test_noalloc_matches_rtw_render_twice(renderer, name, x_pix, prec):
    torch = pytest.importorskip("torch")
    lib = abi.load()
    scene, cam, colors = configs.workload(name, x_pix=x_pix)
    P = cam.x_pix * cam.y_pix
    params = renderer.params(colors, precision=prec)
    t_ref, out_ref = _device_outputs(torch, P)
    renderer.render_raw(scene, [cam], params, out_ref)
    torch.cuda.synchronize()
    ref = _host(t_ref)
    cams = (abi.Camera * 1)(cam)
    for call in range(2):
        t, out = _device_outputs(torch, P)
        st = lib.rtw_render_noalloc(C.byref(scene), cams, 1, C.byref(params), C.byref(out))
        assert st == abi.OK, lib.rtw_noalloc_last_error()
        torch.cuda.synchronize()
        got = _host(t)
        assert np.array_equal(got["class"], ref["class"]), call
        assert np.array_equal(got["steps"], ref["steps"]), call
        assert np.allclose(got["xyz"], ref["xyz"], rtol=1e-6, atol=0), call


def test_noalloc_several_cameras_capped_grid(renderer):
    """Three cameras of different sizes, positions and tolerances in one call,
    128 bins in FP64: one 4-warp CTA then needs 256 KB of spectral scratch, so
    the fixed scratch holds fewer CTAs than the GPU has SMs and the grid is
    capped by it (the launch shape only this entry point has). Spectra,
    classes and step counts must equal rtw_render's, on two calls in a row."""
    torch = pytest.importorskip("torch")
    lib = abi.load()
    scene, cam, _ = configs.workload("schwarzschild_disk", x_pix=24)
    colors = configs.log_spaced_colors(128)
    per_cta = 2 * 32 * 128 * 8 * 4
    assert abi.NOALLOC_SCRATCH_BYTES // per_cta < torch.cuda.get_device_properties(0).multi_processor_count
    far = list(cam.position)
    far[1] = 40.0
    cams = [cam,
            abi.make_camera(far, list(cam.direction), cam.speed, list(cam.pointing), 16, cam.fov_hor, cam.fov_vert,
                            1e-6, cam.max_steps),
            abi.make_camera(list(cam.position), list(cam.direction), cam.speed, list(cam.pointing), 20, 30.0, 20.0,
                            1e-7, cam.max_steps)]
    P = sum(c.x_pix * c.y_pix for c in cams)
    params = renderer.params(colors, precision=abi.PREC_FP64)
    t_ref, out_ref = _device_outputs(torch, P, 128)
    renderer.render_raw(scene, cams, params, out_ref)
    torch.cuda.synchronize()
    ref = _host(t_ref)
    carr = (abi.Camera * 3)(*cams)
    for call in range(2):
        t, out = _device_outputs(torch, P, 128)
        st = lib.rtw_render_noalloc(C.byref(scene), carr, 3, C.byref(params), C.byref(out))
        assert st == abi.OK, lib.rtw_noalloc_last_error()
        torch.cuda.synchronize()
        got = _host(t)
        assert np.array_equal(got["class"], ref["class"]), call
        assert np.array_equal(got["steps"], ref["steps"]), call
        assert np.allclose(got["spectrum"], ref["spectrum"], rtol=1e-6, atol=0), call
        assert np.allclose(got["xyz"], ref["xyz"], rtol=1e-6, atol=0), call


def test_noalloc_refuses_context_features(renderer):
    """graph capture, the autotuner and the step trace keep state in an
    rtw_ctx; without one they are refused, not silently ignored."""
    torch = pytest.importorskip("torch")
    lib = abi.load()
    scene, cam, colors = configs.workload("kerr_thin_disk", x_pix=8)
    t, out = _device_outputs(torch, 64)
    for kw in ({"graph": True}, {"autotune": True}, {"trace_ray": 0}):
        params = renderer.params(colors, precision=abi.PREC_MIXED, **kw)
        st = lib.rtw_render_noalloc(C.byref(scene), (abi.Camera * 1)(cam), 1, C.byref(params), C.byref(out))
        assert st == abi.ERR_UNSUPPORTED and b"rtw_ctx" in lib.rtw_noalloc_last_error(), kw


def test_noalloc_refuses_beyond_limits(renderer):
    torch = pytest.importorskip("torch")
    lib = abi.load()
    scene, cam, colors = configs.workload("kerr_thin_disk", x_pix=8)
    params = renderer.params(colors, precision=abi.PREC_MIXED)
    t, out = _device_outputs(torch, 64)
    many = (abi.Camera * (abi.NOALLOC_MAX_FRAMES + 1))(*([cam] * (abi.NOALLOC_MAX_FRAMES + 1)))
    st = lib.rtw_render_noalloc(C.byref(scene), many, abi.NOALLOC_MAX_FRAMES + 1, C.byref(params), C.byref(out))
    assert st == abi.ERR_INVALID_PARAM and b"RTW_NOALLOC_MAX_FRAMES" in lib.rtw_noalloc_last_error()
    host = abi.Outputs()
    host.on_device = 0
    st = lib.rtw_render_noalloc(C.byref(scene), (abi.Camera * 1)(cam), 1, C.byref(params), C.byref(host))
    assert st == abi.ERR_INVALID_PARAM and b"device output" in lib.rtw_noalloc_last_error()
