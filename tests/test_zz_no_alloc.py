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


def _device_outputs(torch, P):
    dev = torch.device("cuda", 0)
    t = {"xyz": torch.zeros((P, 3), dtype=torch.float32, device=dev),
         "class": torch.zeros(P, dtype=torch.uint8, device=dev),
         "steps": torch.zeros(P, dtype=torch.int32, device=dev)}
    out = abi.Outputs()
    out.xyz, out.term_class, out.steps, out.on_device = (t["xyz"].data_ptr(), t["class"].data_ptr(),
                                                         t["steps"].data_ptr(), 1)
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
