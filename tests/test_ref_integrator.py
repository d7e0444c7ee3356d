"""The C++ oracle's step loop against the independent Python restatement of
the reference's integrate_ray / RKDP_Step_w_buffer! (tests/ref_integrator.py),
both modes, on single rays of each scene."""
import math

import numpy as np
import pytest

from rtwca_b200 import abi, configs
from tests import ref_integrator


@pytest.mark.parametrize("name,pixels", [
    ("schwarzschild_disk", [0, 27, 45, 55, 63]),
    ("kerr_thin_disk", [12, 44, 45, 54, 77]),
    ("minkowski_sphere", [0, 136, 119]),
])
@pytest.mark.parametrize("integ", [abi.DP45_REF_COMPAT, abi.DP45_FSAL])
def test_step_loop_matches_python_restatement(oracle, name, pixels, integ):
    scene, cam, _ = configs.workload(name, x_pix=10 if name != "minkowski_sphere" else 16)
    cam.tolerance = 1e-6  # fewer steps for the Python loop
    colors = configs.log_spaced_colors(2)
    rays = oracle.camera_rays(scene, cam)
    ref = oracle.render(scene, cam, colors, integrator=integ, pixel_ids=pixels)
    for q, pid in enumerate(pixels):
        ray0 = np.zeros(8 + 2 * colors.size)
        ray0[:8] = rays[pid]
        c, steps, ray = ref_integrator.integrate_ray(oracle, scene, colors, ray0, cam.tolerance, cam.max_steps,
                                                     fsal=integ == abi.DP45_FSAL)
        assert c == ref["class"][q], (pid, c, ref["class"][q])
        assert steps == ref["steps"][q], (pid, steps, ref["steps"][q])
        # (rays that end at the horizon are ill-conditioned there: k^t ~ 1/Delta)
        assert np.allclose(ray[:8], ref["state"][q], rtol=1e-7, atol=1e-12)
        assert np.allclose(ray[8::2], ref["spectrum"][q], rtol=1e-9, atol=1e-300)
