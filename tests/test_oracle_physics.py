"""Known-answer pins of the CPU oracle (which has no golden vectors from the
reference itself: the reference's tests are timing runs). Each check is an
analytic property of the geodesic or radiative-transfer problem the
reference's integrator solves.

The pins run the oracle's textbook-FSAL Dormand-Prince mode: the reference's
own step (k1 of the next step = sum b_i k_i of the last one, not f(y)) is not a
convergent 5th-order method - its embedded error estimate shares the stale k1
and cannot see the error it makes - so its results drift from the analytic
answers by 1e-4..1e-2 whatever the tolerance (see the last tests). Everything
else (camera, metric, Christoffel symbols, emitter, radiative transfer, CIE
tables, step controller, termination) is shared by both modes."""
import math

import numpy as np
import pytest

from rtwca_b200 import abi, configs

E_SCALE = 2 * 6.62607015e-34 * 299792458.0 * 1e27
F_FACTOR = 6.62607015e-34 * 299792458.0 * 1e9 / 1.380649e-23


def planck_over_nu3(lam_nm, T):
    """B_nu(T) / nu^3 in the reference's units (calc_planck, nu in nm^-1)."""
    return E_SCALE / (np.exp(F_FACTOR / lam_nm / T) - 1)


def test_constants(oracle):
    e, f = oracle.constants()
    assert e == pytest.approx(E_SCALE, rel=1e-15)
    assert f == pytest.approx(F_FACTOR, rel=1e-15)
    assert f == pytest.approx(1.438776877e7, rel=1e-9)  # second radiation constant in nm K


def cart(x):
    """Cartesian position and velocity of a flat-space state (t, r, th, ph, k)."""
    r, th, ph = x[1], x[2], x[3]
    vr, vth, vph = x[5], x[6], x[7]
    st, ct, sp, cp = math.sin(th), math.cos(th), math.sin(ph), math.cos(ph)
    pos = np.array([r * st * cp, r * st * sp, r * ct])
    vel = np.array([vr * st * cp + r * ct * cp * vth - r * st * sp * vph,
                    vr * st * sp + r * ct * sp * vth + r * st * cp * vph,
                    vr * ct - r * st * vth])
    return pos, vel


def test_flat_space_rays_are_straight_lines(oracle):
    FSAL = abi.DP45_FSAL
    """Minkowski without emitter: every ray ends on the straight line it started on."""
    scene = configs.minkowski_sphere_scene(a_nu=0.0)
    cam = configs.look_at_camera(10.0, math.pi / 2, 60.0, 12, 1e-8)
    colors = configs.log_spaced_colors(2)
    rays = oracle.camera_rays(scene, cam)
    res = oracle.render(scene, cam, colors, integrator=FSAL)
    assert np.all(res["class"] == abi.CLASS_ESCAPE)
    n = 0
    for x0, x1 in zip(rays, res["state"]):
        p0, v0 = cart(x0)
        p1, v1 = cart(x1)
        if np.linalg.norm(np.cross(p0, v0)) / np.linalg.norm(v0) < 0.05:
            # passes within 0.05 of the origin: crosses the coordinate
            # singularity with the reference's Euler escape (first order)
            continue
        n += 1
        u0 = v0 / np.linalg.norm(v0)
        u1 = v1 / np.linalg.norm(v1)
        assert np.allclose(u0, u1, atol=1e-8)
        d = p1 - p0
        assert np.linalg.norm(d - (d @ u0) * u0) < 1e-6 * np.linalg.norm(d)
    assert n > 120


def killing(oracle, scene, x):
    g = oracle.metric(scene, x)
    kl = g @ x[4:]
    return -kl[0], kl[3], kl[2], g


@pytest.mark.parametrize("kind", ["schwarzschild", "kerr"])
def test_null_norm_and_constants_of_motion(oracle, kind):
    """g k k = 0, E = -k_t and L_z = k_phi conserved; Kerr: Carter constant."""
    if kind == "kerr":
        scene = configs.kerr_disk_scene(a_nu=0.0)
        scene.r_in, scene.r_out = 50.0, 40.0  # no emitter
    else:
        scene = configs.schwarzschild_disk_scene(a_nu=0.0)
        scene.r_in, scene.r_out = 50.0, 40.0
    cam = configs.look_at_camera(30.0, math.radians(70.0), 40.0, 10, 1e-8)
    colors = configs.log_spaced_colors(2)
    rays = oracle.camera_rays(scene, cam)
    res = oracle.render(scene, cam, colors, integrator=abi.DP45_FSAL)
    a = scene.spin if kind == "kerr" else 0.0
    checked = 0
    for x0, x1, c in zip(rays, res["state"], res["class"]):
        if c != abi.CLASS_ESCAPE:
            continue
        E0, L0, kth0, g0 = killing(oracle, scene, x0)
        if abs(L0) < 1e-2 * E0:
            continue  # near-axis ray: crosses the pole with the reference's Euler escape
        E1, L1, kth1, g1 = killing(oracle, scene, x1)
        k1 = x1[4:]
        assert abs(k1 @ g1 @ k1) < 1e-6 * E1 * E1
        assert E1 == pytest.approx(E0, rel=1e-7)
        assert L1 == pytest.approx(L0, rel=1e-6, abs=1e-8 * E0)
        Q0 = kth0 ** 2 + math.cos(x0[2]) ** 2 * (L0 ** 2 / math.sin(x0[2]) ** 2 - a * a * E0 ** 2)
        Q1 = kth1 ** 2 + math.cos(x1[2]) ** 2 * (L1 ** 2 / math.sin(x1[2]) ** 2 - a * a * E1 ** 2)
        assert Q1 == pytest.approx(Q0, rel=1e-5, abs=1e-8 * E0 * E0 * 30 * 30)
        checked += 1
    assert checked > 40


def test_schwarzschild_shadow_edge(oracle):
    """Rays with impact parameter b < 3 sqrt(3) M fall in; b > 3 sqrt(3) M escape."""
    scene = configs.schwarzschild_disk_scene(a_nu=0.0)
    scene.r_in, scene.r_out = 50.0, 40.0
    cam = configs.look_at_camera(50.0, math.pi / 2, 30.0, 24, 1e-8)
    colors = configs.log_spaced_colors(2)
    rays = oracle.camera_rays(scene, cam)
    res = oracle.render(scene, cam, colors, integrator=abi.DP45_FSAL)
    bc = 3 * math.sqrt(3.0)
    n_in = n_out = 0
    for x0, c in zip(rays, res["class"]):
        E, Lz, kth, g = killing(oracle, scene, x0)
        L2 = kth ** 2 + Lz ** 2 / math.sin(x0[2]) ** 2
        b = math.sqrt(L2) / E
        if b < bc * (1 - 2e-3):
            assert c == abi.CLASS_HORIZON, b
            n_in += 1
        elif b > bc * (1 + 2e-3):
            assert c == abi.CLASS_ESCAPE, b
            n_out += 1
    assert n_in > 10 and n_out > 100


def test_opaque_blackbody_sphere(oracle):
    """Static emitter, static camera, flat space (g = 1): a ray that stops in the
    opaque sphere carries I_nu/nu^3 = B_nu(T)/nu^3 (1 - exp(-tau))."""
    scene = configs.minkowski_sphere_scene(a_nu=100.0)
    cam = configs.look_at_camera(10.0, math.pi / 2, 20.0, 10, 1e-8)
    colors = configs.log_spaced_colors(8)
    res = oracle.render(scene, cam, colors, integrator=abi.DP45_FSAL)
    hit = res["class"] == abi.CLASS_THICK
    assert hit.sum() >= 4
    expect = planck_over_nu3(colors, scene.temperature)[None, :] * (1 - np.exp(-res["tau"][hit]))
    assert np.allclose(res["spectrum"][hit], expect, rtol=2e-6)
    # and tau reached the reference's stop -log(tol)
    assert np.all(res["tau"][hit] >= -math.log(1e-8))


def test_uniform_slab_transfer(oracle):
    """Optically thin uniform sphere: tau = a_nu x chord, I = B/nu^3 (1 - e^-tau)."""
    a_nu = 0.7
    scene = configs.minkowski_sphere_scene(a_nu=a_nu)
    cam = configs.look_at_camera(10.0, math.pi / 2, 16.0, 10, 1e-9)
    colors = configs.log_spaced_colors(4)
    rays = oracle.camera_rays(scene, cam)
    res = oracle.render(scene, cam, colors, integrator=abi.DP45_FSAL)
    n = 0
    for x0, tau, spec, c in zip(rays, res["tau"], res["spectrum"], res["class"]):
        r, th = x0[1], x0[2]
        L = r * r * math.sqrt(x0[6] ** 2 + math.sin(th) ** 2 * x0[7] ** 2)
        b = L / x0[4]
        if b < 0.98:
            chord = 2 * math.sqrt(1 - b * b)
            assert c == abi.CLASS_ESCAPE
            assert tau[0] == pytest.approx(a_nu * chord, rel=1e-6)
            assert np.allclose(spec, planck_over_nu3(colors, scene.temperature) * (1 - np.exp(-tau)), rtol=1e-6)
            n += 1
        elif b > 1.02:
            assert tau[0] == 0 and np.all(spec == 0)
    assert n >= 8


def test_cie_fit_values(oracle):
    """color_theory.jl:11-61 evaluated directly."""
    m = np.array([[0.362, 1.056, -0.065, 0.821, 0.286, 1.217, 0.681],
                  [442.0, 599.8, 501.1, 568.8, 530.9, 437.0, 459.0],
                  [0.0624, 0.0264, 0.0490, 0.0213, 0.0613, 0.0845, 0.0385],
                  [0.0374, 0.0323, 0.0382, 0.0247, 0.0322, 0.0278, 0.0725]])

    def lobes(wl, idx):
        s = 0.0
        for i in idx:
            d = wl - m[1, i]
            w = m[3, i] if d >= 0 else m[2, i]
            s += m[0, i] * math.exp(-0.5 * (d * w) ** 2)
        return s

    for wl in (380.0, 442.0, 500.0, 555.0, 599.8, 650.0, 720.0):
        assert oracle.cie_eval(0, wl) == pytest.approx(lobes(wl, [0, 1, 2]), rel=1e-14)
        assert oracle.cie_eval(1, wl) == pytest.approx(lobes(wl, [3, 4]), rel=1e-14)
        assert oracle.cie_eval(2, wl) == pytest.approx(lobes(wl, [5, 6]), rel=1e-14)
    # uniform colors: the reference's trapezoid weights (color_theory.jl:79-91)
    colors = np.arange(350.0, 751.0, 30.0)
    wx, wy, wz, fac = oracle.cie(colors)
    step = np.full(colors.size, 30.0)
    step[0] /= 2
    step[-1] /= 2
    assert np.allclose(wy, [lobes(c, [3, 4]) * s for c, s in zip(colors, step)], rtol=1e-14)
    assert np.allclose(fac, (1 / colors) ** 3 * 299792458.0 / colors ** 2, rtol=1e-14)


def test_reference_step_drifts_fsal_converges(oracle):
    """Characterises the reference's step: with the carried average slope the
    null condition drifts by ~1e-3 at tol 1e-8; textbook FSAL keeps it at the
    tolerance level with fewer steps."""
    scene = configs.schwarzschild_disk_scene(a_nu=0.0)
    scene.r_in, scene.r_out = 50.0, 40.0
    cam = configs.look_at_camera(30.0, math.radians(70.0), 40.0, 8, 1e-8)
    colors = configs.log_spaced_colors(2)
    drift = {}
    steps = {}
    for integ in (abi.DP45_REF_COMPAT, abi.DP45_FSAL):
        res = oracle.render(scene, cam, colors, integrator=integ)
        nn = []
        for x1, c in zip(res["state"], res["class"]):
            if c == abi.CLASS_ESCAPE:
                g = oracle.metric(scene, x1)
                nn.append(abs(x1[4:] @ g @ x1[4:]))
        drift[integ] = max(nn)
        steps[integ] = int(res["steps"].sum())
    assert drift[abi.DP45_FSAL] < 1e-7
    assert drift[abi.DP45_REF_COMPAT] > 1e-5
    assert steps[abi.DP45_FSAL] < steps[abi.DP45_REF_COMPAT]


def test_reference_precision_switch(oracle):
    """The reference's CPU path computes Kerr Christoffel symbols in FP32
    (Kerr.source/source_geometry.jl:196-197). The oracle's switch reproduces
    it: escape and disk pixels keep their class, but near the horizon the
    radial acceleration (O(1/Delta) terms that cancel to O(1)) loses every
    digit in FP32, and rays that fall in end as max-steps, NaN or winding
    (frame dragging while stuck) instead of
    reaching the (1 + 10 tol) r+ stop."""
    scene = configs.kerr_disk_scene()
    cam = configs.look_at_camera(50.0, math.radians(80.0), 45.0, 10, 1e-8)
    colors = configs.log_spaced_colors(4)
    a = oracle.render(scene, cam, colors, integrator=abi.DP45_FSAL)
    scene.ref_precision = 1
    b = oracle.render(scene, cam, colors, integrator=abi.DP45_FSAL)
    far = a["class"] != abi.CLASS_HORIZON
    assert np.mean(a["class"][far] == b["class"][far]) >= 0.97
    fell = a["class"] == abi.CLASS_HORIZON
    assert fell.sum() >= 2
    assert np.all(np.isin(b["class"][fell], [abi.CLASS_HORIZON, abi.CLASS_MAXSTEPS, abi.CLASS_NAN, abi.CLASS_WINDING]))
    same = (a["class"] == b["class"]) & far
    ya, yb = a["xyz"][same, 1], b["xyz"][same, 1]
    den = np.maximum(np.abs(ya), 1e-6 * np.abs(ya).max())
    assert np.quantile(np.abs(ya - yb) / den, 0.9) < 1e-3
