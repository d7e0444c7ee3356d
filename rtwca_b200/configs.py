"""The benchmark and parity workloads, as scenes + cameras + spectral grids.

All inputs are synthetic and analytic (no dataset is involved). The parameter
choices that the workload descriptions leave open are stated here:

* 64 log-spaced frequencies 3.7e14..8.6e14 Hz, passed as wavelengths in nm
  (the reference's ``colors``), ascending in wavelength.
* "Opaque" emitters (the blackbody sphere of ``minkowski_sphere`` and the thin
  blackbody disks) use a_nu = 100 per unit length, so a ray reaches the
  reference's optically-thick stop -log(tol) inside the emitter; the reference
  scenes' a_nu (1 and 0.1) leave them optically thin.
* Thin disks keep the reference Schwarzschild wedge half-opening pi/32 around
  the equator (Schwarzschild_Simple_Disk_Spherical.source/source_model.jl:74-75).
* ``kerr_thin_disk`` (the headline workload) is the Schwarzschild thin-disk
  scene with the metric replaced by Kerr a = 0.9: disk 6..20 M, 1e4 K.
* The thick disk uses a_nu(rho0) = 0.05 per M (optically thin) and the
  equatorial Keplerian velocity of radius r off the plane, as the reference's
  Kerr wedge disk does.
* Cameras look at the hole with the reference's default orientation
  (direction [pi/2, 0], pointing [0, 0, -pi/2], initialization.jl:110-119);
  "inclination i" places the camera at theta = i. max_dt_scale = 0.1 and
  max_steps = 1e4 as in the reference's test harness (initialization.jl:380-384).
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

PI = math.pi
C_LIGHT = 299792458.0


def log_spaced_colors(n: int = 64, f_lo: float = 3.7e14, f_hi: float = 8.6e14) -> np.ndarray:
    """n log-spaced frequencies in [f_lo, f_hi] Hz as wavelengths in nm, ascending."""
    f = np.exp(np.linspace(math.log(f_hi), math.log(f_lo), n))
    return C_LIGHT / f * 1e9


def kerr_isco(a: float, M: float = 1.0) -> float:
    """Prograde ISCO (Bardeen, Press & Teukolsky 1972)."""
    chi = a / M
    z1 = 1 + (1 - chi * chi) ** (1 / 3) * ((1 + chi) ** (1 / 3) + (1 - chi) ** (1 / 3))
    z2 = math.sqrt(3 * chi * chi + z1 * z1)
    return M * (3 + z2 - math.sqrt((3 - z1) * (3 + z1 + 2 * z2)))


def circular_orbit_beta(r: float, a: float, M: float = 1.0) -> float:
    """Speed of a prograde equatorial circular orbit relative to the ZAMO
    (calc_circ_geod_beta, Kerr.source/source_geometry.jl:44-49)."""
    d = r * r - 2 * M * r + a * a
    return math.sqrt(M) * (r * r - 2 * a * math.sqrt(M * r) + a * a) / (math.sqrt(d) * (r ** 1.5 + a * math.sqrt(M)))


def _scene(kind: int, **kw) -> abi.Scene:
    s = abi.Scene()
    s.kind = kind
    s.ref_precision = 0
    s.mass = 1.0
    s.spin = 0.0
    s.r_in = 0.0
    s.r_out = 1.0
    s.theta_lo = 0.0
    s.theta_hi = PI
    s.temperature = 5778.0
    s.a_nu = 1.0
    s.escape_radius = 100.0
    s.winding_limit = 8 * PI
    s.rho_r0 = 6.0
    s.rho_h = 0.1
    s.rho_index = -2.0
    s.t_index = -0.75
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def minkowski_sphere_scene(a_nu: float = 100.0) -> abi.Scene:
    return _scene(abi.SCENE_MINKOWSKI_SPHERE, r_out=1.0, temperature=5772.0, a_nu=a_nu)


def schwarzschild_disk_scene(a_nu: float = 100.0) -> abi.Scene:
    return _scene(abi.SCENE_SCHWARZSCHILD_DISK, r_in=6.0, r_out=20.0, theta_lo=15 * PI / 32,
                  theta_hi=17 * PI / 32, temperature=1e4, a_nu=a_nu)


def kerr_disk_scene(a: float = 0.9, a_nu: float = 100.0) -> abi.Scene:
    return _scene(abi.SCENE_KERR_DISK, spin=a, r_in=6.0, r_out=20.0, theta_lo=15 * PI / 32,
                  theta_hi=17 * PI / 32, temperature=1e4, a_nu=a_nu)


def kerr_thick_disk_scene(a: float = 0.9) -> abi.Scene:
    return _scene(abi.SCENE_KERR_THICK_DISK, spin=a, r_in=kerr_isco(a), r_out=30.0, temperature=1e4, a_nu=0.05)


def look_at_camera(r: float, theta: float, fov: float, x_pix: int, tol: float, max_steps: int = 10_000,
                   phi: float = 0.0) -> abi.Camera:
    return abi.make_camera([0.0, r, theta, phi], [PI / 2, 0.0], 0.0, [0.0, 0.0, -PI / 2], x_pix, fov, fov, tol,
                           max_steps)


def orbiting_camera(r: float, theta: float, a: float, fov: float, x_pix: int, tol: float,
                    max_steps: int = 10_000) -> abi.Camera:
    """Camera on a (near-)circular prograde orbit: speed from circular_orbit_beta
    along the +phi tetrad axis, looking towards the hole."""
    beta = circular_orbit_beta(r, a)
    return abi.make_camera([0.0, r, theta, 0.0], [PI / 2, PI / 2], beta, [0.0, 0.0, -PI], x_pix, fov, fov, tol,
                           max_steps)


WORKLOADS = {
    # name: (scene factory, camera factory(x_pix), default x_pix, tolerance)
    "minkowski_sphere": (minkowski_sphere_scene, lambda xp, tol=1e-8: look_at_camera(10.0, PI / 2, 60.0, xp, tol),
                         256, 1e-8),
    "schwarzschild_disk": (schwarzschild_disk_scene,
                           lambda xp, tol=1e-8: look_at_camera(50.0, math.radians(80.0), 45.0, xp, tol), 1024, 1e-8),
    "kerr_thin_disk": (kerr_disk_scene, lambda xp, tol=1e-8: look_at_camera(50.0, math.radians(80.0), 45.0, xp, tol),
                       1024, 1e-8),
    "kerr_thick_disk": (kerr_thick_disk_scene,
                        lambda xp, tol=1e-7: orbiting_camera(5.0, math.radians(80.0), 0.9, 90.0, xp, tol), 2048, 1e-7),
}


def workload(name: str, x_pix: int | None = None, tol: float | None = None):
    """(scene, camera, colors) of a named workload, optionally at another size."""
    sf, cf, xp, t = WORKLOADS[name]
    cam = cf(x_pix or xp, tol or t)
    return sf(), cam, log_spaced_colors(64)


def batched_frames(n_frames: int = 96, seed: int = 0, sizes=(256, 512, 1024), tols=(1e-6, 1e-8)):
    """Cameras of the batched workload: r ~ U[5, 40], inclination ~ U[10, 85] deg
    from numpy default_rng(seed); n_frames/len(sizes) frames per size; frame k
    uses tols[k % 2]. Returns (scene, cameras, colors, meta)."""
    rng = np.random.default_rng(seed)
    rs = rng.uniform(5.0, 40.0, n_frames)
    incs = rng.uniform(10.0, 85.0, n_frames)
    per = n_frames // len(sizes)
    cams, meta = [], []
    for k in range(n_frames):
        xp = sizes[min(k // per, len(sizes) - 1)]
        tol = tols[k % len(tols)]
        cams.append(look_at_camera(float(rs[k]), math.radians(float(incs[k])), 45.0, xp, tol))
        meta.append({"r": float(rs[k]), "inclination_deg": float(incs[k]), "x_pix": xp, "tol": tol})
    return kerr_disk_scene(), cams, log_spaced_colors(64), meta
