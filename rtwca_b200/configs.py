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


# ---------------------------------------------------------------------------
# Differentiable synchrotron torus (Kerr a = 0.94, inclination 17 deg, 512^2,
# 32 bins over 230 GHz +- 20 %), the differentiable-render workload; the camera
# distance, field of view and torus extent are choices of this library.
# ---------------------------------------------------------------------------
TORUS_DEFAULTS = {"spin": 0.94, "inclination_deg": 17.0, "n_e0": 1e5, "b_0": 10.0, "theta_e0": 10.0}


def torus_scene(spin: float = 0.94, n_e0: float = 1e5, b_0: float = 10.0, theta_e0: float = 10.0) -> abi.Scene:
    """n_e = n_e0 (r/6)^-1.5 exp(-z^2 / 2 (0.3 r)^2), B = b_0 (r/6)^-1 G,
    Theta_e = theta_e0 (r/6)^-1, tapered inside r = 6 M (width 0.5 M) and
    beyond 40 M (width 5 M); M87* length scale 9.62e14 cm."""
    s = abi.scene_default(abi.SCENE_KERR_SYNCHRO_TORUS)
    s.spin, s.n_e0, s.b_0, s.theta_e0 = float(spin), float(n_e0), float(b_0), float(theta_e0)
    return s


def torus_colors(n: int = 32, f_center: float = 230e9, rel: float = 0.2) -> np.ndarray:
    """n wavelengths (nm) of frequencies evenly spaced over f_center (1 +- rel),
    ascending in wavelength."""
    f = np.linspace(f_center * (1 + rel), f_center * (1 - rel), n)
    return 299792458.0 * 1e9 / f


def torus_camera(x_pix: int = 512, inclination_deg: float = 17.0, r: float = 100.0, fov: float = 28.0,
                 tol: float = 1e-6, max_steps: int = 20_000) -> abi.Camera:
    """Static camera at r = 100 M and the given inclination, looking at the
    hole; 28 deg covers +- 25 M."""
    return look_at_camera(r, math.radians(inclination_deg), fov, x_pix, tol, max_steps)


def torus_target_params(seed: int = 1, rel: float = 0.05) -> dict:
    """Parameters of the target image: every default perturbed by a relative
    normal deviate of size rel from numpy default_rng(seed)."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(len(TORUS_DEFAULTS))
    return {k: v * (1 + rel * float(e)) for (k, v), e in zip(TORUS_DEFAULTS.items(), d)}


def torus_problem(x_pix: int = 512, tol: float = 1e-6, params: dict | None = None):
    """(scene, camera, colors) of the torus at the given parameters."""
    p = dict(TORUS_DEFAULTS)
    if params:
        p.update(params)
    scene = torus_scene(p["spin"], p["n_e0"], p["b_0"], p["theta_e0"])
    cam = torus_camera(x_pix, p["inclination_deg"], tol=tol)
    return scene, cam, torus_colors()


# ---------------------------------------------------------------------------
# Powehi (the reference's M87* model): its scene constants and its "m87"
# camera (initialization.jl:100-110).
# ---------------------------------------------------------------------------
def powehi_scene() -> abi.Scene:
    return abi.scene_default(abi.SCENE_KERR_POWEHI)


def powehi_camera(x_pix: int = 256, tol: float = 1e-6, max_steps: int = 20_000) -> abi.Camera:
    """position (0, 35, 0.3, 0), direction (pi/2, pi/6), pointing (0, 0, pi),
    beta 0; the reference's default field of view (85 x 60 deg)."""
    return abi.make_camera([0.0, 35.0, 0.3, 0.0], [PI / 2, PI / 6], 0.0, [0.0, 0.0, PI], x_pix, 85.0, 60.0, tol,
                           max_steps)


def synchro_scene() -> abi.Scene:
    """Synchro_Test.source: flat Cartesian space, a static synchrotron cylinder
    of radius 1 around the z axis in B^z = 10 G."""
    return abi.scene_default(abi.SCENE_SYNCHRO_TEST)


def wormhole_scene() -> abi.Scene:
    """Wormhole.source: Interstellar's Dneg wormhole (throat radius 1,
    half-length 0.005, lensing width 0.05)."""
    return abi.scene_default(abi.SCENE_WORMHOLE)


def cart_sphere_scene() -> abi.Scene:
    """Minkowski_Sphere_Cartesian.source: flat Cartesian space, a blackbody
    sphere of radius 1 at 5778 K with a_nu = 1 (optically thin) in front of a
    skybox."""
    return abi.scene_default(abi.SCENE_MINKOWSKI_CART_SPHERE)


def cart_sphere_camera(x_pix: int = 256, tol: float = 1e-6, max_steps: int = 20_000) -> abi.Camera:
    """The reference's "minkowski_t,x,y,z_sphere" world (initialization.jl:
    130-138): position (0, 0, 0, -4) (Cartesian t, x, y, z), direction (0, 0),
    pointing (0, 0, 0), beta 0; default field of view."""
    return abi.make_camera([0.0, 0.0, 0.0, -4.0], [0.0, 0.0], 0.0, [0.0, 0.0, 0.0], x_pix, 85.0, 60.0, tol,
                           max_steps)


def wormhole_camera(x_pix: int = 256, tol: float = 1e-6, max_steps: int = 20_000) -> abi.Camera:
    """The reference's "wormhole" world (initialization.jl:140-148): position
    (0, l = 5, pi/2, 0), direction (pi/2, 0), pointing (0, 0, -pi/2), beta 0;
    default field of view."""
    return abi.make_camera([0.0, 5.0, PI / 2, 0.0], [PI / 2, 0.0], 0.0, [0.0, 0.0, -PI / 2], x_pix, 85.0, 60.0, tol,
                           max_steps)


def synchro_camera(x_pix: int = 256, tol: float = 1e-6, max_steps: int = 20_000) -> abi.Camera:
    """The reference's "synch" world (initialization.jl:120-128): position
    (0, 0, 0, 0) (Cartesian t, x, y, z: inside the cylinder), direction
    (0, 0), pointing (pi/8, 0, pi), beta 0; default field of view."""
    return abi.make_camera([0.0, 0.0, 0.0, 0.0], [0.0, 0.0], 0.0, [PI / 8, 0.0, PI], x_pix, 85.0, 60.0, tol,
                           max_steps)


# ---------------------------------------------------------------------------
# Thermal bremsstrahlung torus (the van Hoof Gaunt-factor lookup of the
# reference's emission_functions.jl:54-78 on the synchrotron torus's fluid).
# ---------------------------------------------------------------------------
def brems_scene(spin: float = 0.94, n_e0: float = 1e8, theta_e0: float = 10.0) -> abi.Scene:
    s = abi.scene_default(abi.SCENE_KERR_BREMS_TORUS)
    s.spin, s.n_e0, s.theta_e0 = float(spin), float(n_e0), float(theta_e0)
    return s


def smooth_gaunt_table() -> np.ndarray:
    """A smooth stand-in for the van Hoof table (the real one is data the
    caller supplies): on the table's grid (log10 u = -16 + 0.2 i, log10
    gamma^2 = -6 + 0.2 j), g = 1 + 0.55 ln(1 + 10^(-0.9 log10 u)) / (1 + 0.05
    |log10 gamma^2|), float32 [146, 81]. It rises towards small u as the
    real factor does; its values are not physical Gaunt factors."""
    lu = -16.0 + 0.2 * np.arange(abi.GAUNT_ROWS)[:, None]
    lg = -6.0 + 0.2 * np.arange(abi.GAUNT_COLS)[None, :]
    return (1.0 + 0.55 * np.log1p(10.0 ** (-0.9 * lu)) / (1.0 + 0.05 * np.abs(lg))).astype(np.float32)
