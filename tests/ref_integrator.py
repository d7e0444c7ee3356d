"""A second, pure-Python restatement of the reference's step loop (test helper).

integrate_ray (main/Iterators/LttM/LttM.jl:11-59) and RKDP_Step_w_buffer!
(main/Iterators/LttM/integrators_LttM.jl:54-224) with the scene guards
pad_max_dt / near_singularity / keepinbounds! / calc_terminate of
Kerr.source, Schwarzschild_Simple_Disk_Spherical.source and
Minkowski_Sphere_Spherical.source, transcribed independently of the C++ oracle
so the two can check each other; the right-hand side comes from the oracle
(oracle.rhs), which tests/test_abi_cpu.py and tests/test_oracle_physics.py pin.
Pure-Python loops: small cases only.
"""
import math

import numpy as np

from rtwca_b200 import abi

PI = 3.141592653589793
NDZ = 1e-24
F32_01 = float(np.float32(0.1))
F32_1EM12 = float(np.float32(1e-12))
F32_1EM32 = float(np.float32(1e-32))

A = np.zeros((10, 9))
A[2, 2] = 1 / 5
A[3, 2], A[3, 3] = 3 / 40, 9 / 40
A[4, 2], A[4, 3], A[4, 4] = 44 / 45, -56 / 15, 32 / 9
A[5, 2], A[5, 3], A[5, 4], A[5, 5] = 19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729
A[6, 2], A[6, 3], A[6, 4], A[6, 5], A[6, 6] = 9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656
A[7, 2], A[7, 4], A[7, 5], A[7, 6], A[7, 7] = 35 / 384, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84
A[9, 2], A[9, 4], A[9, 5], A[9, 6], A[9, 7], A[9, 8] = (5179 / 57600, 7571 / 16695, 393 / 640, -92097 / 339200,
                                                        187 / 2100, 1 / 40)


def jl_mod(x, y):
    r = math.fmod(x, y)
    if r != 0 and ((r < 0) != (y < 0)):
        r += y
    return r


class Scene:
    def __init__(self, s: abi.Scene):
        self.kind = s.kind
        self.M = s.mass
        self.a = s.spin if s.kind in (abi.SCENE_KERR_DISK, abi.SCENE_KERR_THICK_DISK) else 0.0
        self.rs = 2 * self.M
        if self.kind in (abi.SCENE_KERR_DISK, abi.SCENE_KERR_THICK_DISK):
            self.r_ev = self.rs / 2 + math.sqrt(self.rs * self.rs / 4 - self.a * self.a)
        else:
            self.r_ev = self.rs
        self.esc = s.escape_radius
        self.wind = s.winding_limit
        self.kerr = self.kind in (abi.SCENE_KERR_DISK, abi.SCENE_KERR_THICK_DISK)

    def pad_max_dt(self, ray, scale):
        if self.kerr:
            scale = float(np.float32(scale))
        if ray[2] < PI / 8 or ray[2] > 7 * PI / 8:
            eps = min(scale, F32_01)
        elif self.kind == abi.SCENE_SCHWARZSCHILD_DISK and ray[1] <= 1.5 * (3 * self.M):
            eps = scale / 10
        else:
            eps = scale
        with np.errstate(divide="ignore"):
            if self.kerr:
                vr = abs(ray[5])
                first = abs(1 / (eps / vr)) + NDZ if vr != 0 else NDZ
            else:
                first = abs(1 / (eps / (abs(ray[5]) + NDZ))) + NDZ
        second = abs(1 / (eps * min(ray[2], PI - ray[2]) / (abs(ray[6]) + NDZ) + NDZ))
        third = abs(1 / (eps / (abs(ray[7]) + NDZ) + NDZ))
        m = min(1 / (first + second + third + NDZ), 0.5)
        return max(m, F32_1EM12)

    def near_singularity(self, ray, h, tol):
        th_new = ray[2] + h * ray[6]
        r_new = ray[1] + h * ray[5]
        lim = tol
        if self.kind == abi.SCENE_MINKOWSKI_SPHERE:
            lim = 10 * tol / abs(r_new + NDZ)
        if abs(th_new) <= lim:
            return True, 2 * abs(ray[2]) / (abs(ray[6] * 37) + NDZ)
        if abs(th_new - PI) <= lim:
            return True, 2 * abs((ray[2] - PI) / (abs(ray[6] * 37) + NDZ))
        if self.kind == abi.SCENE_MINKOWSKI_SPHERE and abs(r_new) <= 100 * tol:
            return True, 2 * tol / (abs(ray[5] * 37) + NDZ)
        return False, h

    def keepinbounds(self, ray):
        if self.kind == abi.SCENE_MINKOWSKI_SPHERE and ray[1] <= 0:
            ray[1] = -ray[1] + NDZ
            ray[5] = -ray[5]
            ray[2] -= PI
            ray[6] = -ray[6]
        if ray[2] < 0:
            ray[2] = -ray[2]
            ray[3] -= PI
            ray[6] = -ray[6]
        ray[2] = jl_mod(ray[2], 2 * PI)
        if ray[2] >= PI:
            ray[2] = 2 * PI - ray[2]
            ray[3] += PI
            ray[6] = -ray[6]

    def terminate(self, ray, tol, max_steps, step_count):
        """calc_terminate with the class of the first predicate that holds."""
        if step_count >= max_steps:
            return abi.CLASS_MAXSTEPS
        if ray[1] > self.esc:
            return abi.CLASS_ESCAPE
        if self.kind != abi.SCENE_MINKOWSKI_SPHERE and ray[1] <= (1 + 10 * tol) * self.r_ev:
            return abi.CLASS_HORIZON
        if ray[3] > self.wind:
            return abi.CLASS_WINDING
        thick = -math.log(tol)
        for i in range(9, len(ray), 2):
            if ray[i] < thick:
                return 0
        return abi.CLASS_THICK


def integrate_ray(oracle, scene_struct, colors, ray0, tol, max_steps, scale=0.1, fsal=False):
    """Returns (class, step_count, final state) of one ray."""
    sc = Scene(scene_struct)
    L = len(ray0)

    def f(R):
        return oracle.rhs(scene_struct, colors, R)

    ray = np.array(ray0, dtype=float)
    dt = -sc.pad_max_dt(ray, scale)
    last = f(ray)
    rejected = False
    steps = 0
    while True:
        # RKDP_Step_w_buffer!
        k1 = last
        max_dt = sc.pad_max_dt(ray, scale)
        warn, temp = sc.near_singularity(ray, dt, tol)
        done = False
        if warn:
            ray = ray - temp * k1
            sc.keepinbounds(ray)
            for _ in range(36):
                if not sc.terminate(ray, tol, 2, 1):
                    k1 = f(ray)
                    last = k1
                    ray = ray - temp * k1
                    sc.keepinbounds(ray)
            if sc.terminate(ray, tol, 2, 1):
                rejected = False
                done = True
            else:
                k1 = f(ray)
                last = k1
                dt = -sc.pad_max_dt(ray, scale)
        if not done:
            h = dt
            k2 = f(ray + h * k1 * A[2, 2])
            k3 = f(ray + h * (k1 * A[3, 2] + k2 * A[3, 3]))
            k4 = f(ray + h * (k1 * A[4, 2] + k2 * A[4, 3] + k3 * A[4, 4]))
            k5 = f(ray + h * (k1 * A[5, 2] + k2 * A[5, 3] + k3 * A[5, 4] + k4 * A[5, 5]))
            k6 = f(ray + h * (k1 * A[6, 2] + k2 * A[6, 3] + k3 * A[6, 4] + k4 * A[6, 5] + k5 * A[6, 6]))
            ns = k1 * A[7, 2] + k3 * A[7, 4] + k4 * A[7, 5] + k5 * A[7, 6] + k6 * A[7, 7]
            k7 = f(ray + h * ns)
            y = ray + h * ns
            d = y - ray - h * (k1 * A[9, 2] + k3 * A[9, 4] + k4 * A[9, 5] + k5 * A[9, 6] + k6 * A[9, 7] +
                               k7 * A[9, 8])
            tl = tol + np.maximum(np.abs(ray), np.abs(y)) * tol
            err = math.sqrt(float(np.sum((d / tl) ** 2)) / L)
            with np.errstate(divide="ignore", over="ignore"):
                hn = 0.9 * h * (1 / err) ** (1 / 5) if err > 0 else -math.inf * math.copysign(1, h)
            if abs(hn) > max_dt:
                hn = -max_dt
            if err == 0 or not math.isfinite(hn):
                sc.keepinbounds(y)
                last = k7 if fsal else ns
                ray = y
                rejected = False
            elif err > 1:
                if rejected and abs(hn) >= abs(h):
                    hn = h / 2
                sc.keepinbounds(ray)
                dt = hn
                rejected = True
            else:
                if abs(hn) > 5 * abs(h):
                    hn = 5 * h
                sc.keepinbounds(y)
                last = k7 if fsal else ns
                ray = y
                dt = hn
                rejected = False
        steps += 1
        c = sc.terminate(ray, tol, max_steps, steps)
        if c:
            return c, steps, ray
