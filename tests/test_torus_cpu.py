"""The synchrotron torus on the CPU: the library's host evaluation of the
torus right-hand side (the same generic-scalar functions the kernels run)
against the oracle's independent FP64 restatement, the adjoint's generic
geodesic acceleration against the scene functor, and the vector-Jacobian
product against central differences of the right-hand side.
"""
import numpy as np
import pytest

from rtwca_b200 import abi, configs

NB = 8


def _problem():
    sc, cam, col = configs.torus_problem(x_pix=16)
    return sc, col[:: 32 // NB]


def _state(sc, N, r, th, rng):
    """A null ray at (r, theta) with random spatial direction, random tau and I."""
    a, M = sc.spin, sc.mass
    Sig = r * r + a * a * np.cos(th) ** 2
    Del = r * r - 2 * M * r + a * a
    s2 = np.sin(th) ** 2
    gtt, gtp = -(1 - 2 * M * r / Sig), -2 * M * a * r * s2 / Sig
    gpp = (r * r + a * a + 2 * M * a * a * r * s2 / Sig) * s2
    kr, kth, kph = rng.normal(size=3) * np.array([1.0, 0.1, 0.05])
    A, B = gtt, 2 * gtp * kph
    C = gpp * kph ** 2 + Sig / Del * kr ** 2 + Sig * kth ** 2
    kt = (-B - np.sqrt(B * B - 4 * A * C)) / (2 * A)
    y = np.zeros(8 + 2 * N)
    y[:8] = [0.0, r, th, 0.3, kt, kr, kth, kph]
    y[9::2] = rng.uniform(0, 2, N)      # tau_c
    y[8::2] = rng.uniform(0, 1e14, N)   # I_c
    return y


POINTS = [(4.3, 1.57), (5.0, 1.4), (6.5, 1.5), (8.0, 1.2), (12.0, 1.7), (20.0, 1.0), (45.0, 1.5)]


def test_scene_defaults():
    s = abi.scene_default(abi.SCENE_KERR_SYNCHRO_TORUS)
    assert s.kind == abi.SCENE_KERR_SYNCHRO_TORUS
    assert (s.spin, s.r_in, s.n_e0, s.b_0, s.theta_e0) == (0.94, 6.0, 1e5, 10.0, 10.0)
    assert s.length_cm == pytest.approx(9.62e14)


def test_colors_and_target_params():
    c = configs.torus_colors()
    f = 299792458.0 * 1e9 / c
    assert c.size == 32 and np.all(np.diff(c) > 0)
    assert f.max() == pytest.approx(276e9) and f.min() == pytest.approx(184e9)
    t1, t2 = configs.torus_target_params(1), configs.torus_target_params(1)
    assert t1 == t2 and set(t1) == set(configs.TORUS_DEFAULTS)
    for k, v in t1.items():
        assert abs(v / configs.TORUS_DEFAULTS[k] - 1) < 0.25


def test_rhs_matches_oracle(oracle):
    sc, col = _problem()
    rng = np.random.default_rng(3)
    for r, th in POINTS:
        y = _state(sc, NB, r, th, rng)
        ref = oracle.rhs(sc, col, y)
        scale = 1e-12 * np.abs(ref).max()
        for form in (0, 1):
            f = abi.torus_rhs(sc, col, y, form)
            err = np.abs(f - ref) / np.maximum(np.abs(ref), scale)
            assert err.max() < 1e-11, (r, th, form, err.max())


def test_vjp_matches_central_differences():
    sc, col = _problem()
    rng = np.random.default_rng(5)
    names = {0: "spin", 2: "n_e0", 3: "b_0", 4: "theta_e0"}

    def rhs(y, **kw):
        s = configs.torus_scene(**{k: kw.get(k, getattr(sc, k)) for k in ("spin", "n_e0", "b_0", "theta_e0")})
        return abi.torus_rhs(s, col, y, 0)

    for r, th in [(5.0, 1.4), (6.5, 1.5), (8.0, 1.2), (12.0, 1.7)]:
        y = _state(sc, NB, r, th, rng)
        f0 = rhs(y)
        cot = rng.normal(size=y.size) / np.maximum(np.abs(f0), 1e-30)
        mu, pb = abi.torus_vjp(sc, col, y, cot)
        for i in range(y.size):
            if i in (0, 3):  # t and phi enter no slope
                assert mu[i] == 0
                continue
            h = 1e-6 * max(abs(y[i]), 1e-3)
            yp, ym = y.copy(), y.copy()
            yp[i] += h
            ym[i] -= h
            fd = (cot @ rhs(yp) - cot @ rhs(ym)) / (2 * h)
            floor = 1e-6 * np.sum(np.abs(cot * f0)) / max(abs(y[i]), 1e-3)
            assert abs(fd - mu[i]) <= 1e-5 * abs(fd) + floor, (r, th, i, fd, mu[i])
        for q, name in names.items():
            base = getattr(sc, name)
            h = 1e-6 * base
            fd = (cot @ rhs(y, **{name: base + h}) - cot @ rhs(y, **{name: base - h})) / (2 * h)
            assert abs(fd - pb[q]) <= 1e-5 * abs(fd), (r, th, name, fd, pb[q])
        assert pb[1] == 0  # the inclination enters only the initial data


POWEHI_POINTS = [(5.0, np.pi / 2), (8.0, 1.56), (20.0, 0.05), (40.0, 0.02), (60.0, 3.1), (15.0, 0.07), (30.0, 1.0)]


def test_powehi_rhs_matches_oracle(oracle):
    """Powehi (disk zone, jet zone near either pole, empty space): the
    library's per-bin right-hand side against the oracle's restatement of
    Powehi.source/source_model.jl."""
    sc = configs.powehi_scene()
    col = np.array([400.0, 550.0, 700.0])
    rng = np.random.default_rng(1)
    for r, th in POWEHI_POINTS:
        y = _state(sc, 3, r, th, rng)
        y[2] = th
        ref = oracle.rhs(sc, col, y)
        f = abi.torus_rhs(sc, col, y, 0)
        scale = 1e-12 * max(np.abs(ref).max(), 1e-300)
        err = np.abs(f - ref) / np.maximum(np.abs(ref), scale)
        assert err.max() < 1e-11, (r, th, err.max())
    assert abi.scene_default(abi.SCENE_KERR_POWEHI).spin == pytest.approx(0.9, rel=1e-7)


def test_structured_step_vjp_matches_generic():
    """The adjoint kernel's structured reverse of one Dormand-Prince step
    (emitter numbers once per stage, per-bin recursions, geodesic recursion)
    equals the generic reverse over the whole state, and both match central
    differences of the step map through its end state."""
    sc, col = _problem()
    rng = np.random.default_rng(11)
    for r, th in [(5.0, 1.4), (6.5, 1.5), (8.0, 1.2), (12.0, 1.7), (45.0, 1.5)]:
        y = _state(sc, NB, r, th, rng)
        for h in (-0.05, -0.4):
            cot = rng.normal(size=y.size)
            cot[8::2] /= 1e14
            a = abi.torus_step_vjp(sc, col, y, h, cot, 0)
            b = abi.torus_step_vjp(sc, col, y, h, cot, 1)
            back = abi.torus_step_vjp(sc, col, y, h, cot, 2)  # depths run back from the step's end
            for u, v, w in zip(a[:2], b[:2], back[:2]):
                np.testing.assert_allclose(u, v, rtol=1e-11, atol=1e-13 * np.abs(v).max())
                np.testing.assert_allclose(w, v, rtol=1e-10, atol=1e-12 * np.abs(v).max())
            assert a[2] == pytest.approx(b[2], rel=1e-11, abs=1e-13 * abs(b[2]) + 1e-300)
            assert back[2] == pytest.approx(b[2], rel=1e-10, abs=1e-12 * abs(b[2]) + 1e-300)
            # FP32 bin partials (the FP32-mixed adjoint): FP32 rounding, which
            # parameter components that cancel between bins amplify
            f32 = abi.torus_step_vjp(sc, col, y, h, cot, 3)
            np.testing.assert_allclose(f32[0], b[0], rtol=2e-5, atol=1e-5 * np.abs(b[0]).max())
            np.testing.assert_allclose(f32[1], b[1], rtol=1e-3, atol=1e-5 * np.abs(b[1]).max())
            assert f32[2] == pytest.approx(b[2], rel=2e-5, abs=1e-5 * abs(b[2]) + 1e-300)
            # d loss / d h against a central difference of the step
            dh = 1e-6 * abs(h)
            lp = cot @ _step(sc, col, y, h + dh)
            lm = cot @ _step(sc, col, y, h - dh)
            fd = (lp - lm) / (2 * dh)
            assert abs(fd - a[2]) <= 1e-5 * abs(fd) + 1e-9 * np.abs(cot * y).sum() / abs(h), (r, th, h, fd, a[2])


def _step(sc, col, y, h):
    """One DP45 step through the oracle-independent host right-hand side."""
    A = [[], [1 / 5], [3 / 40, 9 / 40], [44 / 45, -56 / 15, 32 / 9],
         [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
         [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
         [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]]
    K = []
    for s in range(6):
        Y = y + h * sum(A[s][j] * K[j] for j in range(s)) if s else y
        K.append(abi.torus_rhs(sc, col, Y, 0))
    return y + h * sum(A[6][j] * K[j] for j in range(6))


def test_synchro_scene_defaults():
    s = configs.synchro_scene()
    assert s.kind == abi.SCENE_SYNCHRO_TEST
    assert (s.r_out, s.n_e0, s.b_0, s.escape_radius) == (1.0, 1e7, 10.0, 100.0)
    assert s.length_cm == pytest.approx(9.62e14)


def _cart_state(N, x, y, z, rng):
    """A null ray at Cartesian (x, y, z) with a random direction, random tau and I."""
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    st = np.zeros(8 + 2 * N)
    st[:8] = [0.0, x, y, z, 1.0, d[0], d[1], d[2]]
    st[9::2] = rng.uniform(0, 2, N)
    st[8::2] = rng.uniform(0, 1e-3, N)
    return st


def test_synchro_rhs_matches_oracle(oracle):
    """Synchro_Test (flat Cartesian space, the synchrotron cylinder): the
    library's per-bin right-hand side against the oracle's restatement of
    Synchro_Test.source/source_model.jl, inside and outside the cylinder."""
    sc = configs.synchro_scene()
    col = np.array([380.0, 450.0, 550.0, 650.0, 750.0])
    rng = np.random.default_rng(2)
    inside = 0
    for x, y, z in [(0.0, 0.0, 0.0), (0.5, -0.3, 4.0), (0.9, 0.1, -20.0), (-0.2, 0.7, 1.0), (1.5, 0.0, 0.0),
                    (30.0, -40.0, 2.0)]:
        for _ in range(3):
            st = _cart_state(col.size, x, y, z, rng)
            ref = oracle.rhs(sc, col, st)
            f = abi.torus_rhs(sc, col, st, 0)
            assert np.array_equal(f[:4], st[4:8]) and np.all(f[4:8] == 0)  # straight lines
            scale = 1e-300 + 1e-12 * np.abs(ref[8:]).max()
            err = np.abs(f[8:] - ref[8:]) / np.maximum(np.abs(ref[8:]), scale)
            assert err.max() < 1e-11, (x, y, z, err.max())
            inside += bool(np.any(ref[8:] != 0))
    assert inside == 12  # the four points inside the cylinder emit, the two outside do not


def test_cart_sphere_rhs_matches_oracle(oracle):
    """The Cartesian blackbody sphere (Minkowski_Sphere_Cartesian.source):
    defaults, and the library's per-bin right-hand side against the oracle's
    generic calc_ray_derivative! with its is_fire and calc_planck, inside and
    outside the sphere; tau' = -a_nu / k^t exactly."""
    sc = configs.cart_sphere_scene()
    assert sc.kind == abi.SCENE_MINKOWSKI_CART_SPHERE
    assert (sc.r_out, sc.temperature, sc.a_nu, sc.escape_radius) == (1.0, 5778.0, 1.0, 100.0)
    col = np.array([380.0, 450.0, 550.0, 650.0, 750.0])
    rng = np.random.default_rng(4)
    inside = 0
    for x, y, z in [(0.0, 0.0, 0.0), (0.5, -0.3, 0.6), (-0.1, 0.2, -0.95), (0.9, 0.5, 0.0), (0.0, 0.0, -4.0),
                    (30.0, -40.0, 2.0)]:
        for _ in range(3):
            st = _cart_state(col.size, x, y, z, rng)
            st[4] = rng.uniform(0.5, 2.0)  # k^t: the frequency shift
            ref = oracle.rhs(sc, col, st)
            f = abi.torus_rhs(sc, col, st, 0)
            assert np.array_equal(f[:4], st[4:8]) and np.all(f[4:8] == 0)  # straight lines
            scale = 1e-300 + 1e-12 * np.abs(ref[8:]).max()
            err = np.abs(f[8:] - ref[8:]) / np.maximum(np.abs(ref[8:]), scale)
            assert err.max() < 1e-11, (x, y, z, err.max())
            if np.any(ref[8:] != 0):
                inside += 1
                assert np.array_equal(f[9::2], np.full(col.size, -1.0 / st[4]))
    assert inside == 9  # the three points inside the sphere emit, (0.9, 0.5, 0) and the others do not


def test_wormhole_rhs_matches_oracle(oracle):
    """The Dneg wormhole (Wormhole.source): the library's geodesic right-hand
    side against the oracle's Christoffel contraction, in the throat, near it
    and far out on both sides; no emission anywhere."""
    sc = configs.wormhole_scene()
    assert sc.kind == abi.SCENE_WORMHOLE and (sc.r_in, sc.edge_in, sc.edge_out) == (1.0, 0.005, 0.05)
    col = np.array([400.0, 550.0, 700.0])
    rng = np.random.default_rng(7)
    for l, th in [(0.0, 1.2), (0.003, 0.7), (0.2, 1.5), (-0.4, 2.0), (5.0, 1.571), (-30.0, 0.3), (80.0, 2.9)]:
        st = np.zeros(8 + 2 * col.size)
        st[:8] = [0.0, l, th, 0.4, 1.0, *rng.normal(size=3)]
        ref = oracle.rhs(sc, col, st)
        f = abi.torus_rhs(sc, col, st, 0)
        err = np.abs(f[:8] - ref[:8]) / np.maximum(np.abs(ref[:8]), 1e-12 * np.abs(ref[:8]).max() + 1e-300)
        assert err.max() < 1e-12, (l, th, err.max())
        assert np.all(f[8:] == 0) and np.all(ref[8:] == 0)
