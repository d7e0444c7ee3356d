"""The bremsstrahlung torus on the host: the Gaunt-factor lookup
(gaunt_ei_therm_van_Hoof, emission_functions.jl:54-78) of the library against
the oracle's separate transcription, its index conventions, a numpy float32
transcription on the reference's own table when that table is present, and
the library's right-hand side against the oracle's."""
from pathlib import Path

import numpy as np
import pytest

from rtwca_b200 import abi, configs

REF_TABLE = Path("/root/reference/main/Gaunt_Factors/gauntff_merged_Z01.dat")


def _points(rng, n):
    lg = rng.uniform(-7.0, 11.0, n)   # log10 gamma^2, beyond the table on both sides
    lu = rng.uniform(-17.0, 14.0, n)  # log10 u
    return 10.0 ** lg, 10.0 ** lu


def _julia_f32(lut, gam2, u):
    """gaunt_ei_therm_van_Hoof in numpy float32 steps (a third transcription)."""
    f = np.float32
    loggam, logu = f(np.log10(gam2)), f(np.log10(u))
    frac_i = f(f(logu + f(16)) / f(0.2))
    frac_j = f(f(loggam + f(6)) / f(0.2))
    if not (np.isfinite(frac_i) and np.isfinite(frac_j)):
        return f(1.2)
    fi, fj = int(np.floor(frac_i)), int(np.floor(frac_j))
    ci, cj = int(np.ceil(f(frac_i + f(1e-3)))), int(np.ceil(f(frac_j + f(1e-3))))
    if not (1 <= fi and 1 <= fj and ci <= 146 and cj <= 81):
        return f(1.2)
    L = lambda i, j: lut[i - 1, j - 1]  # noqa: E731
    a, b = f(f(ci) - frac_i), f(frac_i - f(fi))
    g1 = f(f(a * L(fi, fj)) + f(b * L(ci, fj)))
    g2 = f(f(a * L(fi, cj)) + f(b * L(ci, cj)))
    return f(f(f(f(cj) - frac_j) * g1) + f(f(frac_j - f(fj)) * g2))


def test_gaunt_library_equals_oracle(rtwlib, oracle):
    lut = np.random.default_rng(3).uniform(0.5, 8.0, (abi.GAUNT_ROWS, abi.GAUNT_COLS)).astype(np.float32)
    g2, u = _points(np.random.default_rng(4), 3000)
    for a, b in zip(g2, u):
        lib = abi.gaunt_lookup(lut, a, b)
        orc = oracle.gaunt(lut, a, b)
        py = float(_julia_f32(lut, a, b))
        assert lib == orc == py, (a, b, lib, orc, py)


def test_gaunt_index_conventions(rtwlib):
    """On an indexed table L[i, j] = 1000 i + j (1-based): a point exactly on
    the grid, log10 u = -16 + 0.2 k, reads row k (the reference's fractional
    index (log + 16) / 0.2 addresses the 1-based table directly); just below
    an integer index the two bilinear weights add up to 2; outside the table,
    and for u = 0, the factor is 1.2."""
    i = np.arange(1, abi.GAUNT_ROWS + 1)[:, None]
    j = np.arange(1, abi.GAUNT_COLS + 1)[None, :]
    lut = (1000.0 * i + j).astype(np.float32)
    k, m = 40, 20
    g = abi.gaunt_lookup(lut, 10.0 ** (-6 + 0.2 * m), 10.0 ** (-16 + 0.2 * k))
    assert abs(g - (1000 * k + m)) <= 1e-2 * (1000 * k + m) * 1e-3, g
    # frac_i just below 40 (within 1e-3): floor 39, ceil(frac + 1e-3) = 41
    fr = np.float32(40.0) - np.float32(4e-4)
    lu = float(fr) * 0.2 - 16.0
    g = abi.gaunt_lookup(lut, 10.0 ** (-6 + 0.2 * m), 10.0 ** lu)
    assert g > 1.9 * (1000 * 40 + m), g
    assert abi.gaunt_lookup(lut, 1e-9, 1e-3) == pytest.approx(1.2)   # log gamma^2 below the table
    assert abi.gaunt_lookup(lut, 1.0, 1e20) == pytest.approx(1.2)    # log u above it
    assert abi.gaunt_lookup(lut, 1.0, 0.0) == pytest.approx(1.2)     # u = 0


@pytest.mark.skipif(not REF_TABLE.exists(), reason="the reference's table is not on this machine")
def test_gaunt_on_the_reference_table(rtwlib):
    # the 42 header lines skipped as the reference reads it (emission_functions.jl:15)
    lut = np.loadtxt(REF_TABLE, skiprows=42, dtype=np.float64).astype(np.float32)
    assert lut.shape == (abi.GAUNT_ROWS, abi.GAUNT_COLS)
    g2, u = _points(np.random.default_rng(5), 2000)
    inside = 0
    for a, b in zip(g2, u):
        lib = abi.gaunt_lookup(lut, a, b)
        assert lib == float(_julia_f32(lut, a, b)), (a, b)
        inside += lib != np.float32(1.2)
    assert inside > 500


def test_brems_rhs_matches_oracle(rtwlib, oracle):
    scene = configs.brems_scene()
    lut = configs.smooth_gaunt_table()
    colors = configs.torus_colors(6)
    rng = np.random.default_rng(9)
    checked = 0
    for _ in range(40):
        st = np.zeros(8 + 2 * colors.size)
        st[1] = rng.uniform(4.0, 30.0)
        st[2] = rng.uniform(1.2, 1.9)
        st[3] = rng.uniform(0, 2 * np.pi)
        st[4:8] = [1.0, rng.normal(), rng.normal() / st[1], rng.normal() / st[1]]
        st[9::2] = rng.uniform(0, 1, colors.size)  # optical depths
        a = abi.brems_rhs(scene, colors, lut, st)
        b = oracle.rhs(scene, colors, st, gaunt_lut=lut)
        den = np.abs(b) + 1e-300
        assert np.all(np.abs(a - b) <= 1e-11 * den + 1e-300), np.max(np.abs(a - b) / den)
        checked += np.any(b[8::2] != 0)
    assert checked >= 5
