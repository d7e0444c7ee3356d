"""The bremsstrahlung torus (RTW_SCENE_KERR_BREMS_TORUS) on the GPU against
the FP64 oracle: per-bin forward kernels with the Gaunt-factor lookup of the
reference's gaunt_ei_therm_van_Hoof (emission_functions.jl:54-78) on a device
copy of the caller's table. The table here is a smooth stand-in on the van
Hoof grid (configs.smooth_gaunt_table): the real table is data that the
caller supplies; the lookup itself is checked bit for bit on the host
(tests/test_brems_cpu.py), the real table included."""
import numpy as np
import pytest

from rtwca_b200 import abi, configs

pytestmark = pytest.mark.gpu


def _spec_err(g, ref):
    den = np.maximum(np.abs(ref), 1e-6 * np.abs(ref).max())
    return np.abs(np.asarray(g, np.float64) - ref) / den


@pytest.mark.parametrize("prec,integ,bar", [(abi.PREC_FP64, abi.DP45_FSAL, 0.999),
                                            (abi.PREC_FP64, abi.DP45_REF_COMPAT, 0.999),
                                            (abi.PREC_MIXED, abi.DP45_FSAL, 0.999),
                                            (abi.PREC_MIXED, abi.DP45_REF_COMPAT, 0.99)])
def test_brems_torus_parity(renderer, oracle, prec, integ, bar):
    """Classes on >= 99.9% of pixels; per-bin spectra within 1e-3 on >= 99.9%
    of the pixel-bins (99% for FP32 stages with the reference's step, which
    is not convergent: FP32 and FP64 rounding take slightly different step
    sequences and differ by its error)."""
    scene, lut = configs.brems_scene(), configs.smooth_gaunt_table()
    cam, col = configs.torus_camera(24, tol=1e-6), configs.torus_colors(8)
    g = renderer.render(scene, [cam], col, want=("spectrum", "class", "steps", "xyz"), precision=prec,
                        integrator=integ, gaunt_lut=lut)
    r = oracle.render(scene, cam, col, integrator=integ, gaunt_lut=lut)
    cm = float(np.mean(g["class"] == r["class"]))
    same = g["class"] == r["class"]
    err = _spec_err(g["spectrum"][same], r["spectrum"][same])
    print("class", cm, "within 1e-3", float(np.mean(err <= 1e-3)), "p99", float(np.quantile(err, 0.99)))
    assert np.all(r["spectrum"].max(axis=1) > 0)
    assert cm >= 0.999
    assert np.mean(err <= 1e-3) >= bar


def test_brems_needs_its_table(renderer):
    scene = configs.brems_scene()
    with pytest.raises(abi.RTWError) as e:
        renderer.render(scene, [configs.torus_camera(8, tol=1e-6)], configs.torus_colors(4),
                        precision=abi.PREC_MIXED, integrator=abi.DP45_FSAL)
    assert e.value.status == abi.ERR_INVALID_PARAM


def test_brems_table_scales_the_image(renderer):
    """The table enters as a Gaunt factor should: with a constant table of
    1.2 (the lookup's value outside the table) the image is that of g_ff =
    1.2 everywhere; doubling the table doubles the emission where the fluid
    falls inside the table and leaves the rest (the hot inner torus, where
    gamma^2 drops below the table) at 1.2, so every pixel's intensity grows by
    a factor between 1 and 2 (optically thin)."""
    scene = configs.brems_scene()
    cam, col = configs.torus_camera(12, tol=1e-6), configs.torus_colors(4)
    one = np.full((abi.GAUNT_ROWS, abi.GAUNT_COLS), 1.2, np.float32)
    a = renderer.render(scene, [cam], col, want=("spectrum",), precision=abi.PREC_FP64, integrator=abi.DP45_FSAL,
                        gaunt_lut=one)["spectrum"].astype(np.float64)
    b = renderer.render(scene, [cam], col, want=("spectrum",), precision=abi.PREC_FP64, integrator=abi.DP45_FSAL,
                        gaunt_lut=2 * one)["spectrum"].astype(np.float64)
    on = a > 1e-6 * a.max()
    q = b[on] / a[on]
    print("ratio min", q.min(), "mean", q.mean(), "max", q.max())
    assert q.min() >= 1 - 1e-6 and q.max() <= 2 + 1e-6
    assert q.mean() > 1.3
