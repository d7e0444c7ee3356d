"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the
oracle): the oracle reproduces them, and the CUDA library matches them."""
import numpy as np
import pytest

from rtwca_b200 import abi
from tests.golden.make_golden import CASES, case
from tests.parity import summarize
from tests.conftest import ROOT

GOLDEN = ROOT / "tests" / "golden"
MODES = [(abi.DP45_REF_COMPAT, "ref"), (abi.DP45_FSAL, "fsal")]


def load(name, tag):
    d = np.load(GOLDEN / f"{name}_{tag}.npz")
    return {"xyz": d["xyz"], "class": d["term_class"], "steps": d["steps"], "spectrum": d["spectrum"],
            "tau": d["tau"], "state": d["state"], "colors": d["colors"]}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("integ,tag", MODES)
def test_oracle_reproduces_golden(oracle, name, integ, tag):
    g = load(name, tag)
    scene, cam, colors, _ = case(name, integ)
    assert np.array_equal(colors, g["colors"])
    r = oracle.render(scene, cam, colors, integrator=integ)
    assert np.array_equal(r["class"], g["class"])
    assert np.array_equal(r["steps"], g["steps"])
    assert np.allclose(r["xyz"], g["xyz"], rtol=1e-12, atol=0)
    assert np.allclose(r["state"], g["state"], rtol=1e-12, atol=1e-300)


GPU_CASES = [(i, t, p) for i, t in MODES for p in (abi.PREC_FP64, abi.PREC_MIXED)
             # FSAL with FP32 stages is checked on larger grids in test_gpu_parity
             if not (i == abi.DP45_FSAL and p == abi.PREC_MIXED)]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("integ,tag,prec", GPU_CASES)
def test_gpu_matches_golden(renderer, name, integ, tag, prec):
    g = load(name, tag)
    scene, cam, colors, _ = case(name, integ)
    out = renderer.render(scene, [cam], colors, want=("xyz", "class", "steps", "spectrum"), precision=prec,
                          integrator=integ)
    s = summarize(out, g)
    assert s["class_match"] >= 0.99, s
    assert s["frac_within_1e-3"] >= 0.99, s
    if prec == abi.PREC_FP64:
        assert s["max_rel"] < 1e-5, s
