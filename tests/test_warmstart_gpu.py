"""The learned warm start on the GPU: what the trained network gains over the
reference's conduction start, on held-out cavities the model never saw
(seed 2000; the training set used seed 1000), with the solver judging both by
the same residual criterion; the mixed-precision path's result against FP64;
and the cold-start fallback when a warm start diverges.

The residual criterion bounds the distance to the fixed point only through the
slowest mode's relaxation: at the reference's 1e-6 a warm-started run can stop
with Nu ~1e-4 from the fixed point (a cold start ~2e-5).  The Nusselt checks
below therefore run both arms to 2e-7."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODEL = os.path.join(ROOT, "mpi-multi-process-version_b200", "warmstart_unet.npz")


def _cases(pkg, n=3):
    # held-out cases of the smallest side and moderate Ra, so the test runs in seconds
    cs = [c for c in pkg.warmstart.sample_cases(60, seed=2000) if c["nx"] == 128 and c["Ra"] < 3e4]
    return cs[:n]


@pytest.fixture(scope="module")
def model(pkg):
    return pkg.warmstart.WarmStart.load(MODEL)


def test_model_file_describes_its_training(model):
    assert model.meta["train"] >= 1000 and model.meta["train_seed"] != model.meta["test_seed"]
    assert max(model.meta["heldout_rel_l2"]) < 0.2


EPS = 2e-7


def test_warm_start_needs_fewer_iterations_than_cold(pkg, model):
    W = pkg.warmstart
    cases = _cases(pkg)
    assert len(cases) == 3
    # iterations to the reference's criterion
    cold = W.solve(cases, init="cold", storage="f64", eps=W.F32_EPS, max_steps=1200000)
    warm = W.solve(cases, init="warm", model=model, storage="f64", eps=W.F32_EPS, max_steps=1200000)
    assert (cold["status"] == 1).all() and (warm["status"] == 1).all()
    assert not warm["fallback"].any()
    assert warm["steps"].sum() <= 0.85 * cold["steps"].sum(), (warm["steps"], cold["steps"])
    # both end at the same FP64 fixed point (checked at the tighter criterion)
    cold = W.solve(cases, init="cold", storage="f64", eps=EPS, max_steps=1500000)
    warm = W.solve(cases, init="warm", model=model, storage="f64", eps=EPS, max_steps=1500000)
    assert (cold["status"] == 1).all() and (warm["status"] == 1).all()
    err = np.abs(warm["nu_hot"] - cold["nu_hot"]) / cold["nu_hot"]
    assert err.max() <= 1e-4, err


def test_mixed_precision_reaches_fp64_nusselt(pkg, model):
    W = pkg.warmstart
    cases = _cases(pkg, 2)
    ref = W.solve(cases, init="cold", storage="f64", eps=EPS, max_steps=1200000)
    mixed = W.solve(cases, init="warm", model=model, storage="mixed", eps=EPS, max_steps=1200000)
    assert (mixed["status"] == 1).all()
    assert (mixed["steps_low_precision"] > 0).all()
    err = np.abs(mixed["nu_hot"] - ref["nu_hot"]) / ref["nu_hot"]
    assert err.max() <= 1e-4, err


def test_extrapolated_warm_start_reaches_the_fp64_fixed_point(pkg, model):
    # one extrapolation of each member's slowest mode at residual 3e-5 from
    # states 10,000 iterations apart; the solver's criterion judges the result
    W = pkg.warmstart
    cases = _cases(pkg, 2)
    ref = W.solve(cases, init="cold", storage="f64", eps=EPS, max_steps=1500000)
    ex = W.solve(cases, init="warm", model=model, storage="f64", eps=EPS, max_steps=1500000,
                 extrapolate=(3e-5, 10000))
    assert (ex["status"] == 1).all() and not ex["fallback"].any()
    assert ex["extrapolation_factors"] is not None and (ex["extrapolation_factors"] >= 0).all()
    err = np.abs(ex["nu_hot"] - ref["nu_hot"]) / ref["nu_hot"]
    assert err.max() <= 1e-4, err


def test_diverging_warm_start_falls_back_to_cold(pkg):
    # a prediction far outside the low-Mach regime blows up; the member is
    # stopped (residual not finite or growing) and restarted from the
    # conduction state, then converges like a cold start
    W = pkg.warmstart
    cases = _cases(pkg, 2)
    bad = []
    for c in cases:
        shape = (c["ny"], c["nx"])
        rng = np.random.default_rng(0)
        bad.append({"rho": np.ones(shape), "u": rng.uniform(-0.5, 0.5, shape), "v": rng.uniform(-0.5, 0.5, shape),
                    "T": rng.uniform(-5.0, 5.0, shape)})
    good = W.solve(cases[:1], init="cold", storage="f64", max_steps=800000)
    res = W.solve(cases, init="warm", predictions=bad, storage="f64", max_steps=800000)
    assert res["fallback"].all()
    assert (res["status"] == 1).all()
    assert abs(res["nu_hot"][0] - good["nu_hot"][0]) <= 1e-4 * good["nu_hot"][0]
