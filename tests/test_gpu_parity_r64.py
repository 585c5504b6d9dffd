"""Parity at the production shape (r = 64) against the reference's own build.

The cases (tests/golden/large_cases.py) are regenerated from their seeds and
read back through the reference's file formats; the digests in each spec prove
that the inputs are bitwise the ones the reference saw.  They exercise what the
small golden cases cannot: 64 x 64 knot priors (four 16-wide Cholesky block
columns), the widest product tiles, sibling groups of clustered regions with
hundreds to thousands of observations, the factored posterior up to its 2r
threshold and the dense posterior form above it.

Tolerances, as for the other golden cases:
  FP64 path   log-likelihood within 1e-8 relative, d within 1e-8 of max(1, |d|),
              predictions within 1e-6 (absolute, scaled by max(1, |value|))
  mixed path  errors reported per output (printed).  The mixed path does NOT
              reach the 1e-6 relative log-likelihood target at r = 64: measured
              1.4e-5 to 7.6e-5 on these cases, predictions 3e-5 to 7e-5 (FP32
              storage of the conditioned factors U limits the conditional
              covariances K = C - sum U^T U to an absolute error of about
              2^-24 |C|, which the deep levels' small K amplify).  The assertion
              holds the measured level (log-likelihood 2e-4, predictions 5e-4)
              so that a regression shows.
"""
import numpy as np
import pytest

import large_cases
from nonstationary_mra_b200 import api

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-8
PRED_TOL = 1e-6
MIXED_LL_GUARD = 2e-4      # measured 1.4e-5 .. 7.6e-5; the 1e-6 target is not met
MIXED_PRED_GUARD = 5e-4    # measured 3e-5 .. 7e-5

NAMES = large_cases.names()


def _theta(md):
    return dict(sill=md.sill, range_=md.range_, nugget=md.nugget, sill_scale=md.sill_scale,
                range_scale=md.range_scale, nugget_scale=md.nugget_scale)


def _pred_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


@pytest.fixture(scope="module", params=NAMES)
def case(request):
    st, md, spec = large_cases.load(request.param, mode="prediction")
    return request.param, st, md


def test_r64_fp64_loglik_and_predictions(case):
    name, st, md = case
    g = large_cases.golden(name)
    assert st.n_obs == g["n_obs"]
    ctx = api.Context(st, md)
    ctx.set_theta(**_theta(md))
    d, ll = ctx.loglik()
    err = abs(ll - g["loglik"]) / abs(g["loglik"])
    print(f"{name} fp64 loglik {ll:.12f} reference {g['loglik']:.12f} rel err {err:.3e}")
    assert err <= LL_RTOL, (ll, g["loglik"])
    assert abs(d - g["d"]) <= LL_RTOL * max(1.0, abs(g["d"])), (d, g["d"])
    mean, var = ctx.predict()
    ctx.close()
    gm, gv = large_cases.golden_prediction(name)
    assert mean.shape == gm.shape
    em, ev = _pred_err(mean, gm), _pred_err(var, gv)
    print(f"{name} fp64 prediction err mean {em:.3e} var {ev:.3e}")
    assert em <= PRED_TOL and ev <= PRED_TOL


def test_r64_mixed_errors_per_output(case):
    name, st, md = case
    g = large_cases.golden(name)
    ctx = api.Context(st, md, precision="mixed")
    ctx.set_theta(**_theta(md))
    d, ll = ctx.loglik()
    mean, var = ctx.predict()
    ctx.close()
    gm, gv = large_cases.golden_prediction(name)
    err = abs(ll - g["loglik"]) / abs(g["loglik"])
    em, ev = _pred_err(mean, gm), _pred_err(var, gv)
    print(f"{name} mixed loglik rel err {err:.3e} (d rel err {abs(d - g['d']) / abs(g['d']):.3e}); "
          f"prediction err mean {em:.3e} var {ev:.3e}")
    assert err <= MIXED_LL_GUARD, (ll, g["loglik"], err)
    assert em <= MIXED_PRED_GUARD and ev <= MIXED_PRED_GUARD
