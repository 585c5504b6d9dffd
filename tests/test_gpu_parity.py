"""Parity of the CUDA path (through the C ABI) with the reference.

Tolerances (FP64 path): log-likelihood within 1e-8 relative, predictions within
1e-6 (absolute, scaled by max(1, |value|)); d (the reference's internal sum)
within 1e-8 of max(1, |d|).
"""
import json
import os

import numpy as np
import pytest

import mra_oracle as oracle
from nonstationary_mra_b200 import api, capi, refio
from nonstationary_mra_b200.model import Field, Model, Structure

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-8
PRED_TOL = 1e-6


def theta_of(md):
    return dict(sill=md.sill, range_=md.range_, nugget=md.nugget, sill_scale=md.sill_scale,
                range_scale=md.range_scale, nugget_scale=md.nugget_scale)


def run_loglik(st, md, **kw):
    ctx = api.Context(st, md, **kw)
    ctx.set_theta(**theta_of(md))
    return ctx, ctx.loglik()


def close_pred(a, b):
    scale = np.maximum(1.0, np.abs(b))
    return np.max(np.abs(a - b) / scale) <= PRED_TOL


def test_golden_loglik(case_dir):
    g = json.load(open(os.path.join(case_dir, "golden.json")))
    st, md, _ = refio.load_case(case_dir, mode="likelihood")
    ctx, (d, ll) = run_loglik(st, md)
    assert abs(ll - g["loglik"]) <= LL_RTOL * abs(g["loglik"]), (ll, g["loglik"])
    assert abs(d - g["d"]) <= LL_RTOL * max(1.0, abs(g["d"])), (d, g["d"])
    ctx.close()


def test_golden_predict(case_dir):
    st, md, _ = refio.load_case(case_dir, mode="prediction")
    lon, lat, mean, var = refio.read_prediction_dump(os.path.join(case_dir, "pred_golden.bin"))
    ctx = api.Context(st, md)
    ctx.set_theta(**theta_of(md))
    m, v = ctx.predict()
    assert m.shape == mean.shape
    assert close_pred(m, mean) and close_pred(v, var)
    ctx.close()


def random_case(seed, J, M, r, n, n_pred, clustered=False, nu_x2=1, nonstat=True):
    """Small planar structure with uneven (and some empty) finest regions."""
    rng = np.random.default_rng(seed)
    from nonstationary_mra_b200 import partition, synth
    if clustered:
        c = rng.random((2, 3))
        w = rng.integers(0, 3, n)
        xy = np.clip(c[:, w] + 0.04 * rng.standard_normal((2, n)), 0, 1)
    else:
        xy = rng.random((2, n))
    pxy = rng.random((2, n_pred)) * 0.98 + 0.01
    st = partition.build_by_program(xy[0], xy[1], rng.standard_normal(n), J, M, r, np.exp(1) / 100,
                                    pxy[0], pxy[1], distance=2, all_lon=xy[0], all_lat=xy[1])
    theta = synth.true_theta(synth.Config("t", n, M, J, r, nu_x2, n_pred, "uniform", 0.3), rng)
    md = synth.model_from_theta(theta, nu_x2)
    if not nonstat:
        md.nonstationary = False
        md.sill, md.range_, md.nugget = 1.3, 0.2, 0.07
    return st, md


def to_oracle(st, md):
    ost = oracle.Structure(J=st.J, M=st.M, r=st.r, n_interior=st.n_interior, finest_parent=st.finest_parent,
                           knots=st.knots, obs_offset=st.obs_offset, obs=st.obs, obs_value=st.obs_value,
                           pred_offset=st.pred_offset, pred=st.pred)
    omd = oracle.Model(nonstationary=md.nonstationary, distance=md.distance, nu_x2=md.nu_x2,
                       prefactor_exp=md.prefactor_exp, dist_scale=md.dist_scale, basis=md.basis,
                       basis_len=md.basis_len, fields=[oracle.Field(f.intercept, f.centers, f.weights)
                                                       for f in md.fields],
                       sill=md.sill, range_=md.range_, nugget=md.nugget, sill_scale=md.sill_scale,
                       range_scale=md.range_scale, nugget_scale=md.nugget_scale)
    return ost, omd


RANDOM_CASES = [
    # seed, J, M, r, n, n_pred, clustered, nu_x2, nonstationary
    (1, 4, 2, 16, 300, 40, False, 1, True),      # M = 2: root + finest only
    (2, 2, 5, 7, 500, 60, True, 1, True),        # odd r (7 -> 3x2 = 6 knots), J = 2, empty regions
    (3, 4, 3, 20, 2500, 30, True, 3, True),      # r = 20, large regions (> 64 rows), nu = 3/2
    (4, 4, 4, 9, 900, 50, False, 1, False),      # stationary
    (5, 2, 7, 4, 700, 80, True, 3, True),        # deep tree
    (6, 4, 5, 16, 3000, 200, True, 3, True),     # finest work items both batched and split; children up to 230
    (8, 4, 5, 16, 1200, 60, False, 3, True),     # finest children of about 5 observations: one warp per child
    (9, 4, 5, 12, 1500, 50, True, 1, True),      # clustered: per-warp, grouped and per-child paths side by side
    (10, 4, 3, 128, 3000, 40, True, 3, True),    # r = 120 (12 x 10 knots): factors and tiles beyond 64 rows
    (11, 2, 4, 96, 2000, 30, False, 1, True),    # r = 90, J = 2
    (12, 4, 3, 196, 4000, 40, False, 3, True),   # r = 196: blocked factorization, inverse by triangular solve
    (13, 2, 3, 256, 3000, 30, True, 1, True),    # r = 256, the largest supported
]


@pytest.mark.parametrize("case", RANDOM_CASES, ids=lambda c: f"s{c[0]}J{c[1]}M{c[2]}r{c[3]}")
def test_random_vs_oracle(case):
    st, md = random_case(*case)
    ost, omd = to_oracle(st, md)
    d_ref, ll_ref = oracle.loglik(ost, omd)
    ctx, (d, ll) = run_loglik(st, md)
    assert abs(ll - ll_ref) <= LL_RTOL * abs(ll_ref), (ll, ll_ref)
    m_ref, v_ref = oracle.predict(ost, omd)
    m, v = ctx.predict()
    assert close_pred(m, m_ref) and close_pred(v, v_ref)
    ctx.close()


def test_fields_and_covariance_blocks():
    st, md, _ = refio.load_case(os.path.join(os.path.dirname(__file__), "golden", "example"), mode="likelihood")
    ost, omd = to_oracle(st, md)
    th = dict(sill_scale=md.sill_scale, range_scale=md.range_scale, nugget_scale=md.nugget_scale)
    pts = st.obs[:, :57]
    f = api.eval_fields(md, th, pts)
    fo = oracle.field_values(omd, pts)
    for a, b in zip(f, fo):
        np.testing.assert_allclose(a, b, rtol=1e-13)
    q = st.knots[:, :12]
    c = api.eval_covariance(md, th, pts, q)
    co = oracle.cross_cov(omd, pts, fo, q, oracle.field_values(omd, q))
    np.testing.assert_allclose(c, co, rtol=1e-12, atol=1e-300)
    s = api.eval_covariance(md, th, pts)
    so = oracle.var_cov(omd, pts, fo)
    np.testing.assert_allclose(s, so, rtol=1e-12)


def test_sample_prior_matches_oracle():
    st, md = random_case(7, 4, 3, 9, 400, 10)
    ost, omd = to_oracle(st, md)
    rng = np.random.default_rng(3)
    zi = rng.standard_normal(st.n_interior * st.r)
    zo = rng.standard_normal(st.n_obs)
    ctx = api.Context(st, md)
    ctx.set_theta()
    y = ctx.sample_prior(zi, zo)
    np.testing.assert_allclose(y, oracle.sample_prior(ost, omd, zi, zo), rtol=1e-9, atol=1e-9)
    ctx.close()


def test_graph_replay_and_theta_updates():
    st, md = random_case(8, 4, 4, 16, 1500, 10, clustered=True)
    ctx = api.Context(st, md)
    ctx.set_theta(range_scale=1.0)
    d0, _ = ctx.loglik()
    ctx.capture_graph()
    d1, _ = ctx.loglik()
    assert d1 == d0   # the graph replays the same kernels: bitwise equal
    ctx.set_theta(range_scale=0.7)
    d2, _ = ctx.loglik()
    ost, omd = to_oracle(st, md)
    omd.range_scale = 0.7
    d_ref, _ = oracle.loglik(ost, omd)
    assert d2 != d0 and abs(d2 - d_ref) <= LL_RTOL * max(1.0, abs(d_ref))
    assert ctx.stats()["graph_replays"] >= 2
    # each prior level's time splits into its covariance-block launches and its
    # region launches, also when replayed from the graph
    prior = [l for l in ctx.stats()["launches"] if l["kernel"] == "prior_level"]
    assert len(prior) == st.M - 1
    assert all(0 < l["ms_cov"] < l["ms"] for l in prior), prior
    assert all(l["ms_cov"] == 0 for l in ctx.stats()["launches"] if l["kernel"] != "prior_level")
    ctx.close()


def test_prediction_graph_replay():
    """prior -> posterior -> predict captured in one graph: replays give bitwise
    the eager results, and follow theta changes without recapture."""
    st, md = random_case(13, 4, 4, 16, 1500, 120, clustered=True)
    ctx = api.Context(st, md)
    ctx.set_theta(range_scale=1.0)
    m0, v0 = ctx.predict()
    ctx.capture_graph()
    replays = ctx.stats()["graph_replays"]
    m1, v1 = ctx.predict()
    assert ctx.stats()["graph_replays"] == replays + 1
    assert np.array_equal(m0, m1) and np.array_equal(v0, v1)
    ctx.set_theta(range_scale=0.8)
    m2, v2 = ctx.predict()
    ost, omd = to_oracle(st, md)
    omd.range_scale = 0.8
    m_ref, v_ref = oracle.predict(ost, omd)
    assert not np.array_equal(m2, m0)
    assert close_pred(m2, m_ref) and close_pred(v2, v_ref)
    # the log-likelihood graph is still the one mra_loglik replays
    d, _ = ctx.loglik()
    d_ref, _ = oracle.loglik(ost, omd)
    assert abs(d - d_ref) <= LL_RTOL * max(1.0, abs(d_ref))
    ctx.close()


def test_terms_sum_to_d():
    st, md = random_case(14, 4, 5, 16, 3000, 10, clustered=True)
    ctx, (d, _) = run_loglik(st, md)
    t = ctx.terms()
    assert t.shape == (st.M,)
    assert abs(t.sum() - d) <= 1e-12 * max(1.0, abs(d))
    ctx.close()


def test_autotune_keeps_results_bitwise():
    st, md = random_case(12, 4, 4, 16, 1500, 10, clustered=True)
    ctx, (d0, _) = run_loglik(st, md)
    choice, ms = ctx.autotune(1)
    assert len(choice) == 3 and all(c in (1, 2, 4) for c in choice) and ms > 0
    assert ctx.loglik()[0] == d0
    ctx.close()


def test_deterministic():
    st, md = random_case(9, 4, 3, 16, 1200, 10, clustered=True)
    ctx, (d0, _) = run_loglik(st, md)
    for _ in range(3):
        assert ctx.loglik()[0] == d0
    ctx.close()


def test_non_spd_is_reported_not_faulted():
    # host-side fault injection: a NaN observation coordinate poisons one region's
    # Sigma; the Cholesky reports the region, the device keeps working
    st, md = random_case(10, 4, 3, 9, 300, 5)
    bad = np.array(st.obs, copy=True)
    k = int(np.argmax(np.diff(st.obs_offset)))
    bad[0, st.obs_offset[k]] = np.nan
    st_bad = Structure(**{**st.__dict__, "obs": bad})
    ctx = api.Context(st_bad, md)
    ctx.set_theta()
    with pytest.raises(capi.MRAError) as e:
        ctx.loglik()
    assert e.value.status == capi.MRA_ERR_NOT_SPD
    assert ctx.stats()["bad_region"] == st.n_interior + k
    ctx.close()
    ok = api.Context(st, md)
    ok.set_theta()
    ok.loglik()
    ok.close()


def test_bad_theta_rejected():
    st, md = random_case(11, 4, 3, 9, 200, 5)
    ctx = api.Context(st, md)
    with pytest.raises(capi.MRAError) as e:
        ctx.set_theta(sill_scale=float("nan"))
    assert e.value.status == capi.MRA_ERR_ARG
    ctx.close()


# ---------------------------------------------------------------------------
# mixed path: FP32 tensor-core prior and finest level, FP64 posterior
# ---------------------------------------------------------------------------
MIXED_LL_RTOL = 1e-6


def test_mixed_golden_loglik(case_dir):
    g = json.load(open(os.path.join(case_dir, "golden.json")))
    st, md, _ = refio.load_case(case_dir, mode="likelihood")
    ctx, (d, ll) = run_loglik(st, md, precision="mixed")
    err = abs(ll - g["loglik"]) / abs(g["loglik"])
    print(f"mixed loglik rel err {os.path.basename(case_dir)}: {err:.3e}")
    assert err <= MIXED_LL_RTOL, (ll, g["loglik"], err)
    ctx.close()


def test_mixed_golden_predict_error_report(case_dir):
    st, md, _ = refio.load_case(case_dir, mode="prediction")
    lon, lat, mean, var = refio.read_prediction_dump(os.path.join(case_dir, "pred_golden.bin"))
    ctx = api.Context(st, md, precision="mixed")
    ctx.set_theta(**theta_of(md))
    m, v = ctx.predict()
    em = np.max(np.abs(m - mean) / np.maximum(1.0, np.abs(mean)))
    ev = np.max(np.abs(v - var) / np.maximum(1.0, np.abs(var)))
    print(f"mixed prediction err {os.path.basename(case_dir)}: mean {em:.3e} var {ev:.3e}")
    assert em <= 1e-4 and ev <= 1e-4
    ctx.close()


@pytest.mark.parametrize("stages", ["", "prior", "finest"])
def test_mixed_stage_switch(stages, monkeypatch):
    """The mixed path's per-stage precision switch (MRA_MIXED_FP32): with neither
    stage in FP32 it runs the mixed schedule in FP64 and matches the oracle to the
    FP64 tolerance; with one stage in FP32 it stays within the mixed tolerance."""
    st, md = random_case(15, 4, 4, 16, 2000, 10, clustered=True)
    ost, omd = to_oracle(st, md)
    d_ref, ll_ref = oracle.loglik(ost, omd)
    monkeypatch.setenv("MRA_MIXED_FP32", stages)
    ctx, (d, ll) = run_loglik(st, md, precision="mixed")
    ctx.close()
    tol = LL_RTOL if stages == "" else MIXED_LL_RTOL
    assert abs(ll - ll_ref) <= tol * abs(ll_ref), (stages, ll, ll_ref)
