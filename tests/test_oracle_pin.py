"""Pins the numpy oracle to the reference's own outputs (tests/golden, made by
running the reference's unmodified sources compiled in oracle/Makefile)."""
import json
import os

import numpy as np

import mra_oracle as oracle
from nonstationary_mra_b200 import refio


def test_loglik_matches_reference(case_dir):
    g = json.load(open(os.path.join(case_dir, "golden.json")))
    st, md, _ = oracle.load_case(case_dir, mode="likelihood")
    assert st.n_obs == g["n_obs"]
    d, ll = oracle.loglik(st, md)
    assert abs(d - g["d"]) <= 1e-10 * max(1.0, abs(g["d"]))
    assert abs(ll - g["loglik"]) <= 1e-10 * abs(g["loglik"])


def test_prediction_matches_reference(case_dir):
    st, md, _ = oracle.load_case(case_dir, mode="prediction")
    lon, lat, mean, var = refio.read_prediction_dump(os.path.join(case_dir, "pred_golden.bin"))
    m, v = oracle.predict(st, md)
    assert m.shape == mean.shape
    np.testing.assert_allclose(m, mean, rtol=1e-9, atol=1e-9 * np.abs(mean).max())
    np.testing.assert_allclose(v, var, rtol=1e-9, atol=1e-9 * np.abs(var).max())


def test_oracle_matches_reference_at_r64():
    """The restatement at the production shape (r = 64, clustered, M = 7): the
    regenerated r64_c2s_nu12 case against the reference's recorded outputs."""
    import tempfile
    import large_cases
    name = "r64_c2s_nu12"
    g = large_cases.golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        large_cases.write_inputs(tmp, name, "prediction")
        st, md, _ = oracle.load_case(tmp, mode="prediction")
    d, ll = oracle.loglik(st, md)
    assert abs(d - g["d"]) <= 1e-10 * max(1.0, abs(g["d"]))
    assert abs(ll - g["loglik"]) <= 1e-10 * abs(g["loglik"])
    m, v = oracle.predict(st, md)
    mean, var = large_cases.golden_prediction(name)
    np.testing.assert_allclose(m, mean, rtol=1e-9, atol=1e-9 * np.abs(mean).max())
    np.testing.assert_allclose(v, var, rtol=1e-9, atol=1e-9 * np.abs(var).max())
