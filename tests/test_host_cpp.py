"""The C++ drop-in host (include/mra_host.hpp, executable ``mra_b200``).

CPU: its partition builder gives, bit for bit, the structure of the Python
host (which is pinned to the reference by the golden tests).  GPU: run in the
reference's way -- a directory with user_parameters -- it prints the golden
log-likelihood and writes the golden prediction dump."""
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from nonstationary_mra_b200 import build, refio


@pytest.fixture(scope="module")
def exe():
    return build.build_host()


def read_dump(path):
    raw = open(path, "rb").read()
    head = np.frombuffer(raw, np.uint64, 7, 0).astype(np.int64)
    J, M, r, n_int, n_fin, n_obs, n_pred = (int(x) for x in head)
    off = 56
    out = {}

    def take(name, dtype, n):
        nonlocal off
        out[name] = np.frombuffer(raw, dtype, n, off).copy()
        off += 8 * n

    take("finest_parent", np.uint64, n_fin)
    take("knots", np.float64, 3 * n_int * r)
    take("obs_offset", np.uint64, n_fin + 1)
    take("obs", np.float64, 3 * n_obs)
    take("obs_value", np.float64, n_obs)
    if n_pred:
        take("pred_offset", np.uint64, n_fin + 1)
        take("pred", np.float64, 3 * n_pred)
    return (J, M, r, n_int), out


def case_copy(case_dir, tmp_path, mode):
    d = tmp_path / os.path.basename(case_dir)
    shutil.copytree(case_dir, d)
    P = refio.parse_parameters(str(d / "user_parameters"))
    P["CALCULATION_MODE"] = mode
    P["DUMP_PREDICTION_RESULTS_FLAG"] = "true"
    P["PREDICTION_RESULTS_FILE_NAME"] = "host_pred.bin"
    refio.write_parameters(str(d / "user_parameters"), P)
    return d


@pytest.mark.parametrize("mode", ["likelihood", "prediction"])
def test_structure_matches_python_host(exe, case_dir, tmp_path, mode):
    d = case_copy(case_dir, tmp_path, mode)
    out = tmp_path / "structure.bin"
    subprocess.run([exe, str(d), "--dump-structure", str(out)], check=True, capture_output=True, timeout=300)
    (J, M, r, n_int), cpp = read_dump(str(out))
    st, _, _ = refio.load_case(str(d), mode=mode)
    assert (J, M, r, n_int) == (st.J, st.M, st.r, st.n_interior)
    np.testing.assert_array_equal(cpp["finest_parent"], st.finest_parent)
    np.testing.assert_array_equal(cpp["knots"], np.ascontiguousarray(st.knots).reshape(-1))
    np.testing.assert_array_equal(cpp["obs_offset"], st.obs_offset)
    np.testing.assert_array_equal(cpp["obs"], np.ascontiguousarray(st.obs).reshape(-1))
    np.testing.assert_array_equal(cpp["obs_value"], st.obs_value)
    if mode == "prediction":
        np.testing.assert_array_equal(cpp["pred_offset"], st.pred_offset)
        np.testing.assert_array_equal(cpp["pred"], np.ascontiguousarray(st.pred).reshape(-1))


def test_missing_parameter_file_exits_with_the_reference_message(exe, tmp_path):
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Program exits with an error" in r.stdout


@pytest.mark.gpu
def test_likelihood_mode_prints_golden_value(exe, case_dir, tmp_path):
    g = json.load(open(os.path.join(case_dir, "golden.json")))
    d = case_copy(case_dir, tmp_path, "likelihood")
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    ll = float(re.search(r"The obtained loglikelihood is: (\S+)", r.stdout).group(1))
    dval = float(re.search(r"d=(\S+)", r.stdout).group(1))
    assert abs(dval - g["d"]) <= 1e-8 * max(1.0, abs(g["d"]))
    assert abs(ll - g["loglik"]) <= 1e-5 * abs(g["loglik"])  # printed with 6 significant digits


@pytest.mark.gpu
def test_prediction_mode_writes_golden_dump(exe, case_dir, tmp_path):
    d = case_copy(case_dir, tmp_path, "prediction")
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lon, lat, mean, var = refio.read_prediction_dump(str(d / "host_pred.bin"))
    glon, glat, gmean, gvar = refio.read_prediction_dump(os.path.join(case_dir, "pred_golden.bin"))
    np.testing.assert_array_equal(lon, glon)
    np.testing.assert_array_equal(lat, glat)
    scale = lambda a: np.maximum(1.0, np.abs(a))
    assert np.max(np.abs(mean - gmean) / scale(gmean)) <= 1e-6
    assert np.max(np.abs(var - gvar) / scale(gvar)) <= 1e-6
