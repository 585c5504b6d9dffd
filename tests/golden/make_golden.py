"""Generates the golden fixtures under tests/golden/ (run in the build container).

Each fixture is a directory in the reference's own formats (``user_parameters``,
optional ``ext_parameters``, binary data/basis/knot files) plus the outputs of
the reference's own sources compiled here (oracle/Makefile -> oracle/_ref):

  golden.json       d (Approximation::loglikelihood after likelihood()) and the
                    log-likelihood, from CALCULATION_MODE=likelihood
  pred_golden.bin   the prediction dump (CALCULATION_MODE=prediction)

Cases:
  example         the reference's data/minimal_reproducible_example (user knots,
                  parents file, varying finest J, chordal, Wendland fields)
  ref_prog_j4     reference model, knots by program, J=4, M=4, r=9, NaN rows
  ref_gc_j2       great-circle distance, J=2, M=6, r=6 (3 x 2 knot grid)
  ref_stationary  NONSTATIONARY_FLAG=false, J=4, M=3, r=16
  ext_mix         extension model (planar, Gaussian fields, nu=1/2), clustered
                  points -> uneven and empty finest regions, J=4, M=4, r=16
  ext_nu32        extension model with nu=3/2, J=4, M=5, r=9
  c1              the full CPU-runnable configuration (n=8192, M=4, J=4, r=16)

Observation values are drawn from the MRA prior with the numpy oracle
(oracle/mra_oracle.sample_prior) from PCG64-seeded normals.

    python tests/golden/make_golden.py [--only NAME]
    python tests/golden/make_golden.py --large [--only NAME]   # r = 64 cases, see large_cases.py
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import mra_oracle as oracle  # noqa: E402
from nonstationary_mra_b200 import refio, synth  # noqa: E402

# the reference checkout (read only); override with MRA_REFERENCE=/path/to/nonstationary_mra
REFERENCE = os.environ.get("MRA_REFERENCE", "/root/reference")
REF_EXAMPLE = os.path.join(REFERENCE, "data", "minimal_reproducible_example")
REF_PARAMS = os.path.join(REFERENCE, "user_parameters")
MRA_REF = os.path.join(ROOT, "oracle", "_ref", "mra_ref")
MRA_REF_EXT = os.path.join(ROOT, "oracle", "_ref", "mra_ref_ext")


def ref_params(**over) -> dict:
    p = {
        "DATA_FILE_NAME": "data.bin", "ELIMINATION_DUPLICATES_FLAG": "false", "REGRESSION_FLAG": "false",
        "NONSTATIONARY_FLAG": "true", "OFFSET": "default", "NUM_PARTITIONS_J": 4, "NUM_KNOTS_r": 9,
        "NUM_LEVELS_M": 4, "PRINT_DETAIL_FLAG": "false", "CALCULATION_MODE": "likelihood",
        "PREDICTION_LOCATION_MODE": "A", "PREDICTION_LOCATION_FILE": "pred.bin",
        "DUMP_PREDICTION_RESULTS_FLAG": "true", "PREDICTION_RESULTS_FILE_NAME": "pred_out.bin",
        "SAVE_TO_DISK_FLAG": "false", "TMP_DIRECTORY": "", "DYNAMIC_SCHEDULE_FLAG": "true",
        "SIGMASQ": 2.0, "BETA": 300, "TAUSQ": 0.1, "MAX_ITERATIONS": 1000,
        "SIGMASQ_INITIAL_GUESS": 1, "SIGMASQ_LOWER_BOUND": 0.01, "SIGMASQ_UPPER_BOUND": 10,
        "BETA_INITIAL_GUESS": 0.1, "BETA_LOWER_BOUND": 0.01, "BETA_UPPER_BOUND": 1,
        "TAUSQ_INITIAL_GUESS": 0.05, "TAUSQ_LOWER_BOUND": 0.0, "TAUSQ_UPPER_BOUND": 1,
        "SIGMASQ_FILE_NAME": "log_sill.bin", "BETA_FILE_NAME": "log_range.bin", "TAUSQ_FILE_NAME": "log_nugget.bin",
        "SIGMASQ_SCALE": 1.1, "BETA_SCALE": 0.9, "TAUSQ_SCALE": 1.2, "CHORDAL_DISTANCE_FLAG": "true",
        "PROVIDED_KNOTS_FLAG": "false", "KNOTS_FILE_NAME": "", "OBS_AS_KNOTS_FLAG": "true",
        "NUM_KNOTS_FINEST": 1, "VARIOUS_J_FINEST_LEVEL_FLAG": "false", "PARENT_REGION_FILE_NAME": "",
        "WENDLAND_LEN": 0.22,
    }
    p.update(over)
    return p


def write_ref_case(d, rng, n, n_nan, n_pred, box, params, wendland_len=0.22):
    os.makedirs(d, exist_ok=True)
    lon = rng.uniform(box[0], box[1], n)
    lat = rng.uniform(box[2], box[3], n)
    val = np.zeros(n)
    val[rng.choice(n, n_nan, replace=False)] = np.nan
    refio.write_data(os.path.join(d, "data.bin"), lon, lat, val)
    refio.write_pred(os.path.join(d, "pred.bin"), rng.uniform(box[0], box[1], n_pred),
                     rng.uniform(box[2], box[3], n_pred))
    gl = np.linspace(box[0], box[1], 4)
    gt = np.linspace(box[2], box[3], 4)
    blon, blat = (a.reshape(-1) for a in np.meshgrid(gl, gt, indexing="ij"))
    for name, icpt, sd in (("log_sill.bin", 0.5, 0.3), ("log_range.bin", np.log(800.0), 0.3),
                           ("log_nugget.bin", np.log(0.05), 0.2)):
        refio.write_basis(os.path.join(d, name), icpt, blon, blat, sd * rng.standard_normal(blon.size))
    params = dict(params)
    params["WENDLAND_LEN"] = wendland_len
    refio.write_parameters(os.path.join(d, "user_parameters"), params)


def resample_values(d, seed):
    """Replace the observed values of the data file by a draw from the MRA prior."""
    st, md, P = oracle.load_case(d, mode="likelihood")
    rng = np.random.Generator(np.random.PCG64(seed))
    z_int = rng.standard_normal(st.n_interior * st.r)
    z_obs = rng.standard_normal(st.n_obs)
    y = oracle.sample_prior(st, md, z_int, z_obs)
    provided = P.get("PROVIDED_KNOTS_FLAG", "false") == "true"
    path = os.path.join(d, P["DATA_FILE_NAME"])
    lon, lat, val, reg = refio.read_data(path, provided)
    new = np.where(np.isnan(val), np.nan, 0.0)
    new[st.obs_index] = y
    refio.write_data(path, lon, lat, new, reg)


def run_reference(d, mode, threads=4, pred_npz=False, inputs=None):
    """Runs the reference build on the case in ``d`` (or, for the regenerated
    cases, on ``inputs(tmp)`` written into the scratch directory) and returns
    its ORACLE values."""
    ext = os.path.exists(os.path.join(d, "ext_parameters"))
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    if ext:
        X = refio.parse_parameters(os.path.join(d, "ext_parameters"))
        env.update({k: str(v) for k, v in X.items()})
    with tempfile.TemporaryDirectory() as tmp:
        if inputs is not None:
            inputs(tmp)
            ext = True
            X = refio.parse_parameters(os.path.join(tmp, "ext_parameters"))
            env.update({k: str(v) for k, v in X.items()})
        else:
            for f in os.listdir(d):
                shutil.copy(os.path.join(d, f), tmp)
        P = refio.parse_parameters(os.path.join(tmp, "user_parameters"))
        P["CALCULATION_MODE"] = mode
        refio.write_parameters(os.path.join(tmp, "user_parameters"), P)
        res = subprocess.run([MRA_REF_EXT if ext else MRA_REF], cwd=tmp, env=env, capture_output=True, text=True,
                             timeout=4 * 3600)
        if res.returncode != 0:
            raise RuntimeError(f"reference failed on {d}:\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
        out = {}
        for line in res.stdout.splitlines():
            if line.startswith("ORACLE"):
                for tok in line.split()[1:]:
                    k, v = tok.split("=")
                    out[k] = float(v)
        if mode == "prediction":
            dump = os.path.join(tmp, P["PREDICTION_RESULTS_FILE_NAME"])
            if pred_npz:
                _, _, mean, var = refio.read_prediction_dump(dump)
                np.savez(os.path.join(d, "pred_golden.npz"), mean=mean, var=var)
            else:
                shutil.copy(dump, os.path.join(d, "pred_golden.bin"))
        return out


def finish(d):
    lk = run_reference(d, "likelihood")
    pr = run_reference(d, "prediction")
    g = {"d": lk["d"], "loglik": lk["loglik"], "n_obs": int(lk["n_obs"]),
         "likelihood_seconds": lk["likelihood_seconds"], "predict_seconds": pr["predict_seconds"]}
    with open(os.path.join(d, "golden.json"), "w") as f:
        json.dump(g, f, indent=1)
    print(os.path.basename(d), g)


def case_example(d):
    os.makedirs(d, exist_ok=True)
    for f in os.listdir(REF_EXAMPLE):
        if f != "testTruth.bin":
            shutil.copy(os.path.join(REF_EXAMPLE, f), d)
    P = refio.parse_parameters(REF_PARAMS)
    for k, v in list(P.items()):
        if isinstance(v, str) and v.startswith("data/minimal_reproducible_example/"):
            P[k] = v.split("/")[-1]
    P["PREDICTION_RESULTS_FILE_NAME"] = "pred_out.bin"
    P["PRINT_DETAIL_FLAG"] = "false"
    refio.write_parameters(os.path.join(d, "user_parameters"), P)


def case_ref_prog_j4(d):
    rng = np.random.Generator(np.random.PCG64(11))
    write_ref_case(d, rng, 1800, 40, 300, (-10, 10, -6, 6), ref_params())
    resample_values(d, 111)


def case_ref_gc_j2(d):
    rng = np.random.Generator(np.random.PCG64(12))
    write_ref_case(d, rng, 700, 0, 150, (-4, 8, -5, 5),
                   ref_params(NUM_PARTITIONS_J=2, NUM_LEVELS_M=6, NUM_KNOTS_r=6, CHORDAL_DISTANCE_FLAG="false"),
                   wendland_len=0.3)
    resample_values(d, 112)


def case_ref_stationary(d):
    rng = np.random.Generator(np.random.PCG64(13))
    write_ref_case(d, rng, 1500, 0, 200, (-8, 8, -8, 8),
                   ref_params(NUM_LEVELS_M=3, NUM_KNOTS_r=16, NONSTATIONARY_FLAG="false"))
    resample_values(d, 113)


def synth_case(d, cfg, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    xy, pred = synth.locations(cfg, rng)
    theta = synth.true_theta(cfg, rng)
    synth.write_case(d, cfg, xy, np.zeros(xy.shape[1]), pred, theta)
    resample_values(d, seed + 100)


def case_ext_mix(d):
    synth_case(d, synth.Config("ext_mix", 3000, 4, 4, 16, 1, 200, "mix70", 0.3, 21), 21)


def case_ext_nu32(d):
    synth_case(d, synth.Config("ext_nu32", 2500, 5, 4, 9, 3, 150, "uniform", 0.5, 22), 22)


def case_c1(d):
    synth_case(d, synth.CONFIGS["c1"], 23)


CASES = {"example": case_example, "ref_prog_j4": case_ref_prog_j4, "ref_gc_j2": case_ref_gc_j2,
         "ref_stationary": case_ref_stationary, "ext_mix": case_ext_mix, "ext_nu32": case_ext_nu32, "c1": case_c1}


def make_large(name, threads):
    """A regenerated r = 64 case (tests/golden/large_cases.py): only the spec with
    the input digests, the reference's outputs and its predictions are kept."""
    import platform
    import large_cases
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    cfg = large_cases.SPECS[name]
    dig = {}
    lk = run_reference(d, "likelihood", threads, inputs=lambda tmp: dig.update(large_cases.write_inputs(tmp, name)))
    pr = run_reference(d, "prediction", threads, pred_npz=True,
                       inputs=lambda tmp: large_cases.write_inputs(tmp, name, "prediction"))
    spec = {"config": cfg.__dict__, "generator": "tests/golden/large_cases.py:generate", "digests": dig}
    with open(os.path.join(d, "spec.json"), "w") as f:
        json.dump(spec, f, indent=1)
    g = {"d": lk["d"], "loglik": lk["loglik"], "n_obs": int(lk["n_obs"]),
         "likelihood_seconds": lk["likelihood_seconds"], "predict_seconds": pr["predict_seconds"],
         "threads": threads, "cpu": platform.processor() or platform.machine()}
    with open(os.path.join(d, "golden.json"), "w") as f:
        json.dump(g, f, indent=1)
    print(name, g)


def main():
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    if "--large" in sys.argv:
        sys.path.insert(0, HERE)
        import large_cases
        threads = os.cpu_count() or 4
        for name in large_cases.SPECS:
            if not only or name == only:
                make_large(name, threads)
        return
    for name, fn in CASES.items():
        if only and name != only:
            continue
        d = os.path.join(HERE, name)
        if os.path.exists(d):
            shutil.rmtree(d)
        fn(d)
        finish(d)


if __name__ == "__main__":
    main()
