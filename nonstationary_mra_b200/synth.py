"""Seeded synthetic MRA configurations in the reference's file formats.

No public dataset is involved: the configurations are defined by their sizes
and distributions.  Locations live on [0,1]^2 (planar distance); the
nonstationary fields are

    log sigma^2(s) = 2 * (0 + sum_k a_k phi_k(s)),  a_k ~ N(0, 0.3^2)
    log beta(s)    = log 0.1 + sum_k b_k phi_k(s),   b_k ~ N(0, range_sd^2)
    tau^2          = 0.05 (intercept only)

with phi_k(s) = exp(-|s - c_k|^2 / (2 * 0.35^2)) on a 3x3 grid of centres
c_k in {1/6, 1/2, 5/6}^2.  The covariance is the Paciorek nonstationary
Matern with the d = 2 prefactor (b1 b2 / bbar^2)^1 and nu = 1/2 or 3/2.

Observation values are drawn from the MRA prior at these parameters
(``Context.sample_prior``); the prior's finest-level blocks carry tau^2 on
their diagonal, so the "+ N(0, tau^2)" noise is already included.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import refio
from .model import BASIS_GAUSSIAN, DIST_EUCLID2D, Field, Model


@dataclass
class Config:
    name: str
    n: int
    M: int
    J: int
    r: int
    nu_x2: int
    n_pred: int
    layout: str          # "uniform", "mix70" (70% of points in 16 clusters), "mix10"
    range_sd: float = 0.3
    seed: int = 0


CONFIGS = {
    # CPU-runnable plain FP64 case
    "c1": Config("c1", 8192, 4, 4, 16, 1, 1024, "uniform", 0.3, 1),
    # clustered, uneven regions: FP64 vs mixed
    "c2": Config("c2", 262144, 8, 4, 64, 1, 16384, "mix70", 0.3, 2),
    # large mixed-precision run (read as 90% uniform + 10% clustered), nu = 3/2
    "c3": Config("c3", 1048576, 10, 4, 64, 3, 65536, "mix10", 0.5, 3),
    # c2's layout at a quarter of the points and one level less: the size used for
    # full ncu captures (about 2 GB resident)
    "c2s": Config("c2s", 65536, 7, 4, 64, 1, 4096, "mix70", 0.3, 4),
}

RBF_CENTERS_1D = np.array([1.0 / 6, 0.5, 5.0 / 6])
RBF_WIDTH = 0.35


def rbf_centers() -> np.ndarray:
    gx, gy = np.meshgrid(RBF_CENTERS_1D, RBF_CENTERS_1D, indexing="ij")
    return np.stack([gx.reshape(-1), gy.reshape(-1)])


def locations(cfg: Config, rng: np.random.Generator):
    n = cfg.n
    if cfg.layout == "uniform":
        xy = rng.random((2, n))
    else:
        frac = 0.7 if cfg.layout == "mix70" else 0.1
        nc = int(round(frac * n))
        centres = rng.random((2, 16))
        which = rng.integers(0, 16, nc)
        cl = centres[:, which] + 0.03 * rng.standard_normal((2, nc))
        xy = np.concatenate([np.clip(cl, 0.0, 1.0), rng.random((2, n - nc))], axis=1)
        xy = xy[:, rng.permutation(n)]
    pred = rng.random((2, cfg.n_pred))
    return xy, pred


def true_theta(cfg: Config, rng: np.random.Generator) -> dict:
    a = 0.3 * rng.standard_normal(9)
    b = cfg.range_sd * rng.standard_normal(9)
    return {"log_sigma": a, "log_range": b, "log_tausq": np.log(0.05)}


def model_from_theta(theta: dict, nu_x2: int) -> Model:
    """Extension model for parameters (9 log-sigma, 9 log-range coefficients, log tau^2)."""
    c = rbf_centers()
    c3 = np.vstack([c, np.zeros((1, c.shape[1]))])
    md = Model(nonstationary=True, distance=DIST_EUCLID2D, nu_x2=nu_x2, prefactor_exp=1.0, dist_scale=1.0,
               basis=BASIS_GAUSSIAN, basis_len=RBF_WIDTH)
    md.fields = [Field(0.0, c3, 2.0 * np.asarray(theta["log_sigma"], dtype=np.float64)),
                 Field(float(np.log(0.1)), c3, np.asarray(theta["log_range"], dtype=np.float64)),
                 Field(float(theta["log_tausq"]), np.zeros((3, 0)), np.zeros(0))]
    return md


def theta_vector(theta: dict) -> np.ndarray:
    return np.concatenate([theta["log_sigma"], theta["log_range"], [theta["log_tausq"]]])


def theta_from_vector(v: np.ndarray) -> dict:
    v = np.asarray(v, dtype=np.float64)
    return {"log_sigma": v[:9], "log_range": v[9:18], "log_tausq": float(v[18])}


def log_sigma2_at(theta: dict, xy: np.ndarray) -> np.ndarray:
    """log sigma^2(s) of the synthetic model at points (2, n)."""
    c = rbf_centers()
    d2 = (xy[0][:, None] - c[0][None, :]) ** 2 + (xy[1][:, None] - c[1][None, :]) ** 2
    return 2.0 * (np.exp(-d2 / (2 * RBF_WIDTH ** 2)) @ np.asarray(theta["log_sigma"], dtype=np.float64))


def smooth_values(xy: np.ndarray, theta: dict, seed: int, n_features: int = 512, length: float = 0.1,
                  quantum: float = 2.0 ** -20) -> np.ndarray:
    """Observation values without the MRA prior: sigma(s) times a random
    Fourier-feature draw of a Gaussian field of length scale ``length``, plus
    N(0, tau^2) noise, rounded to multiples of ``quantum``.

    It is vectorised (seconds at n = 262,144) and its output is exactly
    reproducible across machines: the rounding absorbs last-bit differences of
    the vectorised cos/exp of different CPUs, so a run elsewhere gets bitwise the
    same values (callers check a digest)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    omega = rng.standard_normal((2, n_features)) / length
    phase = rng.uniform(0.0, 2.0 * np.pi, n_features)
    amp = rng.standard_normal(n_features) * np.sqrt(2.0 / n_features)
    noise = rng.standard_normal(xy.shape[1])
    g = np.empty(xy.shape[1])
    for s in range(0, xy.shape[1], 8192):       # bounded temporaries
        blk = xy[:, s:s + 8192]
        g[s:s + 8192] = np.cos(blk.T @ omega + phase) @ amp
    y = np.exp(0.5 * log_sigma2_at(theta, xy)) * g + np.sqrt(np.exp(theta["log_tausq"])) * noise
    return np.round(y / quantum) * quantum


def digest(*arrays) -> str:
    """Short SHA-256 of float64 arrays: proves two runs saw the same inputs."""
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()[:16]


def write_case(case_dir: str, cfg: Config, xy: np.ndarray, values: np.ndarray, pred: np.ndarray, theta: dict,
               mode: str = "likelihood") -> None:
    """user_parameters + ext_parameters + binary files for a config."""
    os.makedirs(case_dir, exist_ok=True)
    refio.write_data(os.path.join(case_dir, "data.bin"), xy[0], xy[1], values)
    refio.write_pred(os.path.join(case_dir, "pred.bin"), pred[0], pred[1])
    c = rbf_centers()
    refio.write_basis(os.path.join(case_dir, "log_sill.bin"), 0.0, c[0], c[1], 2.0 * theta["log_sigma"])
    refio.write_basis(os.path.join(case_dir, "log_range.bin"), float(np.log(0.1)), c[0], c[1], theta["log_range"])
    refio.write_basis(os.path.join(case_dir, "log_nugget.bin"), float(theta["log_tausq"]), np.zeros(0), np.zeros(0),
                      np.zeros(0))
    refio.write_parameters(os.path.join(case_dir, "user_parameters"), {
        "DATA_FILE_NAME": "data.bin", "ELIMINATION_DUPLICATES_FLAG": "false", "REGRESSION_FLAG": "false",
        "NONSTATIONARY_FLAG": "true", "OFFSET": "default", "NUM_PARTITIONS_J": cfg.J, "NUM_KNOTS_r": cfg.r,
        "NUM_LEVELS_M": cfg.M, "PRINT_DETAIL_FLAG": "false", "CALCULATION_MODE": mode,
        "PREDICTION_LOCATION_MODE": "A", "PREDICTION_LOCATION_FILE": "pred.bin",
        "DUMP_PREDICTION_RESULTS_FLAG": "true", "PREDICTION_RESULTS_FILE_NAME": "pred_out.bin",
        "SAVE_TO_DISK_FLAG": "false", "TMP_DIRECTORY": "", "DYNAMIC_SCHEDULE_FLAG": "true",
        "SIGMASQ": 1, "BETA": 0.1, "TAUSQ": 0.05, "MAX_ITERATIONS": 1000,
        "SIGMASQ_INITIAL_GUESS": 1, "SIGMASQ_LOWER_BOUND": 0.01, "SIGMASQ_UPPER_BOUND": 10,
        "BETA_INITIAL_GUESS": 0.1, "BETA_LOWER_BOUND": 0.01, "BETA_UPPER_BOUND": 1,
        "TAUSQ_INITIAL_GUESS": 0.05, "TAUSQ_LOWER_BOUND": 0.0, "TAUSQ_UPPER_BOUND": 1,
        "SIGMASQ_FILE_NAME": "log_sill.bin", "BETA_FILE_NAME": "log_range.bin", "TAUSQ_FILE_NAME": "log_nugget.bin",
        "SIGMASQ_SCALE": 1, "BETA_SCALE": 1, "TAUSQ_SCALE": 1, "CHORDAL_DISTANCE_FLAG": "false",
        "PROVIDED_KNOTS_FLAG": "false", "KNOTS_FILE_NAME": "", "OBS_AS_KNOTS_FLAG": "true",
        "NUM_KNOTS_FINEST": 1, "VARIOUS_J_FINEST_LEVEL_FLAG": "false", "PARENT_REGION_FILE_NAME": "",
        "WENDLAND_LEN": RBF_WIDTH,
    })
    refio.write_parameters(os.path.join(case_dir, "ext_parameters"), {
        "MRA_EXT_PLANAR": "true", "MRA_EXT_NU_X2": cfg.nu_x2, "MRA_EXT_PREFACTOR_EXP": 1.0,
        "MRA_EXT_BASIS": "gaussian"})
