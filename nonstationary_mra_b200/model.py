"""Plain containers for a partition (Structure) and a covariance model (Model).

Structure mirrors what the reference's Partition holds for the hot path
(include/class_partition.hpp:16-61) as flat numpy arrays; Model mirrors the
nonstationary covariance (include/class_nonstationary_covariance.hpp:8-68)
plus the model switches of include/constants.hpp (NONSTATIONARY_FLAG,
CHORDAL_DISTANCE_FLAG, WENDLAND_LEN) and the opt-in extensions.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

EARTH_RADIUS_KM = 6371.0

DIST_CHORDAL = 0
DIST_GREAT_CIRCLE = 1
DIST_EUCLID2D = 2
BASIS_WENDLAND = 0
BASIS_GAUSSIAN = 1


@dataclass
class Field:
    """log f(s) = intercept + sum_k weights[k] * basis(|s - centers[:, k]| / basis_len)."""
    intercept: float
    centers: np.ndarray   # (3, nb)
    weights: np.ndarray   # (nb,)


@dataclass
class Model:
    nonstationary: bool = True
    distance: int = DIST_CHORDAL
    nu_x2: int = 1
    prefactor_exp: float = 1.5
    dist_scale: float = EARTH_RADIUS_KM
    basis: int = BASIS_WENDLAND
    basis_len: float = 0.22
    fields: list = field(default_factory=list)   # sill, range, nugget
    sill: float = 1.0
    range_: float = 1.0
    nugget: float = 0.0
    sill_scale: float = 1.0
    range_scale: float = 1.0
    nugget_scale: float = 1.0


@dataclass
class Structure:
    J: int
    M: int
    r: int
    n_interior: int
    finest_parent: np.ndarray   # (n_finest,) int64
    knots: np.ndarray           # (3, n_interior * r)
    obs_offset: np.ndarray      # (n_finest + 1,) int64
    obs: np.ndarray             # (3, n_obs)
    obs_value: np.ndarray       # (n_obs,)
    pred_offset: Optional[np.ndarray] = None
    pred: Optional[np.ndarray] = None
    obs_index: Optional[np.ndarray] = None    # original data-file row of each observation
    pred_index: Optional[np.ndarray] = None   # original row of each prediction location

    @property
    def n_finest(self) -> int:
        return int(self.finest_parent.shape[0])

    @property
    def n_obs(self) -> int:
        return int(self.obs_value.shape[0])

    @property
    def n_pred(self) -> int:
        return 0 if self.pred_offset is None else int(self.pred_offset[-1])
