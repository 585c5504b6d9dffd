"""The reference's file formats and its ``user_parameters`` configuration.

Binary layouts (all little-endian, u64 counts, f64 values):
  data file        u64 n; n lon; n lat; n value; [n u64 region]   class_data.cpp:47-143
  prediction file  u64 n; n lon; n lat; [n u64 region]            class_data.cpp:240-318
  basis file       u64 m; f64 intercept; m lon; m lat; m weight   class_nonstationary_covariance.cpp:80-200
  knots file       u64 k; k lon; k lat; k u64 region              class_partition.cpp:126-203
  parent file      u64 start; u64 end; (end-start+1) u64 parent    class_partition.cpp:685-734
  prediction dump  u64 n; n lon; n lat; n mean; n variance         class_approximation.cpp:493-535
``user_parameters``: KEY=value lines, '#' comments, spaces/tabs/quotes ignored
(read_user_parameters.cpp:10-50).  Opt-in extension keys live in a separate
``ext_parameters`` file of the same format so that the file stays readable by
the reference, which rejects unknown keys (read_user_parameters.cpp:326-329).
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np

from . import partition
from .model import (BASIS_GAUSSIAN, BASIS_WENDLAND, DIST_CHORDAL, DIST_EUCLID2D, DIST_GREAT_CIRCLE,
                    EARTH_RADIUS_KM, Field, Model)


def _u64(raw: bytes, off: int, n: int) -> np.ndarray:
    return np.frombuffer(raw, np.uint64, n, off).astype(np.int64)


def _f64(raw: bytes, off: int, n: int) -> np.ndarray:
    return np.frombuffer(raw, np.float64, n, off).copy()


def _need(raw: bytes, size: int, path: str, what: str):
    if len(raw) < size:
        raise ValueError(f"fail reading data file {path} for {what}. Double check the data file format.")


def read_data(path: str, with_region: bool):
    raw = open(path, "rb").read()
    _need(raw, 8, path, "the number of locations")
    n = int(_u64(raw, 0, 1)[0])
    _need(raw, 8 + 24 * n + (8 * n if with_region else 0), path, "locations and values")
    lon, lat, val = _f64(raw, 8, n), _f64(raw, 8 + 8 * n, n), _f64(raw, 8 + 16 * n, n)
    reg = _u64(raw, 8 + 24 * n, n) if with_region else None
    return lon, lat, val, reg


def read_pred(path: str, with_region: bool):
    raw = open(path, "rb").read()
    _need(raw, 8, path, "the number of locations")
    n = int(_u64(raw, 0, 1)[0])
    _need(raw, 8 + 16 * n + (8 * n if with_region else 0), path, "prediction locations")
    return _f64(raw, 8, n), _f64(raw, 8 + 8 * n, n), (_u64(raw, 8 + 16 * n, n) if with_region else None)


def read_basis(path: str):
    raw = open(path, "rb").read()
    _need(raw, 16, path, "the number of basis functions and the intercept")
    m = int(_u64(raw, 0, 1)[0])
    _need(raw, 16 + 24 * m, path, "basis functions")
    return float(_f64(raw, 8, 1)[0]), _f64(raw, 16, m), _f64(raw, 16 + 8 * m, m), _f64(raw, 16 + 16 * m, m)


def read_knots(path: str):
    raw = open(path, "rb").read()
    _need(raw, 8, path, "the number of knots")
    k = int(_u64(raw, 0, 1)[0])
    _need(raw, 8 + 24 * k, path, "knots")
    return _f64(raw, 8, k), _f64(raw, 8 + 8 * k, k), _u64(raw, 8 + 16 * k, k)


def read_parents(path: str):
    raw = open(path, "rb").read()
    _need(raw, 16, path, "the region range")
    start, end = (int(x) for x in _u64(raw, 0, 2))
    _need(raw, 16 + 8 * (end - start + 1), path, "parent region indices")
    return start, end, _u64(raw, 16, end - start + 1)


def write_data(path: str, lon, lat, val, region=None):
    with open(path, "wb") as f:
        f.write(np.uint64(len(lon)).tobytes())
        for a in (lon, lat, val):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        if region is not None:
            f.write(np.ascontiguousarray(region, dtype=np.uint64).tobytes())


def write_pred(path: str, lon, lat, region=None):
    with open(path, "wb") as f:
        f.write(np.uint64(len(lon)).tobytes())
        for a in (lon, lat):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        if region is not None:
            f.write(np.ascontiguousarray(region, dtype=np.uint64).tobytes())


def write_basis(path: str, intercept: float, lon, lat, weight):
    with open(path, "wb") as f:
        f.write(np.uint64(len(weight)).tobytes())
        f.write(np.float64(intercept).tobytes())
        for a in (lon, lat, weight):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())


def write_prediction_dump(path: str, lon, lat, mean, var):
    with open(path, "wb") as f:
        f.write(np.uint64(len(mean)).tobytes())
        for a in (lon, lat, mean, var):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())


def read_prediction_dump(path: str):
    raw = open(path, "rb").read()
    n = int(_u64(raw, 0, 1)[0])
    a = np.frombuffer(raw, np.float64, 4 * n, 8).reshape(4, n)
    return a[0].copy(), a[1].copy(), a[2].copy(), a[3].copy()


def parse_parameters(path: str) -> dict:
    out = {}
    for line in open(path):
        s = line.lstrip(" \t")
        if not s or s[0] in "#\r\n":
            continue
        s = "".join(ch for ch in s.rstrip("\r\n") if ch not in " \t'\"")
        if "=" not in s:
            continue
        k, v = s.split("=", 1)
        if k:
            out[k] = v
    return out


def write_parameters(path: str, params: dict):
    with open(path, "w") as f:
        for k, v in params.items():
            f.write(f"{k}={v}\n")


def load_case(case_dir: str, mode: Optional[str] = None):
    """(Structure, Model, params) from a directory with ``user_parameters`` (and
    optionally ``ext_parameters``), following the reference's main()
    (src/main.cpp:93-113): load data, split NaN rows, load the fields, build
    the partition."""
    P = parse_parameters(os.path.join(case_dir, "user_parameters"))
    ext_path = os.path.join(case_dir, "ext_parameters")
    X = parse_parameters(ext_path) if os.path.exists(ext_path) else {}
    fp = lambda k: os.path.join(case_dir, P[k])
    flag = lambda k, d="false": P.get(k, d).lower() == "true"
    mode = mode or P.get("CALCULATION_MODE", "likelihood")
    provided = flag("PROVIDED_KNOTS_FLAG")
    chordal = flag("CHORDAL_DISTANCE_FLAG", "true")
    distance = DIST_CHORDAL if chordal else (DIST_EUCLID2D if X.get("MRA_EXT_PLANAR", "false") == "true"
                                             else DIST_GREAT_CIRCLE)
    lon, lat, val, reg = read_data(fp("DATA_FILE_NAME"), provided)
    ok = ~np.isnan(val)
    plon = plat = preg = None
    if mode == "prediction":
        pm = P.get("PREDICTION_LOCATION_MODE", "A")
        if pm == "A":
            plon, plat, preg = read_pred(fp("PREDICTION_LOCATION_FILE"), provided)
        elif pm == "N":
            plon, plat, preg = lon[~ok], lat[~ok], (reg[~ok] if provided else None)
        else:
            plon, plat, preg = lon.copy(), lat.copy(), (reg.copy() if provided else None)
    J, M, r = int(P["NUM_PARTITIONS_J"]), int(P["NUM_LEVELS_M"]), int(P["NUM_KNOTS_r"])
    if provided:
        klon, klat, kreg = read_knots(fp("KNOTS_FILE_NAME"))
        ps, _, par = read_parents(fp("PARENT_REGION_FILE_NAME"))
        st = partition.build_by_user_files(lon[ok], lat[ok], val[ok], reg[ok], J, M, r, klon, klat, kreg, ps, par,
                                           plon, plat, preg, distance)
        st.obs_index = np.nonzero(ok)[0][st.obs_index]
    else:
        off = P.get("OFFSET", "default")
        offset = math.exp(1) / 100 if off == "default" else float(off)
        st = partition.build_by_program(lon[ok], lat[ok], val[ok], J, M, r, offset, plon, plat, distance,
                                        all_lon=lon, all_lat=lat)
        st.obs_index = np.nonzero(ok)[0][st.obs_index]
    md = Model()
    md.nonstationary = flag("NONSTATIONARY_FLAG")
    md.distance = distance
    md.nu_x2 = int(X.get("MRA_EXT_NU_X2", "1"))
    md.prefactor_exp = float(X.get("MRA_EXT_PREFACTOR_EXP", "1.5"))
    md.dist_scale = 1.0 if distance == DIST_EUCLID2D else EARTH_RADIUS_KM
    md.basis = BASIS_GAUSSIAN if X.get("MRA_EXT_BASIS", "wendland") == "gaussian" else BASIS_WENDLAND
    md.basis_len = float(P.get("WENDLAND_LEN", "0.22"))
    md.sill, md.range_, md.nugget = (float(P.get(k, d)) for k, d in (("SIGMASQ", "1"), ("BETA", "1"), ("TAUSQ", "0")))
    md.sill_scale, md.range_scale, md.nugget_scale = (float(P.get(k, "1")) for k in
                                                      ("SIGMASQ_SCALE", "BETA_SCALE", "TAUSQ_SCALE"))
    if md.nonstationary:
        for key in ("SIGMASQ_FILE_NAME", "BETA_FILE_NAME", "TAUSQ_FILE_NAME"):
            icpt, blon, blat, w = read_basis(fp(key))
            md.fields.append(Field(icpt, _coords(blon, blat, distance), w))
    return st, md, P


def _coords(lon, lat, distance):
    if distance == DIST_CHORDAL:
        return np.stack(partition.lonlat_to_xyz(lon, lat))
    return np.stack([lon, lat, np.zeros_like(lon)])
