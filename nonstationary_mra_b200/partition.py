"""Host-side partition builder (vectorised numpy).

Produces the flat Structure that the C ABI uploads once.  It reproduces the
reference's partition exactly -- same boxes, same knot coordinates (bit for
bit: the same floating-point operations in the same order), same assignment of
observations and prediction locations to finest regions, same order inside a
region -- but replaces the reference's O(N * R_finest) scan over finest boxes
(src/class_partition.cpp:525-556, 583-589) by descending the box tree once per
point, and its per-point ancestor-knot coincidence scan (:533-551) by a hashed
lookup.

  build_by_program     src/class_partition.cpp:459-654 (+ create_knots :24-44,
                       create_partitions :49-88, sizes :778-820)
  build_by_user_files  src/class_partition.cpp:93-454 with the finest-level
                       parents of read_parent_region_index (:659-770)
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .model import DIST_CHORDAL, Structure


def lonlat_to_xyz(lon: np.ndarray, lat: np.ndarray):
    """Unit-sphere coordinates (class_partition.cpp:262-270); degrees are
    converted as (deg * pi) / 180, the reference's evaluation order."""
    lat_r = lat * math.pi / 180
    lon_r = lon * math.pi / 180
    cl, sl = np.cos(lat_r), np.sin(lat_r)
    co, so = np.cos(lon_r), np.sin(lon_r)
    return cl * co, cl * so, sl


def _coords(lon, lat, distance):
    if distance == DIST_CHORDAL:
        return np.stack(lonlat_to_xyz(lon, lat))
    return np.stack([lon, lat, np.zeros_like(lon)])


def _n_interior(J: int, M: int) -> int:
    return (J ** (M - 1) - 1) // (J - 1)


def boxes(J: int, M: int, lon_all: np.ndarray, lat_all: np.ndarray):
    """Region boxes of every region (heap order), class_partition.cpp:49-88,476-490."""
    n_int = _n_interior(J, M)
    n_tot = n_int + J ** (M - 1)
    lo0, hi0 = np.empty(n_tot), np.empty(n_tot)
    lo1, hi1 = np.empty(n_tot), np.empty(n_tot)
    mnx, mxx = float(np.min(lon_all)), float(np.max(lon_all))
    mny, mxy = float(np.min(lat_all)), float(np.max(lat_all))
    lo0[0], hi0[0] = mnx, mxx + 1e-6 * (mxx - mnx)   # class_data.cpp:160-165
    lo1[0], hi1[0] = mny, mxy + 1e-6 * (mxy - mny)
    for m in range(M - 1):
        s = (J ** m - 1) // (J - 1)
        reg = np.arange(s, s + J ** m)
        a, b, c, d = lo0[reg], hi0[reg], lo1[reg], hi1[reg]
        if J == 2:
            split_lon = (b - a) >= (d - c)
            mid_lon = (b + a) / 2
            mid_lat = (d + c) / 2
            c1, c2 = 2 * reg + 1, 2 * reg + 2
            lo0[c1] = a
            hi0[c1] = np.where(split_lon, mid_lon, b)
            lo0[c2] = np.where(split_lon, mid_lon, a)
            hi0[c2] = b
            lo1[c1] = c
            hi1[c1] = np.where(split_lon, d, mid_lat)
            lo1[c2] = np.where(split_lon, c, mid_lat)
            hi1[c2] = d
        else:
            lm, tm = (b + a) / 2, (d + c) / 2
            ch = 4 * reg
            lo0[ch + 1], lo0[ch + 2], lo0[ch + 3], lo0[ch + 4] = a, lm, a, lm
            hi0[ch + 1], hi0[ch + 2], hi0[ch + 3], hi0[ch + 4] = lm, b, lm, b
            lo1[ch + 1], lo1[ch + 2], lo1[ch + 3], lo1[ch + 4] = c, c, tm, tm
            hi1[ch + 1], hi1[ch + 2], hi1[ch + 3], hi1[ch + 4] = tm, tm, d, d
    return lo0, hi0, lo1, hi1


def knots_in_boxes(lo0, hi0, lo1, hi1, n_regions: int, r_requested: int, offset: float):
    """create_knots (class_partition.cpp:24-44) for regions 0..n_regions-1."""
    nlon = int(math.ceil(math.sqrt(r_requested)))
    nlat = int(r_requested // nlon)
    a, b, c, d = lo0[:n_regions], hi0[:n_regions], lo1[:n_regions], hi1[:n_regions]
    off_lon, off_lat = (b - a) * offset, (d - c) * offset
    lon_start, lon_end = a + off_lon, b - off_lon
    lat_start, lat_end = c + off_lat, d - off_lat
    lon_inc = np.zeros_like(a) if nlon == 1 else (lon_end - lon_start) / (nlon - 1)
    lat_inc = np.zeros_like(c) if nlat == 1 else (lat_end - lat_start) / (nlat - 1)
    i = np.repeat(np.arange(nlon), nlat)       # knot index i*nlat + j
    j = np.tile(np.arange(nlat), nlon)
    klon = lon_end[:, None] - (nlon - i - 1)[None, :] * lon_inc[:, None]
    klat = lat_end[:, None] - (nlat - j - 1)[None, :] * lat_inc[:, None]
    return klon.reshape(-1), klat.reshape(-1), nlon * nlat


def assign_to_finest(J: int, M: int, lo0, hi0, lo1, hi1, lon, lat) -> np.ndarray:
    """Finest index of each point (-1 outside every box): the box containing it,
    lo <= p < hi in both coordinates, found by descending the tree."""
    idx = np.zeros(len(lon), dtype=np.int64)
    ok = np.ones(len(lon), dtype=bool)
    for _ in range(M - 1):
        nxt = np.full(len(lon), -1, dtype=np.int64)
        for c in range(1, J + 1):
            ch = idx * J + c
            ins = ok & (nxt < 0) & (lon >= lo0[ch]) & (lon < hi0[ch]) & (lat >= lo1[ch]) & (lat < hi1[ch])
            nxt = np.where(ins, ch, nxt)
        ok &= nxt >= 0
        idx = np.where(ok, nxt, 0)
    n_int = _n_interior(J, M)
    return np.where(ok, idx - n_int, -1)


def _pair_hash(lon: np.ndarray, lat: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(lon, dtype=np.float64).view(np.uint64)
    b = np.ascontiguousarray(lat, dtype=np.float64).view(np.uint64)
    return a * np.uint64(0x9E3779B97F4A7C15) ^ b


def _csr(fidx: np.ndarray, n_fin: int):
    order = np.argsort(fidx, kind="stable")
    counts = np.bincount(fidx, minlength=n_fin)
    off = np.zeros(n_fin + 1, dtype=np.int64)
    off[1:] = np.cumsum(counts)
    return order, off


def build_by_program(lon, lat, val, J: int, M: int, r_requested: int, offset: float,
                     pred_lon=None, pred_lat=None, distance: int = DIST_CHORDAL,
                     all_lon=None, all_lat=None) -> Structure:
    """Regular boxes and knot sub-grids, observations as finest-level knots.
    ``all_lon/all_lat``: every location of the data file (observed and NaN rows),
    which sets the domain (class_data.cpp:150-165)."""
    all_lon = lon if all_lon is None else all_lon
    all_lat = lat if all_lat is None else all_lat
    n_int = _n_interior(J, M)
    n_fin = J ** (M - 1)
    lo0, hi0, lo1, hi1 = boxes(J, M, all_lon, all_lat)
    klon, klat, r = knots_in_boxes(lo0, hi0, lo1, hi1, n_int, r_requested, offset)
    fidx = assign_to_finest(J, M, lo0, hi0, lo1, hi1, lon, lat)
    keep = fidx >= 0
    # drop observations that coincide with a knot of one of their ancestors (:533-551)
    kh = _pair_hash(klon, klat)
    cand = np.nonzero(keep & np.isin(_pair_hash(lon, lat), kh))[0]
    if cand.size:
        knot_regions = {}
        for q in np.nonzero(np.isin(kh, _pair_hash(lon[cand], lat[cand])))[0]:
            knot_regions.setdefault((klon[q], klat[q]), set()).add(q // r)
        for t in cand:
            regs = knot_regions.get((lon[t], lat[t]))
            if not regs:
                continue
            anc = n_int + int(fidx[t])
            for _ in range(M - 1):
                anc = (anc - 1) // J
                if anc in regs:
                    keep[t] = False
                    break
    rows = np.nonzero(keep)[0]
    order, off = _csr(fidx[rows], n_fin)
    sel = rows[order]
    st = Structure(J=J, M=M, r=r, n_interior=n_int, finest_parent=(np.arange(n_int, n_int + n_fin) - 1) // J,
                   knots=_coords(klon, klat, distance), obs_offset=off,
                   obs=_coords(lon[sel], lat[sel], distance), obs_value=np.asarray(val, dtype=np.float64)[sel],
                   obs_index=sel)
    if pred_lon is not None:
        pidx = assign_to_finest(J, M, lo0, hi0, lo1, hi1, pred_lon, pred_lat)
        prow = np.nonzero(pidx >= 0)[0]
        porder, poff = _csr(pidx[prow], n_fin)
        psel = prow[porder]
        st.pred_offset, st.pred = poff, _coords(pred_lon[psel], pred_lat[psel], distance)
        st.pred_index = psel
    return st


def build_by_user_files(lon, lat, val, obs_region, J: int, M: int, r: int, knots_lon, knots_lat, knots_region,
                        parent_start: int, parents, pred_lon=None, pred_lat=None, pred_region=None,
                        distance: int = DIST_CHORDAL) -> Structure:
    """User-provided knots and finest-level parents (PROVIDED_KNOTS_FLAG with
    VARIOUS_J_FINEST_LEVEL_FLAG): class_partition.cpp:93-454, 659-770."""
    n_int = _n_interior(J, M)
    if parent_start != n_int:
        raise ValueError(f"the first finest region must be {n_int} (regions 0..{n_int - 1} are interior)")
    n_fin = len(parents)
    klon = np.empty(n_int * r)
    klat = np.empty(n_int * r)
    i = 0
    kr = np.asarray(knots_region, dtype=np.int64)
    while i < len(kr) and kr[i] < n_int:   # class_partition.cpp:247-276
        reg = int(kr[i])
        klon[reg * r:(reg + 1) * r] = knots_lon[i:i + r]
        klat[reg * r:(reg + 1) * r] = knots_lat[i:i + r]
        i += r
    fidx = np.asarray(obs_region, dtype=np.int64) - n_int
    if np.any((fidx < 0) | (fidx >= n_fin)):
        raise ValueError("observation region index outside the finest level")
    order, off = _csr(fidx, n_fin)
    st = Structure(J=J, M=M, r=r, n_interior=n_int, finest_parent=np.asarray(parents, dtype=np.int64),
                   knots=_coords(klon, klat, distance), obs_offset=off,
                   obs=_coords(np.asarray(lon)[order], np.asarray(lat)[order], distance),
                   obs_value=np.asarray(val, dtype=np.float64)[order], obs_index=order)
    if pred_lon is not None:
        pidx = np.asarray(pred_region, dtype=np.int64) - n_int
        porder, poff = _csr(pidx, n_fin)
        st.pred_offset = poff
        st.pred = _coords(np.asarray(pred_lon)[porder], np.asarray(pred_lat)[porder], distance)
        st.pred_index = porder
    return st
