"""FP64 numpy restatement of the reference MRA hot path -- TEST INFRASTRUCTURE.

This module is the CPU oracle.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it,
and only as the checker or the timed CPU baseline; the product never routes
through it.

It restates, in vectorised numpy, the algorithm of hhuang90/nonstationary_mra:

* partition building            src/class_partition.cpp:24-88 (knots, boxes),
                                :459-654 (by program), :93-454 (by user files),
                                :659-770 (finest-level parents), :778-963 (sizes)
* nonstationary parameter fields src/class_nonstationary_covariance.cpp:479-573
* covariance blocks             src/evaluate_covariance.cpp:56-313
* prior, levels 0..M-2          src/class_approximation.cpp:84-169
* prior, finest level           src/class_approximation-loop-regions-at-finest-level-in-prior.cpp:15-409
* w~ / A~ products              src/class_approximation.cpp:52-82
* posterior (log-likelihood)    src/class_approximation-posterior-inference.cpp:14-265,
                                src/class_approximation.cpp:186-306
* prediction                    src/class_approximation-predict.cpp:15-200

Extension models (opt-in, not in the reference): planar Euclidean distance on
[0,1]^2, Gaussian radial basis fields, Matern smoothness 3/2 and a Paciorek
prefactor exponent of d/2 with d = 2.  With the reference settings the
formulas reduce to the reference's exactly.

Pinning: tests/test_oracle_pin.py checks this module against outputs of the
reference's own sources compiled here (oracle/Makefile), stored as fixtures in
tests/golden/.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

EARTH_RADIUS_KM = 6371.0
TWO_PI_TRUNCATED = 2 * 3.14159265359  # the reference's constant, posterior-inference.cpp:244

DIST_CHORDAL = 0       # unit-sphere chord x 6371 (CHORDAL_DISTANCE_FLAG=true)
DIST_GREAT_CIRCLE = 1  # great circle on lon/lat degrees x 6371
DIST_EUCLID2D = 2      # extension: planar distance on (x, y)

BASIS_WENDLAND = 0     # reference: Wendland C4, support WENDLAND_LEN
BASIS_GAUSSIAN = 1     # extension: exp(-d^2 / 2), d = distance / width


# --------------------------------------------------------------------------
# model and structure containers
# --------------------------------------------------------------------------
@dataclass
class Field:
    """log(field) = intercept + sum_k weight_k * basis(dist(s, center_k) / len)."""
    intercept: float
    centers: np.ndarray            # (3, nb) coordinates in the point coordinate system
    weights: np.ndarray            # (nb,)


@dataclass
class Model:
    nonstationary: bool = True
    distance: int = DIST_CHORDAL
    nu_x2: int = 1                 # 2*nu: 1 -> exponential (reference), 3 -> Matern 3/2
    prefactor_exp: float = 1.5     # (b1 b2 / bbar^2)^e ; reference e = 1.5 (evaluate_covariance.cpp:222)
    dist_scale: float = EARTH_RADIUS_KM
    basis: int = BASIS_WENDLAND
    basis_len: float = 0.22
    fields: list = field(default_factory=list)   # [sill, range, nugget] Field objects
    # stationary parameters (NONSTATIONARY_FLAG=false) / nonstationary scales
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
    finest_parent: np.ndarray      # (n_finest,) interior index of each finest region's parent
    knots: np.ndarray              # (3, n_interior * r)
    obs_offset: np.ndarray         # (n_finest + 1,)
    obs: np.ndarray                # (3, n_obs)
    obs_value: np.ndarray          # (n_obs,)
    pred_offset: Optional[np.ndarray] = None
    pred: Optional[np.ndarray] = None
    obs_index: Optional[np.ndarray] = None     # data-file row of each observation

    @property
    def n_finest(self) -> int:
        return int(self.finest_parent.shape[0])

    @property
    def n_obs(self) -> int:
        return int(self.obs_value.shape[0])

    def level_start(self, m: int) -> int:
        J = self.J
        return (J ** m - 1) // (J - 1)

    def level_count(self, m: int) -> int:
        return self.J ** m

    def ancestors_of_interior(self, idx: np.ndarray, m: int) -> np.ndarray:
        """(len(idx), m) ancestors at levels 0..m-1 (class_approximation.cpp:36-43)."""
        out = np.zeros((len(idx), m), dtype=np.int64)
        cur = np.asarray(idx, dtype=np.int64).copy()
        for a in range(m - 1, -1, -1):
            cur = (cur - 1) // self.J
            out[:, a] = cur
        return out

    def ancestors_of_finest(self, k: int) -> np.ndarray:
        L = self.M - 1
        anc = np.zeros(L, dtype=np.int64)
        anc[L - 1] = self.finest_parent[k]
        if L > 1:
            anc[:L - 1] = self.ancestors_of_interior(np.array([anc[L - 1]]), L - 1)[0]
        return anc


# --------------------------------------------------------------------------
# fields and covariance (class_nonstationary_covariance.cpp, evaluate_covariance.cpp)
# --------------------------------------------------------------------------
def lonlat_to_xyz(lon, lat):
    """Unit-sphere coordinates, class_partition.cpp:262-270."""
    cl, sl = np.cos(lat * math.pi / 180), np.sin(lat * math.pi / 180)
    co, so = np.cos(lon * math.pi / 180), np.sin(lon * math.pi / 180)
    return cl * co, cl * so, sl


def pair_distance(p1: np.ndarray, p2: np.ndarray, kind: int) -> np.ndarray:
    """Unscaled distance between every column of p1 (3,n1) and p2 (3,n2) -> (n1, n2)."""
    if kind == DIST_CHORDAL:
        d = (p2[0][None, :] - p1[0][:, None]) ** 2 + (p2[1][None, :] - p1[1][:, None]) ** 2 \
            + (p2[2][None, :] - p1[2][:, None]) ** 2
        return np.sqrt(d)
    if kind == DIST_GREAT_CIRCLE:
        lon1, lat1 = p1[0][:, None] * math.pi / 180, p1[1][:, None] * math.pi / 180
        lon2, lat2 = p2[0][None, :] * math.pi / 180, p2[1][None, :] * math.pi / 180
        ang = np.sin(lat1) * np.sin(lat2) + np.cos(lat1) * np.cos(lat2) * np.cos(lon1 - lon2)
        return np.arccos(np.clip(ang, -1.0, 1.0))
    if kind == DIST_EUCLID2D:
        d = (p2[0][None, :] - p1[0][:, None]) ** 2 + (p2[1][None, :] - p1[1][:, None]) ** 2
        return np.sqrt(d)
    raise ValueError(kind)


def field_values(model: Model, pts: np.ndarray) -> tuple:
    """(sigma^2, beta, tau^2) at points (3, n), scales applied as in
    evaluate_covariance.cpp:166-190,254-270."""
    n = pts.shape[1]
    if not model.nonstationary:
        return (np.full(n, model.sill), np.full(n, model.range_), np.full(n, model.nugget))
    out = []
    for f, scale in zip(model.fields, (model.sill_scale, model.range_scale, model.nugget_scale)):
        val = np.full(n, float(f.intercept))
        if f.weights.size:
            d = pair_distance(pts, f.centers, model.distance) / model.basis_len
            if model.basis == BASIS_WENDLAND:
                dd = np.where(d < 1, d, 1.0)
                phi = np.where(d < 1, (1 - dd) ** 6 * (35 * dd * dd + 18 * dd + 3) / 3, 0.0)
            else:
                phi = np.exp(-0.5 * d * d)
            val = val + phi @ f.weights
        out.append(scale * np.exp(val))
    return tuple(out)


def matern_kernel(h: np.ndarray, nu_x2: int) -> np.ndarray:
    if nu_x2 == 1:
        return np.exp(-h)
    if nu_x2 == 3:
        s = math.sqrt(3.0) * h
        return (1 + s) * np.exp(-s)
    raise ValueError(nu_x2)


def cross_cov(model: Model, p1, f1, p2, f2) -> np.ndarray:
    """C(S1, S2) as an (n1, n2) array; the reference stores it row-major as
    out[i1*n2 + i2] (evaluate_covariance.cpp:82,225), i.e. column-major n2 x n1."""
    D = model.dist_scale * pair_distance(p1, p2, model.distance)
    s1, b1 = f1[0][:, None], f1[1][:, None]
    s2, b2 = f2[0][None, :], f2[1][None, :]
    if not model.nonstationary:
        return s1 * matern_kernel(D / b1, model.nu_x2) * np.ones_like(s2)
    bms = (b1 * b1 + b2 * b2) / 2
    bp = b1 * b2
    return np.sqrt(s1 * s2) * (bp / bms) ** model.prefactor_exp * matern_kernel(D / np.sqrt(bms), model.nu_x2)


def var_cov(model: Model, p, f) -> np.ndarray:
    """Symmetric self block with sigma^2 + tau^2 on the diagonal (evaluate_covariance.cpp:103,307)."""
    C = cross_cov(model, p, f, p, f)
    np.fill_diagonal(C, f[0] + f[2])
    return C


# --------------------------------------------------------------------------
# partition (class_partition.cpp) and reference binary formats
# --------------------------------------------------------------------------
def read_data_file(path, with_region: bool):
    """u64 n; n lon; n lat; n value; [n u64 region] (class_data.cpp:47-143)."""
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    arr = np.frombuffer(raw[8:8 + 24 * n], np.float64).reshape(3, n)
    reg = np.frombuffer(raw[8 + 24 * n:8 + 32 * n], np.uint64).astype(np.int64) if with_region else None
    return arr[0].copy(), arr[1].copy(), arr[2].copy(), reg


def read_pred_file(path, with_region: bool):
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    arr = np.frombuffer(raw[8:8 + 16 * n], np.float64).reshape(2, n)
    reg = np.frombuffer(raw[8 + 16 * n:8 + 24 * n], np.uint64).astype(np.int64) if with_region else None
    return arr[0].copy(), arr[1].copy(), reg


def read_basis_file(path):
    """u64 m; f64 intercept; m lon; m lat; m weight (class_nonstationary_covariance.cpp:80-200)."""
    raw = open(path, "rb").read()
    m = int(np.frombuffer(raw[:8], np.uint64)[0])
    icpt = float(np.frombuffer(raw[8:16], np.float64)[0])
    arr = np.frombuffer(raw[16:16 + 24 * m], np.float64).reshape(3, m)
    return icpt, arr[0].copy(), arr[1].copy(), arr[2].copy()


def read_knots_file(path):
    """u64 k; k lon; k lat; k u64 region (class_partition.cpp:126-203)."""
    raw = open(path, "rb").read()
    k = int(np.frombuffer(raw[:8], np.uint64)[0])
    arr = np.frombuffer(raw[8:8 + 16 * k], np.float64).reshape(2, k)
    reg = np.frombuffer(raw[8 + 16 * k:8 + 24 * k], np.uint64).astype(np.int64)
    return arr[0].copy(), arr[1].copy(), reg


def read_parent_file(path):
    """u64 start; u64 end; (end-start+1) u64 parents (class_partition.cpp:685-734)."""
    raw = open(path, "rb").read()
    start, end = (int(x) for x in np.frombuffer(raw[:16], np.uint64))
    par = np.frombuffer(raw[16:16 + 8 * (end - start + 1)], np.uint64).astype(np.int64)
    return start, end, par


def _create_knots(lonMin, lonMax, nLon, latMin, latMax, nLat, offset):
    """class_partition.cpp:24-44, same floating-point operation order."""
    offLon = (lonMax - lonMin) * offset
    offLat = (latMax - latMin) * offset
    lonStart, lonEnd = lonMin + offLon, lonMax - offLon
    latStart, latEnd = latMin + offLat, latMax - offLat
    lonInc = 0.0 if nLon == 1 else (lonEnd - lonStart) / (nLon - 1)
    latInc = 0.0 if nLat == 1 else (latEnd - latStart) / (nLat - 1)
    lon = np.empty(nLon * nLat)
    lat = np.empty(nLon * nLat)
    for i in range(nLon):
        for j in range(nLat):
            lon[i * nLat + j] = lonEnd - (nLon - i - 1) * lonInc
            lat[i * nLat + j] = latEnd - (nLat - j - 1) * latInc
    return lon, lat


def build_structure_by_program(lon, lat, val, J, M, r_requested, offset,
                               pred_lon=None, pred_lat=None, distance=DIST_CHORDAL,
                               all_lon=None, all_lat=None) -> Structure:
    """build_partition_by_program (class_partition.cpp:459-654) with the sizes of
    Partition() (:778-820).  ``all_lon/all_lat`` are every location of the data
    file (observations and NaN rows), which set the domain (class_data.cpp:150-165)."""
    all_lon = lon if all_lon is None else all_lon
    all_lat = lat if all_lat is None else all_lat
    nLon = int(math.ceil(math.sqrt(r_requested)))
    nLat = int(r_requested // nLon)
    r = nLon * nLat
    n_int = (J ** (M - 1) - 1) // (J - 1)
    n_fin = J ** (M - 1)
    n_tot = n_int + n_fin
    lonMin = np.empty(n_tot); lonMax = np.empty(n_tot); latMin = np.empty(n_tot); latMax = np.empty(n_tot)
    mnLon, mxLon = float(np.min(all_lon)), float(np.max(all_lon))
    mnLat, mxLat = float(np.min(all_lat)), float(np.max(all_lat))
    lonMin[0] = mnLon; lonMax[0] = mxLon + 1e-6 * (mxLon - mnLon)
    latMin[0] = mnLat; latMax[0] = mxLat + 1e-6 * (mxLat - mnLat)
    for reg in range(n_int):  # create_partitions, :49-88
        a, b, c, d = lonMin[reg], lonMax[reg], latMin[reg], latMax[reg]
        if J == 2:
            if (b - a) >= (d - c):
                mid = (b + a) / 2
                lonMin[2 * reg + 1], lonMin[2 * reg + 2] = a, mid
                lonMax[2 * reg + 1], lonMax[2 * reg + 2] = mid, b
                latMin[2 * reg + 1] = latMin[2 * reg + 2] = c
                latMax[2 * reg + 1] = latMax[2 * reg + 2] = d
            else:
                mid = (d + c) / 2
                lonMin[2 * reg + 1] = lonMin[2 * reg + 2] = a
                lonMax[2 * reg + 1] = lonMax[2 * reg + 2] = b
                latMin[2 * reg + 1], latMin[2 * reg + 2] = c, mid
                latMax[2 * reg + 1], latMax[2 * reg + 2] = mid, d
        else:
            lm, tm = (b + a) / 2, (d + c) / 2
            ch = 4 * reg
            lonMin[ch + 1:ch + 5] = (a, lm, a, lm)
            lonMax[ch + 1:ch + 5] = (lm, b, lm, b)
            latMin[ch + 1:ch + 5] = (c, c, tm, tm)
            latMax[ch + 1:ch + 5] = (tm, tm, d, d)
    klon = np.empty(n_int * r); klat = np.empty(n_int * r)
    for reg in range(n_int):
        a, b = _create_knots(lonMin[reg], lonMax[reg], nLon, latMin[reg], latMax[reg], nLat, offset)
        klon[reg * r:(reg + 1) * r] = a
        klat[reg * r:(reg + 1) * r] = b

    def assign(plon, plat):
        # the finest box holding each point (lo <= p < hi), -1 when none does:
        # such points are never collected by the reference's scan (:525-556, 583-589)
        out = np.full(len(plon), -1, dtype=np.int64)
        for t in range(len(plon)):
            for k in range(n_fin):
                reg = n_int + k
                if lonMin[reg] <= plon[t] < lonMax[reg] and latMin[reg] <= plat[t] < latMax[reg]:
                    out[t] = k
                    break
        return out

    fidx = assign(lon, lat)
    inside = fidx >= 0
    # skip observations that coincide with a knot of an ancestor (:533-551)
    keep = inside.copy()
    knot_set = {}
    for reg in range(n_int):
        for q in range(r):
            knot_set.setdefault((klon[reg * r + q], klat[reg * r + q]), set()).add(reg)
    for t in range(len(lon)):
        key = (lon[t], lat[t])
        if keep[t] and key in knot_set:
            anc = n_int + fidx[t]
            regs = knot_set[key]
            for _ in range(M - 1):
                anc = (anc - 1) // J
                if anc in regs:
                    keep[t] = False
                    break
    order = np.argsort(fidx[keep], kind="stable")
    sel = np.nonzero(keep)[0][order]
    counts = np.bincount(fidx[sel], minlength=n_fin)
    off = np.zeros(n_fin + 1, dtype=np.int64); off[1:] = np.cumsum(counts)
    parent = (np.arange(n_int, n_tot) - 1) // J

    def coords(plon, plat):
        if distance == DIST_CHORDAL:
            return np.stack(lonlat_to_xyz(plon, plat))
        return np.stack([plon, plat, np.zeros_like(plon)])

    st = Structure(J=J, M=M, r=r, n_interior=n_int, finest_parent=parent,
                   knots=coords(klon, klat), obs_offset=off, obs=coords(lon[sel], lat[sel]),
                   obs_value=val[sel].copy(), obs_index=sel)
    if pred_lon is not None:
        pidx = assign(pred_lon, pred_lat)
        prow = np.nonzero(pidx >= 0)[0]
        porder = prow[np.argsort(pidx[prow], kind="stable")]
        pc = np.bincount(pidx[prow], minlength=n_fin)
        poff = np.zeros(n_fin + 1, dtype=np.int64); poff[1:] = np.cumsum(pc)
        st.pred_offset = poff
        st.pred = coords(pred_lon[porder], pred_lat[porder])
    return st


def build_structure_by_user_files(lon, lat, val, obs_region, J, M, r, knots_lon, knots_lat, knots_region,
                                  parent_start, parents, pred_lon=None, pred_lat=None, pred_region=None,
                                  distance=DIST_CHORDAL) -> Structure:
    """build_partition_by_user_files (class_partition.cpp:93-454) with
    VARIOUS_J_FINEST_LEVEL_FLAG parents (:659-770)."""
    n_int = (J ** (M - 1) - 1) // (J - 1)
    if parent_start != n_int:
        raise ValueError("finest regions must start right after the interior regions")
    n_fin = len(parents)
    klon = np.empty(n_int * r); klat = np.empty(n_int * r)
    i = 0
    while i < len(knots_region) and knots_region[i] < n_int:
        reg = knots_region[i]
        klon[reg * r:(reg + 1) * r] = knots_lon[i:i + r]
        klat[reg * r:(reg + 1) * r] = knots_lat[i:i + r]
        i += r
    fidx = obs_region - n_int
    order = np.argsort(fidx, kind="stable")
    counts = np.bincount(fidx, minlength=n_fin)
    off = np.zeros(n_fin + 1, dtype=np.int64); off[1:] = np.cumsum(counts)

    def coords(plon, plat):
        if distance == DIST_CHORDAL:
            return np.stack(lonlat_to_xyz(plon, plat))
        return np.stack([plon, plat, np.zeros_like(plon)])

    st = Structure(J=J, M=M, r=r, n_interior=n_int, finest_parent=np.asarray(parents, dtype=np.int64),
                   knots=coords(klon, klat), obs_offset=off, obs=coords(lon[order], lat[order]),
                   obs_value=val[order].copy(), obs_index=order)
    if pred_lon is not None:
        pidx = pred_region - n_int
        porder = np.argsort(pidx, kind="stable")
        pc = np.bincount(pidx, minlength=n_fin)
        poff = np.zeros(n_fin + 1, dtype=np.int64); poff[1:] = np.cumsum(pc)
        st.pred_offset = poff
        st.pred = coords(pred_lon[porder], pred_lat[porder])
    return st


# --------------------------------------------------------------------------
# the MRA (class_approximation*.cpp)
# --------------------------------------------------------------------------
def _trsm(L, B):
    """L^{-1} B for a batch of lower-triangular L."""
    return np.linalg.solve(L, B)


class MRA:
    """Prior -> posterior -> prediction on a Structure, FP64."""

    def __init__(self, st: Structure, model: Model):
        self.st, self.model = st, model

    # ---- prior, levels 0..M-2 : class_approximation.cpp:84-169
    def prior_interior(self):
        st, md = self.st, self.model
        r = st.r
        kf = field_values(md, st.knots)
        self.kf = kf
        L = np.zeros((st.n_interior, r, r))
        U = {}          # level m -> (count, m, r, r): U[i][l] = KCholTimesw[i][l]
        for m in range(st.M - 1):
            s0, cnt = st.level_start(m), st.level_count(m)
            idx = np.arange(s0, s0 + cnt)
            anc = st.ancestors_of_interior(idx, m)
            Um = np.zeros((cnt, m, r, r))
            for q in range(cnt):
                i = idx[q]
                pi = st.knots[:, i * r:(i + 1) * r]
                fi = tuple(f[i * r:(i + 1) * r] for f in kf)
                for j in range(m):
                    a = anc[q, j]
                    pa = st.knots[:, a * r:(a + 1) * r]
                    fa = tuple(f[a * r:(a + 1) * r] for f in kf)
                    # column-major (r_anc x r_own) block == C(S_own, S_anc) transposed
                    V = cross_cov(md, pi, fi, pa, fa).T.copy()
                    a_local = a - st.level_start(j)
                    for l in range(j):
                        V -= U[j][a_local, l].T @ Um[q, l]
                    Um[q, j] = _trsm(L[a], V)
                K = var_cov(md, pi, fi)
                for l in range(m):
                    K -= Um[q, l].T @ Um[q, l]
                L[i] = np.linalg.cholesky(K)
            U[m] = Um
        self.L_prior = L.copy()
        self.U = U

    # ---- prior, finest level : ...-prior.cpp:90-269 (+ prediction half :271-392)
    def prior_finest(self, prediction: bool):
        st, md = self.st, self.model
        r, Lv = st.r, st.M - 1
        of = field_values(md, st.obs)
        self.d_finest = 0.0
        self.fin = []
        pf = field_values(md, st.pred) if (prediction and st.pred is not None) else None
        for k in range(st.n_finest):
            a0, a1 = st.obs_offset[k], st.obs_offset[k + 1]
            n = a1 - a0
            anc = st.ancestors_of_finest(k)
            rec = {"n": n, "anc": anc}
            ps = st.obs[:, a0:a1]
            fs = tuple(f[a0:a1] for f in of)
            if n > 0:
                Ufin = np.zeros((Lv, r, n))
                Vsave = np.zeros((Lv, r, n))
                for j in range(Lv):
                    a = anc[j]
                    pa = st.knots[:, a * r:(a + 1) * r]
                    fa = tuple(f[a * r:(a + 1) * r] for f in self.kf)
                    V = cross_cov(md, ps, fs, pa, fa).T.copy()      # r x n
                    a_local = a - st.level_start(j)
                    for l in range(j):
                        V -= self.U[j][a_local, l].T @ Ufin[l]
                    Vsave[j] = V
                    Ufin[j] = _trsm(self.L_prior[a], V)
                S = var_cov(md, ps, fs)
                for l in range(Lv):
                    S -= Ufin[l].T @ Ufin[l]
                LS = np.linalg.cholesky(S)
                yt = np.linalg.solve(LS, st.obs_value[a0:a1])
                B = np.stack([np.linalg.solve(LS, Vsave[j].T) for j in range(Lv)])  # (Lv, n, r)
                self.d_finest += float(yt @ yt + 2 * np.sum(np.log(np.diag(LS))))
                rec.update(Ufin=Ufin, LS=LS, yt=yt, B=B)
            if prediction and st.pred is not None:
                b0, b1 = st.pred_offset[k], st.pred_offset[k + 1]
                npred = b1 - b0
                rec["np"] = npred
                if npred > 0:
                    pp = st.pred[:, b0:b1]
                    fp = tuple(f[b0:b1] for f in pf)
                    P = np.zeros((Lv, r, npred))
                    Bt = np.zeros((Lv, r, npred))
                    for j in range(Lv):
                        a = anc[j]
                        pa = st.knots[:, a * r:(a + 1) * r]
                        fa = tuple(f[a * r:(a + 1) * r] for f in self.kf)
                        C = cross_cov(md, pp, fp, pa, fa).T.copy()
                        a_local = a - st.level_start(j)
                        for l in range(j):
                            C -= self.U[j][a_local, l].T @ P[l]
                        Bt[j] = C
                        P[j] = _trsm(self.L_prior[a], C)
                    Cpp = var_cov(md, pp, fp)
                    var = np.diag(Cpp).copy() - np.sum(P * P, axis=(0, 1))
                    mean = np.zeros(npred)
                    if n > 0:
                        Pc = cross_cov(md, pp, fp, ps, fs).T.copy()   # n x np
                        for l in range(Lv):
                            Pc -= rec["Ufin"][l].T @ P[l]
                        Pc = np.linalg.solve(rec["LS"], Pc)
                        var -= np.sum(Pc * Pc, axis=0)
                        mean = Pc.T @ rec["yt"]
                        for j in range(Lv):
                            Bt[j] -= rec["B"][j].T @ Pc
                    rec.update(mean=mean, var=var, Bt=Bt)
            self.fin.append(rec)

    # ---- posterior : posterior-inference.cpp:14-265, class_approximation.cpp:186-306
    def posterior(self, keep_factors: bool):
        st = self.st
        r, M = st.r, st.M
        d = 0.0
        Lt = self.L_prior.copy()
        v_all = np.zeros((st.n_interior, r))
        G_all = {}
        child_w, child_A = {}, {}      # level m+1 outputs: dict region -> (w (m+1,r), A dict (j,k)->r x r)
        for m in range(M - 2, -1, -1):
            s0, cnt = st.level_start(m), st.level_count(m)
            out_w, out_A = {}, {}
            for i in range(s0, s0 + cnt):
                if m == M - 2:
                    kids = np.nonzero(st.finest_parent == i)[0]
                    wsum = np.zeros((m + 1, r)); Asum = {}
                    for j in range(m + 1):
                        for k in range(j, m + 1):
                            Asum[(j, k)] = np.zeros((r, r))
                    for c in kids:
                        rec = self.fin[c]
                        if rec["n"] == 0:
                            continue
                        for j in range(m + 1):
                            wsum[j] += rec["B"][j].T @ rec["yt"]
                            for k in range(j, m + 1):
                                Asum[(j, k)] += rec["B"][j].T @ rec["B"][k]
                else:
                    kids = np.arange(i * st.J + 1, i * st.J + st.J + 1)
                    wsum = sum(child_w[c] for c in kids)
                    Asum = {key: sum(child_A[c][key] for c in kids) for key in child_A[kids[0]]}
                d -= 2 * np.sum(np.log(np.diag(Lt[i])))
                Lt[i] = np.linalg.cholesky(Lt[i] @ Lt[i].T + Asum[(m, m)])
                v = np.linalg.solve(Lt[i], wsum[m])
                v_all[i] = v
                d += 2 * np.sum(np.log(np.diag(Lt[i]))) - v @ v
                if m > 0:
                    G = [np.linalg.solve(Lt[i], Asum[(j, m)].T) for j in range(m)]
                    if keep_factors:
                        G_all[i] = G
                    out_w[i] = np.stack([wsum[j] - G[j].T @ v for j in range(m)])
                    out_A[i] = {(j, k): Asum[(j, k)] - G[j].T @ G[k] for j in range(m) for k in range(j, m)}
            child_w, child_A = out_w, out_A
        self.d_posterior = d
        self.L_post, self.v_post, self.G_post = Lt, v_all, G_all
        return d

    # ---- prediction, top-down : predict.cpp:105-189
    def predict_finest(self):
        st = self.st
        Lv = st.M - 1
        means, vars_ = [], []
        for k in range(st.n_finest):
            rec = self.fin[k]
            if rec.get("np", 0) == 0:
                continue
            anc = rec["anc"]
            mean, var = rec["mean"].copy(), rec["var"].copy()
            tmp = [b.copy() for b in rec["Bt"]]
            for j in range(Lv - 1, -1, -1):
                KcB = np.linalg.solve(self.L_post[anc[j]], tmp[j])
                for kk in range(j):
                    tmp[kk] -= self.G_post[anc[j]][kk].T @ KcB
                mean += KcB.T @ self.v_post[anc[j]]
                var += np.sum(KcB * KcB, axis=0)
            means.append(mean)
            vars_.append(var)
        if not means:
            return np.zeros(0), np.zeros(0)
        return np.concatenate(means), np.concatenate(vars_)


def loglik(st: Structure, model: Model) -> tuple:
    """Returns (d, loglik): d is the reference's internal Approximation::loglikelihood
    after likelihood(); loglik = -0.5 (d + n log(2*3.14159265359))."""
    mra = MRA(st, model)
    mra.prior_interior()
    mra.prior_finest(prediction=False)
    d = mra.d_finest + mra.posterior(keep_factors=False)
    return d, -0.5 * (d + st.n_obs * math.log(TWO_PI_TRUNCATED))


def predict(st: Structure, model: Model) -> tuple:
    """Posterior predictive (mean, variance) at st.pred, in finest-region order
    (the order of dump_prediction_result, class_approximation.cpp:493-535)."""
    mra = MRA(st, model)
    mra.prior_interior()
    mra.prior_finest(prediction=True)
    mra.posterior(keep_factors=True)
    return mra.predict_finest()


# --------------------------------------------------------------------------
# reference-format case directories (user_parameters + binary files)
# --------------------------------------------------------------------------
def parse_user_parameters(path) -> dict:
    """KEY=value lines, '#' comments, spaces/tabs/quotes stripped
    (read_user_parameters.cpp:10-50)."""
    out = {}
    for line in open(path):
        s = line.lstrip(" \t")
        if not s or s[0] in "#\n\r":
            continue
        s = "".join(ch for ch in s.rstrip("\r\n") if ch not in " \t'\"")
        if "=" not in s:
            continue
        k, v = s.split("=", 1)
        if k:
            out[k] = v
    return out


def load_case(case_dir, mode: Optional[str] = None):
    """Builds (Structure, Model) from a directory holding ``user_parameters``
    and the binary files it names, the way the reference's main() does
    (src/main.cpp:93-113).  An optional ``ext_parameters`` file (same format,
    keys MRA_EXT_PLANAR / MRA_EXT_NU_X2 / MRA_EXT_PREFACTOR_EXP / MRA_EXT_BASIS)
    selects the opt-in covariance variants; the reference's parser rejects
    unknown keys, so they live outside ``user_parameters`` and the extension
    oracle binary reads them from the environment."""
    import os
    P = parse_user_parameters(os.path.join(case_dir, "user_parameters"))
    fp = lambda k: os.path.join(case_dir, P[k])
    truthy = lambda k, d="false": P.get(k, d).lower() == "true"
    mode = mode or P["CALCULATION_MODE"]
    provided = truthy("PROVIDED_KNOTS_FLAG")
    chordal = truthy("CHORDAL_DISTANCE_FLAG", "true")
    ext_path = os.path.join(case_dir, "ext_parameters")
    ext = parse_user_parameters(ext_path) if os.path.exists(ext_path) else {}
    distance = DIST_CHORDAL if chordal else (DIST_EUCLID2D if ext.get("MRA_EXT_PLANAR", "false") == "true"
                                             else DIST_GREAT_CIRCLE)
    lon, lat, val, reg = read_data_file(fp("DATA_FILE_NAME"), provided)
    ok = ~np.isnan(val)
    plon = plat = preg = None
    if mode == "prediction":
        pm = P.get("PREDICTION_LOCATION_MODE", "A")
        if pm == "A":
            plon, plat, preg = read_pred_file(fp("PREDICTION_LOCATION_FILE"), provided)
        elif pm == "N":
            plon, plat = lon[~ok], lat[~ok]
            preg = reg[~ok] if provided else None
        else:
            plon, plat, preg = lon.copy(), lat.copy(), (reg.copy() if provided else None)
    J = int(P["NUM_PARTITIONS_J"]); M = int(P["NUM_LEVELS_M"]); r = int(P["NUM_KNOTS_r"])
    if provided:
        klon, klat, kreg = read_knots_file(fp("KNOTS_FILE_NAME"))
        ps, pe, par = read_parent_file(fp("PARENT_REGION_FILE_NAME"))
        st = build_structure_by_user_files(lon[ok], lat[ok], val[ok], reg[ok], J, M, r, klon, klat, kreg,
                                           ps, par, plon, plat, preg, distance)
        st.obs_index = np.nonzero(ok)[0][st.obs_index]
    else:
        off = P.get("OFFSET", "default")
        offset = math.exp(1) / 100 if off == "default" else float(off)
        st = build_structure_by_program(lon[ok], lat[ok], val[ok], J, M, r, offset, plon, plat, distance,
                                        all_lon=lon, all_lat=lat)
        st.obs_index = np.nonzero(ok)[0][st.obs_index]
    md = Model()
    md.nonstationary = truthy("NONSTATIONARY_FLAG")
    md.distance = distance
    md.nu_x2 = int(ext.get("MRA_EXT_NU_X2", "1"))
    md.prefactor_exp = float(ext.get("MRA_EXT_PREFACTOR_EXP", "1.5"))
    md.dist_scale = 1.0 if distance == DIST_EUCLID2D else EARTH_RADIUS_KM
    md.basis = BASIS_GAUSSIAN if ext.get("MRA_EXT_BASIS", "wendland") == "gaussian" else BASIS_WENDLAND
    md.basis_len = float(P.get("WENDLAND_LEN", "0.22"))
    md.sill = float(P.get("SIGMASQ", "1")); md.range_ = float(P.get("BETA", "1")); md.nugget = float(P.get("TAUSQ", "0"))
    md.sill_scale = float(P.get("SIGMASQ_SCALE", "1")); md.range_scale = float(P.get("BETA_SCALE", "1"))
    md.nugget_scale = float(P.get("TAUSQ_SCALE", "1"))
    if md.nonstationary:
        for key in ("SIGMASQ_FILE_NAME", "BETA_FILE_NAME", "TAUSQ_FILE_NAME"):
            icpt, blon, blat, w = read_basis_file(fp(key))
            if distance == DIST_CHORDAL:
                centers = np.stack(lonlat_to_xyz(blon, blat))
            else:
                centers = np.stack([blon, blat, np.zeros_like(blon)])
            md.fields.append(Field(icpt, centers, w))
    return st, md, P


def sample_prior(st: Structure, model: Model, z_int: np.ndarray, z_obs: np.ndarray) -> np.ndarray:
    """y = sum_j U_{obs,j}^T z_{a_j} + L_Sigma z_obs, in structure order: a draw from
    the MRA prior (the finest-level Sigma_i already carries tau^2 on its diagonal)."""
    mra = MRA(st, model)
    mra.prior_interior()
    mra.prior_finest(prediction=False)
    y = np.zeros(st.n_obs)
    r = st.r
    for k, rec in enumerate(mra.fin):
        if rec["n"] == 0:
            continue
        a0, a1 = st.obs_offset[k], st.obs_offset[k + 1]
        v = rec["LS"] @ z_obs[a0:a1]
        for j, a in enumerate(rec["anc"]):
            v = v + rec["Ufin"][j].T @ z_int[a * r:(a + 1) * r]
        y[a0:a1] = v
    return y
