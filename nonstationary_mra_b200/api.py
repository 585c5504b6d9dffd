"""Python host mirror of the reference's MRA interface, over the C ABI.

``Context`` holds one resident partition + model on the GPU (the state that
the reference keeps in its global ``partition`` / ``nonstat_cov`` objects,
include/constants.hpp:147-153).  ``Approximation`` mirrors the reference class
of the same name (include/class_approximation.hpp:7-93): it is constructed
with (sill, range, nugget, sill_scale, range_scale, nugget_scale), and
``likelihood()`` / ``predict()`` fill ``loglikelihood`` (the reference's
internal units: sum of log-determinants and quadratic forms, without the -1/2
and the constant) and ``posteriorPredictionMean`` / ``posteriorPredictionVariance``.

Structures and models are plain containers with numpy arrays (see
``nonstationary_mra_b200.model``); any object with the same attribute names
is accepted.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import capi
from .capi import check, f64p, u64p

TWO_PI_TRUNCATED = 2 * 3.14159265359  # src/class_approximation-posterior-inference.cpp:244


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def set_device(device: int):
    check(capi.load().mra_set_device(int(device)), "mra_set_device")


class Context:
    """Device-resident structure + model (one GPU, one CUDA stream)."""

    def __init__(self, structure, model, precision: str = "fp64"):
        lib = capi.load()
        self._keep = []
        st = capi.mra_structure()
        st.J, st.M, st.r = int(structure.J), int(structure.M), int(structure.r)
        st.n_interior = int(structure.n_interior)
        parent = _c(structure.finest_parent, np.uint64)
        knots = _c(structure.knots, np.float64)
        obs_off = _c(structure.obs_offset, np.uint64)
        obs = _c(structure.obs, np.float64)
        y = _c(structure.obs_value, np.float64)
        self._keep += [parent, knots, obs_off, obs, y]
        st.n_finest = parent.shape[0]
        st.finest_parent, st.knots, st.obs_offset = u64p(parent), f64p(knots), u64p(obs_off)
        st.obs, st.obs_value = f64p(obs), f64p(y)
        self.n_obs = int(y.shape[0])
        self.M = int(structure.M)
        self.n_pred = 0
        if getattr(structure, "pred_offset", None) is not None:
            poff = _c(structure.pred_offset, np.uint64)
            pred = _c(structure.pred, np.float64)
            self._keep += [poff, pred]
            st.pred_offset, st.pred = u64p(poff), f64p(pred)
            self.n_pred = int(poff[-1])
        md = capi.mra_model()
        md.nonstationary = 1 if model.nonstationary else 0
        md.distance, md.nu_x2, md.basis = int(model.distance), int(model.nu_x2), int(model.basis)
        md.prefactor_exp, md.dist_scale, md.basis_len = float(model.prefactor_exp), float(model.dist_scale), \
            float(model.basis_len)
        self.n_basis = [0, 0, 0]
        if model.nonstationary:
            for f, fld in enumerate(model.fields):
                cen = _c(fld.centers, np.float64)
                w = _c(fld.weights, np.float64)
                self._keep += [cen, w]
                md.field[f].n_basis = w.shape[0]
                md.field[f].centers, md.field[f].weights = f64p(cen), f64p(w)
                md.field[f].intercept = float(fld.intercept)
                self.n_basis[f] = int(w.shape[0])
        self._model = md
        self.precision = capi.PRECISION_MIXED if precision == "mixed" else capi.PRECISION_FP64
        h = C.c_void_p()
        check(lib.mra_create(C.byref(st), C.byref(md), self.precision, C.byref(h)), "mra_create")
        self._h = h
        self._lib = lib

    # -- parameters ---------------------------------------------------------
    def set_theta(self, sill=1.0, range_=1.0, nugget=0.0, sill_scale=1.0, range_scale=1.0, nugget_scale=1.0,
                  weights: Optional[Sequence] = None, intercepts: Optional[Sequence[float]] = None):
        th = capi.mra_theta()
        th.sill, th.range, th.nugget = sill, range_, nugget
        th.sill_scale, th.range_scale, th.nugget_scale = sill_scale, range_scale, nugget_scale
        keep = []
        if weights is not None:
            for f in range(3):
                if weights[f] is not None:
                    w = _c(weights[f], np.float64)
                    if w.shape[0] != self.n_basis[f]:
                        raise ValueError(f"field {f}: expected {self.n_basis[f]} weights")
                    keep.append(w)
                    th.weights[f] = f64p(w)
        if intercepts is not None:
            ic = _c(intercepts, np.float64)
            keep.append(ic)
            th.intercepts = f64p(ic)
        check(self._lib.mra_set_theta(self._h, C.byref(th)), "mra_set_theta")

    def set_obs_values(self, y: np.ndarray):
        y = _c(y, np.float64)
        check(self._lib.mra_set_obs_values(self._h, f64p(y)), "mra_set_obs_values")

    # -- evaluations --------------------------------------------------------
    def loglik(self) -> tuple:
        d, ll = C.c_double(), C.c_double()
        check(self._lib.mra_loglik(self._h, C.byref(d), C.byref(ll)), "mra_loglik")
        return d.value, ll.value

    def predict(self) -> tuple:
        mean = np.empty(self.n_pred)
        var = np.empty(self.n_pred)
        check(self._lib.mra_predict(self._h, f64p(mean), f64p(var)), "mra_predict")
        return mean, var

    def autotune(self, evals: int = 2):
        """Picks the FP64 tile widths by timing this context (mra_autotune);
        returns (widths per bucket in units of 16 columns, best ms per evaluation)."""
        ch = (C.c_int32 * 3)()
        ms = C.c_double()
        check(self._lib.mra_autotune(self._h, int(evals), ch, C.byref(ms)), "mra_autotune")
        return list(ch), ms.value

    def capture_graph(self):
        check(self._lib.mra_capture_graph(self._h), "mra_capture_graph")

    def sample_prior(self, z_interior: np.ndarray, z_obs: np.ndarray) -> np.ndarray:
        zi, zo = _c(z_interior, np.float64), _c(z_obs, np.float64)
        y = np.empty(self.n_obs)
        check(self._lib.mra_sample_prior(self._h, f64p(zi), f64p(zo), f64p(y)), "mra_sample_prior")
        return y

    def timer_start(self):
        check(self._lib.mra_timer_start(self._h), "mra_timer_start")

    def timer_stop(self) -> float:
        ms = C.c_double()
        check(self._lib.mra_timer_stop(self._h, C.byref(ms)), "mra_timer_stop")
        return ms.value

    def set_obs_values_ptr(self, ptr: int):
        """Replace y from a raw host pointer (e.g. a pinned buffer)."""
        check(self._lib.mra_set_obs_values(self._h, C.cast(C.c_void_p(ptr), capi._p_f64)), "mra_set_obs_values")

    def stats(self) -> dict:
        s = capi.mra_stats()
        check(self._lib.mra_get_stats(self._h, C.byref(s)), "mra_get_stats")
        out = {k: getattr(s, k) for k, _ in capi.mra_stats._fields_ if not k.startswith("timed_")}
        n = s.n_timed
        out["launches"] = [{"kernel": capi.KERNEL_NAMES.get(s.timed_kind[i], "?"), "level": s.timed_level[i],
                            "ms": s.timed_ms[i], "flop": s.timed_flop[i], "ms_cov": s.timed_ms_cov[i]}
                           for i in range(n)]
        return out

    # ---- sub-tree sharding (include/mra_b200.h: mra_shard_*) ----
    def shard_set(self, split_level: int, owned) -> None:
        """Restrict evaluations to the level-`split_level` sub-trees with owned[q]
        true; owned = None returns the context to whole evaluations."""
        if owned is None:
            check(self._lib.mra_shard_set(self._h, 0, None), "mra_shard_set")
            return
        o = np.ascontiguousarray(np.asarray(owned, dtype=np.uint8))
        check(self._lib.mra_shard_set(self._h, int(split_level), o.ctypes.data_as(C.POINTER(C.c_uint8))),
              "mra_shard_set")

    def shard_subtrees(self) -> None:
        check(self._lib.mra_shard_loglik_subtrees(self._h), "mra_shard_loglik_subtrees")

    def shard_export(self, region: int) -> np.ndarray:
        n = C.c_uint64()
        check(self._lib.mra_shard_record_size(self._h, int(region), C.byref(n)), "mra_shard_record_size")
        rec = np.empty(n.value)
        check(self._lib.mra_shard_export(self._h, int(region), f64p(rec), n.value), "mra_shard_export")
        return rec

    def shard_import(self, region: int, record: np.ndarray) -> None:
        rec = _c(record, np.float64)
        check(self._lib.mra_shard_import(self._h, int(region), f64p(rec), rec.shape[0]), "mra_shard_import")

    def shard_top(self):
        d, ll = C.c_double(), C.c_double()
        check(self._lib.mra_shard_loglik_top(self._h, C.byref(d), C.byref(ll)), "mra_shard_loglik_top")
        return d.value, ll.value

    def terms(self) -> np.ndarray:
        """Parts of d from the last evaluation: [m] = level-m posterior terms for
        m < M-1, [M-1] = finest-level plus level M-2 terms (mra_get_terms)."""
        out = np.zeros(self.M)
        check(self._lib.mra_get_terms(self._h, f64p(out), self.M), "mra_get_terms")
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mra_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Approximation:
    """Mirror of the reference's Approximation (include/class_approximation.hpp:7-93)."""

    def __init__(self, ctx: Context, sill: float, range_: float, nugget: float, sill_scale: float,
                 range_scale: float, nugget_scale: float, weights=None, intercepts=None):
        self.ctx = ctx
        self.sill, self.range, self.nugget = sill, range_, nugget
        self.sill_scale, self.range_scale, self.nugget_scale = sill_scale, range_scale, nugget_scale
        self._weights, self._intercepts = weights, intercepts
        self.loglikelihood = 0.0
        self.posteriorPredictionMean = None
        self.posteriorPredictionVariance = None

    def _set(self):
        self.ctx.set_theta(self.sill, self.range, self.nugget, self.sill_scale, self.range_scale,
                           self.nugget_scale, self._weights, self._intercepts)

    def likelihood(self) -> float:
        """Prior + posterior; returns -0.5 (d + n log(2*3.14159265359))."""
        self._set()
        d, ll = self.ctx.loglik()
        self.loglikelihood = d
        return ll

    def predict(self):
        self._set()
        mean, var = self.ctx.predict()
        self.posteriorPredictionMean, self.posteriorPredictionVariance = mean, var
        return mean, var


def eval_covariance(model, theta: dict, p1: np.ndarray, p2: Optional[np.ndarray] = None) -> np.ndarray:
    """evaluate_*covariance on the GPU.  Returns an (n1, n2) array equal to the
    reference's row-major out[i1*n2+i2]; symmetric self block when p2 is None."""
    lib = capi.load()
    md, keep = _model_struct(model)
    th = _theta_struct(theta)
    p1c = _c(p1, np.float64)
    n1 = p1c.shape[1]
    if p2 is None:
        out = np.empty((n1, n1))
        check(lib.mra_eval_covariance(C.byref(md), C.byref(th), f64p(p1c), n1, None, 0, 1, f64p(out)),
              "mra_eval_covariance")
    else:
        p2c = _c(p2, np.float64)
        n2 = p2c.shape[1]
        out = np.empty((n1, n2))
        check(lib.mra_eval_covariance(C.byref(md), C.byref(th), f64p(p1c), n1, f64p(p2c), n2, 0, f64p(out)),
              "mra_eval_covariance")
    del keep
    return out


def eval_fields(model, theta: dict, p: np.ndarray) -> np.ndarray:
    """(3, n): sigma^2, beta, tau^2 (Nonstationary_covariance::get_* times the scales)."""
    lib = capi.load()
    md, keep = _model_struct(model)
    th = _theta_struct(theta)
    pc = _c(p, np.float64)
    out = np.empty((3, pc.shape[1]))
    check(lib.mra_eval_fields(C.byref(md), C.byref(th), f64p(pc), pc.shape[1], f64p(out)), "mra_eval_fields")
    del keep
    return out


def _model_struct(model):
    md = capi.mra_model()
    keep = []
    md.nonstationary = 1 if model.nonstationary else 0
    md.distance, md.nu_x2, md.basis = int(model.distance), int(model.nu_x2), int(model.basis)
    md.prefactor_exp, md.dist_scale, md.basis_len = float(model.prefactor_exp), float(model.dist_scale), \
        float(model.basis_len)
    if model.nonstationary:
        for f, fld in enumerate(model.fields):
            cen, w = _c(fld.centers, np.float64), _c(fld.weights, np.float64)
            keep += [cen, w]
            md.field[f].n_basis = w.shape[0]
            md.field[f].centers, md.field[f].weights = f64p(cen), f64p(w)
            md.field[f].intercept = float(fld.intercept)
    return md, keep


def _theta_struct(theta: dict):
    th = capi.mra_theta()
    th.sill = theta.get("sill", 1.0)
    th.range = theta.get("range", 1.0)
    th.nugget = theta.get("nugget", 0.0)
    th.sill_scale = theta.get("sill_scale", 1.0)
    th.range_scale = theta.get("range_scale", 1.0)
    th.nugget_scale = theta.get("nugget_scale", 1.0)
    return th


def loglik_constant(n_obs: int) -> float:
    return n_obs * math.log(TWO_PI_TRUNCATED)
