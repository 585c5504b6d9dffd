"""Parameter fitting on the exact GPU likelihood: the plain derivative-free
optimizer and the surrogate-assisted variant.

Plain: ``minimize`` runs the library's bound-constrained trust-region
optimizer (``mra_opt_minimize``, the method of the reference's
dlib::find_min_bobyqa call, src/optimization.cpp:158-192) on the reference's
objective, the internal log-likelihood value d = -2 loglik - n log(2 pi)
(src/optimization.cpp:107-150 returns ``approximation.loglikelihood``).

Surrogate-assisted: the same optimizer spends the first ``n_train`` exact
evaluations; an MLP (``Surrogate``: the library's CUDA training and inference
kernels) is trained on those (theta, loglik) pairs and then proposes steps,
each maximising the network inside a box trust region around the best point
found so far.  Every proposal is evaluated exactly on the GPU and is accepted
only if the exact likelihood improves; the new pair joins the training set.
When proposals stop paying (the box shrinks below ``box_min``), the exact
optimizer finishes from the best point.  The exact likelihood is therefore
both the arbiter of every step and the fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import capi
from .capi import check, f32p, f64p


# ---------------------------------------------------------------------------
# plain optimizer
# ---------------------------------------------------------------------------
@dataclass
class OptResult:
    x: np.ndarray
    f: float
    evals: int
    status: int
    rho: float


def minimize(f: Callable[[np.ndarray], float], x0, lower, upper, rho_begin: float, rho_end: float,
             max_evals: int, npt: int = 0) -> OptResult:
    """Minimises f over lower <= x <= upper (mra_opt_minimize).  f may raise
    StopIteration to end the run early (the best point so far is returned)."""
    lib = capi.load()
    x = np.array(x0, dtype=np.float64)
    lo = np.ascontiguousarray(lower, dtype=np.float64)
    hi = np.ascontiguousarray(upper, dtype=np.float64)
    n = x.shape[0]
    err: List[BaseException] = []

    def cb(xp, _user, stop):
        try:
            return float(f(np.ctypeslib.as_array(xp, shape=(n,)).copy()))
        except StopIteration:
            stop[0] = 1
            return 0.0
        except BaseException as e:  # surfaced after the C call returns
            err.append(e)
            stop[0] = 1
            return 0.0

    fn = capi.OBJECTIVE_FN(cb)
    cfg = capi.mra_opt_config(rho_begin=rho_begin, rho_end=rho_end, npt=npt, max_evals=max_evals)
    res = capi.mra_opt_result()
    check(lib.mra_opt_minimize(n, f64p(x), f64p(lo), f64p(hi), C.byref(cfg), fn, None, C.byref(res)),
          "mra_opt_minimize")
    if err:
        raise err[0]
    return OptResult(x, res.f_best, res.evals, res.status, res.rho_final)


# ---------------------------------------------------------------------------
# MLP surrogate (CUDA kernels of libmra_b200.so)
# ---------------------------------------------------------------------------
class Surrogate:
    """n_in -> 128 -> 128 -> 1 SiLU network, BF16 weights / FP32 accumulation."""

    HIDDEN = 128

    def __init__(self, n_in: int, seed: int = 0):
        self._lib = capi.load()
        h = C.c_void_p()
        check(self._lib.mra_mlp_create(int(n_in), self.HIDDEN, int(seed), C.byref(h)), "mra_mlp_create")
        self._h = h
        self.n_in = int(n_in)
        n = C.c_int64()
        check(self._lib.mra_mlp_num_params(self._h, C.byref(n)), "mra_mlp_num_params")
        self.n_params = int(n.value)

    def close(self):
        if self._h:
            self._lib.mra_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        check(self._lib.mra_mlp_get_params(self._h, f32p(p)), "mra_mlp_get_params")
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(self._lib.mra_mlp_set_params(self._h, f32p(p)), "mra_mlp_set_params")

    def set_data(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        check(self._lib.mra_mlp_set_data(self._h, f32p(x), f32p(t), int(t.shape[0])), "mra_mlp_set_data")

    def grad(self):
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_float()
        check(self._lib.mra_mlp_grad(self._h, f32p(g), C.byref(loss)), "mra_mlp_grad")
        return g, float(loss.value)

    def train(self, steps: int, lr: float) -> float:
        loss = C.c_float()
        check(self._lib.mra_mlp_train(self._h, int(steps), float(lr), C.byref(loss)), "mra_mlp_train")
        return float(loss.value)

    def predict(self, x: np.ndarray, with_grad: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        y = np.empty(n, dtype=np.float32)
        g = np.empty((n, self.n_in), dtype=np.float32) if with_grad else None
        check(self._lib.mra_mlp_predict(self._h, f32p(x), n, f32p(y), f32p(g) if with_grad else None),
              "mra_mlp_predict")
        return (y, g) if with_grad else y


# ---------------------------------------------------------------------------
# the MRA objective over the 19 nonstationary parameters
# ---------------------------------------------------------------------------
@dataclass
class Trace:
    """Every exact evaluation: parameters, loglik and wall time since start."""
    theta: list = field(default_factory=list)
    loglik: list = field(default_factory=list)
    seconds: list = field(default_factory=list)
    t0: float = field(default_factory=time.perf_counter)

    def best_loglik(self) -> float:
        return max(self.loglik) if self.loglik else -math.inf

    def time_to_reach(self, target: float) -> Optional[float]:
        """Wall seconds until the first evaluation with loglik >= target."""
        for ll, s in zip(self.loglik, self.seconds):
            if ll >= target:
                return s
        return None

    def evals_to_reach(self, target: float) -> Optional[int]:
        for k, ll in enumerate(self.loglik):
            if ll >= target:
                return k + 1
        return None


class NonstationaryObjective:
    """theta = (9 log-sigma coefficients, 9 log-range coefficients, log tau^2)
    of the Gaussian-RBF extension model -> exact GPU log-likelihood.
    ``__call__`` returns d (the reference's objective, to be minimised)."""

    def __init__(self, ctx, sigma_intercept: float, range_intercept: float, n_sigma: int = 9, n_range: int = 9,
                 max_evals: Optional[int] = None):
        self.ctx = ctx
        self.icpt = (float(sigma_intercept), float(range_intercept))
        self.ns, self.nr = int(n_sigma), int(n_range)
        self.n = self.ns + self.nr + 1
        self.trace = Trace()
        self.max_evals = max_evals

    def loglik(self, theta: np.ndarray) -> float:
        theta = np.asarray(theta, dtype=np.float64)
        if self.max_evals is not None and len(self.trace.loglik) >= self.max_evals:
            raise StopIteration
        self.ctx.set_theta(weights=[2.0 * theta[:self.ns], theta[self.ns:self.ns + self.nr], None],
                           intercepts=[self.icpt[0], self.icpt[1], float(theta[-1])])
        _, ll = self.ctx.loglik()
        self.trace.theta.append(theta.copy())
        self.trace.loglik.append(ll)
        self.trace.seconds.append(time.perf_counter() - self.trace.t0)
        return ll

    def d_of(self, ll: float) -> float:
        return -2.0 * ll - self.ctx.n_obs * math.log(2 * 3.14159265359)

    def __call__(self, theta: np.ndarray) -> float:
        return self.d_of(self.loglik(theta))


# ---------------------------------------------------------------------------
# fitting drivers
# ---------------------------------------------------------------------------
@dataclass
class FitConfig:
    rho_begin: float = 0.5
    rho_end: float = 1e-6
    max_evals: int = 3000
    n_train: int = 200          # exact evaluations before the surrogate takes over
    box0: float = 0.5           # first proposal box half-width (theta units)
    box_min: float = 2e-3       # surrogate phase ends below this box
    train_steps0: int = 3000
    train_steps: int = 300
    lr: float = 2e-3
    starts: int = 64            # multi-start ascent on the network
    ascent_steps: int = 60
    keep_best: int = 160        # training set size
    train_set: str = "best"     # "best": highest loglik; "nearest": pairs closest to the best point
    proposal: str = "ball"      # "ball": gradient path in an L2 trust region; "box": multi-start in a box
    seed: int = 0


def fit_plain(obj: NonstationaryObjective, theta0, lower, upper, cfg: FitConfig) -> OptResult:
    return minimize(obj, theta0, lower, upper, cfg.rho_begin, cfg.rho_end, cfg.max_evals)


def _training_set(trace: Trace, keep: int, center: np.ndarray, scale: np.ndarray, how: str = "best"):
    ll = np.asarray(trace.loglik)
    th = np.asarray(trace.theta)
    if how == "nearest":
        order = np.argsort(np.sum(((th - center) / scale) ** 2, axis=1))[:keep]
    else:
        order = np.argsort(-ll)[:keep]
    x = (th[order] - center) / scale
    t = ll[order]
    mu, sd = float(t.mean()), float(t.std()) or 1.0
    return x.astype(np.float32), ((t - mu) / sd).astype(np.float32), mu, sd


def propose(net: Surrogate, center: np.ndarray, scale: np.ndarray, box: float, lower, upper,
            rng: np.random.Generator, starts: int, steps: int) -> np.ndarray:
    """Multi-start projected gradient ascent of the network inside
    |theta - center| <= box (and the bounds); returns the best theta."""
    n = center.shape[0]
    lo = np.maximum((np.asarray(lower) - center) / scale, -box / scale)
    hi = np.minimum((np.asarray(upper) - center) / scale, box / scale)
    x = rng.uniform(lo, hi, size=(starts, n)).astype(np.float32)
    x[0] = 0.0
    step = (hi - lo) / 10.0
    for _ in range(steps):
        _, g = net.predict(x, with_grad=True)
        x = np.clip(x + step * np.sign(g), lo, hi).astype(np.float32)
        step *= 0.93
    y = net.predict(x)
    return center + scale * x[int(np.argmax(y))].astype(np.float64)


def propose_ball(net: Surrogate, center: np.ndarray, scale: np.ndarray, radius: float, lower, upper,
                 steps: int) -> np.ndarray:
    """Gradient path of the network from the best point, kept inside the L2
    ball |(theta - center) / scale| <= radius and the bounds."""
    lo = (np.asarray(lower) - center) / scale
    hi = (np.asarray(upper) - center) / scale
    x = np.zeros((1, center.shape[0]), dtype=np.float32)
    eta = radius / 10.0
    for _ in range(steps):
        _, g = net.predict(x, with_grad=True)
        gn = float(np.linalg.norm(g))
        if not gn > 0:
            break
        x = x + eta * g / gn
        r = float(np.linalg.norm(x))
        if r > radius:
            x *= radius / r
        x = np.clip(x, lo, hi).astype(np.float32)
    return center + scale * x[0].astype(np.float64)


def _spread(trace: Trace, center: np.ndarray, scale: np.ndarray, k: int = 20) -> float:
    th = np.asarray(trace.theta)
    d = np.sqrt(np.sum(((th - center) / scale) ** 2, axis=1))
    d = np.sort(d)[1:k + 1]
    return float(np.median(d)) if d.size else 1.0


def fit_surrogate(obj: NonstationaryObjective, theta0, lower, upper, cfg: FitConfig, net: Optional[Surrogate] = None):
    """Returns (theta_best, loglik_best, info)."""
    rng = np.random.default_rng(cfg.seed)
    n = len(theta0)
    # phase 1: the exact optimizer's first n_train evaluations
    res = minimize(obj, theta0, lower, upper, cfg.rho_begin, cfg.rho_end, min(cfg.n_train, cfg.max_evals))
    tr = obj.trace
    best = int(np.argmax(tr.loglik))
    theta_b, ll_b = np.array(tr.theta[best]), tr.loglik[best]
    own = net is None
    net = net or Surrogate(n, seed=cfg.seed)
    scale = np.full(n, cfg.box0)
    ball = cfg.proposal == "ball"
    box = _spread(tr, theta_b, scale) if ball else cfg.box0
    box_max = 4.0 * box if ball else cfg.box0
    x, t, mu, sd = _training_set(tr, cfg.keep_best, theta_b, scale, cfg.train_set)
    net.set_data(x, t)
    net.train(cfg.train_steps0, cfg.lr)
    proposals = accepted = 0
    # phase 2: network proposals, each verified exactly
    while box >= cfg.box_min and len(tr.loglik) < cfg.max_evals:
        if ball:
            cand = propose_ball(net, theta_b, scale, box, lower, upper, cfg.ascent_steps)
            small = np.linalg.norm((cand - theta_b) / scale) < 0.05 * box
        else:
            cand = propose(net, theta_b, scale, box, lower, upper, rng, cfg.starts, cfg.ascent_steps)
            small = np.max(np.abs(cand - theta_b)) < 0.05 * box
        if small:
            box *= 0.5
            continue
        try:
            ll = obj.loglik(cand)
        except StopIteration:
            break
        proposals += 1
        if ll > ll_b:
            theta_b, ll_b = cand, ll
            accepted += 1
            box = min(2.0 * box, box_max)
        else:
            box *= 0.5
        x, t, mu, sd = _training_set(tr, cfg.keep_best, theta_b, scale, cfg.train_set)
        net.set_data(x, t)
        net.train(cfg.train_steps, cfg.lr)
    # phase 3: the exact optimizer finishes from the best point
    left = cfg.max_evals - len(tr.loglik)
    rho = max(min(box * (cfg.box0 if ball else 2.0), cfg.rho_begin), cfg.rho_end)
    if left > 2 * n + 2:
        try:
            res = minimize(obj, theta_b, lower, upper, rho, cfg.rho_end, left)
        except StopIteration:
            pass
        best = int(np.argmax(tr.loglik))
        theta_b, ll_b = np.array(tr.theta[best]), tr.loglik[best]
    if own:
        net.close()
    return theta_b, ll_b, {"proposals": proposals, "accepted": accepted, "evals": len(tr.loglik)}
