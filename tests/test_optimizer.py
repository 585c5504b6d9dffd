"""The bound-constrained derivative-free optimizer (mra_opt_minimize, the
method of the reference's dlib::find_min_bobyqa call,
src/optimization.cpp:158-192).  Host code: runs without a GPU."""
import numpy as np
import pytest

from nonstationary_mra_b200 import build, capi
from nonstationary_mra_b200.fit import minimize


@pytest.fixture(scope="module", autouse=True)
def lib():
    build.build()
    return capi.load()


def test_quadratic_with_active_bounds():
    rng = np.random.default_rng(0)
    n = 6
    A = rng.standard_normal((n, n))
    Q = A @ A.T + n * np.eye(n)
    c = rng.standard_normal(n) * 3
    f = lambda x: 0.5 * x @ Q @ x - c @ x
    lo, hi = -0.3 * np.ones(n), 0.4 * np.ones(n)
    r = minimize(f, np.zeros(n), lo, hi, 0.1, 1e-8, 2000)
    # reference solution: projected gradient on the convex QP
    x = np.zeros(n)
    for _ in range(20000):
        x = np.clip(x - 0.01 * (Q @ x - c), lo, hi)
    assert np.max(np.abs(r.x - x)) < 1e-5, (r.x, x)
    assert r.status == 0 and r.f <= f(x) + 1e-9


@pytest.mark.parametrize("x0", [[-1.2, 1.0], [0.0, 0.0, 0.0, 0.0]])
def test_rosenbrock(x0):
    f = lambda x: sum(100 * (x[i + 1] - x[i] ** 2) ** 2 + (1 - x[i]) ** 2 for i in range(len(x) - 1))
    n = len(x0)
    r = minimize(f, np.array(x0), -3 * np.ones(n), 3 * np.ones(n), 0.5, 1e-8, 5000)
    assert r.f < 1e-10 and np.allclose(r.x, 1.0, atol=1e-4), (r.f, r.x, r.evals)


def test_rosenbrock_local_minimum_from_the_chain_start():
    # from (-1.2, 1, -1.2, 1) the 4-d chain has a local minimum near
    # (-0.7757, 0.6131, 0.3821, 0.1460) with f = 3.7014: a valid stopping point
    f = lambda x: sum(100 * (x[i + 1] - x[i] ** 2) ** 2 + (1 - x[i]) ** 2 for i in range(len(x) - 1))
    r = minimize(f, np.array([-1.2, 1.0, -1.2, 1.0]), -3 * np.ones(4), 3 * np.ones(4), 0.5, 1e-8, 5000)
    assert r.status == 0 and (r.f < 1e-10 or abs(r.f - 3.70142861) < 1e-6), (r.f, r.x)


def test_reference_configuration_three_scales():
    # the reference's call: n = 3 scales, x0 = 1, bounds [1e-2, 1e2], npt = 7, rho 0.1 -> 1e-6
    target = np.array([0.7, 2.5, 0.05])
    f = lambda x: float(np.sum(np.log(x / target) ** 2) + 0.1 * np.log(x[0] / target[0]) * np.log(x[1] / target[1]))
    r = minimize(f, np.ones(3), 1e-2 * np.ones(3), 1e2 * np.ones(3), 0.1, 1e-6, 4000, npt=7)
    assert np.allclose(r.x, target, rtol=1e-4), (r.x, r.evals)


def test_budget_and_stop():
    calls = []

    def f(x):
        calls.append(1)
        if len(calls) == 25:
            raise StopIteration
        return float(np.sum((x - 0.3) ** 2))

    r = minimize(f, np.zeros(5), -np.ones(5), np.ones(5), 0.2, 1e-8, 1000)
    assert r.status == 2 and r.evals == 25
    r = minimize(lambda x: float(np.sum(x ** 2)), np.ones(5) * 0.5, -np.ones(5), np.ones(5), 0.2, 1e-12, 40)
    assert r.status == 1 and r.evals == 40


def test_bad_arguments_rejected():
    with pytest.raises(capi.MRAError):
        minimize(lambda x: 0.0, np.zeros(3), -np.ones(3), np.ones(3), 1.5, 1e-6, 100)   # range < 2 rho
    with pytest.raises(capi.MRAError):
        minimize(lambda x: 0.0, np.zeros(3), -np.ones(3), np.ones(3), 0.1, 1e-6, 100, npt=3)
