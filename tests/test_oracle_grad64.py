"""The FP64 gradient references (oracle/grad64.py) checked on the CPU before they check the
engine's adjoints: every analytic gradient against central differences of the FP64 functions
themselves, with a step small enough (1e-6) that the difference's truncation error is far
below the tolerance."""
from __future__ import annotations

import numpy as np

from oracle import grad64 as g

STEP = 1e-6


def _gaussians(k, seed):
    rng = np.random.default_rng(seed)
    G = np.zeros((k, 10))
    G[:, 0:3] = rng.uniform(0, 10, (k, 3))
    G[:, 3:7] = rng.normal(size=(k, 4)) * rng.uniform(0.2, 3.0, (k, 1))  # any quaternion norm
    G[:, 7:10] = rng.uniform(0.05, 1.0, (k, 3))
    P = G[:, 0:3] + rng.normal(size=(k, 3)) * 2.0
    return P, G


def test_gaussian_analytic_matches_differences():
    P, G = _gaussians(400, 1)
    ids = np.arange(len(G))
    d, gp, gG = g.gaussian_analytic(P, G, ids)
    out = d > 1e-3  # points inside (d = 0) have a zero gradient, checked below
    assert out.sum() > 300
    assert np.all(gG[~out] == 0) and np.all(gp[~out] == 0)
    for c in range(10):
        e = np.zeros_like(G)
        e[:, c] = STEP
        fd = (g.ellipsoid_d(P, G + e)[0] - g.ellipsoid_d(P, G - e)[0]) / (2 * STEP)
        assert np.max(g.rel_err(gG[out, c], fd[out], 1e-3)) <= 1e-5, c
    for c in range(3):
        e = np.zeros_like(P)
        e[:, c] = STEP
        fd = (g.ellipsoid_d(P + e, G)[0] - g.ellipsoid_d(P - e, G)[0]) / (2 * STEP)
        assert np.max(g.rel_err(gp[out, c], fd[out], 1e-3)) <= 1e-5, c


def test_gaussian_gradient_sums_per_primitive():
    P, G = _gaussians(300, 2)
    ids = np.random.default_rng(3).integers(0, 20, len(P))
    _, _, gG = g.gaussian_analytic(P, G, ids)
    # a Gaussian no query selects has zero gradient; the rest sum over their queries
    assert np.all(gG[np.setdiff1d(np.arange(len(G)), ids)] == 0)
    one = np.nonzero(ids == ids[0])[0]
    _, _, g1 = g.gaussian_analytic(P[one], G, ids[one])
    assert np.allclose(g1[ids[0]], gG[ids[0]])


def test_ray_analytic_matches_differences():
    rng = np.random.default_rng(4)
    k = 300
    a = rng.uniform(0, 1, (k, 3))
    b = a + rng.uniform(0.2, 1, (k, 3)) * [1, 0, 0.1]
    c = a + rng.uniform(0.2, 1, (k, 3)) * [0, 1, 0.1]
    O = (a + b + c) / 3 + [0, 0, 5] + rng.normal(size=(k, 3)) * [0.05, 0.05, 0]
    D = np.tile([0.0, 0.0, -1.0], (k, 1)) + rng.normal(size=(k, 3)) * 0.05
    tt, w, kk = g.ray_analytic(O, D, a, b, c)
    for j, (wj, vert) in enumerate(zip(w, (a, b, c))):
        for comp in range(3):
            e = np.zeros_like(vert)
            e[:, comp] = STEP
            args_p = [a, b, c]
            args_m = [a, b, c]
            args_p[j] = vert + e
            args_m[j] = vert - e
            fd = (g.ray_t(O, D, *args_p) - g.ray_t(O, D, *args_m)) / (2 * STEP)
            assert np.max(g.rel_err(wj * kk[:, comp], fd, 1e-3)) <= 1e-5
    e = np.zeros_like(O)
    e[:, 2] = STEP
    fd = (g.ray_t(O + e, D, a, b, c) - g.ray_t(O - e, D, a, b, c)) / (2 * STEP)
    assert np.max(g.rel_err(-kk[:, 2], fd, 1e-3)) <= 1e-5


def test_central_difference_and_richardson():
    f = lambda x: np.sin(1.3 + x) * 7.0  # noqa: E731
    fd, rich = g.central(f, 1e-2)
    exact = 7.0 * np.cos(1.3)
    assert abs(rich - exact) < abs(fd - exact) < 1e-3
