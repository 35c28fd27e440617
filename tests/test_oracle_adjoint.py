"""The FP64 reference adjoint (oracle/psc_adjoint.py) against central finite differences, on the CPU."""

import numpy as np
import pytest

from oracle import psc_adjoint as adj
from oracle import psc_oracle as orc

PARTS = np.array([[4.3, 5.1, 4.8, 2.2] + [0.0] * 6,
                  [7.9, 3.2, 6.1, 1.7] + [0.0] * 6,
                  [2.0, 8.5, 1.0, 1.9] + [0.0] * 6])
CASE = dict(n=10, S=2, eps=0.05, tau=0.8, F=(1e-4, 0.0, 0.0), steps=25)


def test_deviation_collision_equals_reference_collision():
    rng = np.random.default_rng(0)
    shp = (5, 5, 5)
    f = orc.equilibrium(1 + rng.normal(0, 1e-3, shp), *rng.normal(0, 1e-3, (3,) + shp))
    solid = rng.uniform(0, 1, shp)
    F = (1e-5, 2e-6, -3e-6)
    post, _ = orc.collide(f, solid, None, 0.8, F)
    dev = adj.collide_dev(f - orc.W[:, None, None, None], adj.bweight(solid, 0.8), 0.8, F)
    assert np.abs(dev + orc.W[:, None, None, None] - post).max() <= 1e-15


def test_collision_vjp_matches_fd():
    rng = np.random.default_rng(1)
    shp = (4, 4, 4)
    g = rng.normal(0, 1e-4, (19,) + shp)
    B = rng.uniform(0, 1, shp)
    lam = rng.normal(0, 1, (19,) + shp)
    F = (1e-5, 0.0, 2e-6)
    mu, dB = adj.collide_dev_vjp(g, B, lam, 0.8, F)
    h = 1e-6
    v = rng.normal(0, 1, g.shape)
    fd = ((adj.collide_dev(g + h * v, B, 0.8, F) - adj.collide_dev(g - h * v, B, 0.8, F)) / (2 * h) * lam).sum()
    assert abs(fd - (mu * v).sum()) <= 1e-8 * abs(fd)
    vb = rng.normal(0, 1, shp)
    fdb = ((adj.collide_dev(g, B + h * vb, 0.8, F) - adj.collide_dev(g, B - h * vb, 0.8, F)) / (2 * h) * lam).sum()
    assert abs(fdb - (dB * vb).sum()) <= 1e-7 * abs(fdb)


@pytest.mark.slow
def test_permeability_gradient_matches_central_differences():
    c = CASE
    K, grad, _ = adj.gradient(PARTS, c["n"], c["S"], c["eps"], c["tau"], c["F"], c["steps"])
    h = 1e-3
    worst = 0.0
    for p in range(len(PARTS)):
        for k in range(4):
            pp = PARTS.copy()
            pp[p, k] += h
            pm = PARTS.copy()
            pm[p, k] -= h
            fd = (adj.forward(pp, c["n"], c["S"], c["eps"], c["tau"], c["F"], c["steps"])[0]
                  - adj.forward(pm, c["n"], c["S"], c["eps"], c["tau"], c["F"], c["steps"])[0]) / (2 * h)
            worst = max(worst, abs(fd - grad[p, k]) / abs(fd))
    # central differences with h = 1e-3 on a sigmoid of width 0.05 carry (h/eps)^2/6 ~ 7e-5
    assert worst <= 2e-4
