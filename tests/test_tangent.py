"""CPU: the FP64 tangent-linear run (oracle/hv_tangent.py) against central
finite differences of the oracle's own forward run (orc_simulate).

The tangent-linear run is the independent reference the GPU adjoint is
checked against (tests/test_gpu_adjoint.py); here it is pinned to finite
differences: dJ/dtheta of J = sum_n w_n D_n for 40Ca on 32^3 (h = 1 fm),
1600 test particles, 16 steps, SOR to relative residual 1e-12, relative step
1e-3; every component within 1e-3 of the largest."""
from __future__ import annotations

import numpy as np
import pytest

from hv_oracle import Oracle, RunSpec


def case():
    import hv_b200 as hv
    from dataclasses import replace
    w = replace(hv.CA40_SMALL, ppn=40)
    parts = hv.workload_particles(w, np.float64)
    theta = np.array([w.t0, w.t3, w.sigma, w.a_sym])
    return w, parts, theta


def spec(w, theta):
    from hv_tangent import skyrme_from_theta
    A, B, C, g = skyrme_from_theta(theta)
    return RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc, eta_exc=w.eta,
                   A=A, B=B, C=C, gamma=g, sor_omega=w.sor_omega, sor_tol=1e-12, sor_criterion=1,
                   sor_max_iter=20000)


def oracle_D(w, parts, theta, steps):
    o = Oracle(np.float64)
    a = [p.copy() for p in parts]
    obs, _ = o.simulate(w.world_tuple(), spec(w, theta), w.protons, w.neutrons, *a, steps)
    return obs["dipole"]


def test_tangent_forward_is_the_oracle_run():
    from hv_tangent import Tangent
    w, parts, theta = case()
    steps = 6
    t = Tangent(w.world_tuple(), spec(w, theta), w.protons, w.neutrons)
    D, _ = t.run(*parts, steps, theta, np.zeros(4))
    assert np.max(np.abs(D - oracle_D(w, parts, theta, steps))) <= 1e-12 * np.abs(D).max()


def test_tangent_linear_matches_central_differences():
    from hv_tangent import Tangent
    w, parts, theta = case()
    steps = 16
    wts = np.random.default_rng(3).standard_normal(steps)
    t = Tangent(w.world_tuple(), spec(w, theta), w.protons, w.neutrons)
    g_tl, g_fd = np.zeros(4), np.zeros(4)
    for i in range(4):
        e = np.zeros(4)
        e[i] = 1.0
        _, dD = t.run(*parts, steps, theta, e)
        g_tl[i] = wts @ dD
        h = 1e-3 * abs(theta[i])
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        g_fd[i] = (wts @ oracle_D(w, parts, tp, steps) - wts @ oracle_D(w, parts, tm, steps)) / (2 * h)
    scale = np.abs(g_fd).max()
    assert scale > 0
    assert np.all(np.abs(g_tl - g_fd) <= 1e-3 * scale), (g_tl, g_fd)
