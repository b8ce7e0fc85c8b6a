"""GPU: the hand-written adjoint (hv_adjoint_forward / hv_adjoint_backward).

The gradient of an objective of D(t) with respect to theta = (t0, t3, sigma,
a_sym) is checked against central finite differences of FP64 forward runs
(relative step 1e-3), with the SOR run to a relative residual of 1e-12 so
that its stopping rule adds no noise to the differences.  Tolerance: every
component within 1e-3 of the finite difference, relative to the largest
component."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(hv, steps, ppn=40):
    w = replace(hv.CA40_SMALL, ppn=ppn, sor_tol=1e-12, deposit_mode=hv.HV_DEPOSIT_SORTED)
    parts = hv.workload_particles(w, np.float64)
    theta = np.array([w.t0, w.t3, w.sigma, w.a_sym])
    return w, parts, theta


def _central_differences(run, theta, fn, rel=1e-3):
    g = np.zeros(4)
    for i in range(4):
        h = rel * abs(theta[i])
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        g[i] = (run.objective(tp, fn) - run.objective(tm, fn)) / (2 * h)
    return g


def test_adjoint_matches_central_differences_linear_objective(hv):
    from hv_b200.adjoint import AdjointRun
    steps = 40
    w, parts, theta = _setup(hv, steps)
    wts = np.random.default_rng(3).standard_normal(steps)
    fn = lambda d: float(wts @ d)
    run = AdjointRun(w, parts, steps, checkpoint_every=10)
    try:
        run.forward(theta)
        g_adj = run.backward(wts)
        g_fd = _central_differences(run, theta, fn)
    finally:
        run.close()
    scale = np.abs(g_fd).max()
    assert scale > 0
    assert np.all(np.abs(g_adj - g_fd) <= 1e-3 * scale), (g_adj, g_fd)


def test_adjoint_spectrum_objective_through_torch(hv):
    """theta.grad of the D(t)-spectrum power in 10-25 MeV (spectrum.power_in_band)
    through the torch.autograd.Function, against central differences, for
    40Ca with 1000 test particles per nucleon.  The objective is only piecewise
    smooth (the CIC weights have kinks at cell faces); with a few thousand
    particles the differences scatter by ~0.5 % between step sizes, with
    40,000 they settle within 1e-3 of the adjoint."""
    import torch

    from hv_b200.adjoint import AdjointRun, dipole_series
    from hv_b200.spectrum import power_in_band
    steps = 160
    w, parts, theta = _setup(hv, steps, ppn=1000)
    t = np.arange(steps) * w.dt
    t_f = steps * w.dt

    def fn(d):
        return float(power_in_band(torch.as_tensor(d), t, t_f, w.dt))

    run = AdjointRun(w, parts, steps, checkpoint_every=40)
    try:
        th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
        J = power_in_band(dipole_series(th, run), t, t_f, w.dt)
        J.backward()
        g_adj = th.grad.numpy().copy()
        g_fd = _central_differences(run, theta, fn)
    finally:
        run.close()
    assert float(J.detach()) > 0
    scale = np.abs(g_fd).max()
    assert np.all(np.abs(g_adj - g_fd) <= 1e-3 * scale), (g_adj, g_fd)


def test_adjoint_independent_of_checkpoint_spacing_and_restores_state(hv):
    from hv_b200.adjoint import AdjointRun
    steps = 30
    w, parts, theta = _setup(hv, steps)
    wts = np.random.default_rng(4).standard_normal(steps)
    grads, finals = [], []
    for every in (1, 7, 30):
        run = AdjointRun(w, parts, steps, checkpoint_every=every)
        try:
            d = run.forward(theta)
            end = run.session.download_particles()
            grads.append(run.backward(wts))
            after = run.session.download_particles()
            assert all(np.array_equal(a, b) for a, b in zip(end, after))
            finals.append(d)
        finally:
            run.close()
    for g in grads[1:]:
        assert np.max(np.abs(g - grads[0])) <= 1e-9 * np.abs(grads[0]).max()
    for d in finals[1:]:
        assert np.array_equal(d, finals[0])


def test_adjoint_forward_matches_plain_run(hv):
    """The checkpointed forward is the plain FP64 run."""
    steps = 12
    w, parts, theta = _setup(hv, steps)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(*parts)
        s.initial_solve()
        a = s.adjoint_forward(steps, 5)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(*parts)
        s.initial_solve()
        b = s.run(steps, hv.HV_PATH_PLAIN)
    assert np.array_equal(a["dipole"], b["dipole"])


def test_adjoint_rejects_float_contexts_and_missing_forward(hv):
    w = hv.CA40_SMALL
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        with pytest.raises(hv.HVError):
            s.adjoint_forward(2, 1)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        with pytest.raises(hv.HVError):
            s.adjoint_backward(np.zeros(2), np.zeros(4))


def test_adjoint_matches_fp64_tangent_linear_cpu_run(hv):
    """The adjoint gradient against the FP64 tangent-linear run on the CPU
    oracle (oracle/hv_tangent.py, itself pinned to finite differences in
    tests/test_tangent.py): both differentiate the same discrete map exactly,
    so they agree far below the finite-difference noise -- within 1e-6 of the
    largest component, in each of the four directions."""
    from hv_oracle import RunSpec
    from hv_tangent import Tangent, skyrme_from_theta

    from hv_b200.adjoint import AdjointRun
    steps = 24
    w, parts, theta = _setup(hv, steps)
    wts = np.random.default_rng(5).standard_normal(steps)
    run = AdjointRun(w, parts, steps, checkpoint_every=8)
    try:
        d_gpu = run.forward(theta)
        g_adj = run.backward(wts)
    finally:
        run.close()
    A, B, C, g = skyrme_from_theta(theta)
    spec = RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc,
                   eta_exc=w.eta, A=A, B=B, C=C, gamma=g, sor_omega=w.sor_omega, sor_tol=w.sor_tol,
                   sor_criterion=w.sor_criterion, sor_max_iter=w.sor_max_iter)
    t = Tangent(w.world_tuple(), spec, w.protons, w.neutrons)
    g_tl = np.zeros(4)
    for i in range(4):
        e = np.zeros(4)
        e[i] = 1.0
        d_cpu, dD = t.run(*parts, steps, theta, e)
        g_tl[i] = wts @ dD
    assert np.max(np.abs(d_cpu - d_gpu)) <= 1e-9 * np.abs(d_cpu).max()
    assert np.all(np.abs(g_adj - g_tl) <= 1e-6 * np.abs(g_tl).max()), (g_adj, g_tl)


def test_adjoint_backward_after_a_resorting_fused_run_keeps_the_caller_order(hv):
    """A fused run between the forward and the backward pass re-sorts the
    particle slots; the backward pass restores the forward's checkpoints with
    their slot permutation, so the state it leaves downloads in the caller's
    order, equal to the forward's final state."""
    steps = 8
    w, parts, theta = _setup(hv, steps)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(*parts)
        s.initial_solve()
        s.adjoint_forward(steps, 4)
        after_forward = s.download_particles()
        s.set_fast_options(sort_every=1)
        s.run(3, hv.HV_PATH_FUSED)
        s.adjoint_backward(np.ones(steps), theta)
        after_backward = s.download_particles()
    for a, b in zip(after_backward, after_forward):
        assert a.tobytes() == b.tobytes()


def test_fused_adjoint_matches_the_plain_adjoint_and_central_differences(hv):
    """hv_adjoint_forward_path(HV_PATH_FUSED): the forward as fused FP64 steps
    and the backward's transposed Poisson solves on the persistent SOR kernel.
    Its D(t) is the plain forward's within 1e-8 of max|D| (both solves to a
    relative residual of 1e-12), its gradient the plain adjoint's within 1e-5
    and central differences of fused forward runs within 1e-3, each relative to
    the largest component."""
    from hv_b200.adjoint import AdjointRun
    steps = 40
    w, parts, theta = _setup(hv, steps)
    wts = np.random.default_rng(5).standard_normal(steps)
    fn = lambda d: float(wts @ d)
    plain = AdjointRun(w, parts, steps, checkpoint_every=10)
    fused = AdjointRun(w, parts, steps, checkpoint_every=10, path=hv.HV_PATH_FUSED)
    try:
        d_p = plain.forward(theta)
        g_p = plain.backward(wts)
        d_f = fused.forward(theta)
        g_f = fused.backward(wts)
        path, its, unconverged = fused.session.adjoint_stats()
        g_fd = _central_differences(fused, theta, fn)
    finally:
        plain.close()
        fused.close()
    assert path == hv.HV_PATH_FUSED and its > 0 and unconverged == 0
    assert np.max(np.abs(d_f - d_p)) <= 1e-8 * np.abs(d_p).max()
    scale = np.abs(g_p).max()
    assert np.all(np.abs(g_f - g_p) <= 1e-5 * scale), (g_f, g_p)
    scale = np.abs(g_fd).max()
    assert np.all(np.abs(g_f - g_fd) <= 1e-3 * scale), (g_f, g_fd)


def test_fused_adjoint_independent_of_checkpoint_spacing_and_restores_state(hv):
    """The fused backward recomputes each segment from a checkpoint that holds
    phi's history, the forces, the smoothed density and the control words, so
    the gradient does not depend on the spacing; the context ends in the
    forward's final state, and slot re-sorting stays off during both passes
    (the default sort_every would otherwise re-sort inside a segment)."""
    from hv_b200.adjoint import AdjointRun
    steps = 30
    w, parts, theta = _setup(hv, steps)
    wts = np.random.default_rng(6).standard_normal(steps)
    grads, finals = [], []
    for every in (1, 7, 30):
        run = AdjointRun(w, parts, steps, checkpoint_every=every, path=hv.HV_PATH_FUSED,
                         fast_options={"sort_every": 4})
        try:
            d = run.forward(theta)
            end = run.session.download_particles()
            grads.append(run.backward(wts))
            after = run.session.download_particles()
            assert all(np.array_equal(a, b) for a, b in zip(end, after))
            finals.append(d)
        finally:
            run.close()
    for g in grads[1:]:
        assert np.max(np.abs(g - grads[0])) <= 1e-9 * np.abs(grads[0]).max()
    for d in finals[1:]:
        assert np.array_equal(d, finals[0])
