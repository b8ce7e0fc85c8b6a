"""GPU: whole steps of the cpu_simulate loop through the C ABI.

* plain HV_F64 path with the reference's SOR settings vs the reference's own
  10-step run (golden): the only operation that is not bit-identical is the
  Skyrme pow (CUDA vs glibc, last bit), so positions agree to ~1e-12 fm;
* plain HV_F64 path with the 40Ca workload's SOR (omega 1.8, relative residual
  1e-6) vs the oracle over 20 steps: D(t) within 1e-9 fm;
* hv_simulate with host buffers equals the session path.
"""
from __future__ import annotations

import numpy as np
import pytest
from conftest import max_rel

pytestmark = pytest.mark.gpu


def test_plain_f64_matches_reference_run(hv, golden):
    g = golden("ca40_run_f64.npz")
    w = hv.CA40_SMALL.with_reference_sor()
    from dataclasses import replace
    w = replace(w, deposit_mode=hv.HV_DEPOSIT_SORTED)
    steps = int(g["steps"])
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(g["x0"], g["y0"], g["z0"], g["kx0"], g["ky0"], g["kz0"])
        s.initial_solve()
        obs = s.run(steps, hv.HV_PATH_PLAIN)
        x, y, z, kx, ky, kz = s.download_particles()
    rows = g["rows"]
    assert np.array_equal(obs["t"], rows[:, 0])
    assert np.max(np.abs(obs["zcm_p"] - rows[:, 3])) < 1e-12
    assert np.max(np.abs(obs["zcm_n"] - rows[:, 4])) < 1e-12
    assert np.max(np.abs(obs["rms_p"] - rows[:, 1])) < 1e-12
    for a, k in zip((x, y, z), ("x", "y", "z")):
        assert np.max(np.abs(a - g[k])) < 1e-10, k
    for a, k in zip((kx, ky, kz), ("kx", "ky", "kz")):
        assert np.max(np.abs(a - g[k])) < 1e-10, k


def _oracle_run(w):
    from hv_oracle import RunSpec
    A, B, C, gm = w.skyrme()
    return RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc,
                   eta_exc=w.eta, A=A, B=B, C=C, gamma=gm, sor_omega=w.sor_omega, sor_tol=w.sor_tol,
                   sor_criterion=w.sor_criterion, sor_max_iter=w.sor_max_iter)


def test_plain_f64_matches_oracle_with_relative_residual_sor(hv):
    from hv_oracle import Oracle
    w = hv.CA40_SMALL
    steps = 20
    x, y, z, kx, ky, kz = hv.workload_particles(w, np.float64)
    run = _oracle_run(w)
    o = Oracle(np.float64)
    o.set_threads(1)
    xo, yo, zo, kxo, kyo, kzo = (a.copy() for a in (x, y, z, kx, ky, kz))
    obs_o, _ = o.simulate(w.world_tuple(), run, w.protons, w.neutrons, xo, yo, zo, kxo, kyo, kzo, steps)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(x, y, z, kx, ky, kz)
        s.initial_solve()
        obs = s.run(steps, hv.HV_PATH_PLAIN)
        xg, yg, zg, *_ = s.download_particles()
    assert np.max(np.abs(obs["dipole"] - obs_o["dipole"])) < 1e-9
    assert np.all(np.abs(obs["sor_iterations"] - obs_o["sor_iterations"]) <= 1)
    assert np.max(np.abs(zg - zo)) < 1e-8


def test_simulate_with_host_buffers_equals_session(hv):
    w = hv.CA40_SMALL
    steps = 5
    x, y, z, kx, ky, kz = hv.workload_particles(w, np.float64)
    a = [v.copy() for v in (x, y, z, kx, ky, kz)]
    obs1 = hv.simulate(w, *a, steps, hv.HV_F64, hv.HV_PATH_PLAIN)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(x, y, z, kx, ky, kz)
        s.initial_solve()
        obs2 = s.run(steps, hv.HV_PATH_PLAIN)
        b = s.download_particles()
    assert max_rel(obs1["dipole"], obs2["dipole"]) < 1e-12
    for u, v in zip(a, b):
        assert max_rel(u, v) < 1e-12


def test_plain_f32_tracks_f64(hv):
    w = hv.CA40_SMALL
    steps = 20
    x, y, z, kx, ky, kz = hv.workload_particles(w, np.float32)
    from dataclasses import replace
    w32 = w.with_reference_sor()  # a float phi cannot reach a 1e-6 relative residual
    with hv.Session.from_workload(w32, hv.HV_F32) as s:
        s.upload_particles(x, y, z, kx, ky, kz)
        s.initial_solve()
        o32 = s.run(steps, hv.HV_PATH_PLAIN)
    with hv.Session.from_workload(replace(w32), hv.HV_F64) as s:
        s.upload_particles(*(v.astype(np.float64) for v in (x, y, z, kx, ky, kz)))
        s.initial_solve()
        o64 = s.run(steps, hv.HV_PATH_PLAIN)
    assert max_rel(o32["dipole"], o64["dipole"]) < 1e-3


def test_simulate_reuses_its_context_as_new(hv):
    """hv_simulate keeps its device context between calls of one shape: a
    second call (after a call of another nucleus shape and one with other
    parameters, on the fused path that re-sorts the slots) computes what the
    first did -- bit for bit on the deterministic plain FP64 path -- and
    hv_simulate_release frees the kept contexts."""
    from dataclasses import replace
    # the deterministic deposit: the atomic one's summation order varies run to run
    w = replace(hv.CA40_SMALL, deposit_mode=hv.HV_DEPOSIT_SORTED)
    steps = 4
    parts = hv.workload_particles(w, np.float64)
    a = [v.copy() for v in parts]
    obs1 = hv.simulate(w, *a, steps, hv.HV_F64, hv.HV_PATH_PLAIN)
    # the same shape on the fused path (slots re-sorted), other parameters
    b = [v.copy() for v in parts]
    hv.simulate(replace(w, t0=-2600.0), *b, 20, hv.HV_F64, hv.HV_PATH_FUSED)
    # another shape in between
    w2 = replace(w, ppn=50)
    hv.simulate(w2, *hv.workload_particles(w2, np.float64), 2, hv.HV_F64, hv.HV_PATH_PLAIN)
    c = [v.copy() for v in parts]
    obs2 = hv.simulate(w, *c, steps, hv.HV_F64, hv.HV_PATH_PLAIN)
    assert obs1.tobytes() == obs2.tobytes()
    for u, v in zip(a, c):
        assert u.tobytes() == v.tobytes()
    hv.simulate_release()
    d = [v.copy() for v in parts]
    obs3 = hv.simulate(w, *d, steps, hv.HV_F64, hv.HV_PATH_PLAIN)
    assert obs3.tobytes() == obs1.tobytes()
    hv.simulate_release()
