"""GPU: the fused fast path (HV_PATH_FUSED) against the oracle and the plain path.

Tolerances
  * D(t): max|D - D_ref| / max|D_ref| <= 1e-3 for the float path against the
    double oracle (the accuracy target of the float form), <= 1e-6 for the
    double fused path against the double plain path;
  * SOR: every step converges to the same stopping rule (relative residual
    1e-6); with plain SOR cycles (sor_coarse = 0) the fused solver checks it
    every few iterations, so it may run up to sor_inner_max iterations more
    than the plain solver, never fewer; with the coarse-grid correction (the
    default) far fewer, and D(t) within 1e-6 of the plain cycles' run;
  * fields after a fused run: smoothed density and potential of the final
    positions within 1e-5 (float) of the oracle's, forces within 1e-4.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest
from conftest import max_rel

pytestmark = pytest.mark.gpu


def _oracle_runspec(w):
    from hv_oracle import RunSpec
    A, B, C, gm = w.skyrme()
    return RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc,
                   eta_exc=w.eta, A=A, B=B, C=C, gamma=gm, sor_omega=w.sor_omega, sor_tol=w.sor_tol,
                   sor_criterion=w.sor_criterion, sor_max_iter=w.sor_max_iter)


def _oracle(w, steps, parts64):
    from hv_oracle import Oracle
    o = Oracle(np.float64)
    o.set_threads(4)
    a = [p.copy() for p in parts64]
    obs, _ = o.simulate(w.world_tuple(), _oracle_runspec(w), w.protons, w.neutrons, *a, steps)
    return obs, a


def _fused(hv, w, steps, prec, parts, **opts):
    with hv.Session.from_workload(w, prec) as s:
        if opts:
            s.set_fast_options(**opts)
        s.upload_particles(*parts)
        s.initial_solve()
        obs = s.run(steps, hv.HV_PATH_FUSED)
        out = s.download_particles()
    return obs, out


def test_fused_f32_dipole_within_1e_3_of_double_oracle(hv):
    """Both initial guesses of the fused SOR: the reference's (the previous
    phi; then every solve takes at least the oracle's iterations, less one) and
    the default extrapolated one (fewer iterations, the same stopping rule)."""
    w = hv.CA40_SMALL
    steps = 200
    p32 = hv.workload_particles(w, np.float32)
    obs_o, _ = _oracle(w, steps, [p.astype(np.float64) for p in p32])
    obs, _ = _fused(hv, w, steps, hv.HV_F32, p32, sor_warm_start=hv.HV_WARM_PREVIOUS, sor_coarse=0)
    assert np.array_equal(obs["t"], obs_o["t"].astype(np.float32).astype(np.float64)) or \
        np.max(np.abs(obs["t"] - obs_o["t"])) < 1e-4
    err = max_rel(obs["dipole"], obs_o["dipole"])
    assert err <= 1e-3, err
    assert not np.any(obs["flags"] & 1)
    assert np.all(obs["sor_iterations"] >= obs_o["sor_iterations"] - 1)
    obs_x, _ = _fused(hv, w, steps, hv.HV_F32, p32)
    assert max_rel(obs_x["dipole"], obs_o["dipole"]) <= 1e-3
    assert not np.any(obs_x["flags"] & 1)
    assert obs_x["sor_iterations"][10:].sum() < obs["sor_iterations"][10:].sum()


def test_fused_f64_matches_plain_f64(hv):
    w = hv.CA40_SMALL
    steps = 30
    p = hv.workload_particles(w, np.float64)
    obs_f, out_f = _fused(hv, w, steps, hv.HV_F64, p, sor_warm_start=hv.HV_WARM_PREVIOUS)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_particles(*p)
        s.initial_solve()
        obs_p = s.run(steps, hv.HV_PATH_PLAIN)
        out_p = s.download_particles()
        inner_max = s.fast_options().sor_inner_max
    assert max_rel(obs_f["dipole"], obs_p["dipole"]) < 1e-6
    assert np.max(np.abs(out_f[2] - out_p[2])) < 1e-6
    d = obs_f["sor_iterations"] - obs_p["sor_iterations"]
    assert np.all(d >= -1) and np.all(d <= inner_max)


def test_fused_reference_sor_rule(hv):
    w = hv.CA40_SMALL.with_reference_sor()
    steps = 20
    p = hv.workload_particles(w, np.float64)
    obs_f, _ = _fused(hv, w, steps, hv.HV_F64, p)
    obs_o, _ = _oracle(w, steps, p)
    assert max_rel(obs_f["dipole"], obs_o["dipole"]) < 1e-4


def test_extrapolated_warm_start_saves_iterations(hv):
    w = hv.CA40_SMALL
    steps = 60
    p32 = hv.workload_particles(w, np.float32)
    obs_a, _ = _fused(hv, w, steps, hv.HV_F32, p32, sor_warm_start=hv.HV_WARM_PREVIOUS, sor_inner_min=1,
                      sor_inner_max=8, sor_coarse=0)
    obs_b, _ = _fused(hv, w, steps, hv.HV_F32, p32, sor_warm_start=hv.HV_WARM_EXTRAPOLATE, sor_inner_min=1,
                      sor_inner_max=8, sor_coarse=0)
    assert obs_b["sor_iterations"][10:].sum() < obs_a["sor_iterations"][10:].sum()
    assert max_rel(obs_b["dipole"], obs_a["dipole"]) < 1e-3
    # the quadratic guess 3 phi_n - 3 phi_(n-1) + phi_(n-2) (the default)
    obs_c, _ = _fused(hv, w, steps, hv.HV_F32, p32, sor_warm_start=hv.HV_WARM_QUADRATIC, sor_inner_min=1,
                      sor_inner_max=8, sor_coarse=0)
    assert obs_c["sor_iterations"][10:].sum() < obs_b["sor_iterations"][10:].sum()
    assert max_rel(obs_c["dipole"], obs_a["dipole"]) < 1e-3
    assert not np.any(obs_c["flags"] & 1)


def test_first_steps_after_the_fused_initial_solve_start_from_solutions(hv):
    """hv_run on the fused path with no earlier solve runs the initial solve
    itself, from phi = 0.  That starting phi must not enter the history that
    the extrapolated guesses are built from: the first steps then need no more
    iterations than from the previous phi (a zero in the history made steps 1
    and 2 start from 2 phi_0 and ~0 and cost as much as the initial solve)."""
    w = hv.CA40_SMALL
    p32 = hv.workload_particles(w, np.float32)
    its = {}
    for ws in (hv.HV_WARM_PREVIOUS, hv.HV_WARM_QUADRATIC):
        with hv.Session.from_workload(w, hv.HV_F32) as s:
            s.set_fast_options(sor_warm_start=ws, sor_inner_min=1, sor_inner_max=8, sor_coarse=0)
            s.upload_particles(*p32)
            its[ws] = s.run(6, hv.HV_PATH_FUSED)["sor_iterations"].astype(np.int64)
    prev, quad = its[hv.HV_WARM_PREVIOUS], its[hv.HV_WARM_QUADRATIC]
    # step 0 starts from the initial solution under both guesses
    assert abs(int(quad[0]) - int(prev[0])) <= 8, (quad, prev)
    # later steps extrapolate from converged solutions only
    assert np.all(quad[1:] <= prev[1:] + 8), (quad, prev)
    assert quad[1:].sum() < prev[1:].sum(), (quad, prev)


@pytest.mark.parametrize("wname", ["208Pb-20.8k-128^3", "208Pb-104k-64^3"])
def test_coarse_cycle_relaxation_keeps_the_rule_with_fewer_iterations(hv, wname):
    """The sweeps after each coarse-grid correction relax at
    hv_fast_options.sor_coarse_omega (default 1.7, 12 sweeps a cycle), not at
    the run's omega: each cycle then removes at least as much of the residual
    as 16 sweeps at the run's 1.8 did, so the solves end at the same FP64
    rule in no more iterations.  D(t) and the Coulomb potential of the two
    settings agree within 1e-6 relative, the tolerance of each solve."""
    w = hv.WORKLOADS[wname]
    p32 = hv.workload_particles(w, np.float32)
    res = []
    for opts in ({}, dict(sor_coarse_sweeps=16, sor_coarse_omega=w.sor_omega)):
        with hv.Session.from_workload(w, hv.HV_F32) as s:
            if opts:
                s.set_fast_options(**opts)
            fo = s.fast_options()
            s.upload_particles(*p32)
            s.initial_solve()
            obs = s.run(10, hv.HV_PATH_FUSED)
            res.append((fo, obs, s.download_field(hv.HV_FIELD_COULOMB)))
    (f0, o0, c0), (f1, o1, c1) = res
    assert f0.sor_coarse_sweeps == 12 and f0.sor_coarse_omega == 0.0
    assert f1.sor_coarse_sweeps == 16 and f1.sor_coarse_omega == w.sor_omega
    assert not np.any(o0["flags"] & 1) and not np.any(o1["flags"] & 1)
    assert o0["sor_iterations"][2:].sum() <= o1["sor_iterations"][2:].sum(), (o0["sor_iterations"],
                                                                             o1["sor_iterations"])
    assert max_rel(o0["dipole"], o1["dipole"]) < 1e-6, max_rel(o0["dipole"], o1["dipole"])
    assert max_rel(c0, c1) < 1e-6, max_rel(c0, c1)
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        for bad in (-0.5, 2.0, 2.5):
            with pytest.raises(hv.HVError):
                s.set_fast_options(sor_coarse_omega=bad)


def test_sor_omega_override_keeps_the_stopping_rule(hv):
    """hv_fast_options.sor_omega relaxes the fused sweeps differently; the
    FP64 residual test is unchanged, so D(t) stays within the float path's
    rounding while the iterations change.  Out-of-range values are refused."""
    w = hv.CA40_SMALL
    steps = 30
    p32 = hv.workload_particles(w, np.float32)
    obs_a, _ = _fused(hv, w, steps, hv.HV_F32, p32, sor_coarse=0)
    obs_b, _ = _fused(hv, w, steps, hv.HV_F32, p32, sor_omega=1.9, sor_coarse=0)
    assert not np.any(obs_b["flags"] & 1)
    assert obs_b["sor_iterations"][5:].sum() != obs_a["sor_iterations"][5:].sum()
    assert max_rel(obs_b["dipole"], obs_a["dipole"]) < 1e-4
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        for bad in (-0.5, 2.0, 2.5):
            with pytest.raises(hv.HVError):
                s.set_fast_options(sor_omega=bad)


def test_slot_resort_keeps_results_and_caller_order(hv):
    """hv_fast_options.sort_every re-sorts the particle slots by cell (species
    kept apart); D(t) and the downloaded particles, in the caller's order,
    match a run without re-sorting to float rounding."""
    w = hv.CA40_SMALL
    p32 = hv.workload_particles(w, np.float32)
    out = {}
    for every in (0, 4):
        with hv.Session.from_workload(w, hv.HV_F32) as s:
            s.set_fast_options(sort_every=every)
            s.upload_particles(*p32)
            obs = s.run(24, hv.HV_PATH_FUSED)
            out[every] = (obs, s.download_particles())
    (o0, p0), (o4, p4) = out[0], out[4]
    assert not np.any(o4["flags"] & 1)
    assert max_rel(o4["dipole"], o0["dipole"]) < 1e-4, max_rel(o4["dipole"], o0["dipole"])
    for a, b in zip(p4, p0):
        assert np.max(np.abs(a.astype(np.float64) - b)) < 1e-3


def _smoothed_after(hv, w, parts, steps, **opts):
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.set_fast_options(**opts)
        s.upload_particles(*parts)
        s.run(steps, hv.HV_PATH_FUSED)
        return s.download_field(hv.HV_FIELD_DENSITY), s.download_field(hv.HV_FIELD_DENSITY_RAW)


@pytest.mark.parametrize("wname", ["40Ca-4k-32^3", "208Pb-20.8k-128^3"])
def test_fft_smoothing_matches_the_direct_form(hv, wname):
    """The FFT convolution (power-of-two grids, no density near a face) gives
    the direct march's smoothed density to float rounding: 1e-5 of the
    maximum, the tolerance of the fused fields against the oracle."""
    w = hv.WORKLOADS[wname]
    p32 = hv.workload_particles(w, np.float32)
    d_fft, raw_fft = _smoothed_after(hv, w, p32, 1, smooth_fft=2)
    d_dir, raw_dir = _smoothed_after(hv, w, p32, 1, smooth_fft=0)
    # the two runs' particles differ by the forces' rounding after the first
    # solve (and the atomic deposit's order): a node's CIC counts by a few
    # 1e-6 of a particle, which the smoothing carries into its output
    e_raw = max_rel(raw_fft, raw_dir)
    assert e_raw < 1e-3, e_raw
    assert max_rel(d_fft, d_dir) < 1e-5 + 2.0 * e_raw, (max_rel(d_fft, d_dir), e_raw)
    # no negative densities from the transform's rounding (rho^gamma follows)
    assert d_fft.min() >= 0.0


def _particles_at_faces(w, parts):
    """Copies of the particles with some moved inside the grid next to faces,
    an edge and a corner, where the circular convolution wraps around."""
    p = [a.copy() for a in parts]
    lo = -float(w.n) * w.h / 2.0
    hi = -lo - 1.5 * w.h  # between the last two nodes
    p[0][:40] = lo + 0.6 * w.h                       # protons at the x = min face
    p[1][40:80] = hi                                 # protons at the y = max face
    p[2][-40:] = lo + 0.3 * w.h                      # neutrons at the z = min face
    p[0][80:90], p[1][80:90], p[2][80:90] = lo + 0.2 * w.h, hi, lo + 0.7 * w.h  # a corner
    p[1][-60:-40], p[2][-60:-40] = hi, hi            # neutrons along the y = z = max edge
    return p


def _fft_and_direct_of_one_raw_density(hv, w, parts, deposit_mode):
    """The fused FFT smoothing of one step's raw density, and the direct sum
    (hv_smooth_density, the plain kernel) of the same raw density."""
    wd = replace(w, deposit_mode=deposit_mode)
    with hv.Session.from_workload(wd, hv.HV_F32) as s:
        s.set_fast_options(smooth_fft=2)
        s.upload_particles(*parts)
        s.run(1, hv.HV_PATH_FUSED)
        raw = s.download_field(hv.HV_FIELD_DENSITY_RAW)
        d_fft = s.download_field(hv.HV_FIELD_DENSITY)
        s.smooth()
        d_dir = s.download_field(hv.HV_FIELD_DENSITY)
    return raw, d_fft, d_dir


@pytest.mark.parametrize("wname", ["40Ca-4k-32^3", "208Pb-20.8k-128^3"])
def test_fft_smoothing_with_density_at_faces_keeps_the_truncated_sum(hv, wname):
    """Density within the stencil of a face wraps around in the circular
    convolution.  With the atomic deposit the transform's wrapped pairs are
    subtracted (the wrap correction); the result is the reference's truncated
    sum, as the direct kernel forms it from the same raw density, to the float
    transform's rounding: 1e-5 of the maximum (a few 1e-6 at 128^3), for the
    generic transform (32^3) and the 128^3 one, with density at three faces,
    an edge and a corner.  Uncorrected, the wrapped density of the 40 moved
    test particles would reach about a tenth of the maximum."""
    w = hv.WORKLOADS[wname]
    p32 = _particles_at_faces(w, hv.workload_particles(w, np.float32))
    raw, d_fft, d_dir = _fft_and_direct_of_one_raw_density(hv, w, p32, hv.HV_DEPOSIT_ATOMIC)
    r = raw.reshape(2, w.n, w.n, w.n)
    assert r[0, :2].sum() > 0 and r[0, :, -2:].sum() > 0 and r[1, :, :, :2].sum() > 0  # density at the faces
    assert max_rel(d_fft, d_dir) < 1e-5, max_rel(d_fft, d_dir)
    assert d_fft.min() >= 0.0


def test_fft_smoothing_with_more_face_particles_than_the_wrap_list_holds(hv):
    """Past the wrap list's capacity (65536 particles near faces) the direct
    march recomputes the field: 70,000 of 2.08 M particles moved to the faces,
    the result still the truncated sum of the same raw density."""
    w = hv.WORKLOADS["208Pb-2.08M-128^3"]
    p32 = [a.copy() for a in hv.workload_particles(w, np.float32)]
    lo = -float(w.n) * w.h / 2.0
    rng = np.random.default_rng(7)
    p32[0][:35000] = lo + rng.uniform(0.1, 1.5, 35000).astype(np.float32) * w.h
    p32[2][-35000:] = -lo - rng.uniform(1.1, 2.5, 35000).astype(np.float32) * w.h
    raw, d_fft, d_dir = _fft_and_direct_of_one_raw_density(hv, w, p32, hv.HV_DEPOSIT_ATOMIC)
    assert raw.reshape(2, w.n, w.n, w.n)[0, :2].sum() > 0
    assert max_rel(d_fft, d_dir) < 1e-5, max_rel(d_fft, d_dir)


def test_fft_smoothing_at_faces_in_the_deterministic_mode_uses_the_direct_form(hv):
    """The sort-by-cell deposit mode keeps the smoothing deterministic: with
    density at a face the direct march recomputes the field instead of the
    atomic wrap correction, and two runs agree bit for bit."""
    w = hv.CA40_SMALL
    p32 = _particles_at_faces(w, hv.workload_particles(w, np.float32))
    raw, d_fft, d_dir = _fft_and_direct_of_one_raw_density(hv, w, p32, hv.HV_DEPOSIT_SORTED)
    raw2, d_fft2, _ = _fft_and_direct_of_one_raw_density(hv, w, p32, hv.HV_DEPOSIT_SORTED)
    assert np.array_equal(raw, raw2) and np.array_equal(d_fft, d_fft2)
    assert max_rel(d_fft, d_dir) < 2e-6, max_rel(d_fft, d_dir)


def test_fused_state_and_fields_match_oracle_on_final_positions(hv):
    """After a fused run the plain buffers describe the final state: density,
    potential and forces of the final positions (computed by the oracle from
    those positions and the GPU's Coulomb potential)."""
    from hv_oracle import Oracle
    w = hv.CA40_SMALL
    p32 = hv.workload_particles(w, np.float32)
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.upload_particles(*p32)
        s.initial_solve()
        s.run(3, hv.HV_PATH_FUSED)
        x, y, z, kx, ky, kz = s.download_particles()
        rho = s.download_field(1)
        U = s.download_field(2)
        phi = s.download_field(3)
        Fx = s.download_field(4)
        fz = s.download_array("fz")
    o = Oracle(np.float64)
    world = w.world_tuple()
    x64, y64, z64 = (a.astype(np.float64) for a in (x, y, z))
    rr = o.smooth(world, w.sigma_r, w.ppn, o.deposit(world, w.protons, w.neutrons, x64, y64, z64))
    assert max_rel(rho, rr) < 1e-5
    A, B, C, gm = w.skyrme()
    Uo = o.skyrme(world, A, B, C, gm, rho.astype(np.float64))
    o.merge(world, Uo, phi.astype(np.float64))
    assert max_rel(U, Uo) < 2e-6
    Fo = o.fdm(world, U.astype(np.float64))
    assert max_rel(Fx, Fo[0]) < 1e-4
    fo = o.gather(world, w.protons, w.neutrons, x64, y64, z64, *o.fdm(world, U.astype(np.float64)))
    assert max_rel(fz, fo[2]) < 1e-4
    # phi solves the Poisson problem to the requested tolerance
    assert o.rel_residual(world, phi.astype(np.float64), rho.astype(np.float64)) < 1e-4


def test_fused_runs_continue_across_calls_and_paths(hv):
    """Two fused calls equal one longer call; a plain step after a fused run
    continues from the same state."""
    w = hv.CA40_SMALL
    p = hv.workload_particles(w, np.float64)
    obs1, out1 = _fused(hv, w, 12, hv.HV_F64, p, graph_steps=4)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.set_fast_options(graph_steps=4)
        s.upload_particles(*p)
        s.initial_solve()
        a = s.run(5, hv.HV_PATH_FUSED)
        b = s.run(7, hv.HV_PATH_FUSED)
        out2 = s.download_particles()
        c = s.run(2, hv.HV_PATH_PLAIN)
    d = np.concatenate([a["dipole"], b["dipole"]])
    assert max_rel(d, obs1["dipole"]) < 1e-9
    assert np.max(np.abs(out2[2] - out1[2])) < 1e-9
    assert np.all(np.isfinite(c["dipole"]))
    assert np.allclose(np.concatenate([a["t"], b["t"], c["t"]]), np.arange(14) * w.dt)


def test_forces_on_the_gathered_rows_only_keep_the_run(hv):
    """A float step with the atomic deposit computes the forces only on the
    row groups of the grid that hold raw density, the nodes its particles'
    next gather reads with a nonzero weight (208Pb on 128^3: about an
    eighth of the row groups hold density); the end of a run computes every row
    again for the plain-path view.  Twelve runs of one step each (every
    gather reading forces computed on every row) and one run of twelve steps
    give D(t) and particles equal to float rounding of the atomic deposit's
    order, and the forces downloaded after the run match those the plain
    path computes from the potential the run left."""
    w = hv.PB208_20K_128
    p32 = hv.workload_particles(w, np.float32)
    opts = dict(sort_every=0)
    obs1, out1 = _fused(hv, w, 12, hv.HV_F32, p32, **opts)
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.set_fast_options(**opts)
        s.upload_particles(*p32)
        s.initial_solve()
        parts = [s.run(1, hv.HV_PATH_FUSED) for _ in range(12)]
        out2 = s.download_particles()
        fields = (hv.HV_FIELD_FORCE_X, hv.HV_FIELD_FORCE_Y, hv.HV_FIELD_FORCE_Z)
        f_fused = [s.download_field(fld) for fld in fields]
        # the plain path's forces of the potential the run left
        s.forces()
        f_plain = [s.download_field(fld) for fld in fields]
    d = np.concatenate([o["dipole"] for o in parts])
    assert np.allclose(np.concatenate([o["t"] for o in parts]), obs1["t"])
    assert max_rel(d, obs1["dipole"]) < 1e-5, max_rel(d, obs1["dipole"])
    for a, b in zip(out1[:6], out2[:6]):
        assert np.max(np.abs(a - b)) <= 1e-5 * max(1.0, float(np.max(np.abs(a))))
    for a, b in zip(f_fused, f_plain):
        scale = float(np.max(np.abs(b)))
        assert scale > 0 and np.max(np.abs(a - b)) <= 1e-5 * scale, (np.max(np.abs(a - b)), scale)


def test_graph_and_direct_launch_agree(hv):
    w = hv.CA40_SMALL
    p = hv.workload_particles(w, np.float64)
    og, _ = _fused(hv, w, 16, hv.HV_F64, p, graph_steps=8)
    od, _ = _fused(hv, w, 16, hv.HV_F64, p, graph_steps=0)
    assert max_rel(og["dipole"], od["dipole"]) < 1e-12


@pytest.mark.parametrize("n", [(20, 16, 24), (33, 17, 9)])
def test_fused_odd_grids(hv, n):
    """Non-cubic and odd grids: fused F64 tracks the plain F64 path."""
    w = replace(hv.CA40_SMALL, name="odd", n=n[0])
    # anisotropic world through the session directly
    from hv_b200 import _lib as L
    world = L.hv_world()
    for a in range(3):
        world.n[a] = n[a]
        world.d_max[a] = 0.5 * n[a] * 1.0
    params = w.run_params()
    p = hv.workload_particles(w, np.float64)
    res = []
    for path in (hv.HV_PATH_PLAIN, hv.HV_PATH_FUSED):
        with hv.Session(world, w.protons, w.neutrons, params, hv.HV_F64) as s:
            s.upload_particles(*p)
            s.initial_solve()
            res.append(s.run(8, path))
    assert max_rel(res[1]["dipole"], res[0]["dipole"]) < 1e-6


def test_sor_cap_is_reported_per_step(hv):
    """A run whose SOR would need more than max_iter iterations reports the
    non-converged steps through the row flags and keeps going."""
    w = replace(hv.CA40_SMALL, sor_max_iter=3)
    p = hv.workload_particles(w, np.float64)
    obs, _ = _fused(hv, w, 4, hv.HV_F64, p)
    assert np.all(obs["flags"] & 1)
    assert np.all(obs["sor_iterations"] <= 3)


def _world(n, h):
    from hv_b200 import _lib as L
    world = L.hv_world()
    for a in range(3):
        world.n[a] = n[a]
        world.d_max[a] = 0.5 * n[a] * h
    return world


@pytest.mark.parametrize("n", [(32, 32, 32), (128, 128, 128), (200, 16, 16), (6, 256, 256)])
def test_tagged_exchange_matches_flag_exchange(hv, n):
    """The tagged and the phase-counter exchange of the fused SOR run the same
    arithmetic in the same order; the float deposit's atomic summation order is
    the only run-to-run difference, so the runs agree to float rounding: D(t)
    and the Coulomb potential within 1e-5 relative, the same iteration counts
    up to one residual check.  The shapes cover one plane per block, several
    planes per block (200 x 16 x 16) and a plane split across blocks along y
    (6 x 256 x 256)."""
    w = hv.PB208_20K_128 if n[0] == 128 else hv.CA40_SMALL
    world = _world(n, w.h)
    p = hv.workload_particles(w, np.float32)
    res = []
    for exchange in (hv.HV_SOR_EXCHANGE_FLAGS, hv.HV_SOR_EXCHANGE_AUTO):
        with hv.Session(world, w.protons, w.neutrons, w.run_params(), hv.HV_F32) as s:
            s.set_fast_options(sor_exchange=exchange, sor_coarse=0)
            s.upload_particles(*p)
            s.initial_solve()
            obs = s.run(4, hv.HV_PATH_FUSED)
            res.append((obs, s.download_particles(), s.download_field(hv.HV_FIELD_COULOMB)))
    (o0, p0, c0), (o1, p1, c1) = res
    assert np.all(o0["sor_iterations"] > 0) and not np.any(o1["flags"] & 1)
    assert np.all(np.abs(o0["sor_iterations"] - o1["sor_iterations"]) <= 64)
    assert max_rel(o1["dipole"], o0["dipole"]) < 1e-5
    assert max_rel(c1, c0) < 1e-5
    assert all(np.max(np.abs(a - b)) < 1e-4 for a, b in zip(p0, p1))


@pytest.mark.parametrize("wname", ["40Ca-4k-32^3", "208Pb-104k-64^3", "208Pb-20.8k-128^3"])
def test_fused_smoothing_matches_direct_sum(hv, wname):
    """The fused path's decomposed smoothing (z-runs and disc sums marched along
    x) on the raw density of a fused run's final state, against the direct tap
    sum of hv_smooth_density in double on the same raw density: within 5e-6
    relative, and no further from it than twice the float direct sum is (both
    float results carry the rounding of sums of up to ~4000 terms)."""
    w = hv.WORKLOADS[wname]
    p = hv.workload_particles(w, np.float32)
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.upload_particles(*p)
        s.run(2, hv.HV_PATH_FUSED)
        fast = s.download_field(hv.HV_FIELD_DENSITY)
        raw = s.download_field(hv._lib.HV_FIELD_DENSITY_RAW)
        s.smooth()
        direct = s.download_field(hv.HV_FIELD_DENSITY)
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        s.upload_field(hv._lib.HV_FIELD_DENSITY_RAW, raw.astype(np.float64))
        s.smooth()
        ref = s.download_field(hv.HV_FIELD_DENSITY)
    assert np.abs(ref).max() > 0
    e_fast, e_direct = max_rel(fast, ref), max_rel(direct, ref)
    assert e_fast < 5e-6
    assert e_fast <= 2 * e_direct + 1e-7


def test_fused_f32_104k_dipole_and_spectrum_match_double_oracle(hv):
    """208Pb with 104,000 test particles on 64^3 at h = 0.5 fm, dt 0.25 fm/c:
    the FP32 fused path (default solve) against the FP64 oracle over 120
    steps -- D(t) within 1e-3 of the oracle's largest |D|, and the strength
    function S(E) of the two D(t) series (detrended, cos^2-windowed FFT as the
    reference's post-processing, scripts/programs.py:82-122) within 1e-3 of
    the oracle's largest |S|."""
    import os
    from hv_b200.spectrum import energy_spectrum
    w = hv.PB208_104K
    steps = 120
    p32 = hv.workload_particles(w, np.float32)
    from hv_oracle import Oracle
    o = Oracle(np.float64)
    o.set_threads(os.cpu_count() or 4)
    a = [p.astype(np.float64) for p in p32]
    obs_o, _ = o.simulate(w.world_tuple(), _oracle_runspec(w), w.protons, w.neutrons, *a, steps)
    obs, _ = _fused(hv, w, steps, hv.HV_F32, p32)
    assert not np.any(obs["flags"] & 1)
    assert max_rel(obs["dipole"], obs_o["dipole"]) <= 1e-3
    t_f = steps * w.dt
    eo, so = energy_spectrum(obs_o["t"], obs_o["zcm_p"], obs_o["zcm_n"], w.Z, w.N, t_f, w.dt, w.eta)
    eg, sg = energy_spectrum(obs["t"], obs["zcm_p"], obs["zcm_n"], w.Z, w.N, t_f, w.dt, w.eta)
    assert np.allclose(eg, eo)
    assert max_rel(sg, so) <= 1e-3


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_fused_sorted_deposit_is_deterministic(hv, prec):
    """HV_DEPOSIT_SORTED on the fused path: every node sums its particles in
    slot order, so two runs give bit-identical D(t) and particles (the atomic
    deposit's summation order varies run to run); the two modes agree to the
    float rounding of the deposit."""
    dt = np.float32 if prec == "f32" else np.float64
    P = hv.HV_F32 if prec == "f32" else hv.HV_F64
    w = replace(hv.CA40_SMALL, deposit_mode=hv.HV_DEPOSIT_SORTED)
    p = hv.workload_particles(w, dt)
    runs = [_fused(hv, w, 30, P, p) for _ in range(2)]
    assert np.array_equal(runs[0][0]["dipole"], runs[1][0]["dipole"])
    assert all(np.array_equal(a, b) for a, b in zip(runs[0][1], runs[1][1]))
    obs_a, _ = _fused(hv, replace(w, deposit_mode=hv.HV_DEPOSIT_ATOMIC), 30, P, p)
    assert max_rel(runs[0][0]["dipole"], obs_a["dipole"]) < (1e-5 if prec == "f32" else 1e-10)


def test_bounded_waits_time_out_and_the_context_recovers(hv):
    """hv_fast_options.sor_wait_limit bounds every device-side wait of the
    fused solver.  With a limit of one poll the blocks' grid barriers and
    neighbour rows give up, the kernel returns and the run reports
    HV_ERR_TIMEOUT (the reference's solver would instead warn and carry on,
    include/physics.hpp:155-156); with the default limit restored, the same
    context solves normally again and matches a new context's run."""
    from hv_b200 import _lib as L
    w = hv.PB208_104K
    p32 = hv.workload_particles(w, np.float32)
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        # 64^3 takes several blocks of the solver, so some of them must wait
        s.set_fast_options(sor_wait_limit=1)
        s.upload_particles(*p32)
        with pytest.raises(hv.HVError) as e:
            s.run(2, hv.HV_PATH_FUSED)
        assert e.value.status == L.HV_ERR_TIMEOUT
        s.set_fast_options(sor_wait_limit=0)
        s.upload_particles(*p32)
        obs = s.run(6, hv.HV_PATH_FUSED)
    assert not np.any(obs["flags"] & 1)
    obs_new, _ = _fused(hv, w, 6, hv.HV_F32, p32)
    assert max_rel(obs["dipole"], obs_new["dipole"]) < 1e-6, max_rel(obs["dipole"], obs_new["dipole"])


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_uploads_and_downloads_follow_the_slot_permutation(hv, prec):
    """After fused runs have re-sorted the slots, particles uploaded (all
    arrays, or one at a time) come back in the caller's order, bit for bit, in
    both precisions; and D(t) after the re-sort matches an unsorted run."""
    w = hv.CA40_SMALL
    dt = np.float32 if prec == "f32" else np.float64
    P = hv.HV_F32 if prec == "f32" else hv.HV_F64
    parts = hv.workload_particles(w, dt)
    rng = np.random.default_rng(5)
    with hv.Session.from_workload(w, P) as s:
        s.set_fast_options(sort_every=4)
        s.upload_particles(*parts)
        s.run(12, hv.HV_PATH_FUSED)
        new = [(p + dt(0.1) * rng.standard_normal(p.size).astype(dt)).astype(dt) for p in parts]
        s.upload_particles(*new)
        got = s.download_particles()
        for a, b in zip(got, new):
            assert a.tobytes() == b.tobytes()
        one = (new[2] * dt(0.5)).astype(dt)
        s.upload_array("z", one)
        assert s.download_array("z").tobytes() == one.tobytes()


@pytest.mark.parametrize("wname,n", [("208Pb-20.8k-128^3", (128, 128, 128)), ("208Pb-104k-64^3", (64, 64, 64)),
                                     ("40Ca-4k-32^3", (32, 32, 32)), ("40Ca-4k-32^3", (64, 32, 128))])
def test_coarse_grid_correction_keeps_the_stopping_rule(hv, wname, n):
    """The coarse-grid correction of the fused float solve (the default) ends
    every solve at the same FP64 stopping rule as plain SOR cycles: D(t) and
    the Coulomb potential agree within 1e-6 relative (the tolerance of each
    solve), the particles to float rounding, and the iterations per step fall
    below the plain cycles' -- to under 0.6 of them on the cubic grids of 64
    nodes and more (coarse factors 8 and 4, and a non-cubic grid with 8 on
    each axis, whose coarse grid has only 3 interior nodes along y).  A grid
    of fewer than 48^3 nodes (32^3) runs plain cycles either way."""
    w = hv.WORKLOADS[wname]
    world = _world(n, w.h)
    p = hv.workload_particles(w, np.float32)
    res = []
    for coarse in (0, 1):
        with hv.Session(world, w.protons, w.neutrons, w.run_params(), hv.HV_F32) as s:
            s.set_fast_options(sor_coarse=coarse)
            s.upload_particles(*p)
            s.initial_solve()
            obs = s.run(12, hv.HV_PATH_FUSED)
            res.append((obs, s.download_particles(), s.download_field(hv.HV_FIELD_COULOMB)))
    (o0, p0, c0), (o1, p1, c1) = res
    assert not np.any(o0["flags"] & 1) and not np.any(o1["flags"] & 1)
    assert max_rel(o1["dipole"], o0["dipole"]) < 1e-6, max_rel(o1["dipole"], o0["dipole"])
    assert max_rel(c1, c0) < 1e-6, max_rel(c1, c0)
    assert all(np.max(np.abs(a - b)) < 1e-4 for a, b in zip(p0, p1))
    its0, its1 = o0["sor_iterations"][2:].mean(), o1["sor_iterations"][2:].mean()
    assert its1 <= its0 + 16, (its1, its0)  # 32^3 (under 48^3 nodes) runs plain cycles either way
    if n[0] * n[1] * n[2] >= 48 ** 3:
        assert its1 < its0, (its1, its0)
    if n[0] == n[1] == n[2] and n[0] >= 64:
        assert its1 < 0.6 * its0, (its1, its0)



@pytest.mark.parametrize("wname", ["40Ca-4k-32^3", "208Pb-104k-64^3"])
def test_warp_aggregated_deposit_matches_the_oracle(hv, wname):
    """The fused float deposit summed over warp runs of equal base nodes
    (hv_fast_options.deposit_aggregate, the default) against one set of
    atomics per particle and against the oracle's deposit of the same final
    positions: the raw density within float rounding (1e-5 of its maximum),
    after re-sorted slots (sort_every = 1) and from unsorted ones."""
    from hv_oracle import Oracle
    w = hv.WORKLOADS[wname]
    p32 = hv.workload_particles(w, np.float32)
    o = Oracle(np.float32)
    for every in (0, 1):
        raws = []
        for agg in (0, 1):
            with hv.Session.from_workload(w, hv.HV_F32) as s:
                s.set_fast_options(deposit_aggregate=agg, sort_every=every)
                s.upload_particles(*p32)
                s.run(3, hv.HV_PATH_FUSED)
                raws.append(s.download_field(hv.HV_FIELD_DENSITY_RAW))
                x, y, z, *_ = s.download_particles()
        ref = o.deposit(w.world_tuple(), w.protons, w.neutrons, x, y, z)
        assert max_rel(raws[1], ref) < 1e-5, (every, max_rel(raws[1], ref))
        assert max_rel(raws[0], raws[1]) < 1e-3  # the two runs' particles differ by rounding


def test_autotune_chooses_a_configuration_and_keeps_results(hv):
    """hv_ctx_autotune times the particle step's block sizes and grids and the
    SOR's best-ranked tiles, keeps the fastest, and the run continues with the
    same physics: D(t) of the steps after it matches a run that advanced the
    same number of steps without it (float rounding of the atomic deposit
    aside: 1e-4)."""
    w = hv.PB208_20K_128
    p32 = hv.workload_particles(w, np.float32)
    trial = 2
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.upload_particles(*p32)
        rep = s.autotune(trial)
        obs_a = s.run(8, hv.HV_PATH_FUSED)
    assert rep["particle_block"] in (128, 256, 512)
    assert rep["particle_grid"] > 0
    assert rep["sor_planes"] >= 1 and rep["sor_rows"] >= 1 and rep["sor_blocks"] >= 1
    assert 0 <= rep["sor_tile_rank"] < 4 and rep["candidates"] >= 10
    assert rep["particle_ms"] > 0 and rep["sor_ms"] > 0
    steps_taken = int(round(obs_a["t"][0] / w.dt))
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.upload_particles(*p32)
        s.run(steps_taken, hv.HV_PATH_FUSED)
        obs_b = s.run(8, hv.HV_PATH_FUSED)
    assert np.allclose(obs_a["t"], obs_b["t"])
    assert max_rel(obs_a["dipole"], obs_b["dipole"]) < 1e-4, max_rel(obs_a["dipole"], obs_b["dipole"])
