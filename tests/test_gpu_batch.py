"""GPU: batched runs (hv_batch_*) against the same instances run one by one.

Six instances drawn like the 64-run batched workload (nuclei 16O..208Pb,
grids 32^3..96^3 at h = 0.5 fm, jittered Skyrme parameters and boosts), with
at most 100 test particles per nucleon to keep the test short.  Tolerance:
D(t) of every instance within 1e-4 of its largest |D| against the instance's
own fused run (the float atomic deposit makes two runs of one instance differ
at ~1e-6); with the instances' own plans, SOR iteration counts within one
residual check (256)."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _instances(hv, n=6, seed=7):
    from hv_b200.workloads import batch_workloads
    return [replace(w, ppn=min(w.ppn, 100)) for w in batch_workloads(n, seed=seed)]


def _sessions(hv, ws):
    out = []
    for w in ws:
        s = hv.Session.from_workload(w, hv.HV_F32)
        s.upload_particles(*hv.workload_particles(w, np.float32))
        out.append(s)
    return out


@pytest.mark.parametrize("cap", [0, 8])
def test_batch_matches_individual_runs(hv, cap):
    from hv_b200.batch import Batch
    ws = _instances(hv)
    steps = 16
    alone = []
    for s in _sessions(hv, ws):
        with s:
            alone.append(s.run(steps, hv.HV_PATH_FUSED))
    sess = _sessions(hv, ws)
    try:
        with Batch(sess) as b:
            b.plan(cap)
            assert b.waves() >= 1
            obs = b.run(steps)
    finally:
        for s in sess:
            s.close()
    for i, a in enumerate(alone):
        d = np.abs(a["dipole"]).max()
        assert d > 0
        assert np.max(np.abs(obs[i]["dipole"] - a["dipole"])) <= 1e-4 * d, ws[i].name
        if cap == 0:
            # the instances' own plans: the same solver as their lone runs (a
            # cap can force the generic sweep, whose plain cycles take more)
            assert np.all(np.abs(obs[i]["sor_iterations"] - a["sor_iterations"]) <= 256)
        assert not np.any(obs[i]["flags"] & 1)
        assert np.allclose(obs[i]["t"], a["t"])


def test_batch_autotune_and_continued_runs(hv):
    """The autotuner picks a cap among its candidates; runs continue across
    calls (step counters and time advance per instance)."""
    from hv_b200.batch import Batch
    ws = _instances(hv, n=4, seed=11)
    sess = _sessions(hv, ws)
    try:
        with Batch(sess) as b:
            cap = b.autotune(2)
            assert cap in (0, 64, 32, 16, 8, 4)
            tiles = b.tiles()
            assert len(tiles) == len(ws)
            assert all(P >= 1 and R >= 1 and nb >= 1 and pb in (128, 256, 512) for P, R, nb, pb in tiles)
            assert len({pb for *_, pb in tiles}) == 1  # one particle block size for all
            o1 = b.run(8)
            o2 = b.run(9)
    finally:
        for s in sess:
            s.close()
    for i, w in enumerate(ws):
        # autotune ran 1 + 2 steps per candidate before o1
        assert np.isclose(o2[i]["t"][0] - o1[i]["t"][0], 8 * w.dt)
        assert np.all(np.isfinite(o2[i]["dipole"]))


def test_batch_rejects_double_contexts(hv):
    from hv_b200.batch import Batch
    w = hv.CA40_SMALL
    with hv.Session.from_workload(w, hv.HV_F64) as s:
        with pytest.raises(hv.HVError):
            Batch([s])


def test_batch_instances_of_every_nucleus_match_the_double_oracle(hv):
    """The 64-run batched workload (full test-particle counts) advanced
    together for 40 steps; for one instance of each nucleus (16O, 40Ca, 90Zr,
    208Pb: the smallest of each), D(t) within 1e-3 of the double oracle's
    largest |D| from the same float particles -- the FP32 form's accuracy
    bound, checked on the batched form."""
    import os

    from hv_b200.batch import Batch
    from hv_b200.workloads import batch_workloads
    from hv_oracle import Oracle, RunSpec
    from conftest import max_rel
    ws = batch_workloads(64, seed=0)
    steps = 40
    pick = {}
    for i, w in enumerate(ws):
        key = w.name.split("-")[0]
        if key not in pick or w.particles + w.G < ws[pick[key]].particles + ws[pick[key]].G:
            pick[key] = i
    assert sorted(pick) == ["16O", "208Pb", "40Ca", "90Zr"]
    sess = _sessions(hv, ws)
    try:
        with Batch(sess) as b:
            obs = b.run(steps)
    finally:
        for s in sess:
            s.close()
    o = Oracle(np.float64)
    o.set_threads(os.cpu_count() or 4)
    for key, i in sorted(pick.items()):
        w = ws[i]
        A, B, C, gm = w.skyrme()
        run = RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc,
                      eta_exc=w.eta, A=A, B=B, C=C, gamma=gm, sor_omega=w.sor_omega, sor_tol=w.sor_tol,
                      sor_criterion=w.sor_criterion, sor_max_iter=w.sor_max_iter)
        p = [a.astype(np.float64) for a in hv.workload_particles(w, np.float32)]
        obs_o, _ = o.simulate(w.world_tuple(), run, w.protons, w.neutrons, *p, steps)
        assert not np.any(obs[i]["flags"] & 1), w.name
        err = max_rel(obs[i]["dipole"], obs_o["dipole"])
        assert err <= 1e-3, (w.name, err)
