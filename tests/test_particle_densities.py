"""compute_particle_densities (include/tools.hpp:170-203).

CPU: the oracle's restatement against the reference's own routine (compiled
from source): bit-identical in double, within 1e-6 relative in float.
GPU: hv_particle_densities (cell lists) against the oracle (index-order sums):
within 1e-12 relative to the largest density in double, 2e-5 in float."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from hv_oracle import Oracle, Reference, reference_available


def _case(hv, ppn=20):
    w = replace(hv.CA40_SMALL, ppn=ppn)
    return w, hv.workload_particles(w, np.float64)


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_particle_densities_match_reference(hv, dtype):
    w, p = _case(hv)
    x, y, z = (a.astype(dtype) for a in p[:3])
    ro = Reference(dtype).particle_densities(w.protons, w.neutrons, x, y, z, w.sigma_r, w.ppn)
    oo = Oracle(dtype).particle_densities(w.protons, w.neutrons, x, y, z, w.sigma_r, w.ppn)
    for a, b in zip(oo, ro):
        if dtype == np.float64:
            assert np.array_equal(a, b)
        else:
            assert np.max(np.abs(a - b)) <= 1e-6 * np.abs(b).max()
    assert np.all(ro[0] > 0) and np.all(ro[1] > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gpu_particle_densities(hv, prec):
    w, p = _case(hv, ppn=50)
    dtype = np.float64 if prec == "f64" else np.float32
    pp = [a.astype(dtype) for a in p]
    with hv.Session.from_workload(w, hv.HV_F64 if prec == "f64" else hv.HV_F32) as s:
        s.upload_particles(*pp)
        dp, dn = s.particle_densities()
    op, on = Oracle(dtype).particle_densities(w.protons, w.neutrons, *pp[:3], w.sigma_r, w.ppn)
    tol = 1e-12 if prec == "f64" else 2e-5
    for a, b in ((dp, op), (dn, on)):
        assert np.max(np.abs(a - b)) <= tol * np.abs(b).max()


@pytest.mark.gpu
def test_gpu_particle_densities_after_a_fused_run(hv):
    """After a fused run (which may reorder the particle slots) the densities
    come back in the caller's particle order."""
    w, p = _case(hv, ppn=30)
    pp = [a.astype(np.float32) for a in p]
    with hv.Session.from_workload(w, hv.HV_F32) as s:
        s.upload_particles(*pp)
        s.run(3, hv.HV_PATH_FUSED)
        x, y, z, *_ = s.download_particles()
        dp, dn = s.particle_densities()
    op, on = Oracle(np.float32).particle_densities(w.protons, w.neutrons, x, y, z, w.sigma_r, w.ppn)
    assert np.max(np.abs(dp - op)) <= 2e-5 * np.abs(op).max()
    assert np.max(np.abs(dn - on)) <= 2e-5 * np.abs(on).max()
