"""GPU: every routine of the plain path, called through the C ABI, against the
golden vectors produced by the reference's own routines.

Tolerances (max|gpu - ref| / max|ref|):
  HV_F64  bit-identical for deposit (sorted mode), boundary, SOR, merge, FDM,
          gather, kick, drift, excite; smoothing bit-identical on grids with
          exact node coordinates and <= 1e-14 otherwise; Skyrme <= 1e-15 (CUDA's
          pow and glibc's may differ in the last bit); atomic deposit <= 1e-14.
  HV_F32  as above where the operation order is the same (float rounding is
          deterministic); Skyrme <= 5e-7 (CUDA's powf and glibc's differ by a
          few ulp), atomic deposit <= 1e-6.
"""
from __future__ import annotations

import numpy as np
import pytest
from conftest import max_rel

pytestmark = pytest.mark.gpu

FIXTURES = [("ca40_stages_f64.npz", "f64", True), ("edge_f64.npz", "f64", False), ("ca40_stages_f32.npz", "f32", True)]


def session_for(hv, g, prec, deposit_mode=0):
    from hv_b200 import _lib as L
    w = L.hv_world()
    for a in range(3):
        w.n[a] = int(g["n"][a])
        w.d_max[a] = float(g["d_max"][a])
    p = L.hv_run_params()
    p.z, p.n, p.part_per_nucleon = int(g["Z"]), int(g["N"]), int(g["ppn"])
    p.sigma_r, p.dt, p.t_exc, p.eta_exc = float(g["sigma_r"]), float(g["dt"]), 0.0, float(g["eta"])
    p.skyrme = L.hv_skyrme(*(float(v) for v in g["skyrme"]))
    p.sor = L.hv_sor_params(1.5, 1e-4, L.HV_SOR_MAX_UPDATE, 512)
    p.deposit_mode = deposit_mode
    return hv.Session(w, int(g["protons"]), int(g["neutrons"]), p, hv.HV_F64 if prec == "f64" else hv.HV_F32)


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_deposit_sorted_is_bit_identical(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec, hv.HV_DEPOSIT_SORTED) as s:
        s.upload_particles(g["x"], g["y"], g["z"], None, None, None)
        s.deposit()
        rho = s.download_field(0)
        assert np.array_equal(rho, g["rho_raw"]), max_rel(rho, g["rho_raw"])
        s.deposit()
        assert np.array_equal(s.download_field(0), rho)


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_deposit_atomic_within_rounding(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec, hv.HV_DEPOSIT_ATOMIC) as s:
        s.upload_particles(g["x"], g["y"], g["z"], None, None, None)
        s.deposit()
        rho = s.download_field(0)
        assert max_rel(rho, g["rho_raw"]) <= (1e-14 if prec == "f64" else 1e-6)
        # the cell assignment is exact: the same nodes are touched
        assert np.array_equal(rho != 0, g["rho_raw"] != 0)
        assert abs(rho.sum() - g["rho_raw"].sum()) <= (1e-9 if prec == "f64" else 1e-2)


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_smoothing(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec) as s:
        s.upload_field(0, g["rho_raw"])
        s.smooth()
        rho = s.download_field(1)
        if exact_grid:
            assert np.array_equal(rho, g["rho"]), max_rel(rho, g["rho"])
        else:
            assert max_rel(rho, g["rho"]) < 1e-14


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_skyrme(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec) as s:
        s.upload_field(1, g["rho"])
        s.skyrme()
        U = s.download_field(2)
        assert max_rel(U, g["U"]) <= (1e-15 if prec == "f64" else 5e-7)


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_boundary_and_sor_bit_identical(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec) as s:
        s.coulomb_boundary()
        phi = s.download_field(3)
        assert np.array_equal(phi, g["phi_boundary"]), max_rel(phi, g["phi_boundary"])
        s.upload_field(1, g["rho"])
        it, m, ok = s.coulomb_sor(allow_not_converged=True)
        phi = s.download_field(3)
        assert np.array_equal(phi, g["phi"]), max_rel(phi, g["phi"])
        assert ok and m < 1e-4


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_merge_fdm_gather_bit_identical(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec) as s:
        s.upload_field(2, g["U"])
        s.upload_field(3, g["phi"])
        s.merge()
        U = s.download_field(2)
        assert np.array_equal(U, g["U_merged"])
        s.forces()
        for f, k in zip((4, 5, 6), ("Fx", "Fy", "Fz")):
            F = s.download_field(f)
            assert np.array_equal(F, g[k]), (k, max_rel(F, g[k]))
        s.upload_particles(g["x"], g["y"], g["z"], None, None, None)
        s.gather()
        for k in ("fx", "fy", "fz"):
            v = s.download_array(k)
            assert np.array_equal(v, g[k]), (k, max_rel(v, g[k]))


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES)
def test_push_and_excite_bit_identical(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    dt = float(g["dt"])
    with session_for(hv, g, prec) as s:
        s.upload_particles(g["x"], g["y"], g["z"], g["kx"], g["ky"], g["kz"])
        for k in ("fx", "fy", "fz"):
            s.upload_array(k, g[k])
        s.kick_half(dt)
        for k in ("kx", "ky", "kz"):
            assert np.array_equal(s.download_array(k), g[k + "_kick"]), k
        s.drift(dt)
        for k in ("x", "y", "z"):
            assert np.array_equal(s.download_array(k), g[k + "_drift"]), k
        s.upload_particles(None, None, None, None, None, g["kz"])
        s.excite(float(g["eta"]))
        assert np.array_equal(s.download_array("kz"), g["kz_excite"])


@pytest.mark.parametrize("fixture,prec,exact_grid", FIXTURES[:2])
def test_observables(hv, golden, fixture, prec, exact_grid):
    g = golden(fixture)
    with session_for(hv, g, prec) as s:
        s.upload_particles(g["x"], g["y"], g["z"], None, None, None)
        o = s.observe()
        assert abs(o.zcm_p - g["com"][0]) < 1e-12 and abs(o.zcm_n - g["com"][1]) < 1e-12
        assert abs(o.rms_p ** 2 - g["msr"][0]) < 1e-11 and abs(o.rms_n ** 2 - g["msr"][1]) < 1e-11
        Z, N = int(g["Z"]), int(g["N"])
        assert abs(o.dipole - N * Z / (N + Z) * (o.zcm_p - o.zcm_n)) < 1e-14
