"""The initialisation loop on the device (hv_initialize_particles and its
parts) against the reference.

* hv_particle_energies vs the reference's compute_particle_energies: 1e-15
  relative in double, 1e-6 in float.
* hv_fit_woods_saxon vs the oracle's restatement of the fit on the same
  particles and densities: parameters within 1e-9 relative in double (only the
  order of the sums differs), same status.
* hv_initialize_particles with HV_RNG_LIBC after srand(128) against the golden
  run of the reference's own loop (tests/golden/init_ca40_f64.npz, 40Ca, 4000
  particles, 32 passes): the same particles (1e-12), Woods-Saxon parameters
  and Fermi levels (1e-9).
* HV_RNG_PHILOX: the same loop with device random numbers reaches the same
  self-consistent state within the sampling noise, in double and float.
* Bad arguments and an unreachable Fermi level end with an error status.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace

import numpy as np
import pytest

from hv_oracle import Oracle

pytestmark = pytest.mark.gpu

LIBC = C.CDLL(None)


def _fixture(golden):
    return golden("init_ca40_f64.npz")


def _ws(g, key):
    w = g[key]
    return (tuple(w[0]), tuple(w[1]))


def _session(hv, g, precision, ppn=None):
    w = replace(hv.CA40_SMALL, Z=int(g["Z"]), N=int(g["N"]), ppn=int(ppn or g["ppn"]), sigma_r=float(g["sigma_r"]))
    p = w.run_params()
    A, B, Cc, gam = (float(v) for v in g["skyrme"])
    p.skyrme = hv._lib.hv_skyrme(A, B, Cc, gam)
    return hv.Session(w.world(), w.protons, w.neutrons, p, precision)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gpu_particle_energies(hv, golden, prec):
    g = _fixture(golden)
    dtype = np.float64 if prec == "f64" else np.float32
    arrs = [g[k].astype(dtype) for k in ("x", "y", "z", "kx", "ky", "kz")]
    ws = _ws(g, "ws")
    with _session(hv, g, hv.HV_F64 if prec == "f64" else hv.HV_F32) as s:
        s.upload_particles(*arrs)
        e = s.particle_energies(ws, float(g["sigma_k"]))
    ref = Oracle(dtype).particle_energies(s.protons, s.neutrons, *arrs, ws, float(g["sigma_k"]), int(g["Z"]))
    tol = 1e-15 if prec == "f64" else 1e-6
    assert np.max(np.abs(e - ref)) <= tol * np.abs(ref).max()
    if prec == "f64":
        assert np.max(np.abs(e - g["energy"])) <= tol * np.abs(g["energy"]).max()


def test_gpu_fit_matches_the_oracle(hv, golden):
    g = _fixture(golden)
    arrs = [g[k] for k in ("x", "y", "z", "kx", "ky", "kz")]
    start = _ws(g, "ws0")
    with _session(hv, g, hv.HV_F64) as s:
        s.upload_particles(*arrs)
        dp, dn = s.particle_densities()
        fitted, iters, status = s.fit_woods_saxon(start)
    P = s.protons
    o = Oracle(np.float64)
    for sp, sl in ((0, slice(0, P)), (1, slice(P, None))):
        x, y, z = (np.ascontiguousarray(a[sl]) for a in arrs[:3])
        ws_o, it_o, st_o = o.fit_woods_saxon(x, y, z, np.ascontiguousarray(dp[sl]), np.ascontiguousarray(dn[sl]), sp,
                                             g["skyrme"], start[sp])
        assert status[sp] == st_o and iters[sp] == it_o
        assert np.allclose(fitted[sp], ws_o, rtol=1e-9, atol=0)


def test_gpu_init_libc_reproduces_the_reference_loop(hv, golden):
    g = _fixture(golden)
    with _session(hv, g, hv.HV_F64) as s:
        LIBC.srand(int(g["seed"]))
        ws, fermi, rep, rows = s.initialize_particles(_ws(g, "ws0"), tuple(g["fermi0"]), sigma_k=float(g["sigma_k"]),
                                                      rng=hv.HV_RNG_LIBC)
        parts = s.download_particles()
    assert rep["iterations"] == int(g["passes"]) == len(rows)
    assert rep["max_test_part"] == int(g["max_test_part"])
    assert rep["r_max"] == pytest.approx(float(g["r_max"]), rel=1e-15)
    for a, k in zip(parts, ("x", "y", "z", "kx", "ky", "kz")):
        assert np.max(np.abs(a - g[k])) <= 1e-12 * np.abs(g[k]).max(), k
    assert np.allclose(np.array(ws), g["ws"], rtol=1e-9, atol=0)
    assert np.allclose(np.array(fermi), g["fermi"], rtol=1e-9, atol=0)
    assert rows[-1]["ws"] == ws and (rows[-1]["epsilon_p"], rows[-1]["epsilon_n"]) == fermi


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gpu_init_philox_reaches_the_same_state(hv, golden, prec):
    """Device random numbers: a different sample of the same distribution.
    200 test particles per nucleon, where the reference's loop converges; the
    self-consistent parameters agree with the HV_RNG_LIBC run within the
    sampling noise."""
    g = _fixture(golden)
    res = {}
    for rng, precision in (("libc", hv.HV_F64), ("philox", hv.HV_F64 if prec == "f64" else hv.HV_F32)):
        with _session(hv, g, precision, ppn=200) as s:
            LIBC.srand(int(g["seed"]))
            res[rng] = s.initialize_particles(_ws(g, "ws0"), tuple(g["fermi0"]), sigma_k=float(g["sigma_k"]),
                                              rng=hv.HV_RNG_LIBC if rng == "libc" else hv.HV_RNG_PHILOX, seed=7)
            parts = s.download_particles()
        x = parts[0]
        assert np.all(np.isfinite(x)) and np.array_equal(x[1::2], -x[0::2])
    (ws_l, f_l, rep_l, _), (ws_p, f_p, rep_p, _) = res["libc"], res["philox"]
    assert rep_l["converged"] and rep_p["iterations"] >= 2
    for sp in range(2):
        assert abs(ws_p[sp][0] - ws_l[sp][0]) < 3.0      # V0 (MeV)
        assert abs(ws_p[sp][1] - ws_l[sp][1]) < 0.15     # R12 (fm)
        assert abs(ws_p[sp][2] - ws_l[sp][2]) < 0.12     # a (fm)
        assert abs(f_p[sp] - f_l[sp]) < 1.0              # Fermi level (MeV)


def test_gpu_init_bad_arguments(hv, golden):
    g = _fixture(golden)
    w = replace(hv.CA40_SMALL, Z=20, N=20, ppn=100, sigma_r=float(g["sigma_r"]))
    # particle counts other than Z ppn / N ppn
    with hv.Session(w.world(), w.protons - 2, w.neutrons, w.run_params(), hv.HV_F64) as s:
        with pytest.raises(hv.HVError):
            s.initialize_particles(_ws(g, "ws0"), tuple(g["fermi0"]))
    # an odd total (the reference would write one particle past its arrays)
    w3 = replace(w, Z=3, N=4, ppn=1)
    with hv.Session(w3.world(), 3, 4, w3.run_params(), hv.HV_F64) as s:
        with pytest.raises(hv.HVError):
            s.initialize_particles(_ws(g, "ws0"), tuple(g["fermi0"]))


def test_gpu_init_unreachable_level_is_an_error(hv, golden):
    """A repulsive well puts every temporary particle above the levels: the
    level update divides by zero (physics.hpp:64-67) and the reference would
    draw candidates for ever; the device loop returns HV_ERR_NOT_CONVERGED."""
    g = _fixture(golden)
    with _session(hv, g, hv.HV_F64, ppn=10) as s:
        ws = ((500.0, 4.0, 0.6), (500.0, 4.0, 0.6))
        with pytest.raises(hv.HVError) as e:
            s.initialize_particles(ws, (-8.0, -12.0), rng=hv.HV_RNG_PHILOX)
        assert e.value.status == hv._lib.HV_ERR_NOT_CONVERGED
