"""The Woods-Saxon initialisation loop, initialize_particles
(include/physics.hpp:34-97), and its parts.

CPU (the checker itself):
* the oracle's compute_energy restatement against the reference's
  compute_particle_energies (compiled from source): bit-identical;
* the oracle's Levenberg-Marquardt restatement of the GSL fit
  (minim_woods_saxon) lands on the least-squares minimum that an independent
  solver (scipy's MINPACK lmder) finds: with the reference's tolerances
  (1e-4) the cost is within 1e-6 and the parameters within 1e-3 of it, with
  tight ones the parameters agree to 1e-6;
* the golden fixture (tests/golden/init_ca40_f64.npz) is what the reference's
  loop produces now, and its particles are consistent: mirrored pairs, the
  densities and energies of the final state.

GPU: tests/test_gpu_init.py."""
from __future__ import annotations

import numpy as np
import pytest

from hv_oracle import Oracle, Reference, reference_available

scipy_opt = pytest.importorskip("scipy.optimize")


def _fixture(golden):
    return golden("init_ca40_f64.npz")


def _ws(g, key="ws"):
    w = g[key]
    return (tuple(w[0]), tuple(w[1]))


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_energies_match_reference(golden, dtype):
    g = _fixture(golden)
    P = int(g["Z"]) * int(g["ppn"])
    Nn = int(g["N"]) * int(g["ppn"])
    arrs = [g[k].astype(dtype) for k in ("x", "y", "z", "kx", "ky", "kz")]
    ws = _ws(g)
    e_ref = Reference(dtype).particle_energies(P, Nn, *arrs, ws, float(g["sigma_k"]), int(g["Z"]))
    e_orc = Oracle(dtype).particle_energies(P, Nn, *arrs, ws, float(g["sigma_k"]), int(g["Z"]))
    assert np.array_equal(e_ref, e_orc)
    if dtype == np.float64:
        # compute_particle_energies(part, ws, param) ends the reference's loop
        assert np.array_equal(e_ref, g["energy"])


def _residual_np(r, vs):
    def f(p):
        V0, R12, a = p
        return vs - V0 / (1.0 + np.exp((r - R12) / a))

    def jac(p):
        V0, R12, a = p
        e = np.exp((r - R12) / a)
        e2 = (1.0 + e) ** 2
        return np.stack([-1.0 / (1.0 + e), -(V0 * e) / (a * e2), -(V0 * (r - R12) * e) / (a * a * e2)], axis=1)

    return f, jac


@pytest.mark.parametrize("species", [0, 1])
def test_oracle_fit_reaches_the_least_squares_minimum(golden, species):
    g = _fixture(golden)
    P = int(g["Z"]) * int(g["ppn"])
    sl = slice(0, P) if species == 0 else slice(P, None)
    x, y, z, dp, dn = (np.ascontiguousarray(g[k][sl]) for k in ("x", "y", "z", "density_p", "density_n"))
    A, B, C, gam = (float(v) for v in g["skyrme"])
    start = tuple(g["ws0"][species])
    (V0, R12, a), iters, status = Oracle(np.float64).fit_woods_saxon(x, y, z, dp, dn, species, g["skyrme"], start)
    assert status in (1, 2) and 1 <= iters <= 100
    # skyrme_potential (physics_formulas.hpp:70-77) and |r| in numpy
    r = np.sqrt(x * x + y * y + z * z)
    t = (dp + dn) / 0.16
    tau = -1.0 if species == 0 else 1.0
    vs = A * t + B * t ** gam + 2.0 * tau * C * ((dn - dp) / 0.16)
    f, jac = _residual_np(r, vs)
    best = scipy_opt.least_squares(f, np.array(start), jac=jac, method="lm", xtol=1e-14, ftol=1e-14, gtol=1e-14)
    cost_orc = 0.5 * np.sum(f(np.array([V0, R12, a])) ** 2)
    # stopped by the reference's tolerances (xtol = gtol = 1e-4)
    assert best.cost * (1 - 1e-12) <= cost_orc <= best.cost * (1 + 1e-6)
    assert np.allclose([V0, R12, a], best.x, rtol=1e-3)
    # with tight tests the same iteration converges onto scipy's minimum
    (V0t, R12t, at), _, st = Oracle(np.float64).fit_woods_saxon(x, y, z, dp, dn, species, g["skyrme"], start,
                                                               max_iter=1000, xtol=1e-13, gtol=1e-13)
    assert st in (1, 2)
    assert np.allclose([V0t, R12t, at], best.x, rtol=1e-6)
    cost_t = 0.5 * np.sum(f(np.array([V0t, R12t, at])) ** 2)
    assert abs(cost_t - best.cost) <= 1e-10 * best.cost


def test_oracle_fit_rejects_too_few_particles():
    x = np.array([1.0, 2.0])
    ws, iters, status = Oracle(np.float64).fit_woods_saxon(x, x, x, x, x, 0, (-356.8, 303.9, 32.0, 7 / 6),
                                                           (-50.0, 3.0, 0.6))
    assert status == -2 and iters == 0 and ws == (-50.0, 3.0, 0.6)


def test_golden_init_is_consistent(golden):
    g = _fixture(golden)
    P = int(g["Z"]) * int(g["ppn"])
    total = P + int(g["N"]) * int(g["ppn"])
    # generate_checking_particles stores (r, k) and (-r, -k) pairs (tools.hpp:271-277)
    for k in ("x", "y", "z", "kx", "ky", "kz"):
        a = g[k]
        assert a.shape == (total,)
        assert np.array_equal(a[1::2], -a[0::2])
    # inside the sampling cube
    assert np.all(np.abs(g["x"]) <= g["r_max"]) and np.all(np.abs(g["kx"]) <= 1.5)
    # every particle's energy is below its species' final... level of its pass
    assert np.all(np.isfinite(g["energy"]))
    o = Oracle(np.float64)
    dp, dn = o.particle_densities(P, total - P, g["x"], g["y"], g["z"], float(g["sigma_r"]), int(g["ppn"]))
    assert np.array_equal(dp, g["density_p"]) and np.array_equal(dn, g["density_n"])


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
def test_golden_init_matches_the_reference_now(golden):
    """The fixture is reproducible: srand(128) and the reference's loop give
    it again bit for bit."""
    g = _fixture(golden)
    out = Reference(np.float64).initialize_particles(int(g["Z"]), int(g["N"]), int(g["ppn"]), float(g["sigma_k"]),
                                                     float(g["sigma_r"]), g["skyrme"], _ws(g, "ws0"),
                                                     tuple(g["fermi0"]), int(g["seed"]))
    for k in ("x", "y", "z", "kx", "ky", "kz", "density_p", "density_n", "energy"):
        assert np.array_equal(out[k], g[k]), k
    assert np.array_equal(np.array(out["ws"]), g["ws"])
    assert np.array_equal(np.array(out["fermi"]), g["fermi"])
    assert out["passes"] == int(g["passes"])
