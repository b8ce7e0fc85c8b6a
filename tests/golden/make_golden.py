"""Generates the golden vectors in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py

Runs the reference's own step routines -- compiled from the reference tree by
oracle/Makefile (target `ref`, -ffp-contract=off) into oracle/_ref/libhvref.so
-- on seeded synthetic inputs from hv_generate_nucleus, and stores every
stage's input and output.  The deposit runs on one OpenMP thread (its array
reduction is order-dependent, include/tools.hpp:45); the O(G^2) smoothing
(include/physics.hpp:202-234) is the reference's own routine, not the
offset-table restatement.

Fixtures:
  ca40_stages_{f64,f32}.npz  one pass of every stage on the 40Ca / 4000
                             particle / 32^3 h = 1 fm workload
  ca40_run_f64.npz           10 steps of the cpu_simulate loop on the same
                             workload: stats rows and final particles
  edge_f64.npz               non-cubic grid (12 x 10 x 14, unequal d_max) with
                             particles outside the grid, on node planes and
                             on the upper faces, through every stage
  init_ca40_f64.npz          the reference's initialize_particles
                             (include/physics.hpp:34-97) after srand(128) for
                             40Ca with 100 test particles per nucleon and the
                             driver's starting values (auto_compute.py), its
                             GSL fit replaced by the oracle's restatement
                             (`python tests/golden/make_golden.py init` writes
                             only this one)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "hyper-vlasov_b200"))

from hv_oracle import Reference, RunSpec  # noqa: E402

import hv_b200  # noqa: E402
from hv_b200.workloads import CA40_SMALL  # noqa: E402

SIGMA_R = CA40_SMALL.sigma_r
A, B, CC, GAMMA = CA40_SMALL.skyrme()


def stages(dtype, world, Z, N, ppn, P, Nn, x, y, z, kx, ky, kz, dt, eta):
    ref = Reference(dtype)
    out = {"x": x.copy(), "y": y.copy(), "z": z.copy(), "kx": kx.copy(), "ky": ky.copy(), "kz": kz.copy()}
    ref.set_threads(1)
    out["rho_raw"] = ref.deposit(world, P, Nn, x, y, z)
    ref.set_threads(os.cpu_count() or 1)
    out["rho"] = ref.smooth(world, SIGMA_R, ppn, out["rho_raw"])
    out["U"] = ref.skyrme(world, A, B, CC, GAMMA, out["rho"])
    phi = ref.coulomb_boundary(world, Z)
    out["phi_boundary"] = phi.copy()
    ref.sor(world, phi, out["rho"])
    out["phi"] = phi
    U = out["U"].copy()
    ref.merge(world, U, phi)
    out["U_merged"] = U
    out["Fx"], out["Fy"], out["Fz"] = ref.fdm(world, U)
    out["fx"], out["fy"], out["fz"] = ref.gather(world, P, Nn, x, y, z, out["Fx"], out["Fy"], out["Fz"])
    k = [kx.copy(), ky.copy(), kz.copy()]
    ref.kick_half(P, Nn, *k, out["fx"], out["fy"], out["fz"], dt)
    out["kx_kick"], out["ky_kick"], out["kz_kick"] = k
    xs = [x.copy(), y.copy(), z.copy()]
    ref.drift(P, Nn, *xs, *k, dt)
    out["x_drift"], out["y_drift"], out["z_drift"] = xs
    kze = kz.copy()
    ref.excite(P, Nn, kze, Z, N, eta)
    out["kz_excite"] = kze
    out["com"] = np.array([ref.center_of_mass(P, Nn, z, 0), ref.center_of_mass(P, Nn, z, 1)])
    out["msr"] = np.array([ref.mean_squared_radius(world, P, Nn, x, y, z, 0),
                           ref.mean_squared_radius(world, P, Nn, x, y, z, 1)])
    meta = {"n": np.array(world[0]), "d_max": np.array(world[1]), "Z": Z, "N": N, "ppn": ppn, "protons": P,
            "neutrons": Nn, "sigma_r": SIGMA_R, "skyrme": np.array([A, B, CC, GAMMA]), "dt": dt, "eta": eta}
    out.update({k_: np.asarray(v) for k_, v in meta.items()})
    return out


def init_fixture():
    from hv_b200.workloads import INIT_K_FWHM, INIT_SKYRME, init_start, sigma_from_fwhm

    Z, N, ppn, seed = 20, 20, 100, 128
    ws, fermi = init_start(Z, N)
    sigma_k, sigma_r = sigma_from_fwhm(INIT_K_FWHM), sigma_from_fwhm(1.444)
    ref = Reference(np.float64)
    ref.set_threads(os.cpu_count() or 1)
    out = ref.initialize_particles(Z, N, ppn, sigma_k, sigma_r, INIT_SKYRME, ws, fermi, seed)
    r_max, mtp = ref.init_sizes(Z, N, ppn)
    np.savez_compressed(os.path.join(HERE, "init_ca40_f64.npz"), Z=Z, N=N, ppn=ppn, seed=seed, sigma_k=sigma_k,
                        sigma_r=sigma_r, skyrme=np.array(INIT_SKYRME), ws0=np.array(ws), fermi0=np.array(fermi),
                        ws=np.array(out["ws"]), fermi=np.array(out["fermi"]), passes=out["passes"],
                        fit_iterations=np.array(out["fit_iterations"]), fit_status=np.array(out["fit_status"]),
                        r_max=r_max, max_test_part=mtp,
                        **{k: out[k] for k in ("x", "y", "z", "kx", "ky", "kz", "density_p", "density_n",
                                               "energy")})
    print("wrote init", out["passes"], out["ws"], out["fermi"])


def main():
    if sys.argv[1:] == ["init"]:
        init_fixture()
        return
    w = CA40_SMALL
    world = w.world_tuple()
    for dtype, tag in ((np.float64, "f64"), (np.float32, "f32")):
        x, y, z, kx, ky, kz = hv_b200.generate_nucleus(w.seed, w.protons, w.neutrons, w.radius, w.k_fermi, dtype)
        out = stages(dtype, world, w.Z, w.N, w.ppn, w.protons, w.neutrons, x, y, z, kx, ky, kz, w.dt, w.eta)
        np.savez_compressed(os.path.join(HERE, f"ca40_stages_{tag}.npz"), **out)
        print("wrote", tag)

    # 10 steps of cpu_simulate with the reference's routines (its SOR settings)
    x, y, z, kx, ky, kz = hv_b200.generate_nucleus(w.seed, w.protons, w.neutrons, w.radius, w.k_fermi, np.float64)
    init = {"x0": x.copy(), "y0": y.copy(), "z0": z.copy(), "kx0": kx.copy(), "ky0": ky.copy(), "kz0": kz.copy()}
    ref = Reference(np.float64)
    ref.set_threads(1)
    run = RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=SIGMA_R, dt=w.dt, t_exc=0.0, eta_exc=w.eta,
                  A=A, B=B, C=CC, gamma=GAMMA)
    rows, fields, secs = ref.simulate(world, run, w.protons, w.neutrons, x, y, z, kx, ky, kz, 10, smooth_mode=1,
                                      want_fields=True)
    np.savez_compressed(os.path.join(HERE, "ca40_run_f64.npz"), rows=rows, x=x, y=y, z=z, kx=kx, ky=ky, kz=kz,
                        steps=10, **init)
    print("wrote run", secs)

    # edge cases: non-cubic grid, particles outside / on planes / on upper faces
    n = (12, 10, 14)
    dm = (6.0, 5.0, 7.5)
    rng = np.random.default_rng(7)
    P, Nn = 300, 200
    tot = P + Nn
    x = rng.uniform(-1.25 * dm[0], 1.25 * dm[0], tot)
    y = rng.uniform(-1.25 * dm[1], 1.25 * dm[1], tot)
    z = rng.uniform(-1.25 * dm[2], 1.25 * dm[2], tot)
    # exact node planes, the last node plane, just below / on the upper face
    special = []
    for ax, (nn, d) in enumerate(zip(n, dm)):
        for v in (-d, d * (2.0 * (nn - 1) / nn - 1.0), d * (1 - 2.0 ** -40), d, 0.0, -d * (1 + 1e-15)):
            special.append((ax, v))
    for i, (ax, v) in enumerate(special):
        (x, y, z)[ax][i] = v
    kx, ky, kz = (rng.uniform(-1, 1, tot) for _ in range(3))
    out = stages(np.float64, (n, dm), 12, 8, 25, P, Nn, x, y, z, kx, ky, kz, 0.3, 0.1)
    np.savez_compressed(os.path.join(HERE, "edge_f64.npz"), **out)
    print("wrote edge")
    init_fixture()


if __name__ == "__main__":
    main()
