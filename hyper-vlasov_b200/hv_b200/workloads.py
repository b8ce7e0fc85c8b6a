"""Named synthetic workloads of the hyper-vlasov hot path.

Each workload is a nucleus, a test-particle count, a box-centred cubic grid and
a time step, with the Skyrme/Coulomb settings of the 40Ca definition below
(t0 = -2645 MeV fm^3, t3 = 15595 MeV fm^(3+3 sigma), sigma = 1/6, a_sym = 32 MeV,
SOR omega = 1.8 to relative residual 1e-6, dipole boost of 30 MeV/c, seed 0).
Positions are uniform in a ball of radius 1.2 A^(1/3) fm and wavenumbers
uniform in a ball of k_F = (3 pi^2 rho_q / 2)^(1/3) with rho_q = 0.08 fm^-3.

The smoothing width is the reference's default FWHM of 1.444 fm
(auto_compute.py:54), sigma_r = FWHM / (2 sqrt(2 ln 2)) (physics_formulas.hpp:59-63).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

from . import _lib as L

HBAR_C = 197.33
RHO0 = 0.16


def sigma_from_fwhm(fwhm: float) -> float:
    return fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0)))


@dataclass
class Workload:
    name: str
    Z: int
    N: int
    ppn: int
    n: int            # grid nodes per axis
    h: float          # grid spacing (fm); d_max = n h / 2
    dt: float         # fm/c
    steps: int
    seed: int = 0
    t0: float = -2645.0
    t3: float = 15595.0
    sigma: float = 1.0 / 6.0
    a_sym: float = 32.0
    boost_mev: float = 30.0
    t_exc: float = 0.0
    sigma_r: float = field(default_factory=lambda: sigma_from_fwhm(1.444))
    sor_omega: float = 1.8
    sor_tol: float = 1e-6
    sor_criterion: int = L.HV_SOR_REL_RESIDUAL
    sor_max_iter: int = 20000
    deposit_mode: int = L.HV_DEPOSIT_ATOMIC

    @property
    def A_nucleons(self) -> int:
        return self.Z + self.N

    @property
    def protons(self) -> int:
        return self.Z * self.ppn

    @property
    def neutrons(self) -> int:
        return self.N * self.ppn

    @property
    def particles(self) -> int:
        return self.protons + self.neutrons

    @property
    def radius(self) -> float:
        return 1.2 * self.A_nucleons ** (1.0 / 3.0)

    @property
    def k_fermi(self) -> float:
        return (3.0 * math.pi ** 2 * 0.08 / 2.0) ** (1.0 / 3.0)

    @property
    def d_max(self) -> float:
        return self.n * self.h / 2.0

    @property
    def G(self) -> int:
        return self.n ** 3

    @property
    def eta(self) -> float:
        """Dipole boost in fm^-1 (nuclear_excitation, include/physics.hpp:236-246)."""
        return self.boost_mev / HBAR_C

    def skyrme(self):
        """(A, B, C, gamma) of Skyrme<T> from (t0, t3, sigma, a_sym)."""
        A = 0.75 * self.t0 * RHO0
        B = (self.sigma + 2.0) / 16.0 * self.t3 * RHO0 ** (self.sigma + 1.0)
        return A, B, self.a_sym, self.sigma + 1.0

    def world(self) -> L.hv_world:
        w = L.hv_world()
        for a in range(3):
            w.n[a] = self.n
            w.d_max[a] = self.d_max
        return w

    def world_tuple(self):
        return ((self.n,) * 3, (self.d_max,) * 3)

    def run_params(self) -> L.hv_run_params:
        p = L.hv_run_params()
        p.z, p.n, p.part_per_nucleon = self.Z, self.N, self.ppn
        p.sigma_r, p.dt, p.t_exc, p.eta_exc = self.sigma_r, self.dt, self.t_exc, self.eta
        A, B, Cc, g = self.skyrme()
        p.skyrme = L.hv_skyrme(A, B, Cc, g)
        p.sor = L.hv_sor_params(self.sor_omega, self.sor_tol, self.sor_criterion, self.sor_max_iter)
        p.deposit_mode = self.deposit_mode
        return p

    def with_grid(self, n: int):
        return replace(self, n=n)

    def with_reference_sor(self):
        """The reference's hard-wired SOR: omega 1.5, max|dphi| < 1e-4, 512
        iterations (include/physics.hpp:103-104,152)."""
        return replace(self, sor_omega=1.5, sor_tol=1e-4, sor_criterion=L.HV_SOR_MAX_UPDATE, sor_max_iter=512)


# Starting values of the initialisation loop in the reference's driver
# (auto_compute.py:41-55): Woods-Saxon V0 = -50 MeV, a = 0.66 fm, R12 = 0.8 r_max
# (include/init.hpp:335-336), Fermi levels -8 / -12 MeV, momentum FWHM 0.346
# fm^-1, Skyrme A = -356.8, B = 303.9, C = 32 MeV, gamma = 7/6.
INIT_V0, INIT_A, INIT_EPS_P, INIT_EPS_N, INIT_K_FWHM = -50.0, 0.66, -8.0, -12.0, 0.346
INIT_SKYRME = (-356.8, 303.9, 32.0, 7.0 / 6.0)


def nuclear_radius(A: int) -> float:
    """r_max = 1.5 A^(1/3) fm (include/physics_formulas.hpp:27-32)."""
    return 1.5 * A ** (1.0 / 3.0)


def init_start(Z: int, N: int):
    """(ws, fermi) starting values: ((V0, R12, a) x 2), (eps_p, eps_n)."""
    r12 = 0.8 * nuclear_radius(Z + N)
    return ((INIT_V0, r12, INIT_A), (INIT_V0, r12, INIT_A)), (INIT_EPS_P, INIT_EPS_N)


# 40Ca, 100 test particles per nucleon, 32^3, h = 1 fm, dt = 0.5 fm/c, 200 steps
CA40_SMALL = Workload("40Ca-4k-32^3", Z=20, N=20, ppn=100, n=32, h=1.0, dt=0.5, steps=200)
# 208Pb, 500 per nucleon (104,000 particles), 64^3, h = 0.5 fm, dt = 0.25, 2000 steps
PB208_104K = Workload("208Pb-104k-64^3", Z=82, N=126, ppn=500, n=64, h=0.5, dt=0.25, steps=2000)
# 208Pb, 10,000 per nucleon (2.08M particles), 128^3, h = 0.25 fm, dt = 0.2, 1000 steps
PB208_2M = Workload("208Pb-2.08M-128^3", Z=82, N=126, ppn=10000, n=128, h=0.25, dt=0.2, steps=1000)

# the 128^3 grid of PB208_2M with 100 test particles per nucleon: the same field
# kernels with a small particle set, for profiling captures that must stay small
PB208_20K_128 = Workload("208Pb-20.8k-128^3", Z=82, N=126, ppn=100, n=128, h=0.25, dt=0.2, steps=1000)

WORKLOADS = {w.name: w for w in (CA40_SMALL, PB208_104K, PB208_2M, PB208_20K_128)}


# Nuclei of the batched workload: (name, Z, N).
BATCH_NUCLEI = (("16O", 8, 8), ("40Ca", 20, 20), ("90Zr", 40, 50), ("208Pb", 82, 126))


def batch_workloads(n: int = 64, seed: int = 0, steps: int = 500, h: float = 0.5, dt: float = 0.25):
    """n independent runs: nuclei drawn from 16O, 40Ca, 90Zr, 208Pb; 200-2000
    test particles per nucleon (log-uniform); cubic grids of 32-96 nodes per
    axis at h (the smallest of 32, 48, ... 96 that leaves 4 fm around the
    nucleus, or larger at random); t0 and t3 jittered +-5 % uniform; dipole
    boosts of 10-40 MeV/c; each run with its own generator seed."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    grids = (32, 48, 64, 80, 96)
    for i in range(n):
        name, Z, N = BATCH_NUCLEI[rng.integers(len(BATCH_NUCLEI))]
        ppn = int(round(math.exp(rng.uniform(math.log(200.0), math.log(2000.0)))))
        radius = 1.2 * (Z + N) ** (1.0 / 3.0)
        fits = [g for g in grids if g * h / 2.0 >= radius + 4.0]
        ng = int(fits[rng.integers(len(fits))])
        w = Workload(f"{name}-{ppn}x{Z + N}-{ng}^3#{i}", Z=Z, N=N, ppn=ppn, n=ng, h=h, dt=dt, steps=steps,
                     seed=seed * 1000 + i,
                     t0=-2645.0 * (1.0 + rng.uniform(-0.05, 0.05)),
                     t3=15595.0 * (1.0 + rng.uniform(-0.05, 0.05)),
                     boost_mev=float(rng.uniform(10.0, 40.0)))
        out.append(w)
    return out
