"""CPU: a NumPy model of the fused float solver's coarse-corrected cycle, the
evidence for its default relaxation (hv_fast_options.sor_coarse_sweeps 12 at
sor_coarse_omega 1.7).

The model takes the cycle's steps in double: the FP64 residual of phi, the
restriction of that residual to every F-th node by the triangle (F - |d|) /
F^2 per axis, the exact solve of the coarse correction equation by a sine
transform (spacing F h, zero boundary), trilinear prolongation back (the
fine grid's n nodes taken as n intervals, node n holding zero), m red-black
SOR sweeps at omega on the correction, and phi += correction; the solve
stops when ||b + lap_h phi|| / ||b|| <= 1e-6.  The densities are those of
successive steps of 208Pb, 104,000 test particles, 64^3 grid, h = 0.5 fm,
computed by the oracle's float stages (deposit, smoothing) with phi solved
in double, as the fused path does; each solve starts from the quadratic
extrapolation 3 phi_n - 3 phi_(n-1) + phi_(n-2) of the previous exact
solutions.  12 sweeps at 1.7 end every solve in two cycles (24 iterations)
where 16 sweeps at the run's omega 1.8 take three (48), and the quadratic
start sits near 7e-4 of the source.
"""
from __future__ import annotations

import numpy as np
import pytest
from scipy.fft import dstn, idstn

from hv_oracle import Oracle

KE = 4.0 * np.pi * 1.44


def _densities(w, steps):
    """Smoothed proton densities (double) of the initial state and of
    `steps` steps, from the oracle's float stages with phi in double."""
    o32, o64 = Oracle(np.float32), Oracle(np.float64)
    o32.set_threads(4)
    o64.set_threads(4)
    world = w.world_tuple()
    A, B, C, g = w.skyrme()
    import hv_b200 as hv
    x, y, z, kx, ky, kz = [a.copy() for a in hv.workload_particles(w, np.float32)]
    P, N = w.protons, w.neutrons
    phi = o64.coulomb_boundary(world, w.Z)
    out = []

    def fields():
        rho = o32.smooth(world, w.sigma_r, w.ppn, o32.deposit(world, P, N, x, y, z))
        U = o32.skyrme(world, A, B, C, g, rho)
        r64 = np.ascontiguousarray(rho.astype(np.float64))
        o64.sor(world, phi, r64, w.sor_omega, w.sor_criterion, w.sor_tol, 100000)
        out.append(r64[: w.G].copy())
        U = o32.merge(world, U, phi.astype(np.float32))
        return o32.gather(world, P, N, x, y, z, *o32.fdm(world, U))

    f = fields()
    dt = np.float32(w.dt)
    for s in range(steps):
        if s == 0:
            o32.excite(P, N, kz, w.Z, w.N, np.float32(w.eta))
        o32.kick_half(kx, ky, kz, *f, dt)
        o32.drift(x, y, z, kx, ky, kz, dt)
        f = fields()
        o32.kick_half(kx, ky, kz, *f, dt)
    return out, o64.coulomb_boundary(world, w.Z)


class CycleModel:
    def __init__(self, n, h, phib):
        self.n, self.h = n, h
        self.phib = phib.reshape(n, n, n)
        self.I = (slice(1, n - 1),) * 3
        self.inside = np.zeros((n, n, n), bool)
        self.inside[self.I] = True
        par = np.indices((n, n, n)).sum(axis=0) & 1
        self.colours = (self.inside & (par == 0), self.inside & (par == 1))

    def nsum(self, p):
        s = np.zeros_like(p)
        a = slice(1, -1)
        s[a, a, a] = p[2:, a, a] + p[:-2, a, a] + p[a, 2:, a] + p[a, :-2, a] + p[a, a, 2:] + p[a, a, :-2]
        return s

    def lap(self, p):
        out = (self.nsum(p) - 6.0 * p) / self.h ** 2
        out[~self.inside] = 0.0
        return out

    def rel(self, p, b):
        r = (b + self.lap(p))[self.I]
        return float(np.sqrt(np.sum(r * r) / np.sum(b[self.I] ** 2)))

    @staticmethod
    def _lam(m, H):
        return (2.0 * np.cos(np.pi * np.arange(1, m + 1) / (m + 1)) - 2.0) / H ** 2

    def _poisson(self, r, H):
        lx, ly, lz = (self._lam(m, H) for m in r.shape)
        L = lx[:, None, None] + ly[None, :, None] + lz[None, None, :]
        return idstn(dstn(-r, type=1) / L, type=1)

    def exact(self, b):
        p = self.phib.copy()
        p[self.I] += self._poisson((b + self.lap(self.phib))[self.I], self.h)
        return p

    def restrict(self, r, F):
        n, m = self.n, self.n // F - 1
        idx = F * np.arange(1, m + 1)
        out = r
        for ax in range(3):
            acc = 0.0
            shape = [1, 1, 1]
            shape[ax] = m
            for d in range(-(F - 1), F):
                j = idx + d
                valid = ((j >= 1) & (j <= n - 2)).reshape(shape)
                acc = acc + (F - abs(d)) / F ** 2 * np.take(out, np.clip(j, 0, n - 1), axis=ax) * valid
            out = acc
        return out

    def prolong(self, e, F):
        n, m = self.n, e.shape[0]
        out = np.zeros((m + 2,) * 3)
        out[1:-1, 1:-1, 1:-1] = e
        x = np.arange(n) / F
        i0 = np.minimum(np.floor(x).astype(int), m)
        t = x - i0
        for ax in range(3):
            shape = [1, 1, 1]
            shape[ax] = n
            tt = t.reshape(shape)
            out = np.take(out, i0, axis=ax) * (1.0 - tt) + np.take(out, i0 + 1, axis=ax) * tt
        out[~self.inside] = 0.0
        return out

    def solve(self, p0, b, F, sweeps, omega, tol=1e-6, max_cycles=12):
        p, cycles = p0.copy(), 0
        while self.rel(p, b) > tol and cycles < max_cycles:
            r = b + self.lap(p)
            d = self.prolong(self._poisson(self.restrict(r, F), F * self.h), F)
            for _ in range(sweeps):
                for colour in self.colours:
                    new = (1.0 - omega) * d + omega * (self.nsum(d) + self.h ** 2 * r) / 6.0
                    d[colour] = new[colour]
            p += d
            cycles += 1
        return cycles, self.rel(p, b)


@pytest.fixture(scope="module")
def solves():
    import hv_b200 as hv
    w = hv.PB208_104K
    rhos, phib = _densities(w, 4)
    model = CycleModel(w.n, 2.0 * w.d_max / w.n, phib)
    bs = [KE * r.reshape((w.n,) * 3) for r in rhos]
    ex = [model.exact(b) for b in bs]
    cases = [(3 * ex[k - 1] - 3 * ex[k - 2] + ex[k - 3], bs[k]) for k in range(3, len(bs))]
    return model, cases


def test_model_exact_solutions_meet_the_rule(solves):
    model, cases = solves
    for p0, b in cases:
        assert model.rel(model.exact(b), b) < 1e-10
        assert 1e-4 < model.rel(p0, b) < 1e-2  # the quadratic start


def test_default_relaxation_ends_solves_in_two_cycles(solves):
    model, cases = solves
    for p0, b in cases:
        cyc_new, rel_new = model.solve(p0, b, F=4, sweeps=12, omega=1.7)
        cyc_old, rel_old = model.solve(p0, b, F=4, sweeps=16, omega=1.8)
        assert cyc_new == 2 and rel_new < 0.5e-6, (cyc_new, rel_new)
        assert cyc_old == 3 and rel_old < 1e-6, (cyc_old, rel_old)
        assert 12 * cyc_new < 16 * cyc_old
