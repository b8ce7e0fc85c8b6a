"""FP64 tangent-linear run of the step.  TEST INFRASTRUCTURE ONLY.

Forward-mode derivative of cpu_simulate's step order
(src/hyper_vlasov.cpp:53-104, restated in hv_oracle_impl.h orc_simulate) in a
direction dtheta of the Skyrme parameters theta = (t0, t3, sigma, a_sym), for
checking the library's adjoint independently of finite differences.  The
linear stages run on the oracle's C routines (hv_oracle.c): smoothing
(physics.hpp:202-234), the Poisson solve on the tangent density with a zero
boundary (physics.hpp:99-157; phi = L^-1(-c rho_p) + boundary, so
dphi = L^-1(-c drho_p)), FDM (physics.hpp:159-200) and gather
(tools.hpp:98-168).  numpy supplies the derivatives of the CIC weights
(tools.hpp:35-168) and of the Skyrme map (physics_formulas.hpp:70-77).

    t = Tangent(world, run, protons, neutrons)
    D, dD = t.run(x, y, z, kx, ky, kz, steps, theta, dtheta)

returns D(t) per step and its derivative in the direction dtheta.
"""
from __future__ import annotations

import numpy as np

from hv_oracle import Oracle, RunSpec

RHO0 = 0.16
HBAR_C = 197.33
MC2 = 935.0


def skyrme_from_theta(theta):
    """(A, B, C, gamma) of (t0, t3, sigma, a_sym) (hv_skyrme_from_t0t3)."""
    t0, t3, s, a = theta
    return 0.75 * t0 * RHO0, (s + 2.0) / 16.0 * t3 * RHO0 ** (s + 1.0), a, s + 1.0


def skyrme_tangent(theta, dtheta):
    """Derivative of (A, B, C, gamma) in the direction dtheta."""
    t0, t3, s, a = theta
    d0, d3, ds, da = dtheta
    r = RHO0 ** (s + 1.0)
    dB = (s + 2.0) / 16.0 * r * d3 + t3 * r * (1.0 / 16.0 + (s + 2.0) / 16.0 * np.log(RHO0)) * ds
    return 0.75 * RHO0 * d0, dB, da, ds


class Tangent:
    def __init__(self, world, run: RunSpec, protons, neutrons):
        self.world, self.spec = world, run
        self.protons, self.neutrons = protons, neutrons
        self.o = Oracle(np.float64)
        self.n = np.array(world[0])
        self.dmax = np.array(world[1], dtype=np.float64)
        self.G = int(np.prod(self.n))

    # ---- CIC geometry (tools.hpp:50-60) and its derivatives
    def _cells(self, x, y, z):
        c = [(self.n[a] / 2.0) * (p / self.dmax[a] + 1.0) for a, p in enumerate((x, y, z))]
        inside = np.ones(len(x), bool)
        for a in range(3):
            inside &= (c[a] >= 0.0) & (c[a] < self.n[a])
        i0 = [np.where(inside, c[a], 0.0).astype(np.int64) for a in range(3)]
        d = [np.where(inside, c[a] - i0[a], 0.0) for a in range(3)]
        h = [self.n[a] / (2.0 * self.dmax[a]) for a in range(3)]  # dc / dpos
        off = np.where(np.arange(len(x)) < self.protons, 0, self.G)
        return inside, i0, d, h, off

    def _corners(self, x, y, z):
        """(linear index, weight, d weight / d(x, y, z)) of the 8 CIC corners;
        dropped corners (index == n) and outside particles get weight 0."""
        inside, i0, d, h, off = self._cells(x, y, z)
        ny, nz = self.n[1], self.n[2]
        out = []
        for a in (0, 1):
            for b in (0, 1):
                for cc in (0, 1):
                    ix, iy, iz = i0[0] + a, i0[1] + b, i0[2] + cc
                    ok = inside & (ix < self.n[0]) & (iy < self.n[1]) & (iz < self.n[2])
                    wx = d[0] if a else 1.0 - d[0]
                    wy = d[1] if b else 1.0 - d[1]
                    wz = d[2] if cc else 1.0 - d[2]
                    gx = h[0] if a else -h[0]
                    gy = h[1] if b else -h[1]
                    gz = h[2] if cc else -h[2]
                    idx = np.where(ok, off + (ix * ny + iy) * nz + iz, 0)
                    m = ok.astype(np.float64)
                    out.append((idx, m * wx * wy * wz, (m * gx * wy * wz, m * wx * gy * wz, m * wx * wy * gz)))
        return out

    def deposit_tangent(self, x, y, z, dx, dy, dz):
        drho = np.zeros(2 * self.G)
        for idx, _, (gx, gy, gz) in self._corners(x, y, z):
            np.add.at(drho, idx, gx * dx + gy * dy + gz * dz)
        return drho

    def gather_tangent(self, x, y, z, F, dx, dy, dz):
        out = [np.zeros(len(x)) for _ in range(3)]
        for idx, _, (gx, gy, gz) in self._corners(x, y, z):
            s = gx * dx + gy * dy + gz * dz
            for k in range(3):
                out[k] += s * F[k][idx]
        return out

    # ---- the force of positions x and its tangent
    def force(self, x, y, z, phi, sk):
        o, w, r = self.o, self.world, self.spec
        rho = o.smooth(w, r.sigma_r, r.part_per_nucleon, o.deposit(w, self.protons, self.neutrons, x, y, z))
        U = o.skyrme(w, *sk, rho)
        o.sor(w, phi, rho, r.sor_omega, r.sor_criterion, r.sor_tol, r.sor_max_iter)
        o.merge(w, U, phi)
        F = o.fdm(w, U)
        f = o.gather(w, self.protons, self.neutrons, x, y, z, *F)
        return f, F, rho

    def force_tangent(self, x, y, z, dx, dy, dz, F, rho, dphi, sk, dsk):
        o, w, r = self.o, self.world, self.spec
        G = self.G
        A, B, C, g = sk
        dA, dB, dC, dg = dsk
        drho = o.smooth(w, r.sigma_r, r.part_per_nucleon, self.deposit_tangent(x, y, z, dx, dy, dz))
        rp, rn = rho[:G], rho[G:]
        t = (rp + rn) / RHO0
        tg = t ** g
        tg1 = np.where(t > 0.0, t ** (g - 1.0), 0.0)
        lnt = np.where(t > 0.0, np.log(np.where(t > 0.0, t, 1.0)), 0.0)
        S = (A + B * g * tg1) / RHO0
        base = S * (drho[:G] + drho[G:]) + dA * t + dB * tg + dg * B * tg * lnt
        iso = 2.0 * C * (drho[G:] - drho[:G]) / RHO0 + dC * 2.0 * (rn - rp) / RHO0
        dU = np.concatenate([base - iso, base + iso])
        o.sor(w, dphi, drho, r.sor_omega, r.sor_criterion, r.sor_tol, r.sor_max_iter)
        dU[:G] += dphi
        dF = o.fdm(w, dU)
        df = o.gather(w, self.protons, self.neutrons, x, y, z, *dF)
        dg_ = self.gather_tangent(x, y, z, F, dx, dy, dz)
        return [df[k] + dg_[k] for k in range(3)]

    def run(self, x, y, z, kx, ky, kz, steps, theta, dtheta):
        x, y, z, kx, ky, kz = (np.array(a, dtype=np.float64, copy=True) for a in (x, y, z, kx, ky, kz))
        o, w, r = self.o, self.world, self.spec
        sk, dsk = skyrme_from_theta(theta), skyrme_tangent(theta, dtheta)
        N = len(x)
        dx, dy, dz, dkx, dky, dkz = (np.zeros(N) for _ in range(6))
        a, b = r.dt / (2.0 * HBAR_C), r.dt * HBAR_C / MC2
        nza = r.n * r.z / (r.n + r.z)
        phi = o.coulomb_boundary(w, r.z)
        dphi = np.zeros(self.G)
        f, F, rho = self.force(x, y, z, phi, sk)
        df = self.force_tangent(x, y, z, dx, dy, dz, F, rho, dphi, sk, dsk)
        D, dD = np.zeros(steps), np.zeros(steps)
        excited = False
        p = self.protons
        for n in range(steps):
            D[n] = nza * (z[:p].mean() - z[p:].mean())
            dD[n] = nza * (dz[:p].mean() - dz[p:].mean())
            if n * r.dt >= r.t_exc and not excited:  # hyper_vlasov.cpp:86-89 (theta-independent)
                excited = True
                o.excite(self.protons, self.neutrons, kz, r.z, r.n, r.eta_exc)
            for k, dk, ff, dff in ((kx, dkx, f[0], df[0]), (ky, dky, f[1], df[1]), (kz, dkz, f[2], df[2])):
                k += a * ff
                dk += a * dff
            for q, dq, k, dk in ((x, dx, kx, dkx), (y, dy, ky, dky), (z, dz, kz, dkz)):
                q += b * k
                dq += b * dk
            f, F, rho = self.force(x, y, z, phi, sk)
            df = self.force_tangent(x, y, z, dx, dy, dz, F, rho, dphi, sk, dsk)
            for k, dk, ff, dff in ((kx, dkx, f[0], df[0]), (ky, dky, f[1], df[1]), (kz, dkz, f[2], df[2])):
                k += a * ff
                dk += a * dff
        return D, dD
