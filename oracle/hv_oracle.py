"""numpy bindings of the checker libraries.  TEST INFRASTRUCTURE ONLY.

Two CPU implementations of the hyper-vlasov step, used to check the CUDA
library and as the timed CPU baseline; the product never imports this module.

* ``Oracle``    -- oracle/libhv_oracle.so, the C restatement (hv_oracle.c).
* ``Reference`` -- oracle/_ref/libhvref*.so, the reference's own routines
  compiled from its include/ directory (ref_harness.cpp, ref_simulate.cpp).
  Built only where the reference tree exists; the built files travel with the
  repository snapshot.

All arrays are numpy, C-contiguous, of the instance's dtype.  Worlds are
``(n, d_max)`` with ``n`` = 3 ints and ``d_max`` = 3 floats.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_P = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class orc_world(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("d_max", C.c_double * 3)]


class orc_skyrme(C.Structure):
    _fields_ = [("A", C.c_double), ("B", C.c_double), ("C", C.c_double), ("gamma", C.c_double)]


class orc_run(C.Structure):
    _fields_ = [
        ("z", C.c_int), ("n", C.c_int), ("part_per_nucleon", C.c_int),
        ("sigma_r", C.c_double), ("dt", C.c_double), ("t_exc", C.c_double), ("eta_exc", C.c_double),
        ("skyrme", orc_skyrme),
        ("sor_omega", C.c_double), ("sor_tol", C.c_double),
        ("sor_criterion", C.c_int), ("sor_max_iter", C.c_int),
    ]


class orc_obs(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("rms_p", C.c_double), ("rms_n", C.c_double),
        ("zcm_p", C.c_double), ("zcm_n", C.c_double), ("dipole", C.c_double),
        ("sor_iterations", C.c_int), ("flags", C.c_int),
    ]


OBS_DTYPE = np.dtype([
    ("t", "f8"), ("rms_p", "f8"), ("rms_n", "f8"), ("zcm_p", "f8"), ("zcm_n", "f8"),
    ("dipole", "f8"), ("sor_iterations", "i4"), ("flags", "i4"),
])
assert OBS_DTYPE.itemsize == C.sizeof(orc_obs)


def make_world(n, d_max):
    w = orc_world()
    for a in range(3):
        w.n[a] = int(n[a])
        w.d_max[a] = float(d_max[a])
    return w


@dataclass
class RunSpec:
    """Parameters of one run (the fields of Parameters<T> the step uses)."""
    z: int
    n: int
    part_per_nucleon: int
    sigma_r: float
    dt: float
    t_exc: float
    eta_exc: float
    A: float
    B: float
    C: float
    gamma: float
    sor_omega: float = 1.5
    sor_tol: float = 1e-4
    sor_criterion: int = 0
    sor_max_iter: int = 512

    def to_c(self):
        r = orc_run()
        r.z, r.n, r.part_per_nucleon = self.z, self.n, self.part_per_nucleon
        r.sigma_r, r.dt, r.t_exc, r.eta_exc = self.sigma_r, self.dt, self.t_exc, self.eta_exc
        r.skyrme = orc_skyrme(self.A, self.B, self.C, self.gamma)
        r.sor_omega, r.sor_tol = self.sor_omega, self.sor_tol
        r.sor_criterion, r.sor_max_iter = self.sor_criterion, self.sor_max_iter
        return r


class Oracle:
    """The C restatement, double (``np.float64``) or float (``np.float32``)."""

    def __init__(self, dtype=np.float64, path=None):
        self.dtype = np.dtype(dtype)
        self.sfx = "d" if self.dtype == np.float64 else "f"
        self.lib = C.CDLL(path or os.path.join(HERE, "libhv_oracle.so"))

    def _f(self, name):
        return getattr(self.lib, f"{name}_{self.sfx}")

    def set_threads(self, n):
        self.lib.orc_set_threads(int(n))

    def _chk(self, *arrs):
        for a in arrs:
            if a is not None:
                assert a.dtype == self.dtype and a.flags.c_contiguous, (a.dtype, self.dtype)

    def deposit(self, world, protons, neutrons, x, y, z):
        G = int(np.prod(world[0]))
        rho = np.zeros(2 * G, self.dtype)
        self._chk(x, y, z)
        self._f("orc_deposit_cic")(C.byref(make_world(*world)), protons, neutrons, _ptr(x), _ptr(y), _ptr(z), _ptr(rho))
        return rho

    def table_size(self, world, sigma_r):
        f = self._f("orc_smooth_table_size")
        f.argtypes = [C.c_void_p, C.c_double]
        return f(C.byref(make_world(*world)), sigma_r)

    def smooth(self, world, sigma_r, ppn, rho_raw):
        rho = np.array(rho_raw, dtype=self.dtype, copy=True)
        tmp = np.empty_like(rho)
        f = self._f("orc_smooth")
        f.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        f(C.byref(make_world(*world)), sigma_r, ppn, _ptr(rho), _ptr(tmp))
        return rho

    def skyrme(self, world, A, B, Cc, gamma, rho):
        self._chk(rho)
        U = np.empty_like(rho)
        s = orc_skyrme(A, B, Cc, gamma)
        self._f("orc_skyrme")(C.byref(make_world(*world)), C.byref(s), _ptr(rho), _ptr(U))
        return U

    def coulomb_boundary(self, world, z, phi=None):
        G = int(np.prod(world[0]))
        phi = np.zeros(G, self.dtype) if phi is None else phi
        self._f("orc_coulomb_boundary")(C.byref(make_world(*world)), z, _ptr(phi))
        return phi

    def sor(self, world, phi, rho, omega=1.5, criterion=0, tol=1e-4, max_iter=512):
        """In-place SOR; returns (iterations, final metric)."""
        self._chk(phi, rho)
        f = self._f("orc_sor")
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_int, C.c_void_p]
        m = C.c_double(0.0)
        it = f(C.byref(make_world(*world)), _ptr(phi), _ptr(rho), omega, criterion, tol, max_iter, C.byref(m))
        return it, m.value

    def rel_residual(self, world, phi, rho):
        f = self._f("orc_rel_residual")
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        f.restype = C.c_double
        return f(C.byref(make_world(*world)), _ptr(phi), _ptr(rho))

    def merge(self, world, U, phi):
        self._f("orc_merge")(C.byref(make_world(*world)), _ptr(U), _ptr(phi))
        return U

    def fdm(self, world, U):
        Fx, Fy, Fz = (np.empty_like(U) for _ in range(3))
        self._f("orc_fdm")(C.byref(make_world(*world)), _ptr(U), _ptr(Fx), _ptr(Fy), _ptr(Fz))
        return Fx, Fy, Fz

    def gather(self, world, protons, neutrons, x, y, z, Fx, Fy, Fz):
        fx, fy, fz = (np.empty_like(x) for _ in range(3))
        self._f("orc_gather_cic")(C.byref(make_world(*world)), protons, neutrons, _ptr(x), _ptr(y), _ptr(z),
                                  _ptr(Fx), _ptr(Fy), _ptr(Fz), _ptr(fx), _ptr(fy), _ptr(fz))
        return fx, fy, fz

    def kick_half(self, kx, ky, kz, fx, fy, fz, dt):
        f = self._f("orc_kick_half")
        ct = C.c_double if self.sfx == "d" else C.c_float
        f.argtypes = [C.c_int] + [C.c_void_p] * 6 + [ct]
        f(len(kx), _ptr(kx), _ptr(ky), _ptr(kz), _ptr(fx), _ptr(fy), _ptr(fz), dt)

    def drift(self, x, y, z, kx, ky, kz, dt):
        f = self._f("orc_drift")
        ct = C.c_double if self.sfx == "d" else C.c_float
        f.argtypes = [C.c_int] + [C.c_void_p] * 6 + [ct]
        f(len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(kx), _ptr(ky), _ptr(kz), dt)

    def excite(self, protons, neutrons, kz, Z, N, eta):
        f = self._f("orc_excite")
        ct = C.c_double if self.sfx == "d" else C.c_float
        f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, ct]
        f(protons, neutrons, _ptr(kz), Z, N, eta)

    def particle_densities(self, protons, neutrons, x, y, z, sigma_r, ppn):
        """(density_p, density_n) per particle (compute_particle_densities)."""
        self._chk(x, y, z)
        dp, dn = np.empty_like(x), np.empty_like(x)
        f = self._f("orc_particle_densities")
        f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 3 + [C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        f(protons, neutrons, _ptr(x), _ptr(y), _ptr(z), sigma_r, ppn, _ptr(dp), _ptr(dn))
        return dp, dn

    def particle_energies(self, protons, neutrons, x, y, z, kx, ky, kz, ws, sigma_k, zc):
        """compute_energy per particle; ws = ((V0, R12, a) protons, neutrons)."""
        self._chk(x, y, z, kx, ky, kz)
        e = np.empty_like(x)
        w = (C.c_double * 6)(*[float(v) for t in ws for v in t])
        f = self._f("orc_particle_energies")
        f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 7 + [C.c_double, C.c_int, C.c_void_p]
        f(protons, neutrons, _ptr(x), _ptr(y), _ptr(z), _ptr(kx), _ptr(ky), _ptr(kz), w, sigma_k, zc, _ptr(e))
        return e

    def fit_woods_saxon(self, x, y, z, dp, dn, species, skyrme, ws, max_iter=100, xtol=1e-4, gtol=1e-4):
        """The Levenberg-Marquardt restatement of minim_woods_saxon for one
        species' particles; returns ((V0, R12, a), iterations, status)."""
        self._chk(x, y, z, dp, dn)
        w = (C.c_double * 3)(*[float(v) for v in ws])
        it = C.c_int(0)
        sk = orc_skyrme(*[float(v) for v in skyrme])
        f = self._f("orc_fit_woods_saxon")
        f.argtypes = [C.c_int] + [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                                     C.c_double, C.c_void_p]
        f.restype = C.c_int
        st = f(len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(dp), _ptr(dn), species, C.byref(sk), w, max_iter, xtol, gtol,
               C.byref(it))
        return (w[0], w[1], w[2]), it.value, st

    def observe(self, world, protons, neutrons, x, y, z):
        o = orc_obs()
        self._f("orc_observe")(C.byref(make_world(*world)), protons, neutrons, _ptr(x), _ptr(y), _ptr(z), C.byref(o))
        return o

    def simulate(self, world, run: RunSpec, protons, neutrons, x, y, z, kx, ky, kz, steps, want_fields=False,
                 step_times=False):
        """cpu_simulate order; particle arrays are advanced in place.
        Returns (observables structured array, fields or None), plus the
        seconds of the initial solve and of each step when step_times."""
        self._chk(x, y, z, kx, ky, kz)
        obs = np.zeros(steps, OBS_DTYPE)
        G = int(np.prod(world[0]))
        fields = np.zeros(11 * G, self.dtype) if want_fields else None
        times = np.zeros(steps + 1, np.float64)
        self._f("orc_simulate")(C.byref(make_world(*world)), C.byref(run.to_c()), protons, neutrons,
                                _ptr(x), _ptr(y), _ptr(z), _ptr(kx), _ptr(ky), _ptr(kz), steps,
                                obs.ctypes.data_as(C.c_void_p), _ptr(fields), _ptr(times))
        return (obs, fields, times) if step_times else (obs, fields)


def split_fields(fields, G):
    """rho(2G) U(2G) phi(G) Fx(2G) Fy(2G) Fz(2G) -> dict."""
    return {
        "rho": fields[0:2 * G], "U": fields[2 * G:4 * G], "phi": fields[4 * G:5 * G],
        "Fx": fields[5 * G:7 * G], "Fy": fields[7 * G:9 * G], "Fz": fields[9 * G:11 * G],
    }


def reference_available(variant=""):
    return os.path.exists(os.path.join(REF_DIR, f"libhvref{variant}.so"))


def _generate(lib, seed, protons, neutrons, radius, k_fermi, dtype):
    """Six arrays x..kz of the seeded synthetic nucleus from the checker
    library `lib` (orc_generate_nucleus_*, hv_oracle.c)."""
    dt = np.dtype(dtype)
    total = int(protons) + int(neutrons)
    arrs = [np.zeros(total, dt) for _ in range(6)]
    f = lib.orc_generate_nucleus_d if dt == np.float64 else lib.orc_generate_nucleus_f
    f.restype = C.c_int
    f.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_double, C.c_double] + [_P] * 6
    if f(int(seed), int(protons), int(neutrons), float(radius), float(k_fermi), *[_ptr(a) for a in arrs]) != 0:
        raise ValueError("orc_generate_nucleus: bad argument")
    return arrs


def workload_inputs(lib, w, dtype):
    """The inputs of workload w (any object with seed, protons, neutrons,
    radius and k_fermi) from the checker library `lib`."""
    return _generate(lib, w.seed, w.protons, w.neutrons, w.radius, w.k_fermi, dtype)


class Reference:
    """The reference's own routines.  variant: "" (-ffp-contract=off),
    "_native" (the reference Makefile's -O3 -march=native), "_portable"
    (same flags, -march=x86-64-v3)."""

    def __init__(self, dtype=np.float64, variant=""):
        self.dtype = np.dtype(dtype)
        self.sfx = "d" if self.dtype == np.float64 else "f"
        self.lib = C.CDLL(os.path.join(REF_DIR, f"libhvref{variant}.so"))
        self.ct = C.c_double if self.sfx == "d" else C.c_float

    def _f(self, name):
        return getattr(self.lib, f"ref_{name}_{self.sfx}")

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def get_threads(self):
        return self.lib.ref_get_threads()

    @staticmethod
    def _w(world):
        n = (C.c_int * 3)(*[int(v) for v in world[0]])
        d = (C.c_double * 3)(*[float(v) for v in world[1]])
        return n, d

    def particle_densities(self, protons, neutrons, x, y, z, sigma_r, ppn):
        """The reference's compute_particle_densities (include/tools.hpp:170-203)."""
        x, y, z = (np.array(v, dtype=self.dtype, copy=True) for v in (x, y, z))
        dp, dn = np.empty_like(x), np.empty_like(x)
        f = self._f("particle_densities")
        f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 3 + [C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        f(protons, neutrons, _ptr(x), _ptr(y), _ptr(z), sigma_r, ppn, _ptr(dp), _ptr(dn))
        return dp, dn

    def particle_energies(self, protons, neutrons, x, y, z, kx, ky, kz, ws, sigma_k, zc):
        """The reference's compute_particle_energies (include/tools.hpp:226-232)."""
        arrs = [np.array(v, dtype=self.dtype, copy=True) for v in (x, y, z, kx, ky, kz)]
        e = np.empty_like(arrs[0])
        w = (C.c_double * 6)(*[float(v) for t in ws for v in t])
        f = self._f("particle_energies")
        f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.c_void_p, C.c_double, C.c_int, C.c_void_p]
        f(protons, neutrons, *[_ptr(a) for a in arrs], w, sigma_k, zc, _ptr(e))
        return e

    def init_sizes(self, z, n, ppn):
        """(r_max, max_test_part) as set_parameters derives them."""
        r, m = C.c_double(), C.c_int()
        self.lib.ref_init_sizes(z, n, ppn, C.byref(r), C.byref(m))
        return r.value, m.value

    def initialize_particles(self, z, n, ppn, sigma_k, sigma_r, skyrme, ws, fermi, seed):
        """srand(seed) and the reference's initialize_particles
        (include/physics.hpp:34-97), its GSL fit replaced by the oracle's
        restatement.  Returns dict: x..kz, density_p/n, energy, ws, fermi,
        passes, fit_iterations, fit_status."""
        total = (z + n) * ppn
        arrs = [np.zeros(total, self.dtype) for _ in range(9)]
        sk = (C.c_double * 4)(*[float(v) for v in skyrme])
        w = (C.c_double * 6)(*[float(v) for t in ws for v in t])
        fe = (C.c_double * 2)(float(fermi[0]), float(fermi[1]))
        info = (C.c_int * 5)()
        f = self._f("initialize_particles")
        f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_uint] + [C.c_void_p] * 10
        f(z, n, ppn, sigma_k, sigma_r, sk, w, fe, seed, *[_ptr(a) for a in arrs], info)
        names = ("x", "y", "z", "kx", "ky", "kz", "density_p", "density_n", "energy")
        out = dict(zip(names, arrs))
        out.update(ws=((w[0], w[1], w[2]), (w[3], w[4], w[5])), fermi=(fe[0], fe[1]), passes=info[0],
                   fit_iterations=(info[1], info[2]), fit_status=(info[3], info[4]))
        return out

    def deposit(self, world, protons, neutrons, x, y, z):
        G = int(np.prod(world[0]))
        rho = np.zeros(2 * G, self.dtype)
        n, d = self._w(world)
        self._f("deposit")(n, d, protons, neutrons, _ptr(x), _ptr(y), _ptr(z), _ptr(rho))
        return rho

    def smooth(self, world, sigma_r, ppn, rho_raw):
        rho = np.array(rho_raw, dtype=self.dtype, copy=True)
        tmp = np.empty_like(rho)
        n, d = self._w(world)
        f = self._f("smooth")
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        f(n, d, sigma_r, ppn, _ptr(rho), _ptr(tmp))
        return rho

    def skyrme(self, world, A, B, Cc, gamma, rho):
        U = np.empty_like(rho)
        n, d = self._w(world)
        f = self._f("skyrme")
        f.argtypes = [C.c_void_p, C.c_void_p] + [C.c_double] * 4 + [C.c_void_p, C.c_void_p]
        f(n, d, A, B, Cc, gamma, _ptr(rho), _ptr(U))
        return U

    def coulomb_boundary(self, world, z, phi=None):
        G = int(np.prod(world[0]))
        phi = np.zeros(G, self.dtype) if phi is None else phi
        n, d = self._w(world)
        self._f("boundary")(n, d, z, _ptr(phi))
        return phi

    def sor(self, world, phi, rho):
        n, d = self._w(world)
        self._f("sor")(n, d, _ptr(phi), _ptr(rho))

    def merge(self, world, U, phi):
        n, d = self._w(world)
        self._f("merge")(n, d, _ptr(U), _ptr(phi))
        return U

    def fdm(self, world, U):
        Fx, Fy, Fz = (np.empty_like(U) for _ in range(3))
        n, d = self._w(world)
        self._f("fdm")(n, d, _ptr(U), _ptr(Fx), _ptr(Fy), _ptr(Fz))
        return Fx, Fy, Fz

    def gather(self, world, protons, neutrons, x, y, z, Fx, Fy, Fz):
        fx, fy, fz = (np.empty_like(x) for _ in range(3))
        n, d = self._w(world)
        self._f("gather")(n, d, protons, neutrons, _ptr(x), _ptr(y), _ptr(z), _ptr(Fx), _ptr(Fy), _ptr(Fz),
                          _ptr(fx), _ptr(fy), _ptr(fz))
        return fx, fy, fz

    def kick_half(self, protons, neutrons, kx, ky, kz, fx, fy, fz, dt):
        f = self._f("kick_half")
        f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.c_double]
        f(protons, neutrons, _ptr(kx), _ptr(ky), _ptr(kz), _ptr(fx), _ptr(fy), _ptr(fz), dt)

    def drift(self, protons, neutrons, x, y, z, kx, ky, kz, dt):
        f = self._f("drift")
        f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.c_double]
        f(protons, neutrons, _ptr(x), _ptr(y), _ptr(z), _ptr(kx), _ptr(ky), _ptr(kz), dt)

    def excite(self, protons, neutrons, kz, Z, N, eta):
        f = self._f("excite")
        f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double]
        f(protons, neutrons, _ptr(kz), Z, N, eta)

    def center_of_mass(self, protons, neutrons, z, species):
        f = self._f("center_of_mass")
        f.restype = C.c_double
        return f(protons, neutrons, _ptr(z), species)

    def mean_squared_radius(self, world, protons, neutrons, x, y, z, species):
        f = self._f("mean_squared_radius")
        f.restype = C.c_double
        n, d = self._w(world)
        return f(n, d, protons, neutrons, _ptr(x), _ptr(y), _ptr(z), species)

    def write_vtk(self, path, world, Fx, Fy, Fz, rho, U):
        """The reference's VTK frame writer (include/init.hpp:159-254)."""
        n, d = self._w(world)
        f = self._f("write_vtk")
        f.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p] + [C.c_void_p] * 5
        return f(str(path).encode(), n, d, _ptr(Fx), _ptr(Fy), _ptr(Fz), _ptr(rho), _ptr(U))

    def simulate(self, world, run: RunSpec, protons, neutrons, x, y, z, kx, ky, kz, steps,
                 smooth_mode=1, want_fields=False, step_times=False):
        """The cpu_simulate loop with the reference's routines (its SOR is
        hard-wired to omega 1.5, |dphi| < 1e-4, 512).  smooth_mode 0 = the
        reference's O(G^2) smoothing, 1 = offset-table restatement.
        Returns (rows[steps,5] = t, rms_p, rms_n, zcm_p, zcm_n; fields; seconds).
        With step_times=True, seconds is an array: [0] the initial field solve,
        [1 + s] step s."""
        G = int(np.prod(world[0]))
        rows = np.zeros((steps, 5), np.float64)
        fields = np.zeros(11 * G, self.dtype) if want_fields else None
        times = np.zeros(steps + 1, np.float64)
        n, d = self._w(world)
        f = self._f("simulate")
        f.restype = C.c_double
        f.argtypes = ([C.c_void_p, C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 6 +
                      [C.c_double, C.c_int, C.c_int, C.c_int] + [C.c_double] * 4 +
                      [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                       C.c_void_p])
        secs = f(n, d, protons, neutrons, _ptr(x), _ptr(y), _ptr(z), _ptr(kx), _ptr(ky), _ptr(kz),
                 run.sigma_r, run.part_per_nucleon, run.z, run.n, run.A, run.B, run.C, run.gamma,
                 run.dt, run.t_exc, run.eta_exc, steps, smooth_mode, _ptr(rows), _ptr(fields), _ptr(times))
        return rows, fields, (times if step_times else secs)
