"""Python mirror of the reference's step interface over libhv_b200.so.

``Session`` owns one device context (one nucleus on one GPU).  Its methods are
the reference's routines, in the reference's vocabulary:

=============================  =============================================
Session method                 reference routine
=============================  =============================================
deposit()                      distribute_volumetric_particles_cic (tools.hpp:35-96)
smooth()                       compute_volumetric_densities (physics.hpp:202-234)
skyrme()                       compute_volumetric_skyrme_potentials (physics.hpp:272-281)
coulomb_boundary()             set_initial_coulomb_boundaries (tools.hpp:283-300)
coulomb_sor()                  compute_volumetric_coulomb_potentials_sor (physics.hpp:99-157)
merge()                        merge_volumetric_potentials (tools.hpp:377-384)
forces()                       compute_volumetric_forces_fdm (physics.hpp:159-200)
gather()                       distribute_forces_to_particles_cic (tools.hpp:98-168)
kick_half(dt) / drift(dt)      update_momenta_half / update_positions_full (physics.hpp:248-270)
excite(eta)                    nuclear_excitation (physics.hpp:236-246)
observe()                      center_of_mass / mean_squared_radius (tools.hpp:302-338)
particle_densities()           compute_particle_densities (tools.hpp:170-203)
particle_energies(ws, sigma_k) compute_particle_energies (tools.hpp:226-232)
fit_woods_saxon(ws)            minim_woods_saxon (fit_algorithm.hpp:95-137), GSL restated
initialize_particles(ws, eps)  initialize_particles (physics.hpp:34-97)
initial_solve() / run(steps)   cpu_simulate (src/hyper_vlasov.cpp:32-104)
=============================  =============================================

Arrays are numpy; the element type follows the session precision (float64 for
HV_F64, float32 for HV_F32).  Errors raise ``HVError``; nothing falls back to
the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .workloads import Workload


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _ws_array(ws):
    w = (L.hv_woods_saxon * 2)()
    for q in range(2):
        w[q].V0, w[q].R12, w[q].a = (float(v) for v in ws[q])
    return w


def _ws_tuple(w):
    return tuple((w[q].V0, w[q].R12, w[q].a) for q in range(2))


def generate_nucleus(seed, protons, neutrons, radius, k_fermi, dtype=np.float64):
    """Seeded synthetic nucleus (hv_generate_nucleus_*): six arrays x..kz."""
    lib = L.load()
    dt = np.dtype(dtype)
    total = protons + neutrons
    arrs = [np.zeros(total, dt) for _ in range(6)]
    f = lib.hv_generate_nucleus_f64 if dt == np.float64 else lib.hv_generate_nucleus_f32
    L.check(f(seed, protons, neutrons, radius, k_fermi, *[_p(a) for a in arrs]), "hv_generate_nucleus")
    return arrs


def workload_particles(w: Workload, dtype=np.float64):
    return generate_nucleus(w.seed, w.protons, w.neutrons, w.radius, w.k_fermi, dtype)


class Session:
    """One hv_ctx: device-resident particles and fields of one run."""

    def __init__(self, world: L.hv_world, protons: int, neutrons: int, params: L.hv_run_params,
                 precision: int = L.HV_F64, device: int = -1):
        self.lib = L.load()
        self.world = world
        self.protons, self.neutrons = protons, neutrons
        self.total = protons + neutrons
        self.precision = precision
        self.dtype = np.dtype(np.float64 if precision == L.HV_F64 else np.float32)
        self.G = world.n[0] * world.n[1] * world.n[2]
        self._ctx = C.c_void_p()
        L.check(self.lib.hv_ctx_create(C.byref(world), protons, neutrons, precision, C.byref(params), device,
                                       C.byref(self._ctx)), "hv_ctx_create")
        self.params = params

    @classmethod
    def from_workload(cls, w: Workload, precision=L.HV_F64, device=-1):
        return cls(w.world(), w.protons, w.neutrons, w.run_params(), precision, device)

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.hv_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._ctx

    def set_params(self, params: L.hv_run_params):
        L.check(self.lib.hv_ctx_set_params(self._ctx, C.byref(params)), "hv_ctx_set_params")
        self.params = params

    def fast_options(self) -> L.hv_fast_options:
        o = L.hv_fast_options()
        L.check(self.lib.hv_ctx_get_fast_options(self._ctx, C.byref(o)), "hv_ctx_get_fast_options")
        return o

    def set_fast_options(self, **kw):
        """Updates fields of hv_fast_options (sor_warm_start, sor_inner_min,
        sor_inner_max, sort_every, graph_steps, sor_exchange, smooth_fft, sor_omega,
        sor_wait_limit, sor_coarse, sor_coarse_sweeps, deposit_aggregate,
        sor_coarse_omega)."""
        o = self.fast_options()
        for k, v in kw.items():
            if not hasattr(o, k):
                raise KeyError(k)
            setattr(o, k, float(v) if k in ("sor_omega", "sor_coarse_omega") else int(v))
        L.check(self.lib.hv_ctx_set_fast_options(self._ctx, C.byref(o)), "hv_ctx_set_fast_options")

    def autotune(self, trial_steps=4):
        """hv_ctx_autotune: times the particle step's launch configurations and
        the SOR tiles over trial_steps fused steps each (the steps advance the
        run) and keeps the fastest; returns what it chose as a dict."""
        r = L.hv_autotune_report()
        L.check(self.lib.hv_ctx_autotune(self._ctx, int(trial_steps), C.byref(r)), "hv_ctx_autotune")
        return {k: getattr(r, k) for k, _ in r._fields_}

    KERNELS = ("particle", "smooth", "skyrme", "sor", "forces")

    def set_profiling(self, enable: bool):
        """Per-kernel CUDA-event timing of fused steps (direct launches)."""
        L.check(self.lib.hv_ctx_set_profiling(self._ctx, int(bool(enable))), "hv_ctx_set_profiling")

    def kernel_times(self):
        """{kernel: (total device ms, launches)} since profiling was enabled."""
        n = len(self.KERNELS)
        ms = (C.c_double * n)()
        ln = (C.c_int * n)()
        L.check(self.lib.hv_ctx_kernel_times(self._ctx, ms, ln, n), "hv_ctx_kernel_times")
        return {k: (ms[i], ln[i]) for i, k in enumerate(self.KERNELS)}

    def stream(self):
        """The context's CUDA stream (cudaStream_t as an integer)."""
        return self.lib.hv_ctx_stream(self._ctx) or 0

    def synchronize(self):
        L.check(self.lib.hv_ctx_synchronize(self._ctx), "hv_ctx_synchronize")

    # -- transfers ----------------------------------------------------------
    def _as(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        if a.size != self.total:
            raise ValueError(f"expected {self.total} elements, got {a.size}")
        return a

    def upload_particles(self, x, y, z, kx, ky, kz):
        arrs = [None if a is None else self._as(a) for a in (x, y, z, kx, ky, kz)]
        L.check(self.lib.hv_upload_particles(self._ctx, *[_p(a) for a in arrs]), "hv_upload_particles")

    def download_particles(self):
        arrs = [np.empty(self.total, self.dtype) for _ in range(6)]
        L.check(self.lib.hv_download_particles(self._ctx, *[_p(a) for a in arrs]), "hv_download_particles")
        return arrs

    def upload_array(self, name, a):
        a = self._as(a)
        L.check(self.lib.hv_upload_particle_array(self._ctx, L.HV_PART[name], _p(a)), "hv_upload_particle_array")

    def download_array(self, name):
        a = np.empty(self.total, self.dtype)
        L.check(self.lib.hv_download_particle_array(self._ctx, L.HV_PART[name], _p(a)), "hv_download_particle_array")
        return a

    def _field_len(self, field):
        return self.G if field == L.HV_FIELD_COULOMB else 2 * self.G

    def upload_field(self, field, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        if a.size != self._field_len(field):
            raise ValueError("field size")
        L.check(self.lib.hv_upload_field(self._ctx, field, _p(a)), "hv_upload_field")

    def download_field(self, field):
        a = np.empty(self._field_len(field), self.dtype)
        L.check(self.lib.hv_download_field(self._ctx, field, _p(a)), "hv_download_field")
        return a

    # -- routines ------------------------------------------------------------
    def deposit(self):
        L.check(self.lib.hv_deposit_cic(self._ctx), "hv_deposit_cic")

    def smooth(self):
        L.check(self.lib.hv_smooth_density(self._ctx), "hv_smooth_density")

    def skyrme(self):
        L.check(self.lib.hv_skyrme_potential(self._ctx), "hv_skyrme_potential")

    def coulomb_boundary(self):
        L.check(self.lib.hv_coulomb_boundary(self._ctx), "hv_coulomb_boundary")

    def coulomb_sor(self, allow_not_converged=False):
        it = C.c_int(0)
        m = C.c_double(0.0)
        st = self.lib.hv_coulomb_sor(self._ctx, C.byref(it), C.byref(m))
        if st == L.HV_ERR_NOT_CONVERGED and allow_not_converged:
            return it.value, m.value, False
        L.check(st, "hv_coulomb_sor")
        return it.value, m.value, True

    def merge(self):
        L.check(self.lib.hv_merge_potentials(self._ctx), "hv_merge_potentials")

    def forces(self):
        L.check(self.lib.hv_forces_fdm(self._ctx), "hv_forces_fdm")

    def gather(self):
        L.check(self.lib.hv_gather_cic(self._ctx), "hv_gather_cic")

    def kick_half(self, dt):
        L.check(self.lib.hv_kick_half(self._ctx, float(dt)), "hv_kick_half")

    def drift(self, dt):
        L.check(self.lib.hv_drift(self._ctx, float(dt)), "hv_drift")

    def excite(self, eta):
        L.check(self.lib.hv_excite(self._ctx, float(eta)), "hv_excite")

    def observe(self):
        o = L.hv_observables()
        L.check(self.lib.hv_observe(self._ctx, C.byref(o)), "hv_observe")
        return o

    def particle_densities(self):
        """(density_p, density_n) of every particle: compute_particle_densities
        (tools.hpp:170-203) on the device, with cell lists."""
        dp, dn = np.empty(self.total, self.dtype), np.empty(self.total, self.dtype)
        L.check(self.lib.hv_particle_densities(self._ctx, _p(dp), _p(dn)), "hv_particle_densities")
        return dp, dn

    def particle_energies(self, ws, sigma_k):
        """compute_particle_energies (tools.hpp:226-232) of every particle with
        Woods-Saxon parameters ws = ((V0, R12, a) protons, (V0, R12, a) neutrons)."""
        w = _ws_array(ws)
        e = np.empty(self.total, self.dtype)
        L.check(self.lib.hv_particle_energies(self._ctx, C.byref(w), float(sigma_k), _p(e)), "hv_particle_energies")
        return e

    def fit_woods_saxon(self, ws, skyrme=None):
        """minim_woods_saxon (fit_algorithm.hpp:95-137) on the particles and
        their densities, from ws; returns (fitted ws, iterations, status)."""
        w = _ws_array(ws)
        it, st = (C.c_int * 2)(), (C.c_int * 2)()
        sk = C.byref(skyrme) if skyrme is not None else None
        L.check(self.lib.hv_fit_woods_saxon(self._ctx, sk, C.byref(w), it, st), "hv_fit_woods_saxon")
        return _ws_tuple(w), tuple(it), tuple(st)

    def initialize_particles(self, ws, fermi, sigma_k=None, rng=L.HV_RNG_PHILOX, seed=128, max_iterations=0,
                             max_test_part=0, r_max=0.0, skyrme=None):
        """initialize_particles (physics.hpp:34-97) on the device: replaces the
        session's particles by the Woods-Saxon loop's.  ws as for
        fit_woods_saxon, fermi = (eps_p, eps_n) starting values; sigma_k None
        takes calc_sigma(0.346).  HV_RNG_LIBC draws rand() in the reference's
        order (seed it with srand first).  Returns (ws, fermi, report, rows):
        the final parameters, the hv_init_report fields as a dict and one
        hv_init_row per pass."""
        ip = L.hv_init_params()
        self.lib.hv_init_params_default(C.byref(ip))
        if sigma_k is not None:
            ip.sigma_k = float(sigma_k)
        ip.rng, ip.seed = int(rng), int(seed)
        ip.max_iterations, ip.max_test_part, ip.r_max = int(max_iterations), int(max_test_part), float(r_max)
        w = _ws_array(ws)
        f = L.hv_fermi(float(fermi[0]), float(fermi[1]))
        rep = L.hv_init_report()
        rows = (L.hv_init_row * (ip.max_iterations or 32))()
        sk = C.byref(skyrme) if skyrme is not None else None
        L.check(self.lib.hv_initialize_particles(self._ctx, sk, C.byref(w), C.byref(f), C.byref(ip), C.byref(rep),
                                                 rows), "hv_initialize_particles")
        report = {k: getattr(rep, k) for k, _ in L.hv_init_report._fields_}
        out_rows = [{"equal_p": r.equal_p, "equal_n": r.equal_n, "epsilon_p": r.epsilon_p,
                     "epsilon_n": r.epsilon_n, "delta_epsilon": r.delta_epsilon,
                     "ws": _ws_tuple(r.ws), "fit_iterations": tuple(r.fit_iterations),
                     "fit_status": tuple(r.fit_status)} for r in rows[:rep.iterations]]
        return _ws_tuple(w), (f.epsilon_p, f.epsilon_n), report, out_rows

    def write_vtk(self, path):
        """One VTK frame of the current forces, density and potential in the
        reference's format (include/init.hpp:159-254)."""
        L.check(self.lib.hv_write_vtk(self._ctx, str(path).encode()), "hv_write_vtk")

    def initial_solve(self):
        it = C.c_int(0)
        L.check(self.lib.hv_initial_solve(self._ctx, C.byref(it)), "hv_initial_solve")
        return it.value

    def run(self, steps, path=L.HV_PATH_PLAIN):
        obs = np.zeros(steps, L.OBS_DTYPE)
        L.check(self.lib.hv_run(self._ctx, steps, path, C.c_void_p(obs.ctypes.data)), "hv_run")
        return obs

    # -- adjoint ---------------------------------------------------------------
    def adjoint_forward(self, steps, checkpoint_every, path=L.HV_PATH_PLAIN):
        """hv_adjoint_forward_path: `steps` FP64 steps on `path` (plain or
        fused) with checkpoints every `checkpoint_every` steps; returns the
        observable rows."""
        obs = np.zeros(steps, L.OBS_DTYPE)
        L.check(self.lib.hv_adjoint_forward_path(self._ctx, path, steps, checkpoint_every,
                                                 C.c_void_p(obs.ctypes.data)),
                "hv_adjoint_forward_path")
        return obs

    def adjoint_stats(self):
        """hv_adjoint_stats: (path, iterations of the last backward pass's
        transposed Poisson solves, how many stopped at the iteration cap)."""
        p, it, un = C.c_int(0), C.c_int(0), C.c_int(0)
        L.check(self.lib.hv_adjoint_stats(self._ctx, C.byref(p), C.byref(it), C.byref(un)), "hv_adjoint_stats")
        return p.value, it.value, un.value

    def adjoint_backward(self, dJ_dD, theta):
        """hv_adjoint_backward: (dJ/d(t0, t3, sigma, a_sym), dJ/d(A, B, C, gamma))
        for dJ/dD of the rows of the last adjoint_forward, at theta."""
        g = np.ascontiguousarray(dJ_dD, dtype=np.float64)
        th = np.ascontiguousarray(theta, dtype=np.float64)
        gt, gs = np.zeros(4), np.zeros(4)
        L.check(self.lib.hv_adjoint_backward(self._ctx, _p(g), _p(th), _p(gt), _p(gs)), "hv_adjoint_backward")
        return gt, gs


def simulate(w: Workload, x, y, z, kx, ky, kz, steps, precision=L.HV_F64, path=L.HV_PATH_PLAIN):
    """hv_simulate: the whole GPU run with host buffers (advanced in place).
    Returns the per-step observables."""
    lib = L.load()
    dt = np.dtype(np.float64 if precision == L.HV_F64 else np.float32)
    arrs = (x, y, z, kx, ky, kz)
    for a in arrs:
        if a.dtype != dt or not a.flags.c_contiguous:
            raise ValueError("particle arrays must be contiguous and match the precision")
    obs = np.zeros(steps, L.OBS_DTYPE)
    world, params = w.world(), w.run_params()
    L.check(lib.hv_simulate(C.byref(world), w.protons, w.neutrons, precision, C.byref(params), path, steps,
                            *[_p(a) for a in arrs], C.c_void_p(obs.ctypes.data)), "hv_simulate")
    return obs


def simulate_release():
    """hv_simulate_release: frees the device contexts hv_simulate keeps
    between calls."""
    L.check(L.load().hv_simulate_release(), "hv_simulate_release")
