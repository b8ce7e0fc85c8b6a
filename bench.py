"""Throughput of the hyper-vlasov hot path on B200, in particle-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one time step of the 208Pb / 2.08M test particle / 128^3 (h = 0.25
fm, dt = 0.2 fm/c) workload: CIC deposit, smoothing, Skyrme potential,
red-black SOR Coulomb solve to relative residual 1e-6 (coarse-grid corrected
cycles whose sweeps relax at omega 1.7; plain cycles at the workload's 1.8),
forces, gather, leapfrog and the D(t) observables.  Inputs are synthetic (seeded
uniform-sphere nucleus), resident on the device before timing.

Our arm (default) prints one JSON line with:
  value        particle-steps/s of K fused FP32 steps, CUDA events on the
               context stream, max over ranks
  e2e          the same metric through hv_simulate with pinned host buffers:
               upload, initial solve, K steps, download of D(t) and particles
               (the context cached by an untimed first call)
  roofline     the dominant kernel (SOR) against measured HBM bandwidth, from
               a per-kernel CUDA-event pass of the same steps
  kernels      per-kernel device time, share and algorithmic GB/s
  plain_f64    the plain FP64 drop-in (one kernel per reference routine,
               host-tested SOR) on the same workload, and the D(t) agreement
  fused_f64    the fused path in double: the FP32 form's gain on one algorithm
  dipole_accuracy
               FP32 fused against plain FP64 over the workload's 1000 steps:
               D(t) and strength-function errors (the metric's 1e-3 bound);
               full_run: the FP32 run's throughput over all 1000 steps, timed
               in windows of 100
  warm_start_previous
               the same steps with each SOR started from the previous step's
               phi (the reference's guess) instead of 3 phi_n - 3 phi_(n-1) + phi_(n-2)
  deposit_sorted
               the deterministic sort-by-cell deposit: throughput and whether
               two runs give bit-identical D(t)
  adjoint      gradient of the D(t)-spectrum objective for 40Ca (40k) and 208Pb
               (104k) over 1000 steps: cost against forward runs, and a
               central-difference check on 208Pb
  particle_densities, initialisation
               the Woods-Saxon initialisation loop and its per-particle
               densities on the device, against the reference's routines
  batched      64 independent runs advanced together (sharded over ranks)
  cpu_baseline the reference's own routines on the host cores (rank 0, N=1)

--adjoint-horizons 100,200,400 prints, instead of the bench line, the adjoint's
gradient against central differences over those step counts (208Pb 104k).

--impl reference times the reference's CPU step routines (compiled from its
sources into oracle/_ref; the restated C oracle when that build is absent) on
the same workload, a bounded number of steps.

With torchrun (N > 1) every rank runs an independent replica of the workload
(weak scaling; the path does not shard), timed between barriers; the legs
that hold one GPU for minutes (plain_f64 onwards) run at N = 1 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hyper-vlasov_b200"))

METRIC = "particle-steps/s (208Pb, 2M tp)"
UNIT = "particle-steps/s"
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "sor_traffic.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="208Pb-2.08M-128^3")
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--warm-start", choices=["previous", "extrapolate", "quadratic"], default="quadratic")
    ap.add_argument("--sor-exchange", choices=["auto", "flags"], default="auto")
    ap.add_argument("--coarse-sweeps", type=int, default=0,
                    help="red+black sweeps after each coarse-grid correction in the headline's session "
                         "(0: the library's default, 12; e2e and the other legs keep the default)")
    ap.add_argument("--coarse-omega", type=float, default=0.0,
                    help="their relaxation in the headline's session (0: the library's default, 1.7)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-init", action="store_true", help="skip the initialisation legs (densities, loop)")
    ap.add_argument("--no-extrap", action="store_true", help="skip the other warm start's comparison run")
    ap.add_argument("--no-sorted", action="store_true", help="skip the deterministic sorted-deposit runs")
    ap.add_argument("--batch-steps", type=int, default=500)
    ap.add_argument("--adjoint-steps", type=int, default=1000)
    ap.add_argument("--adjoint-fd-steps", type=int, default=100)
    ap.add_argument("--adjoint-horizons", default="",
                    help="instead of the bench line: the adjoint against central differences on 208Pb for these "
                         "comma-separated step counts (fused FP64 path, SOR to 1e-12)")
    ap.add_argument("--accuracy-steps", type=int, default=1000)
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP32-against-FP64 D(t) leg")
    ap.add_argument("--autotune-steps", type=int, default=2, help="trial steps per autotuner candidate (0: off)")
    ap.add_argument("--cpu-sample", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--cpu-steps", type=int, default=2, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-warmup", type=int, default=0, help=argparse.SUPPRESS)
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts after nvidia-smi's own start-up (NVML
            # initialisation), once its first sample has arrived
            t0 = time.time()
            while not self.rows and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------- helpers
def dist_setup(gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v):
    from hv_b200 import replicas
    return replicas.max_over_ranks(v, world)


def sor_checks(n_sor, sweeps_per_cycle):
    """FP64 residual checks of a solve of n_sor red+black iterations whose
    cycles run sweeps_per_cycle iterations each (the coarse-corrected solve):
    one before each cycle and one after the last."""
    return math.ceil(n_sor / sweeps_per_cycle) + 1 if sweeps_per_cycle > 0 else 2


def step_bytes(w, n_sor, wordsize=4, checks=2, touched=None, force_frac=None):
    """Algorithmic bytes of one step, per kernel.  The particle step: 48 B per
    particle (x, k read and written) and, per grid node its particles touch
    (`touched`, counted over both species' grids; all 2 G when not given), the
    interleaved force read by the gather (4 words) and the raw density's
    read-modify-write by the deposit (2 words).  The grid kernels: 4 G B per
    word of traffic per node (smoothing 4, Skyrme 4, forces 10: the potential
    and phi read with their neighbours, the interleaved force written; SOR 3
    per red+black iteration).  The solve also streams its FP64 state: the
    extrapolated start (read phi and its two predecessors, write all three:
    48 B per node) and each residual check (read phi and the carried
    residual, write both: 32 B per node).  The float forces kernel with the
    atomic deposit computes only the row groups holding raw density
    (`force_frac` of them); it tests them by reading the raw density of every
    row (1 word per node of both species), except at 128^3, where the FFT
    smoothing's forward pass records the test while it reads that density."""
    G, N = w.G, w.particles
    s = wordsize / 4.0
    nodes = 2 * G if touched is None else touched
    return {
        "particle": s * (48 * N + 4 * nodes * (4 + 2)),
        "smooth": s * 4 * G * 4,
        "skyrme": s * 4 * G * 4,
        "sor": s * 4 * G * 3 * n_sor + G * (48 + 32 * checks),
        "forces": s * 4 * G * 10 if force_frac is None else s * 4 * G * ((0 if w.n == 128 else 2) + 10 * force_frac),
    }


def row_group_fraction(raw, n, rows=4):
    """Share of the forces kernel's work items that hold raw density: per
    species and x plane, groups of `rows` consecutive y rows (the last group
    shorter when n is not a multiple), a group counting when any node of its
    rows has nonzero raw density.  raw: both species' n^3 grids, stacked."""
    import numpy as np
    occupied = np.any(np.asarray(raw).reshape(2, n, n, n) != 0, axis=3)
    pad = (-n) % rows
    groups = np.any(np.pad(occupied, ((0, 0), (0, 0), (0, pad))).reshape(2, n, -1, rows), axis=3)
    return float(np.mean(groups))


# ---------------------------------------------------------------- CPU arm
def inputs_digest(arrays):
    """sha256 (first 16 hex digits) of the six input arrays' bytes, in order:
    both arms print it, so that the driver can see they start from the same
    particles."""
    import hashlib

    import numpy as np
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def product_libraries_loaded():
    """This repository's shared libraries mapped into this process, relative
    to the repository root (from /proc/self/maps)."""
    found = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if line.strip() else ""
                if path.endswith(".so") and path.startswith(ROOT):
                    found.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(found)


def cpu_sample(args):
    """Runs inside a child process with the stack and OpenMP settings the
    reference's deposit needs: the reference's step routines on the host.  The
    inputs come from the checker library's own restatement of the seeded
    generator, so this process never maps the CUDA library."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from hv_b200.workloads import WORKLOADS  # parameters only: loads no library
    from hv_oracle import Oracle, Reference, RunSpec, reference_available, workload_inputs
    w = WORKLOADS[args.workload]
    dt = np.float32 if args.precision == "f32" else np.float64
    A, B, Cc, g = w.skyrme()
    steps = args.cpu_warmup + args.cpu_steps
    run = RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc, eta_exc=w.eta,
                  A=A, B=B, C=Cc, gamma=g, sor_omega=w.sor_omega, sor_tol=w.sor_tol,
                  sor_criterion=w.sor_criterion, sor_max_iter=w.sor_max_iter)
    threads = os.cpu_count() or 1
    if reference_available("_portable"):
        r = Reference(dt, "_portable")
        parts = workload_inputs(r.lib, w, dt)
        digest = inputs_digest(parts)
        r.set_threads(threads)
        _, _, times = r.simulate(w.world_tuple(), run, w.protons, w.neutrons, *parts, steps, smooth_mode=1,
                                 step_times=True)
        kind = "reference"
        what = ("the reference's own routines (include/*.hpp, compiled from source, -O3 -march=x86-64-v3) in "
                "cpu_simulate order; its SOR is hard-wired to omega 1.5, |dphi| < 1e-4, 512 iterations; the "
                "O(G^2) smoothing replaced by the identical-pair-set offset table")
    else:
        o = Oracle(dt)
        parts = workload_inputs(o.lib, w, dt)
        digest = inputs_digest(parts)
        o.set_threads(threads)
        _, _, times = o.simulate(w.world_tuple(), run, w.protons, w.neutrons, *parts, steps, step_times=True)
        kind = "port"
        what = "the C restatement of the reference (oracle/hv_oracle.c) with the workload's SOR settings"
    timed = times[1 + args.cpu_warmup:]
    secs = float(timed.sum())
    print(json.dumps({"kind": kind, "seconds": secs, "steps": int(len(timed)), "init_seconds": float(times[0]),
                      "threads": threads, "what": what, "value": w.particles * len(timed) / secs,
                      "inputs_sha256": digest, "libraries_loaded": product_libraries_loaded()}))


def run_cpu_child(args, steps, warmup):
    env = dict(os.environ)
    env["OMP_STACKSIZE"] = "64M"  # the deposit reduction keeps a private 2G grid per thread
    env["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
    cmd = (f"ulimit -s unlimited; exec {sys.executable} {os.path.abspath(__file__)} --cpu-sample "
           f"--workload '{args.workload}' --precision {args.precision} --cpu-steps {steps} --cpu-warmup {warmup}")
    r = subprocess.run(["bash", "-c", cmd], capture_output=True, text=True, env=env, timeout=1800)
    for line in r.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("CPU sample failed: " + r.stderr[-2000:])


def reference_arm(args, world, rank):
    """The reference's CPU step on the host cores: the same workload, steps and
    warm-up steps as our arm (at most 60 and 5, so that the arm ends within a
    few minutes), in a child process that maps only the checker libraries."""
    if rank != 0:
        return
    from hv_b200.workloads import WORKLOADS  # parameters only: loads no library
    w = WORKLOADS[args.workload]
    steps = max(1, min(args.steps, 60))
    warm = max(0, min(args.warmup, 5))
    s = run_cpu_child(args, steps, warm)
    line = {
        "metric": METRIC, "value": s["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": s["steps"],
        "warmup": warm, "ms_per_step": 1e3 * s["seconds"] / s["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "impl": "reference",
        "config": {"workload": w.name, "particles": w.particles, "grid": f"{w.n}^3", "h_fm": w.h, "dt_fm_c": w.dt,
                   "sor": "the reference's own: omega 1.5, max|dphi| < 1e-4, at most 512 iterations"},
        "cpu_baseline": {"value": s["value"], "unit": UNIT, "cores": s["threads"], "kind": s["kind"],
                         "sample": f"{s['steps']} time steps of {w.name} after {warm} warm-up step(s) and the "
                                   f"initial solve ({s['init_seconds']:.1f} s, untimed); {s['what']}"},
        "e2e": {"value": s["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "inputs_sha256": s["inputs_sha256"],
        "libraries_loaded": s["libraries_loaded"] + product_libraries_loaded(),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- adjoint
def adjoint_cases(args, local):
    """The adjoint workload: the gradient of the power of the D(t) spectrum in
    10-25 MeV with respect to (t0, t3, sigma, a_sym), for 40Ca with 1000 test
    particles per nucleon (32^3, h = 1 fm) and 208Pb with 500 (64^3, h =
    0.5 fm), dt = 0.5 fm/c, args.adjoint_steps steps (1000), checkpoints every
    50 steps, FP64 with the deterministic deposit, on both paths.  Per case
    and path: the forward run, the checkpointed forward and the backward pass
    (host wall time around the synchronous calls) and their ratio -- the cost
    against a forward run of the same precision and path; the fused FP64
    adjoint's gradient against the plain one's, and both against the fused
    FP32 forward of that case.  For 208Pb, central-difference checks of both
    paths (relative step 1e-3, SOR to 1e-12 so that its stopping rule adds no
    noise) over args.adjoint_fd_steps steps."""
    from dataclasses import replace

    import numpy as np
    import torch

    import hv_b200 as hv
    from hv_b200.spectrum import power_in_band
    steps, every = args.adjoint_steps, 50
    cases = {"ca40_40k_32": replace(hv.CA40_SMALL, ppn=1000, dt=0.5, deposit_mode=hv.HV_DEPOSIT_SORTED),
             "pb208_104k_64": replace(hv.PB208_104K, dt=0.5, deposit_mode=hv.HV_DEPOSIT_SORTED)}
    out = {"objective": "power of the D(t) spectrum in 10-25 MeV", "steps": steps, "checkpoint_every": every,
           "timing": "host wall time around the synchronous calls"}

    def objective_grad(obs, w, n):
        d = torch.tensor(obs["dipole"], dtype=torch.float64, requires_grad=True)
        J = power_in_band(d, np.arange(n) * w.dt, n * w.dt, w.dt)
        J.backward()
        return float(J), d.grad.numpy()

    for key, w in cases.items():
        parts = hv.workload_particles(w, np.float64)
        theta = np.array([w.t0, w.t3, w.sigma, w.a_sym])
        with hv.Session.from_workload(w, hv.HV_F64, device=local) as s:
            s.upload_particles(*parts)
            s.initial_solve()
            t0 = time.perf_counter()
            s.run(steps, hv.HV_PATH_PLAIN)
            plain = time.perf_counter() - t0
        with hv.Session.from_workload(w, hv.HV_F32, device=local) as s:
            s.upload_particles(*[p.astype(np.float32) for p in parts])
            s.run(1, hv.HV_PATH_FUSED)
            t0 = time.perf_counter()
            s.run(steps, hv.HV_PATH_FUSED)
            fused = time.perf_counter() - t0
        with hv.Session.from_workload(w, hv.HV_F64, device=local) as s:
            s.upload_particles(*parts)
            s.initial_solve()
            t0 = time.perf_counter()
            obs = s.adjoint_forward(steps, every)
            t1 = time.perf_counter()
            J, dJ = objective_grad(obs, w, steps)
            grad, _ = s.adjoint_backward(dJ, theta)
            t2 = time.perf_counter()
            _, plain_adj_its, _ = s.adjoint_stats()
        # the fused FP64 path: its forward, then its adjoint
        with hv.Session.from_workload(w, hv.HV_F64, device=local) as s:
            s.upload_particles(*parts)
            s.run(1, hv.HV_PATH_FUSED)
            t0f = time.perf_counter()
            s.run(steps, hv.HV_PATH_FUSED)
            fused64 = time.perf_counter() - t0f
        with hv.Session.from_workload(w, hv.HV_F64, device=local) as s:
            s.upload_particles(*parts)
            s.run(0, hv.HV_PATH_FUSED)
            t3 = time.perf_counter()
            obs_f = s.adjoint_forward(steps, every, hv.HV_PATH_FUSED)
            t4 = time.perf_counter()
            Jf, dJf = objective_grad(obs_f, w, steps)
            grad_f, _ = s.adjoint_backward(dJf, theta)
            t5 = time.perf_counter()
            _, fused_adj_its, fused_unconv = s.adjoint_stats()
        gscale = float(np.max(np.abs(grad)))
        out[key] = {"workload": f"{w.Z + w.N} nucleons x {w.ppn} test particles ({w.particles}), {w.n}^3 at "
                                f"h {w.h} fm, dt {w.dt} fm/c",
                    "objective_value": J, "plain_forward_s": plain, "checkpointed_forward_s": t1 - t0,
                    "backward_s": t2 - t1, "gradient_over_forward": (t2 - t0) / plain,
                    "adjoint_sor_iterations_per_step": plain_adj_its / steps,
                    "fused_f32_forward_s": fused, "gradient_over_fused_f32_forward": (t2 - t0) / fused,
                    "grad_t0_t3_sigma_asym": [float(v) for v in grad],
                    "fused_f64": {
                        "objective_value": Jf, "forward_s": fused64, "checkpointed_forward_s": t4 - t3,
                        "backward_s": t5 - t4, "gradient_over_forward": (t5 - t3) / fused64,
                        "gradient_over_fused_f32_forward": (t5 - t3) / fused,
                        "speedup_over_plain_gradient": (t2 - t0) / (t5 - t3),
                        "adjoint_sor_iterations_per_step": fused_adj_its / steps,
                        "adjoint_sor_unconverged": fused_unconv,
                        "grad_t0_t3_sigma_asym": [float(v) for v in grad_f],
                        "max_abs_diff_from_plain_gradient_over_max": (float(np.max(np.abs(grad_f - grad))) / gscale
                                                                      if gscale > 0 else None)}}
    # central differences on 208Pb over fewer steps
    fd_steps = args.adjoint_fd_steps
    if fd_steps > 0:
        from hv_b200.adjoint import AdjointRun
        w = replace(cases["pb208_104k_64"], sor_tol=1e-12)
        parts = hv.workload_particles(w, np.float64)
        theta = np.array([w.t0, w.t3, w.sigma, w.a_sym])

        def fn(dd):
            d = torch.tensor(dd, dtype=torch.float64)
            return float(power_in_band(d, np.arange(fd_steps) * w.dt, fd_steps * w.dt, w.dt))
        for name, path in (("pb208_104k_64_central_differences", hv.HV_PATH_PLAIN),
                           ("pb208_104k_64_central_differences_fused_f64", hv.HV_PATH_FUSED)):
            run = AdjointRun(w, parts, fd_steps, checkpoint_every=every, device=local, path=path)
            try:
                run.forward(theta)
                _, dJ = objective_grad(run.obs, w, fd_steps)
                g_adj = run.backward(dJ)
                g_fd = np.zeros(4)
                for i in range(4):
                    hstep = 1e-3 * abs(theta[i])
                    tp, tm = theta.copy(), theta.copy()
                    tp[i] += hstep
                    tm[i] -= hstep
                    g_fd[i] = (run.objective(tp, fn) - run.objective(tm, fn)) / (2 * hstep)
            finally:
                run.close()
            scale = float(np.max(np.abs(g_fd)))
            out[name] = {
                "steps": fd_steps, "relative_step": 1e-3, "sor_tol": 1e-12, "adjoint": [float(v) for v in g_adj],
                "finite_differences": [float(v) for v in g_fd],
                "max_abs_diff_over_max_abs_fd": float(np.max(np.abs(g_adj - g_fd))) / scale if scale > 0 else None}
        ga = np.array(out["pb208_104k_64_central_differences"]["adjoint"])
        gb = np.array(out["pb208_104k_64_central_differences_fused_f64"]["adjoint"])
        out["pb208_104k_64_fused_vs_plain_adjoint_max_abs_diff_over_max"] = float(
            np.max(np.abs(gb - ga)) / np.max(np.abs(ga)))
    return out


def adjoint_horizons(args):
    """The adjoint's gradient of the spectrum objective against central
    differences at relative steps 1e-3 and 1e-5, for 208Pb with 500 test
    particles per nucleon (64^3, dt 0.5 fm/c, deterministic deposit, SOR to
    1e-12) on the fused FP64 path, over each step count of
    --adjoint-horizons: how far the linearisation of the test-particle
    dynamics holds.  Prints one JSON line."""
    from dataclasses import replace

    import numpy as np
    import torch

    import hv_b200 as hv
    from hv_b200.adjoint import AdjointRun
    from hv_b200.spectrum import power_in_band
    w = replace(hv.PB208_104K, dt=0.5, deposit_mode=hv.HV_DEPOSIT_SORTED, sor_tol=1e-12)
    parts = hv.workload_particles(w, np.float64)
    theta = np.array([w.t0, w.t3, w.sigma, w.a_sym])
    out = {"study": "adjoint against central differences by horizon", "workload": "208Pb 104k 64^3, dt 0.5 fm/c",
           "path": "fused FP64", "objective": "power of the D(t) spectrum in 10-25 MeV", "horizons": {}}
    for steps in (int(v) for v in args.adjoint_horizons.split(",")):
        t = np.arange(steps) * w.dt

        def fn(dd):
            return float(power_in_band(torch.tensor(dd, dtype=torch.float64), t, steps * w.dt, w.dt))
        run = AdjointRun(w, parts, steps, checkpoint_every=50, path=hv.HV_PATH_FUSED)
        try:
            d = torch.tensor(run.forward(theta), dtype=torch.float64, requires_grad=True)
            J = power_in_band(d, t, steps * w.dt, w.dt)
            J.backward()
            g = run.backward(d.grad.numpy())
            res = {"objective": float(J.detach()), "adjoint": [float(v) for v in g]}
            for rel in (1e-3, 1e-5):
                gf = np.zeros(4)
                for i in range(4):
                    h = rel * abs(theta[i])
                    tp, tm = theta.copy(), theta.copy()
                    tp[i] += h
                    tm[i] -= h
                    gf[i] = (run.objective(tp, fn) - run.objective(tm, fn)) / (2 * h)
                res[f"fd_{rel:g}"] = [float(v) for v in gf]
                res[f"max_abs_diff_over_max_abs_fd_{rel:g}"] = float(np.max(np.abs(g - gf)) / np.max(np.abs(gf)))
        finally:
            run.close()
        out["horizons"][str(steps)] = res
    print(json.dumps(out), flush=True)


def dipole_accuracy(args, w, parts32, local):
    """The metric's accuracy qualifier over the workload's full run: the FP32
    fused path (the headline's settings) against the plain FP64 path (every
    stage bit-identical to the reference's routines) from the same particles,
    args.accuracy_steps steps: max|D32 - D64| / max|D64| and the same for the
    strength function S(E) of the two series (detrended, cos^2-windowed FFT,
    scripts/programs.py:82-122)."""
    import numpy as np

    import hv_b200 as hv
    from hv_b200.spectrum import energy_spectrum
    steps = args.accuracy_steps
    t0 = time.perf_counter()
    with hv.Session.from_workload(w, hv.HV_F64, device=local) as s:
        s.upload_particles(*[p.astype(np.float64) for p in parts32])
        s.initial_solve()
        o64 = s.run(steps, hv.HV_PATH_PLAIN)
    t_plain = time.perf_counter() - t0
    # the FP32 run, timed in windows of 100 steps (CUDA events on the context
    # stream, after the initial field solve): the throughput over the whole
    # run, whose later steps see escaping test particles near the faces
    import torch
    win = 100
    with hv.Session.from_workload(w, hv.HV_F32, device=local) as s:
        s.upload_particles(*parts32)
        s.run(0, hv.HV_PATH_FUSED)
        stream = torch.cuda.ExternalStream(s.stream())
        parts_obs, win_ms = [], []
        done = 0
        while done < steps:
            k = min(win, steps - done)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            parts_obs.append(s.run(k, hv.HV_PATH_FUSED))
            e1.record(stream)
            e1.synchronize()
            win_ms.append(e0.elapsed_time(e1) / k)
            done += k
        o32 = np.concatenate(parts_obs)
    run_ms = float(sum(m * min(win, steps - i * win) for i, m in enumerate(win_ms)))
    full_run = {"value": w.particles * steps / (run_ms / 1e3), "unit": UNIT, "steps": steps,
                "ms_per_step": run_ms / steps, "ms_per_step_by_100_steps": [round(m, 4) for m in win_ms],
                "note": "the FP32 fused run of this accuracy leg, from step 0 after the initial field solve"}
    dmax = float(np.max(np.abs(o64["dipole"])))
    t_f = steps * w.dt
    e64, s64 = energy_spectrum(o64["t"], o64["zcm_p"], o64["zcm_n"], w.Z, w.N, t_f, w.dt, w.eta)
    e32, s32 = energy_spectrum(o32["t"], o32["zcm_p"], o32["zcm_n"], w.Z, w.N, t_f, w.dt, w.eta)
    smax = float(np.max(np.abs(s64)))
    return {"steps": steps, "reference": "plain FP64 path (per-routine kernels, bit-identical stages)",
            "dipole_max_rel_err": float(np.max(np.abs(o32["dipole"] - o64["dipole"]))) / dmax,
            "strength_max_rel_err": float(np.max(np.abs(s32 - s64))) / smax,
            "bound": 1e-3, "sor_not_converged_steps": int(np.sum(o32["flags"] & 1) + np.sum(o64["flags"] & 1)),
            "plain_f64_run_s": t_plain, "full_run": full_run}


# ---------------------------------------------------------------- init
def particle_densities_cost(args, local, world):
    """compute_particle_densities (the initialisation's O(N^2) per-particle
    densities) on the device with cell lists: 208Pb with 500 test particles
    per nucleon (104k, FP64) and with 10000 (2.08M, FP32), against the
    reference's own routine on all host threads at 104k (one GPU only)."""
    import numpy as np

    import hv_b200 as hv
    out = {}
    for key, w, prec in (("pb208_104k_f64", hv.PB208_104K, hv.HV_F64), ("pb208_2m_f32", hv.PB208_2M, hv.HV_F32)):
        dt = np.float64 if prec == hv.HV_F64 else np.float32
        p = hv.workload_particles(w, dt)
        with hv.Session.from_workload(w, prec, device=local) as s:
            s.upload_particles(*p)
            s.particle_densities()
            t0 = time.perf_counter()
            s.particle_densities()
            out[key + "_gpu_s"] = time.perf_counter() - t0
    if world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from hv_oracle import Reference, reference_available
        if reference_available("_portable"):
            w = hv.PB208_104K
            p = hv.workload_particles(w, np.float64)
            r = Reference(np.float64, "_portable")
            r.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            r.particle_densities(w.protons, w.neutrons, *p[:3], w.sigma_r, w.ppn)
            out["pb208_104k_f64_cpu_reference_s"] = time.perf_counter() - t0
            out["cpu_cores"] = os.cpu_count()
            out["speedup_104k"] = out["pb208_104k_f64_cpu_reference_s"] / out["pb208_104k_f64_gpu_s"]
    out["timing"] = "host wall time of hv_particle_densities (incl. download), second call"
    return out


def initialisation_cost(args, local, world):
    """initialize_particles (the Woods-Saxon self-consistency loop) on the
    device: 208Pb with 10000 test particles per nucleon (2.08M, FP32, Philox
    random numbers), and 40Ca with 1000 (40k, FP64) drawing the C library's
    rand() in the reference's order -- the reference's own loop, whose GSL fit
    is replaced by the oracle's restatement, runs the same random stream on
    all host threads (one GPU only).  Host wall time around each call."""
    import ctypes

    import numpy as np

    import hv_b200 as hv
    from dataclasses import replace
    from hv_b200.workloads import INIT_K_FWHM, INIT_SKYRME, init_start, sigma_from_fwhm
    libc = ctypes.CDLL(None)
    sigma_k = sigma_from_fwhm(INIT_K_FWHM)
    out = {}
    for key, w, prec, rng in (("pb208_2m_f32_philox", hv.PB208_2M, hv.HV_F32, hv.HV_RNG_PHILOX),
                              ("ca40_40k_f64_libc", replace(hv.CA40_SMALL, ppn=1000), hv.HV_F64, hv.HV_RNG_LIBC)):
        params = w.run_params()
        params.skyrme = hv._lib.hv_skyrme(*INIT_SKYRME)
        ws, fermi = init_start(w.Z, w.N)
        with hv.Session(w.world(), w.protons, w.neutrons, params, prec, device=local) as s:
            libc.srand(128)
            t0 = time.perf_counter()
            _, _, rep, _ = s.initialize_particles(ws, fermi, sigma_k=sigma_k, rng=rng)
            out[key + "_gpu_s"] = time.perf_counter() - t0
        out[key + "_passes"] = rep["iterations"]
        out[key + "_converged"] = bool(rep["converged"])
        out[key + "_candidates"] = rep["candidates"]
    if world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from hv_oracle import Reference, reference_available
        if reference_available("_portable"):
            w = replace(hv.CA40_SMALL, ppn=1000)
            ws, fermi = init_start(w.Z, w.N)
            r = Reference(np.float64, "_portable")
            r.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            ro = r.initialize_particles(w.Z, w.N, w.ppn, sigma_k, w.sigma_r, INIT_SKYRME, ws, fermi, 128)
            out["ca40_40k_f64_cpu_reference_s"] = time.perf_counter() - t0
            out["ca40_40k_f64_cpu_reference_passes"] = ro["passes"]
            out["cpu_cores"] = os.cpu_count()
            out["speedup_40k"] = out["ca40_40k_f64_cpu_reference_s"] / out["ca40_40k_f64_libc_gpu_s"]
    out["timing"] = "host wall time of hv_initialize_particles (incl. the final store of the particles)"
    return out


# ---------------------------------------------------------------- batched
def batched(args, local, world=1, rank=0):
    """The batched form: 64 independent runs (16O..208Pb, 200-2000 test
    particles per nucleon, 32^3-96^3 at h = 0.5 fm, jittered Skyrme
    parameters and boosts) advanced together by hv_batch_run after the
    autotuner chose the SOR block cap; on one GPU, against the same instances
    stepped one after another by their own fused runs.  With N ranks every
    rank takes the runs that longest-processing-time-first assigns it by
    estimated cost (no per-step collective), the timed region is bracketed by
    barriers and maxed over ranks, and the D(t) series are gathered at the
    end.  Host wall time around the calls (each synchronises at its end)."""
    import numpy as np

    import hv_b200 as hv
    from hv_b200 import replicas
    from hv_b200.batch import Batch
    from hv_b200.workloads import batch_workloads
    all_ws = batch_workloads(64, seed=0)
    mine = replicas.assign_runs([replicas.run_cost(w.particles, w.G) for w in all_ws], world)[rank]
    ws = [all_ws[i] for i in mine]
    K = args.batch_steps
    parts = [hv.workload_particles(w, np.float32) for w in ws]
    sess = []
    try:
        for w, p in zip(ws, parts):
            s = hv.Session.from_workload(w, hv.HV_F32, device=local)
            s.upload_particles(*p)
            sess.append(s)
        t0 = time.perf_counter()
        with Batch(sess) as b:
            setup = time.perf_counter() - t0
            cap = b.autotune(2)
            tiles = b.tiles()
            b.run(3)
            barrier(world)
            t0 = time.perf_counter()
            obs = b.run(K)
            el = time.perf_counter() - t0
            barrier(world)
            waves = b.waves()
        seq = None
        if world == 1:  # the same instances one after another, each on its own fused path
            ks = 8
            for s in sess:
                s.run(2, hv.HV_PATH_FUSED)
            t0 = time.perf_counter()
            for s in sess:
                s.run(ks, hv.HV_PATH_FUSED)
            seq = time.perf_counter() - t0
    finally:
        for s in sess:
            s.close()
    el = max_over_ranks(world, el)
    series = replicas.gather_series({i: obs[j]["dipole"].tolist() for j, i in enumerate(mine)}, world)
    N = sum(w.particles for w in all_ws)
    value = N * K / el
    out = {"value": value, "unit": UNIT, "instances": len(all_ws), "particles": N, "n_gpus": world,
           "grid_nodes": sum(w.G for w in all_ws), "steps": K, "ms_per_step": 1e3 * el / K,
           "sor_waves_rank0": waves, "autotuned_sor_block_cap_rank0": cap, "setup_s": setup,
           "autotuned_particle_block_rank0": tiles[0][3] if tiles else None,
           "sor_tiles_rank0": {f"{P}x{R}": sum(1 for t in tiles if t[:2] == (P, R)) for P, R, *_ in tiles},
           "sor_iterations_per_step_mean_rank0": float(obs["sor_iterations"].mean()),
           "dipole_series_gathered": len(series)}
    if seq is not None:
        out.update({"sequential_value": N * ks / seq, "speedup_over_sequential": value / (N * ks / seq)})
    out.update({
            "workload": "64 runs: 16O/40Ca/90Zr/208Pb, 200-2000 tp/nucleon log-uniform, 32^3-96^3 at h 0.5 fm, "
                        "t0 and t3 +-5 %, boosts 10-40 MeV/c, dt 0.25 fm/c, FP32 fused",
            "timing": "host wall time around hv_batch_run, max over ranks"})
    return out


def fused_f64_leg(w, parts, local, K, start, value_f32, obs_f32):
    """The fused path in double (HV_F64 on HV_PATH_FUSED: the same kernels,
    warm start and stopping rule as the headline, with particles, grids and
    the solver's correction in double, in plain SOR cycles), advanced to the
    headline's first timed step and then over its K steps: the FP32 form's
    gain on one algorithm, and the D(t) agreement of the timed steps."""
    import numpy as np
    import torch

    import hv_b200 as hv
    p64 = [p.astype(np.float64) for p in parts]
    with hv.Session.from_workload(w, hv.HV_F64, device=local) as s:
        s.upload_particles(*p64)
        s.run(start, hv.HV_PATH_FUSED)
        st = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        o = s.run(K, hv.HV_PATH_FUSED)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    v = w.particles * K / (ms / 1e3)
    dmax = float(np.max(np.abs(o["dipole"])))
    return {"value": v, "unit": UNIT, "ms_per_step": ms / K, "steps": K,
            "sor_iterations_per_step": float(o["sor_iterations"].mean()),
            "speedup_of_value_f32_over_f64": value_f32 / v,
            "dipole_max_rel_diff_f32": float(np.max(np.abs(obs_f32["dipole"] - o["dipole"]))) / dmax
            if dmax > 0 else None}


def sorted_deposit_leg(args, w, prec, parts, local, K, W):
    """The same workload with the deterministic sort-by-cell deposit
    (HV_DEPOSIT_SORTED): its throughput over K steps, and whether two runs give
    bit-identical D(t)."""
    import numpy as np
    import torch
    from dataclasses import replace

    import hv_b200 as hv
    ws = replace(w, deposit_mode=hv.HV_DEPOSIT_SORTED)
    dips, ms = [], None
    for rep in range(2):
        with hv.Session.from_workload(ws, prec, device=local) as s:
            s.upload_particles(*parts)
            s.run(W, hv.HV_PATH_FUSED)
            st = torch.cuda.ExternalStream(s.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            o = s.run(K, hv.HV_PATH_FUSED)
            e1.record(st)
            e1.synchronize()
            if rep == 0:
                ms = e0.elapsed_time(e1)
            dips.append(np.array(o["dipole"]))
    return {"value": w.particles * K / (ms / 1e3), "ms_per_step": ms / K,
            "deterministic": bool(np.array_equal(dips[0], dips[1])),
            "note": "sort-by-cell deposit, nodes summed in particle-slot order; two runs compared bit for bit"}


# ---------------------------------------------------------------- GPU arm
def our_arm(args, world, rank, local):
    import numpy as np
    import torch

    import hv_b200 as hv
    w = hv.WORKLOADS[args.workload]
    prec = hv.HV_F32 if args.precision == "f32" else hv.HV_F64
    dt = np.float32 if prec == hv.HV_F32 else np.float64
    K, W = args.steps, max(3, args.warmup)
    warm_mode = {"previous": hv.HV_WARM_PREVIOUS, "extrapolate": hv.HV_WARM_EXTRAPOLATE,
                 "quadratic": hv.HV_WARM_QUADRATIC}[args.warm_start]
    parts = hv.workload_particles(w, dt)
    digest = inputs_digest(parts)
    torch.cuda.set_device(local)

    sess = hv.Session.from_workload(w, prec, device=local)
    sess.set_fast_options(sor_warm_start=warm_mode, sor_exchange=hv.HV_SOR_EXCHANGE_FLAGS
                          if args.sor_exchange == "flags" else hv.HV_SOR_EXCHANGE_AUTO)
    if args.coarse_sweeps > 0:
        sess.set_fast_options(sor_coarse_sweeps=args.coarse_sweeps)
    if args.coarse_omega > 0:
        sess.set_fast_options(sor_coarse_omega=args.coarse_omega)
    sess.upload_particles(*parts)
    stream = torch.cuda.ExternalStream(sess.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the clock sampler starts before the autotuner, so that its start-up
    # (up to a second of nvidia-smi initialisation, with the GPU idle) is
    # followed by the autotuner's trial steps and the warm-up steps rather than
    # by the timed steps; it samples through the timed region
    with ClockSampler(local) as clk:
        # the launch configuration chosen by the project's autotuner (its
        # trial steps advance the run), then the warm-up steps
        tune = sess.autotune(args.autotune_steps) if args.autotune_steps > 0 else None
        sess.run(W, hv.HV_PATH_FUSED)  # includes the initial field solve when not tuned
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        obs = sess.run(K, hv.HV_PATH_FUSED)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(world, ms)
    # the step the timed rows start at (the autotuner's trial steps and the
    # warm-up came first): the comparison legs below start there too
    start = int(round(float(obs["t"][0]) / w.dt))
    value = w.particles * K * world / (ms_max / 1e3)
    sor_its = obs["sor_iterations"].astype(np.int64)

    # per-kernel device times over the same number of steps (direct launches)
    sess.set_profiling(True)
    obs_p = sess.run(K, hv.HV_PATH_FUSED)
    kt = sess.kernel_times()
    sess.set_profiling(False)
    its_p = obs_p["sor_iterations"].astype(np.int64)
    fo = sess.fast_options()
    per_cycle = fo.sor_coarse_sweeps if (fo.sor_coarse and prec == hv.HV_F32) else 0
    ws_ = 4 if prec == hv.HV_F32 else 8
    # grid nodes the particle step's gathers and deposit touch: the nonzero
    # nodes of the raw density its last launch deposited (both species); the
    # forces kernel's row groups (4 y rows of one x plane and species in the
    # float steps) that hold any of them are the ones it computes
    raw = sess.download_field(hv.HV_FIELD_DENSITY_RAW)
    touched = int(np.count_nonzero(raw))
    gated = prec == hv.HV_F32 and w.deposit_mode != hv.HV_DEPOSIT_SORTED
    force_frac = row_group_fraction(raw, w.n, 4) if gated else None
    nbytes = step_bytes(w, its_p.mean(), ws_, float(np.mean([sor_checks(n, per_cycle) for n in its_p])),
                        touched=touched, force_frac=force_frac)
    tot_ms = sum(v[0] for v in kt.values())
    kernels = {}
    for k, (kms, n) in kt.items():
        if n == 0:
            continue
        per = kms / n
        b = nbytes[k]
        kernels[k] = {"launches": n, "avg_ms": per, "share": kms / tot_ms if tot_ms else None,
                      "algorithmic_bytes": b, "gbs": b / (per / 1e3) / 1e9}
    if "particle" in kernels:
        kernels["particle"]["touched_nodes"] = touched
    if "forces" in kernels and force_frac is not None:
        kernels["forces"]["computed_row_groups"] = force_frac
    peak, peak_kind = peaks()
    sor_b = sum(step_bytes(w, n, ws_, sor_checks(n, per_cycle))["sor"] for n in its_p)
    sor_ms = kt["sor"][0]
    achieved = sor_b / (sor_ms / 1e3) / 1e9 if sor_ms > 0 else None
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        try:
            with open(PROFILE_TRAFFIC) as f:
                traffic = json.load(f).get("bytes_per_launch")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": traffic,
                "kernel": "k_sor_fast (persistent red-black SOR, coarse-grid corrected)", "peak_source": peak_kind,
                "bytes": "per solve: 12 B per node per red+black iteration (read phi, rho_p; write phi), 48 B per "
                         "node for the extrapolated start, 32 B per node per FP64 residual check",
                "mean_sor_iterations": float(its_p.mean()),
                "sor_checks_per_solve": float(np.mean([sor_checks(n, per_cycle) for n in its_p]))}

    # per step: particle step, smoothing, Skyrme, SOR, forces (which also
    # advances the step counter);
    # the FFT smoothing (power-of-two axes up to 128; by default for stencil
    # half-widths >= 6 nodes, 4 sigma / h) adds its three passes before the
    # march kernel, which then only checks the edge flags
    opts = sess.fast_options()
    pow2 = all(n & (n - 1) == 0 and 2 <= n <= 128 for n in (w.n, w.n, w.n))
    half_width = int(4.0 * w.sigma_r / w.h)
    fft = pow2 and (opts.smooth_fft == 2 or (opts.smooth_fft == 1 and half_width >= 6))
    launches_per_step = 5 + (3 if fft else 0)
    chunk = opts.graph_steps or 8
    # slot re-sorts: one every sort_every steps, at the start of a graph
    # chunk; each launches its key kernel and ten gathers of ours (the radix
    # sort itself is CUB's)
    resorts = math.ceil(K / opts.sort_every) if opts.sort_every > 0 else 0
    gpu_launches = K * launches_per_step + math.ceil(K / chunk) + 11 * resorts
    sess.close()

    # the same K steps from the other initial guess of the solve (the
    # reference's: the previous step's phi), same stopping rule, for comparison
    extrap = None
    other = hv.HV_WARM_PREVIOUS if warm_mode != hv.HV_WARM_PREVIOUS else hv.HV_WARM_QUADRATIC
    if not args.no_extrap:
        with hv.Session.from_workload(w, prec, device=local) as sx:
            sx.set_fast_options(sor_warm_start=other)
            sx.upload_particles(*parts)
            sx.run(start, hv.HV_PATH_FUSED)
            sstream = torch.cuda.ExternalStream(sx.stream())
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            f0.record(sstream)
            obs_x = sx.run(K, hv.HV_PATH_FUSED)
            f1.record(sstream)
            f1.synchronize()
            msx = f0.elapsed_time(f1)
        dref = np.max(np.abs(obs["dipole"]))
        extrap = {"value": w.particles * K / (msx / 1e3), "ms_per_step": msx / K,
                  "sor_iterations_per_step": float(obs_x["sor_iterations"].mean()),
                  "dipole_max_rel_diff_vs_headline": float(np.max(np.abs(obs_x["dipole"] - obs["dipole"])) / dref)
                  if dref > 0 else None,
                  "note": ("SOR started from the previous step's phi (the reference's guess)"
                           if other == hv.HV_WARM_PREVIOUS else "SOR started from 3 phi_n - 3 phi_(n-1) + phi_(n-2)") +
                          ", same stopping rule"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": w.name, "nucleus": f"208Pb (Z={w.Z}, N={w.N})", "particles": w.particles,
                   "grid": f"{w.n}^3", "h_fm": w.h, "dt_fm_c": w.dt,
                   "sor": (f"red-black SOR to relative residual {w.sor_tol:g} (FP64 test): omega {w.sor_omega} in "
                           f"plain cycles; each coarse-grid corrected cycle smooths with {fo.sor_coarse_sweeps} "
                           f"sweeps at omega {fo.sor_coarse_omega if fo.sor_coarse_omega > 0 else 1.7:g}"
                           if (fo.sor_coarse and prec == hv.HV_F32) else
                           f"red-black omega {w.sor_omega} to relative residual {w.sor_tol:g}"),
                   "warm_start": args.warm_start, "sor_exchange": args.sor_exchange, "path": "fused",
                   "precision": "f32 particles/grids, f64 phi, SOR residual and observable sums",
                   "parallelism": f"replicas x{world}",
                   "l2": "working set larger than L2 (particle state 50 MB + 2x128^3 fields ~120 MB)"},
        "sor_iterations_per_step": float(sor_its.mean()), "autotune": tune,
        "roofline": roofline, "kernels": kernels, "gpu_launches": gpu_launches,
        "clocks": clk.summary(), "inputs_sha256": digest,
    }
    if extrap:
        line["warm_start_previous" if other == hv.HV_WARM_PREVIOUS else "warm_start_quadratic"] = extrap
    if not args.no_sorted:
        line["deposit_sorted"] = sorted_deposit_leg(args, w, prec, parts, local, K, W)

    if not args.no_e2e:
        pinned = [torch.from_numpy(p.copy()).pin_memory() for p in parts]
        host = [t.numpy() for t in pinned]
        # an untimed first call creates and plans the device context, which
        # hv_simulate keeps for the later calls of the same shape (a caller
        # running many nuclei pays for it once); then three timed calls, the
        # median reported
        for hb, p in zip(host, parts):
            hb[:] = p
        hv.simulate(w, *host, K, prec, hv.HV_PATH_FUSED)
        runs = []
        for _ in range(3):
            # hv_simulate advances the host arrays in place: every call starts
            # from the same particles (restored outside the timed region)
            for hb, p in zip(host, parts):
                hb[:] = p
            barrier(world)
            t0 = time.perf_counter()
            obs_e = hv.simulate(w, *host, K, prec, hv.HV_PATH_FUSED)
            el = time.perf_counter() - t0
            runs.append(w.particles * K * world / max_over_ranks(world, el))
        es = 4 if prec == hv.HV_F32 else 8
        line["e2e"] = {"value": float(np.median(runs)), "unit": UNIT,
                       "h2d_bytes_per_step": 6 * w.particles * es / K,
                       "d2h_bytes_per_step": (6 * w.particles * es + obs_e.nbytes) / K,
                       "runs": runs, "reported": "median of 3 calls",
                       "includes": "per call: upload from pinned host memory, initial field solve, K steps, "
                                   "download of the particles and the K observable rows (hv_simulate); the "
                                   "device context is the one an untimed first call created and left cached"}
        hv.simulate_release()

    # the last leg with collectives, before the legs that rank 0 runs alone (so
    # that no rank waits on those at a barrier)
    if not args.no_batch:
        bl = batched(args, local, world, rank)  # every rank takes part (its share of the runs)
        if rank == 0:
            line["batched"] = bl

    # the legs below hold one GPU for minutes: single-GPU runs only
    single = world == 1 and rank == 0
    if not args.no_plain and single:
        # the plain FP64 drop-in: per-routine kernels, SOR tested on the host
        p64 = [p.astype(np.float64) for p in parts]
        with hv.Session.from_workload(w, hv.HV_F64, device=local) as s64:
            s64.upload_particles(*p64)
            s64.initial_solve()
            kp = 3
            st = torch.cuda.ExternalStream(s64.stream())
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a0.record(st)
            ob64 = s64.run(kp, hv.HV_PATH_PLAIN)
            a1.record(st)
            a1.synchronize()
            pms = a0.elapsed_time(a1) / kp
        with hv.Session.from_workload(w, prec, device=local) as sf:
            sf.upload_particles(*parts)
            obf = sf.run(kp, hv.HV_PATH_FUSED)
        dmax = float(np.max(np.abs(ob64["dipole"])))
        line["plain_f64"] = {"value": w.particles / (pms / 1e3), "unit": UNIT, "ms_per_step": pms, "steps": kp,
                             "speedup_of_value": value / world / (w.particles / (pms / 1e3)),
                             "sor_iterations_per_step": float(ob64["sor_iterations"].mean()),
                             "dipole_max_rel_diff_fused_f32": float(np.max(np.abs(obf["dipole"] - ob64["dipole"])) /
                                                                    dmax) if dmax > 0 else None}

    if not args.no_plain and single:
        line["fused_f64"] = fused_f64_leg(w, parts, local, K, start, value / world, obs)
    if not args.no_accuracy and single and prec == hv.HV_F32:
        line["dipole_accuracy"] = dipole_accuracy(args, w, parts, local)
    if not args.no_adjoint and single:
        line["adjoint"] = adjoint_cases(args, local)
    if not args.no_init and single:
        line["particle_densities"] = particle_densities_cost(args, local, world)
        line["initialisation"] = initialisation_cost(args, local, world)

    if not args.no_cpu and rank == 0 and world == 1:
        try:
            s = run_cpu_child(args, args.cpu_steps, 0)
            line["cpu_baseline"] = {"value": s["value"], "unit": UNIT, "cores": s["threads"], "kind": s["kind"],
                                    "sample": f"{s['steps']} time step(s) of {w.name} after the initial solve "
                                              f"({s['init_seconds']:.1f} s, untimed); {s['what']}",
                                    "inputs_match": s["inputs_sha256"] == digest}
        except Exception as e:  # reported, never fatal for the GPU number
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"failed: {e}"[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.cpu_sample:
        cpu_sample(args)
        return
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        reference_arm(args, world, rank)
        return
    if args.adjoint_horizons:
        adjoint_horizons(args)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        our_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
