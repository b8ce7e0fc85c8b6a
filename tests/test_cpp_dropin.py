"""The C++ drop-in header (include/hv_b200.hpp): a program written against the
reference's call shapes compiles and links here (CPU), and on the GPU its
cpu_simulate loop and its gpu_simulate stats.txt match the oracle run."""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest
from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")
LIBDIR = os.path.join(ROOT, "hyper-vlasov_b200", "hv_b200", "lib")


def build(tmp):
    exe = os.path.join(tmp, "dropin_main")
    gxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lhv_b200", f"-Wl,-rpath,{LIBDIR}"]
    env = dict(os.environ)
    env.pop("CXX", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_header_compiles_and_links(hv, tmp_path):
    exe = build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_dropin_loop_and_gpu_simulate_match_oracle(hv, tmp_path):
    from hv_oracle import Oracle, RunSpec
    exe = build(str(tmp_path))
    steps = 6
    r = subprocess.run([exe, str(steps), str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[:steps]])
    final = [float(v) for v in lines[steps].split()[1:]]
    w = hv.CA40_SMALL.with_reference_sor()
    A, B, C, gm = w.skyrme()
    run = RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=0.0, eta_exc=w.eta,
                  A=A, B=B, C=C, gamma=gm)
    o = Oracle(np.float64)
    o.set_threads(1)
    parts = hv.workload_particles(w, np.float64)
    obs, _ = o.simulate(w.world_tuple(), run, w.protons, w.neutrons, *parts, steps)
    assert np.max(np.abs(rows[:, 1] - obs["zcm_p"])) < 1e-12
    assert np.max(np.abs(rows[:, 2] - obs["zcm_n"])) < 1e-12
    assert abs(final[0] - parts[0].sum()) < 1e-8 and abs(final[1] - parts[5].sum()) < 1e-8
    stats = np.loadtxt(os.path.join(str(tmp_path), "stats.txt"))
    assert stats.shape == (steps, 5)
    # gpu_simulate (double -> plain path) writes the reference's stats columns
    assert np.max(np.abs(stats[:, 3] - obs["zcm_p"])) < 1e-6
    assert np.max(np.abs(stats[:, 1] - obs["rms_p"])) < 1e-6
