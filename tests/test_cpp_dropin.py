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


INIT_SRC = os.path.join(ROOT, "tests", "cpp", "init_main.cpp")


def build(tmp, src=SRC):
    exe = os.path.join(tmp, os.path.splitext(os.path.basename(src))[0])
    gxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
           "-L", LIBDIR, "-lhv_b200", f"-Wl,-rpath,{LIBDIR}"]
    env = dict(os.environ)
    env.pop("CXX", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_header_compiles_and_links(hv, tmp_path):
    exe = build(str(tmp_path))
    assert os.path.exists(exe)
    assert os.path.exists(build(str(tmp_path), INIT_SRC))


@pytest.mark.gpu
def test_dropin_initialize_particles_matches_the_reference_loop(hv, golden, tmp_path):
    """hvb200::initialize_particles after srand(128), with the reference's
    call shape, against the golden run of the reference's own loop (its fit
    restated): the same particles to 1e-12, Woods-Saxon parameters and Fermi
    levels to 1e-9, densities and energies of the final particles."""
    g = golden("init_ca40_f64.npz")
    exe = build(str(tmp_path), INIT_SRC)
    out = os.path.join(str(tmp_path), "init.bin")
    ws0, fe0, sk = g["ws0"], g["fermi0"], g["skyrme"]
    args = [exe, out] + [str(v) for v in (int(g["Z"]), int(g["N"]), int(g["ppn"]))] + \
        [repr(float(g["sigma_k"])), repr(float(g["sigma_r"])), repr(float(g["r_max"])), str(int(g["max_test_part"])),
         str(int(g["seed"]))] + [repr(float(v)) for v in sk] + [repr(float(v)) for v in ws0.ravel()] + \
        [repr(float(v)) for v in fe0]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("ITERATION") == int(g["passes"])
    data = np.fromfile(out, dtype=np.float64)
    total = (int(g["Z"]) + int(g["N"])) * int(g["ppn"])
    assert data.size == 8 + 9 * total
    assert np.allclose(data[:6], g["ws"].ravel(), rtol=1e-9, atol=0)
    assert np.allclose(data[6:8], g["fermi"], rtol=1e-9, atol=0)
    arrs = data[8:].reshape(9, total)
    for a, k in zip(arrs, ("x", "y", "z", "kx", "ky", "kz", "density_p", "density_n", "energy")):
        tol = 1e-12 if k in ("x", "y", "z", "kx", "ky", "kz") else 1e-9
        assert np.max(np.abs(a - g[k])) <= tol * np.abs(g[k]).max(), k


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
