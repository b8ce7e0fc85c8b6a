"""Builds the sm_100a shared library hv_b200/lib/libhv_b200.so in-tree.

    python hyper-vlasov_b200/build.py [--force] [--jobs N]

Each csrc/*.cu and csrc/*.cpp is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` with line info; the plain-path
kernels (k_plain.cu) and the initialisation (init_ws.cu) additionally get
``--fmad=false`` so that their double results can match the reference's
arithmetic bit for bit.  The CUDA runtime is
linked statically so the library needs only the driver on the GPU host.
Objects go to _build/ (incremental: rebuilt when a source or header changes).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "hv_b200", "lib")
LIB = os.path.join(LIBDIR, "libhv_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", INCLUDE, "-I", CSRC, "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
PER_FILE = {
    "k_plain.cu": ["--fmad=false"],
    "init_ws.cu": ["--fmad=false"],
}


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def host_compiler():
    # the system g++; some images point CXX at a wrapper without OpenMP/spec files
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return "g++"


def _deps():
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def compile_one(src, force):
    name = os.path.basename(src)
    obj = os.path.join(OBJDIR, name + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps()):
        return obj, None
    cmd = [nvcc(), "-ccbin", host_compiler(), *ARCH, *COMMON, *PER_FILE.get(name, []), "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd[cmd.index("-c")] = "-x"
        cmd.insert(cmd.index("-x") + 1, "cu")
        cmd.insert(cmd.index("-x") + 2, "-c")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, (r.stderr if "spill" in r.stderr and "0 bytes spill" not in r.stderr else None) and None


def build(force=False, jobs=None, verbose=False):
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    objs = []
    errors = []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        for obj, err in ex.map(lambda s: compile_one(s, force), srcs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), "-ccbin", host_compiler(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs,
               "-Xlinker", "--no-undefined", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("linked", LIB)
    return LIB


def build_oracle(verbose=False, reference_root=None):
    """Builds the checker libraries under oracle/, and oracle/_ref/ from the
    reference tree at reference_root (or $HV_REFERENCE_ROOT) when one is given
    and present; without one, oracle/_ref/ is left as it is."""
    oracle = os.path.join(ROOT, "oracle")
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(["make", "-s", "-C", oracle, "all"], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    ref_root = reference_root or env.get("HV_REFERENCE_ROOT")
    if ref_root and os.path.isdir(os.path.join(ref_root, "include")):
        r = subprocess.run(["make", "-s", "-C", oracle, "ref", f"REF_ROOT={ref_root}"], capture_output=True,
                           text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError("reference harness build failed:\n" + r.stdout + r.stderr)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--reference-root", default=None, help="reference tree to build oracle/_ref/ from")
    a = ap.parse_args()
    try:
        build(a.force, a.jobs, verbose=True)
        if not a.no_oracle:
            build_oracle(verbose=True, reference_root=a.reference_root)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
