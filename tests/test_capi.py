"""CPU: the C-ABI library loads, exports exactly what include/hv_b200.h
declares, and its host-only entry points behave (generator, parameter helpers,
argument checking).  No compute call needs a GPU here."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest
from conftest import ROOT

HEADER_DIR = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in os.listdir(HEADER_DIR):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(HEADER_DIR, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^HV_API\s+[\w\s\*]*?\b(hv_\w+)\s*\(", src, flags=re.M))
    return names


def exported_functions(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_exports_every_declared_symbol(hv):
    from hv_b200 import _lib
    decl = declared_functions()
    assert len(decl) >= 30
    exp = exported_functions(_lib.LIB_PATH)
    missing = decl - exp
    assert not missing, missing
    # and exports nothing undeclared (hidden visibility by default)
    assert not {e for e in exp if e.startswith("hv_")} - decl
    lib = C.CDLL(_lib.LIB_PATH)
    for name in decl:
        assert getattr(lib, name) is not None


def test_python_signatures_cover_the_header(hv):
    from hv_b200 import _lib
    assert set(_lib.SIGNATURES) == declared_functions()


def test_library_has_no_dynamic_cuda_dependency(hv):
    from hv_b200 import _lib
    deps = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcudart" not in deps


def test_generator_is_deterministic_and_in_the_balls(hv):
    a = hv.generate_nucleus(0, 20, 30, 4.0, 1.05)
    b = hv.generate_nucleus(0, 20, 30, 4.0, 1.05)
    c = hv.generate_nucleus(1, 20, 30, 4.0, 1.05)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    assert not np.array_equal(a[0], c[0])
    r2 = a[0] ** 2 + a[1] ** 2 + a[2] ** 2
    k2 = a[3] ** 2 + a[4] ** 2 + a[5] ** 2
    assert r2.max() < 16.0 and k2.max() < 1.05 ** 2
    f = hv.generate_nucleus(0, 20, 30, 4.0, 1.05, np.float32)
    for u, v in zip(a, f):
        assert np.array_equal(u.astype(np.float32), v)


def test_generator_uniform_statistics(hv):
    x, y, z, kx, ky, kz = hv.generate_nucleus(3, 5000, 5000, 7.0, 1.0)
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    # uniform ball: P(r < R/2) = 1/8, <z> = 0
    assert abs(np.mean(r < 3.5) - 0.125) < 0.01
    assert abs(np.mean(z)) < 0.1 and abs(np.mean(kz)) < 0.02


def test_generator_rejects_bad_arguments(hv):
    from hv_b200 import _lib
    lib = _lib.load()
    x = np.zeros(4)
    p = C.c_void_p(x.ctypes.data)
    assert lib.hv_generate_nucleus_f64(0, 2, 2, -1.0, 1.0, p, p, p, p, p, p) == _lib.HV_ERR_BAD_ARG
    assert lib.hv_generate_nucleus_f64(0, -1, 2, 1.0, 1.0, p, p, p, p, p, p) == _lib.HV_ERR_BAD_ARG
    assert lib.hv_generate_nucleus_f64(0, 2, 2, 1.0, 1.0, None, p, p, p, p, p) == _lib.HV_ERR_BAD_ARG


def test_parameter_helpers(hv):
    from hv_b200 import _lib
    lib = _lib.load()
    s = _lib.hv_sor_params()
    lib.hv_sor_reference_defaults(C.byref(s))
    assert (s.omega, s.tol, s.criterion, s.max_iter) == (1.5, 1e-4, 0, 512)
    k = _lib.hv_skyrme()
    lib.hv_skyrme_from_t0t3(-2645.0, 15595.0, 1.0 / 6.0, 32.0, C.byref(k))
    assert abs(k.A - (-317.4)) < 1e-9 and abs(k.B - 248.96) < 0.01 and abs(k.gamma - 7.0 / 6.0) < 1e-15
    assert k.C == 32.0
    assert lib.hv_status_string(3) == b"SOR not converged"
    assert lib.hv_version().startswith(b"hv_b200")


def test_fast_option_defaults(hv):
    """hv_fast_options_default gives the documented defaults of the fused
    path (host only: no device needed)."""
    from hv_b200 import _lib
    lib = _lib.load()
    o = _lib.hv_fast_options()
    lib.hv_fast_options_default(C.byref(o))
    assert o.sor_warm_start == _lib.HV_WARM_QUADRATIC
    assert (o.sor_inner_min, o.sor_inner_max, o.sort_every, o.graph_steps) == (8, 256, 16, 8)
    assert o.sor_exchange == _lib.HV_SOR_EXCHANGE_AUTO and o.smooth_fft == 1
    assert o.sor_omega == 0.0 and o.sor_wait_limit == 0
    # coarse-corrected cycles: 12 sweeps at the default relaxation (0: 1.7)
    assert (o.sor_coarse, o.sor_coarse_sweeps, o.sor_coarse_omega) == (1, 12, 0.0)
    assert o.deposit_aggregate == 1


def test_workload_definitions(hv):
    w = hv.PB208_2M
    assert w.particles == 2_080_000 and w.n == 128 and w.h == 0.25 and w.d_max == 16.0
    assert hv.PB208_104K.particles == 104_000 and hv.CA40_SMALL.particles == 4000
    assert abs(w.radius - 1.2 * 208 ** (1 / 3)) < 1e-12
    assert abs(w.k_fermi - 1.0580) < 1e-4
    A, B, Cc, g = w.skyrme()
    assert abs(A + 317.4) < 1e-9 and abs(B - 248.96) < 0.05


@pytest.mark.skipif(os.environ.get("HV_EXPECT_GPU") == "1", reason="GPU host")
def test_context_creation_fails_cleanly_without_a_device(hv):
    from hv_b200 import _lib
    lib = _lib.load()
    if lib.hv_device_count() > 0:
        pytest.skip("a device is present")
    w = hv.CA40_SMALL
    ctx = C.c_void_p()
    st = lib.hv_ctx_create(C.byref(w.world()), w.protons, w.neutrons, 0, C.byref(w.run_params()), -1,
                           C.byref(ctx))
    assert st == _lib.HV_ERR_NO_DEVICE and not ctx.value
    with pytest.raises(hv.HVError):
        hv.Session.from_workload(w)


def test_context_rejects_bad_arguments_before_touching_a_device(hv):
    from hv_b200 import _lib
    lib = _lib.load()
    w = hv.CA40_SMALL
    ctx = C.c_void_p()
    bad = w.world()
    bad.n[1] = 2
    assert lib.hv_ctx_create(C.byref(bad), 10, 10, 0, C.byref(w.run_params()), -1, C.byref(ctx)) == _lib.HV_ERR_BAD_ARG
    p = w.run_params()
    p.sor.omega = 2.0
    assert lib.hv_ctx_create(C.byref(w.world()), 10, 10, 0, C.byref(p), -1, C.byref(ctx)) == _lib.HV_ERR_BAD_ARG
    p = w.run_params()
    p.sigma_r = float("nan")
    assert lib.hv_ctx_create(C.byref(w.world()), 10, 10, 0, C.byref(p), -1, C.byref(ctx)) == _lib.HV_ERR_BAD_ARG
    assert lib.hv_ctx_create(C.byref(w.world()), -1, 10, 0, C.byref(w.run_params()), -1, C.byref(ctx)) == \
        _lib.HV_ERR_BAD_ARG
    assert lib.hv_ctx_create(C.byref(w.world()), 10, 10, 7, C.byref(w.run_params()), -1, C.byref(ctx)) == \
        _lib.HV_ERR_BAD_ARG
    assert lib.hv_ctx_destroy(None) == _lib.HV_OK
    assert lib.hv_run(None, 1, 0, None) == _lib.HV_ERR_BAD_ARG


def test_ctypes_structs_match_the_c_layout(hv, tmp_path):
    """Every struct that the Python mirror declares has the C header's size
    and field offsets (gcc on a generated program that prints them)."""
    from hv_b200 import _lib
    structs = [(n, c) for n, c in vars(_lib).items()
               if isinstance(c, type) and issubclass(c, C.Structure) and n.startswith("hv_")]
    assert len(structs) >= 8
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hv_b200.h"', 'int main(void) {']
    for name, cls in structs:
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", HEADER_DIR, str(src), "-o", str(exe)], check=True)
    out = dict(ln.rsplit(" ", 1) for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                          check=True).stdout.split("\n") if ln)
    for name, cls in structs:
        assert int(out[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(out[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def test_oracle_generator_matches_the_library_byte_for_byte(hv):
    """The checker's restatement of the seeded generator (MT19937-64 in C,
    oracle/hv_oracle.c) gives the CUDA library's host generator's particles bit
    for bit, in double and float, so that the CPU baseline starts from the same
    inputs without mapping the library."""
    import ctypes as C

    from hv_oracle import Oracle, workload_inputs
    o = Oracle(np.float64)
    # MT19937-64's published check value: the 10000th output after the default
    # seed 5489 (the C++ standard's [rand.predef] requirement on mt19937_64)
    o.lib.orc_mt64_nth.restype = C.c_uint64
    o.lib.orc_mt64_nth.argtypes = [C.c_uint64, C.c_longlong]
    assert o.lib.orc_mt64_nth(5489, 10000) == 9981545732273789042
    for w in (hv.CA40_SMALL, hv.PB208_104K):
        for dt in (np.float64, np.float32):
            ours = hv.workload_particles(w, dt)
            theirs = workload_inputs(o.lib, w, dt)
            for a, b in zip(ours, theirs):
                assert a.dtype == b.dtype and a.tobytes() == b.tobytes()
