"""CPU: the algorithmic byte counts bench.py divides by kernel times.

The roofline and the per-kernel GB/s of the bench line rest on these
formulas, so they are pinned here: the particle step's bytes over the grid
nodes its particles touch, the forces kernel's over the row groups it
computes, the SOR's per iteration and per FP64 check, and the share of row
groups holding raw density, on small hand-built grids.
"""
from __future__ import annotations

import importlib.util
import os
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("hv_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_sor_checks_count_one_per_cycle_and_one_after_the_last():
    b = _bench()
    assert b.sor_checks(32, 16) == 3
    assert b.sor_checks(33, 16) == 4
    assert b.sor_checks(48, 16) == 4
    assert b.sor_checks(170, 0) == 2  # plain cycles: the first and the last check


def test_step_bytes_per_kernel():
    b = _bench()
    n, N = 128, 2_080_000
    w = SimpleNamespace(G=n ** 3, particles=N, n=n)
    G = w.G
    full = b.step_bytes(w, 32, 4, 3)
    assert full["particle"] == 48 * N + 4 * 2 * G * 6
    assert full["smooth"] == full["skyrme"] == 16 * G
    assert full["sor"] == 12 * G * 32 + G * (48 + 32 * 3)
    assert full["forces"] == 40 * G
    part = b.step_bytes(w, 32, 4, 3, touched=127_050, force_frac=0.125)
    assert part["particle"] == 48 * N + 24 * 127_050
    # at 128^3 the FFT pass records the occupancy: no raw-density read
    assert part["forces"] == 40 * G * 0.125
    w64 = SimpleNamespace(G=64 ** 3, particles=N, n=64)
    assert b.step_bytes(w64, 32, 4, 3, force_frac=0.25)["forces"] == 4 * w64.G * (2 + 10 * 0.25)
    # double: every word twice as wide, the FP64 state of the solve unchanged
    d = b.step_bytes(w, 32, 8, 3)
    assert d["sor"] == 24 * G * 32 + G * (48 + 32 * 3)


def test_row_group_fraction():
    b = _bench()
    n = 8
    raw = np.zeros((2, n, n, n), np.float32)
    assert b.row_group_fraction(raw, n, 4) == 0.0
    raw[0, 3, 5, 7] = 1.0  # protons, plane 3, group 1 of 2
    raw[1, 0, 0, 0] = 2.0  # neutrons, plane 0, group 0
    raw[1, 0, 3, 2] = 1.0  # the same group again
    assert b.row_group_fraction(raw.ravel(), n, 4) == 2 / (2 * n * 2)
    # n not a multiple of the group: the last group is shorter
    n = 6
    raw = np.zeros((2, n, n, n), np.float32)
    raw[0, 5, 5, 0] = 1.0  # rows 4..5 form the last group
    assert b.row_group_fraction(raw, n, 4) == 1 / (2 * n * 2)
