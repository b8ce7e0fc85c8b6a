"""Batched runs: many independent nuclei advanced together on one GPU
(hv_batch_* of the C ABI).

    sessions = [Session.from_workload(w, HV_F32) for w in batch_workloads(64)]
    for s, w in zip(sessions, ws): s.upload_particles(*workload_particles(w, np.float32))
    with Batch(sessions) as b:
        b.autotune(2)               # SOR block cap and particle block size chosen by timing
                                    # (advances every run)
        obs = b.run(500)            # obs[i] = rows of instance i

Each instance's rows are those of its own Session.run(steps, HV_PATH_FUSED),
up to float rounding.  The sessions must outlive the batch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class Batch:
    def __init__(self, sessions):
        self.lib = L.load()
        self.sessions = list(sessions)
        arr = (C.c_void_p * len(self.sessions))(*[s.handle.value for s in self.sessions])
        self._b = C.c_void_p()
        L.check(self.lib.hv_batch_create(len(self.sessions), arr, C.byref(self._b)), "hv_batch_create")

    def plan(self, sor_max_blocks=0):
        L.check(self.lib.hv_batch_plan(self._b, int(sor_max_blocks)), "hv_batch_plan")

    def autotune(self, trial_steps=2):
        cap = C.c_int(0)
        L.check(self.lib.hv_batch_autotune(self._b, int(trial_steps), C.byref(cap)), "hv_batch_autotune")
        return cap.value

    def waves(self):
        return self.lib.hv_batch_waves(self._b)

    def tiles(self):
        """Per instance: (SOR planes, rows, blocks, particle-step block size)."""
        n = len(self.sessions)
        arrs = [np.zeros(n, np.int32) for _ in range(4)]
        L.check(self.lib.hv_batch_tiles(self._b, *[C.c_void_p(a.ctypes.data) for a in arrs], n), "hv_batch_tiles")
        return list(zip(*[a.tolist() for a in arrs]))

    def run(self, steps):
        obs = np.zeros((len(self.sessions), steps), L.OBS_DTYPE)
        L.check(self.lib.hv_batch_run(self._b, int(steps), C.c_void_p(obs.ctypes.data)), "hv_batch_run")
        return obs

    def close(self):
        if self._b:
            self.lib.hv_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
