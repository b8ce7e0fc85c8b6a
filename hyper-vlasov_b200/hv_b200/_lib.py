"""ctypes binding of libhv_b200.so (the C ABI declared in include/hv_b200.h).

Loading fails loudly when the library has not been built: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libhv_b200.so")

HV_OK = 0
HV_ERR_BAD_ARG = 1
HV_ERR_CUDA = 2
HV_ERR_NOT_CONVERGED = 3
HV_ERR_NO_DEVICE = 4
HV_ERR_OOM = 5
HV_ERR_TIMEOUT = 6
HV_ERR_UNSUPPORTED = 7
HV_ERR_NONFINITE = 8

HV_F64 = 0
HV_F32 = 1
HV_DEPOSIT_ATOMIC = 0
HV_DEPOSIT_SORTED = 1
HV_SOR_MAX_UPDATE = 0
HV_SOR_REL_RESIDUAL = 1
HV_PATH_PLAIN = 0
HV_PATH_FUSED = 1

HV_FIELD_DENSITY_RAW = 0
HV_FIELD_DENSITY = 1
HV_FIELD_POTENTIAL = 2
HV_FIELD_COULOMB = 3
HV_FIELD_FORCE_X = 4
HV_FIELD_FORCE_Y = 5
HV_FIELD_FORCE_Z = 6

HV_PART = {"x": 0, "y": 1, "z": 2, "kx": 3, "ky": 4, "kz": 5, "fx": 6, "fy": 7, "fz": 8}
HV_OBS_SOR_NOT_CONVERGED = 1


class hv_world(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("d_max", C.c_double * 3)]


class hv_skyrme(C.Structure):
    _fields_ = [("A", C.c_double), ("B", C.c_double), ("C", C.c_double), ("gamma", C.c_double)]


class hv_sor_params(C.Structure):
    _fields_ = [("omega", C.c_double), ("tol", C.c_double), ("criterion", C.c_int), ("max_iter", C.c_int)]


class hv_run_params(C.Structure):
    _fields_ = [
        ("z", C.c_int), ("n", C.c_int), ("part_per_nucleon", C.c_int),
        ("sigma_r", C.c_double), ("dt", C.c_double), ("t_exc", C.c_double), ("eta_exc", C.c_double),
        ("skyrme", hv_skyrme), ("sor", hv_sor_params), ("deposit_mode", C.c_int),
    ]


class hv_fast_options(C.Structure):
    _fields_ = [("sor_warm_start", C.c_int), ("sor_inner_min", C.c_int), ("sor_inner_max", C.c_int),
                ("sort_every", C.c_int), ("graph_steps", C.c_int), ("sor_exchange", C.c_int),
                ("smooth_fft", C.c_int), ("sor_omega", C.c_double), ("sor_wait_limit", C.c_int),
                ("sor_coarse", C.c_int), ("sor_coarse_sweeps", C.c_int), ("deposit_aggregate", C.c_int),
                ("sor_coarse_omega", C.c_double)]


HV_WARM_PREVIOUS = 0
HV_WARM_EXTRAPOLATE = 1
HV_WARM_QUADRATIC = 2
HV_SOR_EXCHANGE_AUTO = 0
HV_SOR_EXCHANGE_FLAGS = 1


class hv_observables(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("rms_p", C.c_double), ("rms_n", C.c_double),
        ("zcm_p", C.c_double), ("zcm_n", C.c_double), ("dipole", C.c_double),
        ("sor_iterations", C.c_int), ("flags", C.c_int),
    ]


class hv_autotune_report(C.Structure):
    _fields_ = [("particle_block", C.c_int), ("particle_grid", C.c_int), ("sor_planes", C.c_int),
                ("sor_rows", C.c_int), ("sor_blocks", C.c_int), ("sor_tile_rank", C.c_int),
                ("candidates", C.c_int), ("particle_ms", C.c_double), ("sor_ms", C.c_double)]


class hv_woods_saxon(C.Structure):
    _fields_ = [("V0", C.c_double), ("R12", C.c_double), ("a", C.c_double)]


class hv_fermi(C.Structure):
    _fields_ = [("epsilon_p", C.c_double), ("epsilon_n", C.c_double)]


HV_RNG_LIBC = 0
HV_RNG_PHILOX = 1


class hv_init_params(C.Structure):
    _fields_ = [("sigma_k", C.c_double), ("r_max", C.c_double), ("max_test_part", C.c_int),
                ("max_iterations", C.c_int), ("rng", C.c_int), ("seed", C.c_uint64)]


class hv_init_row(C.Structure):
    _fields_ = [("equal_p", C.c_int), ("equal_n", C.c_int), ("epsilon_p", C.c_double), ("epsilon_n", C.c_double),
                ("delta_epsilon", C.c_double), ("ws", hv_woods_saxon * 2), ("fit_iterations", C.c_int * 2),
                ("fit_status", C.c_int * 2)]


class hv_init_report(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("delta_epsilon", C.c_double),
                ("chi_squared_p", C.c_double), ("chi_squared_n", C.c_double), ("candidates", C.c_longlong),
                ("max_test_part", C.c_int), ("r_max", C.c_double)]


OBS_DTYPE = np.dtype([
    ("t", "f8"), ("rms_p", "f8"), ("rms_n", "f8"), ("zcm_p", "f8"), ("zcm_n", "f8"),
    ("dipole", "f8"), ("sor_iterations", "i4"), ("flags", "i4"),
])
assert OBS_DTYPE.itemsize == C.sizeof(hv_observables)

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_S = C.c_int  # hv_status

# name -> (restype, argtypes); every name here must be declared in include/hv_b200.h
SIGNATURES = {
    "hv_version": (C.c_char_p, []),
    "hv_status_string": (C.c_char_p, [_S]),
    "hv_last_error": (C.c_char_p, []),
    "hv_device_count": (_I, []),
    "hv_sor_reference_defaults": (None, [_P]),
    "hv_skyrme_from_t0t3": (None, [_D, _D, _D, _D, _P]),
    "hv_generate_nucleus_f64": (_S, [C.c_uint64, _I, _I, _D, _D, _P, _P, _P, _P, _P, _P]),
    "hv_generate_nucleus_f32": (_S, [C.c_uint64, _I, _I, _D, _D, _P, _P, _P, _P, _P, _P]),
    "hv_ctx_create": (_S, [_P, _I, _I, _I, _P, _I, _P]),
    "hv_ctx_destroy": (_S, [_P]),
    "hv_ctx_set_params": (_S, [_P, _P]),
    "hv_ctx_get_params": (_S, [_P, _P]),
    "hv_ctx_stream": (_P, [_P]),
    "hv_ctx_synchronize": (_S, [_P]),
    "hv_upload_particles": (_S, [_P, _P, _P, _P, _P, _P, _P]),
    "hv_download_particles": (_S, [_P, _P, _P, _P, _P, _P, _P]),
    "hv_upload_particle_array": (_S, [_P, _I, _P]),
    "hv_download_particle_array": (_S, [_P, _I, _P]),
    "hv_upload_field": (_S, [_P, _I, _P]),
    "hv_download_field": (_S, [_P, _I, _P]),
    "hv_field_device_ptr": (_S, [_P, _I, _P]),
    "hv_deposit_cic": (_S, [_P]),
    "hv_smooth_density": (_S, [_P]),
    "hv_skyrme_potential": (_S, [_P]),
    "hv_coulomb_boundary": (_S, [_P]),
    "hv_coulomb_sor": (_S, [_P, _P, _P]),
    "hv_merge_potentials": (_S, [_P]),
    "hv_forces_fdm": (_S, [_P]),
    "hv_gather_cic": (_S, [_P]),
    "hv_kick_half": (_S, [_P, _D]),
    "hv_drift": (_S, [_P, _D]),
    "hv_excite": (_S, [_P, _D]),
    "hv_observe": (_S, [_P, _P]),
    "hv_observe_noalloc": (_S, [_P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "hv_fast_options_default": (None, [_P]),
    "hv_ctx_set_fast_options": (_S, [_P, _P]),
    "hv_ctx_get_fast_options": (_S, [_P, _P]),
    "hv_ctx_set_profiling": (_S, [_P, _I]),
    "hv_ctx_autotune": (_S, [_P, _I, _P]),
    "hv_ctx_kernel_times": (_S, [_P, _P, _P, _I]),
    "hv_write_vtk": (_S, [_P, C.c_char_p]),
    "hv_initial_solve": (_S, [_P, _P]),
    "hv_run": (_S, [_P, _I, _I, _P]),
    "hv_simulate": (_S, [_P, _I, _I, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "hv_simulate_release": (_S, []),
    "hv_adjoint_forward": (_S, [_P, _I, _I, _P]),
    "hv_adjoint_backward": (_S, [_P, _P, _P, _P, _P]),
    "hv_adjoint_forward_path": (_S, [_P, _I, _I, _I, _P]),
    "hv_adjoint_stats": (_S, [_P, _P, _P, _P]),
    "hv_particle_densities": (_S, [_P, _P, _P]),
    "hv_init_params_default": (None, [_P]),
    "hv_initialize_particles": (_S, [_P, _P, _P, _P, _P, _P, _P]),
    "hv_fit_woods_saxon": (_S, [_P, _P, _P, _P, _P]),
    "hv_particle_energies": (_S, [_P, _P, _D, _P]),
    "hv_batch_create": (_S, [_I, _P, _P]),
    "hv_batch_destroy": (_S, [_P]),
    "hv_batch_plan": (_S, [_P, _I]),
    "hv_batch_autotune": (_S, [_P, _I, _P]),
    "hv_batch_run": (_S, [_P, _I, _P]),
    "hv_batch_waves": (_I, [_P]),
    "hv_batch_tiles": (_S, [_P, _P, _P, _P, _P, _I]),
}

_lib = None


def load(path: str | None = None):
    """Loads and types the library once; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libhv_b200.so not built ({p}); run python hyper-vlasov_b200/build.py")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


class HVError(RuntimeError):
    def __init__(self, status, where=""):
        lib = load()
        msg = lib.hv_status_string(status).decode()
        detail = lib.hv_last_error().decode()
        super().__init__(f"{where}: {msg} ({status})" + (f" [{detail}]" if detail else ""))
        self.status = status


def check(status, where=""):
    if status != HV_OK:
        raise HVError(status, where)
    return status
