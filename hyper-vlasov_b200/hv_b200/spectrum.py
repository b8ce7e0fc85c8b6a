"""Dipole strength function from D(t), as scripts/programs.py:82-122 computes
it, in numpy and (differentiably) in torch.

The reference reads t and the proton/neutron centres of mass from
stats.txt, forms D = N Z / A (z_p - z_n) (programs.py:99), removes a linear
least-squares trend (scipy.signal.detrend, :100), applies the window
cos^2(pi (t - t0) / (2 (t_f - t0))) (:104), takes conj(FFT(D)) dt (:109) and
keeps S(E) = Im / (pi eta hbar c) at E = hbar omega > 0 (:111-117).

``power_in_band`` is the objective of the adjoint runs: the spectral power
|D~(E)|^2 summed over the band [e_lo, e_hi] MeV.
"""
from __future__ import annotations

import math

import numpy as np

HBAR_C = 197.33


def detrend_linear(x):
    """x minus its least-squares line over the sample index (the default of
    scipy.signal.detrend)."""
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    if n < 2:
        return x - x.mean() if n else x.copy()
    i = np.arange(n, dtype=np.float64)
    ic = i - i.mean()
    slope = np.dot(ic, x - x.mean()) / np.dot(ic, ic)
    return x - (x.mean() + slope * ic)


def start_index(t_exc, t_f, steps, substeps):
    """First recorded row at or after the excitation (programs.py:95)."""
    return int(t_exc / t_f * steps / substeps)


def dipole(zcm_p, zcm_n, Z, N):
    """D = N Z / A (z_p - z_n) (programs.py:99)."""
    return (N * Z) / (N + Z) * (np.asarray(zcm_p) - np.asarray(zcm_n))


def energy_spectrum(t, zcm_p, zcm_n, Z, N, t_f, dt_row, eta_exc):
    """(E [MeV], S(E)) for rows that start at the excitation.

    t, zcm_p, zcm_n: the rows used (the reference slices them from
    start_index); dt_row: time between rows (t_f / steps * substeps)."""
    t = np.asarray(t, dtype=np.float64)
    d = detrend_linear(dipole(zcm_p, zcm_n, Z, N))
    t0 = t[0]
    d = d * np.cos(np.pi * (t - t0) / (2.0 * (t_f - t0))) ** 2
    freq = np.fft.fftfreq(d.size, d=dt_row)
    omega = 2.0 * np.pi * freq
    raw = np.conjugate(np.fft.fft(d)) * dt_row
    if eta_exc > 1e-5:
        strength = np.imag(raw) / (np.pi * eta_exc * HBAR_C)
    else:
        strength = np.imag(raw) / (np.pi * HBAR_C)
    pos = omega > 0
    return omega[pos] * HBAR_C, strength[pos]


# ---------------------------------------------------------------- torch
def _torch():
    import torch
    return torch


def windowed_dipole_torch(d, t, t_f):
    """Detrended, windowed D(t) (differentiable in d)."""
    torch = _torch()
    n = d.shape[-1]
    i = torch.arange(n, dtype=d.dtype, device=d.device)
    ic = i - i.mean()
    dm = d.mean(dim=-1, keepdim=True)
    slope = ((d - dm) * ic).sum(-1, keepdim=True) / (ic * ic).sum()
    dd = d - (dm + slope * ic)
    t = torch.as_tensor(t, dtype=d.dtype, device=d.device)
    t0 = t[0]
    w = torch.cos(math.pi * (t - t0) / (2.0 * (t_f - t0))) ** 2
    return dd * w


def energy_spectrum_torch(d, t, t_f, dt_row, eta_exc):
    """(E, S(E)) as energy_spectrum, differentiable in d (a tensor of D rows)."""
    torch = _torch()
    dw = windowed_dipole_torch(d, t, t_f)
    n = dw.shape[-1]
    raw = torch.conj(torch.fft.fft(dw.to(torch.complex128 if dw.dtype == torch.float64 else torch.complex64))) * dt_row
    freq = torch.fft.fftfreq(n, d=dt_row, dtype=d.dtype, device=d.device)
    omega = 2.0 * math.pi * freq
    scale = math.pi * (eta_exc if eta_exc > 1e-5 else 1.0) * HBAR_C
    strength = raw.imag / scale
    pos = omega > 0
    return omega[pos] * HBAR_C, strength[..., pos]


def power_in_band(d, t, t_f, dt_row, e_lo=10.0, e_hi=25.0):
    """sum over E in [e_lo, e_hi] of |conj(FFT(windowed D)) dt|^2 (torch,
    differentiable in d): the power of the D(t) spectrum in the band."""
    torch = _torch()
    dw = windowed_dipole_torch(d, t, t_f)
    n = dw.shape[-1]
    spec = torch.fft.fft(dw.to(torch.complex128 if dw.dtype == torch.float64 else torch.complex64)) * dt_row
    e = 2.0 * math.pi * torch.fft.fftfreq(n, d=dt_row, dtype=d.dtype, device=d.device) * HBAR_C
    band = (e >= e_lo) & (e <= e_hi)
    return (spec.abs() ** 2)[..., band].sum(-1)
