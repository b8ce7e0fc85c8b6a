"""CPU: the spectrum post-processing (scripts/programs.py:82-122) restated in
hv_b200.spectrum agrees with the reference's own scipy calls on D(t) series,
and the torch form agrees with the numpy form."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.fft
import scipy.signal

from hv_b200 import spectrum


def reference_spectrum(t, cm_p, cm_n, Z, N, t_f, steps, substeps, eta_exc):
    """The reference's computation, line by line (scripts/programs.py:97-117)."""
    h_bar_c = 197.33
    dipole = (N * Z) / (N + Z) * (cm_p - cm_n)
    dipole = scipy.signal.detrend(dipole)
    t0 = t[0]
    dt = t_f / steps * substeps
    dipole = dipole * np.cos(np.pi * (t - t0) / (2.0 * (t_f - t0))) ** 2.0
    freq = scipy.fft.fftfreq(np.size(dipole), d=dt)
    omega = 2.0 * np.pi * freq
    strength_raw = np.conjugate(scipy.fft.fft(dipole)) * dt
    if eta_exc > 1e-5:
        strength = np.imag(strength_raw) / (np.pi * eta_exc * h_bar_c)
    else:
        strength = np.imag(strength_raw) / (np.pi * h_bar_c)
    pos = omega > 0
    return omega[pos] * h_bar_c, strength[pos]


def synthetic(n=400, dt=0.5, seed=1):
    rng = np.random.default_rng(seed)
    t = np.arange(n) * dt
    w = 13.5 / 197.33
    cm_p = 0.4 * np.sin(w * t) * np.exp(-t / 150) + 0.01 * t / t[-1] + 1e-3 * rng.standard_normal(n)
    cm_n = -0.26 * np.sin(w * t) * np.exp(-t / 150) + 2e-3 + 1e-3 * rng.standard_normal(n)
    return t, cm_p, cm_n


@pytest.mark.parametrize("eta", [30.0 / 197.33, 0.0])
def test_numpy_spectrum_matches_reference_scipy_pipeline(eta):
    t, cp, cn = synthetic()
    steps, substeps = 400, 1
    t_f = t[-1] + 0.5
    E, S = spectrum.energy_spectrum(t, cp, cn, 82, 126, t_f, t_f / steps * substeps, eta)
    Er, Sr = reference_spectrum(t, cp, cn, 82, 126, t_f, steps, substeps, eta)
    assert np.allclose(E, Er, rtol=1e-14, atol=0)
    assert np.max(np.abs(S - Sr)) <= 1e-12 * np.max(np.abs(Sr))


def test_detrend_matches_scipy():
    x = np.random.default_rng(3).standard_normal(777) + np.linspace(0, 5, 777)
    assert np.max(np.abs(spectrum.detrend_linear(x) - scipy.signal.detrend(x))) < 1e-12


def test_torch_spectrum_and_gradient():
    torch = pytest.importorskip("torch")
    t, cp, cn = synthetic()
    t_f, dt = t[-1] + 0.5, 0.5
    d = spectrum.dipole(cp, cn, 82, 126)
    E, S = spectrum.energy_spectrum(t, cp, cn, 82, 126, t_f, dt, 0.152)
    dt_ = torch.tensor(d, dtype=torch.float64, requires_grad=True)
    Et, St = spectrum.energy_spectrum_torch(dt_, t, t_f, dt, 0.152)
    assert np.allclose(Et.detach().numpy(), E, rtol=1e-13)
    assert np.max(np.abs(St.detach().numpy() - S)) < 1e-12 * np.max(np.abs(S))
    J = spectrum.power_in_band(dt_, t, t_f, dt)
    J.backward()
    g = dt_.grad.numpy().copy()
    # central differences on a few components
    for i in (0, 57, 200, 399):
        e = np.zeros_like(d)
        e[i] = 1e-6
        jp = spectrum.power_in_band(torch.tensor(d + e), t, t_f, dt).item()
        jm = spectrum.power_in_band(torch.tensor(d - e), t, t_f, dt).item()
        assert abs((jp - jm) / 2e-6 - g[i]) <= 1e-6 * max(1.0, abs(g[i]))
