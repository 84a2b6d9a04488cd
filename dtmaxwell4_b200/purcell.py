"""Purcell post-processing on the engine's FP64 running DFTs.

The reference computes its Purcell factor offline: calc_purcell.sh runs an
external Fourier script over the sensor trace of E at the dipole and over the
dipole signal (files fE.dat and fdip.dat: omega, amplitude, phase), and
purcell.gp:3 plots, against wavelength 2 pi/omega,

    (A_E cos(phi_E) A_d sin(phi_d) - A_E sin(phi_E) A_d cos(phi_d)) * omega / 2
        / (A_d^2 omega^4 / 3) + 1

labelled "Purcell factor, W/W_0+1".  Here the spectra come from the engine's
own accumulators (a one-point DFT window on the dipole's E node, or the
source waveform below), and a second estimator uses the power through a
closed flux box (dtmx_add_flux_box) of a structure run and a vacuum run.

DFT convention of the engine (dtmx_add_dft_plane): X(omega) = sum_n x(t_n)
exp(-i omega t_n) dt with each quantity at its own time level.
"""
import math

import numpy as np

from . import abi


def purcell_reference(e_hat, d_hat, omega):
    """The purcell.gp:3 expression with the spectra as complex values
    A exp(i phi):  Im(d_hat conj(e_hat)) * omega / 2 / (|d_hat|^2 omega^4 / 3) + 1,
    since A_E A_d (cos phi_E sin phi_d - sin phi_E cos phi_d) = Im(d_hat conj(e_hat))."""
    e_hat = np.asarray(e_hat, dtype=np.complex128)
    d_hat = np.asarray(d_hat, dtype=np.complex128)
    omega = np.asarray(omega, dtype=np.float64)
    return (d_hat * np.conj(e_hat)).imag * omega / 2.0 / (np.abs(d_hat) ** 2 * omega ** 4 / 3.0) + 1.0


def source_spectrum(src, omegas, dt, nsteps):
    """DFT of a soft point source's waveform as the engine injects it: during
    step n (n = 0 .. nsteps-1) the E node gets amp sin(2 pi f0 u) exp(-(u/tau)^2)
    with u = (n + 1/2) dt - t0 (point_source_kernel), i.e. at time (n + 1/2) dt."""
    if src.waveform != abi.WAVE_GAUSS_SINE:
        raise ValueError("unknown waveform %d" % src.waveform)
    n = np.arange(nsteps, dtype=np.float64)
    t = (n + 0.5) * dt
    u = t - src.t0
    s = src.amp * np.sin(2.0 * math.pi * src.f0 * u) * np.exp(-(u / src.tau) ** 2)
    om = np.asarray(omegas, dtype=np.float64)
    return (s[None, :] * np.exp(-1j * om[:, None] * t[None, :])).sum(axis=1) * dt


def purcell_flux(power, power0, eps_src=1.0, eps_src0=1.0):
    """W/W0 from the total outward flux-box power of a structure run (power)
    and of a vacuum run with the same source and box (power0).  A soft source
    adds s(t) to E after the E update, which is the current J = -eps s / dt in
    a medium of permittivity eps at the source node; radiated power scales as
    |J|^2, so each run is normalised by its eps_src^2 to compare equal currents."""
    power = np.asarray(power, dtype=np.float64)
    power0 = np.asarray(power0, dtype=np.float64)
    return (power / eps_src ** 2) / (power0 / eps_src0 ** 2)
