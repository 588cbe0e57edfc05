"""Physical constants (SI, CODATA 2018) used by the rate-equation path.

Values equal molmot/constants.py:5-99 so that inputs built here are
bit-identical to the reference's.  Two hbar values exist in the reference:
the CODATA one used by its pure-Python solver (molmot/constants.py:18) and a
truncated one hard-coded in its numba core and CUDA kernels
(molmot/obe/rate_equations_jit.py:27).  The force kernels take hbar as a
parameter; ``HBAR_JIT`` is their default because the reference's dispatcher
routes DCMOTSimulator.force through the numba core.
"""
import math

c = 299792458.0
h = 6.62607015e-34
hbar = 1.054571817e-34
HBAR_JIT = 1.0545718e-34
mu_B = 9.2740100783e-24
k_B = 1.380649e-23
amu = 1.66053906660e-27
gS = 2.0023193043617


def wavenumber(wavelength: float) -> float:
    """k = 2 pi / lambda (1/m)."""
    return 2.0 * math.pi / wavelength


def v_recoil(k: float, mass: float) -> float:
    """Single-photon recoil velocity hbar k / m (m/s)."""
    return hbar * k / mass


def T_doppler(Gamma: float) -> float:
    """Doppler temperature hbar Gamma / (2 k_B) (K)."""
    return hbar * Gamma / (2.0 * k_B)


def I_sat(Gamma_hz: float, wavelength: float) -> float:
    """Two-level saturation intensity pi h c Gamma / (3 lambda^3) (W/m^2);
    Gamma_hz is the linewidth in the units the caller uses for Gamma."""
    return math.pi * h * c * Gamma_hz / (3.0 * wavelength ** 3)
