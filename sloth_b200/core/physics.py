"""Plasma-optics formulas used on the host to parameterise the kernels.

Same formulas and constants as the reference (src/core/propagator.py:31-37,
:72-89, :116-164); the kernels evaluate them per ray stage in factored form.
"""
from __future__ import annotations

import numpy as np
from scipy.constants import c as C
from scipy.constants import e as E_CHARGE
from scipy.constants import epsilon_0 as EPS0

ALPHA = 3.14207787e-4   # m_e*eps0/e^2 as used by the reference (propagator.py:73, :88)
NRL_OPE = 5.64e4        # omega_pe = 5.64e4*sqrt(ne[cm^-3]) (NRL formulary, propagator.py:33)


def omega_pe(ne):
    """Electron plasma frequency (rad/s); ne in cm^-3 (propagator.py:31-33)."""
    return NRL_OPE * np.sqrt(ne)


def n_refrac(ne, omega):
    """Plasma refractive index; ne in m^-3 (propagator.py:36-37)."""
    return np.sqrt(1.0 - (omega_pe(ne * 1e-6) / omega) ** 2)


def omega_of(lwl):
    """Laser angular frequency 2*pi*c/lambda (propagator.py:467)."""
    return 2.0 * np.pi * (C / lwl)


def critical_density(omega):
    """ncr = m_e eps0 omega^2/e^2 in m^-3 (propagator.py:73)."""
    return ALPHA * float(omega) ** 2


def kappa_inv_brems(ne, Te, Z, omega):
    """Inverse-bremsstrahlung amplitude absorption rate, 1/s (propagator.py:116-164).
    ne in m^-3, Te in eV, Z mean ion charge; scalars or arrays."""
    ne_cc = np.asarray(ne, dtype=np.float64) * 1e-6
    v_the = 4.19e5 * np.sqrt(Te)
    o_pe = NRL_OPE * np.sqrt(ne_cc)
    o_max = np.maximum(o_pe, omega)
    b_min = Z * E_CHARGE / (4.0 * np.pi * EPS0 * Te)
    CL = np.maximum(2.0, np.log(v_the / (o_max * b_min)))
    return 3.1e-5 * Z * C * (ne_cc / omega) ** 2 * CL * np.power(Te, -1.5)


def kappa_factors(Te, Z, omega):
    """Factorisation of kappa_inv_brems for uniform Te, Z used by the tracers:

        kappa / c = kappa_q2 * q^2 * CL(q),  q = ne/nc,
        CL(q) = max(2, cl_w - 0.5*ln(max(ope2*q, 1))),

    where ope2*q = (omega_pe/omega)^2. Returns (kappa_q2 [1/m], cl_w, ope2).
    """
    Te = float(Te)
    Z = float(Z)
    nc = critical_density(omega)
    kappa_q2 = 3.1e-5 * Z * (nc * 1e-6 / omega) ** 2 * Te ** (-1.5)
    v_the = 4.19e5 * np.sqrt(Te)
    b_min = Z * E_CHARGE / (4.0 * np.pi * EPS0 * Te)
    cl_w = float(np.log(v_the / (omega * b_min)))
    return float(kappa_q2), cl_w, ope_ratio2(omega)


def ope_ratio2(omega):
    """(omega_pe/omega)^2 per unit ne/nc with the NRL omega_pe."""
    return float(NRL_OPE ** 2 * critical_density(omega) * 1e-6 / float(omega) ** 2)
