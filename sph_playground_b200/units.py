"""CGS physical constants and code-unit systems for the experiment runners.

The reference's runners import ``PhysicalConstants`` from its driver package
(playground/runner/fortdriver/units.py) to convert physical set-ups (the
radiation-hydrodynamics shock tubes, runner/004.*_fluxlimdif_*.py) into code
units.  The names and values below are the ones those runners use, so their
set-ups come out with the same numbers; ``Scale`` builds a unit system from
given scales, either with c = 1 (``ic``) or G = 1 (``ig``), and ``Unit``
derives the remaining units from length, mass and time.
"""
import math

# name: value (CGS) — the table the runners index by attribute
_CONSTANTS = {
    "PI": 3.1415926536e0,
    "C": 2.997924e10,               # speed of light, cm/s
    "GG": 6.672041e-8,              # gravitational constant, dyn cm^2 g^-2
    "RG": 8.314e7,                  # gas constant, erg mol^-1 K^-1
    "ELECTRON_MASS_CGS": 9.10938291e-28,
    "PROTON_MASS_CGS": 1.67262158e-24,
    "ATOMIC_MASS_UBIT": 1.660538921e-24,
    "CROSS_SECTION_H2_CGS": 2.367e-15,
    "RADCONST": 7.5646e-15,         # radiation constant, erg cm^-3 K^-4
    "KBOLTZ": 1.38066e-16,          # erg/K
    "EV": 1.60219e-12,              # erg
    "QE": 4.8032068e-10,            # esu
    "PLANCKH": 6.6260755e-27,       # erg s
    "PLANCKHBAR": 1.05457266e-27,   # erg s
    "THOMCS": 6.6525e-25,           # cm^2
    "FINESTR": 7.2974e-3,
    "STEBOLTZ": 5.67051e-5,         # erg cm^-2 K^-4 s^-1
    "AVOGADRO": 6.0221408577e23,    # mol^-1
    "RO": 3.00000000,
    "SOLARM": 1.9891e33, "SOLARR": 6.959500e10, "SOLARL": 3.9e33,
    "EARTHM": 5.979e27, "EARTHR": 6.371315e8,
    "JUPITERM": 1.89813e30, "CERESM": 8.958e23,
    "AU": 1.496e13, "LY": 9.4605e17, "PC": 3.086e18, "KPC": 3.086e21, "MPC": 3.086e24,
    "KM": 1.0e5,
    "SECONDS": 1.0e0, "MINUTES": 6.0e1, "HOURS": 3.6e3, "DAYS": 8.64e4, "YEARS": 3.1556926e7,
    "EVTOK": 1.1604519e4,           # K per eV
}


class PhysicalConstants(object):
    """CGS constants as class attributes (the table above, plus mu0 = 4 pi
    and k_B / m_H), and ``Scale``."""

    CGSMU0 = 4.0 * _CONSTANTS["PI"]
    KB_ON_MH = _CONSTANTS["KBOLTZ"] / _CONSTANTS["PROTON_MASS_CGS"]

    def Scale(self, idist=None, imass=None, itime=None, ig=None, ic=None):
        """A unit system from the given scales (1 for those not given).
        With ``ic`` set, c = 1: one given scale fixes the other two through
        dist = G mass / c^2 and time = dist / c (mass alone when nothing
        is given).  With ``ig`` set, G = 1: time^2 = dist^3 / (G mass) ties
        the three, the missing one solved from the other two — except that
        a mass solved from length and time is dist^2 / (G time^2), as the
        reference computes it (runner/fortdriver/units.py:80, 84), kept so that runner
        set-ups get the same numbers."""
        c, G = self.C, self.GG
        dist = 1.0 if idist is None else idist
        mass = 1.0 if imass is None else imass
        time = 1.0 if itime is None else itime
        if ic is not None:
            if imass is not None or (idist is None and itime is None):
                dist = G * mass / (c * c)
                time = dist / c
            elif idist is not None:
                time = dist / c
                mass = c * c * dist / G
            else:
                dist = time * c
                mass = c * c * dist / G
        elif ig is not None:
            if imass is not None and idist is not None:
                time = math.sqrt(dist ** 3 / (G * mass))
            elif idist is not None and itime is not None:
                mass = dist ** 2 / (G * time ** 2)
            elif imass is not None and itime is not None:
                dist = (time ** 2 * (G * mass)) ** (1.0 / 3.0)
            elif itime is not None:
                mass = dist ** 2 / (G * time ** 2)
            else:
                time = math.sqrt(dist ** 3 / (G * mass))
        return Unit(dist, mass, time)


for _name, _value in _CONSTANTS.items():
    setattr(PhysicalConstants, _name, _value)


class Unit:
    """Length, mass and time units and the ones derived from them (Gaussian
    charge with mu0 = 4 pi, magnetic field, velocity, acceleration, density,
    pressure, specific and total energy)."""

    def __init__(self, dist, mass, time):
        self.dist = dist
        self.mass = mass
        self.time = time
        self.charge = math.sqrt(mass * dist / PhysicalConstants.CGSMU0)
        self.Bfield = mass / (time * self.charge)
        self.velocity = dist / time
        self.accel = dist / time / time
        self.density = mass / dist ** 3
        self.pressure = mass / (dist * time ** 2)
        self.ergg = self.velocity ** 2
        self.energ = mass * self.ergg

    def print(self):
        for key, val in self.__dict__.items():
            print(key, " = ", val)
