"""Atomic-unit constants (Hartree, bohr, electron mass, kelvin).

The reference expresses every quantity in atomic units through
``molmod.units`` / ``molmod.constants`` (e.g. cmmdft/system.py:12-13,
cmmdft/functionals.py:11-12).  molmod is not installed here, so this module
defines the same names with CODATA values.  The test harness that imports the
unmodified reference exposes this very module as ``molmod.units`` and
``molmod.constants``, so parity never depends on the constant choice.
"""

import math

# --- constants (molmod.constants names) ---
avogadro = 6.0221415e23
# Boltzmann constant in Hartree/K (1.3806504e-23 J/K).
boltzmann = 3.1668154051341965e-06
# h in atomic units is 2*pi*hbar with hbar = 1.
planck = 2.0 * math.pi
lightspeed = 137.03599975303575

# --- units (molmod.units names) ---
au = 1.0
meter = 1.0 / 0.5291772083e-10
angstrom = 1.0e-10 * meter
centimeter = 1.0e-2 * meter
nanometer = 1.0e-9 * meter
bohr = 1.0

gram = 1.0e-3 / 9.10938188e-31
kilogram = 1.0e3 * gram
amu = 1.66053873e-27 * kilogram

joule = 1.0 / 4.35974381e-18
calorie = 4.184 * joule
kjmol = 1.0e3 * joule / avogadro
kcalmol = 1.0e3 * calorie / avogadro
electronvolt = 1.0 / 27.21138386
mol = avogadro

kelvin = 1.0
second = 1.0 / 2.418884326505e-17

newton = joule / meter
pascal = newton / meter ** 2
bar = 1.0e5 * pascal
atm = 1.01325e5 * pascal

_UNIT_TABLE = {
    "au": au, "bohr": bohr, "meter": meter, "m": meter, "angstrom": angstrom,
    "A": angstrom, "centimeter": centimeter, "cm": centimeter, "nm": nanometer,
    "nanometer": nanometer, "gram": gram, "g": gram, "kilogram": kilogram,
    "kg": kilogram, "amu": amu, "joule": joule, "J": joule, "calorie": calorie,
    "cal": calorie, "kjmol": kjmol, "kcalmol": kcalmol, "eV": electronvolt,
    "electronvolt": electronvolt, "kelvin": kelvin, "K": kelvin, "mol": mol,
    "pascal": pascal, "Pa": pascal, "bar": bar, "atm": atm, "newton": newton,
    "N": newton, "second": second, "s": second,
}


def parse_unit(expression):
    """Evaluate a unit expression such as ``kcalmol`` or ``angstrom**3``.

    Mirrors ``molmod.units.parse_unit`` for the unit names used by LJ
    parameter files (cmmdft/extpot_calculator.py:705-716).
    """
    try:
        return float(eval(expression, {"__builtins__": {}}, dict(_UNIT_TABLE)))
    except Exception as exc:  # pragma: no cover - defensive
        raise ValueError("Unknown unit expression %r" % expression) from exc
