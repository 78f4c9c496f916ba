"""
Element symbols, atomic numbers and IUPAC standard atomic weights for H-Ar
(the range the built-in basis sets cover; reference ``aimd/elements.py:10-33``).
"""

from __future__ import annotations

_SYMBOLS = ("H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
            "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar")
_MASSES = (1.008, 4.002602, 6.94, 9.0121831, 10.81, 12.011, 14.007, 15.999, 18.998403163,
           20.1797, 22.98976928, 24.305, 26.9815385, 28.085, 30.973761998, 32.06, 35.45, 39.948)

ATOMIC_NUMBERS: dict[str, int] = {s: z for z, s in enumerate(_SYMBOLS, start=1)}
ATOMIC_MASSES_AMU: dict[str, float] = dict(zip(_SYMBOLS, _MASSES))


def normalize_symbol(symbol: str) -> str:
    """Canonical capitalisation of an element symbol ('cl' -> 'Cl'); ValueError if unknown."""
    s = str(symbol).strip()
    sym = s[:1].upper() + s[1:].lower()
    if sym not in ATOMIC_NUMBERS:
        raise ValueError(f"Unknown element symbol: {symbol!r}")
    return sym
