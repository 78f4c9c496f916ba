"""
Hartree atomic units and the conversion factors used at the I/O boundary
(CODATA 2018, the same constants as the reference's ``aimd/units.py:14-26``).
"""

BOHR_TO_ANG = 0.529177210903
ANG_TO_BOHR = 1.0 / BOHR_TO_ANG
AMU_TO_AU = 1822.888486209           # unified atomic mass unit in electron masses
AU_TIME_TO_FS = 2.4188843265857e-2   # atomic time unit in femtoseconds
FS_TO_AU_TIME = 1.0 / AU_TIME_TO_FS
KB_AU = 3.166811563455546e-6         # Boltzmann constant, hartree / kelvin
HARTREE_TO_EV = 27.211386245988
HARTREE_TO_KCALMOL = 627.5094740631
