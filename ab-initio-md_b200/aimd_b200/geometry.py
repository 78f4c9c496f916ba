"""
Seeded synthetic geometries for the benchmark workloads (positions in bohr).

  water()              O at the origin, r(OH) = 0.9572 A, angle HOH = 104.52 deg
  methanol()           staggered CH3OH: C-O 1.43, C-H 1.09, O-H 0.96 A,
                       tetrahedral angles
  water_cluster(n, s)  n rigid gas-phase waters at random positions in a cube
                       sized for 1 g/cm^3, O-O >= 2.7 A, uniformly random
                       orientations (QR of a Gaussian matrix)
  random_molecule(s)   a random H/C/N/O tree of 3-20 atoms with standard bond
                       lengths and tetrahedral angles, then Gaussian noise
                       sigma = 0.05 A

No public dataset is involved: these stand in for the workloads' shapes and
sizes (atom counts, basis sizes, interatomic distances).
"""

from __future__ import annotations

import numpy as np

from .units import ANG_TO_BOHR

_TETRA = np.arccos(-1.0 / 3.0)       # 109.47 deg


def water() -> tuple[list[str], np.ndarray]:
    th = np.deg2rad(104.52)
    r = 0.9572
    pos = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0], [r * np.cos(th), r * np.sin(th), 0.0]])
    return ["O", "H", "H"], pos * ANG_TO_BOHR


def _dir(polar: float, azim: float) -> np.ndarray:
    return np.array([np.sin(polar) * np.cos(azim), np.sin(polar) * np.sin(azim), np.cos(polar)])


def methanol() -> tuple[list[str], np.ndarray]:
    """C at the origin, O on +z; methyl H staggered against the hydroxyl H."""
    C = np.zeros(3)
    O = np.array([0.0, 0.0, 1.43])
    pos = [C, O]
    sym = ["C", "O"]
    for k in range(3):                                   # H-C-O = tetrahedral
        pos.append(C + 1.09 * _dir(_TETRA, np.deg2rad(120.0 * k)))
        sym.append("H")
    pos.append(O + 0.96 * _dir(np.pi - _TETRA, np.deg2rad(60.0)))   # C-O-H tetrahedral
    sym.append("H")
    return sym, np.array(pos) * ANG_TO_BOHR


def water_cluster(n: int, seed: int = 0, min_oo: float = 2.7, density: float = 1.0
                  ) -> tuple[list[str], np.ndarray]:
    """n rigid waters in a cube of side (n * 18.015 / (0.6022 density))^(1/3) A."""
    rng = np.random.default_rng(seed)
    side = (n * 18.015 / (0.6022 * density)) ** (1.0 / 3.0)
    _, mono = water()
    mono = mono / ANG_TO_BOHR
    mono = mono - mono[0]
    oxy: list[np.ndarray] = []
    tries = 0
    while len(oxy) < n:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place the waters; lower min_oo or the density")
        c = rng.uniform(0.0, side, size=3)
        if all(np.linalg.norm(c - o) >= min_oo for o in oxy):
            oxy.append(c)
    sym, pos = [], []
    for o in oxy:
        q, r = np.linalg.qr(rng.normal(size=(3, 3)))
        q = q * np.sign(np.diag(r))                      # Haar-uniform rotation
        if np.linalg.det(q) < 0:
            q[:, 0] = -q[:, 0]
        for s, x in zip(["O", "H", "H"], mono):
            sym.append(s)
            pos.append(o + q @ x)
    return sym, np.array(pos) * ANG_TO_BOHR


_BONDS = {frozenset(("C", "H")): 1.09, frozenset(("C", "C")): 1.54, frozenset(("C", "N")): 1.47,
          frozenset(("C", "O")): 1.43, frozenset(("N", "H")): 1.01, frozenset(("O", "H")): 0.96,
          frozenset(("N", "N")): 1.45, frozenset(("N", "O")): 1.40, frozenset(("O", "O")): 1.48,
          frozenset(("H", "H")): 0.74}
_VALENCE = {"H": 1, "C": 4, "N": 3, "O": 2}


def random_molecule(seed: int, min_atoms: int = 3, max_atoms: int = 20, noise: float = 0.05
                    ) -> tuple[list[str], np.ndarray]:
    """
    A random tree of heavy atoms (C/N/O) with hydrogens filling the remaining
    valences, built with tetrahedral bond directions, then displaced by
    Gaussian noise (sigma ``noise`` A). Retries until the atom count is in
    [min_atoms, max_atoms] and no two atoms are closer than 0.7 A.
    """
    rng = np.random.default_rng(seed)
    for _ in range(1000):
        nheavy = int(rng.integers(1, 7))
        heavy = list(rng.choice(["C", "C", "C", "N", "O"], size=nheavy))
        sym = [heavy[0]]
        pos = [np.zeros(3)]
        free = {0: _VALENCE[heavy[0]]}
        dirs: dict[int, list[np.ndarray]] = {0: []}
        ok = True
        for el in heavy[1:]:
            cands = [i for i, f in free.items() if f > 0 and sym[i] != "H"]
            if not cands:
                ok = False
                break
            parent = int(rng.choice(cands))
            d = _new_direction(dirs[parent], rng)
            sym.append(el)
            pos.append(pos[parent] + _BONDS[frozenset((sym[parent], el))] * d)
            i = len(sym) - 1
            free[parent] -= 1
            free[i] = _VALENCE[el] - 1
            dirs[parent].append(d)
            dirs[i] = [-d]
        if not ok:
            continue
        for i in range(len(heavy)):
            while free[i] > 0:
                d = _new_direction(dirs[i], rng)
                sym.append("H")
                pos.append(pos[i] + _BONDS[frozenset((sym[i], "H"))] * d)
                dirs[i].append(d)
                free[i] -= 1
        if not min_atoms <= len(sym) <= max_atoms:
            continue
        x = np.array(pos) + rng.normal(scale=noise, size=(len(sym), 3))
        r = np.linalg.norm(x[:, None] - x[None], axis=-1) + np.eye(len(sym)) * 10
        if r.min() < 0.7:
            continue
        return sym, x * ANG_TO_BOHR
    raise RuntimeError("random_molecule: no valid molecule found")


def _new_direction(existing: list[np.ndarray], rng: np.random.Generator) -> np.ndarray:
    """A unit vector at a tetrahedral angle to the existing bonds when possible."""
    if not existing:
        v = rng.normal(size=3)
        return v / np.linalg.norm(v)
    a = existing[0]
    perp = np.cross(a, rng.normal(size=3))
    perp /= np.linalg.norm(perp)
    best, best_score = None, -1.0
    for k in range(12):
        phi = 2 * np.pi * k / 12 + rng.uniform(0, 0.1)
        p2 = np.cross(a, perp)
        d = np.cos(_TETRA) * a + np.sin(_TETRA) * (np.cos(phi) * perp + np.sin(phi) * p2)
        d /= np.linalg.norm(d)
        score = min(np.arccos(np.clip(np.dot(d, e), -1, 1)) for e in existing)
        if score > best_score:
            best, best_score = d, score
    return best
