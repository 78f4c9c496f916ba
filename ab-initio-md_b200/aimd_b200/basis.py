"""
Contracted Cartesian Gaussian basis sets as flat host arrays.

Same conventions as the reference (``aimd/qc/basis.py:1-64``), so that AO
matrices are interchangeable between the two codes:

* every Cartesian component is kept (6 d functions), each AO has unit norm;
  ``prim_coef`` normalises the axis-aligned component x^l and component
  (lx, ly, lz) carries ``cartesian_factor(lx, ly, lz)``;
* AO order: atoms in input order, shells of an atom sorted by l (stable),
  a general contraction becomes consecutive segmented shells (one per
  column), Cartesian components in PySCF order (xx, xy, xz, yy, yz, zz);
* "blocks": consecutive shells of one atom with the same l whose exponent
  sets are nested share their primitives (general contraction). The
  two-electron kernels work on blocks, evaluating each primitive quartet once
  for all contraction combinations. The grouping rule is the reference's
  (``aimd/qc/basis.py:185-228``), because the Schwarz bounds are per block
  pair and the screening decisions must agree.

The basis data (``data/basis_sets.json``) are the published basis sets in
the PySCF/NWChem row layout, identical to the reference's library.
"""

from __future__ import annotations

import copy
import functools
import json
import math
import os
from typing import Sequence

import numpy as np

from .elements import ATOMIC_NUMBERS, normalize_symbol

_L_LABELS = "spdfghi"
_ALIASES = {"sto3g": "sto-3g", "631g": "6-31g", "6-31g(d)": "6-31g*", "631g*": "6-31g*",
            "6-31g(d,p)": "6-31g**", "631g**": "6-31g**", "ccpvdz": "cc-pvdz"}


@functools.lru_cache(maxsize=1)
def _library() -> dict:
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "basis_sets.json")
    with open(path) as f:
        return json.load(f)


def available_basis_sets() -> list[str]:
    return list(_library())


def normalize_basis_name(name: str) -> str:
    """Canonical lower-case basis name ('6-31G(d)' -> '6-31g*'); ValueError if unknown."""
    key = "".join(str(name).split()).lower()
    key = _ALIASES.get(key, key)
    if key not in _library():
        raise ValueError(f"Unknown basis set {name!r}. Available: {', '.join(available_basis_sets())}")
    return key


def get_basis_shells(name: str, symbol: str) -> list[tuple[int, np.ndarray, np.ndarray]]:
    """Shells of ``symbol`` as (l, exponents (nprim,), coefficients (nprim, ncol)) in file order."""
    key = normalize_basis_name(name)
    sym = normalize_symbol(symbol)
    data = _library()[key]
    if sym not in data:
        raise ValueError(f"Basis set {key!r} has no data for element {sym!r} "
                         f"(available: {', '.join(data)})")
    out = []
    for entry in data[sym]:
        rows = np.array(entry[1:], dtype=float)
        out.append((int(entry[0]), rows[:, 0].copy(), rows[:, 1:].copy()))
    return out


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def cartesian_components(l: int) -> list[tuple[int, int, int]]:
    """(lx, ly, lz) in PySCF order."""
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def _odd_factorial(n: int) -> int:
    """(n)!! for odd n >= -1, with (-1)!! = 1."""
    return math.prod(range(n, 0, -2)) if n > 0 else 1


def cartesian_factor(lx: int, ly: int, lz: int) -> float:
    """sqrt((2l-1)!! / ((2lx-1)!! (2ly-1)!! (2lz-1)!!)): norm of (lx,ly,lz) relative to x^l."""
    l = lx + ly + lz
    num = _odd_factorial(2 * l - 1)
    den = _odd_factorial(2 * lx - 1) * _odd_factorial(2 * ly - 1) * _odd_factorial(2 * lz - 1)
    return float(np.sqrt(num / den))


def normalized_contraction(l: int, exponents: np.ndarray, coefficients: np.ndarray) -> np.ndarray:
    """
    Coefficients c_k giving x^l sum_k c_k exp(-a_k r^2) unit norm, from
    coefficients of normalised primitives (the standard renormalisation).
    """
    a = np.asarray(exponents, dtype=float)
    d = np.asarray(coefficients, dtype=float)
    df = _odd_factorial(2 * l - 1)
    # norm of each primitive x^l exp(-a r^2), formed first so that the
    # coefficients round exactly as the reference's do
    prim_norm = (2.0 * a / np.pi) ** 0.75 * (4.0 * a) ** (0.5 * l) / np.sqrt(df)
    c = d * prim_norm
    s = a[:, None] + a[None, :]
    gram = df * np.pi ** 1.5 / ((2.0 * s) ** l * s ** 1.5)
    return c / np.sqrt(c @ gram @ c)


def _frozen(a: np.ndarray) -> np.ndarray:
    a.flags.writeable = False
    return a


class BasisSet:
    """
    Cartesian Gaussian basis of one molecule. Attribute names follow the
    reference's ``BasisSet`` (``aimd/qc/basis.py:140-283``):

      shell_atom, shell_l, shell_prim, shell_ao, prim_exp, prim_coef
      blk_shell, blk_atom, blk_l, blk_ncon, blk_ao, blk_prim, blk_exp, blk_coef
      ao_shell, ao_atom, ao_l, ao_lxyz, atom_ao, positions (bohr)
    """

    def __init__(self, name: str, symbols: Sequence[str], positions: np.ndarray,
                 shell_atom, shell_l, shell_prim, prim_exp, prim_coef) -> None:
        self.name = name
        self.symbols = [normalize_symbol(s) for s in symbols]
        self.natm = len(self.symbols)
        self.atomic_numbers = _frozen(np.array([ATOMIC_NUMBERS[s] for s in self.symbols], dtype=np.int64))
        self.shell_atom = _frozen(np.asarray(shell_atom, dtype=np.int64).copy())
        self.shell_l = _frozen(np.asarray(shell_l, dtype=np.int64).copy())
        self.shell_prim = _frozen(np.asarray(shell_prim, dtype=np.int64).copy())
        self.prim_exp = _frozen(np.asarray(prim_exp, dtype=float).copy())
        self.prim_coef = _frozen(np.asarray(prim_coef, dtype=float).copy())
        self.nshell = int(self.shell_l.size)
        self.nprim = int(self.prim_exp.size)
        nc = (self.shell_l + 1) * (self.shell_l + 2) // 2
        self.shell_ao = _frozen(np.concatenate([[0], np.cumsum(nc)]).astype(np.int64))
        self.nao = int(self.shell_ao[-1])
        self.lmax = int(self.shell_l.max()) if self.nshell else 0
        self.ao_shell = _frozen(np.repeat(np.arange(self.nshell, dtype=np.int64), nc))
        self.ao_atom = _frozen(self.shell_atom[self.ao_shell].copy())
        self.ao_l = _frozen(self.shell_l[self.ao_shell].copy())
        lxyz = [c for l in self.shell_l for c in cartesian_components(int(l))]
        self.ao_lxyz = _frozen(np.array(lxyz, dtype=np.int64).reshape(-1, 3))
        rng = np.zeros((self.natm, 2), dtype=np.int64)
        for a in range(self.natm):
            idx = np.flatnonzero(self.ao_atom == a)
            if idx.size:
                rng[a] = (idx[0], idx[-1] + 1)
        self.atom_ao = _frozen(rng)
        self._group_blocks()
        # state shared by every geometry of this basis (with_positions copies
        # the reference): the device engine lives here
        self._shared: dict = {}
        self._set_positions(positions)

    # ------------------------------------------------------------------ blocks
    def _group_blocks(self) -> None:
        """General-contraction blocks (see module docstring)."""
        groups: list[list[int]] = []        # shells of each block
        members: list[list[float]] = []     # exponents of each block, first-seen order
        for s in range(self.nshell):
            k0, k1 = self.shell_prim[s], self.shell_prim[s + 1]
            exps = list(dict.fromkeys(self.prim_exp[k0:k1].tolist()))
            joins = (groups and self.shell_atom[s] == self.shell_atom[s - 1]
                     and self.shell_l[s] == self.shell_l[s - 1])
            if joins:
                cur, new = set(members[-1]), set(exps)
                joins = new <= cur or cur <= new
            if joins:
                groups[-1].append(s)
                members[-1].extend(e for e in exps if e not in members[-1])
            else:
                groups.append([s])
                members.append(exps)
        nblk = len(groups)
        maxcon = max((len(g) for g in groups), default=1)
        blk_prim = np.zeros(nblk + 1, dtype=np.int64)
        blk_prim[1:] = np.cumsum([len(m) for m in members])
        coef = np.zeros((int(blk_prim[-1]), maxcon))
        for b, (g, m) in enumerate(zip(groups, members)):
            row = {e: blk_prim[b] + i for i, e in enumerate(m)}
            for c, s in enumerate(g):
                for k in range(self.shell_prim[s], self.shell_prim[s + 1]):
                    coef[row[float(self.prim_exp[k])], c] += self.prim_coef[k]
        first = np.array([g[0] for g in groups], dtype=np.int64)
        self.nblock = nblk
        self.blk_shell = _frozen(np.append(first, self.nshell).astype(np.int64))
        self.blk_atom = _frozen(self.shell_atom[first].copy())
        self.blk_l = _frozen(self.shell_l[first].copy())
        self.blk_ncon = _frozen(np.array([len(g) for g in groups], dtype=np.int64))
        self.blk_ao = _frozen(self.shell_ao[first].copy())
        self.blk_prim = _frozen(blk_prim)
        self.blk_exp = _frozen(np.array([e for m in members for e in m], dtype=float))
        self.blk_coef = _frozen(coef)

    # ---------------------------------------------------------------- geometry
    def _set_positions(self, positions: np.ndarray) -> None:
        x = np.array(positions, dtype=float).reshape(-1, 3)
        if x.shape[0] != self.natm:
            raise ValueError(f"expected {self.natm} positions, got {x.shape[0]}")
        if not np.all(np.isfinite(x)):
            raise ValueError("atomic positions must be finite (got NaN or inf)")
        self.positions = _frozen(x)
        self._cache: dict = {}

    def with_positions(self, positions: np.ndarray) -> "BasisSet":
        """The same basis on moved atoms; shares every other array (O(1))."""
        new = copy.copy(self)
        new._set_positions(positions)
        return new

    @property
    def shell_centers(self) -> np.ndarray:
        return self.positions[self.shell_atom]

    @property
    def nuclear_charges(self) -> np.ndarray:
        return self.atomic_numbers.astype(float)

    def ao_labels(self) -> list[str]:
        out = []
        for mu in range(self.nao):
            a = int(self.ao_atom[mu])
            lx, ly, lz = (int(v) for v in self.ao_lxyz[mu])
            out.append(f"{a} {self.symbols[a]} {_L_LABELS[lx + ly + lz]}{'x' * lx + 'y' * ly + 'z' * lz}")
        return out

    def __repr__(self) -> str:
        return (f"BasisSet({self.name!r}, natm={self.natm}, nshell={self.nshell}, "
                f"nao={self.nao}, nprim={self.nprim}, nblock={self.nblock})")


def build_basis(symbols: Sequence[str], positions: np.ndarray, basis: str) -> BasisSet:
    """Basis ``basis`` (case-insensitive name) for atoms ``symbols`` at ``positions`` (bohr)."""
    name = normalize_basis_name(basis)
    shell_atom, shell_l, shell_prim, prim_exp, prim_coef = [], [], [0], [], []
    for a, sym in enumerate(symbols):
        for l, exps, cols in sorted(get_basis_shells(name, sym), key=lambda sh: sh[0]):
            for j in range(cols.shape[1]):
                used = cols[:, j] != 0.0
                e = exps[used]
                prim_exp.extend(e)
                prim_coef.extend(normalized_contraction(l, e, cols[used, j]))
                shell_atom.append(a)
                shell_l.append(l)
                shell_prim.append(len(prim_exp))
    return BasisSet(name, symbols, positions, shell_atom, shell_l, shell_prim, prim_exp, prim_coef)
