"""
Force-backend boundary: the reference's plugin interface
(aimd/backends/base.py:42-84, aimd/backends/registry.py:21-39) and a GPU
Hartree-Fock backend with the constructor arguments, density-guess protocol
and ``info`` keys of the reference's ``hf`` backend (aimd/backends/hf.py:
150-369), registered as ``"hf-gpu"``.

Integrators, thermostats and XL-BOMD call only ``compute(positions)`` and
``set_density_guess(D)``, so this backend is a drop-in for them. When the
reference package ``aimd`` is importable, ``register_with_reference()``
adds it to the reference's registry (``aimd run --backend hf-gpu``).
"""

from __future__ import annotations

import time
from abc import ABC, abstractmethod
from dataclasses import dataclass, field
from typing import Any, ClassVar, Sequence

import numpy as np

from . import integrals as I
from .basis import BasisSet
from .gradients import scf_gradient
from .scf import SCFOptions, SCFResult, SCFSolver


@dataclass
class GradientResult:
    """Energy (Eh) and gradient dE/dR (Eh/bohr, (N, 3)) for one geometry."""
    energy: float
    gradient: np.ndarray
    converged: bool = True
    density: np.ndarray | None = None
    dipole: np.ndarray | None = None
    info: dict[str, Any] = field(default_factory=dict)

    @property
    def forces(self) -> np.ndarray:
        return -self.gradient


class ForceBackend(ABC):
    """Energy/gradient provider: positions in bohr (N, 3) -> GradientResult."""
    name: ClassVar[str] = ""
    supports_density_guess: ClassVar[bool] = False

    def __init__(self, symbols: Sequence[str], charge: int = 0, multiplicity: int = 1) -> None:
        self.symbols = list(symbols)
        self.charge = int(charge)
        self.multiplicity = int(multiplicity)

    @abstractmethod
    def compute(self, positions: np.ndarray) -> GradientResult:
        """Energy and gradient at ``positions`` (bohr, shape (N, 3))."""

    def set_density_guess(self, density: np.ndarray) -> None:
        raise NotImplementedError(f"backend '{self.name}' does not support density guesses")

    def close(self) -> None:
        """Release resources. Optional."""


_REGISTRY: dict[str, type] = {}


def register_backend(cls: type) -> type:
    key = str(cls.name).strip().lower()
    if not key:
        raise ValueError(f"{cls.__name__} must define a non-empty 'name'")
    _REGISTRY[key] = cls
    return cls


def get_backend(name: str) -> type:
    key = str(name).strip().lower()
    if key not in _REGISTRY:
        raise ValueError(f"Unknown backend '{name}'. Available backends: {list_backends()}")
    return _REGISTRY[key]


def list_backends() -> list[str]:
    return sorted(_REGISTRY)


_REFERENCES = {"auto": None, "rhf": "rhf", "restricted": "rhf", "uhf": "uhf", "unrestricted": "uhf"}
_METHODS = {"hf": None, "scf": None, "rhf": "rhf", "uhf": "uhf"}
_GUESSES = {"auto": "sad", "sad": "sad", "core": "core", "gwh": "gwh"}
_OWN_OPTIONS = {"conv_energy": "conv_tol", "conv_commutator": "conv_tol_grad", "max_iter": "max_cycles",
                "guess": "guess", "warn_unconverged": None}


@register_backend
class HFGPUBackend(ForceBackend):
    """
    RHF/UHF energies and analytic gradients on one B200. Arguments as the
    reference's HFBackend (aimd/backends/hf.py:181-197); ``threads`` is
    accepted and ignored (no CPU threads in the integral path).
    """

    name = "hf-gpu"
    description = "RHF / UHF with analytic gradients, McMurchie-Davidson integrals on the GPU"
    supports_density_guess = True

    def __init__(self, symbols: Sequence[str], charge: int = 0, multiplicity: int = 1,
                 basis: str | BasisSet = "sto-3g", reference: str | None = "auto", method: str = "hf",
                 conv_tol: float = 1e-10, conv_tol_grad: float = 1e-7, max_cycles: int = 100,
                 guess: str = "auto", reuse_density: bool = True,
                 gradient_screening: float = I.DEFAULT_SCHWARZ_GRAD, threads: int | None = None,
                 scf_options: dict[str, Any] | None = None) -> None:
        super().__init__(symbols, charge, multiplicity)
        ref = self._parse_reference(reference, method)
        key = str(guess).strip().lower()
        if key not in _GUESSES:
            raise ValueError(f"unknown guess {guess!r}; use one of {sorted(_GUESSES)}")
        self.init_guess = _GUESSES[key]
        if not gradient_screening >= 0.0:
            raise ValueError("gradient_screening must be >= 0")
        self.gradient_screening = float(gradient_screening)
        self.reuse_density = bool(reuse_density)
        extra = dict(scf_options or {})
        for k in extra:
            if k in _OWN_OPTIONS:
                arg = _OWN_OPTIONS[k]
                raise ValueError(f"set SCF option {k!r} through the backend argument {arg!r}"
                                 if arg else f"SCF option {k!r} is managed by the backend")
        try:
            options = SCFOptions(conv_energy=float(conv_tol), conv_commutator=float(conv_tol_grad),
                                 max_iter=int(max_cycles), guess=self.init_guess, warn_unconverged=False, **extra)
        except TypeError as e:
            raise ValueError(f"invalid scf_options: {e}") from e
        self.solver = SCFSolver(self.symbols, basis, charge=self.charge, multiplicity=self.multiplicity,
                                reference=ref, options=options)
        self.threads = None if threads is None else int(threads)
        self._guess: np.ndarray | None = None
        self._last_density: np.ndarray | None = None
        self.last_scf: SCFResult | None = None

    def _parse_reference(self, reference: str | None, method: str) -> str | None:
        m = str(method).strip().lower()
        if m not in _METHODS:
            raise ValueError(f"the hf-gpu backend does Hartree-Fock only; unknown method {method!r}")
        r = "auto" if reference is None else str(reference).strip().lower()
        if r not in _REFERENCES:
            raise ValueError(f"unknown reference {reference!r}; use 'auto', 'rhf' or 'uhf'")
        ref, forced = _REFERENCES[r], _METHODS[m]
        if ref is not None and forced is not None and ref != forced:
            raise ValueError(f"method {method!r} conflicts with reference {reference!r}")
        return ref or forced

    @property
    def options(self) -> SCFOptions:
        return self.solver.options

    @property
    def unrestricted(self) -> bool:
        return self.solver.unrestricted

    @property
    def nao(self) -> int:
        return self.solver.nao

    @property
    def basis(self) -> BasisSet:
        return self.solver.basis

    @property
    def density_shape(self) -> tuple[int, ...]:
        return self.solver.density_shape

    @property
    def label(self) -> str:
        return "UHF" if self.unrestricted else "RHF"

    def set_density_guess(self, density: np.ndarray) -> None:
        d = np.array(density, dtype=float)
        if d.shape != self.density_shape:
            raise ValueError(f"density guess has shape {d.shape}, expected {self.density_shape} "
                             f"({'unrestricted' if self.unrestricted else 'restricted'} reference)")
        if not np.all(np.isfinite(d)):
            raise ValueError("density guess contains non-finite values")
        self._guess = d

    def reset_guess(self) -> None:
        self._guess = None
        self._last_density = None

    def compute(self, positions: np.ndarray) -> GradientResult:
        t0 = time.perf_counter()
        x = np.array(positions, dtype=float)
        if x.ndim != 2 or x.shape != (len(self.symbols), 3):
            raise ValueError(f"expected positions of shape ({len(self.symbols)}, 3), got {x.shape}")
        if self._guess is not None:
            guess, label = self._guess, "external"
        elif self.reuse_density and self._last_density is not None:
            guess, label = self._last_density, "previous"
        else:
            guess, label = self.init_guess, "init"
        self._guess = None
        res = self.solver.run(x, guess=guess)
        t1 = time.perf_counter()
        gradient = scf_gradient(res, schwarz_threshold=self.gradient_screening,
                                fp32_cutoff=self.solver.options.fp32_cutoff)
        t2 = time.perf_counter()
        density = res.guess_density
        if self.reuse_density:
            self._last_density = density
        self.last_scf = res
        warnings_: list[str] = []
        if not res.converged:
            warnings_.append(f"SCF not converged after {res.iterations} iterations (energy change "
                             f"{res.energy_change:.2e} Eh, commutator {res.commutator_norm:.2e}); "
                             "energy and gradient are those of the last iterate")
        if res.n_removed:
            warnings_.append(f"{res.n_removed} near-linearly-dependent basis combination(s) removed; "
                             "the analytic gradient is then not the exact derivative of the energy")
        info: dict[str, Any] = {
            "method": self.label, "basis": res.basis.name, "reference": res.reference,
            "scf_converged": bool(res.converged), "scf_iterations": int(res.iterations),
            "scf_energy": float(res.energy), "electronic_energy": float(res.electronic_energy),
            "nuclear_repulsion": float(res.nuclear_repulsion), "energy_change": float(res.energy_change),
            "commutator_norm": float(res.commutator_norm), "s2": float(res.s2), "s2_exact": float(res.s2_exact),
            "mulliken_charges": res.mulliken_charges.copy(), "guess": label, "init_guess": self.init_guess,
            "n_removed": int(res.n_removed), "warnings": warnings_,
            "fp32_cutoff": float(self.solver.options.fp32_cutoff),
            "timings": {"integrals": float(res.timings.get("integrals", 0.0)),
                        "guess": float(res.timings.get("guess", 0.0)),
                        "scf_iterations": float(res.timings.get("iterations", 0.0)),
                        "scf": t1 - t0, "gradient": t2 - t1, "total": time.perf_counter() - t0},
        }
        return GradientResult(energy=float(res.energy), gradient=gradient, converged=bool(res.converged),
                              density=density.copy(), dipole=np.array(res.dipole, dtype=float), info=info)

    def close(self) -> None:
        self.solver.clear_cache()
        self.reset_guess()
        self.last_scf = None


def register_with_reference() -> bool:
    """Add HFGPUBackend to the reference's registry if ``aimd`` is importable."""
    try:
        from aimd.backends import registry  # type: ignore
    except ImportError:
        return False
    registry.register_backend(HFGPUBackend)
    return True
