"""
Many geometries at once: SCF + analytic gradient for a list of molecules of
uneven size (the batched benchmark configuration: 64 random H/C/N/O
molecules of 3-20 atoms in 6-31G*).

Each molecule is small (tens to ~150 AOs), so one molecule at a time leaves
most of the 148 SMs idle: its class kernels have a few dozen CTAs. The batch
runs molecules concurrently instead:

  * one SCFSolver (one native context) per molecule, created up front on
    the calling thread, which is the only step that allocates device memory;
    the atomic-HF cache of the SAD guess is filled there too;
  * ``workers`` threads, each with its own CUDA stream, take molecules from
    a queue (largest first) and run SCF + gradient on their stream. The
    integral work is C-ABI calls and the SCF's host decisions wait on torch
    copies; both release the Python GIL, so the streams keep the GPU busy
    with the kernels of several molecules at the same time.

Results are those of running each molecule alone (same kernels, same
screening; only the summation order of the FP64 atomics may differ).
"""

from __future__ import annotations

import concurrent.futures as cf
import threading
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from .elements import ATOMIC_NUMBERS, normalize_symbol
from .gradients import scf_gradient_device
from .scf import SCFOptions, SCFSolver, run_device, sad_density


@dataclass
class BatchResult:
    """Energy (Eh), gradient dE/dR (Eh/bohr, (natm, 3)) and SCF status of one molecule."""
    energy: float
    gradient: np.ndarray
    converged: bool
    iterations: int
    dipole: np.ndarray
    info: dict = field(default_factory=dict)


def default_multiplicity(symbols: Sequence[str], charge: int = 0) -> int:
    """1 for an even electron count, 2 (doublet) for an odd one."""
    n = sum(ATOMIC_NUMBERS[normalize_symbol(s)] for s in symbols) - int(charge)
    return 1 if n % 2 == 0 else 2


class BatchSolver:
    """
    SCF + gradient for a fixed list of molecules ``[(symbols, positions_bohr), ...]``;
    ``run()`` may be called again with new positions for the same molecules.
    """

    def __init__(self, molecules: Sequence[tuple[Sequence[str], np.ndarray]], basis: str = "6-31g*",
                 options: SCFOptions | None = None, workers: int = 8, charges: Sequence[int] | None = None,
                 multiplicities: Sequence[int] | None = None) -> None:
        if workers < 1:
            raise ValueError("workers must be >= 1")
        self.options = options or SCFOptions(warn_unconverged=False)
        self.workers = int(workers)
        self.solvers: list[SCFSolver] = []
        self.positions: list[np.ndarray] = []
        for i, (sym, pos) in enumerate(molecules):
            q = 0 if charges is None else int(charges[i])
            m = default_multiplicity(sym, q) if multiplicities is None else int(multiplicities[i])
            solver = SCFSolver(sym, basis, charge=q, multiplicity=m, options=self.options)
            x = np.asarray(pos, dtype=float).reshape(-1, 3)
            solver.integrals(x)              # native context + device buffers: allocate here, serially
            sad_density(solver.basis)        # fills the atomic-HF cache for the elements
            self.solvers.append(solver)
            self.positions.append(x)
        # largest molecules first, so the tail of the batch is short
        self.order = sorted(range(len(self.solvers)), key=lambda i: -self.solvers[i].nao)
        self._local = threading.local()

    def _stream(self) -> torch.cuda.Stream:
        s = getattr(self._local, "stream", None)
        if s is None:
            s = torch.cuda.Stream()
            self._local.stream = s
        return s

    def _one(self, i: int) -> BatchResult:
        solver = self.solvers[i]
        s = self._stream()
        with torch.cuda.stream(s):
            st = run_device(solver, self.positions[i])
            g = scf_gradient_device(st, fp32_cutoff=self.options.fp32_cutoff)
            dip = -torch.einsum("xmn,mn->x", st.dipole_ints, st.spin[0] + st.spin[1])
            g_h, dip_h = g.cpu().numpy(), dip.cpu().numpy()
        basis = st.basis                     # the basis at this call's positions
        dip_h = dip_h + (basis.nuclear_charges[:, None] * basis.positions).sum(axis=0)
        return BatchResult(st.energy, g_h, st.converged, st.iterations, dip_h, {"nao": solver.nao})

    def run(self, positions: Sequence[np.ndarray] | None = None) -> list[BatchResult]:
        """Results in input order; ``positions`` replaces the stored geometries."""
        if positions is not None:
            if len(positions) != len(self.solvers):
                raise ValueError(f"expected {len(self.solvers)} geometries, got {len(positions)}")
            self.positions = [np.asarray(p, dtype=float).reshape(-1, 3) for p in positions]
        out: list[BatchResult | None] = [None] * len(self.solvers)
        if self.workers == 1:
            for i in self.order:
                out[i] = self._one(i)
        else:
            with cf.ThreadPoolExecutor(max_workers=self.workers) as ex:
                futs = {ex.submit(self._one, i): i for i in self.order}
                for f in cf.as_completed(futs):
                    out[futs[f]] = f.result()
        torch.cuda.synchronize()
        return out  # type: ignore[return-value]


def run_batch(molecules, basis: str = "6-31g*", options: SCFOptions | None = None,
              workers: int = 8) -> list[BatchResult]:
    """One-shot BatchSolver(molecules, basis, options, workers).run()."""
    return BatchSolver(molecules, basis, options, workers).run()
